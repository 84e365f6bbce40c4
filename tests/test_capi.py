"""The C-ABI library loads and exports every entry point include/tct_b200.h
declares (no device calls)."""
import ctypes
import os
import re

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(REPO, "include", "tct_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tct_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header():
    lib = ctypes.CDLL(os.path.join(REPO, "tectosaur_b200", "libtct_b200.so"))
    names = declared_symbols()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n


def test_binding_covers_header():
    from tectosaur_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.EXPORTED)


def test_kernel_ids_and_errors():
    from tectosaur_b200 import _lib
    assert _lib.kernel_id("elasticRH3") == 6
    assert _lib.lib.tct_kernel_id(b"nope") == -1
    # host-only entry point reports a bad argument with a message
    rc = _lib.lib.tct_make_bsr_index(2, 1, _lib.i64ptr(np.array([5], np.int64)),
                                     _lib.i64ptr(np.array([0], np.int64)),
                                     _lib.i64ptr(np.zeros(3, np.int64)),
                                     _lib.i64ptr(np.zeros(1, np.int64)),
                                     _lib.i64ptr(np.zeros(1, np.int64)))
    assert rc == _lib.TCT_ERR_ARG and "out of range" in _lib.last_error()
    assert _lib.lib.tct_farfield_workspace_bytes(6, 0, 100, 100, 5) == 0
    assert _lib.lib.tct_farfield_workspace_bytes(6, 0, 100, 100, 3) > 0


def test_make_bsr_index_matches_oracle(orc):
    from tectosaur_b200.util.sparse import make_bsr_index
    rng = np.random.default_rng(1)
    rows = rng.integers(0, 40, 500)
    cols = rng.integers(0, 40, 500)
    data = rng.standard_normal((500, 9, 9))
    indptr, indices, slot = make_bsr_index(40, rows, cols)
    i2, j2, d2 = orc.make_bsr(40, rows, cols, data)
    assert np.array_equal(indptr, i2) and np.array_equal(indices, j2)
    out = np.empty_like(data)
    out[slot] = data
    assert np.array_equal(out, d2)


def test_padded_rows_layout():
    """Padded BSR rows: every row starts on a multiple of the alignment, the
    blocks keep their CSR order inside the row, and the padding fills only
    the gap up to the next row."""
    from tectosaur_b200.util.sparse import auto_row_align, padded_rows
    counts = np.array([0, 1, 7, 8, 9, 0, 33, 2])
    indptr = np.concatenate([[0], np.cumsum(counts)])
    pstart, pos = padded_rows(indptr, 8)
    assert pstart.tolist() == [0, 0, 8, 16, 24, 40, 40, 80, 88]
    for r in range(len(counts)):
        k = np.arange(indptr[r], indptr[r + 1])
        assert np.array_equal(pos[k], pstart[r] + np.arange(counts[r]))
    assert np.unique(pos).shape[0] == pos.shape[0] == indptr[-1]
    p1, q1 = padded_rows(indptr, 1)
    assert np.array_equal(p1, indptr) and np.array_equal(q1, np.arange(indptr[-1]))
    # mean padding (align - 1) / 2 at most a fifth of the mean row length
    assert auto_row_align(100, 9150) == 32 and auto_row_align(100, 7750) == 32
    assert auto_row_align(100, 7749) == 16 and auto_row_align(100, 3750) == 16
    assert auto_row_align(100, 3749) == 8 and auto_row_align(100, 1750) == 8
    assert auto_row_align(100, 1749) == 1 and auto_row_align(100, 150) == 1
    assert auto_row_align(0, 0) == 1


def test_mass_op_matches_reference(golden):
    from tectosaur_b200.ops.mass_op import MassOp
    g = golden("mass_op.npz")
    for nq in [2, 3]:
        for td in [1, 3]:
            m = MassOp(nq, g["pts"], g["tris"], tensor_dim=td).mat.toarray()
            np.testing.assert_allclose(m, g["mat_%d_%d" % (nq, td)], rtol=1e-14, atol=1e-16)


def test_make_rect_matches_reference_order():
    from tectosaur_b200.mesh.mesh_gen import make_rect
    pts, tris = make_rect(3, 3, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]])
    assert tris.shape == (8, 3)
    assert np.array_equal(tris[:4], [[0, 3, 1], [3, 4, 1], [3, 6, 4], [6, 7, 4]])


def test_panel_workspace_sizes():
    """The tensor-core panels report 0 bytes (unsupported) outside R = 16 and
    their rules: RH 3/4/7 points, RT 3 points, point form any R = 16."""
    from tectosaur_b200 import _lib
    L = _lib.lib
    assert L.tct_farfield_rt_panel_workspace_bytes(100, 100, 8, 3) == 0
    assert L.tct_farfield_rt_panel_workspace_bytes(100, 100, 16, 4) == 0
    assert L.tct_farfield_rt_panel_workspace_bytes(100, 100, 16, 3) > 0
    assert L.tct_farfield_rh_panel_workspace_bytes(100, 100, 16, 5) == 0
    assert L.tct_farfield_rh_panel_workspace_bytes(100, 100, 16, 7) > 0


def test_new_entry_points_reject_bad_arguments():
    """The batched quasidynamic steps and the RT panel check their
    arguments before any device work (these calls launch nothing)."""
    import ctypes
    from tectosaur_b200 import _lib
    L = _lib.lib
    nul = None
    # RK combinations take 1 to 4 terms and their arrays
    k = (ctypes.c_void_p * 5)(*([None] * 5))
    st = (ctypes.c_int64 * 5)(*([0] * 5))
    cs = (ctypes.c_double * 5)(*([1.0] * 5))
    # (null device pointers only: a check that stopped working is caught by
    # the null-pointer check, never by a launch)
    for n_terms in (5, 0, 2):
        assert L.tct_qd_combine_batch(10, 2, n_terms, k, st, cs, nul, nul, 0, nul, 10,
                                      nul) == _lib.TCT_ERR_ARG
        assert L.tct_qd_error_norm_batch(10, 2, n_terms, k, st, cs, nul, nul, 10, nul, 10, 1e-4,
                                         nul, nul) == _lib.TCT_ERR_ARG
    assert L.tct_qd_combine_batch(0, 2, 2, k, st, cs, nul, nul, 0, nul, 10, nul) == _lib.TCT_OK
    # null arrays, negative sizes; empty problems are no-ops
    assert L.tct_qd_deficit_batch(9, 2, nul, 1.0, nul, nul, nul, 9, _lib.TCT_F64, nul, 9,
                                  nul) == _lib.TCT_ERR_ARG
    assert L.tct_qd_deficit_batch(-9, 2, nul, 1.0, nul, nul, nul, 9, _lib.TCT_F64, nul, 9,
                                  nul) == _lib.TCT_ERR_ARG
    assert L.tct_qd_deficit_batch(0, 2, nul, 1.0, nul, nul, nul, 9, _lib.TCT_F64, nul, 9,
                                  nul) == _lib.TCT_OK
    assert L.tct_qd_finish_batch(9, 3, 2, nul, 12, nul, 9, nul, 3, 1.2, nul, 12,
                                 nul) == _lib.TCT_ERR_ARG
    assert L.tct_qd_finish_batch(9, 3, 0, nul, 12, nul, 9, nul, 3, 1.2, nul, 12,
                                 nul) == _lib.TCT_OK
    # the RT panel: R = 16 and the 3-point rule only
    dp = _lib.dptr(np.zeros(8))
    assert L.tct_farfield_rt_panel_matvec(nul, nul, nul, nul, 10, nul, 10, 8, 3, dp, dp, dp, 0,
                                          nul, 0, nul) == _lib.TCT_ERR_ARG
    assert "R must be 16" in _lib.last_error()
    assert L.tct_farfield_rt_panel_matvec(nul, nul, nul, nul, 10, nul, 10, 16, 4, dp, dp, dp, 0,
                                          nul, 0, nul) == _lib.TCT_ERR_ARG
    assert L.tct_farfield_rt_panel_matvec(nul, nul, nul, nul, 10, nul, 10, 16, 3, dp, dp, dp, 0,
                                          nul, 0, nul) == _lib.TCT_ERR_ARG  # no workspace
    assert "workspace" in _lib.last_error()
