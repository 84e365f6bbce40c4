"""Parity at the benched configuration: the 60k-triangle topographic surface
(59,858 triangles, 538,722 DOF) with the production operator
RegularizedSparseIntegralOp(6, 6, 6, 1, 5, 2.5, 'elasticRH3', 'elasticRH3',
[1, 0.25], ..., TriToTriDirectFarfieldOp), against the FP64 oracle of the
reference operator on seeded observation rows (oracle/ref_pipeline.py: the
reference's compiled near-pair finder and rule arrays, the C++ kernel
restatement).  Bars: FP32 apply within 1e-5 relative per matvec, FP64 apply
within 1e-10, the tensor-core multi-RHS farfield within 1e-5 per vector."""
import numpy as np
import pytest

from oracle import ref_pipeline as rp

from helpers import PARAMS, c2_mesh, rel

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not rp.available(), reason="oracle/_ref not built")]

NQ = (6, 6, 6, 1, 5, 2.5)
FP32_TOL = 1e-5
FP64_TOL = 1e-10


@pytest.fixture(scope="module")
def c2():
    pts, tris = c2_mesh()
    classes = rp.classify(tris, rp.near_pairs(pts, tris, NQ[5]))
    return pts, tris, classes


def _op(pts, tris, ft):
    import tectosaur_b200 as tct
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    return tct.RegularizedSparseIntegralOp(*NQ, "elasticRH3", "elasticRH3", PARAMS, pts, tris,
                                           ft, TriToTriDirectFarfieldOp, keep_uncorrected=False)


def _rows(pts, tris, classes, n_rows, seed, ft=np.float64):
    rows = np.sort(np.random.default_rng(seed).choice(tris.shape[0], n_rows, replace=False))
    return rp.SampledRows(pts, tris, rows, *NQ, "elasticRH3", PARAMS, ft, classes=classes)


def test_c2_structure_matches_reference_finder(cuda, c2):
    pts, tris, classes = c2
    op = _op(pts, tris, np.float32)
    assert op.nearfield.bsr.nnzb == sum(v.shape[0] for v in classes.values())


@pytest.mark.parametrize("ft,tol,n_rows", [(np.float32, FP32_TOL, 512),
                                           (np.float64, FP64_TOL, 256)])
def test_c2_apply_vs_fp64_oracle(cuda, c2, ft, tol, n_rows):
    pts, tris, classes = c2
    op = _op(pts, tris, ft)
    x = np.random.default_rng(3).standard_normal(9 * tris.shape[0])
    y = op.dot(x.astype(ft))
    s = _rows(pts, tris, classes, n_rows, 17)
    want = s.apply(x.astype(ft).astype(np.float64))
    got = y.reshape(-1, 9)[s.rows].reshape(-1)
    err = rel(got, want)
    assert err <= tol, (np.dtype(ft).name, err)


def test_c2_panel_farfield_vs_fp64_oracle(cuda, c2):
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    pts, tris, classes = c2
    n = tris.shape[0]
    idx = np.arange(n)
    far = TriToTriDirectFarfieldOp(1, "elasticRH3", PARAMS, pts, tris, np.float32, idx, idx)
    assert far.panel_supported()
    X = np.random.default_rng(4).standard_normal((16, 9 * n)).astype(np.float32)
    Y = far.dot_panel(X)
    assert far.panel_error(16) == 0
    s = _rows(pts, tris, classes, 128, 23)
    for r in (0, 9, 15):
        want = s.farfield(X[r].astype(np.float64))
        got = Y[r].reshape(-1, 9)[s.rows].reshape(-1)
        assert rel(got, want) <= FP32_TOL, (r, rel(got, want))
