"""Tuned launch shapes on the GPU: every shape the autotuner can pick gives
the default shape's result (up to summation order), and the tuner's choice
is one of its candidates.  Forced shapes go through the same cache the
tuner writes (tct_tune_set)."""
import numpy as np
import pytest
import scipy.sparse

import tectosaur_b200 as tct
from tectosaur_b200 import _lib, autotune
from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
from tectosaur_b200.util import device
from tectosaur_b200.util.sparse import DeviceBSR9

from helpers import PARAMS, bumpy_mesh, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _empty_cache():
    autotune.clear()
    yield
    autotune.clear()


def _short_row_bsr(ft, n_rows=5000, seed=0):
    # rows of 0-3 blocks (the shape of the batched pair-quadrature matrices)
    rng = np.random.default_rng(seed)
    counts = rng.integers(0, 4, n_rows)
    indptr = np.concatenate([[0], np.cumsum(counts)])
    nnzb = int(indptr[-1])
    indices = rng.integers(0, n_rows, nnzb)
    blocks = rng.standard_normal((nnzb, 9, 9))
    m = DeviceBSR9((9 * n_rows, 9 * n_rows), indptr, indices, ft)
    m.data = device.to_dev(np.ascontiguousarray(blocks.reshape(nnzb, 81).T).reshape(-1), ft)
    A = scipy.sparse.bsr_matrix((blocks, indices, indptr), shape=(9 * n_rows, 9 * n_rows))
    return m, A


@pytest.mark.parametrize("ft,tol", [(np.float64, 1e-13), (np.float32, 2e-6)])
def test_bsr_every_shape_matches_scipy(cuda, ft, tol):
    m, A = _short_row_bsr(ft)
    x = np.random.default_rng(3).standard_normal(A.shape[1])
    want = A @ x
    xd = device.to_dev(x, ft)
    for lanes in (32, 16, 8, 4, 2, 1):
        for ctas in (4, 6, 8, 12, 16):
            _lib.lib.tct_tune_set(_lib.TCT_TUNE_BSR9, -1, _lib.prec_of(ft), 0, 1,
                                  m.n_row_blocks, max(1, m.nnzb // m.n_row_blocks), lanes, ctas)
            y = device.torch().full((A.shape[0],), 7.0, dtype=xd.dtype, device="cuda")
            m.matvec(xd, y)
            assert rel(y.cpu().numpy(), want) < tol, (lanes, ctas)
            y2 = device.torch().ones_like(y)
            m.matvec(xd, y2, accumulate=True)
            assert rel(y2.cpu().numpy(), want + 1.0) < tol, (lanes, ctas)
    autotune.clear()
    lanes, ctas = autotune.tune_bsr(m)
    assert lanes in (32, 16, 8, 4, 2, 1) and ctas in (4, 6, 8, 12, 16)
    y = device.torch().empty_like(xd)
    m.matvec(xd, y)
    assert rel(y.cpu().numpy(), want) < tol


@pytest.mark.parametrize("ft,tol", [(np.float64, 1e-13), (np.float32, 1e-6)])
def test_farfield_chunk_counts_match_default(cuda, ft, tol):
    pts, tris = bumpy_mesh(23, seed=4)
    n = tris.shape[0]
    idx = np.arange(n)
    far = TriToTriDirectFarfieldOp(1, "elasticRH3", PARAMS, pts, tris, ft, idx, idx)
    x = device.to_dev(np.random.default_rng(5).standard_normal(9 * n), ft)
    y0 = device.torch().empty_like(x)
    far.dot_device(x, y0)
    want = y0.cpu().numpy()
    chosen = far.autotune(x)
    assert chosen in (1, 2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 48, 64)
    for c in (1, 3, chosen, 64):
        _lib.lib.tct_tune_set(_lib.TCT_TUNE_FARFIELD, far.kid, far.prec, far.n_q, 1, far.n_obs,
                              far.n_src, c, 1)
        y = device.torch().empty_like(x)
        far.dot_device(x, y)
        assert rel(y.cpu().numpy(), want) < tol, c


def test_operator_autotune_keeps_the_apply(cuda):
    pts, tris = bumpy_mesh(14, seed=6)
    op = tct.RegularizedSparseIntegralOp(3, 3, 3, 2, 3, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                         pts, tris, np.float64, TriToTriDirectFarfieldOp)
    x = np.random.default_rng(7).standard_normal(op.shape[1])
    want = op.dot(x)
    shapes = op.autotune()
    assert set(shapes) == {"farfield_chunks", "bsr_lanes_per_row", "bsr_ctas_per_sm"}
    assert rel(op.dot(x), want) < 1e-13
    assert len(autotune.entries()) == 2
