"""The BSR nearfield matvec applied to a panel of vectors in one launch
(tct_bsr9_matvec_panel) against the single-vector kernel, and the operator's
panel apply (RegularizedSparseIntegralOp.dot_panel) against dot per vector."""
import numpy as np
import pytest
import torch

import tectosaur_b200 as tct
from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
from tectosaur_b200.util.sparse import DeviceBSR9, auto_row_align, make_bsr_index

from helpers import PARAMS, bumpy_mesh, rel

pytestmark = pytest.mark.gpu


def _random_bsr(n_rows, n_cols, nnz, ft, seed, row_align=1):
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, n_rows, nnz)
    cols = rng.integers(0, n_cols, nnz)
    # one empty row and one long row (more than 32 blocks: several lane passes)
    rows[rows == 1] = 0
    rows[:70] = 2
    indptr, indices, slot = make_bsr_index(n_rows, rows, cols)
    m = DeviceBSR9((9 * n_rows, 9 * n_cols), indptr, indices, ft, row_align=row_align)
    blocks = rng.standard_normal((nnz, 81))
    planes = torch.from_numpy(np.ascontiguousarray(blocks.T)).to(m.data.dtype).cuda()
    if m.pos is None:
        m.data.copy_(planes.reshape(-1))
    else:
        m.data.view(81, m.stride)[:, torch.from_numpy(m.pos).cuda()] = planes
    return m


@pytest.mark.parametrize("align", [1, 32])
def test_autotune_times_the_padded_layout(cuda, align):
    """The BSR tuner runs the matrix in its own layout (slot stride, not the
    block count): its output after tuning is the product."""
    from tectosaur_b200 import autotune
    autotune.clear()
    b = _random_bsr(300, 250, 6000, np.float32, seed=4, row_align=align)
    x = torch.from_numpy(np.random.default_rng(5).standard_normal(b.shape[1])
                         .astype(np.float32)).cuda()
    want = torch.empty(b.shape[0], device="cuda")
    b.matvec(x, want)
    y = torch.full((b.shape[0],), 7.0, device="cuda")
    try:
        autotune.tune_bsr(b, x, y)
    finally:
        autotune.clear()
    assert float(torch.linalg.norm(y - want) / torch.linalg.norm(want)) < 2e-6


@pytest.mark.parametrize("ft", [np.float32, np.float64])
@pytest.mark.parametrize("align", [8, 32])
def test_padded_rows_match_unpadded(cuda, ft, align):
    """Rows padded to `align` slots: the same lane takes the same block of a
    row as unpadded, so single and panel applies agree bit for bit, and the
    padding (index -1) is never read."""
    a = _random_bsr(300, 250, 6000, ft, seed=3)
    b = _random_bsr(300, 250, 6000, ft, seed=3, row_align=align)
    assert b.stride % align == 0 and b.stride > b.nnzb
    assert torch.all(b.indices.view(-1)[torch.from_numpy(b.pos).cuda()] >= 0)
    assert int((b.indices < 0).sum()) == b.stride - b.nnzb
    # poison the padding: a padded slot that were read would show
    pad = torch.ones(b.stride, dtype=torch.bool, device="cuda")
    pad[torch.from_numpy(b.pos).cuda()] = False
    b.data.view(81, b.stride)[:, pad] = float("nan")
    tdt = torch.float32 if ft == np.float32 else torch.float64
    x = torch.randn(9 * 250, dtype=tdt, device="cuda")
    assert torch.equal(a.matvec(x, torch.empty(9 * 300, dtype=tdt, device="cuda")),
                       b.matvec(x, torch.empty(9 * 300, dtype=tdt, device="cuda")))
    X = torch.randn((5, 9 * 250), dtype=tdt, device="cuda")
    Ya = a.matvec_panel(X, torch.empty((5, 9 * 300), dtype=tdt, device="cuda"))
    Yb = b.matvec_panel(X, torch.empty((5, 9 * 300), dtype=tdt, device="cuda"))
    assert torch.equal(Ya, Yb)
    assert np.array_equal(a.blocks_host(), b.blocks_host())


@pytest.mark.parametrize("ft", [np.float32, np.float64])
@pytest.mark.parametrize("R", [1, 3, 8, 13, 16])
def test_bsr_panel_matches_single(cuda, ft, R):
    m = _random_bsr(300, 250, 6000, ft, seed=R)
    tdt = torch.float32 if ft == np.float32 else torch.float64
    X = torch.randn((R, 9 * 250), dtype=torch.float64, device="cuda").to(tdt)
    Y = torch.empty((R, 9 * 300), dtype=tdt, device="cuda")
    m.matvec_panel(X, Y)
    want = torch.empty_like(Y)
    for r in range(R):
        m.matvec(X[r], want[r])
    tol = 1e-6 if ft == np.float32 else 1e-14
    assert rel(Y.cpu().numpy(), want.cpu().numpy()) < tol
    assert np.all(Y[:, 9:18].cpu().numpy() == 0)  # the empty row


def test_bsr_panel_strides_and_accumulate(cuda):
    m = _random_bsr(200, 200, 3000, np.float32, seed=9)
    R = 10
    Xbig = torch.randn((R, 9 * 200 + 37), device="cuda")
    Ybig = torch.randn((R, 9 * 200 + 5), device="cuda")
    X, Y = Xbig[:, :9 * 200], Ybig[:, :9 * 200]
    Y0 = Y.clone()
    tail = Ybig[:, 9 * 200:].clone()
    m.matvec_panel(X, Y, accumulate=True)
    want = Y0.clone()
    for r in range(R):
        m.matvec(X[r].contiguous(), want[r], accumulate=True)
    assert rel(Y.cpu().numpy(), want.cpu().numpy()) < 1e-6
    assert torch.equal(Ybig[:, 9 * 200:], tail)  # nothing written past a row


@pytest.mark.parametrize("ft", [np.float32, np.float64])
def test_operator_panel_matches_dot(cuda, ft):
    pts, tris = bumpy_mesh(10, seed=4)
    op = tct.RegularizedSparseIntegralOp(3, 3, 3, 1, 3, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                         pts, tris, ft, TriToTriDirectFarfieldOp)
    X = np.random.default_rng(2).standard_normal((5, op.shape[1])).astype(ft)
    got = op.dot_panel(X)
    want = np.stack([op.dot(X[r]) for r in range(5)])
    tol = 1e-5 if ft == np.float32 else 1e-13
    assert rel(got, want) < tol


def test_operator_nearfield_rows_padded(cuda):
    """The operator's nearfield matrix pads its rows (their average length is
    above the threshold) and gives the unpadded matrix's apply bit for bit."""
    pts, tris = bumpy_mesh(10, seed=4)
    op = tct.RegularizedSparseIntegralOp(3, 3, 3, 1, 3, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                         pts, tris, np.float32, TriToTriDirectFarfieldOp)
    bsr = op.nearfield.bsr
    assert bsr.row_align == auto_row_align(bsr.n_row_blocks, bsr.nnzb) > 1
    assert bsr.stride % bsr.row_align == 0 and bsr.stride >= bsr.nnzb
    flat = DeviceBSR9(bsr.shape, bsr.indptr_host, bsr.indices_host, np.float32)
    flat.data.copy_(torch.from_numpy(
        np.ascontiguousarray(bsr.blocks_host().reshape(-1, 81).T).ravel()).cuda())
    x = torch.randn(op.shape[1], device="cuda")
    assert torch.equal(bsr.matvec(x, torch.empty(op.shape[0], device="cuda")),
                       flat.matvec(x, torch.empty(op.shape[0], device="cuda")))
