"""Row shards of the operator on one GPU: the applies of
RegularizedSparseIntegralOp(..., row_range=(r0, r1)) over a partition of the
rows, stacked, against the full operator's apply -- the nearfield bit for bit
(same pairs, same blocks, same per-row summation); with the direct farfield
the whole apply to FP64 rounding (the farfield's source chunking depends on
the row count), with the FMM farfield bit for bit (the same trees and
lists, evaluated on the shard's nodes)."""
import numpy as np
import pytest

import tectosaur_b200 as tct
from tectosaur_b200.ops.sparse_farfield_op import FMMFarfieldOp, TriToTriDirectFarfieldOp
from tectosaur_b200.sharded import row_ranges

from helpers import PARAMS, bumpy_mesh, rel

pytestmark = pytest.mark.gpu

ARGS = (3, 3, 3, 2, 3, 2.5, "elasticRH3", "elasticRH3", PARAMS)


@pytest.mark.parametrize("ft", [np.float64, np.float32])
@pytest.mark.parametrize("world", [2, 3])
def test_row_shards_stack_to_the_full_apply(cuda, ft, world):
    pts, tris = bumpy_mesh(21, seed=8, amp=0.3)
    n = tris.shape[0]
    full = tct.RegularizedSparseIntegralOp(*ARGS, pts, tris, ft, TriToTriDirectFarfieldOp)
    x = np.random.default_rng(2).standard_normal(9 * n).astype(ft)
    near_full = full.nearfield.dot(x)
    y_full = full.dot(x)
    near_parts, y_parts = [], []
    for r0, r1 in row_ranges(n, world):
        sh = tct.RegularizedSparseIntegralOp(*ARGS, pts, tris, ft, TriToTriDirectFarfieldOp,
                                             row_range=(r0, r1))
        assert sh.shape == (9 * (r1 - r0), 9 * n)
        near_parts.append(sh.nearfield.dot(x))
        y_parts.append(sh.dot(x))
    assert np.array_equal(np.concatenate(near_parts), near_full)
    tol = 1e-12 if ft == np.float64 else 1e-6
    assert rel(np.concatenate(y_parts), y_full) <= tol


@pytest.mark.parametrize("ft", [np.float64, np.float32])
@pytest.mark.parametrize("mode", ["fmm", "treecode"])
def test_fmm_row_shards_bit_identical(cuda, ft, mode):
    """An FMM operator's row shards keep the whole observation set's trees and
    lists and evaluate only the nodes holding their rows: stacked, they are
    the full apply bit for bit (farfield and whole operator)."""
    pts, tris = bumpy_mesh(24, seed=9, amp=0.3)
    n = tris.shape[0]
    fmm = FMMFarfieldOp(3.0, 30, 5, mode=mode)
    full = tct.RegularizedSparseIntegralOp(*ARGS, pts, tris, ft, fmm)
    x = np.random.default_rng(4).standard_normal(9 * n).astype(ft)
    far_full = full.farfield.dot(x)
    y_full = full.dot(x)
    for world in (2, 3):
        far_parts, y_parts = [], []
        for r0, r1 in row_ranges(n, world):
            sh = tct.RegularizedSparseIntegralOp(*ARGS, pts, tris, ft, fmm, row_range=(r0, r1))
            assert sh.shape == (9 * (r1 - r0), 9 * n)
            far_parts.append(sh.farfield.dot(x))
            y_parts.append(sh.dot(x))
        assert np.array_equal(np.concatenate(far_parts), far_full)
        assert np.array_equal(np.concatenate(y_parts), y_full)
    # a shard evaluates fewer observation leaves than the full operator
    sh = tct.RegularizedSparseIntegralOp(*ARGS, pts, tris, ft, fmm, row_range=(0, n // 3))
    assert sh.farfield.fmm.p2p.obs_n_idxs.shape[0] < full.farfield.fmm.p2p.obs_n_idxs.shape[0]


def test_fmm_row_shard_astype_and_accumulate(cuda):
    """astype keeps the row range (the FP32 twin of an FP64 shard); an
    accumulating apply adds the rows to the given vector."""
    import torch
    pts, tris = bumpy_mesh(18, seed=3, amp=0.3)
    n = tris.shape[0]
    fmm = FMMFarfieldOp(3.0, 30, 5, mode="fmm")
    rr = (n // 4, 3 * n // 4)
    sh = tct.RegularizedSparseIntegralOp(*ARGS, pts, tris, np.float64, fmm, row_range=rr)
    full32 = tct.RegularizedSparseIntegralOp(*ARGS, pts, tris, np.float32, fmm)
    tw = sh.astype(np.float32)
    x = np.random.default_rng(7).standard_normal(9 * n).astype(np.float32)
    want = full32.farfield.dot(x)[9 * rr[0]:9 * rr[1]]
    assert np.array_equal(tw.farfield.dot(x), want)
    y = torch.ones(9 * (rr[1] - rr[0]), dtype=torch.float32, device="cuda")
    tw.farfield.dot_device(torch.from_numpy(x).cuda(), y, accumulate=True)
    assert np.array_equal(y.cpu().numpy(), (torch.from_numpy(want) + 1.0).numpy())
