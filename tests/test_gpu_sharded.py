"""Row shards of the operator on one GPU: the applies of
RegularizedSparseIntegralOp(..., row_range=(r0, r1)) over a partition of the
rows, stacked, against the full operator's apply -- the nearfield bit for bit
(same pairs, same blocks, same per-row summation), the whole apply to FP64
rounding (the farfield's source chunking depends on the row count)."""
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


def test_fmm_operator_refuses_row_range(cuda):
    pts, tris = bumpy_mesh(9)
    with pytest.raises(ValueError, match="row_range"):
        tct.RegularizedSparseIntegralOp(*ARGS, pts, tris, np.float64, FMMFarfieldOp(3.0, 20, 4),
                                        row_range=(0, 10))
