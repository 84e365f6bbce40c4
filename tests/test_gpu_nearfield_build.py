"""The nearfield operator built by the persistent batched pair kernel (all
four classes in one launch, the corrections in a second) against the
per-class launches (one single_pairs-style launch per class and rule, as the
reference's RegularizedNearfieldIntegralOp integrates): the same blocks in
the same BSR slots, up to summation order."""
import numpy as np
import pytest

import tectosaur_b200 as tct
from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp

from helpers import PARAMS, bumpy_mesh, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("K", ["elasticRH3", "elasticH3", "elasticU3", "elasticRT3"])
@pytest.mark.parametrize("ft,tol", [(np.float64, 1e-13), (np.float32, 2e-6)])
def test_batched_build_matches_per_class_launches(cuda, K, ft, tol):
    pts, tris = bumpy_mesh(12, seed=9, amp=0.2)
    args = (4, 4, 4, 2, 3, 2.5, K, K, PARAMS, pts, tris, ft, TriToTriDirectFarfieldOp)
    a = tct.RegularizedSparseIntegralOp(*args, batched=True)
    b = tct.RegularizedSparseIntegralOp(*args, batched=False)
    na, nb = a.nearfield, b.nearfield
    assert np.array_equal(na.bsr.indptr_host, nb.bsr.indptr_host)
    assert np.array_equal(na.bsr.indices_host, nb.bsr.indices_host)
    Da, Db = na.bsr.blocks_host(), nb.bsr.blocks_host()
    assert rel(Da, Db) < tol
    Ca, Cb = na.bsr.blocks_host(na.correction), nb.bsr.blocks_host(nb.correction)
    assert rel(Ca, Cb) < tol
    x = np.random.default_rng(1).standard_normal(a.shape[1]).astype(ft)
    assert rel(a.dot(x), b.dot(x)) < 10 * tol
    assert rel(na.nearfield_no_correction_dot(x), nb.nearfield_no_correction_dot(x)) < 10 * tol


def test_batched_build_is_deterministic(cuda):
    pts, tris = bumpy_mesh(10, seed=2)
    args = (5, 5, 5, 1, 4, 2.5, "elasticRH3", "elasticRH3", PARAMS, pts, tris, np.float64,
            TriToTriDirectFarfieldOp)
    a = tct.RegularizedSparseIntegralOp(*args).nearfield.bsr.blocks_host()
    b = tct.RegularizedSparseIntegralOp(*args).nearfield.bsr.blocks_host()
    assert np.array_equal(a, b)
