"""Multi-RHS elasticRT3 farfield on the tensor cores (A generated into
tensor memory, split TF32; csrc/rt_mrhs.cu) against the FP32 direct farfield
applied vector by vector and against the FP64 oracle."""
import numpy as np
import pytest
import torch

import tectosaur_b200 as tct
from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp

from helpers import PARAMS, bumpy_mesh, rel

pytestmark = pytest.mark.gpu


def _setup(n, R, seed=0, obs=None):
    pts, tris = bumpy_mesh(n, seed=seed)
    nt = tris.shape[0]
    idx = np.arange(nt)
    obs = idx if obs is None else obs
    op = TriToTriDirectFarfieldOp(1, "elasticRT3", PARAMS, pts, tris, np.float32, obs, idx)
    X = np.random.default_rng(seed + 1).standard_normal((R, 9 * nt)).astype(np.float32)
    return pts, tris, op, X


def _per_vector(op, X):
    Xd = torch.from_numpy(X).cuda()
    Y = torch.empty((X.shape[0], op.shape[0]), dtype=torch.float32, device="cuda")
    for r in range(X.shape[0]):
        op.dot_device(Xd[r].contiguous(), Y[r])
    return Y.cpu().numpy()


def _row_err(got, want):
    return np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)


@pytest.mark.parametrize("n,R", [(12, 16), (17, 32), (16, 20), (9, 5), (30, 16)])
def test_rt_panel_matches_per_vector(cuda, n, R):
    pts, tris, op, X = _setup(n, R)
    assert op.panel_supported() and op.n_q == 3
    got = op.dot_panel(X)
    want = _per_vector(op, X)
    assert op.panel_error(16) == 0
    err = _row_err(got, want)
    assert np.all(err < 1e-5), err


def test_rt_panel_vs_fp64_oracle(cuda, orc):
    from tectosaur_b200.util.quadrature import gauss2d_tri
    pts, tris, op, X = _setup(14, 16, seed=3)
    got = op.dot_panel(X)
    for r in [0, 7, 15]:
        want = orc.farfield_tris("elasticRT3", np.float64, gauss2d_tri(1), pts, tris, tris,
                                 X[r].astype(np.float64), PARAMS)
        assert np.linalg.norm(got[r] - want) / np.linalg.norm(want) < 1e-5


def test_rt_panel_unequal_weights(cuda):
    # a 3-point rule with unequal weights takes the kernel's other branch
    # (weights in A, not folded into B); the per-vector kernel gets the same rule
    pts, tris, op, X = _setup(11, 16, seed=8)
    op.qx = np.ascontiguousarray([[0.2, 0.3], [0.55, 0.15], [0.1, 0.6]], dtype=np.float64)
    op.qw = np.ascontiguousarray([0.22, 0.17, 0.11], dtype=np.float64)
    got = op.dot_panel(X)
    want = _per_vector(op, X)
    assert op.panel_error(16) == 0
    assert np.all(_row_err(got, want) < 1e-5)


def test_rt_panel_subset_and_accumulate(cuda):
    # observation points not a multiple of 128; accumulate into a given panel
    pts, tris, op, X = _setup(15, 16, seed=5, obs=np.arange(0, 300, 2))
    Xd = torch.from_numpy(X).cuda()
    Y = torch.ones((16, op.shape[0]), dtype=torch.float32, device="cuda")
    op.dot_panel_device(Xd, Y, accumulate=True)
    want = _per_vector(op, X) + 1.0
    assert rel(Y.cpu().numpy(), want) < 1e-5


def test_rt_operator_panel_matches_dot(cuda):
    """RegularizedSparseIntegralOp with elasticRT3: the panel apply (farfield
    panels on the tensor cores + the BSR panel) equals dot per vector."""
    pts, tris = bumpy_mesh(12, seed=4)
    op = tct.RegularizedSparseIntegralOp(3, 3, 3, 1, 3, 2.5, "elasticRT3", "elasticRT3", PARAMS,
                                         pts, tris, np.float32, TriToTriDirectFarfieldOp)
    X = np.random.default_rng(2).standard_normal((16, op.shape[1])).astype(np.float32)
    got = op.dot_panel(X)
    want = np.stack([op.dot(X[r]) for r in range(16)])
    assert np.all(_row_err(got, want) < 1e-5)

