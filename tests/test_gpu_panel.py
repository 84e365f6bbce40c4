"""Multi-RHS elasticRH3 farfield on the tensor cores (split TF32,
csrc/far_mrhs.cu) against the FP32 direct farfield applied vector by vector
and against the FP64 oracle."""
import numpy as np
import pytest
import torch

from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp

from helpers import PARAMS, bumpy_mesh

pytestmark = pytest.mark.gpu


def _setup(n, R, seed=0, obs=None, nq_far=1):
    pts, tris = bumpy_mesh(n, seed=seed)
    nt = tris.shape[0]
    idx = np.arange(nt)
    obs = idx if obs is None else obs
    op = TriToTriDirectFarfieldOp(nq_far, "elasticRH3", PARAMS, pts, tris, np.float32, obs, idx)
    X = np.random.default_rng(seed + 1).standard_normal((R, 9 * nt)).astype(np.float32)
    return pts, tris, op, X


def _per_vector(op, X):
    Xd = torch.from_numpy(X).cuda()
    Y = torch.empty((X.shape[0], op.shape[0]), dtype=torch.float32, device="cuda")
    for r in range(X.shape[0]):
        op.dot_device(Xd[r].contiguous(), Y[r])
    return Y.cpu().numpy()


@pytest.mark.parametrize("n,R", [(12, 16), (17, 32), (16, 20), (9, 5), (30, 16)])
def test_panel_matches_per_vector(cuda, n, R):
    pts, tris, op, X = _setup(n, R)
    assert op.panel_supported()
    got = op.dot_panel(X)
    want = _per_vector(op, X)
    assert op.panel_error(16) == 0
    err = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
    assert np.all(err < 1e-5), err


@pytest.mark.parametrize("nq_far", [2, 3])
def test_panel_rules_match_per_vector(cuda, nq_far):
    # the 4-point (negative centre weight) and 7-point rules
    pts, tris, op, X = _setup(13, 20, seed=7, nq_far=nq_far)
    assert op.panel_supported() and op.n_q == {2: 4, 3: 7}[nq_far]
    got = op.dot_panel(X)
    want = _per_vector(op, X)
    assert op.panel_error(16) == 0
    err = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
    assert np.all(err < 1e-5), err


@pytest.mark.parametrize("nq_far", [1, 2])
def test_panel_vs_fp64_oracle(cuda, orc, nq_far):
    from tectosaur_b200.util.quadrature import gauss2d_tri
    pts, tris, op, X = _setup(14, 16, seed=3, nq_far=nq_far)
    got = op.dot_panel(X)
    for r in [0, 7, 15]:
        want = orc.farfield_tris("elasticRH3", np.float64, gauss2d_tri(nq_far), pts, tris, tris,
                                 X[r].astype(np.float64), PARAMS)
        assert np.linalg.norm(got[r] - want) / np.linalg.norm(want) < 1e-5


def test_panel_subset_and_accumulate(cuda):
    # observation rows not a multiple of 128; accumulate into a given panel
    pts, tris, op, X = _setup(15, 16, seed=5, obs=np.arange(0, 300, 2))
    Xd = torch.from_numpy(X).cuda()
    Y = torch.ones((16, op.shape[0]), dtype=torch.float32, device="cuda")
    op.dot_panel_device(Xd, Y, accumulate=True)
    want = _per_vector(op, X) + 1.0
    got = Y.cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-5
