"""Interior evaluation on the device against the oracle restatements
(pinned to the reference's interior golden master in test_interior.py):
point-triangle integrals, vertex integrals, the triangle-to-point farfield
and InteriorOp.dot."""
import numpy as np
import pytest
import torch

import tectosaur_b200 as tct
from tectosaur_b200.interior import make_pairs_mat
from tectosaur_b200.mesh.find_near_adj import get_nearfield, get_tri_centroids_rs, \
    split_vertex_nearfield
from tectosaur_b200.mesh.mesh_gen import make_rect
from tectosaur_b200.util.quadrature import gauss2d_tri, gaussxw, map_to

from test_interior import _golden_case

pytestmark = pytest.mark.gpu
PARAMS = [1.0, 0.25]


def _case(seed=3):
    rng = np.random.default_rng(seed)
    pts, tris = make_rect(5, 4, [[-1, -1, 0], [1, -1, 0.2], [1, 1, 0], [-1, 1, 0.1]])
    obs = np.concatenate([rng.uniform(-1.5, 1.5, (30, 3)), pts[:6]])  # some at vertices
    ns = rng.standard_normal(obs.shape)
    ns /= np.linalg.norm(ns, axis=1)[:, None]
    return pts, tris, obs, ns


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("K", ["elasticU3", "elasticT3", "elasticA3", "elasticH3"])
@pytest.mark.parametrize("ft", [np.float32, np.float64])
def test_interior_pairs_kernel(cuda, orc, K, ft):
    pts, tris, obs, ns = _case()
    rng = np.random.default_rng(4)
    pairs = np.column_stack([rng.integers(0, 30, 200), rng.integers(0, tris.shape[0], 200),
                             rng.integers(0, 3, 200)])
    far = tct.interior.TriToPtDirectFarfieldOp(obs, ns, (pts, tris), K, 2, PARAMS, ft)
    q = gauss2d_tri(5)
    got = tct.interior.interior_pairs_quad(K, pairs, q, far, ft)
    want = orc.interior_pairs(K, ft, q, obs, ns, pts, tris, pairs, PARAMS)
    assert _rel(got, want) < (2e-6 if ft == np.float32 else 1e-13)
    got_fp = tct.interior.interior_pairs_quad(K, pairs, q, far, ft, finite_part=True)
    want_fp = orc.interior_pairs(K, ft, q, obs, ns, pts, tris, pairs, PARAMS, finite_part=True)
    assert _rel(got_fp, want_fp) < (2e-6 if ft == np.float32 else 1e-13)


@pytest.mark.parametrize("ft", [np.float32, np.float64])
def test_interior_corners_kernel(cuda, orc, ft):
    pts, tris, obs, ns = _case()
    pairs, _ = split_vertex_nearfield(
        np.array([[i, j] for i in range(30, 36) for j in range(tris.shape[0])]), obs, pts, tris)
    assert pairs.shape[0] > 0
    far = tct.interior.TriToPtDirectFarfieldOp(obs, ns, (pts, tris), "elasticH3", 2, PARAMS, ft)
    q = map_to(gaussxw(8), [0.0, np.pi / 2])
    got = tct.interior.interior_corners_quad(pairs, q, far, ft)
    want = orc.interior_corners(ft, q, ns, pts, tris, pairs, PARAMS)
    assert _rel(got, want) < (2e-6 if ft == np.float32 else 1e-13)


@pytest.mark.parametrize("K", ["elasticU3", "elasticT3", "elasticA3", "elasticH3"])
def test_tris_to_pts_kernel(cuda, orc, K):
    pts, tris, obs, ns = _case()
    v = np.random.default_rng(6).standard_normal(tris.shape[0] * 9)
    for ft, tol in [(np.float32, 1e-5), (np.float64, 1e-12)]:
        op = tct.interior.TriToPtDirectFarfieldOp(obs, ns, (pts, tris), K, 3, PARAMS, ft)
        want = orc.farfield_tris_to_pts(K, ft, gauss2d_tri(3), obs, ns, pts, tris, v, PARAMS)
        assert _rel(op.dot(v), want) < tol


def test_interior_op_reference_golden(cuda, golden):
    want = golden("ref_goldens.npz")["test_interior"]
    pts, tris, obs_pts, obs_ns, v = _golden_case()
    op = tct.InteriorOp(obs_pts, obs_ns, (pts, tris), "elasticH3", 4, 8, 2, 4, PARAMS,
                        np.float32)
    assert op.vertex_pairs.shape[0] == 0
    got = op.dot(v)
    assert np.abs(got - want).max() / np.abs(want).max() < 5e-6


def test_interior_op_vs_oracle(cuda, orc):
    pts, tris, obs, ns = _case()
    K, nq_vertex, nq_far, nq_near = "elasticH3", 8, 2, 5
    op = tct.InteriorOp(obs, ns, (pts, tris), K, 4, nq_vertex, nq_far, nq_near, PARAMS,
                        np.float64)
    # the oracle composition of interior.py:77-83
    pairs = get_nearfield(obs, np.zeros(obs.shape[0]), *get_tri_centroids_rs(pts, tris), 4.0)
    vp, npairs = split_vertex_nearfield(pairs, obs, pts, tris)
    assert vp.shape[0] > 0 and npairs.shape[0] > 0
    allp = np.vstack((npairs, vp))
    allp[:, 2] = 0
    shape = (obs.shape[0] * 3, tris.shape[0] * 9)
    M = (make_pairs_mat(npairs, orc.interior_pairs(K, np.float64, gauss2d_tri(nq_near), obs, ns,
                                                   pts, tris, npairs, PARAMS), shape)
         - make_pairs_mat(allp, orc.interior_pairs(K, np.float64, gauss2d_tri(nq_far), obs, ns,
                                                   pts, tris, allp, PARAMS), shape)
         + make_pairs_mat(vp, orc.interior_corners(np.float64, map_to(gaussxw(nq_vertex),
                                                                      [0.0, np.pi / 2]),
                                                   ns, pts, tris, vp, PARAMS), shape))
    v = np.random.default_rng(7).standard_normal(tris.shape[0] * 9)
    want = orc.farfield_tris_to_pts(K, np.float64, gauss2d_tri(nq_far), obs, ns, pts, tris, v,
                                    PARAMS) + M @ v
    got = op.dot(v)
    assert _rel(got, want) < 1e-11
    assert torch.is_tensor(op.dot(torch.from_numpy(v).cuda()))
