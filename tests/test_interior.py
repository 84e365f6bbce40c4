"""Interior evaluation, host side: the oracle restatements of the
point-triangle integrals and the triangle-to-point farfield pinned to the
reference's own golden master (tests/golden_masters/test_interior.npy:
elasticH3 at points one unit above a 3 x 3 plate, FP32), and the
vertex/near split of point-triangle pairs against the reference's
split_vertex_nearfield semantics."""
import numpy as np

from tectosaur_b200.mesh.find_near_adj import split_vertex_nearfield
from tectosaur_b200.mesh.mesh_gen import make_rect
from tectosaur_b200.util.quadrature import gauss2d_tri


def _golden_case():
    # test_integral_op.py:199-217 of the reference
    np.random.seed(10)
    corners = [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]]
    pts, tris = make_rect(3, 3, corners)
    obs_pts = pts.copy()
    obs_pts[:, 2] += 1.0
    obs_ns = np.random.rand(*obs_pts.shape)
    obs_ns /= np.linalg.norm(obs_ns, axis=1)[:, np.newaxis]
    return pts, tris, obs_pts, obs_ns, np.ones(tris.shape[0] * 9)


def test_interior_oracle_matches_reference_golden(orc, golden):
    # Every pair is near (threshold 4): far - near_far cancels and the
    # result is the nq = 4 point-triangle integrals, the configuration the
    # golden master was made with.
    want = golden("ref_goldens.npz")["test_interior"]
    pts, tris, obs_pts, obs_ns, v = _golden_case()
    n_obs, n_src = obs_pts.shape[0], tris.shape[0]
    pairs = np.array([[i, j, 0] for i in range(n_obs) for j in range(n_src)])
    E = orc.interior_pairs("elasticH3", np.float32, gauss2d_tri(4), obs_pts, obs_ns, pts, tris,
                           pairs, [1.0, 0.25])
    out = np.zeros(n_obs * 3)
    for k, (i, j, _) in enumerate(pairs):
        out[3 * i:3 * i + 3] += E[k].reshape(3, 9) @ v[9 * j:9 * j + 9]
    assert np.abs(out - want).max() / np.abs(want).max() < 1e-6
    far = orc.farfield_tris_to_pts("elasticH3", np.float32, gauss2d_tri(4), obs_pts, obs_ns,
                                   pts, tris, v, [1.0, 0.25])
    assert np.abs(far - want).max() / np.abs(want).max() < 1e-6


def test_split_vertex_nearfield():
    pts, tris = make_rect(4, 4, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]])
    obs = np.concatenate([pts[[0, 5, 9]], [[0.1, 0.2, 0.3], [0.0, 0.0, 1e-12]]])
    pairs = np.array([[i, j] for i in range(obs.shape[0]) for j in range(tris.shape[0])])
    vert, near = split_vertex_nearfield(pairs, obs, pts, tris)
    assert vert.shape[0] + near.shape[0] == pairs.shape[0]
    for i, j, d in vert:
        assert np.linalg.norm(obs[i] - pts[tris[j, d]]) < 1e-9
    for i, j, d in near:
        assert d == 0 and np.min(np.linalg.norm(obs[i] - pts[tris[j]], axis=1)) >= 1e-9
    # order kept within each class
    assert np.all(np.diff(near[:, 0] * 1000 + near[:, 1]) > 0)
    assert np.all(np.diff(vert[:, 0] * 1000 + vert[:, 1]) > 0)
