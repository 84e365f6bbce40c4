"""GPU parity: every device kernel through the C ABI against the oracle.

Tolerances (relative 2-norm over the whole output):
  FP64 device vs FP64 oracle: 1e-10 (the plain path's parity bar); observed ~1e-14.
  FP32 device vs FP32 oracle: 2e-5 (float rounding, rsqrt vs 1/sqrt, FMA contraction).
"""
import numpy as np
import pytest

from tectosaur_b200.mesh import find_near_adj as fna
from tectosaur_b200.nearfield import triangle_rules as tr
from tectosaur_b200.nearfield.nearfield_op import nearfield_pairs
from tectosaur_b200.nearfield.pairs_integrator import PairsIntegrator
from tectosaur_b200.util.quadrature import gauss2d_tri, gauss4d_tri

from helpers import ALL_KERNELS, PARAMS, bumpy_mesh, rel, two_surfaces

pytestmark = pytest.mark.gpu

TOL = {np.float64: 1e-10, np.float32: 2e-5}


@pytest.fixture(scope="module")
def mesh_classes():
    pts, tris = bumpy_mesh(9, seed=11)
    cl = nearfield_pairs(pts, tris, np.arange(tris.shape[0]), np.arange(tris.shape[0]), 2.5)
    return pts, tris, cl


@pytest.mark.parametrize("ft", [np.float64, np.float32])
@pytest.mark.parametrize("K", ALL_KERNELS)
def test_pairs_all_classes(cuda, orc, mesh_classes, K, ft):
    pts, tris, cl = mesh_classes
    pi = PairsIntegrator(K, PARAMS, ft, 2, 3, pts, tris)
    cases = [
        ("coincident", lambda: pi.coincident(3, cl["co"][0]), tr.coincident_quad(3),
         cl["co"][0], False, True),
        ("edge", lambda: pi.edge_adj(3, cl["ea"][0]), tr.edge_adj_quad(3), cl["ea"][0], True, True),
        ("vertex", lambda: pi.vert_adj(3, cl["va"][0]), tr.vertex_adj_quad(3, 3, 3), cl["va"][0],
         True, True),
        ("near", lambda: pi.nearfield(cl["near"][0]), gauss4d_tri(3, 3), cl["near"][0], False, False),
        ("correction", lambda: pi.correction(cl["ea"][0][:, :2], False), gauss4d_tri(2, 2),
         cl["ea"][0][:, :2], False, False),
        ("correction0", lambda: pi.correction(cl["co"][0], True), gauss4d_tri(2, 2), cl["co"][0],
         False, True),
    ]
    for name, run, rule, recs, adj, check0 in cases:
        assert recs.shape[0] > 0, name
        got = run()
        assert got.dtype == np.dtype(ft) and got.shape == (recs.shape[0], 3, 3, 3, 3)
        want = orc.pairs(K, ft, rule, pts, tris, recs, PARAMS, adj=adj, check0=check0)
        assert np.all(np.isfinite(got)), name
        assert rel(got, want) < TOL[ft], (K, name, rel(got, want))


def test_pairs_flip_and_rotation_records(cuda, orc):
    # every (obs_clicks, src_clicks, flip) combination on one edge-adjacent pair
    pts = np.array([[0, 0, 0], [1, 0, 0], [0.3, 1, 0.2], [0.6, -0.9, 0.1]], float)
    tris = np.array([[0, 1, 2], [1, 0, 3]])
    recs = np.array([[0, 1, oc, sc, f] for oc in range(3) for sc in range(3) for f in (0, 1)])
    for K in ["elasticH3", "elasticRH3", "elasticRT3", "elasticRA3"]:
        pi = PairsIntegrator(K, PARAMS, np.float64, 2, 3, pts, tris)
        got = pi.pairs_quad(pi.edge_adj_rule(4), recs, True, True)
        want = orc.pairs(K, np.float64, tr.edge_adj_quad(4), pts, tris, recs, PARAMS, adj=True,
                         check0=True)
        assert rel(got, want) < 1e-12


@pytest.mark.parametrize("ft", [np.float64, np.float32])
@pytest.mark.parametrize("K", ALL_KERNELS)
def test_farfield_tris_matvec(cuda, orc, K, ft):
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    rng = np.random.default_rng(5)
    (pts, tris), s1, s2 = two_surfaces(n=9, sep=1.0)
    pts = pts + 0.01 * rng.standard_normal(pts.shape)
    all_t = np.arange(tris.shape[0])
    for nq in [1, 2, 3]:
        for obs, src in [(s1, s2), (all_t, all_t)]:
            op = TriToTriDirectFarfieldOp(nq, K, PARAMS, pts, tris, ft, obs, src)
            v = rng.standard_normal(op.shape[1])
            got = op.dot(v)
            want = orc.farfield_tris(K, ft, gauss2d_tri(nq), pts, tris[obs], tris[src], v, PARAMS)
            assert got.dtype == np.dtype(ft)
            assert rel(got, want) < TOL[ft], (K, nq, rel(got, want))


def test_farfield_chunked_grid_and_tail_tiles(cuda, orc):
    # sizes that exercise several source chunks, partial tiles and a partial
    # obs block (n_obs not a multiple of 128)
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    pts, tris = bumpy_mesh(31, seed=2)
    rng = np.random.default_rng(0)
    obs = np.arange(0, tris.shape[0], 3)
    src = np.arange(tris.shape[0])
    for K in ["elasticRH3", "elasticU3"]:
        op = TriToTriDirectFarfieldOp(1, K, PARAMS, pts, tris, np.float64, obs, src)
        v = rng.standard_normal(op.shape[1])
        want = orc.farfield_tris(K, np.float64, gauss2d_tri(1), pts, tris[obs], tris[src], v, PARAMS)
        assert rel(op.dot(v), want) < 1e-12


@pytest.mark.parametrize("ft", [np.float64, np.float32])
@pytest.mark.parametrize("K", ["elasticU3", "elasticT3", "elasticA3", "elasticH3"])
def test_farfield_pts(cuda, orc, K, ft):
    from tectosaur_b200.farfield import farfield_pts_direct
    rng = np.random.default_rng(100)
    n = 300
    obs = rng.random((n, 3))
    obs_n = rng.random((n, 3))
    obs_n /= np.linalg.norm(obs_n, axis=1)[:, None]
    src = rng.random((n + 17, 3))
    src_n = rng.random((n + 17, 3))
    src_n /= np.linalg.norm(src_n, axis=1)[:, None]
    src[:5] = obs[:5]  # coincident points are skipped (r^2 == 0)
    w = rng.random((n + 17) * 3)
    got = farfield_pts_direct(K, obs, obs_n, src, src_n, w, PARAMS, ft)
    want = orc.farfield_pts(K, ft, obs, obs_n, src, src_n, w, PARAMS)
    assert rel(got, want) < TOL[ft]


def test_point_kernels_vs_sympy_on_device(cuda, golden):
    from tectosaur_b200.farfield import farfield_pts_direct
    d = golden("kernel_values.npz")
    names = ["elasticU3", "elasticT3", "elasticA3", "elasticH3"]
    for c, v in zip(d["cases"], d["values"]):
        k, i, j = map(int, c[:3])
        p = c[3:]
        V = np.zeros(3)
        V[j] = 1.0
        out = farfield_pts_direct(names[k], p[7:10][None], p[13:16][None], p[4:7][None],
                                  p[10:13][None], V, p[0:2], np.float64)
        assert abs(out[i] - v) <= 1e-12 * max(abs(v), 1e-12)


def test_dense_farfield_golden_and_oracle(cuda, orc, golden):
    from tectosaur_b200.ops.dense_integral_op import farfield_tris
    g = golden("ref_goldens.npz")["test_farfield_two_tris"]
    pts = np.array([[1, 0, 0], [2, 0, 0], [1, 1, 0], [5, 0, 0], [6, 0, 0], [5, 1, 0]], float)
    out = farfield_tris("elasticH3", PARAMS, pts, np.array([[0, 1, 2]]), np.array([[3, 4, 5]]),
                        3, np.float32)
    np.testing.assert_almost_equal(out, g, 6)
    pts, tris = bumpy_mesh(6, seed=4)
    for K in ALL_KERNELS:
        out = farfield_tris(K, PARAMS, pts, tris[:20], tris[30:], 2, np.float64)
        want = orc.farfield_tris_dense(K, np.float64, gauss4d_tri(2, 2), pts, tris[:20],
                                       tris[30:], PARAMS)
        assert rel(out, want) < 1e-12


@pytest.mark.parametrize("ft", [np.float64, np.float32])
def test_bsr_matvec(cuda, orc, ft):
    from tectosaur_b200.util.sparse import BCOOMatrix
    rng = np.random.default_rng(9)
    for n, nb in [(1, 1), (50, 400), (300, 30000), (7, 0)]:
        rows = rng.integers(0, n, nb)
        cols = rng.integers(0, n, nb)
        data = rng.standard_normal((nb, 9, 9)).astype(ft)
        x = rng.standard_normal(9 * n)
        got = BCOOMatrix(rows, cols, data, (9 * n, 9 * n)).dot(x)
        want = orc.bcoo_matvec(np.float64, rows, cols, data.astype(np.float64), x, 9 * n)
        if nb == 0:
            assert np.all(got == 0)
        else:
            assert rel(got, want) < TOL[ft] / 10


def test_reference_sparse_unit_cases(cuda):
    # tests/test_sparse.py:8-73 (BSR / BCOO vs dense, block size 9 here)
    import scipy.sparse
    from tectosaur_b200.util.sparse import BCOOMatrix, from_scipy_bsr
    rng = np.random.default_rng(1)
    A = rng.random((90, 90))
    x = rng.random(90)
    np.testing.assert_almost_equal(from_scipy_bsr(scipy.sparse.bsr_matrix(A, blocksize=(9, 9))).dot(x),
                                   A.dot(x))
    nbr = 10
    data = np.swapaxes(A.reshape(nbr, 9, nbr, 9), 1, 2).reshape(-1, 9, 9).copy()
    rows = np.repeat(np.arange(nbr), nbr)
    cols = np.tile(np.arange(nbr), nbr)
    m = BCOOMatrix(rows, cols, data, A.shape)
    np.testing.assert_almost_equal(m.dot(x), A.dot(x))
    np.testing.assert_almost_equal(m.to_bsr().dot(x), A.dot(x))
