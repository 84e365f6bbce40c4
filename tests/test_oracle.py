"""The oracle (CPU restatement of the reference kernel math) pinned against
the reference's golden vectors and self-consistency checks."""
import numpy as np
import pytest

from tectosaur_b200.util.quadrature import gauss2d_tri, gauss4d_tri

from helpers import ALL_KERNELS, rel, two_surfaces


def test_farfield_two_tris_golden(orc, golden):
    # tests/test_integral_op.py:82-94 (elasticH3, nq=3, float32, 6 decimals)
    g = golden("ref_goldens.npz")["test_farfield_two_tris"]
    pts = np.array([[1, 0, 0], [2, 0, 0], [1, 1, 0], [5, 0, 0], [6, 0, 0], [5, 1, 0]], float)
    for ft in [np.float32, np.float64]:
        out = orc.farfield_tris_dense("elasticH3", ft, gauss4d_tri(3, 3), pts, [[0, 1, 2]],
                                      [[3, 4, 5]], [1.0, 0.25])
        np.testing.assert_almost_equal(out, g, 6)
        assert rel(out, g) < 1e-6


def test_point_kernels_vs_sympy(orc, golden):
    # tests/test_elastic.py:21-72: U/T/A/H point values vs the Carini &
    # Salvadori sympy derivation (relative 1e-4 there; FP64 here: 1e-12)
    d = golden("kernel_values.npz")
    names = ["elasticU3", "elasticT3", "elasticA3", "elasticH3"]
    for c, v in zip(d["cases"], d["values"]):
        k, i, j = map(int, c[:3])
        p = c[3:]
        V = np.zeros(3)
        V[j] = 1.0
        out = orc.farfield_pts(names[k], np.float64, p[7:10][None], p[13:16][None],
                               p[4:7][None], p[10:13][None], V, p[0:2])
        assert abs(out[i] - v) <= 1e-12 * max(abs(v), 1e-12), (names[k], i, j)


@pytest.mark.parametrize("K", ALL_KERNELS)
def test_vector_form_equals_tensor_form(orc, K):
    # matrix_free.cl (vector forms) and assemble.cl (tensor forms) are two
    # independent restatements of each kernel; contracted with v they agree
    rng = np.random.default_rng(3)
    pts = rng.random((12, 3)) * 2
    pts[6:, 0] += 4
    obs = np.array([[0, 1, 2], [3, 4, 5], [1, 3, 5]])
    src = np.array([[6, 7, 8], [9, 10, 11], [7, 9, 11], [8, 6, 10]])
    v = rng.standard_normal(src.shape[0] * 9)
    for nq in [1, 2, 3]:
        y1 = orc.farfield_tris(K, np.float64, gauss2d_tri(nq), pts, obs, src, v, [1.3, 0.27])
        M = orc.farfield_tris_dense(K, np.float64, gauss4d_tri(nq, nq), pts, obs, src,
                                    [1.3, 0.27]).reshape(27, 36)
        assert rel(y1, M @ v) < 1e-13


@pytest.mark.parametrize("K", ["T", "A", "H"])
def test_regularized_matches_unregularized_far(orc, K):
    # tests/test_regularized.py:168-215: for a continuous input that vanishes
    # on the source boundary, the integration-by-parts (surface-curl) forms
    # RT/RA/RH agree with T/A/H on separated surfaces
    (pts, tris), s1, s2 = two_surfaces(n=14, sep=1.5)
    cent = pts[tris[s2]]
    x = cent[..., 0]
    z = cent[..., 2]
    bump = ((1 - x ** 2) * (1 - z ** 2)) ** 2
    v = np.zeros((s2.shape[0], 3, 3))
    for d in range(3):
        v[:, :, d] = bump * (0.5 + 0.25 * d)
    v = v.reshape(-1)
    q = gauss2d_tri(4)
    y_plain = orc.farfield_tris("elastic%s3" % K, np.float64, q, pts, tris[s1], tris[s2], v,
                                [1.0, 0.25])
    y_reg = orc.farfield_tris("elasticR%s3" % K, np.float64, q, pts, tris[s1], tris[s2], v,
                              [1.0, 0.25])
    if K == "T":
        assert rel(y_reg, y_plain) < 2e-3
    else:
        # A and H act through the observation surface: compare the
        # observation-basis sums (what a continuity constraint projects onto)
        def node_sum(y):
            yy = y.reshape(-1, 3, 3)
            out = np.zeros((pts.shape[0], 3))
            np.add.at(out, tris[s1].reshape(-1), yy.reshape(-1, 3))
            return out
        a, b = node_sum(y_reg), node_sum(y_plain)
        inner = np.abs(pts[:, 0]) < 0.7
        inner &= np.abs(pts[:, 2]) < 0.7
        inner &= np.abs(pts[:, 1]) < 1e-9
        assert rel(a[inner], b[inner]) < 2e-3


def test_bsr_matches_bcoo(orc):
    rng = np.random.default_rng(0)
    nb, n = 200, 30
    rows = rng.integers(0, n, nb)
    cols = rng.integers(0, n, nb)
    data = rng.standard_normal((nb, 9, 9))
    x = rng.standard_normal(9 * n)
    indptr, indices, d2 = orc.make_bsr(n, rows, cols, data)
    y1 = orc.bsr_matvec(np.float64, indptr, indices, d2, x)
    y2 = orc.bcoo_matvec(np.float64, rows, cols, data, x, 9 * n)
    A = np.zeros((9 * n, 9 * n))
    for r, c, b in zip(rows, cols, data):
        A[9 * r:9 * r + 9, 9 * c:9 * c + 9] += b
    assert rel(y1, A @ x) < 1e-14 and rel(y2, A @ x) < 1e-14
