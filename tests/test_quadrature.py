"""Quadrature rules: bit-exact against the reference's rules (fixtures made
by tests/golden/make_golden.py) and the reference's closed-form checks
(tests/test_quadrature.py:55-147)."""
import hashlib

import numpy as np
import pytest

from tectosaur_b200.nearfield import triangle_rules as tr
from tectosaur_b200.util import quadrature as q


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def test_gauss_legendre_bit_exact(golden):
    g = golden("quad_rules.npz")
    for n in range(1, 21):
        x, w = q.gaussxw(n)
        assert np.array_equal(x, g["gaussxw_%d_x" % n])
        assert np.array_equal(w, g["gaussxw_%d_w" % n])


def test_tri_rules_bit_exact(golden):
    g = golden("quad_rules.npz")
    for n in range(1, 12):
        p, w = q.gauss2d_tri(n)
        assert np.array_equal(p, g["gauss2d_tri_%d_p" % n]), n
        assert np.array_equal(w, g["gauss2d_tri_%d_w" % n]), n


def test_singular_rules_bit_exact(golden):
    g = golden("quad_rules.npz")
    makers = {"coincident": tr.coincident_quad, "edge_adj": tr.edge_adj_quad,
              "vertex_adj": lambda k: tr.vertex_adj_quad(k, k, k)}
    for n in [2, 3]:
        for name, f in makers.items():
            p, w = f(n)
            assert np.array_equal(p, g["%s_%d_p" % (name, n)]), (name, n)
            assert np.array_equal(w, g["%s_%d_w" % (name, n)]), (name, n)
    for line in g["digests"]:
        parts = str(line).split()
        name, n = parts[0], parts[1]
        if name == "gauss4d_tri":
            a, b = map(int, n.split(","))
            p, w = q.gauss4d_tri(a, b)
        else:
            p, w = makers[name](int(n))
        assert p.shape[0] == int(parts[2]), line
        assert sha(p) == parts[3] and sha(w) == parts[4], line


def test_gauss_kat():
    est = q.quadrature(lambda x: x ** 7, q.map_to(q.gaussxw(4), [0, 1]))
    np.testing.assert_almost_equal(est, 1.0 / 8.0)


def test_gauss2d_tri_kats():
    np.testing.assert_almost_equal(q.quadrature(lambda x: 1, q.gauss2d_tri(2)), 0.5)
    res = q.quadrature(lambda x: x[:, 0] ** 3 * x[:, 1] ** 4, q.gauss2d_tri(5))
    np.testing.assert_almost_equal(res, 1.0 / 2520.0, 12)
    res = q.quadrature(lambda x: np.sin(np.exp(x[:, 0] * x[:, 1] * 5)), q.gauss2d_tri(7))
    np.testing.assert_almost_equal(res, 0.426659055902, 4)
    assert q.gauss2d_tri(3)[0].shape[0] == 7


def test_gauss4d_tri_kat():
    r = q.gauss4d_tri(3, 3)
    np.testing.assert_almost_equal(q.quadrature(lambda x: 1, r), 0.25)
    np.testing.assert_almost_equal(
        q.quadrature(lambda x: (x[:, 0] * x[:, 1] * x[:, 2] * x[:, 3]) ** 2, r),
        1.0 / 180.0 ** 2, 10)


def check_simple(rule, digits):
    np.testing.assert_almost_equal(q.quadrature(lambda p: 1.0, rule), 0.25, digits)
    np.testing.assert_almost_equal(
        q.quadrature(lambda p: p[:, 0] * p[:, 1] * p[:, 2] * p[:, 3], rule), 1.0 / 576.0, digits)
    np.testing.assert_almost_equal(
        q.quadrature(lambda p: p[:, 0] ** 6 * p[:, 1] * p[:, 3], rule), 1.0 / 3024.0, digits)
    np.testing.assert_almost_equal(
        q.quadrature(lambda p: p[:, 0] * p[:, 1] * p[:, 3] ** 6, rule), 1.0 / 1344.0, digits)
    np.testing.assert_almost_equal(
        q.quadrature(lambda p: p[:, 0] * p[:, 2] ** 6 * p[:, 3], rule), 1.0 / 3024.0, digits)


def test_vertex_adjacent_simple():
    check_simple(tr.vertex_adj_quad(8, 8, 8), 7)


def test_coincident_simple():
    check_simple(tr.coincident_quad(10), 7)


def test_edge_adj_simple():
    check_simple(tr.edge_adj_quad(6), 7)


# The reference's edge-adjacent variant of this check (test_edge_adj_real)
# assumes an older source reflection (y -> -y); with the rule the reference
# now ships (bit-identical to this one) it does not converge, so only the
# coincident and vertex checks are kept.
@pytest.mark.parametrize("maker,fn", [
    ("coincident", lambda p: 1.0 / np.sqrt((p[:, 0] - p[:, 2]) ** 2 + (p[:, 1] - p[:, 3]) ** 2)),
    ("vertex", lambda p: 1.0 / np.sqrt((p[:, 0] + p[:, 2]) ** 2 + (p[:, 1] + p[:, 3]) ** 2)),
])
def test_singular_rules_converge(maker, fn):
    mk = {"coincident": tr.coincident_quad,
          "vertex": lambda n: tr.vertex_adj_quad(n, n, n)}[maker]
    est = [q.quadrature(fn, mk(n)) for n in [9, 10]]
    np.testing.assert_almost_equal(est[0], est[1])


def test_rule_sizes():
    assert tr.coincident_quad(6)[0].shape[0] == 6048
    assert tr.edge_adj_quad(6)[0].shape[0] == 6480
    assert tr.vertex_adj_quad(6, 6, 6)[0].shape[0] == 2592
    assert q.gauss4d_tri(5, 5)[0].shape[0] == 361
