"""The product-free CPU pipeline of the reference operator (oracle/ref_pipeline.py)
that bench.py's CPU legs time and check against: its pieces against the
reference's own outputs, and the composed sampled rows against the oracle
composition the rest of the suite uses."""
import numpy as np
import pytest

from oracle import oracle as orc
from oracle import ref_pipeline as rp

from helpers import PARAMS, bumpy_mesh, oracle_sparse_op_dot, rel

pytestmark = pytest.mark.skipif(not rp.available(),
                                reason="oracle/_ref (reference modules) not built")

SPLIT = np.load("tests/golden/near_split.npz") if rp.os.path.exists(
    "tests/golden/near_split.npz") else None


def test_make_rect_matches_product_mesh():
    from tectosaur_b200.mesh.mesh_gen import make_rect
    c = [[-1, -1, 0], [1, -1, 0.2], [1, 1, 0], [-1, 1, 0.3]]
    a = rp.make_rect(7, 5, c)
    b = make_rect(7, 5, c)
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[0], b[0])


@pytest.mark.parametrize("mesh", ["rect", "sphere", "bumpy"])
@pytest.mark.parametrize("thr", ["1p25", "2p5"])
def test_pairs_split_and_rotation_match_reference(mesh, thr):
    key = "%s_%s" % (mesh, thr)
    pts, tris = SPLIT[key + "_pts"], SPLIT[key + "_tris"]
    raw = SPLIT[key + "_pairs_raw"]
    got = rp.near_pairs(pts, tris, float(thr.replace("p", ".")))
    want = raw[np.lexsort((raw[:, 1], raw[:, 0]))]
    assert np.array_equal(got, want)
    ea = SPLIT[key + "_ea"]
    assert np.array_equal(rp.resolve_ea_rotation(tris, ea), SPLIT[key + "_ea_rot"])


def test_rules_are_the_reference_rules():
    q = np.load("tests/golden/quad_rules.npz")
    for n in (3,):
        for name in ("coincident", "edge_adj", "vertex_adj"):
            p, w = rp.rule(name, n)
            assert np.array_equal(p, q["%s_%d_p" % (name, n)])
            assert np.array_equal(w, q["%s_%d_w" % (name, n)])
    p, w = rp.rule("gauss2d_tri", 2)
    assert np.array_equal(p, q["gauss2d_tri_2_p"]) and np.array_equal(w, q["gauss2d_tri_2_w"])
    # the larger rules against the digests the reference produced
    import hashlib
    dig = set(str(d) for d in q["digests"])

    def sha(a):
        return hashlib.sha256(np.ascontiguousarray(a, np.float64).tobytes()).hexdigest()
    for name in ("coincident", "edge_adj", "vertex_adj"):
        p, w = rp.rule(name, 6)
        assert "%s 6 %d %s %s" % (name, p.shape[0], sha(p), sha(w)) in dig
    p, w = rp.rule("gauss4d", 5)
    assert "gauss4d_tri 5,5 %d %s %s" % (p.shape[0], sha(p), sha(w)) in dig


@pytest.mark.parametrize("ft,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_sampled_rows_match_oracle_composition(ft, tol):
    pts, tris = bumpy_mesh(9, seed=3)
    n = tris.shape[0]
    x = np.random.default_rng(5).standard_normal(9 * n)
    want = oracle_sparse_op_dot(orc, 3, 3, 3, 2, 3, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                pts, tris, ft, x)
    rows = np.sort(np.random.default_rng(6).choice(n, 40, replace=False))
    s = rp.SampledRows(pts, tris, rows, 3, 3, 3, 2, 3, 2.5, "elasticRH3", PARAMS, ft)
    got = s.apply(x)
    w = want.reshape(n, 9)[rows].reshape(-1)
    assert rel(got, w) < tol
    # the timed build agrees with the checker build
    s.fast = True
    assert rel(s.apply(x), w) < 1e-5
