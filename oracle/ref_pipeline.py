"""Test infrastructure: the reference operator's CPU pipeline for sampled
observation rows, built without the product package (tectosaur_b200).

Used by tests/ and by bench.py's CPU legs (the timed CPU baseline, and the
FP64 parity figure of the benched configuration).  Nothing here is imported
by the product.  The pieces, each from the reference or restated from it:

  * meshes: ``make_rect`` (mesh/mesh_gen.py:7-47), restated;
  * near pairs and their classes: the reference's own compiled finder
    (oracle/_ref/fast_find_nearfield: ``get_nearfield`` and
    ``split_adjacent_close``, called as mesh/find_near_adj.py:13-35 calls
    them);
  * edge-adjacent orientation: ``resolve_ea_rotation``
    (nearfield/nearfield_op.py:44-64), restated;
  * quadrature rules: the reference's own rule arrays, saved by
    tests/golden/make_golden.py (op_rules);
  * pair integrals, farfield and BCOO matvec: liboracle (oracle.cpp).

The composition is RegularizedNearfieldIntegralOp (nearfield/nearfield_op.py:
76-150) plus the direct farfield on all pairs (ops/sparse_integral_op.py:
11-55), restricted to a set of observation rows.
"""
import importlib.machinery
import importlib.util
import os

import numpy as np

from . import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
RULES_PATH = os.path.join(REPO, "tests", "golden", "op_rules.npz")

_mods = {}
_rules = None


def ref_module(name):
    """A reference C++ module compiled by `make -C oracle ref` into oracle/_ref."""
    if name not in _mods:
        for suffix in importlib.machinery.EXTENSION_SUFFIXES:
            path = os.path.join(HERE, "_ref", name + suffix)
            if os.path.exists(path):
                spec = importlib.util.spec_from_file_location(name, path)
                mod = importlib.util.module_from_spec(spec)
                spec.loader.exec_module(mod)
                _mods[name] = mod
                break
        else:
            raise ImportError("oracle/_ref/%s is not built (make -C oracle ref REF=...)" % name)
    return _mods[name]


def available():
    try:
        ref_module("fast_find_nearfield")
    except ImportError:
        return False
    return os.path.exists(RULES_PATH)


# ---- meshes (mesh/mesh_gen.py:7-47) ----------------------------------------
def make_rect(nx, ny, corners):
    """Bilinear patch on an nx x ny vertex grid; cells column-major, two
    triangles [tl, bl, tr], [bl, br, tr] per cell (mesh_gen.py:7-47)."""
    corners = np.asarray(corners, dtype=np.float64)
    X, Y = np.meshgrid(np.linspace(0, 1, nx), np.linspace(0, 1, ny))
    x = X.reshape(-1)
    y = Y.reshape(-1)
    basis = [x * y, (1 - x) * y, (1 - x) * (1 - y), x * (1 - y)]
    pts = np.sum([np.outer(basis[i], corners[i]) for i in range(4)], axis=0)
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="ij")
    i = i.reshape(-1)
    j = j.reshape(-1)
    tl, tr = j * nx + i, j * nx + i + 1
    bl, br = (j + 1) * nx + i, (j + 1) * nx + i + 1
    tris = np.empty((2 * i.shape[0], 3), dtype=np.int64)
    tris[0::2] = np.stack([tl, bl, tr], axis=1)
    tris[1::2] = np.stack([bl, br, tr], axis=1)
    return pts, tris


# ---- quadrature rules (the reference's arrays) -------------------------------
def rule(name, n):
    """(points, weights) of the reference rule `name` in {coincident,
    edge_adj, vertex_adj, gauss4d, gauss2d_tri} of order n."""
    global _rules
    if _rules is None:
        _rules = dict(np.load(RULES_PATH))
    return _rules["%s_%d_p" % (name, n)], _rules["%s_%d_w" % (name, n)]


# ---- near pairs (mesh/find_near_adj.py:13-35) --------------------------------
def tri_centroids_rs(pts, tris):
    """Centroids and circumscribing radii (find_near_adj.py:13-20)."""
    tri_pts = pts[tris]
    c = np.sum(tri_pts, axis=1) / 3.0
    r = np.sqrt(np.max(np.sum((tri_pts - c[:, None, :]) ** 2, axis=2), axis=1))
    return c, r


def near_pairs(pts, tris, threshold):
    """All (obs, src) triangle pairs within the ball threshold, by the
    reference's compiled octree finder (leaf size 50), lexsorted (the raw
    order depends on OpenMP thread completion)."""
    ffn = ref_module("fast_find_nearfield")
    c, r = tri_centroids_rs(pts, tris)
    p = np.asarray(ffn.get_nearfield(c, r, c, r, threshold, 50))
    if p.shape[0] == 0:
        return p.reshape(0, 2)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def edge_adj_orient(a, b):
    """edge_adj_orient of nearfield_op.py:44-50 on arrays of the two touching
    vertex positions: 0 for {0,1}, 2 for {0,2}, 1 for {1,2}."""
    lo = np.minimum(a, b)
    hi = np.maximum(a, b)
    return np.where(lo == 0, np.where(hi == 2, 2, 0), 1)


def resolve_ea_rotation(tris, ea):
    """(obs, src, obs_clicks, src_clicks, src_flip) per edge-adjacent pair
    (nearfield_op.py:52-64)."""
    ea = np.asarray(ea, dtype=np.int64).reshape(-1, 6)
    oc = edge_adj_orient(ea[:, 2], ea[:, 4])
    sc = edge_adj_orient(ea[:, 3], ea[:, 5])
    to, ts = tris[ea[:, 0]], tris[ea[:, 1]]
    k = np.arange(ea.shape[0])
    flip = (to[k, (0 + oc) % 3] != ts[k, (1 + sc) % 3]) | \
           (to[k, (1 + oc) % 3] != ts[k, (0 + sc) % 3])
    return np.stack([ea[:, 0], ea[:, 1], oc, sc, flip.astype(np.int64)], axis=1)


def classify(tris, pairs):
    """The four pair classes of RegularizedNearfieldIntegralOp for a self
    operator (obs_subset = src_subset = all triangles): records and the
    (obs, src) block indices, by the reference's split_adjacent_close."""
    ffn = ref_module("fast_find_nearfield")
    tris = np.asarray(tris)
    close, va, ea = ffn.split_adjacent_close(np.asarray(pairs, dtype=np.int64), tris, tris)
    close = np.asarray(close).reshape(-1, 2)
    va = np.asarray(va).reshape(-1, 4)
    ea = np.asarray(ea).reshape(-1, 6)
    n = tris.shape[0]
    co = np.stack([np.arange(n), np.arange(n)], axis=1)
    va5 = np.hstack([va, np.zeros((va.shape[0], 1), dtype=va.dtype)])
    return {"co": co, "ea": resolve_ea_rotation(tris, ea), "va": va5, "near": close}


def restrict_rows(classes, rows):
    """Keep the records whose observation triangle is in `rows`."""
    keep = np.zeros(max(int(np.max(rows)) + 1, 1), dtype=bool)
    keep[rows] = True
    out = {}
    for c, recs in classes.items():
        m = recs[:, 0] < keep.shape[0]
        m[m] = keep[recs[m, 0]]
        out[c] = recs[m]
    return out


# ---- the sampled operator -----------------------------------------------------
class SampledRows:
    """Rows `rows` (observation triangles) of RegularizedSparseIntegralOp(
    nq_co, nq_ea, nq_va, nq_far, nq_near, thr, K, K, params, pts, tris,
    float_type, TriToTriDirectFarfieldOp) for a self operator: the corrected
    nearfield blocks of those rows are integrated once here (setup);
    `apply(x)` is the farfield of those rows against all sources plus their
    BCOO nearfield rows, the reference operator's apply restricted to them."""

    def __init__(self, pts, tris, rows, nq_co, nq_ea, nq_va, nq_far, nq_near, thr, K, params,
                 float_type, classes=None, n_threads=None, fast=False):
        self.pts = np.asarray(pts, dtype=np.float64)
        self.tris = np.asarray(tris)
        self.rows = np.asarray(rows, dtype=np.int64)
        self.K = K
        self.params = params
        self.float_type = float_type
        self.nq_far = nq_far
        self.n_threads = n_threads
        self.fast = fast
        if classes is None:
            classes = classify(self.tris, near_pairs(self.pts, self.tris, thr))
        cl = restrict_rows(classes, self.rows)
        # row position of each observation triangle in the sample
        pos = np.full(self.tris.shape[0], -1, dtype=np.int64)
        pos[self.rows] = np.arange(self.rows.shape[0])
        far4 = rule("gauss4d", nq_far)
        rules = {"co": (rule("coincident", nq_co), False, True),
                 "ea": (rule("edge_adj", nq_ea), True, True),
                 "va": (rule("vertex_adj", nq_va), True, True),
                 "near": (rule("gauss4d", nq_near), False, False)}
        ft = np.dtype(float_type)
        rr, cc, bb = [], [], []
        for c, (q, adj, check0) in rules.items():
            recs = cl[c]
            if recs.shape[0] == 0:
                continue
            b = orc.pairs(K, float_type, q, self.pts, self.tris, recs[:, :5 if adj else 2],
                          params, adj=adj, check0=check0, n_threads=n_threads).astype(ft)
            corr = orc.pairs(K, float_type, far4, self.pts, self.tris, recs[:, :2], params,
                             adj=False, check0=(c == "co"), n_threads=n_threads).astype(ft)
            rr.append(pos[recs[:, 0]])
            cc.append(recs[:, 1])
            bb.append((b - corr).reshape(-1, 9, 9))
        self.n_blocks = int(sum(r.shape[0] for r in rr))
        self.brows = np.concatenate(rr) if rr else np.zeros(0, np.int64)
        self.bcols = np.concatenate(cc) if cc else np.zeros(0, np.int64)
        self.blocks = (np.concatenate(bb) if bb else np.zeros((0, 9, 9))).astype(np.float64)
        self.far_rule = rule("gauss2d_tri", nq_far)

    def farfield(self, x):
        return orc.farfield_tris(self.K, self.float_type, self.far_rule, self.pts,
                                 self.tris[self.rows], self.tris, x, self.params,
                                 n_threads=self.n_threads, fast=self.fast)

    def nearfield(self, x):
        return orc.bcoo_matvec(self.float_type, self.brows, self.bcols, self.blocks, x,
                               self.rows.shape[0] * 9, n_threads=self.n_threads or 0,
                               fast=self.fast)

    def apply(self, x):
        return self.farfield(x) + self.nearfield(x)
