"""Shared test inputs and oracle compositions (test infrastructure)."""
import numpy as np

from tectosaur_b200.mesh.mesh_gen import make_rect, concat_no_dedupe

ALL_KERNELS = ["elasticU3", "elasticT3", "elasticA3", "elasticH3",
               "elasticRT3", "elasticRA3", "elasticRH3"]
PARAMS = [1.0, 0.25]


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def c1_mesh():
    """Config 1: 2x2 planar fault from a 20x20 vertex grid (722 tris, 6498 DOF)."""
    return make_rect(20, 20, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]])


def c2_mesh(n=174, seed=2):
    """The 60k-triangle direct-farfield surface: an n x n vertex grid over
    [-10, 10]^2 with z = 0.5 exp(-(x^2 + y^2)/8) + 0.02 N(0, 1) (seed 2);
    59,858 triangles at n = 174."""
    pts, tris = make_rect(n, n, [[-10, -10, 0], [10, -10, 0], [10, 10, 0], [-10, 10, 0]])
    rng = np.random.default_rng(seed)
    pts = pts.copy()
    pts[:, 2] = 0.5 * np.exp(-(pts[:, 0] ** 2 + pts[:, 1] ** 2) / 8.0) + \
        0.02 * rng.standard_normal(pts.shape[0])
    return pts, tris


def bumpy_mesh(n, seed=0, amp=0.05, size=1.0):
    pts, tris = make_rect(n, n, [[-size, -size, 0], [size, -size, 0], [size, size, 0],
                                 [-size, size, 0]])
    rng = np.random.default_rng(seed)
    pts = pts.copy()
    pts[:, 2] = 0.3 * np.exp(-(pts[:, 0] ** 2 + pts[:, 1] ** 2)) + amp * rng.standard_normal(
        pts.shape[0]) * (size / n)
    return pts, tris


def two_surfaces(n=8, sep=2.0, w=1.0):
    """The reference's make_meshes (tests/test_farfield.py:9-24) without the
    duplicate-vertex merge (the surfaces do not touch)."""
    m1 = make_rect(n, n, [[-w, 0, w], [-w, 0, -w], [w, 0, -w], [w, 0, w]])
    m2 = make_rect(n, n, [[-w, sep, w], [-w, sep, -w], [w, sep, -w], [w, sep, w]])
    m = concat_no_dedupe(m1, m2)
    s1 = np.arange(m1[1].shape[0])
    s2 = s1[-1] + 1 + s1
    return m, s1, s2


def oracle_sparse_op_dot(orc, nq_co, nq_ea, nq_va, nq_far, nq_near, thr, Kn, Kf, params, pts,
                         tris, float_type, v, obs_subset=None, src_subset=None,
                         correction=True, n_threads=None):
    """CPU composition of RegularizedSparseIntegralOp.dot from oracle pieces:
    farfield (matrix_free.cl restatement) on all pairs + per-class BCOO blocks
    (assemble.cl restatement) minus far-rule corrections."""
    from tectosaur_b200.nearfield import triangle_rules as tr
    from tectosaur_b200.nearfield.nearfield_op import nearfield_pairs
    from tectosaur_b200.util.quadrature import gauss2d_tri, gauss4d_tri
    tris = np.asarray(tris)
    if obs_subset is None:
        obs_subset = np.arange(tris.shape[0])
    if src_subset is None:
        src_subset = np.arange(tris.shape[0])
    classes = nearfield_pairs(pts, tris, obs_subset, src_subset, thr)
    far_rule = gauss4d_tri(nq_far, nq_far)
    rules = {"co": (tr.coincident_quad(nq_co), False, True),
             "ea": (tr.edge_adj_quad(nq_ea), True, True),
             "va": (tr.vertex_adj_quad(nq_va, nq_va, nq_va), True, True),
             "near": (gauss4d_tri(nq_near, nq_near), False, False)}
    y = orc.farfield_tris(Kf, float_type, gauss2d_tri(nq_far), pts, tris[obs_subset],
                          tris[src_subset], v, params, n_threads=n_threads)
    ft = np.dtype(float_type)
    for c, (rule, adj, check0) in rules.items():
        recs, dofs = classes[c]
        if dofs.shape[0] == 0:
            continue
        blocks = orc.pairs(Kn, float_type, rule, pts, tris, recs[:, :5 if adj else 2], params,
                           adj=adj, check0=check0, n_threads=n_threads).astype(ft)
        if correction:
            corr = orc.pairs(Kf, float_type, far_rule, pts, tris, recs[:, :2], params, adj=False,
                             check0=(c == "co"), n_threads=n_threads).astype(ft)
            blocks = blocks - corr
        y = y + orc.bcoo_matvec(float_type, dofs[:, 0], dofs[:, 1],
                                blocks.reshape(-1, 9, 9).astype(np.float64), v, y.shape[0])
    return y


def oracle_sparse_op(orc, nq_co, nq_ea, nq_va, nq_far, nq_near, thr, K, params, pts, tris,
                     float_type):
    """v -> the oracle composition of RegularizedSparseIntegralOp.dot with the
    corrected nearfield blocks integrated once (for repeated applies)."""
    from oracle import qd_oracle
    return qd_oracle.sparse_op(nq_co, nq_ea, nq_va, nq_far, nq_near, thr, K, params, pts, tris,
                               float_type)
