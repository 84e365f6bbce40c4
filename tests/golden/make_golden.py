"""Generate the golden fixtures in tests/golden/ from the reference.

Run once on a machine that has the reference checkout (TCT_REFERENCE, else a
directory named "reference" beside this repository) and the reference's C++
modules built by ``make -C oracle ref REF=<checkout>``:

    python tests/golden/make_golden.py

Outputs (all small, committed):
  ref_goldens.npz   the reference's own golden masters for the near-pair
                    finder, the two-triangle farfield and the interior
                    evaluation (copied verbatim from tests/golden_masters/
                    *.npy), plus the sphere mesh test_find_adjacency is
                    computed on.
  quad_rules.npz    reference quadrature rules: small ones in full, larger
                    ones as SHA-256 digests of their FP64 bytes.
  kernel_values.npz pointwise U/T/A/H values of the reference's sympy
                    derivation (kernels/elastic.py, Carini & Salvadori 2002,
                    the expressions tests/test_elastic.py checks its GPU kernels
                    against) at seeded points.  The pickled copy of the same
                    expressions (tests/3d_kernels.pkl) does not load under
                    Python 3.12, so the derivation is evaluated directly.
  near_split.npz    reference find_close_or_touching + split_adjacent_close +
                    resolve_ea_rotation on two meshes (lexsorted).
  mass_op.npz       reference MassOp matrix (dense) on a small mesh.
  qd.npz            the reference's quasidynamic pieces on seeded inputs:
                    qd/newton.cpp rate_state_solver (shear-magnitude and
                    separate-dimension forms, zero-shear DOFs included),
                    qd/pt_average.cpp pt_averageD, and free_edge_constraints
                    + build_constraint_matrix of the qd model's edge
                    conditions (the DOFs it holds at zero).
"""
import hashlib
import os
import sys

import numpy as np

# one OpenMP thread: the reference's near-pair output order is then
# reproducible (with more threads it depends on thread completion order)
os.environ["OMP_NUM_THREADS"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refshim  # noqa: E402  (installs the import shims)

REF = refshim.REF
GM = os.path.join(REF, "tests", "golden_masters")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def ref_goldens():
    import tectosaur.mesh.mesh_gen as mesh_gen
    out = {}
    for name in ["test_close_or_touching", "test_find_nearfield_real",
                 "test_find_adjacency", "test_find_close_notself",
                 "test_farfield_two_tris", "test_interior"]:
        out[name] = np.load(os.path.join(GM, name + ".npy"))
    sphere = mesh_gen.make_sphere([0, 0, 0], 1.0, 3)
    out["sphere_pts"] = sphere[0]
    out["sphere_tris"] = sphere[1]
    np.savez_compressed(os.path.join(HERE, "ref_goldens.npz"), **out)


def quad_rules():
    import tectosaur.util.quadrature as rq
    import tectosaur.nearfield.triangle_rules as rtr
    out = {}
    for n in range(1, 21):
        x, w = rq.gaussxw(n)
        out["gaussxw_%d_x" % n] = x
        out["gaussxw_%d_w" % n] = w
    for n in range(1, 12):
        p, w = rq.gauss2d_tri(n)
        out["gauss2d_tri_%d_p" % n] = p
        out["gauss2d_tri_%d_w" % n] = w
    for n in [2, 3]:
        for name, f in [("coincident", rtr.coincident_quad), ("edge_adj", rtr.edge_adj_quad),
                        ("vertex_adj", lambda k: rtr.vertex_adj_quad(k, k, k))]:
            p, w = f(n)
            out["%s_%d_p" % (name, n)] = p
            out["%s_%d_w" % (name, n)] = w
    digests = []
    for n in [4, 5, 6, 8, 10, 12]:
        for name, f in [("coincident", rtr.coincident_quad), ("edge_adj", rtr.edge_adj_quad),
                        ("vertex_adj", lambda k: rtr.vertex_adj_quad(k, k, k))]:
            p, w = f(n)
            digests.append("%s %d %d %s %s" % (name, n, p.shape[0], sha(p), sha(w)))
    for a, b in [(2, 2), (3, 3), (5, 5), (2, 5)]:
        p, w = rq.gauss4d_tri(a, b)
        digests.append("gauss4d_tri %d,%d %d %s %s" % (a, b, p.shape[0], sha(p), sha(w)))
    out["digests"] = np.array(digests)
    np.savez_compressed(os.path.join(HERE, "quad_rules.npz"), **out)


def op_rules():
    """The reference's own rules for the operator configurations the CPU
    baseline and the sampled-row parity check run without the product package
    (oracle/ref_pipeline.py): (nq_co, nq_ea, nq_va, nq_far, nq_near) =
    (6, 6, 6, 2, 5) for the 722-triangle fault, (6, 6, 6, 1, 5) for the 60k
    surface, (3, 3, 3, 2, 3) for small test operators."""
    import tectosaur.util.quadrature as rq
    import tectosaur.nearfield.triangle_rules as rtr
    out = {}
    for n in (3, 6):
        for name, f in [("coincident", rtr.coincident_quad), ("edge_adj", rtr.edge_adj_quad),
                        ("vertex_adj", lambda k: rtr.vertex_adj_quad(k, k, k))]:
            p, w = f(n)
            out["%s_%d_p" % (name, n)] = p
            out["%s_%d_w" % (name, n)] = w
    for n in (1, 2, 3, 5):
        p, w = rq.gauss4d_tri(n, n)
        out["gauss4d_%d_p" % n] = p
        out["gauss4d_%d_w" % n] = w
        p, w = rq.gauss2d_tri(n)
        out["gauss2d_tri_%d_p" % n] = p
        out["gauss2d_tri_%d_w" % n] = w
    np.savez_compressed(os.path.join(HERE, "op_rules.npz"), **out)


def kernel_values():
    import sympy
    from tectosaur.kernels.elastic import U, T, A, H, all_args
    builders = [U, T, A, H]
    rng = np.random.default_rng(1234)
    params = []
    vals = []
    for k in range(4):
        for i in range(3):
            for j in range(3):
                f = sympy.lambdify(all_args, builders[k](i, j)["expr"], "mpmath")
                for t in range(6):
                    # argument order (test_elastic.py:38-50): G, nu, b0, b1,
                    # src pt, obs pt, src normal, obs normal
                    p = rng.random(16)
                    p[-3:] /= np.linalg.norm(p[-3:])
                    p[-6:-3] /= np.linalg.norm(p[-6:-3])
                    params.append(np.concatenate([[k, i, j], p]))
                    vals.append(float(f(*[sympy.Float(v, 30) for v in p])))
    np.savez_compressed(os.path.join(HERE, "kernel_values.npz"),
                        cases=np.array(params), values=np.array(vals))


def near_split():
    import tectosaur.mesh.mesh_gen as mesh_gen
    from tectosaur.mesh.find_near_adj import find_close_or_touching, split_adjacent_close
    from tectosaur.nearfield.nearfield_op import resolve_ea_rotation
    out = {}
    rng = np.random.default_rng(7)
    meshes = {
        "rect": mesh_gen.make_rect(12, 12, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]]),
        "sphere": mesh_gen.make_sphere([0, 0, 0], 1.0, 2),
    }
    pts, tris = mesh_gen.make_rect(9, 7, [[-1, 0, 1], [-1, 0, -1], [1, 0, -1], [1, 0, 1]])
    pts = pts + 0.01 * rng.standard_normal(pts.shape)
    meshes["bumpy"] = (pts, tris)
    for name, (pts, tris) in meshes.items():
        for thr in [1.25, 2.5]:
            key = "%s_%s" % (name, str(thr).replace(".", "p"))
            pairs = find_close_or_touching(pts, tris, pts, tris, thr)
            close, va, ea = split_adjacent_close(pairs, tris, tris)
            ea_rot = resolve_ea_rotation(tris, ea)
            out[key + "_pts"] = pts
            out[key + "_tris"] = tris
            out[key + "_pairs_raw"] = pairs
            out[key + "_close"] = close
            out[key + "_va"] = va
            out[key + "_ea"] = ea
            out[key + "_ea_rot"] = ea_rot.astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "near_split.npz"), **out)


def mass_op():
    import tectosaur.mesh.mesh_gen as mesh_gen
    from tectosaur.ops.mass_op import MassOp
    m = mesh_gen.make_rect(4, 3, [[0, 0, 0], [1, 0, 0], [1, 1, 0.3], [0, 1, 0]])
    out = {"pts": m[0], "tris": m[1]}
    for nq in [2, 3]:
        for td in [1, 3]:
            out["mat_%d_%d" % (nq, td)] = MassOp(nq, m[0], m[1], tensor_dim=td).mat.toarray()
    np.savez_compressed(os.path.join(HERE, "mass_op.npz"), **out)


def qd_inputs(seed=12, n_tris=40):
    """Seeded rate-state inputs in the units of the reference's qd runs
    (Pa, m/s; sm 3e10, density 2670 -> eta = sm / (2 cs))."""
    rng = np.random.default_rng(seed)
    n = rng.standard_normal((n_tris, 3))
    n /= np.linalg.norm(n, axis=1)[:, None]
    traction = rng.standard_normal((n_tris * 3, 3)) * rng.uniform(1e5, 3e7, (n_tris * 3, 1))
    traction[::7] = 0.0  # zero shear: the solver returns zero velocity
    state = rng.uniform(0.5, 0.85, n_tris * 3)
    a = rng.uniform(0.008, 0.012, n_tris * 3)
    sm, density = 3e10, 2670.0
    eta = sm / (2 * np.sqrt(sm / density))
    normal_stress = np.full(n_tris * 3, 50e6)
    return dict(tri_normals=n, traction=traction, state=state, a=a, eta=eta, V0=1e-6, C=0.0,
                normal_stress=normal_stress)


def qd():
    import tectosaur.mesh.mesh_gen as mesh_gen
    from tectosaur.constraint_builders import free_edge_constraints
    from tectosaur.constraints import build_constraint_matrix
    newton = refshim._load_ext("newton")
    pt_average = refshim._load_ext("pt_average")
    inp = qd_inputs()
    out = {"in_" + k: np.asarray(v) for k, v in inp.items()}
    for sep in (False, True):
        V = np.zeros_like(inp["traction"])
        newton.rate_state_solver(inp["tri_normals"], inp["traction"], inp["state"], V, inp["a"],
                                 inp["eta"], inp["V0"], inp["C"], inp["normal_stress"], 1e-12,
                                 50, 3, sep)
        out["V_sep%d" % int(sep)] = V
    m = mesh_gen.make_rect(5, 4, [[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]])
    field = np.random.default_rng(13).standard_normal(m[1].size)
    out["avg_pts"], out["avg_tris"], out["avg_field"] = m[0], m[1], field
    out["avg_out"] = pt_average.pt_averageD(m[0], m[1].astype(np.int64), field)
    cs = free_edge_constraints(m[1])
    cm, _, _ = build_constraint_matrix(cs, m[1].shape[0] * 9)
    out["edge_ones_interior"] = cm.dot(np.ones(cm.shape[1]))
    np.savez_compressed(os.path.join(HERE, "qd.npz"), **out)


if __name__ == "__main__":
    # no arguments: every fixture; otherwise only the named generators
    gens = [qd, ref_goldens, quad_rules, op_rules, kernel_values, near_split, mass_op]
    names = sys.argv[1:]
    for g in gens:
        if not names or g.__name__ in names:
            g()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
