"""Test infrastructure only: CPU restatement (numpy, FP64) of the reference's
quasidynamic (rate-and-state) stepper, the checker for tectosaur_b200.qd.

Nothing in the product imports this module; tests/ and bench.py's CPU
baseline leg use it as the oracle.

Follows, function by function:
  * rate_state_solver  - qd/newton.cpp:18-131 (newton, F, dFdV, newton_rs,
    solve_for_dof_mag, solve_for_dof_separate_dims, rate_state_solver), in
    the same operation order, so that it agrees bit for bit with the
    reference module compiled by oracle/Makefile (tested);
  * pt_average         - qd/pt_average.cpp:10-35 (sum in DOF order, divide);
  * aging_law / state_evolution - qd/model_helpers.py:122-130;
  * rate_state_solve   - qd/model_helpers.py:79-119;
  * cg                 - the conjugate-gradient solve of
    qd/full_model.py:160-176 (scipy.sparse.linalg.cg, x0 = 0, stop when
    ||r|| < max(atol, rtol ||b||); scipy 1.18.1's algorithm);
  * FullspaceModel     - qd/full_model.py:19-150 (derivs: slip deficit ->
    traction by H and the constrained mass solve -> rate-state velocity ->
    state evolution), with the elastic operator and mass matrix passed in
    (the oracle operator composition and the mass matrix).
The time stepper of the reference is scipy.integrate.RK23 (qd/integrator.py:
44-54), used here as is.
"""
import math

import numpy as np

# Scalar libm functions (math.asinh / exp / sqrt), as the compiled reference
# calls them; numpy's own arcsinh differs from libm's in the last bit for
# some arguments.


def F(V, sigma_n, state, a, V0, C):
    return a * sigma_n * math.asinh(V / (2 * V0) * math.exp(state / a)) - C


def dFdV(V, sigma_n, state, a, V0):
    expsa = math.exp(state / a)
    Q = (V * expsa) / (2 * V0)
    return a * expsa * sigma_n / (2 * V0 * math.sqrt(1 + (Q * Q)))


def newton_rs(tau_qs, eta, sigma_n, state, a, V0, C, V_guess, tol, maxiter):
    """Scalar Newton iteration of newton.cpp:18-31/61-76: (V, converged)."""
    x0 = V_guess
    for _ in range(maxiter):
        y = tau_qs - eta * x0 - F(x0, sigma_n, state, a, V0, C)
        yp = -eta - dFdV(x0, sigma_n, state, a, V0)
        x1 = x0 - y / yp
        if abs(x1 - x0) <= tol * abs(x0):
            return x1, True
        x0 = x1
    return x0, False


def rate_state_solver(tri_normals, traction, state, a, eta, V0, C, normal_stress, tol,
                      maxiter, basis_dim=3, separate_dims=False):
    """Velocity (n_dofs, 3) per DOF (newton.cpp:107-150); also returns the
    number of DOFs whose Newton iteration did not converge."""
    tri_normals = np.asarray(tri_normals, np.float64).reshape(-1, 3).tolist()
    traction = np.asarray(traction, np.float64).reshape(-1, 3).tolist()
    state = np.asarray(state, np.float64).tolist()
    a = np.broadcast_to(np.asarray(a, np.float64), (len(traction),)).tolist()
    normal_stress = np.asarray(normal_stress, np.float64).tolist()
    n_tris = len(tri_normals)
    V = np.zeros((n_tris * basis_dim, 3))
    failed = 0
    eps = 1e-14
    for i in range(n_tris):
        n = tri_normals[i]
        for d in range(basis_dim):
            dof = i * basis_dim + d
            t = traction[dof]

            def rs(shear_mag, normal_mag):
                nonlocal failed
                v, ok = newton_rs(shear_mag, eta, normal_mag + normal_stress[dof], state[dof],
                                  a[dof], V0, C, 0.0, tol, maxiter)
                failed += not ok
                return v

            if separate_dims:
                for k in range(3):
                    V[dof, k] = rs(abs(t[k]), 0.0) * ((t[k] > 0) - (t[k] < 0))
                continue
            nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2]
            f = (t[0] * n[0] + t[1] * n[1] + t[2] * n[2]) / nn
            nvec = [n[0] * f, n[1] * f, n[2] * f]
            shear = [t[0] - nvec[0], t[1] - nvec[1], t[2] - nvec[2]]
            normal_mag = math.sqrt(nvec[0] * nvec[0] + nvec[1] * nvec[1] + nvec[2] * nvec[2])
            shear_mag = math.sqrt(shear[0] * shear[0] + shear[1] * shear[1] + shear[2] * shear[2])
            if shear_mag < eps:
                continue
            vmag = rs(shear_mag, normal_mag)
            inv = 1.0 / shear_mag
            V[dof] = [shear[0] * inv * vmag, shear[1] * inv * vmag, shear[2] * inv * vmag]
    return V, failed


def pt_average(n_pts, tris, field):
    """Average of a per-corner field over the corners sharing a vertex
    (pt_average.cpp:10-35)."""
    tris = np.asarray(tris).reshape(-1)
    field = np.asarray(field, np.float64).reshape(-1)
    vals = np.zeros(n_pts)
    count = np.zeros(n_pts, np.int64)
    for k in range(tris.shape[0]):
        vals[tris[k]] += field[k]
        count[tris[k]] += 1
    with np.errstate(invalid="ignore", divide="ignore"):
        vals = vals / count
    return vals[tris]


def aging_law(b, V0, Dc, f0, V, state):
    return (b * V0 / Dc) * (np.exp((f0 - state) / b) - (V / V0))


def state_evolution(cfg, V, state):
    V_mag = np.linalg.norm(V.reshape(-1, 3), axis=1)
    return aging_law(cfg["b"], cfg["V0"], cfg["Dc"], cfg["f0"], V_mag, state)


def cg(A, b, rtol, atol, maxiter=None):
    """scipy.sparse.linalg.cg (scipy 1.18.1) without a preconditioner, x0 = 0:
    returns (x, n_iterations)."""
    n = b.shape[0]
    maxiter = 10 * n if maxiter is None else maxiter
    bnrm2 = np.linalg.norm(b)
    if bnrm2 == 0.0:
        return b.copy(), 0
    atol = max(float(atol), float(rtol) * float(bnrm2))
    x = np.zeros_like(b)
    r = b.copy()
    rho_prev, p = None, None
    for it in range(maxiter):
        if np.linalg.norm(r) < atol:
            return x, it
        z = r
        rho_cur = np.dot(r, z)
        if it > 0:
            beta = rho_cur / rho_prev
            p *= beta
            p += z
        else:
            p = np.empty_like(r)
            p[:] = z[:]
        q = A @ p
        alpha = rho_cur / np.dot(p, q)
        x += alpha * p
        r -= alpha * q
        rho_prev = rho_cur
    return x, maxiter


def calc_derived_constants(cfg):
    out = dict(cfg)
    out["cs"] = np.sqrt(out["sm"] / out["density"])
    out["eta"] = out["sm"] / (2 * out["cs"])
    return out


class FullspaceModel:
    """derivs(t, y) of qd/full_model.py:19-150 on the host.

    H_dot: v -> H v (the elastic operator; the oracle composition of the
    regularized hypersingular operator), mass: scipy sparse mass matrix,
    cm: continuity + free-edge constraint matrix, cm_edges: free-edge-only
    constraint matrix (setup_edge_bcs)."""

    def __init__(self, pts, tris, cfg, H_dot, mass, cm, cm_edges, normals):
        self.cfg = calc_derived_constants(cfg)
        self.pts, self.tris = pts, np.asarray(tris)
        self.n_tris = self.tris.shape[0]
        self.H_dot, self.cm = H_dot, cm
        self.cmT = cm.T.tocsr()
        self.mass_c = (cm.T @ mass @ cm).tocsr()
        self.tri_normals = normals
        ones_interior = cm_edges.dot(np.ones(cm_edges.shape[1]))
        self.field_inslipdir_interior = ones_interior.copy()
        self.field_inslipdir = ones_interior.copy()
        sd = self.cfg.get("slipdir", (1.0, 0.0, 0.0))
        for d in range(3):
            self.field_inslipdir_interior.reshape(-1, 3)[:, d] *= sd[d]
            self.field_inslipdir.reshape(-1, 3)[:, d] = sd[d]
        self.field_inslipdir_edges = self.field_inslipdir - self.field_inslipdir_interior
        self.ones_interior = ones_interior
        self.cg_iters = []

    def slip_to_traction(self, slip):
        rhs = -self.H_dot(slip)
        soln, it = cg(self.mass_c, self.cmT.dot(rhs), rtol=1e-5, atol=1e-12)
        self.cg_iters.append(it)
        return self.cfg["sm"] * self.cm.dot(soln)

    def rate_state_solve(self, traction, state):
        cfg = self.cfg
        n_dofs = self.n_tris * 3
        normal_stress = np.ones(n_dofs) * cfg["additional_normal_stress"]
        V, failed = rate_state_solver(self.tri_normals, traction, state, cfg["a"], cfg["eta"],
                                      cfg["V0"], cfg.get("C", 0.0), normal_stress, 1e-12, 50, 3,
                                      cfg.get("rs_separate_dims", False))
        self.newton_failed = failed
        ptavg = np.empty_like(V)
        for d in range(3):
            ptavg[:, d] = pt_average(self.pts.shape[0], self.tris, V[:, d])
        interior = self.field_inslipdir_interior.reshape(-1, 3)
        with np.errstate(invalid="ignore", divide="ignore"):
            speed = np.sum(ptavg * interior, axis=1) / np.linalg.norm(interior, axis=1)
        if cfg.get("no_backslip", False):
            ptavg[speed < 0, :] = 0.0
            ptavg[np.isnan(speed)] = 0.0
        return self.field_inslipdir_edges * cfg["plate_rate"] + ptavg.reshape(-1)

    def derivs(self, t, y):
        """full_model.py:27-85: inf * y when y is not finite, the state leaves
        [0, 1.2] or V is not finite."""
        if np.any(~np.isfinite(y)):
            return np.inf * y
        n_slip = y.shape[0] // 4 * 3
        slip, state = y[:n_slip], y[n_slip:]
        if np.any(state < 0) or np.any(state > 1.2):
            return np.inf * y
        plate_motion = (t * self.cfg["plate_rate"]) * self.field_inslipdir
        slip_deficit = self.ones_interior * (plate_motion.reshape(-1) - slip)
        traction = self.slip_to_traction(slip_deficit)
        V = self.rate_state_solve(traction, state)
        if np.any(~np.isfinite(V)):
            return np.inf * y
        dstatedt = state_evolution(self.cfg, V, state)
        return np.concatenate((V, dstatedt))


def sparse_op(nq_co, nq_ea, nq_va, nq_far, nq_near, thr, K, params, pts, tris, float_type):
    """v -> the oracle composition of RegularizedSparseIntegralOp.dot (the
    farfield restatement on all pairs + corrected nearfield blocks, the
    blocks integrated once) for repeated applies by the qd oracle."""
    from oracle import oracle as orc
    from tectosaur_b200.nearfield import triangle_rules as tr
    from tectosaur_b200.nearfield.nearfield_op import nearfield_pairs
    from tectosaur_b200.util.quadrature import gauss2d_tri, gauss4d_tri
    tris = np.asarray(tris)
    idx = np.arange(tris.shape[0])
    classes = nearfield_pairs(pts, tris, idx, idx, thr)
    far_rule = gauss4d_tri(nq_far, nq_far)
    rules = {"co": (tr.coincident_quad(nq_co), False, True),
             "ea": (tr.edge_adj_quad(nq_ea), True, True),
             "va": (tr.vertex_adj_quad(nq_va, nq_va, nq_va), True, True),
             "near": (gauss4d_tri(nq_near, nq_near), False, False)}
    ft = np.dtype(float_type)
    near = []
    for c, (rule, adj, check0) in rules.items():
        recs, dofs = classes[c]
        if dofs.shape[0] == 0:
            continue
        blocks = orc.pairs(K, float_type, rule, pts, tris, recs[:, :5 if adj else 2], params,
                           adj=adj, check0=check0).astype(ft)
        corr = orc.pairs(K, float_type, far_rule, pts, tris, recs[:, :2], params, adj=False,
                         check0=(c == "co")).astype(ft)
        near.append((dofs, (blocks - corr).reshape(-1, 9, 9).astype(np.float64)))
    q2 = gauss2d_tri(nq_far)

    def dot(v):
        y = orc.farfield_tris(K, float_type, q2, pts, tris, tris, v, params)
        for dofs, blocks in near:
            y = y + orc.bcoo_matvec(float_type, dofs[:, 0], dofs[:, 1], blocks, v, y.shape[0])
        return y

    return dot
