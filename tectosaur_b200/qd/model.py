"""Quasidynamic full-space fault model with its state on the device
(reference: tectosaur/qd/full_model.py:19-197 and qd/model_helpers.py).

derivs(t, y), y = (slip (9 n_tris), state (3 n_tris)), runs as in the
reference, every step on the GPU and without host synchronisation:
  slip deficit = ones_interior (t plate_rate slipdir - slip)
  traction     = sm cm (cm^T M cm)^-1 cm^T (-H slip_deficit)
                 H: RegularizedSparseIntegralOp elasticRH3 (its dot_device),
                 the mass solve: conjugate gradients in one CTA (tct_cg_csr,
                 rtol 1e-5, atol 1e-12 as the reference's scipy cg call)
  V            = rate-state Newton solve per DOF (tct_qd_rate_state), vertex
                 average, plate rate on the free edges (tct_qd_velocity_state)
  dstate/dt    = aging law (same kernel)
A y with non-finite entries or a state outside [0, 1.2], or a non-finite V,
gives inf * y (the reference's signal to its time stepper to shrink the
step); it is selected on the device.  Newton solves that stop at maxiter
are counted on the device (newton_failures()).
"""
import ctypes

import numpy as np

from .. import _lib
from ..ops.mass_op import MassOp, unscaled_normals
from ..simple_solver import DeviceCSR, free_edge_vertices, shared_vertex_matrix
from ..util import device


def calc_derived_constants(cfg):
    """model_helpers.py:60-73: shear wave speed and radiation damping."""
    out = dict(cfg)
    out["cs"] = np.sqrt(out["sm"] / out["density"])
    out["eta"] = out["sm"] / (2 * out["cs"])
    return out


def aging_law(cfg, V, state):
    """model_helpers.py:122-125 (host form)."""
    return (cfg["b"] * cfg["V0"] / cfg["Dc"]) * (
        np.exp((cfg["f0"] - state) / cfg["b"]) - (V / cfg["V0"]))


def build_elastic_op(pts, tris, cfg, K="H", float_type=None):
    """model_helpers.py:23-42: the regularized elastic operator of the qd
    model (direct or FMM farfield per tectosaur_cfg)."""
    from ..ops.sparse_farfield_op import FMMFarfieldOp, TriToTriDirectFarfieldOp
    from ..ops.sparse_integral_op import RegularizedSparseIntegralOp
    op_cfg = cfg["tectosaur_cfg"]
    name = "elastic" + K + "3" if K == "U" else "elasticR" + K + "3"
    if op_cfg.get("use_fmm", False):
        far = FMMFarfieldOp(op_cfg["fmm_mac"], op_cfg["pts_per_cell"], op_cfg["fmm_order"])
    else:
        far = TriToTriDirectFarfieldOp
    return RegularizedSparseIntegralOp(
        op_cfg["quad_coincident_order"], op_cfg["quad_edgeadj_order"],
        op_cfg["quad_vertadj_order"], op_cfg["quad_far_order"], op_cfg["quad_near_order"],
        op_cfg["quad_near_threshold"], name, name, [1.0, cfg["pr"]], pts, tris,
        float_type or op_cfg["float_type"], far)


def edge_ones_interior(tris):
    """1 at every slip DOF (9 per triangle) not held by the free-edge
    constraints, 0 at those held: cm.dot(ones) for the constraint matrix of
    free_edge_constraints (full_model.py:119-124, constraint_builders.py:
    74-135), i.e. the DOFs of triangle corners at free-edge vertices."""
    tris = np.asarray(tris)
    interior_dof = ~np.isin(tris.reshape(-1), free_edge_vertices(tris))
    return np.repeat(interior_dof.astype(np.float64), 3)


def _per_dof(v, n):
    return np.ascontiguousarray(np.broadcast_to(np.asarray(v, np.float64), (n,)))


class FullspaceModel:
    """FullspaceModel(m, cfg) of qd/full_model.py:19-150 for a fault-only
    mesh m = (pts, tris).  H: an already built elastic operator (default:
    build_elastic_op from cfg['tectosaur_cfg'])."""

    def __init__(self, m, cfg, H=None):
        t = device.require_cuda()
        self.cfg = calc_derived_constants(cfg)
        pts, tris = np.asarray(m[0], np.float64), np.asarray(m[1], np.int64)
        self.m = (pts, tris)
        # setup_mesh (full_model.py:105-117)
        self.unscaled_tri_normals = unscaled_normals(pts[tris])
        self.tri_size = np.linalg.norm(self.unscaled_tri_normals, axis=1)
        self.tri_normals = self.unscaled_tri_normals / self.tri_size[:, None]
        self.n_tris = tris.shape[0]
        self.basis_dim = 3
        self.n_dofs = self.basis_dim * self.n_tris
        # setup_edge_bcs (full_model.py:119-135): DOFs at free-edge vertices
        fixed = free_edge_vertices(tris)
        self.ones_interior = edge_ones_interior(tris)
        sd = self.cfg.get("slipdir", (1.0, 0.0, 0.0))
        self.field_inslipdir_interior = self.ones_interior.copy()
        self.field_inslipdir = self.ones_interior.copy()
        for d in range(3):
            self.field_inslipdir_interior.reshape(-1, 3)[:, d] *= sd[d]
            self.field_inslipdir.reshape(-1, 3)[:, d] = sd[d]
        self.field_inslipdir_edges = self.field_inslipdir - self.field_inslipdir_interior
        # slip -> traction (full_model.py:152-176): continuity + free edges
        self.H = H if H is not None else build_elastic_op(pts, tris, self.cfg)
        self.H_dtype = device.torch_dtype(getattr(self.H, "float_type", np.float64))
        self.mass = MassOp(self.cfg["tectosaur_cfg"]["quad_mass_order"], pts, tris)
        self.cm_host = shared_vertex_matrix(tris, fixed_vertices=fixed)
        self.cm, self.cmT = DeviceCSR(self.cm_host), DeviceCSR(self.cm_host.T)
        mc = (self.cm_host.T @ self.mass.mat @ self.cm_host).tocsr()
        mc.sort_indices()
        self.n_free = mc.shape[0]
        self.mass_c = (device.to_dev(mc.indptr.astype(np.int64)),
                       device.to_dev(mc.indices.astype(np.int64)),
                       device.to_dev(mc.data.astype(np.float64)))
        # vertex averaging: the DOFs at each vertex in increasing order
        dof_vert = tris.reshape(-1)
        order = np.argsort(dof_vert, kind="stable")
        counts = np.bincount(dof_vert, minlength=pts.shape[0])
        self.vert_start = device.to_dev(np.concatenate([[0], np.cumsum(counts)]), np.int32)
        self.vert_dofs = device.to_dev(order, np.int32)
        self.dof_vert = device.to_dev(dof_vert, np.int32)
        # device copies of the per-DOF fields and parameters
        f64 = t.float64
        self.d_normals = device.to_dev(self.tri_normals)
        self.d_interior = device.to_dev(self.ones_interior)
        self.d_inslipdir = device.to_dev(self.field_inslipdir)
        self.d_edges = device.to_dev(self.field_inslipdir_edges)
        self.d_int_dir = device.to_dev(self.field_inslipdir_interior)
        self.d_a = device.to_dev(_per_dof(self.cfg["a"], self.n_dofs))
        self.d_b = device.to_dev(_per_dof(self.cfg["b"], self.n_dofs))
        self.d_sigma = device.to_dev(np.full(self.n_dofs, float(self.cfg["additional_normal_stress"])))
        n9 = 9 * self.n_tris
        self._x = t.zeros(n9, dtype=self.H_dtype, device="cuda")
        self._y = t.zeros(n9, dtype=self.H_dtype, device="cuda")
        self._rhs_c = t.zeros(self.n_free, dtype=f64, device="cuda")
        self._soln = t.zeros(self.n_free, dtype=f64, device="cuda")
        self._cg_work = t.zeros(3 * max(self.n_free, 1), dtype=f64, device="cuda")
        self._cg_iters = t.zeros(1, dtype=t.int32, device="cuda")
        self._vn = t.zeros(n9, dtype=f64, device="cuda")
        self.n_failed = t.zeros(1, dtype=t.int32, device="cuda")
        self.n_evals = 0
        self.graph_kernel_launches = 0  # library kernels run by derivative graph replays

    # -- pieces ---------------------------------------------------------------
    def slip_to_traction(self, slip):
        """sm cm (cm^T M cm)^-1 cm^T (-H slip) on device FP64 vectors."""
        t = device.torch()
        self._x.copy_(slip)
        self.H.dot_device(self._x, self._y)
        rhs = -self._y.to(t.float64)
        self.cmT.dot_device(rhs, self._rhs_c)
        ip, ix, dv = self.mass_c
        _lib.check(_lib.lib.tct_cg_csr(
            self.n_free, _lib.tptr(ip), _lib.tptr(ix), _lib.tptr(dv), _lib.tptr(self._rhs_c),
            _lib.tptr(self._soln), _lib.tptr(self._cg_work), 1e-5, 1e-12, 10 * self.n_free,
            _lib.tptr(self._cg_iters), _lib.stream_ptr()), "tct_cg_csr")
        out = t.empty(9 * self.n_tris, dtype=t.float64, device="cuda")
        self.cm.dot_device(self._soln, out)
        out *= self.cfg["sm"]
        if self.cfg.get("only_x", False):
            out.view(-1, 3)[:, 1:] = 0.0
        return out

    def rate_state_solve(self, traction, state):
        """(V, dstate/dt): model_helpers.py:79-119 and the aging law."""
        t = device.torch()
        cfg = self.cfg
        _lib.check(_lib.lib.tct_qd_rate_state(
            self.n_tris, 3, _lib.tptr(self.d_normals), _lib.tptr(traction), _lib.tptr(state),
            _lib.tptr(self.d_a), float(cfg["eta"]), float(cfg["V0"]), float(cfg.get("C", 0.0)),
            _lib.tptr(self.d_sigma), 1e-12, 50, int(bool(cfg.get("rs_separate_dims", False))),
            _lib.tptr(self._vn), _lib.tptr(self.n_failed), _lib.stream_ptr()),
            "tct_qd_rate_state")
        V = t.empty(9 * self.n_tris, dtype=t.float64, device="cuda")
        dstate = t.empty(self.n_dofs, dtype=t.float64, device="cuda")
        _lib.check(_lib.lib.tct_qd_velocity_state(
            self.n_dofs, _lib.tptr(self.vert_start), _lib.tptr(self.vert_dofs),
            _lib.tptr(self.dof_vert), _lib.tptr(self._vn), _lib.tptr(self.d_edges),
            _lib.tptr(self.d_int_dir), float(cfg["plate_rate"]),
            int(bool(cfg.get("no_backslip", False))), _lib.tptr(state), _lib.tptr(self.d_b),
            float(cfg["V0"]), float(cfg["Dc"]), float(cfg["f0"]), _lib.tptr(V), _lib.tptr(dstate),
            _lib.stream_ptr()), "tct_qd_velocity_state")
        return V, dstate

    def solve_for_full_state(self, t_, y):
        """full_model.py:42-85 on device tensors: (slip, slip_deficit,
        state, traction, V, dstatedt, bad) with bad a device bool."""
        t = device.torch()
        n_slip = y.shape[0] // 4 * 3
        slip, state = y[:n_slip], y[n_slip:].contiguous()
        plate_motion = (t_ * self.cfg["plate_rate"]) * self.d_inslipdir
        slip_deficit = self.d_interior * (plate_motion - slip)
        traction = self.slip_to_traction(slip_deficit)
        V, dstate = self.rate_state_solve(traction, state)
        bad = (~t.isfinite(y).all()) | (state < 0).any() | (state > 1.2).any() | \
            (~t.isfinite(V).all())
        return slip, slip_deficit, state, traction, V, dstate, bad

    def make_derivs(self, graph=True):
        """The derivative function (t, y) -> dy/dt of one state (full_model.py
        make_derivs).  With graph (the default) the evaluation -- the
        operator apply, the constrained mass solve, Newton, averaging and
        the rejection, ~30 launches -- is captured once as a CUDA graph on
        private buffers and replayed: the time and state are copied in, the
        derivative is copied out.  The graph holds the same kernels with the
        same arguments, so its values are the eager evaluation's bit for
        bit (the time enters as a device scalar: t * plate_rate is the same
        one rounding); the eager form is used where capture fails."""
        t = device.torch()

        def eager(t_, y):
            *_, V, dstate, bad = self.solve_for_full_state(t_, y)
            out = t.cat((V, dstate))
            return t.where(bad, y * float("inf"), out)

        st = {}

        def capture(t_, y):
            ts = t.zeros((), dtype=t.float64, device="cuda")
            yin = t.empty_like(y)
            ts.fill_(float(t_))
            yin.copy_(y)
            side = t.cuda.Stream()
            side.wait_stream(t.cuda.current_stream())
            with t.cuda.stream(side):
                eager(ts, yin)  # warm-up outside the capture
            t.cuda.current_stream().wait_stream(side)
            g = t.cuda.CUDAGraph()
            n0 = _lib.launch_count()
            with t.cuda.graph(g):
                out = eager(ts, yin)
            # library kernels recorded in the graph: a replay runs them
            # without passing the launch counter
            st.update(g=g, ts=ts, yin=yin, out=out, kernels=_lib.launch_count() - n0)

        def derivs(t_, y):
            self.n_evals += 1
            if not graph or st.get("off"):
                return eager(t_, y)
            if "g" not in st:
                try:
                    capture(t_, y)
                except RuntimeError:
                    st.clear()
                    st["off"] = True
                    return eager(t_, y)
            st["ts"].fill_(float(t_))
            st["yin"].copy_(y)
            st["g"].replay()
            self.graph_kernel_launches += st["kernels"]
            return st["out"].clone()

        return derivs

    # -- several states at once (the served form) ----------------------------------
    def _panel(self, X, Y):
        """Y = H X for (R, 9 n) panels of H's float type."""
        if hasattr(self.H, "dot_panel_device"):
            return self.H.dot_panel_device(X, Y)
        for r in range(X.shape[0]):
            self.H.dot_device(X[r], Y[r])
        return Y

    def _csr_panel(self, mat, X, Y):
        _lib.check(_lib.lib.tct_csr_matvec_panel(
            _lib.TCT_F64, mat.shape[0], _lib.tptr(mat.indptr), _lib.tptr(mat.indices),
            _lib.tptr(mat.data), _lib.tptr(X), X.stride(0), _lib.tptr(Y), Y.stride(0),
            X.shape[0], 0, _lib.stream_ptr()), "tct_csr_matvec_panel")
        return Y

    def slip_to_traction_batch(self, D):
        """slip_to_traction for the rows of D (R, 9 n): one panel apply of H,
        one CG launch with a CTA per row.  The constrained mass solve runs on
        H D instead of -H D and the sign goes into the final scale: every
        step of the CSR products and of CG commutes exactly with negation,
        so the result is bit-identical and two element-wise passes fewer."""
        t = device.torch()
        R = D.shape[0]
        X = D.to(self.H_dtype).contiguous()
        Yh = t.empty_like(X)
        self._panel(X, Yh)
        rhs = Yh if Yh.dtype == t.float64 else Yh.to(t.float64)
        rc = t.empty((R, self.n_free), dtype=t.float64, device="cuda")
        self._csr_panel(self.cmT, rhs, rc)
        soln = t.empty_like(rc)
        work = t.empty(3 * max(self.n_free, 1) * R, dtype=t.float64, device="cuda")
        iters = t.empty(R, dtype=t.int32, device="cuda")
        ip, ix, dv = self.mass_c
        _lib.check(_lib.lib.tct_cg_csr_batch(
            self.n_free, R, _lib.tptr(ip), _lib.tptr(ix), _lib.tptr(dv), _lib.tptr(rc),
            rc.stride(0), _lib.tptr(soln), soln.stride(0), _lib.tptr(work), 1e-5, 1e-12,
            10 * self.n_free, _lib.tptr(iters), _lib.stream_ptr()), "tct_cg_csr_batch")
        out = t.empty((R, 9 * self.n_tris), dtype=t.float64, device="cuda")
        self._csr_panel(self.cm, soln, out)
        out *= -self.cfg["sm"]
        if self.cfg.get("only_x", False):
            out.view(R, -1, 3)[:, :, 1:] = 0.0
        return out

    def rate_state_solve_batch(self, traction, state):
        """(V, dstate/dt) for the rows of traction (R, 9 n) and state
        (R, 3 n; any row stride)."""
        t = device.torch()
        cfg = self.cfg
        R = traction.shape[0]
        n9 = 9 * self.n_tris
        vn = t.empty((R, n9), dtype=t.float64, device="cuda")
        _lib.check(_lib.lib.tct_qd_rate_state_batch(
            self.n_tris, 3, R, _lib.tptr(self.d_normals), _lib.tptr(traction),
            traction.stride(0), _lib.tptr(state), state.stride(0), _lib.tptr(self.d_a),
            float(cfg["eta"]), float(cfg["V0"]), float(cfg.get("C", 0.0)),
            _lib.tptr(self.d_sigma), 1e-12, 50, int(bool(cfg.get("rs_separate_dims", False))),
            _lib.tptr(vn), vn.stride(0), _lib.tptr(self.n_failed), _lib.stream_ptr()),
            "tct_qd_rate_state_batch")
        V = t.empty((R, n9), dtype=t.float64, device="cuda")
        dstate = t.empty((R, self.n_dofs), dtype=t.float64, device="cuda")
        _lib.check(_lib.lib.tct_qd_velocity_state_batch(
            self.n_dofs, R, _lib.tptr(self.vert_start), _lib.tptr(self.vert_dofs),
            _lib.tptr(self.dof_vert), _lib.tptr(vn), vn.stride(0), _lib.tptr(self.d_edges),
            _lib.tptr(self.d_int_dir), float(cfg["plate_rate"]),
            int(bool(cfg.get("no_backslip", False))), _lib.tptr(state), state.stride(0),
            _lib.tptr(self.d_b), float(cfg["V0"]), float(cfg["Dc"]), float(cfg["f0"]),
            _lib.tptr(V), V.stride(0), _lib.tptr(dstate), dstate.stride(0), _lib.stream_ptr()),
            "tct_qd_velocity_state_batch")
        return V, dstate

    def derivs_batch(self, ts, Y):
        """derivs for R states at once: ts (R,) device float64, Y (R, n_y).
        The slip deficit (cast to H's precision) and the derivative's
        assembly with the rejection of non-finite or out-of-range states
        are one fused launch each (tct_qd_deficit_batch,
        tct_qd_finish_batch), bit-identical to the element-wise forms
        plate = (ts rate) dir, deficit = interior (plate - slip);
        where(bad, Y inf, (V, dstate))."""
        t = device.torch()
        R = Y.shape[0]
        self.n_evals += R
        n9 = 9 * self.n_tris
        if Y.stride(1) != 1:
            Y = Y.contiguous()
        ts = ts.contiguous()
        state = Y[:, n9:]
        D = t.empty((R, n9), dtype=self.H_dtype, device="cuda")
        _lib.check(_lib.lib.tct_qd_deficit_batch(
            n9, R, _lib.tptr(ts), float(self.cfg["plate_rate"]), _lib.tptr(self.d_inslipdir),
            _lib.tptr(self.d_interior), _lib.tptr(Y), Y.stride(0),
            _lib.prec_of(np.float32 if self.H_dtype == t.float32 else np.float64),
            _lib.tptr(D), D.stride(0), _lib.stream_ptr()), "tct_qd_deficit_batch")
        traction = self.slip_to_traction_batch(D)
        V, dstate = self.rate_state_solve_batch(traction, state)
        out = t.empty((R, Y.shape[1]), dtype=t.float64, device="cuda")
        _lib.check(_lib.lib.tct_qd_finish_batch(
            n9, Y.shape[1] - n9, R, _lib.tptr(Y), Y.stride(0), _lib.tptr(V), V.stride(0),
            _lib.tptr(dstate), dstate.stride(0), 1.2, _lib.tptr(out), out.stride(0),
            _lib.stream_ptr()), "tct_qd_finish_batch")
        return out

    def newton_failures(self, reset=True):
        """DOFs whose Newton iteration stopped at maxiter since the last call
        (a host sync).  The reference's assert on them is compiled out
        (extension builds define NDEBUG), so such a DOF keeps its last
        iterate there too; an attempted step that meets them is normally
        rejected by the error control."""
        n = int(self.n_failed.item())
        if reset and n:
            self.n_failed.zero_()
        return n

    @property
    def last_cg_iterations(self):
        return int(self._cg_iters.item())


def _terms(Ks, coeffs):
    n = len(Ks)
    for k in Ks:
        if k.dtype != device.torch().float64 or k.stride(1) != 1:
            raise ValueError("RK terms: float64 rows with unit stride")
    return (n, (ctypes.c_void_p * n)(*[k.data_ptr() for k in Ks]),
            (ctypes.c_int64 * n)(*[k.stride(0) for k in Ks]),
            (ctypes.c_double * n)(*[float(c) for c in coeffs]))


def combine_batch(Ks, coeffs, h, y, out):
    """out = y + (((K0 c0 + K1 c1) + K2 c2) + K3 c3) * h[:, None] for 1-4
    (R, n) float64 terms (y None: no y term), rounded as that element-wise
    expression; one launch (tct_qd_combine_batch)."""
    n, kp, ks, cs = _terms(Ks, coeffs)
    R, m = out.shape
    _lib.check(_lib.lib.tct_qd_combine_batch(
        m, R, n, kp, ks, cs, _lib.tptr(h.contiguous()), _lib.tptr(y) if y is not None else None,
        y.stride(0) if y is not None else 0, _lib.tptr(out), out.stride(0), _lib.stream_ptr()),
        "tct_qd_combine_batch")
    return out


def error_norm_batch(Ks, coeffs, h, y, y_new, tol, out):
    """out[r] = || (combination of the terms) h[r] / (tol + max(|y|, |y_new|) tol) ||_2
    per row (tct_qd_error_norm_batch)."""
    n, kp, ks, cs = _terms(Ks, coeffs)
    R, m = y.shape
    _lib.check(_lib.lib.tct_qd_error_norm_batch(
        m, R, n, kp, ks, cs, _lib.tptr(h.contiguous()), _lib.tptr(y), y.stride(0),
        _lib.tptr(y_new), y_new.stride(0), float(tol), _lib.tptr(out), _lib.stream_ptr()),
        "tct_qd_error_norm_batch")
    return out
