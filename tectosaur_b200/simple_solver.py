"""Constrained iterative solve with the Krylov state on the device
(reference: tectosaur/simple_solver.py:14-33 and examples/solve.py:25-61).

The reference forms `cm^T A cm` with scipy sparse products on the host and
runs scipy's GMRES (restart 200, tol 1e-8) with one host<->device round trip
of the operator per iteration.  Here the constrained operator, the Arnoldi
basis and every vector stay on the GPU:
  * cm and cm^T are CSR matrices applied by `tct_csr_matvec`;
  * the operator runs through its `dot_device` (FP32 or FP64 operators; the
    Krylov vectors are FP64 either way);
  * GMRES(m) with classical Gram-Schmidt applied twice (two matrix-vector
    products against the basis per step), Givens rotations of the small
    Hessenberg system on the host (one scalar column per step comes back).
`gmres` takes any callable matvec on torch tensors, so the algorithm is the
same on the CPU (tested there against scipy).
"""
import logging

import numpy as np

from . import _lib
from .util import device

logger = logging.getLogger(__name__)

defaults = dict(solver_tol=1e-8, restart=200)


def gmres(A, b, tol=1e-8, restart=200, maxiter=None, x0=None, M=None, callback=None):
    """Restarted GMRES for A x = b on torch tensors (b float64, any device).

    A, M: callables tensor -> tensor (M = right preconditioner, default none).
    Stops when the Arnoldi residual estimate ||b - A x|| <= tol ||b|| or after
    maxiter inner steps (default 10 n).  Returns (x, info, n_iter, residuals)
    with info = 0 on convergence, else the step count (scipy's convention)."""
    t = device.torch()
    n = b.shape[0]
    bnorm = float(t.linalg.norm(b))
    x = t.zeros_like(b) if x0 is None else x0.clone()
    hist = []
    if bnorm == 0.0:
        return x, 0, 0, hist
    maxiter = 10 * n if maxiter is None else maxiter
    m = max(1, min(restart, n))
    V = t.empty((m + 1, n), dtype=b.dtype, device=b.device)
    total = 0
    first = x0 is None
    while True:
        r = b.clone() if first else b - A(x)
        first = False
        beta = float(t.linalg.norm(r))
        if beta <= tol * bnorm:
            return x, 0, total, hist
        V[0] = r / beta
        H = np.zeros((m + 1, m))
        cs = np.zeros(m)
        sn = np.zeros(m)
        g = np.zeros(m + 1)
        g[0] = beta
        done = False
        j_end = m
        for j in range(m):
            w = A(V[j] if M is None else M(V[j]))
            Vj = V[: j + 1]
            h = Vj @ w
            w = w - h @ Vj
            h2 = Vj @ w
            w = w - h2 @ Vj
            h = h + h2
            hn = t.linalg.norm(w)
            col = t.cat([h, hn.reshape(1)]).cpu().numpy()  # the one sync of a step
            H[: j + 2, j] = col
            if col[-1] > 0.0:
                V[j + 1] = w / hn
            for i in range(j):
                a, c = H[i, j], H[i + 1, j]
                H[i, j] = cs[i] * a + sn[i] * c
                H[i + 1, j] = -sn[i] * a + cs[i] * c
            den = np.hypot(H[j, j], H[j + 1, j])
            cs[j] = H[j, j] / den if den > 0 else 1.0
            sn[j] = H[j + 1, j] / den if den > 0 else 0.0
            H[j, j] = den
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            total += 1
            res = abs(g[j + 1]) / bnorm
            hist.append(res)
            if callback is not None:
                callback(res)
            if res <= tol or total >= maxiter or col[-1] == 0.0:
                done = True
                j_end = j + 1
                break
        y = np.linalg.solve(np.triu(H[:j_end, :j_end]), g[:j_end]) if j_end > 0 else np.zeros(0)
        upd = t.as_tensor(y, dtype=b.dtype, device=b.device) @ V[:j_end]
        x = x + (upd if M is None else M(upd))
        if done:
            return x, (0 if hist and hist[-1] <= tol else total), total, hist


class DeviceCSR:
    """A scipy CSR matrix (double values) on the device; dot_device via
    tct_csr_matvec."""

    def __init__(self, mat):
        import scipy.sparse
        mat = scipy.sparse.csr_matrix(mat)
        mat.sort_indices()
        self.shape = mat.shape
        self.indptr = device.to_dev(mat.indptr.astype(np.int64))
        self.indices = device.to_dev(mat.indices.astype(np.int64) if mat.nnz else
                                     np.zeros(1, np.int64))
        self.data = device.to_dev(mat.data.astype(np.float64) if mat.nnz else np.zeros(1))

    def dot_device(self, x, y, accumulate=False, stream=None):
        prec = _lib.TCT_F64 if x.dtype == device.torch().float64 else _lib.TCT_F32
        _lib.check(_lib.lib.tct_csr_matvec(
            prec, self.shape[0], _lib.tptr(self.indptr), _lib.tptr(self.indices),
            _lib.tptr(self.data), _lib.tptr(x), _lib.tptr(y), int(bool(accumulate)),
            _lib.stream_ptr(stream)), "tct_csr_matvec")
        return y


def free_edge_vertices(tris):
    """Vertices on free edges (edges of exactly one triangle), the vertex set
    of the reference's find_free_edges / free_edge_dofs
    (constraint_builders.py:74-105)."""
    tris = np.asarray(tris)
    e = np.sort(np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]]), axis=1)
    uniq, counts = np.unique(e, axis=0, return_counts=True)
    return np.unique(uniq[counts == 1].reshape(-1))


def shared_vertex_matrix(tris, fixed_vertices=None):
    """Continuity constraint matrix tying together the DOFs of triangle
    corners that share a mesh vertex (component by component): cm[i, j] = 1
    when total DOF i = 9 tri + 3 corner + d sits at the j-th free (vertex, d).
    Vertices in `fixed_vertices` get no column (their DOFs are held at zero,
    the reference's free_edge_constraints with a zero field).  The reference
    builds such matrices from continuity constraints (constraint_builders.py,
    constraints.py:10-18); this one covers meshes whose vertices are shared by
    index.  The regularized hypersingular operator on an open surface is
    singular without zero slip on its free edges, so solves with it pass
    fixed_vertices=free_edge_vertices(tris)."""
    import scipy.sparse
    tris = np.asarray(tris)
    verts, inv = np.unique(tris.reshape(-1), return_inverse=True)
    col_of_vert = np.arange(verts.size)
    if fixed_vertices is not None and len(fixed_vertices):
        fixed = np.isin(verts, fixed_vertices)
        col_of_vert = np.where(fixed, -1, np.cumsum(~fixed) - 1)
    vcol = col_of_vert[inv]
    keep = np.repeat(vcol >= 0, 3)
    rows = np.arange(tris.size * 3)[keep]
    cols = (vcol[:, None] * 3 + np.arange(3)).reshape(-1)[keep]
    n_cols = int((col_of_vert >= 0).sum()) * 3
    return scipy.sparse.csr_matrix((np.ones(rows.size), (rows, cols)),
                                   shape=(tris.size * 3, n_cols))


class ConstrainedOperator:
    """v -> cm^T A cm v on the device (float64 vectors; the operator itself
    runs in its own float_type)."""

    def __init__(self, iop, cm=None):
        t = device.torch()
        self.iop = iop
        self.ft = device.torch_dtype(getattr(iop, "float_type", np.float64))
        self.cm = DeviceCSR(cm) if cm is not None else None
        self.cmT = DeviceCSR(cm.T) if cm is not None else None
        self.n = cm.shape[1] if cm is not None else iop.shape[1]
        self.x_full = t.zeros(iop.shape[1], dtype=self.ft, device="cuda")
        self.y_full = t.zeros(iop.shape[0], dtype=self.ft, device="cuda")
        self._tmp = t.zeros(iop.shape[1], dtype=t.float64, device="cuda")
        self.n_matvecs = 0

    def __call__(self, v):
        t = device.torch()
        self.n_matvecs += 1
        if self.cm is not None:
            self.cm.dot_device(v, self._tmp)
            self.x_full.copy_(self._tmp)
        else:
            self.x_full.copy_(v)
        self.iop.dot_device(self.x_full, self.y_full)
        yd = self.y_full.to(t.float64)
        if self.cmT is None:
            return yd
        out = t.empty(self.n, dtype=t.float64, device="cuda")
        return self.cmT.dot_device(yd, out)


def iterative_solve(iop, cm, rhs, prec=None, cfg=None):
    """Drop-in for simple_solver.iterative_solve (simple_solver.py:14-33):
    solves cm^T A cm x = cm^T rhs by GMRES and returns cm x as a host float64
    array.  cm: scipy sparse (n_total x n_free) or None for no constraints;
    prec: None, or a device callable (tensor -> tensor) used as a right
    preconditioner; cfg: dict with solver_tol (default 1e-8) and restart."""
    t = device.torch()
    cfg = dict(defaults, **(cfg or {}))
    op = ConstrainedOperator(iop, cm)
    rhs_d = device.to_dev(np.asarray(rhs, dtype=np.float64).reshape(-1))
    if cm is not None:
        b = t.empty(op.n, dtype=t.float64, device="cuda")
        op.cmT.dot_device(rhs_d, b)
    else:
        b = rhs_d

    def report(res):
        logger.debug("residual: %g", res)

    x, info, n_iter, hist = gmres(op, b, tol=cfg["solver_tol"], restart=cfg["restart"],
                                  M=prec, callback=report)
    iterative_solve.last = dict(info=info, n_iter=n_iter, residuals=hist,
                                n_matvecs=op.n_matvecs)
    if cm is not None:
        full = t.empty(cm.shape[0], dtype=t.float64, device="cuda")
        op.cm.dot_device(x, full)
        return full.cpu().numpy()
    return x.cpu().numpy()


# ---- many right-hand sides at once -----------------------------------------

def gmres_batch(A, B, tol=1e-8, restart=200, maxiter=None):
    """R independent restarted GMRES solves advancing in lockstep.

    A: callable (R, n) -> (R, n) on torch tensors; B: (R, n) float64.  Every
    step applies A to all R current basis vectors at once (the panel apply)
    and brings back one (R, j + 2) Hessenberg block; each system keeps its own
    Krylov basis, Givens rotations and stopping step, so a system that
    converges or breaks down early stops updating.  Returns (X, info, n_iter)
    with info[r] = 0 when system r reached ||b - A x|| <= tol ||b||."""
    t = device.torch()
    R, n = B.shape
    bnorm = t.linalg.norm(B, dim=1).cpu().numpy()
    X = t.zeros_like(B)
    maxiter = 10 * n if maxiter is None else maxiter
    m = max(1, min(restart, n))
    V = t.empty((R, m + 1, n), dtype=B.dtype, device=B.device)
    total = 0
    first = True
    bsafe = np.where(bnorm > 0, bnorm, 1.0)
    while True:
        Rr = B.clone() if first else B - A(X)
        first = False
        beta = t.linalg.norm(Rr, dim=1).cpu().numpy()
        done0 = beta <= tol * bnorm
        if done0.all():
            return X, np.zeros(R, np.int64), total
        bt = t.as_tensor(np.where(beta > 0, beta, 1.0), dtype=B.dtype, device=B.device)
        V[:, 0] = Rr / bt[:, None]
        H = np.zeros((R, m + 1, m))
        cs = np.zeros((R, m))
        sn = np.zeros((R, m))
        g = np.zeros((R, m + 1))
        g[:, 0] = beta
        stop = np.where(done0, 0, -1)  # per system: steps used in this cycle (-1 = running)
        j_end = m
        for j in range(m):
            W = A(V[:, j])
            Vj = V[:, : j + 1]
            h = t.bmm(Vj, W[:, :, None])[:, :, 0]
            W = W - t.bmm(h[:, None, :], Vj)[:, 0]
            h2 = t.bmm(Vj, W[:, :, None])[:, :, 0]
            W = W - t.bmm(h2[:, None, :], Vj)[:, 0]
            h = h + h2
            hn = t.linalg.norm(W, dim=1)
            col = t.cat([h, hn[:, None]], dim=1).cpu().numpy()  # the one sync of a step
            H[:, : j + 2, j] = col
            hs = t.where(hn > 0, hn, t.ones_like(hn))
            V[:, j + 1] = W / hs[:, None]
            for i in range(j):
                a, c = H[:, i, j].copy(), H[:, i + 1, j].copy()
                H[:, i, j] = cs[:, i] * a + sn[:, i] * c
                H[:, i + 1, j] = -sn[:, i] * a + cs[:, i] * c
            den = np.hypot(H[:, j, j], H[:, j + 1, j])
            ok = den > 0
            cs[:, j] = np.where(ok, H[:, j, j] / np.where(ok, den, 1.0), 1.0)
            sn[:, j] = np.where(ok, H[:, j + 1, j] / np.where(ok, den, 1.0), 0.0)
            H[:, j, j] = den
            H[:, j + 1, j] = 0.0
            g[:, j + 1] = -sn[:, j] * g[:, j]
            g[:, j] = cs[:, j] * g[:, j]
            total += 1
            res = np.abs(g[:, j + 1]) / bsafe
            newly = (stop < 0) & ((res <= tol) | (col[:, -1] == 0.0))
            stop[newly] = j + 1
            if (stop >= 0).all() or total >= maxiter:
                j_end = j + 1
                break
        k = np.where(stop < 0, j_end, stop)
        Y = np.zeros((R, j_end))
        for r in range(R):
            if k[r] > 0:
                Y[r, : k[r]] = np.linalg.solve(np.triu(H[r, : k[r], : k[r]]), g[r, : k[r]])
        X = X + t.bmm(t.as_tensor(Y, dtype=B.dtype, device=B.device)[:, None, :],
                      V[:, :j_end])[:, 0]
        if (stop >= 0).all() or total >= maxiter:
            final = np.abs(g[np.arange(R), k]) / bsafe
            return X, np.where(final <= tol, 0, total).astype(np.int64), total


class ConstrainedPanelOperator:
    """V (R, n_free) float64 -> cm^T A cm V for a panel of R vectors.  An
    operator with dot_panel_device applies all R vectors at once (FP32
    elasticRH3: tensor-core farfield panel + one BSR panel launch); other
    operators apply dot_device vector by vector."""

    def __init__(self, iop, cm, R):
        t = device.torch()
        self.iop = iop
        self.R = R
        self.ft = device.torch_dtype(getattr(iop, "float_type", np.float64))
        self.cm = DeviceCSR(cm)
        self.cmT = DeviceCSR(cm.T)
        self.n = cm.shape[1]
        self.n_full_in, self.n_full_out = iop.shape[1], iop.shape[0]
        self.U = t.zeros((R, self.n_full_in), dtype=t.float64, device="cuda")
        self.Xf = t.zeros((R, self.n_full_in), dtype=self.ft, device="cuda")
        self.Yf = t.zeros((R, self.n_full_out), dtype=self.ft, device="cuda")
        self.panel = hasattr(iop, "dot_panel_device")

    def _csr_panel(self, mat, X, Y):
        _lib.check(_lib.lib.tct_csr_matvec_panel(
            _lib.TCT_F64, mat.shape[0], _lib.tptr(mat.indptr), _lib.tptr(mat.indices),
            _lib.tptr(mat.data), _lib.tptr(X), X.shape[1], _lib.tptr(Y), Y.shape[1], X.shape[0],
            0, _lib.stream_ptr()), "tct_csr_matvec_panel")
        return Y

    def __call__(self, V):
        t = device.torch()
        R = V.shape[0]
        U = self._csr_panel(self.cm, V.contiguous(), self.U[:R])
        self.Xf[:R].copy_(U)
        if self.panel:
            self.iop.dot_panel_device(self.Xf[:R], self.Yf[:R])
        else:
            for r in range(R):
                self.iop.dot_device(self.Xf[r], self.Yf[r])
        out = t.empty((R, self.n), dtype=t.float64, device="cuda")
        return self._csr_panel(self.cmT, self.Yf[:R].to(t.float64), out)


def iterative_solve_batch(iop64, iop32, cm, rhs, tol=1e-8, inner_tol=1e-5, restart=200,
                          max_refine=8):
    """R constrained solves at once, mixed precision: GMRES on the FP32
    operator (tensor-core panel farfield) inside FP64 iterative refinement
    with residuals of the FP64 operator, to ||cm^T (rhs - A u)|| <= tol
    ||cm^T rhs|| in FP64 for every system; each correction solve stops at
    max(inner_tol, tol / (2 r)) relative, r the current relative residual.
    rhs: (R, n_total) host or device;
    returns (R, n_total) host float64 and records the refinement history in
    iterative_solve_batch.last."""
    t = device.torch()
    rhs_d = (rhs if device.is_device_tensor(rhs) else
             device.to_dev(np.asarray(rhs, np.float64))).to(t.float64)
    R = rhs_d.shape[0]
    A64 = ConstrainedPanelOperator(iop64, cm, R)
    A32 = ConstrainedPanelOperator(iop32, cm, R)
    b = A64._csr_panel(A64.cmT, rhs_d.contiguous(),
                       t.empty((R, A64.n), dtype=t.float64, device="cuda"))
    bn = t.linalg.norm(b, dim=1)
    x = t.zeros_like(b)
    steps, resid = [], []
    for _ in range(max_refine):
        r = b - A64(x) if steps else b.clone()
        rel = float((t.linalg.norm(r, dim=1) / t.where(bn > 0, bn, t.ones_like(bn))).max())
        resid.append(rel)
        if rel <= tol:
            break
        # no more accurate than the outer tolerance needs
        eta = max(inner_tol, 0.5 * tol / rel) if rel > 0 else inner_tol
        d, info, n_it = gmres_batch(A32, r, tol=eta, restart=restart)
        steps.append(n_it)
        x = x + d
    else:
        r = b - A64(x)
        resid.append(float((t.linalg.norm(r, dim=1) / t.where(bn > 0, bn, t.ones_like(bn))).max()))
    iterative_solve_batch.last = dict(gmres_steps=steps, residuals=resid)
    full = t.empty((R, cm.shape[0]), dtype=t.float64, device="cuda")
    A64._csr_panel(A64.cm, x.contiguous(), full)
    return full.cpu().numpy()
