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
