"""Served solve stream: continuous batching of constrained BEM solves.

The reference solves one system at a time (examples/solve.py:25-61,
simple_solver.py:14-33): each solve builds its own operator and drives
scipy's GMRES with a host round trip per iteration.  This module keeps the
operators of several meshes resident on the device and serves a stream of
solve requests (mesh, right-hand side, tolerance) arriving at any time.

Continuous batching.  Each resident mesh owns a SolveEngine with S slots
(S = 16, the width of the tensor-core farfield panel).  A request takes a
free slot of its mesh's engine and leaves it when its FP64 residual reaches
its tolerance; free slots are refilled between Arnoldi steps, so requests
that arrive while others are on the GPU join the running batch rather than
wait for it to drain.

Per slot, mixed-precision iterative refinement: FP64 residual r = b - A x
with the FP64 operator, a correction by restarted GMRES(m) on the FP32
operator to max(inner_tol, tol ||b|| / 2 ||r||) ||r|| (no more accurate than
the request needs), x += correction, until ||r|| <= tol ||b||.  The
slots of an engine that are in their GMRES phase advance together, each at
its own step count: one panel apply of the FP32 operator for all slots
(tensor-core farfield panel + BSR panel + CSR panels), classical
Gram-Schmidt applied twice as batched products against each slot's own
basis (columns past a slot's step masked out), one device-to-host copy of
the new Hessenberg columns, and the Givens updates on the host
(tct_gmres_givens).  A slot's arithmetic never mixes with another slot's,
so a request's result does not depend on what else is in the batch beyond
the summation order of library reductions.

Engines of different meshes run on their own CUDA streams.  The scheduling
loop completes an engine's tick as soon as the device has finished it (an
event query, no wait) and enqueues its next one, so the work of different
meshes overlaps on the device and a slow engine holds back no other.

HBM admission.  A mesh's operators (FP64 nearfield blocks, their FP32 cast,
farfield workspaces) and its engine state are built when its first request
is admitted.  Before a build, idle meshes (no occupied slot) are released,
least recently used first, until the mesh's footprint (measured on earlier
builds, else estimated) fits the budget; requests whose mesh does not fit
wait in the queue without blocking requests for resident meshes.
"""
import collections
import contextlib
import itertools
import time

import numpy as np

from . import _lib
from .util import device

FREE, RESID, INNER = 0, 1, 2


class Request:
    """One solve: u = cm x with cm^T A cm x = cm^T rhs, ||cm^T (rhs - A u)||
    <= tol ||cm^T rhs|| in FP64."""

    _ids = itertools.count()

    def __init__(self, key, rhs, tol, t_submit=None):
        self.id = next(Request._ids)
        self.key = key
        self.rhs = np.ascontiguousarray(rhs, dtype=np.float64).reshape(-1)
        self.tol = float(tol)
        self.t_submit = time.perf_counter() if t_submit is None else t_submit
        self.t_admit = None
        self.t_done = None
        self.x = None
        self.residual = None
        self.gmres_steps = 0
        self.refinements = 0
        self.converged = False
        self.error = None

    @property
    def done(self):
        return self.t_done is not None

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit


def _givens(sys_idx, j, m, cols, H, cs, sn, g):
    res = np.empty(sys_idx.shape[0])
    cols = np.ascontiguousarray(cols, dtype=np.float64)
    _lib.check(_lib.lib.tct_gmres_givens(
        sys_idx.shape[0], _lib.i64ptr(sys_idx), _lib.i64ptr(j), m, _lib.dptr(cols),
        cols.shape[1], _lib.dptr(H), _lib.dptr(cs), _lib.dptr(sn), _lib.dptr(g),
        _lib.dptr(res)), "tct_gmres_givens")
    return res


class SolveEngine:
    """S solve slots on one operator pair.

    A32, A64: callables (k, n) float64 tensor -> (k, n) float64 (the
    constrained FP32 and FP64 operators, k <= S); to_free(rhs (n_total,)
    float64 tensor) -> (n,) = cm^T rhs; to_full(x (n,)) -> (n_total,) = cm x.
    dev: torch device of the vectors; stream: CUDA stream (None on the CPU).
    """

    def __init__(self, A32, A64, to_free, to_full, n, slots=16, restart=64, inner_tol=1e-6,
                 max_refine=20, dev="cuda", stream=None):
        t = device.torch()
        self.t = t
        self.A32, self.A64 = A32, A64
        self.to_free, self.to_full = to_free, to_full
        self.n = int(n)
        self.S = int(slots)
        self.m = max(1, min(int(restart), self.n))
        self.inner_tol = float(inner_tol)
        self.max_refine = int(max_refine)
        self.dev = t.device(dev)
        self.stream = stream
        S, m, f64 = self.S, self.m, t.float64
        self.V = t.zeros((S, m + 1, self.n), dtype=f64, device=self.dev)
        self.X = t.zeros((S, self.n), dtype=f64, device=self.dev)
        self.B = t.zeros((S, self.n), dtype=f64, device=self.dev)
        self.Rv = t.zeros((S, self.n), dtype=f64, device=self.dev)
        pin = self.dev.type == "cuda"
        self._pin = pin
        # the new Hessenberg columns of a tick, (S, J + 1) row-major in the
        # first S (J + 1) entries: a contiguous destination, so the copy from
        # the device is one asynchronous memcpy (a copy into a strided slice
        # of pinned memory falls back to a synchronous one, which held the
        # host on every engine's tick until the tick had run on the device)
        self._cols = t.zeros(S * (m + 2), dtype=f64, pin_memory=pin)
        self._norms = t.zeros(S, dtype=f64, pin_memory=pin)
        # host -> device control block of a tick (slot lists and step counts)
        # and back-substitution results, staged in pinned memory so that no
        # copy blocks the host (a pinned buffer is rewritten only after the
        # tick that read it has completed)
        self._ctl = t.zeros(5 * S, dtype=t.int64, pin_memory=pin)
        self._ctl_d = t.zeros(5 * S, dtype=t.int64, device=self.dev)
        self._ybuf = t.zeros((S, m), dtype=f64, pin_memory=pin)
        self._yd = t.zeros((S, m), dtype=f64, device=self.dev)
        self._rhs_pin = None
        self._event = t.cuda.Event() if pin else None
        self.state = np.full(S, FREE, np.int64)
        self.fresh = np.zeros(S, bool)      # x = 0: the residual is b
        self.j = np.zeros(S, np.int64)
        self.H = np.zeros((S, m, m + 1))    # column-major per slot: H[s, col, row]
        self.cs = np.zeros((S, m))
        self.sn = np.zeros((S, m))
        self.g = np.zeros((S, m + 1))
        self.beta = np.zeros(S)
        self.eta = np.zeros(S)              # this cycle's relative GMRES tolerance
        self.bnorm = np.zeros(S)
        self.req = [None] * S
        self.last_used = time.perf_counter()
        self.n_panel_applies = 0
        self.n_vector_applies = 0
        self._pending = None

    # -- slots ---------------------------------------------------------------
    def _ctx(self):
        if self.stream is None:
            return contextlib.nullcontext()
        return self.t.cuda.stream(self.stream)

    @property
    def free_slots(self):
        return int((self.state == FREE).sum())

    @property
    def busy(self):
        return bool((self.state != FREE).any())

    @property
    def pending(self):
        """A tick enqueued and not yet completed."""
        return getattr(self, "_pending", None) is not None

    def ready(self):
        """The enqueued tick has finished on the device (no wait)."""
        return self._event is None or self._event.query()

    def admit(self, req):
        """Put a request into a free slot (False if none)."""
        free = np.flatnonzero(self.state == FREE)
        if free.size == 0:
            return False
        s = int(free[0])
        t = self.t
        with self._ctx():
            rhs = t.from_numpy(req.rhs)
            if self._pin:
                if self._rhs_pin is None or self._rhs_pin.shape[1] != rhs.shape[0]:
                    self._rhs_pin = t.zeros((self.S, rhs.shape[0]), dtype=t.float64,
                                            pin_memory=True)
                self._rhs_pin[s].copy_(rhs)
                rhs = self._rhs_pin[s].to(self.dev, non_blocking=True)
            self.B[s] = self.to_free(rhs)
            self.X[s].zero_()
        self.state[s] = RESID
        self.fresh[s] = True
        self.req[s] = req
        req.t_admit = time.perf_counter()
        self.last_used = req.t_admit
        return True

    # -- one scheduling tick: enqueue, then complete -----------------------------
    def launch(self):
        """Enqueue this tick's device work: FP64 residuals of the slots in
        the residual phase, one Arnoldi step of the slots in the GMRES phase."""
        t = self.t
        resid = np.flatnonzero(self.state == RESID)
        inner = np.flatnonzero(self.state == INNER)
        if resid.size == 0 and inner.size == 0:
            self._pending = None
            return
        J = 0
        S = self.S
        stale = resid[~self.fresh[resid]]
        fr = resid[self.fresh[resid]]
        ctl = self._ctl.numpy()
        for k, lst in enumerate((resid, stale, fr, inner)):
            ctl[k * S: k * S + lst.size] = lst
        ctl[4 * S:] = self.j
        with self._ctx():
            cd = self._ctl_d
            cd.copy_(self._ctl, non_blocking=True)
            if resid.size:
                ri = cd[: resid.size]
                if stale.size:
                    si = cd[S: S + stale.size]
                    self.Rv[si] = self.B[si] - self.A64(self.X[si])
                    self.n_vector_applies += stale.size
                if fr.size:
                    fi = cd[2 * S: 2 * S + fr.size]
                    self.Rv[fi] = self.B[fi]
                self._norms[: resid.size].copy_(t.linalg.norm(self.Rv[ri], dim=1),
                                                non_blocking=True)
            if inner.size:
                J = int(self.j[inner].max()) + 1
                ii = cd[3 * S: 3 * S + inner.size]
                jt = cd[4 * S:]
                # index_fill_ passes the value as a kernel argument; an
                # assignment `act[ii] = True` would make it a host tensor and
                # copy it synchronously, holding the host on every tick
                act = t.zeros(S, dtype=t.bool, device=self.dev).index_fill_(0, ii, True)
                # the operator is applied to the active slots' columns only
                # (an FMM farfield costs one pass per column; columns are
                # independent, so a slot's result does not depend on the others)
                W = t.zeros((S, self.n), dtype=t.float64, device=self.dev)
                W[ii] = self.A32(self.V[ii, jt[ii]])
                self.n_panel_applies += 1
                self.n_vector_applies += inner.size
                mask = ((t.arange(J, device=self.dev)[None, :] <= jt[:, None]) & act[:, None])
                mask = mask.to(t.float64)
                Vj = self.V[:, :J]
                h = t.bmm(Vj, W[:, :, None])[:, :, 0] * mask
                W = W - t.bmm(h[:, None, :], Vj)[:, 0]
                h2 = t.bmm(Vj, W[:, :, None])[:, :, 0] * mask
                W = W - t.bmm(h2[:, None, :], Vj)[:, 0]
                h = h + h2
                hn = t.linalg.norm(W, dim=1)
                hs = t.where(hn > 0, hn, t.ones_like(hn))
                self.V[ii, jt[ii] + 1] = W[ii] / hs[ii, None]
                hc = t.cat((h, hn[:, None]), dim=1)
                self._cols[: S * (J + 1)].copy_(hc.reshape(-1), non_blocking=True)
            if self._event is not None:
                self._event.record()
        self._pending = (resid, inner, J)

    def complete(self):
        """Finish this tick on the host; returns the requests that completed."""
        if self._pending is None:
            return []
        resid, inner, J = self._pending
        self._pending = None
        if self._event is not None:
            self._event.synchronize()
        t = self.t
        finished = []
        norms = self._norms.numpy()[: resid.size].copy()
        cols = (self._cols.numpy()[: self.S * (J + 1)].reshape(self.S, J + 1).copy()
                if inner.size else None)
        now = time.perf_counter()
        self.last_used = now
        # residual phase: finish, or start a GMRES cycle on the residual
        for i, s in enumerate(resid):
            req = self.req[s]
            if self.fresh[s]:
                self.bnorm[s] = norms[i]
                self.fresh[s] = False
            rel = norms[i] / self.bnorm[s] if self.bnorm[s] > 0 else 0.0
            req.residual = rel
            if rel <= req.tol or req.refinements >= self.max_refine:
                req.converged = rel <= req.tol
                with self._ctx():
                    u = self.to_full(self.X[s])
                    req.x = u.cpu().numpy()
                req.t_done = time.perf_counter()
                finished.append(req)
                self.req[s] = None
                self.state[s] = FREE
                continue
            req.refinements += 1
            beta = norms[i]
            with self._ctx():
                self.V[s, 0] = self.Rv[s] / beta
            self.beta[s] = beta
            # the correction need not be more accurate than the request needs
            self.eta[s] = max(self.inner_tol, 0.5 * req.tol / rel) if rel > 0 else self.inner_tol
            self.g[s] = 0.0
            self.g[s, 0] = beta
            self.j[s] = 0
            self.state[s] = INNER
        if inner.size == 0:
            return finished
        # GMRES phase: Givens updates, then cycle ends
        c = cols[inner]
        c[np.arange(inner.size), self.j[inner] + 1] = c[:, J]
        res = _givens(np.ascontiguousarray(inner, dtype=np.int64), self.j, self.m, c,
                      self.H, self.cs, self.sn, self.g)
        for i, s in enumerate(inner):
            req = self.req[s]
            req.gmres_steps += 1
            k = int(self.j[s]) + 1
            broke = cols[s, J] == 0.0
            if res[i] <= self.eta[s] * self.beta[s] or k == self.m or broke:
                Rm = self.H[s, :k, :k].T
                self._ybuf.numpy()[s, :k] = _back_substitute(Rm, self.g[s, :k])
                with self._ctx():
                    yd = self._yd[s, :k]
                    yd.copy_(self._ybuf[s, :k], non_blocking=True)
                    self.X[s] += yd @ self.V[s, :k]
                self.state[s] = RESID
            else:
                self.j[s] = k
        return finished


class QdRequest:
    """n_steps quasidynamic RK23 steps of a fault model from (t0, y0)."""

    _ids = itertools.count()

    def __init__(self, key, y0, n_steps, t0=0.0, first_step=None, t_submit=None):
        self.id = next(QdRequest._ids)
        self.key = key
        self.y0 = np.ascontiguousarray(y0, dtype=np.float64).reshape(-1)
        self.n_steps = int(n_steps)
        self.t0 = float(t0)
        self.first_step = first_step
        self.t_submit = time.perf_counter() if t_submit is None else t_submit
        self.t_admit = None
        self.t_done = None
        self.y = None
        self.ts = []
        self.steps = 0
        self.rejected = 0
        self.error = None
        self.converged = False

    @property
    def done(self):
        return self.t_done is not None

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit


class QdEngine:
    """S quasidynamic integrations on one fault model, advancing together:
    each tick every occupied slot makes one RK23 attempt (scipy's RK23 step
    control per slot, restated in qd/rk23.py), its three derivative
    evaluations batched over the slots (one panel apply of H, one CG launch,
    one Newton launch, one averaging launch per evaluation); slots are
    refilled between ticks."""

    def __init__(self, model, slots=16, stream=None):
        t = device.torch()
        from .qd import model as qd_model
        from .qd import rk23 as rk
        self.t, self.rk, self.qm = t, rk, qd_model
        self.model = model
        self.derivs = model.derivs_batch
        self.S = int(slots)
        self.stream = stream
        self.n_y = 12 * model.n_tris
        self.tol = float(model.cfg["timestep_tol"])
        self.Y = t.zeros((self.S, self.n_y), dtype=t.float64, device="cuda")
        self.F = t.zeros_like(self.Y)
        self.tv = np.zeros(self.S)
        self.h = np.zeros(self.S)
        self.rejected_now = np.zeros(self.S, bool)
        self.req = [None] * self.S
        self._norms = t.zeros(self.S, dtype=t.float64, pin_memory=True)
        self._ndev = t.zeros(self.S, dtype=t.float64, device="cuda")
        self._tpin = t.zeros((4, self.S), dtype=t.float64, pin_memory=True)
        self._tdev = t.zeros((4, self.S), dtype=t.float64, device="cuda")
        self._ipin = t.zeros(self.S, dtype=t.int64, pin_memory=True)
        self._idev = t.zeros(self.S, dtype=t.int64, device="cuda")
        self._event = t.cuda.Event()
        self._pending = None
        self.last_used = time.perf_counter()

    def _ctx(self):
        if self.stream is None:
            return contextlib.nullcontext()
        return self.t.cuda.stream(self.stream)

    @property
    def free_slots(self):
        return sum(r is None for r in self.req)

    @property
    def busy(self):
        return any(r is not None for r in self.req)

    @property
    def pending(self):
        return self._pending is not None

    def ready(self):
        return self._event.query()

    def admit(self, req):
        free = [s for s in range(self.S) if self.req[s] is None]
        if not free:
            return False
        if req.y0.shape[0] != self.n_y:
            req.error = "state of %d values, the model has %d" % (req.y0.shape[0], self.n_y)
            req.t_done = time.perf_counter()
            return True
        s = free[0]
        t = self.t
        with self._ctx():
            self.Y[s] = t.from_numpy(req.y0).to("cuda")
            ts = t.full((1,), req.t0, dtype=t.float64, device="cuda")
            self.F[s] = self.derivs(ts, self.Y[s:s + 1])[0]
        self.tv[s] = req.t0
        self.h[s] = req.first_step if req.first_step is not None else 3.15576e6
        self.rejected_now[s] = False
        self.req[s] = req
        req.t_admit = time.perf_counter()
        if req.n_steps <= 0:
            self._finish(s)
        return True

    def _finish(self, s, error=None):
        req = self.req[s]
        with self._ctx():
            req.y = self.Y[s].cpu().numpy()
        req.error = error
        req.converged = error is None
        req.t_done = time.perf_counter()
        self.req[s] = None
        return req

    def launch(self):
        t, rk = self.t, self.rk
        act = [s for s in range(self.S) if self.req[s] is not None]
        self._pending = None
        if not act:
            return
        k = len(act)
        h = np.array([self.h[s] for s in act])
        tv = np.array([self.tv[s] for s in act])
        tp = self._tpin.numpy()
        tp[0, :k] = h
        tp[1, :k] = tv + rk.C[1] * h
        tp[2, :k] = tv + rk.C[2] * h
        tp[3, :k] = tv + h
        self._ipin.numpy()[:k] = act
        with self._ctx():
            self._tdev.copy_(self._tpin, non_blocking=True)
            self._idev.copy_(self._ipin, non_blocking=True)
            idx = self._idev[:k]
            hdev = self._tdev[0, :k]  # the step sizes on the device (h stays on the host)
            y, K0 = self.Y[idx], self.F[idx]
            # stage inputs, the new state and the error norm: one fused
            # launch each, rounded as y + (K0 a10) h, y + (K0 a20 + K1 a21) h,
            # y + h (K0 b0 + K1 b1 + K2 b2), ||(sum_j K_j e_j) h / scale||
            ys = t.empty_like(y)
            self.qm.combine_batch([K0], [rk.A[1][0]], hdev, y, ys)
            K1 = self.derivs(self._tdev[1, :k], ys)
            self.qm.combine_batch([K0, K1], [rk.A[2][0], rk.A[2][1]], hdev, y, ys)
            K2 = self.derivs(self._tdev[2, :k], ys)
            y_new = t.empty_like(y)
            self.qm.combine_batch([K0, K1, K2], rk.B[:3], hdev, y, y_new)
            f_new = self.derivs(self._tdev[3, :k], y_new)
            self.qm.error_norm_batch([K0, K1, K2, f_new], rk.E[:4], hdev, y, y_new, self.tol,
                                     self._ndev[:k])
            self._norms[:k].copy_(self._ndev[:k], non_blocking=True)
            self._event.record()
        self._pending = (act, h, y_new, f_new)

    def complete(self):
        if self._pending is None:
            return []
        rk = self.rk
        act, h, y_new, f_new = self._pending
        self._pending = None
        self._event.synchronize()
        norms = self._norms.numpy()[: len(act)] / np.sqrt(self.n_y)
        self.last_used = time.perf_counter()
        done = []
        for i, s in enumerate(act):
            req = self.req[s]
            en = float(norms[i])
            t_old = self.tv[s]
            min_step = 10 * abs(np.nextafter(t_old, np.inf) - t_old)
            if en < 1:
                factor = rk.MAX_FACTOR if en == 0 else min(rk.MAX_FACTOR,
                                                           rk.SAFETY * en ** rk.ERROR_EXPONENT)
                if self.rejected_now[s]:
                    factor = min(1.0, factor)
                with self._ctx():
                    self.Y[s] = y_new[i]
                    self.F[s] = f_new[i]
                self.tv[s] = t_old + h[i]
                self.h[s] = h[i] * factor
                self.rejected_now[s] = False
                req.steps += 1
                req.ts.append(self.tv[s])
                if req.steps >= req.n_steps:
                    done.append(self._finish(s))
            else:
                shrink = rk.SAFETY * en ** rk.ERROR_EXPONENT if en == en else 0.0
                self.h[s] = h[i] * max(rk.MIN_FACTOR, shrink)
                self.rejected_now[s] = True
                req.rejected += 1
                if self.h[s] < min_step:
                    done.append(self._finish(s, error="step size below the spacing of t"))
        return done


def _back_substitute(R, g):
    k = g.shape[0]
    y = np.zeros(k)
    for i in range(k - 1, -1, -1):
        d = R[i, i]
        y[i] = (g[i] - R[i, i + 1:] @ y[i + 1:]) / d if d != 0 else 0.0
    return y


class MeshSpec:
    """A mesh the server can make resident: geometry, constraints and the
    RegularizedSparseIntegralOp arguments."""

    def __init__(self, key, pts, tris, cm=None, nq=(6, 6, 6, 2, 5, 2.5), kernel="elasticRH3",
                 params=(1.0, 0.25), farfield_op_type=None, op64=None,
                 inner_farfield_op_type=None, inner_tol=None):
        self.key = key
        # relative tolerance floor of the FP32 correction solves (None: the
        # server's); an FP32 operator whose rounding floor is above the
        # server's floor (the FP32 FMM) needs a looser one
        self.inner_tol = inner_tol
        # farfield of the FP32 correction operator when it differs from the
        # FP64 residual operator's (None: the same type)
        self.inner_farfield_op_type = inner_farfield_op_type
        self.op64 = op64  # an FP64 operator built by the caller (kept while registered)
        self.pts = np.asarray(pts, np.float64)
        self.tris = np.asarray(tris, np.int64)
        self.cm = cm
        self.nq = tuple(nq)
        self.kernel = kernel
        self.params = list(params)
        self.farfield_op_type = farfield_op_type
        self.measured_bytes = None

    @property
    def n_tris(self):
        return self.tris.shape[0]

    def estimate_bytes(self, slots, restart):
        """Footprint before the first build: ~100 nearfield blocks per
        triangle in FP64 + FP32, the panel farfield operand, the Krylov
        bases of the slots."""
        n = self.n_tris
        if getattr(self, "kind", "solve") == "qd":
            return int(n * 100 * 648 + n * 8100 + slots * 4 * 12 * n * 8)
        n_free = self.cm.shape[1] if self.cm is not None else 9 * n
        return int(n * 100 * (648 + 324) + n * 8100 + slots * (restart + 4) * n_free * 8)


def _op_bytes(op):
    """Device bytes held by a RegularizedSparseIntegralOp (nearfield blocks,
    farfield workspace)."""
    near = op.nearfield
    n = near.bsr.nbytes
    if getattr(near, "correction", None) is not None:
        n += near.correction.numel() * near.correction.element_size()
    ws = getattr(op.farfield, "workspace", None)
    if ws is not None:
        n += ws.numel() * ws.element_size()
    return int(n)


class _Resident:
    def __init__(self, spec, op64, op32, engine, nbytes):
        self.spec, self.op64, self.op32, self.engine = spec, op64, op32, engine
        self.nbytes = nbytes


class SolveServer:
    """Continuous-batching solve server over resident meshes (module docstring).

    hbm_budget: bytes the resident meshes may take (None: 85 % of the
    device's free memory at construction).  builder(server, spec) ->
    _Resident makes a mesh resident (default: the device operators of
    RegularizedSparseIntegralOp in FP64 and its FP32 cast)."""

    def __init__(self, hbm_budget=None, slots=16, restart=64, inner_tol=1e-6, max_refine=20,
                 builder=None):
        if builder is None:
            t = device.require_cuda()
            if hbm_budget is None:
                free, _ = t.cuda.mem_get_info()
                hbm_budget = int(0.85 * free)
        elif hbm_budget is None:
            raise ValueError("hbm_budget is required with a custom builder")
        self.builder = builder or SolveServer._build
        self.hbm_budget = int(hbm_budget)
        self.slots, self.restart = slots, restart
        self.inner_tol, self.max_refine = inner_tol, max_refine
        self.specs = {}
        self.resident = collections.OrderedDict()
        self.queue = collections.deque()
        self.completed = []
        self.n_builds = 0
        self.n_evictions = 0

    # -- meshes ------------------------------------------------------------------
    def add_qd_mesh(self, key, pts, tris, cfg, model=None):
        """A fault for quasidynamic requests (qd.FullspaceModel(m, cfg))."""
        spec = MeshSpec(key, pts, tris)
        spec.kind = "qd"
        spec.qd_cfg = cfg
        spec.model = model
        self.specs[key] = spec
        return spec

    def add_mesh(self, key, pts, tris, cm=None, **op_args):
        from .ops.sparse_farfield_op import TriToTriDirectFarfieldOp
        op_args.setdefault("farfield_op_type", TriToTriDirectFarfieldOp)
        self.specs[key] = MeshSpec(key, pts, tris, cm, **op_args)
        return self.specs[key]

    @property
    def resident_bytes(self):
        return sum(r.nbytes for r in self.resident.values())

    def _footprint(self, spec):
        if spec.measured_bytes is not None:
            return spec.measured_bytes
        return spec.estimate_bytes(self.slots, self.restart)

    def _release(self, key):
        r = self.resident.pop(key)
        r.engine = r.op64 = r.op32 = None
        self.n_evictions += 1

    def _make_room(self, need):
        for key in list(self.resident):
            if self.resident_bytes + need <= self.hbm_budget:
                break
            e = self.resident[key].engine
            if not (e.busy or e.pending):
                self._release(key)
        return self.resident_bytes + need <= self.hbm_budget

    @staticmethod
    def _build(self, spec):
        if getattr(spec, "kind", "solve") == "qd":
            return SolveServer._build_qd(self, spec)
        from .ops.sparse_integral_op import RegularizedSparseIntegralOp
        from .simple_solver import ConstrainedPanelOperator, DeviceCSR
        t = device.torch()
        t.cuda.synchronize()
        before = t.cuda.memory_allocated()
        op64 = spec.op64
        if op64 is None:
            op64 = RegularizedSparseIntegralOp(*spec.nq, spec.kernel, spec.kernel, spec.params,
                                               spec.pts, spec.tris, np.float64,
                                               spec.farfield_op_type, keep_uncorrected=False)
        op32 = op64.astype(np.float32, keep_uncorrected=False,
                           farfield_op_type=getattr(spec, "inner_farfield_op_type", None))
        cm = spec.cm
        S = self.slots
        if cm is None:
            import scipy.sparse
            cm = scipy.sparse.identity(op64.shape[1], format="csr")
        A32 = ConstrainedPanelOperator(op32, cm, S)
        A64 = ConstrainedPanelOperator(op64, cm, S)
        cmd, cmtd = DeviceCSR(cm), DeviceCSR(cm.T)
        n = cm.shape[1]

        def to_free(rhs):
            out = t.empty(n, dtype=t.float64, device="cuda")
            return cmtd.dot_device(rhs, out)

        def to_full(x):
            out = t.empty(cm.shape[0], dtype=t.float64, device="cuda")
            return cmd.dot_device(x.contiguous(), out)

        inner_tol = spec.inner_tol if spec.inner_tol is not None else self.inner_tol
        engine = SolveEngine(A32, A64, to_free, to_full, n, S, self.restart, inner_tol,
                             self.max_refine, "cuda", t.cuda.Stream())
        t.cuda.synchronize()
        nbytes = t.cuda.memory_allocated() - before
        if spec.op64 is not None:  # built before, outside the measurement
            nbytes += _op_bytes(spec.op64)
        spec.measured_bytes = max(nbytes, 1)
        self.n_builds += 1
        return _Resident(spec, op64, op32, engine, spec.measured_bytes)

    @staticmethod
    def _build_qd(self, spec):
        from .qd import FullspaceModel
        t = device.torch()
        t.cuda.synchronize()
        before = t.cuda.memory_allocated()
        model = spec.model or FullspaceModel((spec.pts, spec.tris), spec.qd_cfg)
        # a high-priority stream: an RK23 tick is a chain of small,
        # latency-bound kernels and a host sync, which would otherwise queue
        # behind the solve engines' panel and FMM kernels
        engine = QdEngine(model, self.slots,
                          t.cuda.Stream(priority=t.cuda.Stream.priority_range()[1]))
        t.cuda.synchronize()
        spec.measured_bytes = max(t.cuda.memory_allocated() - before, 1)
        self.n_builds += 1
        return _Resident(spec, None, None, engine, spec.measured_bytes)

    def submit_qd(self, key, y0, n_steps, t0=0.0, first_step=None, t_submit=None):
        """A quasidynamic request: n_steps RK23 steps from (t0, y0) on a
        fault registered with add_qd_mesh; its result is req.y (host) and
        req.ts (the accepted step times)."""
        if getattr(self.specs.get(key), "kind", None) != "qd":
            raise KeyError("no quasidynamic mesh %r" % (key,))
        req = QdRequest(key, y0, n_steps, t0, first_step, t_submit)
        self.queue.append(req)
        return req

    def _engine_for(self, key):
        if key in self.resident:
            self.resident.move_to_end(key)
            return self.resident[key].engine
        spec = self.specs[key]
        if not self._make_room(self._footprint(spec)):
            return None
        r = self.builder(self, spec)
        self.resident[key] = r
        if self.resident_bytes > self.hbm_budget:
            self._make_room(0)
        return r.engine

    # -- requests ----------------------------------------------------------------
    def submit(self, key, rhs, tol=1e-8, t_submit=None):
        if key not in self.specs:
            raise KeyError("unknown mesh %r" % (key,))
        req = Request(key, rhs, tol, t_submit)
        self.queue.append(req)
        return req

    def _admit(self):
        waiting = collections.deque()
        while self.queue:
            req = self.queue.popleft()
            eng = self._engine_for(req.key)
            if eng is None and not self.resident and \
                    self._footprint(self.specs[req.key]) > self.hbm_budget:
                # larger than the whole budget: refused, not queued for ever
                req.error = "mesh footprint %d bytes exceeds the HBM budget %d" % (
                    self._footprint(self.specs[req.key]), self.hbm_budget)
                req.t_done = time.perf_counter()
                self.completed.append(req)
                continue
            if eng is None or not eng.admit(req):
                waiting.append(req)
            elif req.done:  # refused by the engine (e.g. a state of the wrong size)
                self.completed.append(req)
        self.queue = waiting

    @property
    def idle(self):
        return not self.queue and not any(r.engine.busy or r.engine.pending
                                          for r in self.resident.values())

    def step(self):
        """One pass of the scheduling loop: admit, then for every resident
        engine complete its tick if the device has finished it (an event
        query, no wait) and enqueue its next tick.  Engines of different
        meshes and kinds advance at their own pace: a slow engine (a batch
        of quasidynamic RK23 attempts) does not hold back the Arnoldi steps
        of the others.  Returns the requests finished in this pass."""
        self._admit()
        done = []
        waiting = True

        def service(e):
            nonlocal waiting
            if e.pending and e.ready():
                done.extend(e.complete())
                waiting = False
            if not e.pending and e.busy:
                e.launch()
                waiting = False

        engines = [r.engine for r in self.resident.values()]
        # quasidynamic engines are chains of short RK23 attempts, each waiting
        # for the host to accept or reject the previous one: they are
        # serviced again after every other engine, so a finished attempt is
        # followed at once rather than after a whole pass over the solve
        # engines (whose host work is a millisecond or more each)
        quick = [e for e in engines if isinstance(e, QdEngine)]
        for e in engines:
            service(e)
            if not isinstance(e, QdEngine):
                for q in quick:
                    service(q)
        if waiting and done == []:
            time.sleep(20e-6)  # every engine is waiting for the device
        self.completed.extend(done)
        return done

    def run_until_idle(self, max_ticks=None):
        ticks = 0
        while not self.idle:
            self.step()
            ticks += 1
            if max_ticks is not None and ticks >= max_ticks:
                break
        return self.completed

    def replay(self, arrivals):
        """Serve a timed stream: arrivals = [(t_offset_s, key, rhs, tol)] for
        solves and [(t_offset_s, "qd", key, y0, n_steps)] for quasidynamic
        integrations, each submitted once the wall clock passes its offset
        (its latency is counted from the offset).  Returns the requests in
        arrival order."""
        arrivals = sorted(arrivals, key=lambda a: a[0])
        t0 = time.perf_counter()
        reqs = []
        i = 0
        while i < len(arrivals) or not self.idle:
            now = time.perf_counter() - t0
            while i < len(arrivals) and arrivals[i][0] <= now:
                a = arrivals[i]
                if len(a) == 5 and a[1] == "qd":
                    off, _, key, y0, n_steps = a
                    reqs.append(self.submit_qd(key, y0, n_steps, t_submit=t0 + off))
                else:
                    off, key, rhs, tol = a
                    reqs.append(self.submit(key, rhs, tol, t_submit=t0 + off))
                i += 1
            if self.idle:
                if i < len(arrivals):
                    time.sleep(max(0.0, min(arrivals[i][0] - now, 0.01)))
                continue
            self.step()
        return reqs
