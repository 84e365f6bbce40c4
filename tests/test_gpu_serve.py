"""The continuous-batching solve server on the device: served results
against the plain FP64 one-solve-at-a-time path (simple_solver.
iterative_solve), and a request's result alone against the same request in
a mix of meshes and right-hand sides."""
import numpy as np
import pytest

from tectosaur_b200 import _lib, serve
from tectosaur_b200.mesh.mesh_gen import make_rect
from tectosaur_b200.simple_solver import (free_edge_vertices, iterative_solve,
                                          shared_vertex_matrix)

from helpers import PARAMS, bumpy_mesh

pytestmark = pytest.mark.gpu

NQ = (6, 6, 6, 2, 5, 2.5)


def _meshes():
    a = make_rect(10, 10, [[-1, -1, 0], [-1, 1, 0], [1, 1, 0], [1, -1, 0]])
    b = bumpy_mesh(9, seed=2)
    return {k: (np.asarray(p), np.asarray(t)) for k, (p, t) in {"fault": a, "surface": b}.items()}


def _server(meshes):
    srv = serve.SolveServer(slots=16, restart=64)
    for k, (pts, tris) in meshes.items():
        cm = shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))
        srv.add_mesh(k, pts, tris, cm, nq=NQ, params=PARAMS)
    return srv


def test_served_matches_plain_fp64(cuda):
    meshes = _meshes()
    srv = _server(meshes)
    rng = np.random.default_rng(0)
    reqs = []
    for i in range(6):
        k = "fault" if i % 2 == 0 else "surface"
        reqs.append(srv.submit(k, rng.standard_normal(9 * meshes[k][1].shape[0]), tol=1e-8))
    n0 = _lib.launch_count()
    srv.run_until_idle(max_ticks=20_000)
    assert _lib.launch_count() > n0  # the library's kernels ran
    for k in meshes:
        r = srv.resident[k]
        assert r.op32.farfield.panel_supported()  # the tensor-core panel path
    for r in reqs:
        assert r.converged and r.residual <= 1e-8, (r.residual, r.error)
        op64 = srv.resident[r.key].op64
        pts, tris = meshes[r.key]
        cm = shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))
        want = iterative_solve(op64, cm, r.rhs, cfg=dict(solver_tol=1e-10))
        assert np.linalg.norm(r.x - want) / np.linalg.norm(want) < 1e-6


def test_same_alone_and_in_mix(cuda):
    meshes = _meshes()
    rng = np.random.default_rng(1)
    target = rng.standard_normal(9 * meshes["fault"][1].shape[0])
    alone = _server(meshes)
    r0 = alone.submit("fault", target, tol=1e-8)
    alone.run_until_idle(max_ticks=20_000)
    mixed = _server(meshes)
    for _ in range(5):
        mixed.submit("surface", rng.standard_normal(9 * meshes["surface"][1].shape[0]), 1e-8)
    mixed.step()
    mixed.submit("fault", rng.standard_normal(target.shape[0]), 1e-6)
    mixed.step()
    r1 = mixed.submit("fault", target, tol=1e-8)
    for _ in range(4):
        mixed.submit("fault", rng.standard_normal(target.shape[0]), 1e-7)
    mixed.run_until_idle(max_ticks=20_000)
    assert r0.converged and r1.converged
    assert all(r.converged for r in mixed.completed)
    assert np.linalg.norm(r1.x - r0.x) / np.linalg.norm(r0.x) < 1e-9


def _qd_setup(ft=np.float64, n=6):
    from tectosaur_b200 import qd
    pts, tris = make_rect(n, n, [[-1, 0, 1], [-1, 0, -1], [1, 0, -1], [1, 0, 1]])
    nt = tris.shape[0]
    cfg = dict(sm=3e10, pr=0.25, density=2670.0, Dc=2e-6, f0=0.6, V0=1e-6,
               a=np.full(nt * 3, 0.010), b=np.full(nt * 3, 0.015), plate_rate=1e-9,
               additional_normal_stress=50e6, timestep_tol=1e-4,
               tectosaur_cfg=dict(quad_coincident_order=6, quad_edgeadj_order=6,
                                  quad_vertadj_order=6, quad_near_order=5,
                                  quad_near_threshold=2.5, quad_far_order=2,
                                  quad_mass_order=4, float_type=ft, use_fmm=False))
    model = qd.FullspaceModel((pts, tris), cfg)
    rng = np.random.default_rng(3)
    y0s = [np.concatenate([np.zeros(9 * nt), 0.7 + 0.01 * rng.standard_normal(3 * nt)])
           for _ in range(3)]
    return pts, tris, cfg, model, y0s


def test_qd_served_matches_integrator(cuda):
    from tectosaur_b200 import qd
    pts, tris, cfg, model, y0s = _qd_setup()
    steps = 15
    integ = qd.Integrator(model, (0.0, y0s[0]))
    integ.integrate(steps)
    srv = serve.SolveServer(slots=4)
    srv.add_qd_mesh("fault", pts, tris, cfg, model=model)
    req = srv.submit_qd("fault", y0s[0], steps)
    n0 = _lib.launch_count()
    srv.run_until_idle(max_ticks=10_000)
    assert _lib.launch_count() > n0
    assert req.converged and req.steps == steps and req.error is None
    np.testing.assert_allclose(req.ts, integ.h_t, rtol=1e-10)
    want = integ.h_y[-1].cpu().numpy()
    assert np.linalg.norm(req.y - want) / np.linalg.norm(want) < 1e-10


def test_qd_same_alone_and_in_mix(cuda):
    pts, tris, cfg, model, y0s = _qd_setup(np.float32)
    alone = serve.SolveServer(slots=4)
    alone.add_qd_mesh("fault", pts, tris, cfg, model=model)
    r0 = alone.submit_qd("fault", y0s[0], 12)
    alone.run_until_idle(max_ticks=10_000)
    mixed = serve.SolveServer(slots=4)
    mixed.add_qd_mesh("fault", pts, tris, cfg, model=model)
    others = [mixed.submit_qd("fault", y0s[1], 20)]
    mixed.step()
    r1 = mixed.submit_qd("fault", y0s[0], 12)
    others.append(mixed.submit_qd("fault", y0s[2], 5))
    mixed.run_until_idle(max_ticks=10_000)
    assert r0.converged and r1.converged and all(o.converged for o in others)
    assert r1.steps == r0.steps == 12
    np.testing.assert_allclose(r1.ts, r0.ts, rtol=1e-9)
    # a pending tick's step sizes stay on the host: its completion reads
    # them per slot, and a device scalar there would be a blocking copy
    srv = serve.SolveServer(slots=4)
    srv.add_qd_mesh("fault", pts, tris, cfg, model=model)
    srv.submit_qd("fault", y0s[0], 3)
    srv.step()
    eng = srv.resident["fault"].engine
    assert eng.pending and isinstance(eng._pending[1], np.ndarray)
    srv.run_until_idle(max_ticks=10_000)
    assert np.linalg.norm(r1.y - r0.y) / np.linalg.norm(r0.y) < 1e-9


def _elementwise_derivs(model, ts, Y):
    """The batched derivative as element-wise tensor operations (deficit,
    -H D through the constrained mass solve, rate-state, rejection)."""
    import torch as t
    n9 = 9 * model.n_tris
    slip, state = Y[:, :n9], Y[:, n9:]
    plate = (ts[:, None] * model.cfg["plate_rate"]) * model.d_inslipdir[None, :]
    deficit = model.d_interior[None, :] * (plate - slip)
    X = deficit.to(model.H_dtype).contiguous()
    Yh = t.empty_like(X)
    model._panel(X, Yh)
    rhs = (-Yh).to(t.float64)
    R = Y.shape[0]
    rc = t.empty((R, model.n_free), dtype=t.float64, device="cuda")
    model._csr_panel(model.cmT, rhs, rc)
    soln = t.empty_like(rc)
    work = t.empty(3 * max(model.n_free, 1) * R, dtype=t.float64, device="cuda")
    iters = t.empty(R, dtype=t.int32, device="cuda")
    ip, ix, dv = model.mass_c
    _lib.check(_lib.lib.tct_cg_csr_batch(
        model.n_free, R, _lib.tptr(ip), _lib.tptr(ix), _lib.tptr(dv), _lib.tptr(rc),
        rc.stride(0), _lib.tptr(soln), soln.stride(0), _lib.tptr(work), 1e-5, 1e-12,
        10 * model.n_free, _lib.tptr(iters), _lib.stream_ptr()), "cg")
    traction = t.empty((R, n9), dtype=t.float64, device="cuda")
    model._csr_panel(model.cm, soln, traction)
    traction *= model.cfg["sm"]
    V, dstate = model.rate_state_solve_batch(traction, state)
    bad = (~t.isfinite(Y).all(dim=1)) | (state < 0).any(dim=1) | (state > 1.2).any(dim=1) | \
        (~t.isfinite(V).all(dim=1))
    return t.where(bad[:, None], Y * float("inf"), t.cat((V, dstate), dim=1))


@pytest.mark.parametrize("ft", [np.float64, np.float32])
def test_fused_derivs_batch_bit_identical(cuda, ft):
    """derivs_batch's fused deficit / rejection kernels and the sign folded
    into the traction scale give the element-wise computation bit for bit,
    rejected rows (a NaN, a state above 1.2, a negative state) included."""
    import torch as t
    pts, tris, cfg, model, y0s = _qd_setup(ft)
    nt = tris.shape[0]
    rng = np.random.default_rng(5)
    Y = np.stack([np.concatenate([1e-3 * rng.standard_normal(9 * nt),
                                  0.7 + 0.05 * rng.standard_normal(3 * nt)]) for _ in range(5)])
    Y[1, 3] = np.nan
    Y[2, 9 * nt + 4] = 1.3
    Y[3, 9 * nt] = -0.1
    Yd = t.from_numpy(Y).cuda()
    ts = t.from_numpy(rng.uniform(0, 1e7, 5)).cuda()
    got = model.derivs_batch(ts, Yd)
    want = _elementwise_derivs(model, ts, Yd)
    t.testing.assert_close(got, want, rtol=0, atol=0, equal_nan=True)
    assert t.isinf(got[2]).any() and t.isinf(got[3]).any() and not t.isfinite(got[1]).all()
    assert t.isfinite(got[0]).all() and t.isfinite(got[4]).all()


def test_fused_rk_combinations(cuda):
    """The RK23 stage combinations bit for bit against their element-wise
    expressions; the error norm to rounding."""
    import torch as t
    from tectosaur_b200.qd import model as qm, rk23 as rk
    rng = np.random.default_rng(6)
    R, n = 7, 3001
    y, K0, K1, K2, f = [t.from_numpy(rng.standard_normal((R, n))).cuda() for _ in range(5)]
    K1[2, 7] = float("inf")
    h = t.from_numpy(rng.uniform(1e-3, 1e3, R)).cuda()
    hd = h[:, None]
    out = t.empty_like(y)
    cases = [([K0], [rk.A[1][0]], y + (K0 * rk.A[1][0]) * hd),
             ([K0, K1], [rk.A[2][0], rk.A[2][1]], y + (K0 * rk.A[2][0] + K1 * rk.A[2][1]) * hd),
             ([K0, K1, K2], rk.B[:3], y + hd * (K0 * rk.B[0] + K1 * rk.B[1] + K2 * rk.B[2]))]
    for Ks, cs, want in cases:
        qm.combine_batch(Ks, cs, h, y, out)
        t.testing.assert_close(out, want, rtol=0, atol=0, equal_nan=True)
    qm.combine_batch([K0, K2], [0.3, -0.7], h, None, out)
    t.testing.assert_close(out, (K0 * 0.3 + K2 * -0.7) * hd, rtol=0, atol=0)
    y_new = y + 0.01 * K2
    tol = 1e-4
    err = (K0 * rk.E[0] + K1 * rk.E[1] + K2 * rk.E[2] + f * rk.E[3]) * hd
    scale = tol + t.maximum(y.abs(), y_new.abs()) * tol
    want = t.linalg.norm(err / scale, dim=1)
    norms = t.empty(R, dtype=t.float64, device="cuda")
    qm.error_norm_batch([K0, K1, K2, f], rk.E[:4], h, y, y_new, tol, norms)
    assert not t.isfinite(norms[2]) and not t.isfinite(want[2])
    ok = t.arange(R, device="cuda") != 2
    t.testing.assert_close(norms[ok], want[ok], rtol=1e-13, atol=0)
