"""Host logic of the continuous-batching solve server (tectosaur_b200.serve)
on the CPU: the native Givens update against a numpy restatement, and the
scheduler (slots, refills between steps, per-slot stopping, mixed-precision
refinement, HBM admission and eviction) with dense CPU operators."""
import numpy as np
import pytest
import torch

from tectosaur_b200 import serve


def _givens_numpy(H, cs, sn, g, j, col):
    """One step of the Givens QR as in simple_solver.gmres."""
    H[: j + 2, j] = col
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
    return abs(g[j + 1])


def test_gmres_givens_matches_numpy():
    rng = np.random.default_rng(0)
    S, m = 5, 12
    H = np.zeros((S, m, m + 1))
    cs, sn, g = np.zeros((S, m)), np.zeros((S, m)), np.zeros((S, m + 1))
    g[:, 0] = rng.uniform(1, 2, S)
    Hn = np.zeros((S, m + 1, m))
    csn, snn, gn = cs.copy(), sn.copy(), g.copy()
    j = np.zeros(S, np.int64)
    for step in range(m):
        # systems advance at different rates: a subset takes a step
        active = np.flatnonzero((rng.random(S) < 0.7) & (j < m))
        if active.size == 0:
            continue
        cols = np.zeros((active.size, m + 2))
        for i, s in enumerate(active):
            cols[i, : j[s] + 2] = rng.standard_normal(j[s] + 2)
        res = serve._givens(active.astype(np.int64), j, m, cols, H, cs, sn, g)
        for i, s in enumerate(active):
            want = _givens_numpy(Hn[s], csn[s], snn[s], gn[s], j[s], cols[i, : j[s] + 2])
            assert res[i] == want
            j[s] += 1
    for s in range(S):
        np.testing.assert_array_equal(H[s].T, Hn[s])
    np.testing.assert_array_equal(g, gn)
    with pytest.raises(RuntimeError):
        jj = np.full(S, m, np.int64)  # step past the restart length
        serve._givens(np.array([0], np.int64), jj, m, np.zeros((1, m + 2)), H, cs, sn, g)


def _dense_problem(n, seed):
    rng = np.random.default_rng(seed)
    A = np.eye(n) * 4.0 + rng.standard_normal((n, n)) / np.sqrt(n)
    return A


def _cpu_builder(mats, nbytes):
    """builder(server, spec) making a CPU engine over the dense matrix
    mats[spec.key] (FP32-rounded for the inner operator)."""

    def build(server, spec):
        A = torch.from_numpy(mats[spec.key])
        A32 = A.float()

        def op64(V):
            return V @ A.T

        def op32(V):
            return (V.float() @ A32.T).double()

        eng = serve.SolveEngine(op32, op64, lambda r: r.clone(), lambda x: x.clone(),
                                A.shape[0], server.slots, server.restart, server.inner_tol,
                                server.max_refine, dev="cpu", stream=None)
        spec.measured_bytes = nbytes[spec.key]
        return serve._Resident(spec, None, None, eng, spec.measured_bytes)

    return build


def _server(mats, nbytes, budget, slots=4, restart=8):
    srv = serve.SolveServer(hbm_budget=budget, slots=slots, restart=restart, inner_tol=1e-4,
                            builder=_cpu_builder(mats, nbytes))
    for key, A in mats.items():
        n = A.shape[0]
        spec = srv.add_mesh(key, np.zeros((3, 3)), np.zeros((n // 9, 3), np.int64),
                            farfield_op_type=None)
        spec.measured_bytes = nbytes[key]
    return srv


def test_server_solves_and_refills_slots():
    mats = {"a": _dense_problem(45, 1)}
    srv = _server(mats, {"a": 100}, budget=1000, slots=3, restart=6)
    rng = np.random.default_rng(2)
    rhs = [rng.standard_normal(45) for _ in range(7)]
    tols = [1e-3] + [1e-10] * 6  # the first request stops early
    reqs = [srv.submit("a", b, tol=tl) for b, tl in zip(rhs[:5], tols)]
    # two ticks in, more requests arrive; they wait for slots, then join
    srv.step()
    srv.step()
    assert len(srv.queue) == 2
    reqs += [srv.submit("a", b, tol=tl) for b, tl in zip(rhs[5:], tols[5:])]
    srv.run_until_idle(max_ticks=10_000)
    assert srv.idle
    for r, b, tl in zip(reqs, rhs, tols):
        assert r.converged and r.error is None and r.residual <= tl
        want = np.linalg.solve(mats["a"], b)
        assert np.linalg.norm(r.x - want) / np.linalg.norm(want) < 10 * tl
    # restart 6 < the steps needed: several GMRES cycles and FP64 refinements
    assert all(r.refinements >= 2 for r in reqs[1:])
    # continuous batching: the slot freed by the early request was refilled
    # while the rest of its batch was still running
    assert reqs[0].t_done < reqs[3].t_admit < min(reqs[1].t_done, reqs[2].t_done)


def test_result_same_alone_and_in_mix():
    mats = {"a": _dense_problem(36, 3), "b": _dense_problem(54, 4)}
    nb = {"a": 10, "b": 10}
    rng = np.random.default_rng(5)
    target = rng.standard_normal(36)
    alone = _server(mats, nb, 100)
    r0 = alone.submit("a", target, tol=1e-9)
    alone.run_until_idle(max_ticks=10_000)
    mixed = _server(mats, nb, 100)
    others = [mixed.submit("b", rng.standard_normal(54), tol=1e-7) for _ in range(3)]
    mixed.step()
    r1 = mixed.submit("a", target, tol=1e-9)
    others += [mixed.submit("a", rng.standard_normal(36), tol=1e-6) for _ in range(4)]
    mixed.run_until_idle(max_ticks=10_000)
    assert r0.converged and r1.converged and all(o.converged for o in others)
    assert np.linalg.norm(r1.x - r0.x) / np.linalg.norm(r0.x) < 1e-12


def test_admission_and_eviction():
    mats = {"a": _dense_problem(27, 6), "b": _dense_problem(27, 7), "c": _dense_problem(18, 8)}
    nb = {"a": 60, "b": 60, "c": 500}
    srv = _server(mats, nb, budget=100, slots=2)
    rng = np.random.default_rng(9)
    ra = [srv.submit("a", rng.standard_normal(27), 1e-8) for _ in range(3)]
    rb = [srv.submit("b", rng.standard_normal(27), 1e-8) for _ in range(2)]
    srv.step()
    # "a" is resident and busy; "b" does not fit beside it and waits
    assert list(srv.resident) == ["a"] and all(r.t_admit is None for r in rb)
    srv.run_until_idle(max_ticks=10_000)
    assert all(r.converged for r in ra + rb)
    # "b" was admitted only after "a" went idle and was released
    assert min(r.t_admit for r in rb) >= max(r.t_done for r in ra[:2])
    assert srv.n_evictions >= 1 and srv.resident_bytes <= 100
    # a mesh larger than the whole budget is refused, not queued for ever
    rc = srv.submit("c", rng.standard_normal(18), 1e-8)
    srv.run_until_idle(max_ticks=100)
    assert rc.error is not None and rc.x is None and srv.idle
