"""Quasidynamic stepper, host side: the oracle (oracle/qd_oracle.py) pinned
bit for bit to the reference's own rate-state Newton solve and vertex
averaging (fixtures from qd/newton.cpp and qd/pt_average.cpp, compiled from
the reference sources), the RK23 restatement against scipy's RK23, the CG
restatement against scipy's cg, and the free-edge DOF field against the
reference's constraint builders."""
import numpy as np
import pytest
import scipy.sparse
import scipy.sparse.linalg
import torch
from scipy.integrate import RK23 as ScipyRK23

from tectosaur_b200.qd.model import edge_ones_interior
from tectosaur_b200.qd.rk23 import RK23

import os

from oracle import qd_oracle

QD = np.load(os.path.join(os.path.dirname(__file__), "golden", "qd.npz"))


def _inputs():
    return dict(tri_normals=QD["in_tri_normals"], traction=QD["in_traction"],
                state=QD["in_state"], a=QD["in_a"], eta=float(QD["in_eta"]),
                V0=float(QD["in_V0"]), C=float(QD["in_C"]), normal_stress=QD["in_normal_stress"])


@pytest.mark.parametrize("sep", [False, True])
def test_rate_state_oracle_bit_exact(sep):
    i = _inputs()
    V, failed = qd_oracle.rate_state_solver(i["tri_normals"], i["traction"], i["state"], i["a"],
                                            i["eta"], i["V0"], i["C"], i["normal_stress"],
                                            1e-12, 50, 3, sep)
    assert failed == 0
    np.testing.assert_array_equal(V, QD["V_sep%d" % int(sep)])
    if not sep:
        # zero traction -> zero velocity
        assert np.all(V[::7] == 0.0)


def test_pt_average_oracle_bit_exact():
    out = qd_oracle.pt_average(QD["avg_pts"].shape[0], QD["avg_tris"], QD["avg_field"])
    np.testing.assert_array_equal(out, QD["avg_out"])


def test_edge_ones_interior_matches_reference_constraints():
    np.testing.assert_array_equal(edge_ones_interior(QD["avg_tris"]), QD["edge_ones_interior"])


def test_rk23_restatement_matches_scipy():
    # a stiff nonlinear oscillator: many rejected steps
    def f_np(t, y):
        return np.array([y[1], -1000 * y[0] - 30 * y[1] * (y[0] ** 2 - 1) + np.sin(t)])

    def f_t(t, y):
        return torch.stack([y[1], -1000 * y[0] - 30 * y[1] * (y[0] ** 2 - 1) + np.sin(t)])

    y0 = np.array([1.0, 0.3])
    ref = ScipyRK23(f_np, 0.0, y0, 1e50, rtol=1e-4, atol=1e-4)
    ref.h_abs = 1e-3
    ours = RK23(f_t, 0.0, torch.tensor(y0), 1e50, rtol=1e-4, atol=1e-4, first_step=1e-3)
    for _ in range(300):
        assert ref.step() is None and ours.step() is None
        assert abs(ref.t - ours.t) <= 1e-11 * abs(ref.t)
        np.testing.assert_allclose(ours.y.numpy(), ref.y, rtol=1e-9, atol=1e-12)
    assert ours.n_rejected > 10
    # scipy's own initial step selection
    ref2 = ScipyRK23(f_np, 0.0, y0, 1e50, rtol=1e-4, atol=1e-4)
    ours2 = RK23(f_t, 0.0, torch.tensor(y0), 1e50, rtol=1e-4, atol=1e-4)
    assert abs(ref2.h_abs - ours2.h_abs) <= 1e-14 * ref2.h_abs


def test_rk23_rejects_infinite_derivatives():
    # derivatives that are infinite beyond t = 0.5 (the qd model's signal of
    # an invalid state): steps reaching past it are rejected as by scipy
    def f_np(t, y):
        return y * np.inf if t > 0.5 else -y

    def f_t(t, y):
        return y * float("inf") if t > 0.5 else -y

    ref = ScipyRK23(f_np, 0.0, np.array([1.0]), 1e50, rtol=1e-6, atol=1e-6)
    ref.h_abs = 0.01
    ours = RK23(f_t, 0.0, torch.tensor([1.0], dtype=torch.float64), 1e50, rtol=1e-6, atol=1e-6,
                first_step=0.01)
    for _ in range(30):  # to within 1e-7 of the boundary
        r1, r2 = ref.step(), ours.step()
        assert (r1 is None) == (r2 is None)
        if r1 is not None:
            break
        assert ours.t == pytest.approx(ref.t, rel=1e-10) and ours.t <= 0.5
    assert ours.n_rejected > 0


def test_cg_restatement_matches_scipy():
    rng = np.random.default_rng(3)
    n = 60
    M = scipy.sparse.random(n, n, density=0.1, random_state=4)
    A = (M @ M.T + scipy.sparse.identity(n) * 2.0).tocsr()
    b = rng.standard_normal(n)
    x, it = qd_oracle.cg(A, b, rtol=1e-5, atol=1e-12)
    count = []
    xs, info = scipy.sparse.linalg.cg(A, b, rtol=1e-5, atol=1e-12,
                                      callback=lambda xk: count.append(1))
    assert info == 0 and it == len(count)
    np.testing.assert_allclose(x, xs, rtol=1e-12, atol=1e-14)


def test_oracle_against_reference_module_if_built():
    import importlib.machinery
    import importlib.util
    base = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref")
    path = None
    for suf in importlib.machinery.EXTENSION_SUFFIXES:
        if os.path.exists(os.path.join(base, "newton" + suf)):
            path = os.path.join(base, "newton" + suf)
    if path is None:
        pytest.skip("reference newton module not built (make -C oracle ref)")
    spec = importlib.util.spec_from_file_location("newton", path)
    newton = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(newton)
    rng = np.random.default_rng(21)
    i = _inputs()
    tr = rng.standard_normal(i["traction"].shape) * 1e7
    st = rng.uniform(0.3, 0.9, tr.shape[0])
    V = np.zeros_like(tr)
    newton.rate_state_solver(i["tri_normals"], tr, st, V, i["a"], i["eta"], i["V0"], i["C"],
                             i["normal_stress"], 1e-12, 50, 3, False)
    Vo, _ = qd_oracle.rate_state_solver(i["tri_normals"], tr, st, i["a"], i["eta"], i["V0"],
                                        i["C"], i["normal_stress"], 1e-12, 50)
    np.testing.assert_array_equal(V, Vo)
