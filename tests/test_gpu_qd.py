"""Quasidynamic stepper on the device against the oracle (oracle/qd_oracle.py,
pinned to the reference's own newton.cpp / pt_average.cpp): the rate-state
Newton kernel, the vertex-average + aging-law kernel, the one-CTA CG mass
solve, the model's derivatives and a short RK23 integration."""
import os

import numpy as np
import pytest
import scipy.sparse
import torch

from tectosaur_b200 import _lib, qd
from tectosaur_b200.mesh.mesh_gen import make_rect
from tectosaur_b200.ops.mass_op import MassOp
from tectosaur_b200.qd.model import edge_ones_interior
from tectosaur_b200.simple_solver import free_edge_vertices, shared_vertex_matrix

from helpers import oracle_sparse_op
from oracle import qd_oracle

pytestmark = pytest.mark.gpu

QD = np.load(os.path.join(os.path.dirname(__file__), "golden", "qd.npz"))


def qd_cfg(n_tris, float_type=np.float64):
    return dict(sm=3e10, pr=0.25, density=2670.0, Dc=2e-6, f0=0.6, V0=1e-6,
                a=np.full(n_tris * 3, 0.010), b=np.full(n_tris * 3, 0.015), plate_rate=1e-9,
                additional_normal_stress=50e6, timestep_tol=1e-4,
                tectosaur_cfg=dict(quad_coincident_order=6, quad_edgeadj_order=6,
                                   quad_vertadj_order=6, quad_near_order=5,
                                   quad_near_threshold=2.5, quad_far_order=2, quad_mass_order=4,
                                   float_type=float_type, use_fmm=False))


def dev(a, dt=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dt)


@pytest.mark.parametrize("sep", [0, 1])
def test_rate_state_kernel(cuda, sep):
    n_tris = QD["in_tri_normals"].shape[0]
    V = torch.zeros((n_tris * 3, 3), dtype=torch.float64, device="cuda")
    failed = torch.zeros(1, dtype=torch.int32, device="cuda")
    keep = [dev(QD[k]) for k in ("in_tri_normals", "in_traction", "in_state", "in_a",
                                 "in_normal_stress")]
    _lib.check(_lib.lib.tct_qd_rate_state(
        n_tris, 3, _lib.tptr(keep[0]), _lib.tptr(keep[1]), _lib.tptr(keep[2]),
        _lib.tptr(keep[3]), float(QD["in_eta"]), float(QD["in_V0"]), float(QD["in_C"]),
        _lib.tptr(keep[4]), 1e-12, 50, sep, _lib.tptr(V), _lib.tptr(failed), None), "rate_state")
    got, want = V.cpu().numpy(), QD["V_sep%d" % sep]
    assert int(failed.item()) == 0
    zero = np.all(want == 0, axis=1)
    assert np.all(got[zero] == 0)
    rel = np.linalg.norm(got - want, axis=1)[~zero] / np.linalg.norm(want, axis=1)[~zero]
    assert rel.max() < 1e-12, rel.max()


@pytest.mark.parametrize("no_backslip", [0, 1])
def test_velocity_state_kernel(cuda, no_backslip):
    pts, tris = make_rect(6, 5, [[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]])
    n_dofs = tris.size
    rng = np.random.default_rng(5)
    vn = rng.standard_normal((n_dofs, 3)) * 1e-9
    state = rng.uniform(0.5, 0.8, n_dofs)
    b = rng.uniform(0.012, 0.018, n_dofs)
    ones = edge_ones_interior(tris)
    slipdir = np.array([1.0, 0.2, 0.0])
    interior = (ones.reshape(-1, 3) * slipdir).reshape(-1)
    full = np.tile(slipdir, n_dofs)
    edges = full - interior
    # oracle: the tail of model_helpers.rate_state_solve + the aging law
    avg = np.stack([qd_oracle.pt_average(pts.shape[0], tris, vn[:, d]) for d in range(3)], 1)
    if no_backslip:
        ii = interior.reshape(-1, 3)
        with np.errstate(invalid="ignore", divide="ignore"):
            speed = np.sum(avg * ii, axis=1) / np.linalg.norm(ii, axis=1)
        avg[speed < 0] = 0.0
        avg[np.isnan(speed)] = 0.0
    V_want = edges * 1e-9 + avg.reshape(-1)
    ds_want = qd_oracle.aging_law(b, 1e-6, 2e-6, 0.6, np.linalg.norm(V_want.reshape(-1, 3), axis=1),
                                  state)
    dof_vert = tris.reshape(-1)
    order = np.argsort(dof_vert, kind="stable")
    start = np.concatenate([[0], np.cumsum(np.bincount(dof_vert, minlength=pts.shape[0]))])
    a_ = [dev(x, torch.int32) for x in (start, order, dof_vert)]
    f_ = [dev(x) for x in (vn, edges, interior, state, b)]
    V = torch.empty(n_dofs * 3, dtype=torch.float64, device="cuda")
    ds = torch.empty(n_dofs, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib.tct_qd_velocity_state(
        n_dofs, *[_lib.tptr(x) for x in a_], _lib.tptr(f_[0]), _lib.tptr(f_[1]), _lib.tptr(f_[2]),
        1e-9, no_backslip, _lib.tptr(f_[3]), _lib.tptr(f_[4]), 1e-6, 2e-6, 0.6, _lib.tptr(V),
        _lib.tptr(ds), None), "velocity_state")
    np.testing.assert_allclose(V.cpu().numpy(), V_want, rtol=1e-13, atol=1e-25)
    np.testing.assert_allclose(ds.cpu().numpy(), ds_want, rtol=1e-12)


def test_cg_kernel(cuda):
    pts, tris = make_rect(9, 7, [[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]])
    cm = shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))
    M = (cm.T @ MassOp(4, pts, tris).mat @ cm).tocsr()
    M.sort_indices()
    n = M.shape[0]
    b = np.random.default_rng(2).standard_normal(n) * 1e7
    x_want, it_want = qd_oracle.cg(M, b, rtol=1e-5, atol=1e-12)
    d = [dev(M.indptr, torch.int64), dev(M.indices, torch.int64), dev(M.data), dev(b)]
    x = torch.empty(n, dtype=torch.float64, device="cuda")
    work = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    it = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(_lib.lib.tct_cg_csr(n, *[_lib.tptr(v) for v in d], _lib.tptr(x), _lib.tptr(work),
                                   1e-5, 1e-12, 10 * n, _lib.tptr(it), None), "cg")
    assert int(it.item()) == it_want
    np.testing.assert_allclose(x.cpu().numpy(), x_want, rtol=1e-10, atol=1e-12 * np.abs(x_want).max())


def test_cg_kernel_non_finite_rhs(cuda):
    # a non-finite right-hand side (an oversized trial step): the NaN
    # solution at once (scipy's cg returns NaN only after maxiter iterations)
    pts, tris = make_rect(9, 7, [[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]])
    cm = shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))
    M = (cm.T @ MassOp(4, pts, tris).mat @ cm).tocsr()
    M.sort_indices()
    n = M.shape[0]
    for bad in (np.nan, np.inf):
        b = np.random.default_rng(2).standard_normal(n)
        b[n // 2] = bad
        d = [dev(M.indptr, torch.int64), dev(M.indices, torch.int64), dev(M.data), dev(b)]
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        work = torch.empty(3 * n, dtype=torch.float64, device="cuda")
        it = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.check(_lib.lib.tct_cg_csr(n, *[_lib.tptr(v) for v in d], _lib.tptr(x),
                                       _lib.tptr(work), 1e-5, 1e-12, 10 * n, _lib.tptr(it), None),
                   "cg")
        assert int(it.item()) == -1
        assert np.all(np.isnan(x.cpu().numpy()))


def _pair(n=7, seed=0):
    pts, tris = make_rect(n, n, [[-1, 0, 1], [-1, 0, -1], [1, 0, -1], [1, 0, 1]])
    cfg = qd_cfg(tris.shape[0])
    model = qd.FullspaceModel((pts, tris), cfg)
    return pts, tris, cfg, model


def _oracle_model(orc, pts, tris, cfg, model):
    op = cfg["tectosaur_cfg"]
    H_dot = oracle_sparse_op(orc, op["quad_coincident_order"], op["quad_edgeadj_order"],
                             op["quad_vertadj_order"], op["quad_far_order"],
                             op["quad_near_order"], op["quad_near_threshold"], "elasticRH3",
                             [1.0, cfg["pr"]], pts, tris, np.float64)
    ones = edge_ones_interior(tris)
    cm_edges = scipy.sparse.diags(ones).tocsc()[:, ones > 0]
    cm = shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))
    return qd_oracle.FullspaceModel(pts, tris, cfg, H_dot, MassOp(4, pts, tris).mat, cm, cm_edges,
                                    model.tri_normals)


def test_model_derivs(cuda, orc):
    pts, tris, cfg, model = _pair()
    om = _oracle_model(orc, pts, tris, cfg, model)
    rng = np.random.default_rng(4)
    n = tris.shape[0]
    y = np.concatenate([rng.standard_normal(9 * n) * 1e-6, rng.uniform(0.6, 0.8, 3 * n)])
    for t in (0.0, 1e4):
        want = om.derivs(t, y)
        got = model.make_derivs()(t, torch.from_numpy(y).cuda()).cpu().numpy()
        assert model.newton_failures() == 0 and om.newton_failed == 0
        n9 = 9 * n
        rv = np.linalg.norm(got[:n9] - want[:n9]) / np.linalg.norm(want[:n9])
        rs = np.linalg.norm(got[n9:] - want[n9:]) / np.linalg.norm(want[n9:])
        assert rv < 1e-9 and rs < 1e-9, (rv, rs)
    # an invalid state: inf * y, as the reference's derivs returns
    y_bad = y.copy()
    y_bad[-1] = 1.5
    out = model.make_derivs()(0.0, torch.from_numpy(y_bad).cuda()).cpu().numpy()
    assert np.all(np.isinf(out[y_bad != 0])) and np.all(np.isinf(om.derivs(0.0, y_bad)[y_bad != 0]))


def test_integrate_matches_oracle(cuda, orc):
    from scipy.integrate import RK23
    pts, tris, cfg, model = _pair(6)
    om = _oracle_model(orc, pts, tris, cfg, model)
    n = tris.shape[0]
    rng = np.random.default_rng(8)
    y0 = np.concatenate([np.zeros(9 * n), 0.7 + 0.02 * rng.standard_normal(3 * n)])
    integ = qd.Integrator(model, (0.0, y0))
    ref = RK23(om.derivs, 0.0, y0, 1e50, atol=cfg["timestep_tol"], rtol=cfg["timestep_tol"])
    ref.h_abs = qd.siay / 10.0
    steps = 12
    integ.integrate(steps)
    for i in range(steps):
        assert ref.step() is None
        t_got, y_got = integ.h_t[i], integ.h_y[i].cpu().numpy()
        assert abs(t_got - ref.t) <= 1e-8 * abs(ref.t), (i, t_got, ref.t)
        assert np.linalg.norm(y_got - ref.y) <= 1e-8 * np.linalg.norm(ref.y), i


@pytest.mark.parametrize("ft", [np.float64, np.float32])
def test_graph_derivs_bit_identical(cuda, ft):
    """The single-state derivative replayed as a CUDA graph equals the eager
    evaluation bit for bit, over several times and states (a rejected one
    included), and the Integrator's trajectory with it is the eager one's."""
    pts, tris = make_rect(7, 7, [[-1, 0, 1], [-1, 0, -1], [1, 0, -1], [1, 0, 1]])
    cfg = qd_cfg(tris.shape[0], ft)
    model = qd.FullspaceModel((pts, tris), cfg)
    n = tris.shape[0]
    rng = np.random.default_rng(8)
    fg, fe = model.make_derivs(graph=True), model.make_derivs(graph=False)
    for k, t in enumerate((0.0, 3.3e3, 1e7, 2.5)):
        y = np.concatenate([rng.standard_normal(9 * n) * 1e-6, rng.uniform(0.6, 0.8, 3 * n)])
        if k == 3:
            y[-2] = 1.5  # rejected: inf * y
        yd = torch.from_numpy(y).cuda()
        a, b = fg(t, yd), fe(t, yd)
        torch.testing.assert_close(a, b, rtol=0, atol=0, equal_nan=True)
    y0 = np.concatenate([np.zeros(9 * n), 0.7 + 0.01 * rng.standard_normal(3 * n)])
    runs = []
    for graph in (True, False):
        integ = qd.Integrator(model, (0.0, y0))
        integ.derivs = model.make_derivs(graph=graph)
        integ.rk23.fun = integ.derivs
        integ.integrate(8)
        runs.append((list(integ.h_t), integ.h_y[-1].cpu().numpy()))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1])
