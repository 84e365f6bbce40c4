"""Device-resident constrained GMRES (tectosaur_b200/simple_solver.py):
the CSR kernel against scipy, and solves whose residuals are checked with
the FP64 oracle operator (the reference's examples/solve.py:25-61 solve)."""
import numpy as np
import pytest
import scipy.sparse
import torch

from tectosaur_b200 import _lib
from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
from tectosaur_b200.ops.sparse_integral_op import RegularizedSparseIntegralOp
from tectosaur_b200.simple_solver import (DeviceCSR, free_edge_vertices, iterative_solve,
                                          shared_vertex_matrix)

from helpers import PARAMS, bumpy_mesh, oracle_sparse_op_dot

pytestmark = pytest.mark.gpu

NQS = (6, 6, 6, 2, 5, 2.5)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_csr_matvec_matches_scipy(cuda, dt):
    rng = np.random.default_rng(0)
    A = scipy.sparse.random(700, 500, density=0.01, random_state=1, format="csr")
    x = rng.standard_normal(500).astype(dt)
    m = DeviceCSR(A)
    xt = torch.from_numpy(x).cuda()
    y = torch.empty(700, dtype=xt.dtype, device="cuda")
    m.dot_device(xt, y)
    want = A @ x.astype(np.float64)
    tol = 1e-14 if dt == np.float64 else 1e-6
    assert np.linalg.norm(y.cpu().numpy() - want) <= tol * np.linalg.norm(want)
    m.dot_device(xt, y, accumulate=True)
    assert np.linalg.norm(y.cpu().numpy() - 2 * want) <= 2 * tol * np.linalg.norm(want)


def _op(pts, tris, ft, K="elasticRH3"):
    return RegularizedSparseIntegralOp(*NQS, K, K, PARAMS, pts, tris, ft,
                                       TriToTriDirectFarfieldOp)


def _oracle_apply(orc, pts, tris, v, K="elasticRH3"):
    return oracle_sparse_op_dot(orc, *NQS, K, K, PARAMS, pts, tris, np.float64, v)


def _cm(tris):
    # continuity + zero slip on the free edges (the hypersingular system on an
    # open surface is singular without the latter)
    return shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))


def test_constrained_solve_fp64(cuda, orc):
    pts, tris = bumpy_mesh(8, seed=3)
    cm = _cm(tris)
    rhs = np.random.default_rng(1).standard_normal(tris.shape[0] * 9)
    u = iterative_solve(_op(pts, tris, np.float64), cm, rhs, cfg=dict(solver_tol=1e-10))
    info = iterative_solve.last
    assert info["info"] == 0 and info["residuals"][-1] <= 1e-10
    # the solution is continuous and vanishes on the free edges
    corner = np.repeat(tris.reshape(-1), 3)
    fixed = np.isin(corner, free_edge_vertices(tris))
    assert np.all(u[fixed] == 0.0)
    assert np.allclose(cm @ (cm.T @ u / np.asarray(cm.sum(axis=0)).reshape(-1)), u, atol=1e-12)
    r = cm.T @ (_oracle_apply(orc, pts, tris, u) - rhs)
    assert np.linalg.norm(r) / np.linalg.norm(cm.T @ rhs) < 1e-8


def test_unconstrained_single_layer_solve_fp64(cuda, orc):
    # the single-layer (elasticU3) system is well posed without constraints
    pts, tris = bumpy_mesh(6, seed=4)
    rhs = np.random.default_rng(2).standard_normal(tris.shape[0] * 9)
    u = iterative_solve(_op(pts, tris, np.float64, "elasticU3"), None, rhs,
                        cfg=dict(solver_tol=1e-10))
    assert iterative_solve.last["info"] == 0
    r = _oracle_apply(orc, pts, tris, u, "elasticU3") - rhs
    assert np.linalg.norm(r) / np.linalg.norm(rhs) < 1e-8


def test_fp32_operator_solve_reaches_fp32_accuracy(cuda, orc):
    pts, tris = bumpy_mesh(8, seed=3)
    cm = _cm(tris)
    rhs = np.random.default_rng(1).standard_normal(tris.shape[0] * 9)
    u32 = iterative_solve(_op(pts, tris, np.float32), cm, rhs, cfg=dict(solver_tol=1e-5))
    u64 = iterative_solve(_op(pts, tris, np.float64), cm, rhs, cfg=dict(solver_tol=1e-10))
    assert np.linalg.norm(u32 - u64) / np.linalg.norm(u64) < 1e-3


def test_batched_mixed_precision_solves(cuda, orc):
    """16 right-hand sides solved together (FP32 tensor-core panel operator
    inside FP64 refinement) agree with the plain FP64 one-at-a-time solve,
    reach the FP64 residual bar, and a system's answer does not depend on the
    batch it is solved in."""
    from tectosaur_b200.simple_solver import iterative_solve_batch
    pts, tris = bumpy_mesh(8, seed=3)
    cm = _cm(tris)
    op64 = _op(pts, tris, np.float64)
    op32 = _op(pts, tris, np.float32)
    rhs = np.random.default_rng(4).standard_normal((16, tris.shape[0] * 9))
    U = iterative_solve_batch(op64, op32, cm, rhs, tol=1e-9)
    assert iterative_solve_batch.last["residuals"][-1] <= 1e-9
    for r in [0, 9]:
        u64 = iterative_solve(op64, cm, rhs[r], cfg=dict(solver_tol=1e-11))
        assert np.linalg.norm(U[r] - u64) / np.linalg.norm(u64) < 1e-7
        res = cm.T @ (_oracle_apply(orc, pts, tris, U[r]) - rhs[r])
        assert np.linalg.norm(res) / np.linalg.norm(cm.T @ rhs[r]) < 2e-9
    alone = iterative_solve_batch(op64, op32, cm, rhs[5:6], tol=1e-9)
    mixed = iterative_solve_batch(op64, op32, cm, np.concatenate([rhs[5:6], rhs[:3]]), tol=1e-9)
    assert np.linalg.norm(alone[0] - U[5]) / np.linalg.norm(U[5]) < 1e-7
    assert np.linalg.norm(mixed[0] - U[5]) / np.linalg.norm(U[5]) < 1e-7
