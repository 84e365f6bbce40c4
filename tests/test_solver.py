"""GMRES of the constrained solve (tectosaur_b200/simple_solver.py): the
algorithm on CPU tensors against dense solves and scipy; the continuity
matrix against its definition."""
import numpy as np
import pytest
import scipy.sparse.linalg
import torch

from tectosaur_b200.simple_solver import free_edge_vertices, gmres, shared_vertex_matrix


def _system(n=160, seed=0):
    rng = np.random.default_rng(seed)
    A = np.eye(n) + 0.4 * rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal(n)
    return A, b


@pytest.mark.parametrize("restart", [200, 25, 7])
def test_gmres_solves_dense_system(restart):
    A, b = _system()
    At = torch.from_numpy(A)
    x, info, n_iter, hist = gmres(lambda v: At @ v, torch.from_numpy(b), tol=1e-11,
                                  restart=restart)
    assert info == 0 and hist[-1] <= 1e-11
    xs = np.linalg.solve(A, b)
    assert np.linalg.norm(x.numpy() - xs) / np.linalg.norm(xs) < 1e-9
    assert np.linalg.norm(A @ x.numpy() - b) / np.linalg.norm(b) < 2e-11


def test_gmres_iterations_match_scipy():
    A, b = _system(seed=1)
    At = torch.from_numpy(A)
    _, _, n_iter, _ = gmres(lambda v: At @ v, torch.from_numpy(b), tol=1e-8, restart=200)
    count = [0]

    def cb(_):
        count[0] += 1
    xs, info = scipy.sparse.linalg.gmres(A, b, rtol=1e-8, restart=200, callback=cb,
                                         callback_type="pr_norm")
    assert info == 0
    assert abs(n_iter - count[0]) <= 1


def test_gmres_right_preconditioner():
    rng = np.random.default_rng(2)
    n = 120
    d = np.exp(rng.uniform(-3, 3, n))
    A = np.diag(d) + 0.05 * rng.standard_normal((n, n))
    b = rng.standard_normal(n)
    At = torch.from_numpy(A)
    Minv = torch.from_numpy(1.0 / d)
    x, info, it_p, _ = gmres(lambda v: At @ v, torch.from_numpy(b), tol=1e-10,
                             M=lambda v: Minv * v)
    _, _, it_0, _ = gmres(lambda v: At @ v, torch.from_numpy(b), tol=1e-10)
    assert info == 0 and it_p < it_0
    assert np.linalg.norm(A @ x.numpy() - b) / np.linalg.norm(b) < 1e-9


def test_gmres_zero_rhs_and_maxiter():
    A, b = _system(n=50)
    At = torch.from_numpy(A)
    x, info, n, _ = gmres(lambda v: At @ v, torch.zeros(50, dtype=torch.float64))
    assert info == 0 and n == 0 and float(x.abs().max()) == 0.0
    x, info, n, _ = gmres(lambda v: At @ v, torch.from_numpy(b), tol=1e-14, maxiter=5)
    assert info == 5 and n == 5


def test_shared_vertex_matrix():
    tris = np.array([[0, 1, 2], [2, 1, 3], [3, 4, 2]])
    cm = shared_vertex_matrix(tris).toarray()
    assert cm.shape == (27, 15)
    assert np.all(cm.sum(axis=1) == 1)
    # DOF of corner c, component d of triangle i maps to column 3 * vertex + d
    for i in range(3):
        for c in range(3):
            for d in range(3):
                assert cm[9 * i + 3 * c + d, 3 * tris[i, c] + d] == 1


def test_free_edges_and_fixed_vertices():
    from tectosaur_b200.mesh.mesh_gen import make_rect
    pts, tris = make_rect(5, 4, [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]])
    fv = free_edge_vertices(tris)
    on_boundary = np.nonzero((pts[:, 0] % 1 == 0) | (pts[:, 1] % 1 == 0))[0]
    assert np.array_equal(fv, on_boundary)
    cm = shared_vertex_matrix(tris, fixed_vertices=fv)
    n_interior = pts.shape[0] - fv.size
    assert cm.shape == (tris.shape[0] * 9, 3 * n_interior)
    rows_hit = np.asarray(cm.sum(axis=1)).reshape(-1)
    corner_vert = np.repeat(tris.reshape(-1), 3)
    assert np.all(rows_hit[np.isin(corner_vert, fv)] == 0)
    assert np.all(rows_hit[~np.isin(corner_vert, fv)] == 1)


def test_gmres_batch_matches_single_solves():
    from tectosaur_b200.simple_solver import gmres_batch
    rng = np.random.default_rng(7)
    n, R = 120, 5
    As = [np.eye(n) + 0.35 * rng.standard_normal((n, n)) / np.sqrt(n) for _ in range(R)]
    # one operator for all systems (as in the solve), different right-hand sides
    A = torch.from_numpy(As[0])
    B = torch.from_numpy(rng.standard_normal((R, n)))
    B[3] = 0.0  # a zero right-hand side converges at once
    X, info, n_it = gmres_batch(lambda V: V @ A.T, B, tol=1e-11, restart=20)
    assert np.all(info == 0)
    for r in range(R):
        want = np.linalg.solve(As[0], B[r].numpy())
        assert np.linalg.norm(X[r].numpy() - want) <= 1e-9 * max(np.linalg.norm(want), 1e-300)
    assert float(X[3].abs().max()) == 0.0
