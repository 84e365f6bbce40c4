"""Mass operator: block-diagonal Galerkin mass matrix J * int phi_a phi_b
(reference: tectosaur/ops/mass_op.py:9-42 and ops/_mass_op.cpp:11-40).

Entry (tri i, basis a, basis b, component d): row (3i + a) * tensor_dim + d,
col (3i + b) * tensor_dim + d, value J_i * sum_q w_q phi_a(q) phi_b(q).
"""
import numpy as np
import scipy.sparse

from ..util.quadrature import gauss2d_tri


def unscaled_normals(tri_pts):
    return np.cross(tri_pts[:, 2, :] - tri_pts[:, 0, :], tri_pts[:, 2, :] - tri_pts[:, 1, :])


def jacobians(unscaled_normals):
    return np.linalg.norm(unscaled_normals, axis=1)


def linear_basis_tri_arr(pts):
    return np.array([1 - pts[:, 0] - pts[:, 1], pts[:, 0], pts[:, 1]]).T


class MassOp:
    def __init__(self, nq, pts, tris, tensor_dim=3):
        qx, qw = gauss2d_tri(nq)
        tri_pts = np.asarray(pts)[np.asarray(tris)]
        basis = linear_basis_tri_arr(qx)
        J = jacobians(unscaled_normals(tri_pts))
        bf = np.array([np.sum(qw * (basis[:, b1] * basis[:, b2]))
                       for b1 in range(3) for b2 in range(3)])
        n_tris = tri_pts.shape[0]
        i = np.arange(n_tris)[:, None, None, None]
        b1 = np.arange(3)[None, :, None, None]
        b2 = np.arange(3)[None, None, :, None]
        d = np.arange(tensor_dim)[None, None, None, :]
        shape4 = (n_tris, 3, 3, tensor_dim)
        rows = np.broadcast_to((i * 3 + b1) * tensor_dim + d, shape4).reshape(-1)
        cols = np.broadcast_to((i * 3 + b2) * tensor_dim + d, shape4).reshape(-1)
        vals = np.broadcast_to(J[:, None, None, None] * bf.reshape(3, 3)[None, :, :, None],
                               shape4).reshape(-1)
        n_rows = n_tris * 3 * tensor_dim
        self.shape = (n_rows, n_rows)
        self.mat = scipy.sparse.csr_matrix((vals, (rows, cols)), shape=self.shape)

    def dot(self, v):
        return self.mat.dot(v)

    def nearfield_dot(self, v):
        return self.dot(v)

    def nearfield_no_correction_dot(self, v):
        return self.dot(v)

    def farfield_dot(self, v):
        shape = [self.shape[0]]
        shape.extend(v.shape[1:])
        return np.zeros(shape)
