"""Mass operator: block-diagonal Galerkin mass matrix J * int phi_a phi_b
(reference: tectosaur/ops/mass_op.py:9-42 and ops/_mass_op.cpp:11-40).

Entry (tri i, basis a, basis b, component d): row (3i + a) * tensor_dim + d,
col (3i + b) * tensor_dim + d, value J_i * sum_q w_q phi_a(q) phi_b(q).

On the device (the apply; the reference applies a scipy CSR on the host):
with tensor_dim = 3 the matrix is one 9x9 block per triangle on the
diagonal, stored as a DeviceBSR9 (one block row per triangle, the nearfield's
SoA layout) and applied by tct_bsr9_matvec, so sums with the integral
operators (SumOp([H, MultOp(MassOp, 0.5)]), examples/okada.py:354-358) stay
on the device; with tensor_dim = 1 (3x3 blocks) it is a device CSR applied
by tct_csr_matvec.  ``.mat`` (the host CSR, as the reference) is built in
the constructor; the device matrix on first use, once per precision.
"""
import numpy as np
import scipy.sparse

from ..util import device
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
        self.tensor_dim = tensor_dim
        self.n_tris = n_tris
        self._J = J
        self._bf = bf.reshape(3, 3)
        self._dev = {}

    # -- device matrix ----------------------------------------------------
    def device_matrix(self, float_type=np.float64):
        """The device form in float_type (cached): DeviceBSR9 for
        tensor_dim 3, DeviceCSR otherwise."""
        ft = np.dtype(float_type)
        if ft not in self._dev:
            if self.tensor_dim == 3:
                from ..util.sparse import DeviceBSR9
                n = self.n_tris
                # block element (3a + d, 3b + d') = J bf[a, b] delta(d, d')
                blk = np.kron(self._bf, np.eye(3))
                soa = np.outer(blk.reshape(81), self._J)  # element e of block i at [e, i]
                m = DeviceBSR9(self.shape, np.arange(n + 1), np.arange(n), ft,
                               data=device.to_dev(np.ascontiguousarray(soa.reshape(-1)), ft))
            else:
                from ..simple_solver import DeviceCSR
                m = DeviceCSR(self.mat)
            self._dev[ft] = m
        return self._dev[ft]

    def dot_device(self, x, y, accumulate=False, stream=None):
        """y (+)= M x on device tensors (FP32 or FP64, the matrix in x's
        precision)."""
        ft = np.float64 if x.dtype == device.torch().float64 else np.float32
        m = self.device_matrix(ft)
        if self.tensor_dim == 3:
            return m.matvec(x, y, accumulate=accumulate, stream=stream)
        return m.dot_device(x, y, accumulate=accumulate, stream=stream)

    def dot_panel_device(self, X, Y, accumulate=False, stream=None):
        """Y[r] (+)= M X[r] for device tensors X, Y (R, n)."""
        if self.tensor_dim == 3:
            ft = np.float64 if X.dtype == device.torch().float64 else np.float32
            return self.device_matrix(ft).matvec_panel(X, Y, accumulate=accumulate,
                                                       stream=stream)
        for r in range(X.shape[0]):
            self.dot_device(X[r], Y[r], accumulate=accumulate, stream=stream)
        return Y

    def dot(self, v):
        """M v on the device.  A host array comes back as float64 (as the
        reference's scipy product); a CUDA tensor stays on the device in its
        own precision."""
        if device.is_device_tensor(v):
            x = v.contiguous()
            if x.dtype not in (device.torch().float32, device.torch().float64):
                x = x.double()
            return self.dot_device(x, device.torch().empty_like(x))
        x = device.to_dev(np.asarray(v, dtype=np.float64).reshape(-1), np.float64)
        y = device.torch().empty_like(x)
        self.dot_device(x, y)
        return y.cpu().numpy()

    def nearfield_dot(self, v):
        return self.dot(v)

    def nearfield_no_correction_dot(self, v):
        return self.dot(v)

    def farfield_dot(self, v):
        shape = [self.shape[0]]
        shape.extend(v.shape[1:])
        return np.zeros(shape)
