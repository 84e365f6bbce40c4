"""Interior evaluation: a boundary field's kernel integral at observation
points off the surface or at its vertices (reference: tectosaur/interior.py).

InteriorOp(obs_pts, obs_ns, src_mesh, K_name, threshold, nq_vertex, nq_far,
nq_near, params, float_type).dot(v) =
    far(v)                       all triangles, gauss2d_tri(nq_far), on the
                                 device (tct_farfield_tris_to_pts)
  + near(v) - near_far(v)        point-triangle pairs within 4 radii (the
                                 reference fixes the threshold at 4.0,
                                 interior.py:31), integrated with
                                 gauss2d_tri(nq_near) minus the same pairs
                                 with the farfield rule (tct_interior_pairs)
  + vertex(v)                    pairs whose point is a triangle vertex:
                                 the closed-form radial integral of
                                 elasticH3 (tct_interior_corners, as the
                                 reference's interior_corners.cl whatever
                                 the kernel)
The three pair terms are assembled once into one device CSR matrix of FP64
entries (rows obs * 3 + d, columns tri * 9 + b * 3 + d) and applied with
tct_csr_matvec; the far term is recomputed per apply.
"""
import numpy as np
import scipy.sparse

from . import _lib
from .kernels import kernels
from .mesh import find_near_adj
from .simple_solver import DeviceCSR
from .util import device
from .util.quadrature import gauss2d_tri, gaussxw, map_to


def make_pairs_mat(pairs, entries, shape):
    """CSR of (n, 3, 3, 3) pair entries (interior.py:13-26)."""
    pairs = np.asarray(pairs).reshape(-1, 3)
    n = pairs.shape[0]
    rows = np.broadcast_to((pairs[:, 0][:, None, None] * 3 + np.arange(3)[None, :, None]),
                           (n, 3, 9))
    cols = np.broadcast_to((pairs[:, 1][:, None, None] * 9 + np.arange(9)[None, None, :]),
                           (n, 3, 9))
    return scipy.sparse.csr_matrix(
        (np.asarray(entries).reshape(n, 3, 9).ravel(), (rows.ravel(), cols.ravel())),
        shape=shape)


class TriToPtDirectFarfieldOp:
    """Direct farfield from source triangles to points (interior.py:131-185)."""

    def __init__(self, obs_pts, obs_ns, src_mesh, K_name, nq, params, float_type):
        self.K_name = K_name
        self.kid = _lib.kernel_id(K_name)
        self.float_type = np.dtype(float_type)
        self.prec = _lib.prec_of(float_type)
        obs_pts = np.asarray(obs_pts, np.float64)
        self.n_obs = obs_pts.shape[0]
        self.n_src = np.asarray(src_mesh[1]).shape[0]
        self.tensor_dim = kernels[K_name].tensor_dim
        self.shape = (self.n_obs * 3, self.n_src * 9)
        self.q = gauss2d_tri(nq)
        self.qx = np.ascontiguousarray(self.q[0], np.float64)
        self.qw = np.ascontiguousarray(self.q[1], np.float64)
        self.gpu_obs_pts = device.to_dev(obs_pts, self.float_type)
        self.gpu_obs_ns = device.to_dev(np.asarray(obs_ns, np.float64), self.float_type)
        self.gpu_src_pts = device.to_dev(np.asarray(src_mesh[0], np.float64), self.float_type)
        self.gpu_src_tris = device.to_dev(np.asarray(src_mesh[1]), np.int32)
        self.params = np.ascontiguousarray(np.asarray(params, np.float64)[:2])
        self.ws_bytes = _lib.lib.tct_farfield_tris_to_pts_workspace_bytes(
            self.prec, self.n_obs, self.n_src, self.qx.shape[0])
        self.workspace = device.workspace(self.ws_bytes)

    def dot_device(self, x, y, stream=None):
        _lib.check(_lib.lib.tct_farfield_tris_to_pts(
            self.kid, self.prec, _lib.tptr(y), _lib.tptr(x), _lib.tptr(self.gpu_obs_pts),
            _lib.tptr(self.gpu_obs_ns), self.n_obs, _lib.tptr(self.gpu_src_pts),
            _lib.tptr(self.gpu_src_tris), self.n_src, self.qx.shape[0], _lib.dptr(self.qx),
            _lib.dptr(self.qw), _lib.dptr(self.params), _lib.tptr(self.workspace), self.ws_bytes,
            _lib.stream_ptr(stream)), "tct_farfield_tris_to_pts")
        return y

    def dot(self, v):
        x = device.to_dev(np.asarray(v).reshape(-1), self.float_type)
        y = device.empty(max(self.shape[0], 1), self.float_type)
        self.dot_device(x, y)
        return y[: self.shape[0]].cpu().numpy()


def interior_pairs_quad(K_name, pairs, quad, far, float_type, finite_part=False):
    """(n, 3, 3, 3) point-triangle integrals on the device
    (interior.py:105-127)."""
    pairs = np.ascontiguousarray(np.asarray(pairs).reshape(-1, 3), dtype=np.int32)
    n = pairs.shape[0]
    if n == 0:
        return np.zeros((0, 3, 3, 3))
    ft = np.dtype(float_type)
    out = device.empty(n * 27, ft)
    qp = device.to_dev(np.ascontiguousarray(quad[0]), ft)
    qw = device.to_dev(np.ascontiguousarray(quad[1]), ft)
    pl = device.to_dev(pairs, np.int32)
    _lib.check(_lib.lib.tct_interior_pairs(
        _lib.kernel_id(K_name), _lib.prec_of(ft), _lib.tptr(out), qw.shape[0], _lib.tptr(qp),
        _lib.tptr(qw), _lib.tptr(far.gpu_obs_pts), _lib.tptr(far.gpu_obs_ns),
        _lib.tptr(far.gpu_src_pts), _lib.tptr(far.gpu_src_tris), _lib.tptr(pl), n,
        _lib.dptr(far.params), int(bool(finite_part)), _lib.stream_ptr()), "tct_interior_pairs")
    return out.cpu().numpy().reshape(n, 3, 3, 3)


def interior_corners_quad(pairs, quad, far, float_type):
    pairs = np.ascontiguousarray(np.asarray(pairs).reshape(-1, 3), dtype=np.int32)
    n = pairs.shape[0]
    if n == 0:
        return np.zeros((0, 3, 3, 3))
    ft = np.dtype(float_type)
    out = device.empty(n * 27, ft)
    qt = device.to_dev(np.ascontiguousarray(quad[0]), ft)
    qw = device.to_dev(np.ascontiguousarray(quad[1]), ft)
    pl = device.to_dev(pairs, np.int32)
    _lib.check(_lib.lib.tct_interior_corners(
        _lib.prec_of(ft), _lib.tptr(out), qt.shape[0], _lib.tptr(qt), _lib.tptr(qw),
        _lib.tptr(far.gpu_obs_ns), _lib.tptr(far.gpu_src_pts), _lib.tptr(far.gpu_src_tris),
        _lib.tptr(pl), n, _lib.dptr(far.params), _lib.stream_ptr()), "tct_interior_corners")
    return out.cpu().numpy().reshape(n, 3, 3, 3)


class InteriorOp:
    def __init__(self, obs_pts, obs_ns, src_mesh, K_name, threshold, nq_vertex, nq_far,
                 nq_near, params, float_type):
        device.require_cuda()
        self.K_name = K_name
        self.float_type = np.dtype(float_type)
        # the reference replaces the threshold argument by 4.0 (interior.py:31)
        self.threshold = 4.0
        obs_pts = np.asarray(obs_pts, np.float64)
        src_pts, src_tris = np.asarray(src_mesh[0], np.float64), np.asarray(src_mesh[1])
        pairs = find_near_adj.get_nearfield(
            obs_pts, np.zeros(obs_pts.shape[0]),
            *find_near_adj.get_tri_centroids_rs(src_pts, src_tris), self.threshold)
        self.vertex_pairs, self.near_pairs = find_near_adj.split_vertex_nearfield(
            pairs, obs_pts, src_pts, src_tris)
        self.all_near_pairs = np.vstack((self.near_pairs, self.vertex_pairs))
        self.all_near_pairs[:, 2] = 0
        self.farfield = TriToPtDirectFarfieldOp(obs_pts, obs_ns, (src_pts, src_tris), K_name,
                                                nq_far, params, float_type)
        shape = self.farfield.shape
        self.shape = shape
        near = interior_pairs_quad(K_name, self.near_pairs, gauss2d_tri(nq_near),
                                   self.farfield, float_type)
        corr = interior_pairs_quad(K_name, self.all_near_pairs, gauss2d_tri(nq_far),
                                   self.farfield, float_type)
        vert = interior_corners_quad(self.vertex_pairs,
                                     map_to(gaussxw(nq_vertex), [0.0, np.pi / 2]),
                                     self.farfield, float_type)
        self.near_mat = make_pairs_mat(self.near_pairs, near, shape)
        self.near_mat_correction = make_pairs_mat(self.all_near_pairs, corr, shape)
        self.vertex_mat = make_pairs_mat(self.vertex_pairs, vert, shape)
        self._pairs = DeviceCSR(self.near_mat - self.near_mat_correction + self.vertex_mat)
        t = device.torch()
        self._x = t.zeros(shape[1], dtype=device.torch_dtype(float_type), device="cuda")
        self._yf = t.zeros(max(shape[0], 1), dtype=device.torch_dtype(float_type), device="cuda")

    def dot_device(self, v, y=None):
        """far(v) + (near - near_far + vertex) v on device tensors (FP64 out)."""
        t = device.torch()
        v64 = v.to(t.float64).contiguous()
        self._x.copy_(v64)
        self.farfield.dot_device(self._x, self._yf)
        if y is None:
            y = t.empty(self.shape[0], dtype=t.float64, device="cuda")
        y.copy_(self._yf[: self.shape[0]])
        self._pairs.dot_device(v64, y, accumulate=True)
        return y

    def dot(self, v):
        if device.is_device_tensor(v):
            return self.dot_device(v)
        x = device.to_dev(np.asarray(v, np.float64).reshape(-1))
        return self.dot_device(x).cpu().numpy()
