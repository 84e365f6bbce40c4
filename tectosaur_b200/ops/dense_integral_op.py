"""Dense operators (reference: tectosaur/ops/dense_integral_op.py:11-84).

farfield_tris / FarfieldTriMatrix assemble every (obs, src) 9x9 block with a
gauss4d_tri(n_q, n_q) product rule on the device (tct_farfield_tris_dense,
one launch per 1024 obs triangles, as the reference chunks its calls).
RegularizedDenseIntegralOp keeps the uncorrected nearfield blocks where they
exist and the farfield blocks elsewhere.
"""
import numpy as np

from .. import _lib
from ..nearfield.nearfield_op import RegularizedNearfieldIntegralOp
from ..util import device
from ..util.quadrature import gauss4d_tri
from .dense_op import DenseOp


def farfield_tris(kernel, params, pts, obs_tris, src_tris, n_q, float_type):
    return FarfieldTriMatrix(kernel, params, n_q, float_type).assemble(pts, obs_tris, src_tris)


class FarfieldTriMatrix:
    def __init__(self, kernel, params, n_q, float_type):
        self.float_type = np.dtype(float_type)
        self.prec = _lib.prec_of(float_type)
        self.kid = _lib.kernel_id(kernel)
        self.params = np.ascontiguousarray(np.asarray(params, dtype=np.float64)[:2])
        self.q = gauss4d_tri(n_q, n_q)
        self.gpu_qx = device.to_dev(self.q[0], self.float_type)
        self.gpu_qw = device.to_dev(self.q[1], self.float_type)

    def assemble(self, pts, obs_tris, src_tris):
        gpu_pts = device.to_dev(np.asarray(pts, dtype=np.float64), self.float_type)
        gpu_src = device.to_dev(np.asarray(src_tris), np.int32)
        obs_tris = np.asarray(obs_tris)
        n, m = obs_tris.shape[0], np.asarray(src_tris).shape[0]
        out = np.empty((n, 3, 3, m, 3, 3), dtype=self.float_type)
        for start in range(0, n, 1024):
            end = min(n, start + 1024)
            res = device.empty((end - start) * 81 * m, self.float_type)
            gpu_obs = device.to_dev(obs_tris[start:end], np.int32)
            _lib.check(_lib.lib.tct_farfield_tris_dense(
                self.kid, self.prec, _lib.tptr(res), self.q[0].shape[0], _lib.tptr(self.gpu_qx),
                _lib.tptr(self.gpu_qw), _lib.tptr(gpu_pts), _lib.tptr(gpu_obs), end - start,
                _lib.tptr(gpu_src), m, _lib.dptr(self.params), _lib.stream_ptr()),
                "tct_farfield_tris_dense")
            out[start:end] = res.cpu().numpy().reshape(end - start, 3, 3, m, 3, 3)
        return out


class RegularizedDenseIntegralOp(DenseOp):
    def __init__(self, nq_coincident, nq_edge_adj, nq_vert_adjacent, nq_far, nq_near,
                 near_threshold, K_near_name, K_far_name, params, pts, tris, float_type,
                 obs_subset=None, src_subset=None):
        tris = np.asarray(tris)
        if obs_subset is None:
            obs_subset = np.arange(tris.shape[0])
        if src_subset is None:
            src_subset = np.arange(tris.shape[0])
        self.float_type = float_type
        nearfield = np.asarray(RegularizedNearfieldIntegralOp(
            pts, tris, obs_subset, src_subset,
            nq_coincident, nq_edge_adj, nq_vert_adjacent, nq_far, nq_near,
            near_threshold, K_near_name, K_far_name, params, float_type
        ).no_correction_to_dense())
        farfield = farfield_tris(
            K_far_name, params, pts, tris[obs_subset], tris[src_subset], nq_far, float_type
        ).reshape(nearfield.shape)
        self.mat = np.where(np.abs(nearfield) > 0, nearfield, farfield)
        self.mat[np.isnan(self.mat)] = 0.0
        self.shape = self.mat.shape
        self.gpu_mat = None
