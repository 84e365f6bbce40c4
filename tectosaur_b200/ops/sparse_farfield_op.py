"""Direct farfield operator (reference: tectosaur/ops/sparse_farfield_op.py:16-71).

TriToTriDirectFarfieldOp applies the farfield rule gauss2d_tri(nq_far) between
every (obs, src) triangle pair of the subsets -- nearfield pairs included; the
nearfield operator subtracts the same rule from its blocks -- through
tct_farfield_tris_matvec.  ``dot`` takes a host array (copied in, result
copied out in float_type, as the reference) or a CUDA tensor (no copies).
"""
import numpy as np

from .. import _lib
from ..kernels import kernels
from ..util import device
from ..util.quadrature import gauss2d_tri


class TriToTriDirectFarfieldOp:
    def __init__(self, nq_far, K_name, params, pts, tris, float_type, obs_subset, src_subset):
        device.require_cuda()
        obs_subset = np.asarray(obs_subset)
        src_subset = np.asarray(src_subset)
        tris = np.asarray(tris)
        self.shape = (obs_subset.shape[0] * 9, src_subset.shape[0] * 9)
        self.dim = np.asarray(pts).shape[1]
        self.tensor_dim = kernels[K_name].tensor_dim
        self.n_obs = obs_subset.shape[0]
        self.n_src = src_subset.shape[0]
        self.float_type = np.dtype(float_type)
        self.prec = _lib.prec_of(float_type)
        self.kid = _lib.kernel_id(K_name)
        self.K_name = K_name
        self.params = np.ascontiguousarray(np.asarray(params, dtype=np.float64)[:2])
        q = gauss2d_tri(nq_far)
        self.q = q
        self.n_q = q[0].shape[0]
        self.qx = np.ascontiguousarray(q[0], dtype=np.float64)
        self.qw = np.ascontiguousarray(q[1], dtype=np.float64)
        self.gpu_pts = device.to_dev(np.asarray(pts, dtype=np.float64), self.float_type)
        self.gpu_obs_tris = device.to_dev(tris[obs_subset], np.int32)
        self.gpu_src_tris = device.to_dev(tris[src_subset], np.int32)
        self.ws_bytes = _lib.lib.tct_farfield_workspace_bytes(
            self.kid, self.prec, self.n_obs, self.n_src, self.n_q)
        if self.ws_bytes == 0 and self.n_src > 0:
            raise ValueError("farfield: unsupported kernel/rule (%s, %d points)" % (K_name, self.n_q))
        self.workspace = device.workspace(self.ws_bytes)

    def dot_device(self, x, y, accumulate=False, stream=None):
        """y (+)= Far x on device tensors of float_type."""
        _lib.check(_lib.lib.tct_farfield_tris_matvec(
            self.kid, self.prec, _lib.tptr(y), _lib.tptr(x), _lib.tptr(self.gpu_pts),
            _lib.tptr(self.gpu_obs_tris), self.n_obs, _lib.tptr(self.gpu_src_tris), self.n_src,
            self.n_q, _lib.dptr(self.qx), _lib.dptr(self.qw), _lib.dptr(self.params),
            int(bool(accumulate)), _lib.tptr(self.workspace), self.ws_bytes,
            _lib.stream_ptr(stream)), "tct_farfield_tris_matvec")
        return y

    def dot(self, v):
        if device.is_device_tensor(v):
            x = v.to(device.torch_dtype(self.float_type)).contiguous()
            y = device.empty(self.shape[0], self.float_type)
            return self.dot_device(x, y)
        x = device.to_dev(np.asarray(v).reshape(-1), self.float_type)
        y = device.empty(self.shape[0], self.float_type)
        self.dot_device(x, y)
        return y.cpu().numpy()

    async def async_dot(self, v):
        return self.dot(v)

    def nearfield_dot(self, v):
        return self.dot(v)

    def nearfield_no_correction_dot(self, v):
        return self.dot(v)

    def farfield_dot(self, v):
        return self.dot(v)


from ..fmm.tsfmm import FMMFarfieldOp, FMMFarfieldOpImpl  # noqa: E402,F401
