"""Point-to-point farfield sum (reference: tectosaur/farfield.py:15-38,
farfield_pts{K} of tectosaur/farfield_direct.cl:15-113), U/T/A/H only."""
import numpy as np

from . import _lib
from .util import device


def farfield_pts_direct(K, obs_pts, obs_ns, src_pts, src_ns, vec, params, float_type):
    ft = np.dtype(float_type)
    obs_pts = np.asarray(obs_pts)
    n_obs = obs_pts.shape[0]
    n_src = np.asarray(src_pts).shape[0]
    tensor_dim = int(np.asarray(vec).shape[0] / max(n_src, 1))
    if tensor_dim != 3:
        raise ValueError("farfield_pts_direct: elastic kernels take 3 components per point")
    out = device.empty(max(n_obs * 3, 1), ft)
    args = [device.to_dev(a, ft) for a in (obs_pts, obs_ns, src_pts, src_ns, vec)]
    params = np.ascontiguousarray(np.asarray(params, dtype=np.float64)[:2])
    _lib.check(_lib.lib.tct_farfield_pts(
        _lib.kernel_id(K), _lib.prec_of(ft), _lib.tptr(out), _lib.tptr(args[0]),
        _lib.tptr(args[1]), n_obs, _lib.tptr(args[2]), _lib.tptr(args[3]), n_src,
        _lib.tptr(args[4]), _lib.dptr(params), _lib.stream_ptr()), "tct_farfield_pts")
    return out[:n_obs * 3].cpu().numpy()
