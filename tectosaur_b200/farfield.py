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


PANEL_R = 16


def farfield_pts_panel_device(K, obs_pts, obs_ns, src_pts, src_ns, W, params, out=None,
                              accumulate=False, stream=None):
    """An addition: the point farfield for R weight vectors at once, FP32 on
    the tensor cores (tct_farfield_pts_panel: the kernel's 3x3 point-pair
    matrices generated on the fly, times the weight panel, split TF32 with
    compensated accumulation) in panels of 16.  Device float32 tensors:
    obs_pts/obs_ns (n_obs, 3), src_pts/src_ns (n_src, 3), W (R, 3 n_src);
    returns (R, 3 n_obs)."""
    t = device.torch()
    kid = _lib.kernel_id(K)
    n_obs, n_src = obs_pts.shape[0], src_pts.shape[0]
    R = W.shape[0]
    if out is None:
        out = t.empty((R, 3 * n_obs), dtype=t.float32, device="cuda")
    params = np.ascontiguousarray(np.asarray(params, dtype=np.float64)[:2])
    nbytes = int(_lib.lib.tct_farfield_pts_panel_workspace_bytes(n_obs, n_src, PANEL_R))
    ws = device.workspace(max(nbytes, 256))
    for r0 in range(0, R, PANEL_R):
        k = min(PANEL_R, R - r0)
        Wp = W[r0:r0 + k]
        Yp = out[r0:r0 + k]
        if k < PANEL_R or not (Wp.is_contiguous() and Yp.is_contiguous()):
            Wf = t.zeros((PANEL_R, 3 * n_src), dtype=t.float32, device="cuda")
            Wf[:k] = Wp
            Yf = t.empty((PANEL_R, 3 * n_obs), dtype=t.float32, device="cuda")
            if accumulate:
                Yf[:k] = Yp
        else:
            Wf, Yf = Wp, Yp
        _lib.check(_lib.lib.tct_farfield_pts_panel(
            kid, _lib.tptr(Yf), _lib.tptr(Wf), _lib.tptr(obs_pts), _lib.tptr(obs_ns), n_obs,
            _lib.tptr(src_pts), _lib.tptr(src_ns), n_src, PANEL_R, _lib.dptr(params),
            int(bool(accumulate)), _lib.tptr(ws), nbytes, _lib.stream_ptr(stream)),
            "tct_farfield_pts_panel")
        if Yf is not Yp:
            Yp.copy_(Yf[:k])
    flag = np.zeros(1, np.int32)
    _lib.check(_lib.lib.tct_farfield_pts_panel_error(
        _lib.tptr(ws), n_obs, n_src, PANEL_R, _lib.stream_ptr(stream),
        flag.ctypes.data_as(_lib.ctypes.POINTER(_lib.ctypes.c_int))),
        "tct_farfield_pts_panel_error")
    if flag[0]:
        raise RuntimeError("tct_farfield_pts_panel: a bounded tensor-core wait timed out")
    return out


def farfield_pts_panel(K, obs_pts, obs_ns, src_pts, src_ns, V, params):
    """Host form of farfield_pts_panel_device: V (R, 3 n_src) -> (R, 3 n_obs)
    float32 host arrays (the reference's farfield_pts_direct, vector by
    vector, on R vectors)."""
    f32 = np.float32
    args = [device.to_dev(np.asarray(a).reshape(-1, 3), f32)
            for a in (obs_pts, obs_ns, src_pts, src_ns)]
    W = device.to_dev(np.asarray(V, dtype=f32).reshape(np.asarray(V).shape[0], -1), f32)
    return farfield_pts_panel_device(K, *args, W, params).cpu().numpy()
