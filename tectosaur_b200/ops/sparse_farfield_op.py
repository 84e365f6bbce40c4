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
        self._panel_ws = {}

    def autotune(self, x=None):
        """Tune the source chunking of this operator's launch (cached in the
        library, tectosaur_b200.autotune); returns the chosen chunk count."""
        from .. import autotune
        return autotune.tune_farfield(self, x)

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

    # -- many right-hand sides ------------------------------------------------
    def panel_supported(self):
        """The tensor-core panel path: FP32 elasticRH3 (a 3-, 4- or 7-point
        rule) or elasticRT3 (a 3-point rule)."""
        if self.prec != _lib.TCT_F32:
            return False
        return ((self.K_name == "elasticRH3" and self.n_q in (3, 4, 7))
                or (self.K_name == "elasticRT3" and self.n_q == 3))

    def _panel_fns(self):
        pre = "tct_farfield_rh_panel" if self.K_name == "elasticRH3" else "tct_farfield_rt_panel"
        return (getattr(_lib.lib, pre + "_workspace_bytes"), getattr(_lib.lib, pre + "_matvec"),
                getattr(_lib.lib, pre + "_error"), pre)

    def dot_panel_device(self, X, Y, accumulate=False, stream=None):
        """Y[r] (+)= Far X[r] for device tensors X (R, 9 n_src), Y (R, 9 n_obs).
        FP32 elasticRH3 (3-, 4- or 7-point rule) and elasticRT3 (3-point
        rule) run on the tensor cores in panels of 16 vectors (split TF32,
        compensated FP32 accumulation); other kernels apply dot_device
        vector by vector."""
        t = device.torch()
        R = X.shape[0]
        if not self.panel_supported():
            for r in range(R):
                self.dot_device(X[r].contiguous(), Y[r], accumulate=accumulate, stream=stream)
            return Y
        ws_fn, mv_fn, _, name = self._panel_fns()
        r0 = 0
        while r0 < R:
            width = 16
            take = min(width, R - r0)
            if take == width:
                xin = X[r0:r0 + take].contiguous()
            else:
                xin = t.zeros((width, X.shape[1]), dtype=X.dtype, device=X.device)
                xin[:take] = X[r0:r0 + take]
            out = Y[r0:r0 + take] if take == width else t.empty(
                (width, Y.shape[1]), dtype=Y.dtype, device=Y.device)
            if take != width and accumulate:
                out[:take] = Y[r0:r0 + take]
            nbytes = ws_fn(self.n_obs, self.n_src, width, self.n_q)
            ws = self._panel_ws.get(width)
            if ws is None or ws.numel() < nbytes:
                ws = device.workspace(nbytes)
                self._panel_ws[width] = ws
            _lib.check(mv_fn(
                _lib.tptr(out), _lib.tptr(xin), _lib.tptr(self.gpu_pts),
                _lib.tptr(self.gpu_obs_tris), self.n_obs, _lib.tptr(self.gpu_src_tris), self.n_src,
                width, self.n_q, _lib.dptr(self.qx), _lib.dptr(self.qw), _lib.dptr(self.params),
                int(bool(accumulate)), _lib.tptr(ws), nbytes,
                _lib.stream_ptr(stream)), name + "_matvec")
            if take != width:
                Y[r0:r0 + take] = out[:take]
            r0 += take
        return Y

    def panel_error(self, width=16, stream=None):
        """Error word of the last panel apply (0 = ok)."""
        import ctypes
        flag = ctypes.c_int(0)
        ws = self._panel_ws.get(width)
        if ws is None:
            return 0
        _, _, err_fn, name = self._panel_fns()
        _lib.check(err_fn(
            _lib.tptr(ws), self.n_obs, self.n_src, width, self.n_q, _lib.stream_ptr(stream),
            ctypes.byref(flag)), name + "_error")
        return flag.value

    def dot_panel(self, X):
        """Host (R, 9 n_src) in, host (R, 9 n_obs) out."""
        t = device.torch()
        Xd = device.to_dev(np.asarray(X, dtype=self.float_type).reshape(-1, self.shape[1]),
                           self.float_type)
        Yd = t.empty((Xd.shape[0], self.shape[0]), dtype=Xd.dtype, device="cuda")
        self.dot_panel_device(Xd, Yd)
        return Yd.cpu().numpy()

    async def async_dot(self, v):
        return self.dot(v)

    def nearfield_dot(self, v):
        return self.dot(v)

    def nearfield_no_correction_dot(self, v):
        return self.dot(v)

    def farfield_dot(self, v):
        return self.dot(v)


from ..fmm.tsfmm import FMMFarfieldOp, FMMFarfieldOpImpl  # noqa: E402,F401
