"""The elastic BEM operator: corrected nearfield + farfield on all pairs
(reference: tectosaur/ops/sparse_integral_op.py:10-62).

``dot(v)`` = farfield(v) + nearfield(v).  On the device both terms write into
one output buffer on one stream (farfield overwrites, the BSR nearfield
accumulates), so a host-array apply costs one copy in and one copy out, and
``capture_graph`` records the whole apply as a CUDA graph for repeated use.
"""
import numpy as np

from ..nearfield.nearfield_op import RegularizedNearfieldIntegralOp
from ..util import device


class RegularizedSparseIntegralOp:
    def __init__(self, nq_coincident, nq_edge_adj, nq_vert_adjacent,
                 nq_far, nq_near, near_threshold,
                 K_near_name, K_far_name, params, pts, tris, float_type, farfield_op_type,
                 obs_subset=None, src_subset=None, keep_uncorrected=True, row_range=None,
                 batched=True):
        """row_range=(r0, r1) (an addition, for row shards): the operator is
        block rows r0..r1-1 of the one over obs_subset x src_subset -- the
        same near pairs and blocks (the search runs over the whole
        obs_subset) and the farfield of those observation triangles (an FMM
        farfield: the whole set's trees and lists, evaluated on the leaves
        that hold the rows) -- so stacking the applies of a partition of the
        rows gives the full operator's apply."""
        tris = np.asarray(tris)
        if obs_subset is None:
            obs_subset = np.arange(tris.shape[0])
        if src_subset is None:
            src_subset = np.arange(tris.shape[0])
        obs_subset = np.asarray(obs_subset)
        self.float_type = np.dtype(float_type)
        self.row_range = row_range
        self.nearfield = RegularizedNearfieldIntegralOp(
            pts, tris, obs_subset, src_subset,
            nq_coincident, nq_edge_adj, nq_vert_adjacent, nq_far, nq_near,
            near_threshold, K_near_name, K_far_name, params, float_type,
            keep_uncorrected=keep_uncorrected, row_range=row_range, batched=batched)
        self._far_args = (farfield_op_type, nq_far, K_far_name, params, pts, tris, obs_subset,
                          src_subset)
        self.farfield = self._make_far(farfield_op_type, float_type)
        self.shape = self.nearfield.shape
        self._graph = None

    def _make_far(self, factory, float_type):
        """The farfield of this operator's rows: the direct farfield over
        the row range's observation triangles; an FMM farfield keeps the
        whole observation set's trees and lists and evaluates the rows'
        leaves (FMMFarfieldOpImpl(row_range=)), so its rows are exactly the
        unsharded FMM's."""
        from ..fmm.tsfmm import FMMFarfieldOp
        _, nq_far, K_far, params, pts, tris, obs_subset, src_subset = self._far_args
        rr = self.row_range
        if rr is not None and isinstance(factory, FMMFarfieldOp):
            return factory(nq_far, K_far, params, pts, tris, float_type, obs_subset, src_subset,
                           row_range=rr)
        far_obs = obs_subset if rr is None else obs_subset[rr[0]:rr[1]]
        return factory(nq_far, K_far, params, pts, tris, float_type, far_obs, src_subset)

    def autotune(self):
        """Tune this operator's launch shapes (direct-farfield source
        chunking, nearfield BSR shape) on its own data and keep them in the
        library's shape cache (tectosaur_b200.autotune); returns them."""
        from .. import autotune
        return autotune.tune_operator(self)

    def astype(self, float_type, keep_uncorrected=True, farfield_op_type=None):
        """The same operator in another precision (an addition, for mixed-
        precision solves): the nearfield blocks are cast from this operator's
        (structure shared, no re-integration), the farfield is set up anew in
        float_type -- with this operator's farfield type, or with
        `farfield_op_type` (e.g. the direct farfield, whose multi-RHS form runs
        on the tensor cores, as the inner operator of a solve whose FP64
        residual uses an FMM farfield)."""
        import copy
        twin = copy.copy(self)
        twin.float_type = np.dtype(float_type)
        twin.nearfield = self.nearfield.astype(float_type, keep_uncorrected)
        factory = self._far_args[0]
        if farfield_op_type is not None:
            factory = farfield_op_type
            twin._far_args = (factory,) + self._far_args[1:]
        twin.farfield = twin._make_far(factory, float_type)
        twin._graph = None
        return twin

    # -- device apply -------------------------------------------------------
    # operators from this many rows run the nearfield next to an FMM farfield
    OVERLAP_MIN_ROWS = 9 * 100_000

    def _overlap_near(self):
        from ..fmm.tsfmm import FMMFarfieldOpImpl
        return (isinstance(self.farfield, FMMFarfieldOpImpl)
                and hasattr(self.nearfield, "dot_device") and self.shape[0] >= self.OVERLAP_MIN_ROWS)

    def _overlapped(self, x, y, stream, near_into, far):
        """near_into(buf, side stream) next to far(main stream); y += buf."""
        t = device.torch()
        main = stream if stream is not None else t.cuda.current_stream()
        if getattr(self, "_near_stream", None) is None:
            self._near_stream = t.cuda.Stream(priority=t.cuda.Stream.priority_range()[1])
        side = self._near_stream
        buf = getattr(self, "_near_buf", None)
        if buf is None or buf.dtype != y.dtype or buf.shape != y.shape:
            buf = self._near_buf = t.empty_like(y)
        side.wait_stream(main)
        near_into(buf, side)
        far(main)
        main.wait_stream(side)
        with t.cuda.stream(main):
            y.add_(buf)
        return y

    def dot_device(self, x, y, stream=None, accumulate=False):
        """y (+)= (Far + Near) x on device tensors of float_type.  With an
        FMM farfield on a large mesh the nearfield BSR (HBM-bound) runs on a
        high-priority second stream into its own buffer while the FMM
        (compute-bound) runs, and is added at the end."""
        acc = bool(accumulate)
        if self._overlap_near():
            return self._overlapped(
                x, y, stream, lambda b, s: self.nearfield.dot_device(x, b, accumulate=False,
                                                                      stream=s),
                lambda s: self.farfield.dot_device(x, y, accumulate=acc, stream=s))
        if hasattr(self.farfield, "dot_device"):
            self.farfield.dot_device(x, y, accumulate=acc, stream=stream)
        else:
            far = device.torch().as_tensor(self.farfield.dot(x.cpu().numpy()), device="cuda")
            y.add_(far) if acc else y.copy_(far)
        self.nearfield.dot_device(x, y, accumulate=True, stream=stream)
        return y

    def dot_panel_device(self, X, Y, stream=None, accumulate=False):
        """Y[r] (+)= (Far + Near) X[r] for device tensors X (R, 9 n_src),
        Y (R, 9 n_obs) of float_type (an addition: R vectors per apply; the
        FP32 elasticRH3 / elasticRT3 farfield runs on the tensor cores, the
        nearfield BSR in one launch)."""
        far = self.farfield
        acc = bool(accumulate)
        if self._overlap_near() and not hasattr(far, "dot_panel_device"):
            def far_all(s):
                for r in range(X.shape[0]):
                    far.dot_device(X[r], Y[r], accumulate=acc, stream=s)
            return self._overlapped(
                X, Y, stream, lambda b, s: self.nearfield.dot_panel_device(X, b, accumulate=False,
                                                                            stream=s), far_all)
        if hasattr(far, "dot_panel_device"):
            far.dot_panel_device(X, Y, accumulate=acc, stream=stream)
        else:
            for r in range(X.shape[0]):
                far.dot_device(X[r], Y[r], accumulate=acc, stream=stream)
        self.nearfield.dot_panel_device(X, Y, accumulate=True, stream=stream)
        return Y

    def dot_panel(self, X):
        """Host (R, 9 n_src) in, host (R, 9 n_obs) out."""
        t = device.torch()
        X = np.asarray(X).reshape(-1, self.shape[1])
        Xd = device.to_dev(np.ascontiguousarray(X, dtype=self.float_type), self.float_type)
        Yd = t.empty((Xd.shape[0], self.shape[0]), dtype=Xd.dtype, device="cuda")
        self.dot_panel_device(Xd, Yd)
        return Yd.cpu().numpy()

    def capture_graph(self):
        """Record one full apply (farfield + nearfield) as a CUDA graph on
        private input/output buffers; returns (graph, x, y): fill x, call
        graph.replay(), read y."""
        t = device.torch()
        x = device.zeros(self.shape[1], self.float_type)
        y = device.zeros(self.shape[0], self.float_type)
        s = t.cuda.Stream()
        s.wait_stream(t.cuda.current_stream())
        with t.cuda.stream(s):
            self.dot_device(x, y)  # warm-up outside the capture
        t.cuda.current_stream().wait_stream(s)
        g = t.cuda.CUDAGraph()
        with t.cuda.graph(g):
            self.dot_device(x, y)
        self._graph = (g, x, y)
        return self._graph

    def dot(self, v):
        if device.is_device_tensor(v):
            x = v.to(device.torch_dtype(self.float_type)).contiguous()
            y = device.empty(self.shape[0], self.float_type)
            return self.dot_device(x, y)
        x = device.to_dev(np.asarray(v).reshape(-1), self.float_type)
        y = device.empty(self.shape[0], self.float_type)
        self.dot_device(x, y)
        return y.cpu().numpy()

    async def nearfield_dot(self, v):
        return self.nearfield.dot(v)

    def nearfield_no_correction_dot(self, v):
        return self.nearfield.nearfield_no_correction_dot(v)

    async def farfield_dot(self, v):
        return await self.farfield.async_dot(v)
