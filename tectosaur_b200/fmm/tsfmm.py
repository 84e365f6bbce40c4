"""Treecode / FMM farfield operator (reference: FMMFarfieldOp / FMMFarfieldOpImpl,
tectosaur/ops/sparse_farfield_op.py:73-120, and TSFMM, tectosaur/fmm/tsfmm.py).

Same construction as the reference: the mesh is scaled by L = max(pts) (the
largest coordinate, as the reference does), ball octrees are built on the
observation and source triangles (max_pts_per_cell per leaf), the dual
traversal with MAC outer_r * R_src + inner_r * R_obs < 0.98 * separation
yields the interaction lists, and the result is multiplied by
L^(-scale_type).  The expansions are Cartesian multipoles / locals of order
`order` (csrc/fmm.cu).

mode="treecode" is the reference's scheme (inner_r 1, outer_r mac; P2P and
M2P).  mode="fmm" adds local expansions: the traversal runs without the
treecode flag and with inner_r = outer_r = mac, every accepted pair becomes an
M2L, locals are pushed down by L2L and evaluated by L2P.
Kernels: elasticU3, elasticRT3, elasticRA3, elasticRH3.
"""
import ctypes

import numpy as np

from .. import _lib
from ..kernels import kernels
from ..util import device
from ..util.quadrature import gauss2d_tri
from .tree import Tree, interactions, tri_centers_radii

SUPPORTED = ("elasticU3", "elasticRT3", "elasticRA3", "elasticRH3")
MODES = {"treecode": 0, "fmm": 1}


class TSFMM:
    def __init__(self, obs_m, src_m, params, order, quad_order, float_type, K_name, mac,
                 max_pts_per_cell, mode="treecode"):
        if K_name not in SUPPORTED:
            raise ValueError("treecode supports %s, not %s" % (", ".join(SUPPORTED), K_name))
        if mode not in MODES:
            raise ValueError("mode must be 'treecode' or 'fmm'")
        if not 0 <= int(order) <= 12:
            raise ValueError("treecode order must be 0..12")
        device.require_cuda()
        self.K = kernels[K_name]
        self.kid = _lib.kernel_id(K_name)
        self.mode = mode
        self.float_type = np.dtype(float_type)
        self.prec = _lib.prec_of(float_type)
        self.order = int(order)
        self.params = np.ascontiguousarray(np.asarray(params, np.float64)[:2])
        self.obs_m, self.src_m = obs_m, src_m
        self.obs_tree = Tree(*tri_centers_radii(*obs_m), max_pts_per_cell)
        same = (obs_m[0] is src_m[0] or np.array_equal(obs_m[0], src_m[0])) and \
            np.array_equal(obs_m[1], src_m[1])
        # a self operator (the same triangles on both sides) shares one tree
        self.src_tree = self.obs_tree if same else Tree(*tri_centers_radii(*src_m),
                                                        max_pts_per_cell)
        if mode == "treecode":
            lists = interactions(self.obs_tree, self.src_tree, 1.0, mac, 0, True)
            far = lists["m2p"]
        else:
            lists = interactions(self.obs_tree, self.src_tree, mac, mac, 0, False)
            far = lists["m2l"]
        self.lists = lists
        self.p2p, self.m2p, self.m2l = lists["p2p"], lists["m2p"], lists["m2l"]
        q = gauss2d_tri(quad_order)
        self.qx = np.ascontiguousarray(q[0], np.float64)
        self.qw = np.ascontiguousarray(q[1], np.float64)
        self.nq = self.qx.shape[0]
        ft = self.float_type
        self._keep = []  # device arrays the descriptors point at

        def dev(a, dt=None):
            if dt is None:
                a = np.ascontiguousarray(a, dtype=np.int64)
                if a.size == 0:
                    a = np.zeros(1, np.int64)
            t = device.to_dev(a, dt)
            self._keep.append(t)
            return t

        self.obs_pts = dev(obs_m[0], ft)
        self.src_pts = dev(src_m[0], ft)
        self.obs_tris = dev(np.asarray(obs_m[1])[self.obs_tree.orig_idxs], np.int32)
        self.src_tris = dev(np.asarray(src_m[1])[self.src_tree.orig_idxs], np.int32)
        self.obs_desc, self._obs_off = self._tree_desc(self.obs_tree, dev, ft, obs=True)
        self.src_desc, self._src_off = self._tree_desc(self.src_tree, dev, ft, obs=False)
        self.p2p_desc = self._list_desc(self.p2p, dev)
        self.far_desc = self._list_desc(far, dev)
        self.n_obs = np.asarray(obs_m[1]).shape[0]
        self.n_src = np.asarray(src_m[1]).shape[0]
        self.ws_bytes = _lib.lib.tct_fmm_workspace_bytes(
            self.kid, self.prec, MODES[mode], self.order, self.nq, self.n_obs, self.n_src,
            self.obs_tree.n_nodes, self.src_tree.n_nodes)
        if self.ws_bytes == 0:
            raise ValueError("unsupported treecode configuration (rule of %d points)" % self.nq)
        self.workspace = device.workspace(self.ws_bytes)

    @staticmethod
    def _tree_desc(tree, dev, ft, obs):
        nodes, offsets = tree.l2l_levels() if obs else tree.m2m_levels()
        offsets = np.ascontiguousarray(offsets, np.int64)
        leaves = tree.leaves()
        radii = np.where(tree.R > 0, tree.R, 1.0)
        desc = _lib.FmmTree(
            n_nodes=tree.n_nodes, start=dev(tree.start).data_ptr(), end=dev(tree.end).data_ptr(),
            centers=dev(tree.centers, ft).data_ptr(), radii=dev(radii, ft).data_ptr(),
            children=dev(tree.children).data_ptr(), parent=dev(tree.parent).data_ptr(),
            orig=dev(tree.orig_idxs).data_ptr(), leaves=dev(leaves).data_ptr(),
            n_leaves=leaves.shape[0], levels=dev(nodes).data_ptr(),
            level_offsets=_lib.i64ptr(offsets), n_levels=offsets.shape[0] - 1)
        return desc, offsets

    @staticmethod
    def _list_desc(lst, dev):
        """Device copy of a compressed list with its obs entries ordered longest
        list first (one block or warp per entry: the long ones start first)."""
        obs, start, src = lst.obs_n_idxs, lst.obs_src_starts, lst.src_n_idxs
        lens = np.diff(start)
        order = np.argsort(-lens, kind="stable")
        new_start = np.concatenate([[0], np.cumsum(lens[order])]).astype(np.int64)
        new_src = (np.concatenate([src[start[i]:start[i + 1]] for i in order])
                   if order.size else src)
        return _lib.FmmList(obs=dev(obs[order]).data_ptr(), start=dev(new_start).data_ptr(),
                            src=dev(new_src).data_ptr(), n_obs=obs.shape[0])

    def dot_device(self, x, y, scale=1.0, accumulate=False, stream=None):
        """y (+)= scale * farfield(x) for device tensors in original order."""
        t = _lib.tptr
        _lib.check(_lib.lib.tct_fmm_matvec(
            self.kid, self.prec, MODES[self.mode], self.order, self.nq, _lib.dptr(self.qx),
            _lib.dptr(self.qw), _lib.dptr(self.params), float(scale), t(self.obs_pts),
            t(self.obs_tris), self.n_obs, ctypes.byref(self.obs_desc), t(self.src_pts),
            t(self.src_tris), self.n_src, ctypes.byref(self.src_desc),
            ctypes.byref(self.p2p_desc), ctypes.byref(self.far_desc), t(x), t(y),
            int(bool(accumulate)), t(self.workspace), self.ws_bytes, _lib.stream_ptr(stream)),
            "tct_fmm_matvec")
        return y

    def dot(self, v):
        x = device.to_dev(np.asarray(v).reshape(-1), self.float_type)
        y = device.empty(self.n_obs * 9, self.float_type)
        self.dot_device(x, y)
        return y.cpu().numpy()


class FMMFarfieldOp:
    """Factory with the reference's signature: FMMFarfieldOp(mac, pts_per_cell, order);
    `mode` ("treecode" as in the reference, or "fmm") is an addition."""

    def __init__(self, mac, pts_per_cell, order, mode="treecode"):
        self.mac = mac
        self.pts_per_cell = pts_per_cell
        self.order = order
        self.mode = mode

    def __call__(self, nq_far, K_name, params, pts, tris, float_type, obs_subset, src_subset):
        return FMMFarfieldOpImpl(nq_far, K_name, params, pts, tris, float_type, obs_subset,
                                 src_subset, self.mac, self.pts_per_cell, self.order, self.mode)


class FMMFarfieldOpImpl:
    def __init__(self, nq_far, K_name, params, pts, tris, float_type, obs_subset, src_subset,
                 mac, pts_per_cell, order, mode="treecode"):
        pts = np.asarray(pts, dtype=np.float64)
        tris = np.asarray(tris)
        obs_subset = np.asarray(obs_subset)
        src_subset = np.asarray(src_subset)
        # the reference scales by the largest coordinate (not the extent)
        L_scale = np.max(pts)
        scaled = pts / L_scale
        self.L_factor = L_scale ** (-kernels[K_name].scale_type)
        self.float_type = np.dtype(float_type)
        self.shape = (obs_subset.shape[0] * 9, src_subset.shape[0] * 9)
        self.fmm = TSFMM((scaled, tris[obs_subset].copy()), (scaled, tris[src_subset].copy()),
                         params, order, nq_far, float_type, K_name, mac, pts_per_cell, mode)

    def dot_device(self, x, y, accumulate=False, stream=None):
        return self.fmm.dot_device(x, y, scale=self.L_factor, accumulate=accumulate,
                                   stream=stream)

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
