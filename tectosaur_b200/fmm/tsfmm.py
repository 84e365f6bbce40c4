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
import contextlib
import ctypes

import numpy as np

from .. import _lib
from ..kernels import kernels
from ..util import device
from ..util.quadrature import gauss2d_tri
from .tree import CompressedList, Tree, interactions, tri_centers_radii

SUPPORTED = ("elasticU3", "elasticRT3", "elasticRA3", "elasticRH3")
MODES = {"treecode": 0, "fmm": 1}


def touching_nodes(tree, r0, r1):
    """Boolean per node: the node's triangles include one whose original
    index is in [r0, r1) (a node's triangles are the contiguous tree
    positions start..end-1)."""
    inside = (tree.orig_idxs >= r0) & (tree.orig_idxs < r1)
    cs = np.concatenate([[0], np.cumsum(inside, dtype=np.int64)])
    return (cs[tree.end] - cs[tree.start]) > 0


def restrict_list(lst, keep_obs):
    """The entries of a compressed list whose observation node is kept
    (each kept entry with its whole source list, in the same order)."""
    obs, starts, src = lst.obs_n_idxs, lst.obs_src_starts, lst.src_n_idxs
    keep = keep_obs[obs] if obs.size else np.zeros(0, bool)
    lens = np.diff(starts)
    owner_keep = np.repeat(keep, lens)
    new_lens = lens[keep]
    return CompressedList(obs[keep].astype(np.int64),
                          np.concatenate([[0], np.cumsum(new_lens)]).astype(np.int64),
                          src[owner_keep].astype(np.int64))


class TSFMM:
    def __init__(self, obs_m, src_m, params, order, quad_order, float_type, K_name, mac,
                 max_pts_per_cell, mode="treecode", obs_rows=None):
        """obs_rows=(r0, r1) (an addition, for row shards): evaluate only the
        observation nodes that hold triangles r0..r1-1 -- their P2P and
        far-list entries, their L2L chain and L2P -- on the trees and lists
        of the whole observation set; the moments are computed in full.  The
        rows in the range are then exactly the full apply's (every stage
        computes a node from its own list entries only); other rows are
        partial or zero."""
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
        self.obs_rows = obs_rows
        touch = None
        if obs_rows is not None:
            touch = touching_nodes(self.obs_tree, int(obs_rows[0]), int(obs_rows[1]))
            lists = {k: restrict_list(v, touch) for k, v in lists.items()}
            far = lists["m2p"] if mode == "treecode" else lists["m2l"]
        self.touch = touch
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
        self.obs_desc, self._obs_off = self._tree_desc(self.obs_tree, dev, ft, obs=True,
                                                       keep=touch)
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
    def _tree_desc(tree, dev, ft, obs, keep=None):
        """Device descriptor of a tree; with `keep` (a row shard's
        observation side) only the kept nodes' L2L levels and leaves."""
        nodes, offsets = tree.l2l_levels() if obs else tree.m2m_levels()
        leaves = tree.leaves()
        if keep is not None:
            level_of = np.repeat(np.arange(offsets.shape[0] - 1), np.diff(offsets))
            k = keep[nodes]
            nodes = nodes[k]
            offsets = np.concatenate([[0], np.cumsum(
                np.bincount(level_of[k], minlength=offsets.shape[0] - 1))])
            leaves = leaves[keep[leaves]]
        offsets = np.ascontiguousarray(offsets, np.int64)
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

    def __call__(self, nq_far, K_name, params, pts, tris, float_type, obs_subset, src_subset,
                 row_range=None):
        return FMMFarfieldOpImpl(nq_far, K_name, params, pts, tris, float_type, obs_subset,
                                 src_subset, self.mac, self.pts_per_cell, self.order, self.mode,
                                 row_range=row_range)


class FMMFarfieldOpImpl:
    """row_range=(r0, r1) (an addition, for row shards): rows r0..r1-1 of the
    farfield over obs_subset, exactly those of the unsharded operator (the
    whole observation set's trees and lists, TSFMM(obs_rows=)); shape and
    dot cover the range's rows only."""

    def __init__(self, nq_far, K_name, params, pts, tris, float_type, obs_subset, src_subset,
                 mac, pts_per_cell, order, mode="treecode", row_range=None):
        pts = np.asarray(pts, dtype=np.float64)
        tris = np.asarray(tris)
        obs_subset = np.asarray(obs_subset)
        src_subset = np.asarray(src_subset)
        # the reference scales by the largest coordinate (not the extent)
        L_scale = np.max(pts)
        scaled = pts / L_scale
        self.L_factor = L_scale ** (-kernels[K_name].scale_type)
        self.float_type = np.dtype(float_type)
        n_obs = obs_subset.shape[0]
        self.row_range = None if row_range is None else (int(row_range[0]), int(row_range[1]))
        r0, r1 = self.row_range if row_range is not None else (0, n_obs)
        if not 0 <= r0 <= r1 <= n_obs:
            raise ValueError("row_range (%d, %d) outside 0..%d" % (r0, r1, n_obs))
        self.shape = ((r1 - r0) * 9, src_subset.shape[0] * 9)
        self.fmm = TSFMM((scaled, tris[obs_subset].copy()), (scaled, tris[src_subset].copy()),
                         params, order, nq_far, float_type, K_name, mac, pts_per_cell, mode,
                         obs_rows=self.row_range)
        self._full = device.empty(n_obs * 9, float_type) if row_range is not None else None

    def dot_device(self, x, y, accumulate=False, stream=None):
        if self.row_range is None:
            return self.fmm.dot_device(x, y, scale=self.L_factor, accumulate=accumulate,
                                       stream=stream)
        self.fmm.dot_device(x, self._full, scale=self.L_factor, accumulate=False, stream=stream)
        r0, r1 = self.row_range
        seg = self._full[9 * r0:9 * r1]
        t = device.torch()
        ctx = t.cuda.stream(stream) if stream is not None else contextlib.nullcontext()
        with ctx:
            if accumulate:
                y.add_(seg)
            else:
                y.copy_(seg)
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
