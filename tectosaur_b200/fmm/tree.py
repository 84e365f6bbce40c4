"""Treecode trees and interaction lists (reference: tectosaur/fmm/tsfmm.py:22-28,
66-70; fmm/octree.cpp; fmm/traversal.cpp), built in libtct_b200.so."""
import ctypes

import numpy as np

from .. import _lib


def tri_centers_radii(pts, tris):
    """Centre (vertex mean) and max centre-vertex distance of each triangle
    (make_tree of fmm/tsfmm.py:22-28)."""
    tri_pts = pts[tris]
    centers = np.mean(tri_pts, axis=1)
    Rs = np.max(np.linalg.norm(tri_pts - centers[:, np.newaxis, :], axis=2), axis=1)
    return centers, Rs


# trees from this many balls are built on the GPU when one is visible (the
# same tree, node for node)
DEVICE_TREE_MIN = 100_000


class Tree:
    """Ball octree: node arrays in depth-first preorder and the permutation
    from tree positions to original indices.  device: build on the GPU
    (tct_tree_build_device) -- None picks the GPU from DEVICE_TREE_MIN balls
    when one is visible."""

    def __init__(self, centers, radii, max_pts_per_cell, device=None):
        c = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
        r = np.ascontiguousarray(radii, dtype=np.float64).reshape(-1)
        if device is None:
            from ..util import device as dev
            device = c.shape[0] >= DEVICE_TREE_MIN and dev.cuda_available()
        h = ctypes.c_void_p()
        if device:
            _lib.check(_lib.lib.tct_tree_build_device(
                _lib.dptr(c), _lib.dptr(r), c.shape[0], int(max_pts_per_cell),
                _lib.stream_ptr(), ctypes.byref(h)), "tct_tree_build_device")
        else:
            _lib.check(_lib.lib.tct_tree_build(_lib.dptr(c), _lib.dptr(r), c.shape[0],
                                               int(max_pts_per_cell), ctypes.byref(h)),
                       "tct_tree_build")
        self.on_device = bool(device)
        self._h = h
        n = _lib.lib.tct_tree_n_nodes(h)
        self.n_nodes = n
        self.max_height = _lib.lib.tct_tree_max_height(h)
        self.orig_idxs = np.empty(c.shape[0], np.int64)
        self.start = np.empty(n, np.int64)
        self.end = np.empty(n, np.int64)
        self.centers = np.empty((n, 3))
        self.R = np.empty(n)
        self.is_leaf = np.empty(n, np.int32)
        self.depth = np.empty(n, np.int32)
        self.height = np.empty(n, np.int32)
        self.children = np.empty((n, 8), np.int64)
        i32 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        _lib.check(_lib.lib.tct_tree_export(
            h, _lib.i64ptr(self.orig_idxs), _lib.i64ptr(self.start), _lib.i64ptr(self.end),
            _lib.dptr(self.centers), _lib.dptr(self.R), i32(self.is_leaf), i32(self.depth),
            i32(self.height), _lib.i64ptr(self.children)), "tct_tree_export")
        self.parent = np.full(n, -1, np.int64)
        inner = np.nonzero(self.is_leaf == 0)[0]
        self.parent[self.children[inner].reshape(-1)] = np.repeat(inner, 8)

    def leaves(self):
        return np.nonzero(self.is_leaf)[0].astype(np.int64)

    def m2m_levels(self):
        """Non-leaf nodes grouped by height 1, 2, ... (children before parents)."""
        groups = [np.nonzero((self.is_leaf == 0) & (self.height == h))[0]
                  for h in range(1, self.max_height + 1)]
        return _grouped(groups)

    def l2l_levels(self):
        """Non-root nodes grouped by depth 1, 2, ... (parents before children)."""
        groups = [np.nonzero(self.depth == d)[0] for d in range(1, int(self.depth.max()) + 1)]
        return _grouped(groups)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None and _lib.lib is not None:
            _lib.lib.tct_tree_free(self._h)
            self._h = None


def _grouped(groups):
    offsets = np.concatenate([[0], np.cumsum([g.shape[0] for g in groups])]).astype(np.int64)
    nodes = np.concatenate(groups).astype(np.int64) if groups else np.zeros(0, np.int64)
    return nodes, offsets


class CompressedList:
    def __init__(self, obs_n_idxs, obs_src_starts, src_n_idxs):
        self.obs_n_idxs = obs_n_idxs
        self.obs_src_starts = obs_src_starts
        self.src_n_idxs = src_n_idxs


LIST_NAMES = ("p2p", "m2p", "p2l", "m2l")


def interactions(obs_tree, src_tree, inner_r, outer_r, order=0, treecode=True):
    """All four compressed lists of the dual traversal, keyed by name."""
    h = ctypes.c_void_p()
    _lib.check(_lib.lib.tct_treecode_lists(obs_tree._h, src_tree._h, float(inner_r),
                                           float(outer_r), int(order), int(bool(treecode)),
                                           ctypes.byref(h)), "tct_treecode_lists")
    out = {}
    try:
        sizes = np.zeros(8, np.int64)
        _lib.check(_lib.lib.tct_lists_sizes(h, _lib.i64ptr(sizes)), "tct_lists_sizes")
        for k, name in enumerate(LIST_NAMES):
            arrs = [np.empty(sizes[2 * k], np.int64), np.empty(sizes[2 * k] + 1, np.int64),
                    np.empty(sizes[2 * k + 1], np.int64)]
            _lib.check(_lib.lib.tct_lists_export(h, k, *[_lib.i64ptr(a) for a in arrs]),
                       "tct_lists_export")
            out[name] = CompressedList(*arrs)
    finally:
        _lib.lib.tct_lists_free(h)
    return out


def treecode_interactions(obs_tree, src_tree, inner_r, outer_r, order=0, treecode=True):
    """(p2p, m2p) compressed lists of the dual traversal."""
    lists = interactions(obs_tree, src_tree, inner_r, outer_r, order, treecode)
    return lists["p2p"], lists["m2p"]
