"""Treecode farfield operator (reference: FMMFarfieldOp / FMMFarfieldOpImpl,
tectosaur/ops/sparse_farfield_op.py:73-120, and TSFMM, tectosaur/fmm/tsfmm.py).

Same construction as the reference: the mesh is scaled by L = max(pts) (the
largest coordinate, as the reference does), ball octrees are built on the
observation and source triangles (max_pts_per_cell per leaf), the dual
traversal with MAC mac * R_src + R_obs < 0.98 * separation yields P2P and
M2P lists, and the result is multiplied by L^(-scale_type).  The expansions
are this build's Cartesian multipoles of order `order` (csrc/fmm.cu).
Kernels: elasticU3, elasticRT3, elasticRA3, elasticRH3.
"""
import numpy as np

from .. import _lib
from ..kernels import kernels
from ..util import device
from ..util.quadrature import gauss2d_tri
from .tree import Tree, tri_centers_radii, treecode_interactions

SUPPORTED = ("elasticU3", "elasticRT3", "elasticRA3", "elasticRH3")


class TSFMM:
    def __init__(self, obs_m, src_m, params, order, quad_order, float_type, K_name, mac,
                 max_pts_per_cell):
        if K_name not in SUPPORTED:
            raise ValueError("treecode supports %s, not %s" % (", ".join(SUPPORTED), K_name))
        device.require_cuda()
        self.K = kernels[K_name]
        self.kid = _lib.kernel_id(K_name)
        self.float_type = np.dtype(float_type)
        self.prec = _lib.prec_of(float_type)
        self.order = int(order)
        if not 0 <= self.order <= 12:
            raise ValueError("treecode order must be 0..12")
        self.params = np.ascontiguousarray(np.asarray(params, np.float64)[:2])
        self.obs_m, self.src_m = obs_m, src_m
        oc, orr = tri_centers_radii(*obs_m)
        sc, sr = tri_centers_radii(*src_m)
        self.obs_tree = Tree(oc, orr, max_pts_per_cell)
        self.src_tree = Tree(sc, sr, max_pts_per_cell)
        self.p2p, self.m2p = treecode_interactions(self.obs_tree, self.src_tree, 1.0, mac, 0,
                                                   True)
        q = gauss2d_tri(quad_order)
        self.nq = q[0].shape[0]
        ft = self.float_type
        ot, st = self.obs_tree, self.src_tree
        d = device.to_dev
        self.dev = {
            "qx": d(q[0], ft), "qw": d(q[1], ft),
            "obs_pts": d(obs_m[0], ft), "src_pts": d(src_m[0], ft),
            "obs_tris": d(np.asarray(obs_m[1])[ot.orig_idxs], np.int32),
            "src_tris": d(np.asarray(src_m[1])[st.orig_idxs], np.int32),
            "obs_orig": d(ot.orig_idxs), "src_orig": d(st.orig_idxs),
            "o_start": d(ot.start), "o_end": d(ot.end),
            "s_start": d(st.start), "s_end": d(st.end),
            "s_cent": d(st.centers, ft), "s_children": d(st.children),
            "src_leaves": d(np.nonzero(st.is_leaf)[0].astype(np.int64)),
        }
        parents = [np.nonzero((st.is_leaf == 0) & (st.height == h))[0]
                   for h in range(1, st.max_height + 1)]
        self.height_counts = np.concatenate([[0], np.cumsum([p.shape[0] for p in parents])]) \
            .astype(np.int64)
        allp = np.concatenate(parents) if parents else np.zeros(0, np.int64)
        self.dev["m2m_parents"] = d(allp.astype(np.int64) if allp.size else np.zeros(1, np.int64))
        self.n_heights = len(parents)
        for name, lst in [("p2p", self.p2p), ("m2p", self.m2p)]:
            self.dev[name + "_obs"] = d(lst.obs_n_idxs if lst.obs_n_idxs.size else np.zeros(1, np.int64))
            self.dev[name + "_start"] = d(lst.obs_src_starts)
            self.dev[name + "_src"] = d(lst.src_n_idxs if lst.src_n_idxs.size else np.zeros(1, np.int64))
        self.n_obs = np.asarray(obs_m[1]).shape[0]
        self.n_src = np.asarray(src_m[1]).shape[0]
        self.ws_bytes = _lib.lib.tct_treecode_workspace_bytes(
            self.kid, self.prec, self.order, self.n_obs, self.n_src, st.n_nodes, self.nq)
        self.workspace = device.workspace(self.ws_bytes)

    def dot_device(self, x, y, scale=1.0, accumulate=False, stream=None):
        """y (+)= scale * treecode(x) for device tensors in original order."""
        dv = self.dev
        st = self.src_tree
        t = _lib.tptr
        _lib.check(_lib.lib.tct_treecode_matvec(
            self.kid, self.prec, self.order, self.nq, t(dv["qx"]), t(dv["qw"]),
            _lib.dptr(self.params), float(scale), t(dv["obs_pts"]), t(dv["obs_tris"]), self.n_obs,
            t(dv["obs_orig"]), t(dv["o_start"]), t(dv["o_end"]), t(dv["src_pts"]),
            t(dv["src_tris"]), self.n_src, t(dv["src_orig"]), t(dv["s_start"]), t(dv["s_end"]), t(dv["s_cent"]),
            t(dv["s_children"]), st.n_nodes, t(dv["src_leaves"]), int(np.sum(st.is_leaf)),
            t(dv["m2m_parents"]), _lib.i64ptr(self.height_counts), self.n_heights,
            t(dv["p2p_obs"]), t(dv["p2p_start"]), t(dv["p2p_src"]), self.p2p.obs_n_idxs.shape[0],
            t(dv["m2p_obs"]), t(dv["m2p_start"]), t(dv["m2p_src"]), self.m2p.obs_n_idxs.shape[0],
            t(x), t(y), int(bool(accumulate)), t(self.workspace), self.ws_bytes,
            _lib.stream_ptr(stream)), "tct_treecode_matvec")
        return y

    def dot(self, v):
        x = device.to_dev(np.asarray(v).reshape(-1), self.float_type)
        y = device.empty(self.n_obs * 9, self.float_type)
        self.dot_device(x, y)
        return y.cpu().numpy()


class FMMFarfieldOp:
    """Factory with the reference's signature: FMMFarfieldOp(mac, pts_per_cell, order)."""

    def __init__(self, mac, pts_per_cell, order):
        self.mac = mac
        self.pts_per_cell = pts_per_cell
        self.order = order

    def __call__(self, nq_far, K_name, params, pts, tris, float_type, obs_subset, src_subset):
        return FMMFarfieldOpImpl(nq_far, K_name, params, pts, tris, float_type, obs_subset,
                                 src_subset, self.mac, self.pts_per_cell, self.order)


class FMMFarfieldOpImpl:
    def __init__(self, nq_far, K_name, params, pts, tris, float_type, obs_subset, src_subset,
                 mac, pts_per_cell, order):
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
                         params, order, nq_far, float_type, K_name, mac, pts_per_cell)

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
