"""Near-pair search and adjacency split (reference: tectosaur/mesh/find_near_adj.py
and mesh/fast_find_nearfield.cpp), on the C++ side of libtct_b200.so."""
import ctypes

import numpy as np

from .. import _lib


def get_tri_centroids_rs(pts, tris):
    """Centroid and bounding radius (max centroid-vertex distance) of each
    triangle, with the reference's NumPy reductions (find_near_adj.py:13-20),
    so the radii -- and hence the near-pair set -- match bit for bit."""
    tri_pts = pts[tris]
    centroid = np.sum(tri_pts, axis=1) / 3.0
    r = np.sqrt(np.max(np.sum((tri_pts - centroid[:, np.newaxis, :]) ** 2, axis=2), axis=1))
    return centroid, r


def get_nearfield(obs_centers, obs_radii, src_centers, src_radii, threshold, n_threads=0):
    """All (i, j) with |c_i - c_j|^2 <= ((r_i + r_j) threshold)^2, int64 (P, 2),
    lexicographically ordered."""
    oc = np.ascontiguousarray(obs_centers, dtype=np.float64).reshape(-1, 3)
    orr = np.ascontiguousarray(obs_radii, dtype=np.float64).reshape(-1)
    sc = np.ascontiguousarray(src_centers, dtype=np.float64).reshape(-1, 3)
    sr = np.ascontiguousarray(src_radii, dtype=np.float64).reshape(-1)
    handle = ctypes.c_void_p()
    _lib.check(_lib.lib.tct_find_near_pairs(
        _lib.dptr(oc), _lib.dptr(orr), oc.shape[0], _lib.dptr(sc), _lib.dptr(sr), sc.shape[0],
        float(threshold), int(n_threads), ctypes.byref(handle)), "tct_find_near_pairs")
    try:
        n = _lib.lib.tct_pairs_count(handle)
        out = np.empty((n, 2), dtype=np.int64)
        _lib.check(_lib.lib.tct_pairs_copy(handle, _lib.i64ptr(out)), "tct_pairs_copy")
    finally:
        _lib.lib.tct_pairs_free(handle)
    return out


def near_plan(obs_centers, obs_radii, src_centers, src_radii, threshold, n_threads=0,
              device_tree=False, stream=None):
    """The octrees and dual traversal of the device search, down to leaf
    pairs (an opaque handle; free with `_lib.lib.tct_near_plan_free`): built
    on the host, or with device_tree on the GPU (the same leaf pairs)."""
    oc = np.ascontiguousarray(obs_centers, dtype=np.float64).reshape(-1, 3)
    orr = np.ascontiguousarray(obs_radii, dtype=np.float64).reshape(-1)
    if src_centers is obs_centers and src_radii is obs_radii:
        sc, sr = oc, orr  # a self search: one tree
    else:
        sc = np.ascontiguousarray(src_centers, dtype=np.float64).reshape(-1, 3)
        sr = np.ascontiguousarray(src_radii, dtype=np.float64).reshape(-1)
    handle = ctypes.c_void_p()
    if device_tree:
        _lib.check(_lib.lib.tct_near_plan_build_device(
            _lib.dptr(oc), _lib.dptr(orr), oc.shape[0], _lib.dptr(sc), _lib.dptr(sr),
            sc.shape[0], float(threshold), _lib.stream_ptr(stream), ctypes.byref(handle)),
            "tct_near_plan_build_device")
        return handle
    _lib.check(_lib.lib.tct_near_plan_build(
        _lib.dptr(oc), _lib.dptr(orr), oc.shape[0], _lib.dptr(sc), _lib.dptr(sr), sc.shape[0],
        float(threshold), int(n_threads), ctypes.byref(handle)), "tct_near_plan_build")
    return handle


def get_nearfield_device(obs_centers, obs_radii, src_centers, src_radii, threshold,
                         n_threads=0, stream=None, device_tree=True):
    """get_nearfield on the GPU -- octrees, dual traversal (device_tree;
    else on the host), ball tests, row fill and row sort: the same pairs in
    the same order, as an int64 (P, 2) CUDA tensor."""
    from ..util import device
    t = device.require_cuda()
    handle = near_plan(obs_centers, obs_radii, src_centers, src_radii, threshold, n_threads,
                       device_tree=device_tree, stream=stream)
    try:
        s = _lib.stream_ptr(stream)
        total = ctypes.c_int64()
        _lib.check(_lib.lib.tct_near_device_count(handle, s, ctypes.byref(total)),
                   "tct_near_device_count")
        out = t.empty((total.value, 2), dtype=t.int64, device="cuda")
        _lib.check(_lib.lib.tct_near_device_fill(handle, ctypes.c_void_p(out.data_ptr()), s),
                   "tct_near_device_fill")
        # the plan's device buffers are released after the fill has run
        t.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
    finally:
        _lib.lib.tct_near_plan_free(handle)
    return out


# meshes from this many triangles search on the GPU when one is visible
DEVICE_NEAR_MIN_TRIS = 100_000


def find_close_or_touching(a_pts, a_tris, b_pts, b_tris, threshold):
    """Pairs (i in a, j in b) whose bounding balls, scaled by `threshold`,
    touch (find_near_adj.py:29-35).  Large meshes use the device search when
    a GPU is visible; both give the same pairs in the same order."""
    ca, ra = get_tri_centroids_rs(a_pts, a_tris)
    if (a_pts is b_pts or np.array_equal(a_pts, b_pts)) and np.array_equal(a_tris, b_tris):
        cb, rb = ca, ra  # a self search: one set of balls (and one octree)
    else:
        cb, rb = get_tri_centroids_rs(b_pts, b_tris)
    if max(ca.shape[0], cb.shape[0]) >= DEVICE_NEAR_MIN_TRIS:
        from ..util import device
        if device.cuda_available():
            return get_nearfield_device(ca, ra, cb, rb, threshold).cpu().numpy()
    return get_nearfield(ca, ra, cb, rb, threshold)


def split_adjacent_close(close_pairs, tris_a, tris_b):
    """(near (n,2), vertex-adjacent (n,4), edge-adjacent (n,6)) by shared-vertex
    count; coincident pairs are dropped (fast_find_nearfield.cpp:143-182)."""
    cp = np.ascontiguousarray(close_pairs, dtype=np.int64).reshape(-1, 2)
    ta = np.ascontiguousarray(tris_a, dtype=np.int64).reshape(-1, 3)
    tb = np.ascontiguousarray(tris_b, dtype=np.int64).reshape(-1, 3)
    n = cp.shape[0]
    near = np.empty((max(n, 1), 2), dtype=np.int64)
    va = np.empty((max(n, 1), 4), dtype=np.int64)
    ea = np.empty((max(n, 1), 6), dtype=np.int64)
    nn, nv, ne = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    _lib.check(_lib.lib.tct_split_adjacent_close(
        _lib.i64ptr(cp), n, _lib.i64ptr(ta), _lib.i64ptr(tb), _lib.i64ptr(near), ctypes.byref(nn),
        _lib.i64ptr(va), ctypes.byref(nv), _lib.i64ptr(ea), ctypes.byref(ne)),
        "tct_split_adjacent_close")
    return near[:nn.value].copy(), va[:nv.value].copy(), ea[:ne.value].copy()


def split_vertex_nearfield(close_pairs, obs_pts, src_pts, src_tris):
    """(vertex_pairs, near_pairs) of point-triangle pairs
    (fast_find_nearfield.cpp:184-215): a pair whose observation point lies
    within 1e-9 of a source vertex d becomes (obs, tri, d) (the last such d),
    any other (obs, tri, 0); input order kept."""
    close_pairs = np.asarray(close_pairs, dtype=np.int64).reshape(-1, 2)
    obs_pts = np.asarray(obs_pts, dtype=np.float64)
    src_pts = np.asarray(src_pts, dtype=np.float64)
    src_tris = np.asarray(src_tris, dtype=np.int64)
    if close_pairs.shape[0] == 0:
        e = np.empty((0, 3), dtype=np.int64)
        return e, e.copy()
    o = obs_pts[close_pairs[:, 0]]
    corner = np.full(close_pairs.shape[0], -1, dtype=np.int64)
    for d in range(3):
        v = src_pts[src_tris[close_pairs[:, 1], d]]
        dist = np.sqrt(np.sum((o - v) ** 2, axis=1))
        corner[dist < 1e-9] = d
    isv = corner >= 0
    vertex = np.column_stack([close_pairs[isv], corner[isv]])
    near = np.column_stack([close_pairs[~isv], np.zeros((~isv).sum(), dtype=np.int64)])
    return vertex, near
