"""Treecode trees and interaction lists vs the reference's compiled C++
(fmm/octree.cpp + fmm/traversal.cpp in oracle/_ref) -- bit-exact."""
import importlib.machinery
import importlib.util
import os

import numpy as np
import pytest

from tectosaur_b200.fmm.tree import Tree, interactions, tri_centers_radii, treecode_interactions

from helpers import bumpy_mesh, two_surfaces

REF_BUILD = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                         "_ref")


def _ref():
    for suffix in importlib.machinery.EXTENSION_SUFFIXES:
        path = os.path.join(REF_BUILD, "traversal_wrapper" + suffix)
        if os.path.exists(path):
            spec = importlib.util.spec_from_file_location("traversal_wrapper", path)
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            return mod.three.octree
    pytest.skip("reference C++ not compiled (make -C oracle ref)")


@pytest.mark.parametrize("n,leaf", [(12, 2), (25, 20), (40, 100), (180, 50), (200, 128)])
def test_tree_matches_reference(n, leaf):
    # n = 180, 200: 64 k and 79 k balls, built with threads (subtrees spliced
    # into the serial depth-first order)
    ref = _ref()
    pts, tris = bumpy_mesh(n, seed=n)
    c, r = tri_centers_radii(pts, tris)
    mine = Tree(c, r, leaf)
    theirs = ref.Tree.build(c, r, leaf)
    assert mine.n_nodes == theirs.n_nodes
    assert mine.max_height == theirs.max_height
    assert np.array_equal(mine.orig_idxs, np.array(theirs.orig_idxs))
    assert np.array_equal(mine.centers, np.array(theirs.node_centers))
    assert np.array_equal(mine.R, np.array(theirs.node_Rs))
    for k, nd in enumerate(theirs.nodes):
        assert (mine.start[k], mine.end[k], bool(mine.is_leaf[k]), mine.depth[k],
                mine.height[k]) == (nd.start, nd.end, nd.is_leaf, nd.depth, nd.height)
        if not nd.is_leaf:
            assert list(mine.children[k]) == list(nd.children)


@pytest.mark.parametrize("mac,leaf,offset", [(2.5, 2, 0.0), (3.0, 20, 0.0), (2.5, 10, 6.0)])
def test_treecode_lists_match_reference(mac, leaf, offset):
    ref = _ref()
    (pts, tris), s1, s2 = two_surfaces(n=16, sep=1.0)
    pts = pts.copy()
    pts[tris[s1].reshape(-1), 0] += offset
    co, ro = tri_centers_radii(pts, tris[s1])
    cs, rs = tri_centers_radii(pts, tris[s2])
    mo, ms = Tree(co, ro, leaf), Tree(cs, rs, leaf)
    to, ts = ref.Tree.build(co, ro, leaf), ref.Tree.build(cs, rs, leaf)
    p2p, m2p = treecode_interactions(mo, ms, 1.0, mac, 0, True)
    ri = ref.fmmmm_interactions(to, ts, 1.0, mac, 0, True)
    for mine, theirs in [(p2p, ri.p2p), (m2p, ri.m2p)]:
        assert np.array_equal(mine.obs_n_idxs, np.array(theirs.obs_n_idxs))
        assert np.array_equal(mine.obs_src_starts, np.array(theirs.obs_src_starts))
        assert np.array_equal(mine.src_n_idxs, np.array(theirs.src_n_idxs))


@pytest.mark.parametrize("order,inner", [(0, 2.5), (10, 1.0), (60, 2.0)])
def test_fmm_lists_match_reference(order, inner):
    """Without the treecode flag the traversal also yields P2L and M2L lists
    (and M2P / P2P for small nodes, by `order`)."""
    ref = _ref()
    (pts, tris), s1, s2 = two_surfaces(n=18, sep=0.7)
    co, ro = tri_centers_radii(pts, tris[s1])
    cs, rs = tri_centers_radii(pts, tris[s2])
    mo, ms = Tree(co, ro, 8), Tree(cs, rs, 8)
    to, ts = ref.Tree.build(co, ro, 8), ref.Tree.build(cs, rs, 8)
    mine = interactions(mo, ms, inner, 2.5, order, False)
    ri = ref.fmmmm_interactions(to, ts, inner, 2.5, order, False)
    if order == 0:
        assert mine["m2l"].src_n_idxs.shape[0] > 0 and mine["m2p"].src_n_idxs.shape[0] == 0
    for name in ["p2p", "m2p", "p2l", "m2l"]:
        theirs = getattr(ri, name)
        assert np.array_equal(mine[name].obs_n_idxs, np.array(theirs.obs_n_idxs)), name
        assert np.array_equal(mine[name].obs_src_starts, np.array(theirs.obs_src_starts)), name
        assert np.array_equal(mine[name].src_n_idxs, np.array(theirs.src_n_idxs)), name


def test_tree_parent_and_levels():
    pts, tris = bumpy_mesh(20, seed=4)
    t = Tree(*tri_centers_radii(pts, tris), 5)
    inner = np.nonzero(t.is_leaf == 0)[0]
    for k in inner:
        assert np.all(t.parent[t.children[k]] == k)
    assert t.parent[0] == -1 and np.sum(t.parent < 0) == 1
    nodes, off = t.m2m_levels()
    assert np.all(np.diff(t.height[nodes]) >= 0) and np.all(t.is_leaf[nodes] == 0)
    assert nodes.shape[0] == inner.shape[0]
    nodes, off = t.l2l_levels()
    assert np.all(np.diff(t.depth[nodes]) >= 0) and nodes.shape[0] == t.n_nodes - 1


def test_treecode_rejects_unsupported_kernel():
    from tectosaur_b200.fmm.tsfmm import TSFMM
    from tectosaur_b200.mesh.mesh_gen import make_rect
    m = make_rect(4, 4, [[-1, -1, 0], [-1, 1, 0], [1, 1, 0], [1, -1, 0]])
    with pytest.raises(ValueError, match="treecode supports"):
        TSFMM(m, m, [1.0, 0.25], 4, 2, np.float64, "elasticH3", 2.5, 2)


def test_fmm_abi_rejects_bad_arguments():
    from tectosaur_b200 import _lib
    ws = _lib.lib.tct_fmm_workspace_bytes
    assert ws(6, 1, 0, 13, 3, 10, 10, 5, 5) == 0  # order > 12
    assert ws(3, 1, 0, 8, 3, 10, 10, 5, 5) == 0  # elasticH3
    assert ws(6, 1, 2, 8, 3, 10, 10, 5, 5) == 0  # mode
    assert ws(6, 1, 0, 8, 6, 10, 10, 5, 5) == 0  # 6-point rule
    assert ws(6, 1, 0, 8, 3, 10, 10, 5, 5) > 0
    assert ws(6, 1, 1, 8, 3, 10, 10, 5, 5) > ws(6, 1, 0, 8, 3, 10, 10, 5, 5)  # locals


@pytest.mark.parametrize("lanes", [192, 224])
@pytest.mark.parametrize("nb", [1, 2, 3, 4, 6, 9])
@pytest.mark.parametrize("p", range(13))
def test_m2l_plan_covers_every_pair(p, nb, lanes):
    """The M2L work plan (csrc/fmm.cu m2l3_make_plan, built on the host here)
    covers every (a, b) with |a| + |b| <= p exactly once, within the lanes.
    FP32 uses nb = 3 (elasticRH3), 4 (RA), 6 (RT) or 9 (U) terms per lane, on
    192 lanes (two source nodes per stage) or 224 (one)."""
    import ctypes
    from tectosaur_b200 import _lib
    out = (ctypes.c_int64 * 5)()
    rc = _lib.lib.tct_fmm_m2l_plan_stats(p, nb, lanes, out)
    nt = (p + 1) * (p + 2) * (p + 3) // 6
    if nb < 3 and -(-nt // nb) > lanes - 10:
        return  # more tuples than lanes: the item form runs instead (rc may be 0 or 1)
    assert rc == 0  # every FP32 configuration (nb >= 3) fits
    covered, bad, L, used, steps = list(out)
    total = (p + 1) * (p + 2) * (p + 3) * (p + 4) * (p + 5) * (p + 6) // 720
    assert covered == total and bad == 0
    assert 1 <= used <= lanes
    if p == 8 and nb == 3:
        assert (L, used) == ((7, 181) if lanes == 192 else (6, 209))


def test_m2l_plan_rejects_bad_lane_counts():
    import ctypes
    from tectosaur_b200 import _lib
    out = (ctypes.c_int64 * 5)()
    for lanes in (0, 100, 256):
        assert _lib.lib.tct_fmm_m2l_plan_stats(8, 3, lanes, out) != 0


@pytest.mark.parametrize("world", [2, 3, 5])
def test_row_shard_restriction(world):
    """A row shard's FMM observation side: a node is kept iff it holds a
    triangle of the range, every ancestor of a kept node is kept, the kept
    leaves hold every row of the range, and each kept list entry keeps its
    whole source list; over a partition of the rows every list entry is
    kept by some shard (but those of empty octree children)."""
    from tectosaur_b200.fmm.tsfmm import restrict_list, touching_nodes
    from tectosaur_b200.sharded import row_ranges
    pts, tris = bumpy_mesh(20, seed=1, amp=0.3)
    c, r = tri_centers_radii(pts, tris)
    tree = Tree(c, r, 25, device=False)
    lists = interactions(tree, tree, 3.0, 3.0, 0, False)
    n = tris.shape[0]
    pos_of = np.empty(n, np.int64)
    pos_of[tree.orig_idxs] = np.arange(n)
    seen = {k: np.zeros(v.obs_n_idxs.shape[0], bool) for k, v in lists.items()}
    for r0, r1 in row_ranges(n, world):
        touch = touching_nodes(tree, r0, r1)
        for k in range(tree.n_nodes):
            rows = tree.orig_idxs[tree.start[k]:tree.end[k]]
            assert touch[k] == bool(((rows >= r0) & (rows < r1)).any())
        kept = np.nonzero(touch)[0]
        par = tree.parent[kept]
        assert touch[par[par >= 0]].all()
        leaves = tree.leaves()[touch[tree.leaves()]]
        covered = np.zeros(n, bool)
        for lf in leaves:
            covered[tree.orig_idxs[tree.start[lf]:tree.end[lf]]] = True
        assert covered[r0:r1].all()
        for name, lst in lists.items():
            sub = restrict_list(lst, touch)
            assert np.all(touch[sub.obs_n_idxs])
            for j, o in enumerate(sub.obs_n_idxs):
                i = int(np.nonzero(lst.obs_n_idxs == o)[0][0])
                full_src = lst.src_n_idxs[lst.obs_src_starts[i]:lst.obs_src_starts[i + 1]]
                assert np.array_equal(
                    sub.src_n_idxs[sub.obs_src_starts[j]:sub.obs_src_starts[j + 1]], full_src)
            seen[name] |= touch[lst.obs_n_idxs]
    nonempty = tree.end > tree.start  # empty octree children hold no rows and do no work
    for name, lst in lists.items():
        assert seen[name][nonempty[lst.obs_n_idxs]].all()
