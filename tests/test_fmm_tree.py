"""Treecode trees and interaction lists vs the reference's compiled C++
(fmm/octree.cpp + fmm/traversal.cpp in oracle/_ref) -- bit-exact."""
import importlib.machinery
import importlib.util
import os

import numpy as np
import pytest

from tectosaur_b200.fmm.tree import Tree, tri_centers_radii, treecode_interactions

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


@pytest.mark.parametrize("n,leaf", [(12, 2), (25, 20), (40, 100)])
def test_tree_matches_reference(n, leaf):
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


def test_treecode_rejects_unsupported_kernel():
    from tectosaur_b200.fmm.tsfmm import TSFMM
    from tectosaur_b200.mesh.mesh_gen import make_rect
    m = make_rect(4, 4, [[-1, -1, 0], [-1, 1, 0], [1, 1, 0], [1, -1, 0]])
    with pytest.raises(ValueError, match="treecode supports"):
        TSFMM(m, m, [1.0, 0.25], 4, 2, np.float64, "elasticH3", 2.5, 2)


def test_treecode_abi_rejects_bad_order():
    from tectosaur_b200 import _lib
    assert _lib.lib.tct_treecode_workspace_bytes(6, 1, 13, 10, 10, 5, 3) == 0
    assert _lib.lib.tct_treecode_workspace_bytes(3, 1, 8, 10, 10, 5, 3) == 0  # elasticH3
    assert _lib.lib.tct_treecode_workspace_bytes(6, 1, 8, 10, 10, 5, 3) > 0
