"""Near-pair search, adjacency split and edge orientation (host C++ in
libtct_b200.so) against the reference's golden masters and its compiled
C++ (oracle/_ref, when built)."""
import importlib.machinery
import importlib.util
import os

import numpy as np
import pytest

from tectosaur_b200.mesh import find_near_adj as fna
from tectosaur_b200.mesh.mesh_gen import make_rect
from tectosaur_b200.nearfield.nearfield_op import resolve_ea_rotation, to_dof_space

from helpers import bumpy_mesh

REF_BUILD = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                         "_ref")


def lexsorted(a):
    a = np.asarray(a)
    if a.shape[0] == 0:
        return a
    return a[np.lexsort(a.T[::-1])]


def test_find_adjacents_small():
    # tests/test_find_near_adj.py:11-23 (there the edge-adjacent rows carry
    # only their two triangle indices; now they carry 6 columns)
    tris = np.array([[0, 1, 2], [2, 1, 3], [0, 4, 5]])
    pts = np.random.default_rng(0).random((6, 3))
    close = fna.find_close_or_touching(pts, tris, pts, tris, 1.0)
    _, va, ea = fna.split_adjacent_close(close, tris, tris)
    assert va.size == 8
    assert np.all(lexsorted(va).flatten() == (0, 2, 0, 0, 2, 0, 0, 0))
    assert np.all(lexsorted(ea)[:, :2].flatten() == (0, 1, 1, 0))


def test_nearfield_3x3():
    # tests/test_find_near_adj.py:25-37
    pts, tris = make_rect(3, 3, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]])
    assert tris.shape[0] == 8
    close = fna.find_close_or_touching(pts, tris, pts, tris, 1.0)
    near, va, ea = fna.split_adjacent_close(close, tris, tris)
    check_for = [(0, 5), (0, 6), (0, 3), (1, 7), (2, 7), (3, 0), (4, 7), (5, 0), (6, 0), (7, 2),
                 (7, 1), (7, 4)]
    assert len(near) == len(check_for)
    found = set(map(tuple, near.tolist()))
    assert found == set(check_for)


def test_close_or_touching_golden(golden):
    g = golden("ref_goldens.npz")
    pts, tris = make_rect(20, 20, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]])
    pairs = fna.find_close_or_touching(pts, tris, pts, tris, 1.25)
    assert np.array_equal(np.sort(pairs, axis=0), g["test_close_or_touching"])


def test_find_nearfield_real_golden(golden):
    g = golden("ref_goldens.npz")
    pts, tris = make_rect(20, 20, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]])
    close, va, ea = fna.split_adjacent_close(
        fna.find_close_or_touching(pts, tris, pts, tris, 1.25), tris, tris)
    assert np.array_equal(close[np.lexsort([close[:, 1], close[:, 0]])].flatten(),
                          g["test_find_nearfield_real"])


def test_find_adjacency_golden(golden):
    g = golden("ref_goldens.npz")
    sp, st = g["sphere_pts"], g["sphere_tris"]
    close, va, ea = fna.split_adjacent_close(fna.find_close_or_touching(sp, st, sp, st, 1.25),
                                             st, st)
    allp = np.zeros((va.shape[0] + ea.shape[0], 4))
    allp[:va.shape[0]] = va
    allp[va.shape[0]:, :2] = ea[:, :2]
    out = allp[np.lexsort([allp[:, 1], allp[:, 0]])]
    assert np.array_equal(out, g["test_find_adjacency"])


def test_find_close_notself_golden(golden):
    g = golden("ref_goldens.npz")
    pts, tris = make_rect(2, 2, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]])
    obs = np.array([0.5 * np.ones(5), 0.5 * np.ones(5), np.linspace(0, 2, 5)]).T.copy()
    c, r = fna.get_tri_centroids_rs(pts, tris)
    out = fna.get_nearfield(obs, np.zeros(5), c, r, 1.0)
    assert np.array_equal(lexsorted(out), lexsorted(g["test_find_close_notself"]))


@pytest.mark.parametrize("name", ["rect_1p25", "rect_2p5", "sphere_1p25", "sphere_2p5",
                                  "bumpy_1p25", "bumpy_2p5"])
def test_split_and_orientation_vs_reference(golden, name):
    g = golden("near_split.npz")
    pts, tris = g[name + "_pts"], g[name + "_tris"]
    thr = float(name.split("_")[1].replace("p", "."))
    pairs = fna.find_close_or_touching(pts, tris, pts, tris, thr)
    # canonical order == reference order after lexsort (the reference's raw
    # order depends on OpenMP thread completion)
    assert np.array_equal(pairs, lexsorted(g[name + "_pairs_raw"]))
    close, va, ea = fna.split_adjacent_close(pairs, tris, tris)
    assert np.array_equal(lexsorted(close), lexsorted(g[name + "_close"]))
    assert np.array_equal(lexsorted(va), lexsorted(g[name + "_va"]))
    assert np.array_equal(lexsorted(ea), lexsorted(g[name + "_ea"]))
    rot = resolve_ea_rotation(tris, ea)
    assert np.array_equal(lexsorted(rot), lexsorted(g[name + "_ea_rot"]))
    # same rows in the reference's raw order give the same records
    rot_ref_order = resolve_ea_rotation(tris, g[name + "_ea"])
    assert np.array_equal(rot_ref_order, g[name + "_ea_rot"])


def test_empty_and_degenerate_inputs():
    out = fna.get_nearfield(np.zeros((0, 3)), np.zeros(0), np.zeros((4, 3)), np.ones(4), 1.0)
    assert out.shape == (0, 2)
    out = fna.get_nearfield(np.zeros((3, 3)), np.zeros(3), np.zeros((0, 3)), np.zeros(0), 1.0)
    assert out.shape == (0, 2)
    # coincident centres, zero radii: touching at distance 0
    out = fna.get_nearfield(np.zeros((2, 3)), np.zeros(2), np.zeros((3, 3)), np.zeros(3), 1.0)
    assert out.shape == (6, 2)
    near, va, ea = fna.split_adjacent_close(np.zeros((0, 2), np.int64), np.zeros((0, 3), np.int64),
                                            np.zeros((0, 3), np.int64))
    assert near.shape == (0, 2) and va.shape == (0, 4) and ea.shape == (0, 6)


def test_to_dof_space_subsets():
    obs = np.array([5, 2, 9])
    src = np.array([1, 9, 5])
    out = to_dof_space(np.array([[5, 9], [9, 1], [2, 5]]), obs, src)
    assert np.array_equal(out, [[0, 1], [2, 0], [1, 2]])


def _load_ref_finder():
    for suffix in importlib.machinery.EXTENSION_SUFFIXES:
        path = os.path.join(REF_BUILD, "fast_find_nearfield" + suffix)
        if os.path.exists(path):
            spec = importlib.util.spec_from_file_location("fast_find_nearfield", path)
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            return mod
    return None


@pytest.mark.parametrize("n,thr", [(40, 2.5), (75, 1.25), (120, 2.5), (180, 2.5)])
def test_bit_exact_vs_compiled_reference(n, thr):
    ref = _load_ref_finder()
    if ref is None:
        pytest.skip("reference C++ not compiled (make -C oracle ref)")
    pts, tris = bumpy_mesh(n, seed=n)
    c, r = fna.get_tri_centroids_rs(pts, tris)
    mine = fna.get_nearfield(c, r, c, r, thr)
    theirs = ref.get_nearfield(c, r, c, r, thr, 50)
    assert np.array_equal(mine, lexsorted(theirs))
    a = ref.split_adjacent_close(theirs, tris, tris)
    b = fna.split_adjacent_close(mine, tris, tris)
    for x, y in zip(a, b):
        assert np.array_equal(lexsorted(x), lexsorted(y))


def test_device_plan_builds_on_host():
    """The host half of the device search (octrees + traversal to leaf pairs)
    needs no GPU: leaf pairs exist for a touching mesh, none for far meshes."""
    from tectosaur_b200 import _lib
    pts, tris = bumpy_mesh(40, seed=40)
    c, r = fna.get_tri_centroids_rs(pts, tris)
    h = fna.near_plan(c, r, c, r, 2.5)
    try:
        assert _lib.lib.tct_near_plan_leaf_pairs(h) > 0
    finally:
        _lib.lib.tct_near_plan_free(h)
    h = fna.near_plan(c, r, c + 1e3, r, 2.5)
    try:
        assert _lib.lib.tct_near_plan_leaf_pairs(h) == 0
    finally:
        _lib.lib.tct_near_plan_free(h)

