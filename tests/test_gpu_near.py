"""Device near-pair search against the host search, which is pinned
bit-exactly to the reference's compiled finder and golden masters
(tests/test_near_adj.py): the same pairs in the same (obs, src) order, with
the octrees and traversal on the GPU (csrc/tree_dev.cu, the default) and on
the host (host.cpp); and the device octree against the host octree, node for
node."""
import numpy as np
import pytest

from tectosaur_b200.mesh import find_near_adj as fna
from tectosaur_b200.mesh.mesh_gen import make_rect

from helpers import bumpy_mesh

pytestmark = pytest.mark.gpu

CORNERS = [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]]


def both(c, r, sc, sr, thr):
    host = fna.get_nearfield(c, r, sc, sr, thr)
    dev = fna.get_nearfield_device(c, r, sc, sr, thr).cpu().numpy()
    dev_hostplan = fna.get_nearfield_device(c, r, sc, sr, thr, device_tree=False).cpu().numpy()
    assert np.array_equal(dev_hostplan, host)
    return host, dev


def test_golden_rect(cuda, golden):
    g = golden("ref_goldens.npz")
    pts, tris = make_rect(20, 20, CORNERS)
    c, r = fna.get_tri_centroids_rs(pts, tris)
    host, dev = both(c, r, c, r, 1.25)
    assert np.array_equal(dev, host)
    assert np.array_equal(np.sort(dev, axis=0), g["test_close_or_touching"])


def test_golden_sphere(cuda, golden):
    g = golden("ref_goldens.npz")
    sp, st = g["sphere_pts"], g["sphere_tris"]
    c, r = fna.get_tri_centroids_rs(sp, st)
    for thr in (1.25, 2.5):
        host, dev = both(c, r, c, r, thr)
        assert np.array_equal(dev, host)


def test_notself_zero_radius_obs(cuda):
    pts, tris = make_rect(2, 2, CORNERS)
    obs = np.array([0.5 * np.ones(5), 0.5 * np.ones(5), np.linspace(0, 2, 5)]).T.copy()
    c, r = fna.get_tri_centroids_rs(pts, tris)
    host, dev = both(obs, np.zeros(5), c, r, 1.0)
    assert np.array_equal(dev, host)


@pytest.mark.parametrize("n,thr", [(40, 2.5), (75, 1.25), (120, 2.5), (300, 2.5)])
def test_bumpy_meshes(cuda, n, thr):
    pts, tris = bumpy_mesh(n, seed=n)
    c, r = fna.get_tri_centroids_rs(pts, tris)
    host, dev = both(c, r, c, r, thr)
    assert dev.shape[0] > 0 and np.array_equal(dev, host)


def test_two_meshes_and_empty(cuda):
    a_pts, a_tris = bumpy_mesh(30, seed=1)
    b_pts, b_tris = bumpy_mesh(45, seed=2)
    ca, ra = fna.get_tri_centroids_rs(a_pts, a_tris)
    cb, rb = fna.get_tri_centroids_rs(b_pts, b_tris)
    host, dev = both(ca, ra, cb, rb, 2.0)
    assert np.array_equal(dev, host)
    out = fna.get_nearfield_device(np.zeros((0, 3)), np.zeros(0), cb, rb, 1.0)
    assert tuple(out.shape) == (0, 2)
    out = fna.get_nearfield_device(ca, ra, cb + 1e3, rb, 1.0)  # far apart: nothing
    assert tuple(out.shape) == (0, 2)


def _trees_equal(c, r, leaf):
    from tectosaur_b200.fmm.tree import Tree
    a = Tree(c, r, leaf, device=True)
    b = Tree(c, r, leaf, device=False)
    assert a.on_device and not b.on_device
    assert a.n_nodes == b.n_nodes and a.max_height == b.max_height
    for name in ("orig_idxs", "start", "end", "centers", "R", "is_leaf", "depth", "height",
                 "children"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    return a


@pytest.mark.parametrize("n,leaf", [(40, 50), (120, 50), (300, 50), (300, 128), (60, 1)])
def test_device_octree_equals_host_octree(cuda, n, leaf):
    pts, tris = bumpy_mesh(n, seed=n + 1)
    c, r = fna.get_tri_centroids_rs(pts, tris)
    t = _trees_equal(c, r, leaf)
    assert t.n_nodes > 1


def test_device_octree_edge_cases(cuda, golden):
    g = golden("ref_goldens.npz")
    c, r = fna.get_tri_centroids_rs(g["sphere_pts"], g["sphere_tris"])
    _trees_equal(c, r, 50)
    _trees_equal(c, r, 3)
    # 120 identical centres: the depth cap ends the splitting
    cc = np.tile([[0.3, -0.2, 0.1]], (120, 1))
    _trees_equal(cc, np.full(120, 0.01), 50)
    _trees_equal(cc[:1], np.full(1, 0.01), 50)       # one ball
    _trees_equal(np.zeros((0, 3)), np.zeros(0), 50)  # none
    rng = np.random.default_rng(3)
    pc = rng.standard_normal((5000, 3))
    _trees_equal(pc, np.zeros(5000), 50)             # zero-radius points


def test_c4_like_two_part_mesh(cuda):
    # a surface and a buried dipping fault in one mesh (the 1M-triangle
    # configuration's layout), at 75k triangles
    from tectosaur_b200.mesh.mesh_gen import concat_no_dedupe
    s = make_rect(181, 181, [[-50, -50, 0], [50, -50, 0], [50, 50, 0], [-50, 50, 0]])
    f = make_rect(37, 19, [[-10, 0, -0.5], [10, 0, -0.5], [10, 8.66, -5.5], [-10, 8.66, -5.5]])
    pts, tris = concat_no_dedupe(s, f)
    c, r = fna.get_tri_centroids_rs(pts, tris)
    _trees_equal(c, r, 128)
    host, dev = both(c, r, c, r, 2.5)
    assert np.array_equal(dev, host)
