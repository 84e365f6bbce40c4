"""Device near-pair search (csrc/near.cu + the host traversal in host.cpp)
against the host search, which is pinned bit-exactly to the reference's
compiled finder and golden masters (tests/test_near_adj.py): the same pairs
in the same (obs, src) order."""
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
