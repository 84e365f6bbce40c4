"""Synthetic triangle meshes (same vertex and triangle order as the
reference's tectosaur/mesh/mesh_gen.py:7-47): a bilinear quadrilateral patch
sampled on an nx x ny grid, two triangles per cell."""
import numpy as np


def rect_points(corners, xhat_vals, yhat_vals):
    """Bilinear map of the grid (xhat, yhat) onto the quadrilateral with
    corners ordered lower-left, lower-right, upper-right, upper-left."""
    nx = xhat_vals.shape[0]
    ny = yhat_vals.shape[0]
    corners = np.array(corners)
    rect_basis = [
        lambda x, y: x * y,
        lambda x, y: (1 - x) * y,
        lambda x, y: (1 - x) * (1 - y),
        lambda x, y: x * (1 - y),
    ]
    X, Y = np.meshgrid(xhat_vals, yhat_vals)
    vertices = np.vstack((X.reshape(nx * ny), Y.reshape(nx * ny))).T
    return np.sum([
        np.outer(rect_basis[i](vertices[:, 0], vertices[:, 1]), corners[i, :])
        for i in range(4)
    ], axis=0)


def rect_topology(nx, ny):
    """Cells in column-major order (i outer, j inner); cell (i, j) gives
    [tl, bl, tr] and [bl, br, tr] with v(i, j) = j * nx + i."""
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="ij")
    i = i.reshape(-1)
    j = j.reshape(-1)
    tl = j * nx + i
    tr = j * nx + i + 1
    bl = (j + 1) * nx + i
    br = (j + 1) * nx + i + 1
    tris = np.empty((2 * i.shape[0], 3), dtype=np.int64)
    tris[0::2] = np.stack([tl, bl, tr], axis=1)
    tris[1::2] = np.stack([bl, br, tr], axis=1)
    return tris


def make_rect(nx, ny, corners):
    x = np.linspace(0, 1, nx)
    y = np.linspace(0, 1, ny)
    return rect_points(corners, x, y), rect_topology(nx, ny)


def concat_no_dedupe(*ms):
    """Stack meshes (vertex indices of later meshes offset)."""
    pts = []
    tris = []
    off = 0
    for p, t in ms:
        pts.append(p)
        tris.append(np.asarray(t) + off)
        off += p.shape[0]
    return np.vstack(pts), np.vstack(tris)
