"""Singular 4-D quadrature rules over a pair of reference triangles (host, FP64).

Each rule returns ``(pts, wts)`` with ``pts[:, 0:2]`` the observation-triangle
reference coordinates (xhat, yhat) and ``pts[:, 2:4]`` the source-triangle
ones, ordered exactly as the reference's nested loops emit them
(``tectosaur/nearfield/triangle_rules.py``), so the device kernels see the
reference's rules point for point.  The loops are vectorised here over their
inner dimensions with the same floating-point expression order.

* ``coincident_quad(nq)``  – Erichsen & Sauter (1998) six-simplex split of the
  coincident pair (triangle_rules.py:71-139): 6 x |tri(nq)| x nq x nq points.
* ``edge_adj_quad(nq)``    – Sauter & Schwab edge-adjacent split, five
  4-cube mappings with polynomial Jacobians (:141-206): 5 x nq^4 points; the
  source triangle is reflected so the shared edge is (0,0)-(1,0) in both.
* ``vertex_adj_quad(nt, nb, na)`` – polar coordinates about the shared vertex
  in both triangles, the radial pair written as (a cos b, a sin b) with the b
  range split where one triangle's radial limit takes over (:24-69):
  2 x nt^2 x nb x na points.
"""
import functools

import numpy as np

from ..util import quadrature as quad


def _spow(x, k):
    """Elementwise x**k through the C library's scalar pow.

    NumPy's vectorised power may differ from scalar pow in the last bit; the
    reference evaluates these powers one scalar at a time.
    """
    flat = np.asarray(x, dtype=np.float64)
    out = np.array([float(v) ** k for v in flat.reshape(-1)])
    return out.reshape(flat.shape)


def _rho_max(theta):
    return 1.0 / (np.cos(theta) + np.sin(theta))


@functools.lru_cache(maxsize=None)
def _vertex_adj_cached(n_theta, n_beta, n_alpha):
    theta_q = quad.map_to(quad.gaussxw(n_theta), [0, np.pi / 2])
    beta_quad = quad.gaussxw(n_beta)
    alpha_quad = quad.gaussxw(n_alpha)
    pts = []
    wts = []
    for tp, tpw in zip(*theta_q):
        for tq, tqw in zip(*theta_q):
            w_pq = tpw * tqw
            beta_split = np.arctan(_rho_max(tq) / _rho_max(tp))
            for beta_min, beta_max, first in ((0, beta_split, True),
                                             (beta_split, np.pi / 2, False)):
                bq = quad.map_to(beta_quad, [beta_min, beta_max])
                for b, bw in zip(*bq):
                    if first:
                        alpha_max = _rho_max(tp) / np.cos(b)
                    else:
                        alpha_max = _rho_max(tq) / np.sin(b)
                    a, aw = quad.map_to(alpha_quad, [0, alpha_max])
                    cb = np.cos(b)
                    sb = np.sin(b)
                    jac = _spow(a, 3) * cb * sb
                    rho_p = a * cb
                    rho_q = a * sb
                    blk = np.empty((a.shape[0], 4))
                    blk[:, 0] = rho_p * np.cos(tp)
                    blk[:, 1] = rho_p * np.sin(tp)
                    blk[:, 2] = rho_q * np.cos(tq)
                    blk[:, 3] = rho_q * np.sin(tq)
                    pts.append(blk)
                    wts.append(jac * aw * (bw * w_pq))
    return np.concatenate(pts), np.concatenate(wts)


def vertex_adj_quad(n_theta, n_beta, n_alpha):
    p, w = _vertex_adj_cached(int(n_theta), int(n_beta), int(n_alpha))
    return p.copy(), w.copy()


def _coincident_maps(eta, w1, w2, w3):
    a = w1 + w2 + w3
    b = w1 * (1 - eta) + w2 + w3
    c = w1 * (1 - eta) + w2
    return [
        (a, w1 + w2, b, w2),
        (b, c, a, w2),
        (a, w1 * eta + w2, w2 + w3, w2),
        (b, w2, a, w1 + w2),
        (a, w2, b, c),
        (w2 + w3, w2, a, w1 * eta + w2),
    ]


@functools.lru_cache(maxsize=None)
def _coincident_cached(nq):
    qtri = quad.gauss2d_tri(nq)
    qline = quad.map_to(quad.gaussxw(nq), [0.0, 1.0])
    w1 = qtri[0][:, 0][:, None, None]
    w2 = qtri[0][:, 1][:, None, None]
    f12 = qtri[1][:, None, None]
    x3 = qline[0][None, :, None]
    f3 = qline[1][None, :, None]
    eta = qline[0][None, None, :]
    feta = qline[1][None, None, :]
    w3 = x3 * (1 - w1 - w2)
    f3s = f3 * (1 - w1 - w2)
    F = f12 * f3s * feta * w1
    shape = np.broadcast(w1, x3, eta).shape
    pts = []
    wts = []
    for x1, x2, y1, y2 in _coincident_maps(eta, w1, w2, w3):
        blk = np.empty(shape + (4,))
        blk[..., 0] = 1 - np.broadcast_to(x1, shape)
        blk[..., 1] = np.broadcast_to(x2, shape)
        blk[..., 2] = 1 - np.broadcast_to(y1, shape)
        blk[..., 3] = np.broadcast_to(y2, shape)
        pts.append(blk.reshape(-1, 4))
        wts.append(np.broadcast_to(F, shape).reshape(-1))
    return np.concatenate(pts), np.concatenate(wts)


def coincident_quad(nq):
    p, w = _coincident_cached(int(nq))
    return p.copy(), w.copy()


def _edge_maps(e1, e2, e3, P):
    P3 = _spow(P, 3)
    e1sq = _spow(e1, 2)
    return [
        (P, P * e1 * e3, P * (1 - e1 * e2), P * e1 * (1 - e2), P3 * e1sq),
        (P, P * e1, P * (1 - e1 * e2 * e3), P * e1 * e2 * (1 - e3),
         P3 * e1sq * e2),
        (P * (1 - e1 * e2), P * e1 * (1 - e2), P, P * e1 * e2 * e3,
         P3 * e1sq * e2),
        (P * (1 - e1 * e2 * e3), P * e1 * e2 * (1 - e3), P, P * e1,
         P3 * e1sq * e2),
        (P * (1 - e1 * e2 * e3), P * e1 * (1 - e2 * e3), P, P * e1 * e2,
         P3 * e1sq * e2),
    ]


@functools.lru_cache(maxsize=None)
def _edge_adj_cached(nq):
    x, f = quad.map_to(quad.gaussxw(nq), [0.0, 1.0])
    e1 = x[:, None, None, None]
    e2 = x[None, :, None, None]
    e3 = x[None, None, :, None]
    P = x[None, None, None, :]
    f1 = f[:, None, None, None]
    f2 = f[None, :, None, None]
    f3 = f[None, None, :, None]
    f4 = f[None, None, None, :]
    F0 = f1 * f2 * f3 * f4
    shape = (nq, nq, nq, nq)
    pts = []
    wts = []
    for x1, x2, y1, y2, jac in _edge_maps(e1, e2, e3, P):
        blk = np.empty(shape + (4,))
        blk[..., 0] = 1 - np.broadcast_to(x1, shape)
        blk[..., 1] = np.broadcast_to(x2, shape)
        srcy = np.broadcast_to(y2, shape)
        srcx = 1 - np.broadcast_to(y1, shape)
        blk[..., 2] = (1 - srcy) - srcx
        blk[..., 3] = srcy
        pts.append(blk.reshape(-1, 4))
        wts.append((F0 * jac).reshape(-1))
    return np.concatenate(pts), np.concatenate(wts)


def edge_adj_quad(nq):
    p, w = _edge_adj_cached(int(nq))
    return p.copy(), w.copy()
