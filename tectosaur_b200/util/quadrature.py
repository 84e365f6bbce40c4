"""Host-side FP64 quadrature rules.

Same rules, node order and FP64 values as the reference's
``tectosaur/util/quadrature.py`` and ``tectosaur/util/tri_gauss.py``, so the
device kernels integrate with exactly the rules the reference feeds its own
kernels:

* ``gaussxw``     – Gauss–Legendre by the Golub–Welsch eigenvalue method on the
                    symmetric tridiagonal Jacobi matrix (util/quadrature.py:6-12).
* ``map_to``      – affine map of a [-1, 1] rule onto an interval (:15-19).
* ``gauss2d_tri`` – symmetric triangle rules of Strang & Fix (1973) and
                    Dunavant / ACM TOMS 612 and 706 up to degree 13, falling back
                    to a collapsed (Duffy) tensor rule above that (:33-45,
                    util/tri_gauss.py:180-212).
* ``gauss4d_tri`` – tensor product of two triangle rules (:47-60).

The symmetric rules are stored below as orbits (a weight and one generating
point per orbit) and expanded in the fixed point order the published tables
use; the weights are scaled by 1/2 to integrate over the reference triangle
{x, y >= 0, x + y <= 1}.
"""
import functools

import numpy as np
import scipy.linalg


def gaussxw(n):
    """n-point Gauss–Legendre rule on [-1, 1] (Golub–Welsch).

    The Jacobi matrix of the Legendre polynomials has zero diagonal and
    off-diagonal k / sqrt(4k^2 - 1); its eigenvalues are the nodes and the
    squared first components of its eigenvectors, times 2, the weights.
    Follows util/quadrature.py:6-12 (same banded eigen-solver, so the same bits).
    """
    k = np.arange(1.0, n)
    band = np.zeros((2, n))
    band[1, 0:n - 1] = k / np.sqrt(4 * k * k - 1)
    x, V = scipy.linalg.eig_banded(band, lower=True)
    w = 2 * np.real(np.power(V[0, :], 2))
    return x, w


def map_to(qr, interval):
    """Affine map of a rule on [-1, 1] onto ``interval`` (util/quadrature.py:15-19)."""
    x01 = (qr[0] + 1) / 2
    outx = interval[0] + (interval[1] - interval[0]) * x01
    outw = (qr[1] / 2) * (interval[1] - interval[0])
    return outx, outw


def quadrature(f, qr):
    return sum(f(qr[0]) * qr[1])


def gauss2d_rect(N):
    qg = gaussxw(N)
    qx, qy = np.meshgrid(qg[0], qg[0])
    pts = np.array([qx.flatten(), qy.flatten()]).T
    w = np.outer(qg[1], qg[1]).flatten()
    return pts, w


# --- symmetric triangle rules ---------------------------------------------
# Orbit notation (area coordinates are implied by the two stored coordinates):
#   ("c", w, t)       centroid (t, t); the tables print 1/3 to 15 or 16 digits
#   ("s2", w, a, b)   3 points  (b, a), (a, b), (a, a)
#   ("s3", w, a, b, c) 6 points (a, b), (a, c), (b, a), (b, c), (c, a), (c, b)
# Weights are normalised to sum to 1 (the tables' convention).
_T16 = 0.3333333333333333
_T15 = 0.333333333333333
_TRI_RULES = [
    # (max polynomial degree, orbits)  -- Strang & Fix "strang1"
    (2, [("s2", 0.3333333333333333, 0.16666666666666666, 0.6666666666666666)]),
    # strang3 (degree 3; note the negative centroid weight)
    (3, [("c", -0.5625, _T16),
         ("s2", 0.5208333333333334, 0.2, 0.6)]),
    # strang5 (degree 4)
    (4, [("s2", 0.109951743655322, 0.091576213509771, 0.816847572980459),
         ("s2", 0.223381589678011, 0.445948490915965, 0.10810301816807)]),
    # strang7 (degree 5)
    (5, [("c", 0.225, _T16),
         ("s2", 0.12593918054482717, 0.10128650732345633, 0.7974269853530872),
         ("s2", 0.13239415278850616, 0.47014206410511505, 0.05971587178976981)]),
    # strang8 (degree 6)
    (6, [("s2", 0.205950504760887, 0.437525248383384, 0.124949503233232),
         ("s3", 0.063691414286223, 0.797112651860071, 0.165409927389841,
          0.037477420750088)]),
    # strang10 (degree 7; negative centroid weight)
    (7, [("c", -0.14957004446767, _T15),
         ("s2", 0.175615257433204, 0.260345966079038, 0.479308067841923),
         ("s2", 0.053347235608839, 0.065130102902216, 0.869739794195568),
         ("s3", 0.077113760890257, 0.638444188569809, 0.312865496004875,
          0.048690315425316)]),
    # TOMS 612, 19 points (degree 9)
    (9, [("c", 0.0971357962827961, _T16),
         ("s2", 0.03133470022713983, 0.489682519198737, 0.02063496160252593),
         ("s2", 0.07782754100477543, 0.4370895914929355, 0.125820817014129),
         ("s2", 0.0796477389272091, 0.1882035356190322, 0.6235929287619356),
         ("s2", 0.0255776756586981, 0.04472951339445297, 0.9105409732110941),
         ("s3", 0.0432835393772894, 0.741198598784498, 0.03683841205473626,
          0.22196298916076573)]),
    # TOMS 612, 28 points (degree 11)
    (11, [("c", 0.0879773011622219, _T16),
          ("s2", 0.00874431155373619, 0.02598914092828833, 0.9480217181434233),
          ("s2", 0.03808157199393533, 0.0942875026479227, 0.8114249947041546),
          ("s2", 0.01885544805613125, 0.4946367750172147, 0.0107264499655706),
          ("s2", 0.072159697544741, 0.2073433826145142, 0.5853132347709715),
          ("s2", 0.0693291387055372, 0.4389078057004907, 0.1221843885990187),
          ("s3", 0.0410563154292886, 0.6779376548825902, 0.04484167758913055,
           0.27722066752827923),
          ("s3", 0.007362383783300573, 0.8588702812826364, 0.0,
           0.1411297187173636)]),
    # TOMS 706, 37 points (degree 13)
    (13, [("c", 0.05173976606574413, _T16),
          ("s2", 0.008007799555564802, 0.02486216853794722, 0.9502756629241056),
          ("s2", 0.046868898981821644, 0.41419254253808235, 0.17161491492383535),
          ("s2", 0.04659094018397649, 0.23029387816140479, 0.5394122436771904),
          ("s2", 0.031016943313796383, 0.11391998166173371, 0.7721600366765325),
          ("s2", 0.010791612736631274, 0.4954573000250823, 0.009085399949835354),
          ("s2", 0.03219553424243162, 0.4688613548470565, 0.062277290305886995),
          ("s3", 0.015445834210701583, 0.022076289653624404, 0.8513065041743485,
           0.1266172061720271),
          ("s3", 0.017822989923178663, 0.01862052280252097, 0.6894419707285913,
           0.2919375064688878),
          ("s3", 0.037038683681384625, 0.09650648129215923, 0.6358678594338728,
           0.267625659273968)]),
]


def _expand(orbits):
    pts = []
    wts = []
    for orb in orbits:
        kind, w = orb[0], orb[1]
        if kind == "c":
            pts.append((orb[2], orb[2]))
            wts.append(w)
        elif kind == "s2":
            a, b = orb[2], orb[3]
            pts.extend([(b, a), (a, b), (a, a)])
            wts.extend([w] * 3)
        else:
            a, b, c = orb[2], orb[3], orb[4]
            pts.extend([(a, b), (a, c), (b, a), (b, c), (c, a), (c, b)])
            wts.extend([w] * 6)
    return pts, wts


def symmetric_tri_rule(degree):
    """Published symmetric rule exact to ``degree``, or (None, None) above 13.

    Lookup by the smallest table degree >= ``degree`` (util/tri_gauss.py:180-212).
    """
    if degree <= 0:
        raise ValueError("triangle rule degree must be positive")
    for max_deg, orbits in _TRI_RULES:
        if degree <= max_deg:
            return _expand(orbits)
    return None, None


@functools.lru_cache(maxsize=None)
def _gauss2d_tri_cached(N):
    pts, wts = symmetric_tri_rule(N * 2 - 1)
    if pts is not None:
        return np.array(pts), np.array(wts) * 0.5
    q_rect_pts, q_rect_w = gauss2d_rect(N)
    q_x01 = (q_rect_pts[:, 0] + 1) / 2
    q_y01 = (q_rect_pts[:, 1] + 1) / 2
    q_tri_pts = np.empty_like(q_rect_pts)
    q_tri_pts[:, 0] = q_x01 * (1 - q_y01)
    q_tri_pts[:, 1] = q_y01
    q_tri_w = (q_rect_w / 4.0) * (1 - q_y01)
    return q_tri_pts, q_tri_w


def gauss2d_tri(N):
    """Rule on the reference triangle exact to degree 2N - 1 (util/quadrature.py:33-45)."""
    p, w = _gauss2d_tri_cached(int(N))
    return p.copy(), w.copy()


def gauss4d_tri(N_outer, N_inner):
    """Tensor-product rule over a pair of reference triangles (util/quadrature.py:47-60).

    Point order: outer index slowest.  Rows are (obs xhat, obs yhat, src xhat, src yhat).
    """
    po, wo = gauss2d_tri(N_outer)
    pi, wi = gauss2d_tri(N_inner)
    no, ni = po.shape[0], pi.shape[0]
    pts = np.empty((no * ni, 4))
    pts[:, 0] = np.repeat(po[:, 0], ni)
    pts[:, 1] = np.repeat(po[:, 1], ni)
    pts[:, 2] = np.tile(pi[:, 0], no)
    pts[:, 3] = np.tile(pi[:, 1], no)
    w = (wo[:, None] * wi[None, :]).reshape(-1)
    return pts, w
