"""Test infrastructure: ctypes binding of liboracle.so (the CPU restatement of
the reference's kernel math, oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker or the timed CPU baseline.  The product
(tectosaur_b200) never imports it.

Two builds of the same source: liboracle.so (no FMA contraction, portable
x86-64-v2: the parity checker) and a timed build for the host that runs it
(-O3 -march=native), selected by ``fast=True`` on the calls the CPU baseline
times.
"""
import ctypes
import hashlib
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

KERNEL_IDS = {
    "elasticU3": 0, "elasticT3": 1, "elasticA3": 2, "elasticH3": 3,
    "elasticRT3": 4, "elasticRA3": 5, "elasticRH3": 6,
}

_lib = None
_fast = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])


def lib(fast=False):
    global _lib
    if fast:
        return fast_lib()
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _host_key():
    """Identifies the host CPU (model and feature flags) for -march=native."""
    model, flags = "", ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if not model and line.startswith("model name"):
                    model = line
                elif not flags and line.startswith("flags"):
                    flags = line
                if model and flags:
                    break
    except OSError:
        pass
    return hashlib.sha1((model + flags).encode()).hexdigest()[:12]


def fast_lib_path():
    return os.path.join(HERE, "_native", "liboracle_fast_%s.so" % _host_key())


def fast_lib():
    """The timed CPU build, compiled for this host on first use (a few
    seconds; a library built for another CPU could use instructions this one
    lacks)."""
    global _fast
    if _fast is None:
        path = fast_lib_path()
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", HERE, "fast",
                                   "FAST_OUT=" + os.path.relpath(path, HERE)])
        _fast = ctypes.CDLL(path)
    return _fast


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _l(a):
    a = np.ascontiguousarray(a, dtype=np.int64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_long))


def _prec(float_type):
    return 0 if np.dtype(float_type) == np.float32 else 1


def _check(rc, what):
    if rc != 0:
        raise RuntimeError("oracle %s failed with status %d" % (what, rc))


def _threads(n):
    return int(n if n else os.cpu_count() or 1)


def pairs(kernel, float_type, quad, pts, tris, pair_list, params, adj=False,
          check0=False, n_threads=None, fast=False):
    """(n, 3, 3, 3, 3) pair integrals (assemble.cl single_pairs{Z,N}[_adj])."""
    pair_list = np.asarray(pair_list)
    n = pair_list.shape[0]
    out = np.zeros((n, 81))
    qp, qpp = _d(quad[0])
    qw, qwp = _d(quad[1])
    p, pp = _d(pts)
    t, tp = _i(tris)
    pl, plp = _i(pair_list.reshape(n, 5 if adj else 2))
    pr, prp = _d(params)
    _, op = _d(out)
    rc = lib(fast).orc_pairs(KERNEL_IDS[kernel], _prec(float_type), int(adj), int(check0),
                         op, qp.shape[0], qpp, qwp, pp, tp, plp, n, prp,
                         _threads(n_threads))
    _check(rc, "pairs")
    return out.reshape((n, 3, 3, 3, 3))


def farfield_tris(kernel, float_type, quad2d, pts, obs_tris, src_tris, v, params,
                  n_threads=None, fast=False):
    """Matrix-free tri-to-tri farfield matvec (matrix_free.cl farfield_tris_to_tris)."""
    obs_tris = np.asarray(obs_tris)
    src_tris = np.asarray(src_tris)
    out = np.zeros(obs_tris.shape[0] * 9)
    vin, vp = _d(v)
    p, pp = _d(pts)
    ot, otp = _i(obs_tris)
    st, stp = _i(src_tris)
    qp, qpp = _d(quad2d[0])
    qw, qwp = _d(quad2d[1])
    pr, prp = _d(params)
    _, op = _d(out)
    rc = lib(fast).orc_farfield_tris(KERNEL_IDS[kernel], _prec(float_type), op, vp, pp,
                                 otp, ot.shape[0], stp, st.shape[0], qp.shape[0], qpp,
                                 qwp, prp, _threads(n_threads))
    _check(rc, "farfield_tris")
    return out


def farfield_pts(kernel, float_type, obs_pts, obs_ns, src_pts, src_ns, v, params,
                 n_threads=None, fast=False):
    """Point-to-point farfield (farfield_direct.cl farfield_pts{K})."""
    out = np.zeros(np.asarray(obs_pts).shape[0] * 3)
    a, ap = _d(obs_pts)
    b, bp = _d(obs_ns)
    c, cp = _d(src_pts)
    d, dp = _d(src_ns)
    vin, vp = _d(v)
    pr, prp = _d(params)
    _, op = _d(out)
    rc = lib(fast).orc_farfield_pts(KERNEL_IDS[kernel], _prec(float_type), op, ap, bp,
                                a.shape[0], cp, dp, c.shape[0], vp, prp,
                                _threads(n_threads))
    _check(rc, "farfield_pts")
    return out


def interior_pairs(kernel, float_type, quad2d, obs_pts, obs_ns, pts, tris, pair_list, params,
                   finite_part=False, n_threads=None):
    """(n, 3, 3, 3) point-triangle integrals (assemble.cl interior_pairs)."""
    pair_list = np.asarray(pair_list).reshape(-1, 3)
    n = pair_list.shape[0]
    out = np.zeros((n, 27))
    qp, qpp = _d(quad2d[0])
    qw, qwp = _d(quad2d[1])
    a, ap = _d(obs_pts)
    b, bp = _d(obs_ns)
    p, pp = _d(pts)
    t, tp = _i(tris)
    pl, plp = _i(pair_list)
    pr, prp = _d(params)
    _, op = _d(out)
    rc = lib().orc_interior_pairs(KERNEL_IDS[kernel], _prec(float_type), op, qp.shape[0], qpp,
                                  qwp, ap, bp, a.shape[0], pp, p.shape[0], tp, plp, ctypes.c_long(n), prp,
                                  int(bool(finite_part)), _threads(n_threads))
    _check(rc, "interior_pairs")
    return out.reshape((n, 3, 3, 3))


def interior_corners(float_type, quad1d, obs_ns, pts, tris, pair_list, params, n_threads=None):
    """(n, 3, 3, 3) vertex integrals of elasticH3 (interior_corners.cl)."""
    pair_list = np.asarray(pair_list).reshape(-1, 3)
    n = pair_list.shape[0]
    out = np.zeros((n, 27))
    qp, qpp = _d(quad1d[0])
    qw, qwp = _d(quad1d[1])
    b, bp = _d(obs_ns)
    p, pp = _d(pts)
    t, tp = _i(tris)
    pl, plp = _i(pair_list)
    pr, prp = _d(params)
    _, op = _d(out)
    rc = lib().orc_interior_corners(_prec(float_type), op, qp.shape[0], qpp, qwp, bp,
                                    b.shape[0], pp, p.shape[0], tp, plp, ctypes.c_long(n), prp,
                                    _threads(n_threads))
    _check(rc, "interior_corners")
    return out.reshape((n, 3, 3, 3))


def farfield_tris_to_pts(kernel, float_type, quad2d, obs_pts, obs_ns, pts, src_tris, v, params,
                         n_threads=None):
    """Triangle sources -> points (matrix_free.cl farfield_tris_to_pts{K})."""
    out = np.zeros(np.asarray(obs_pts).shape[0] * 3)
    qp, qpp = _d(quad2d[0])
    qw, qwp = _d(quad2d[1])
    a, ap = _d(obs_pts)
    b, bp = _d(obs_ns)
    p, pp = _d(pts)
    t, tp = _i(src_tris)
    vin, vp = _d(v)
    pr, prp = _d(params)
    _, op = _d(out)
    rc = lib().orc_farfield_tris_to_pts(KERNEL_IDS[kernel], _prec(float_type), op, vp, ap, bp,
                                        a.shape[0], pp, p.shape[0], tp, t.shape[0], qp.shape[0],
                                        qpp, qwp, prp, _threads(n_threads))
    _check(rc, "farfield_tris_to_pts")
    return out


def farfield_tris_dense(kernel, float_type, quad4d, pts, obs_tris, src_tris, params,
                        n_threads=None):
    """Dense (n_obs, 3, 3, n_src, 3, 3) farfield blocks (assemble.cl farfield_tris)."""
    obs_tris = np.asarray(obs_tris)
    src_tris = np.asarray(src_tris)
    n_o, n_s = obs_tris.shape[0], src_tris.shape[0]
    out = np.zeros((n_o, 3, 3, n_s, 3, 3))
    qp, qpp = _d(quad4d[0])
    qw, qwp = _d(quad4d[1])
    p, pp = _d(pts)
    ot, otp = _i(obs_tris)
    st, stp = _i(src_tris)
    pr, prp = _d(params)
    _, op = _d(out)
    rc = lib().orc_farfield_tris_dense(KERNEL_IDS[kernel], _prec(float_type), op,
                                       qp.shape[0], qpp, qwp, pp, otp, n_o, stp, n_s,
                                       prp, _threads(n_threads))
    _check(rc, "farfield_tris_dense")
    return out


def make_bsr(n_row_blocks, rows, cols, data):
    """(indptr, indices, data) exactly as fast_sparse.make_bsr_matrix builds them."""
    data = np.ascontiguousarray(data, dtype=np.float64)
    nb, bs = data.shape[0], data.shape[1]
    indptr = np.zeros(n_row_blocks + 1, dtype=np.int64)
    indices = np.zeros(nb, dtype=np.int64)
    dout = np.zeros_like(data)
    r, rp = _l(rows)
    c, cp = _l(cols)
    _, dp = _d(data)
    _, ipp = _l(indptr)
    _, inp = _l(indices)
    _, dop = _d(dout)
    rc = lib().orc_make_bsr(ctypes.c_long(n_row_blocks), ctypes.c_long(nb), bs, rp, cp,
                            dp, ipp, inp, dop)
    _check(rc, "make_bsr")
    return indptr, indices, dout


def bsr_matvec(float_type, indptr, indices, data, x):
    data = np.ascontiguousarray(data, dtype=np.float64)
    bs = data.shape[1]
    mb = indptr.shape[0] - 1
    y = np.zeros(mb * bs)
    a, ap = _l(indptr)
    b, bp = _l(indices)
    _, dp = _d(data)
    xx, xp = _d(x)
    _, yp = _d(y)
    rc = lib().orc_bsr_matvec(_prec(float_type), ctypes.c_long(mb), bs, ap, bp, dp, xp, yp)
    _check(rc, "bsr_matvec")
    return y


def bcoo_matvec(float_type, rows, cols, data, x, n_rows, n_threads=1, fast=False):
    data = np.ascontiguousarray(data, dtype=np.float64)
    bs = data.shape[1]
    y = np.zeros(n_rows)
    a, ap = _l(rows)
    b, bp = _l(cols)
    _, dp = _d(data)
    xx, xp = _d(x)
    _, yp = _d(y)
    rc = lib(fast).orc_bcoo_matvec(_prec(float_type), ctypes.c_long(data.shape[0]), bs, ap,
                               bp, dp, xp, yp, _threads(n_threads))
    _check(rc, "bcoo_matvec")
    return y
