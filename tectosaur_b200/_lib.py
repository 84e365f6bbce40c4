"""ctypes binding of libtct_b200.so (the C ABI declared in include/tct_b200.h).

The shared library is the only compute path: if it is missing this module
raises at import, and every non-zero status becomes a RuntimeError carrying
the library's last error message.  There is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtct_b200.so")

TCT_OK = 0
TCT_ERR_ARG = 1
TCT_ERR_KERNEL = 2
TCT_ERR_CUDA = 3
TCT_ERR_OOM = 4
TCT_ERR_TIMEOUT = 5
TCT_ERR_PREC = 6
TCT_F32 = 0
TCT_F64 = 1

_STATUS = {1: "bad argument", 2: "unsupported kernel", 3: "CUDA error", 4: "out of memory",
           5: "timeout", 6: "unsupported precision"}

if not os.path.exists(LIB_PATH):
    raise ImportError(
        "tectosaur_b200: %s is not built; run `python tectosaur_b200/build.py` "
        "(there is no CPU fallback)" % LIB_PATH)

lib = ctypes.CDLL(LIB_PATH)

c_p = ctypes.c_void_p
c_i = ctypes.c_int
c_i64 = ctypes.c_int64
c_sz = ctypes.c_size_t
c_dp = ctypes.POINTER(ctypes.c_double)
c_i64p = ctypes.POINTER(ctypes.c_int64)

_SIGS = {
    "tct_version": ([], ctypes.c_char_p),
    "tct_last_error": ([], ctypes.c_char_p),
    "tct_kernel_id": ([ctypes.c_char_p], c_i),
    "tct_pairs_integrate": ([c_i, c_i, c_i, c_i, c_p, c_p, c_i64, c_i, c_i, c_i, c_p, c_p, c_p,
                             c_p, c_p, c_i64, c_dp, c_p], c_i),
    "tct_pairs_integrate_batched": ([c_i, c_i, c_p, c_i64, c_p, c_p, c_p, c_p, c_p, c_p, c_p,
                                     c_p, c_i64, c_i64, c_dp, c_i, c_i, c_p, c_sz, c_p], c_i),
    "tct_farfield_workspace_bytes": ([c_i, c_i, c_i64, c_i64, c_i], c_sz),
    "tct_farfield_tris_matvec": ([c_i, c_i, c_p, c_p, c_p, c_p, c_i64, c_p, c_i64, c_i, c_dp,
                                  c_dp, c_dp, c_i, c_p, c_sz, c_p], c_i),
    "tct_farfield_pts": ([c_i, c_i, c_p, c_p, c_p, c_i64, c_p, c_p, c_i64, c_p, c_dp, c_p], c_i),
    "tct_farfield_tris_dense": ([c_i, c_i, c_p, c_i, c_p, c_p, c_p, c_p, c_i64, c_p, c_i64, c_dp,
                                 c_p], c_i),
    "tct_fp32_fma_probe": ([c_p, c_i64, c_i, c_p], c_i),
    "tct_fp32x2_fma_probe": ([c_p, c_i64, c_i, c_p], c_i),
    "tct_farfield_noalloc_capacity": ([], c_sz),
    "tct_farfield_tris_matvec_noalloc": ([c_i, c_i, c_p, c_p, c_p, c_p, c_i64, c_p, c_i64, c_i,
                                          c_dp, c_dp, c_dp, c_i, c_p], c_i),
    "tct_bsr9_matvec": ([c_i, c_i64, c_p, c_p, c_p, c_p, c_i64, c_p, c_p, c_i, c_p], c_i),
    "tct_bsr9_matvec_panel": ([c_i, c_i64, c_p, c_p, c_p, c_i64, c_p, c_i64, c_p, c_i64, c_i,
                               c_i, c_p], c_i),
    "tct_find_near_pairs": ([c_dp, c_dp, c_i64, c_dp, c_dp, c_i64, ctypes.c_double, c_i,
                             ctypes.POINTER(c_p)], c_i),
    "tct_pairs_count": ([c_p], c_i64),
    "tct_pairs_copy": ([c_p, c_i64p], c_i),
    "tct_pairs_free": ([c_p], None),
    "tct_near_plan_build": ([c_dp, c_dp, c_i64, c_dp, c_dp, c_i64, ctypes.c_double, c_i,
                             ctypes.POINTER(c_p)], c_i),
    "tct_near_plan_leaf_pairs": ([c_p], c_i64),
    "tct_near_device_count": ([c_p, c_p, ctypes.POINTER(c_i64)], c_i),
    "tct_near_device_fill": ([c_p, c_p, c_p], c_i),
    "tct_near_plan_free": ([c_p], None),
    "tct_split_adjacent_close": ([c_i64p, c_i64, c_i64p, c_i64p, c_i64p, c_i64p, c_i64p, c_i64p,
                                  c_i64p, c_i64p], c_i),
    "tct_resolve_ea_rotation": ([c_i64p, c_i64p, c_i64, c_i64p], c_i),
    "tct_make_bsr_index": ([c_i64, c_i64, c_i64p, c_i64p, c_i64p, c_i64p, c_i64p], c_i),
    "tct_gmres_givens": ([c_i64, c_i64p, c_i64p, c_i64, c_dp, c_i64, c_dp, c_dp, c_dp, c_dp,
                          c_dp], c_i),
}

for _name, (_args, _res) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res

EXPORTED = sorted(_SIGS)


def last_error():
    msg = lib.tct_last_error()
    return msg.decode() if msg else ""


def check(status, what):
    if status != TCT_OK:
        raise RuntimeError("%s failed (%s): %s" % (what, _STATUS.get(status, status), last_error()))


def prec_of(float_type):
    dt = np.dtype(float_type)
    if dt == np.float32:
        return TCT_F32
    if dt == np.float64:
        return TCT_F64
    raise ValueError("float_type must be float32 or float64, got %s" % dt)


def kernel_id(name):
    k = lib.tct_kernel_id(name.encode())
    if k < 0:
        raise ValueError("unknown kernel %r (supported: elasticU3, elasticT3, elasticA3, "
                         "elasticH3, elasticRT3, elasticRA3, elasticRH3)" % name)
    return k


def dptr(a):
    """ctypes double* of a C-contiguous float64 numpy array."""
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(c_dp)


def i64ptr(a):
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(c_i64p)


def tptr(t):
    """Raw device pointer of a torch tensor (None for an empty/None tensor)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)

_TREE_SIGS = {
    "tct_tree_build": ([c_dp, c_dp, c_i64, c_i64, ctypes.POINTER(c_p)], c_i),
    "tct_tree_n_nodes": ([c_p], c_i64),
    "tct_tree_max_height": ([c_p], c_i),
    "tct_tree_export": ([c_p, c_i64p, c_i64p, c_i64p, c_dp, c_dp, c_p, c_p, c_p, c_i64p], c_i),
    "tct_tree_free": ([c_p], None),
    "tct_treecode_lists": ([c_p, c_p, ctypes.c_double, ctypes.c_double, c_i64, c_i,
                            ctypes.POINTER(c_p)], c_i),
    "tct_lists_sizes": ([c_p, c_i64p], c_i),
    "tct_lists_export": ([c_p, c_i, c_i64p, c_i64p, c_i64p], c_i),
    "tct_lists_free": ([c_p], None),
}
for _name, (_args, _res) in _TREE_SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res
EXPORTED = sorted(set(EXPORTED) | set(_TREE_SIGS))

class FmmTree(ctypes.Structure):
    """Mirror of tct_fmm_tree (include/tct_b200.h)."""
    _fields_ = [("n_nodes", c_i64), ("start", c_p), ("end", c_p), ("centers", c_p),
                ("radii", c_p), ("children", c_p), ("parent", c_p), ("orig", c_p),
                ("leaves", c_p), ("n_leaves", c_i64), ("levels", c_p),
                ("level_offsets", c_i64p), ("n_levels", c_i)]


class FmmList(ctypes.Structure):
    """Mirror of tct_fmm_list."""
    _fields_ = [("obs", c_p), ("start", c_p), ("src", c_p), ("n_obs", c_i64)]


_FMM_SIGS = {
    "tct_fmm_workspace_bytes": ([c_i, c_i, c_i, c_i, c_i, c_i64, c_i64, c_i64, c_i64], c_sz),
    "tct_fmm_m2l_plan_stats": ([c_i, c_i, c_i, ctypes.POINTER(c_i64)], c_i),
    "tct_fmm_matvec": ([c_i, c_i, c_i, c_i, c_i, c_dp, c_dp, c_dp, ctypes.c_double, c_p, c_p,
                        c_i64, ctypes.POINTER(FmmTree), c_p, c_p, c_i64,
                        ctypes.POINTER(FmmTree), ctypes.POINTER(FmmList),
                        ctypes.POINTER(FmmList), c_p, c_p, c_i, c_p, c_sz, c_p], c_i),
}
for _name, (_args, _res) in _FMM_SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res
EXPORTED = sorted(set(EXPORTED) | set(_FMM_SIGS))

_SOLVE_SIGS = {
    "tct_csr_matvec": ([c_i, c_i64, c_p, c_p, c_p, c_p, c_p, c_i, c_p], c_i),
    "tct_csr_matvec_panel": ([c_i, c_i64, c_p, c_p, c_p, c_p, c_i64, c_p, c_i64, c_i, c_i, c_p],
                             c_i),
    "tct_fp64_fma_probe": ([c_p, c_i64, c_i, c_p], c_i),
    "tct_launch_count": ([], ctypes.c_uint64),
    "tct_qd_rate_state": ([c_i64, c_i, c_p, c_p, c_p, c_p, ctypes.c_double, ctypes.c_double,
                           ctypes.c_double, c_p, ctypes.c_double, c_i, c_i, c_p, c_p, c_p], c_i),
    "tct_qd_velocity_state": ([c_i64, c_p, c_p, c_p, c_p, c_p, c_p, ctypes.c_double, c_i, c_p,
                               c_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, c_p, c_p,
                               c_p], c_i),
    "tct_farfield_tris_to_pts_workspace_bytes": ([c_i, c_i64, c_i64, c_i], c_sz),
    "tct_farfield_tris_to_pts": ([c_i, c_i, c_p, c_p, c_p, c_p, c_i64, c_p, c_p, c_i64, c_i,
                                  c_dp, c_dp, c_dp, c_p, c_sz, c_p], c_i),
    "tct_interior_pairs": ([c_i, c_i, c_p, c_i, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, c_dp,
                            c_i, c_p], c_i),
    "tct_interior_corners": ([c_i, c_p, c_i, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, c_dp, c_p],
                             c_i),
    "tct_qd_rate_state_batch": ([c_i64, c_i, c_i, c_p, c_p, c_i64, c_p, c_i64, c_p,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_double, c_p,
                                 ctypes.c_double, c_i, c_i, c_p, c_i64, c_p, c_p], c_i),
    "tct_qd_velocity_state_batch": ([c_i64, c_i, c_p, c_p, c_p, c_p, c_i64, c_p, c_p,
                                     ctypes.c_double, c_i, c_p, c_i64, c_p, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, c_p, c_i64, c_p, c_i64,
                                     c_p], c_i),
    "tct_qd_deficit_batch": ([c_i64, c_i, c_p, ctypes.c_double, c_p, c_p, c_p, c_i64, c_i, c_p,
                              c_i64, c_p], c_i),
    "tct_qd_finish_batch": ([c_i64, c_i64, c_i, c_p, c_i64, c_p, c_i64, c_p, c_i64,
                             ctypes.c_double, c_p, c_i64, c_p], c_i),
    "tct_qd_combine_batch": ([c_i64, c_i, c_i, c_p, c_p, c_p, c_p, c_p, c_i64, c_p, c_i64, c_p],
                             c_i),
    "tct_qd_error_norm_batch": ([c_i64, c_i, c_i, c_p, c_p, c_p, c_p, c_p, c_i64, c_p, c_i64,
                                 ctypes.c_double, c_p, c_p], c_i),
    "tct_cg_csr_batch": ([c_i64, c_i, c_p, c_p, c_p, c_p, c_i64, c_p, c_i64, c_p,
                          ctypes.c_double, ctypes.c_double, c_i, c_p, c_p], c_i),
    "tct_cg_csr": ([c_i64, c_p, c_p, c_p, c_p, c_p, c_p, ctypes.c_double, ctypes.c_double, c_i,
                    c_p, c_p], c_i),
    "tct_farfield_rh_panel_workspace_bytes": ([c_i64, c_i64, c_i, c_i], c_sz),
    "tct_farfield_rh_panel_matvec": ([c_p, c_p, c_p, c_p, c_i64, c_p, c_i64, c_i, c_i, c_dp, c_dp,
                                      c_dp, c_i, c_p, c_sz, c_p], c_i),
    "tct_farfield_rh_panel_error": ([c_p, c_i64, c_i64, c_i, c_i, c_p, ctypes.POINTER(c_i)], c_i),
    "tct_farfield_rt_panel_workspace_bytes": ([c_i64, c_i64, c_i, c_i], c_sz),
    "tct_farfield_rt_panel_matvec": ([c_p, c_p, c_p, c_p, c_i64, c_p, c_i64, c_i, c_i, c_dp, c_dp,
                                      c_dp, c_i, c_p, c_sz, c_p], c_i),
    "tct_farfield_rt_panel_error": ([c_p, c_i64, c_i64, c_i, c_i, c_p, ctypes.POINTER(c_i)], c_i),
}
for _name, (_args, _res) in _SOLVE_SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res
EXPORTED = sorted(set(EXPORTED) | set(_SOLVE_SIGS))

c_ip = ctypes.POINTER(c_i)
_TUNE_SIGS = {
    "tct_tune_set": ([c_i, c_i, c_i, c_i, c_i, c_i64, c_i64, c_i, c_i], c_i),
    "tct_tune_get": ([c_i, c_i, c_i, c_i, c_i, c_i64, c_i64, c_ip, c_ip], c_i),
    "tct_tune_bucket": ([c_i64], c_i),
    "tct_tune_size": ([], c_i64),
    "tct_tune_entry": ([c_i64, c_ip, c_ip, c_ip], c_i),
    "tct_tune_put_entry": ([c_ip, c_i, c_i], c_i),
    "tct_tune_clear": ([], None),
    "tct_farfield_autotune": ([c_i, c_i, c_p, c_p, c_p, c_p, c_i64, c_p, c_i64, c_i, c_dp, c_dp,
                               c_dp, c_p, c_sz, c_p, c_ip], c_i),
    "tct_bsr9_autotune": ([c_i, c_i64, c_p, c_p, c_p, c_i64, c_p, c_p, c_p, c_ip, c_ip], c_i),
    "tct_farfield_workspace_bytes_chunks": ([c_i, c_i, c_i64, c_i64, c_i, c_i], c_sz),
    "tct_farfield_pts_panel_workspace_bytes": ([c_i64, c_i64, c_i], c_sz),
    "tct_farfield_pts_panel": ([c_i, c_p, c_p, c_p, c_p, c_i64, c_p, c_p, c_i64, c_i, c_dp, c_i,
                                c_p, c_sz, c_p], c_i),
    "tct_farfield_pts_panel_error": ([c_p, c_i64, c_i64, c_i, c_p, ctypes.POINTER(c_i)], c_i),
    "tct_tree_build_device": ([c_dp, c_dp, c_i64, c_i64, c_p, ctypes.POINTER(c_p)], c_i),
    "tct_near_plan_build_device": ([c_dp, c_dp, c_i64, c_dp, c_dp, c_i64, ctypes.c_double, c_p,
                                    ctypes.POINTER(c_p)], c_i),
    "tct_pairs_integrate_batched_slots": ([c_i, c_i, c_p, c_p, c_i64, ctypes.c_double, c_i,
                                           c_i64, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64,
                                           c_i64, c_dp, c_i, c_p, c_sz, c_p], c_i),
}
for _name, (_args, _res) in _TUNE_SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res
EXPORTED = sorted(set(EXPORTED) | set(_TUNE_SIGS))
TCT_TUNE_FARFIELD, TCT_TUNE_BSR9, TCT_TUNE_FAR_PANEL = 1, 2, 3


def launch_count():
    """Kernels launched by libtct_b200.so so far in this process."""
    return int(lib.tct_launch_count())
