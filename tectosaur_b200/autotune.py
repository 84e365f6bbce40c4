"""Launch-shape autotuner (an addition: the reference's launch shapes are
fixed; its only per-configuration cache is the compiled-module cache of
tectosaur/util/gpu.py:63-77).

libtct_b200.so looks every direct-farfield and BSR launch shape up in an
in-library cache keyed by (operation, kernel, precision, rule points,
right-hand sides, log2 size buckets) and falls back to its heuristics when
the key has no entry (include/tct_b200.h, "tuned launch shapes").  This
module fills the cache by timing the candidates on an operator's own data
(tct_farfield_autotune, tct_bsr9_autotune: CUDA events, the fastest kept),
and saves / restores it as JSON so that a tuned shape outlives the process:

    op = RegularizedSparseIntegralOp(...)
    op.autotune()          # tune this operator's launches (a few seconds)
    autotune.save()        # ~/.cache/tectosaur_b200/tune-<gpu>.json
    ...
    autotune.load()        # in a later process, before building operators

A shape changes how the work is cut into CTAs (and so the floating-point
summation order), never the quantity computed.
"""
import ctypes
import json
import os

import numpy as np

from . import _lib
from .util import device

OPS = {_lib.TCT_TUNE_FARFIELD: "farfield", _lib.TCT_TUNE_BSR9: "bsr9",
       _lib.TCT_TUNE_FAR_PANEL: "farfield_panel"}
KEY_FIELDS = ("op", "kernel", "prec", "nq", "rhs", "bucket0", "bucket1")


def _gpu_name():
    try:
        t = device.torch()
        return t.cuda.get_device_name() if t.cuda.is_available() else "none"
    except Exception:
        return "none"


def cache_path(path=None):
    """TCT_TUNE_CACHE, else ~/.cache/tectosaur_b200/tune-<gpu name>.json."""
    if path:
        return path
    env = os.environ.get("TCT_TUNE_CACHE")
    if env:
        return env
    name = "".join(c if c.isalnum() else "_" for c in _gpu_name())
    return os.path.join(os.path.expanduser("~"), ".cache", "tectosaur_b200",
                        "tune-%s.json" % name)


def entries():
    """The cache as a list of dicts (key fields + v0, v1)."""
    out = []
    key = (ctypes.c_int * 7)()
    v0, v1 = ctypes.c_int(), ctypes.c_int()
    for i in range(int(_lib.lib.tct_tune_size())):
        _lib.check(_lib.lib.tct_tune_entry(i, key, ctypes.byref(v0), ctypes.byref(v1)),
                   "tct_tune_entry")
        e = dict(zip(KEY_FIELDS, [int(k) for k in key]))
        e.update(v0=int(v0.value), v1=int(v1.value))
        out.append(e)
    return out


def clear():
    _lib.lib.tct_tune_clear()


def save(path=None):
    """Write the cache (and the GPU it was tuned on) as JSON; returns the path."""
    path = cache_path(path)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump({"gpu": _gpu_name(), "entries": entries()}, f, indent=1)
    return path


def load(path=None, any_gpu=False):
    """Restore entries saved by `save` (only those tuned on a GPU of the same
    name unless any_gpu); returns the number restored."""
    path = cache_path(path)
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        doc = json.load(f)
    if not any_gpu and doc.get("gpu") != _gpu_name():
        return 0
    n = 0
    for e in doc.get("entries", []):
        key = (ctypes.c_int * 7)(*[int(e[k]) for k in KEY_FIELDS])
        _lib.check(_lib.lib.tct_tune_put_entry(key, int(e["v0"]), int(e["v1"])),
                   "tct_tune_put_entry")
        n += 1
    return n


def lookup(op, kernel, prec, nq, rhs, n0, n1):
    """(v0, v1) of a key, or None."""
    v0, v1 = ctypes.c_int(), ctypes.c_int()
    if _lib.lib.tct_tune_get(op, kernel, prec, nq, rhs, n0, n1, ctypes.byref(v0),
                             ctypes.byref(v1)):
        return int(v0.value), int(v1.value)
    return None


def tune_farfield(far, x=None, stream=None):
    """Tune a TriToTriDirectFarfieldOp's source chunking; its workspace is
    grown to hold the partial sums of the largest candidate while tuning and
    kept at the size the chosen count needs.  Returns the chosen count."""
    t = device.torch()
    max_ws = int(_lib.lib.tct_farfield_workspace_bytes_chunks(
        far.kid, far.prec, far.n_obs, far.n_src, far.n_q, 64))
    if max_ws > far.ws_bytes:
        far.workspace = device.workspace(max_ws)
        far.ws_bytes = max_ws
    if x is None:
        x = t.from_numpy(np.random.default_rng(0).standard_normal(far.shape[1])).to(
            device.torch_dtype(far.float_type)).cuda()
    y = t.empty(far.shape[0], dtype=x.dtype, device="cuda")
    chunks = ctypes.c_int()
    _lib.check(_lib.lib.tct_farfield_autotune(
        far.kid, far.prec, _lib.tptr(y), _lib.tptr(x), _lib.tptr(far.gpu_pts),
        _lib.tptr(far.gpu_obs_tris), far.n_obs, _lib.tptr(far.gpu_src_tris), far.n_src, far.n_q,
        _lib.dptr(far.qx), _lib.dptr(far.qw), _lib.dptr(far.params), _lib.tptr(far.workspace),
        far.ws_bytes, _lib.stream_ptr(stream), ctypes.byref(chunks)), "tct_farfield_autotune")
    need = int(_lib.lib.tct_farfield_workspace_bytes_chunks(
        far.kid, far.prec, far.n_obs, far.n_src, far.n_q, chunks.value))
    need = max(need, int(_lib.lib.tct_farfield_workspace_bytes(
        far.kid, far.prec, far.n_obs, far.n_src, far.n_q)))
    if need < far.ws_bytes:
        far.workspace = device.workspace(need)
        far.ws_bytes = need
    return int(chunks.value)


def tune_bsr(bsr, x=None, y=None, stream=None):
    """Tune a DeviceBSR9's launch shape on its own (padded) layout; returns
    (lanes per row, CTAs per SM).  `y` (optional) receives A x."""
    t = device.torch()
    if x is None:
        x = t.from_numpy(np.random.default_rng(1).standard_normal(bsr.shape[1])).to(
            device.torch_dtype(bsr.float_type)).cuda()
    if y is None:
        y = t.empty(bsr.shape[0], dtype=x.dtype, device="cuda")
    lanes, ctas = ctypes.c_int(), ctypes.c_int()
    _lib.check(_lib.lib.tct_bsr9_autotune(
        _lib.prec_of(bsr.float_type), bsr.n_row_blocks, _lib.tptr(bsr.indptr),
        _lib.tptr(bsr.indices), _lib.tptr(bsr.data), bsr.stride, _lib.tptr(x),
        _lib.tptr(y), _lib.stream_ptr(stream), ctypes.byref(lanes), ctypes.byref(ctas)),
        "tct_bsr9_autotune")
    return int(lanes.value), int(ctas.value)


def tune_operator(op):
    """Tune the launches of a RegularizedSparseIntegralOp (direct farfield
    chunking, nearfield BSR shape); returns the chosen shapes."""
    from .ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    out = {}
    if isinstance(op.farfield, TriToTriDirectFarfieldOp) and op.farfield.n_obs and \
            op.farfield.n_src:
        out["farfield_chunks"] = tune_farfield(op.farfield)
    bsr = getattr(op.nearfield, "bsr", None)
    if bsr is not None and bsr.n_row_blocks > 0 and bsr.nnzb > 0:
        lanes, ctas = tune_bsr(bsr)
        out["bsr_lanes_per_row"] = lanes
        out["bsr_ctas_per_sm"] = ctas
    return out
