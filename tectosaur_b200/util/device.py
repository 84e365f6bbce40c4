"""Device-memory helpers over torch (plumbing only: allocation, copies and the
current stream; all arithmetic of the hot path runs in libtct_b200.so)."""
import numpy as np


def torch():
    import torch as _torch
    return _torch


def cuda_available():
    try:
        return torch().cuda.is_available()
    except ImportError:
        return False


def require_cuda():
    t = torch()
    if not t.cuda.is_available():
        raise RuntimeError("tectosaur_b200 needs a CUDA device (sm_100a); none is visible")
    return t


def torch_dtype(float_type):
    t = torch()
    dt = np.dtype(float_type)
    if dt == np.float32:
        return t.float32
    if dt == np.float64:
        return t.float64
    raise ValueError("float_type must be float32 or float64")


def to_dev(arr, dtype=None):
    """Copy a host array to the current CUDA device (C-contiguous)."""
    t = require_cuda()
    a = np.ascontiguousarray(arr if dtype is None else np.asarray(arr).astype(dtype, copy=False))
    return t.from_numpy(a).to("cuda", non_blocking=False)


def empty(n, float_type):
    t = require_cuda()
    return t.empty(n, dtype=torch_dtype(float_type), device="cuda")


def zeros(n, float_type):
    t = require_cuda()
    return t.zeros(n, dtype=torch_dtype(float_type), device="cuda")


def workspace(nbytes):
    """Scratch buffer of at least nbytes, 256-byte aligned (torch allocations are)."""
    t = require_cuda()
    buf = t.empty(max(int(nbytes), 256), dtype=t.uint8, device="cuda")
    assert buf.data_ptr() % 256 == 0
    return buf


def is_device_tensor(v):
    try:
        t = torch()
    except ImportError:
        return False
    return isinstance(v, t.Tensor) and v.is_cuda


def host_or_device_apply(op, v, float_type):
    """op.dot_device on v: a CUDA tensor stays on the device (in its own
    precision when float_type is not fixed by op), a host array is copied in
    as float_type and the result copied back."""
    t = torch()
    ft = np.dtype(float_type)
    if is_device_tensor(v):
        x = v.to(torch_dtype(ft)).contiguous()
        return op.dot_device(x, t.empty(op.shape[0], dtype=x.dtype, device=x.device))
    x = to_dev(np.asarray(v).reshape(-1), ft)
    y = t.empty(op.shape[0], dtype=x.dtype, device=x.device)
    op.dot_device(x, y)
    return y.cpu().numpy()
