"""Block-sparse matrices of 9x9 blocks.

``DeviceBSR9`` is the device-resident nearfield matrix the operator apply
uses: block-row pointers and block-column indices (int32) plus the blocks in
structure-of-arrays order (element e = i*9 + j of the block in slot s at
data[e * stride + s]), applied by tct_bsr9_matvec (one warp per block row, no
atomics).

``BCOOMatrix`` / ``BSRMatrix`` mirror the reference's host classes
(tectosaur/util/sparse.py:14-70) for callers that read ``op.mat`` directly:
same attributes and ``dot``, ``to_bsr``, ``to_scipy``, ``to_dense``.  Their
``dot`` runs on the device through the same BSR kernel.
"""
import ctypes

import numpy as np
import scipy.sparse

from .. import _lib
from . import device


def make_bsr_index(n_row_blocks, rows, cols):
    """(indptr, indices, slot) of the reference's make_bsr_matrix
    (util/fast_sparse.cpp:14-68): stable counting sort by block row,
    duplicates kept; slot[i] = BSR position of input block i."""
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    n = rows.shape[0]
    indptr = np.empty(n_row_blocks + 1, dtype=np.int64)
    indices = np.empty(max(n, 1), dtype=np.int64)
    slot = np.empty(max(n, 1), dtype=np.int64)
    _lib.check(_lib.lib.tct_make_bsr_index(n_row_blocks, n, _lib.i64ptr(rows), _lib.i64ptr(cols),
                                           _lib.i64ptr(indptr), _lib.i64ptr(indices),
                                           _lib.i64ptr(slot)), "tct_make_bsr_index")
    return indptr, indices[:n].copy(), slot[:n].copy()


def padded_rows(indptr, align):
    """Row starts rounded up to multiples of `align` slots: (pstart, pos),
    pstart[r] the first slot of block row r (pstart[-1] the slot count, a
    multiple of `align`) and pos[k] the slot of the k-th block in CSR order."""
    indptr = np.asarray(indptr, dtype=np.int64)
    counts = np.diff(indptr)
    pstart = np.zeros(counts.shape[0] + 1, dtype=np.int64)
    np.cumsum((counts + align - 1) // align * align, out=pstart[1:])
    rows = np.repeat(np.arange(counts.shape[0], dtype=np.int64), counts)
    pos = pstart[rows] + (np.arange(int(indptr[-1]), dtype=np.int64) - indptr[rows])
    return pstart, pos


def auto_row_align(n_row_blocks, nnzb):
    """Row alignment (in slots) for an operator's nearfield matrix: the
    largest of 32, 16, 8 slots (128, 64, 32 bytes of an FP32 element plane)
    whose mean padding, (align - 1) / 2 slots per row, is at most a fifth of
    the mean row length; 1 (no padding) for rows too short for any.  A line
    that two rows (or two steps of one row) share is fetched from DRAM once
    per reader: unpadded rows of ~90 blocks cost 1.37x the algorithmic bytes,
    rows aligned to 8 / 16 / 32 slots 1.24x / 1.13x / 1.05x."""
    if n_row_blocks <= 0:
        return 1
    mean = nnzb / n_row_blocks
    for a in (32, 16, 8):
        if (a - 1) / 2 <= 0.2 * mean:
            return a
    return 1


class DeviceBSR9:
    """Device 9x9-block BSR matrix, SoA block storage (see module docstring).

    With row_align > 1 each block row starts on a multiple of row_align
    slots (the slots between rows are padding, column index -1, zero data,
    never read by the kernels): with 32 FP32 (16 FP64) slots no 128-byte
    line of an element plane then holds blocks of two rows, and none is
    fetched from DRAM twice (at 8 or 16 FP32 slots, fewer lines are shared).  `nnzb`
    counts the blocks, `stride` the slots (the element-plane length);
    `pos[k]` is the slot of the k-th block in CSR order, and the host
    views (`indptr_host`, `indices_host`, `blocks_host`) are unpadded.
    "auto" pads by auto_row_align."""

    def __init__(self, shape, indptr, indices, float_type, data=None, row_align=1):
        self.shape = tuple(shape)
        self.float_type = np.dtype(float_type)
        self.n_row_blocks = self.shape[0] // 9
        self.nnzb = int(indices.shape[0])
        self.indptr_host = np.asarray(indptr, dtype=np.int64)
        self.indices_host = np.asarray(indices, dtype=np.int64)
        if row_align == "auto":
            row_align = auto_row_align(self.n_row_blocks, self.nnzb)
        self.row_align = int(row_align)
        if self.row_align < 1:
            raise ValueError("row_align must be >= 1")
        if self.row_align > 1 and data is not None:
            raise ValueError("data= takes the unpadded layout (row_align 1)")
        if self.row_align > 1:
            pstart, self.pos = padded_rows(self.indptr_host, self.row_align)
            self.stride = max(int(pstart[-1]), 1)
            idx = np.full(self.stride, -1, dtype=np.int32)
            idx[self.pos] = self.indices_host
        else:
            pstart, self.pos = self.indptr_host, None
            self.stride = max(self.nnzb, 1)
            idx = np.maximum(self.indices_host, 0).astype(np.int32) if self.nnzb > 0 \
                else np.zeros(1, dtype=np.int32)
        if self.stride >= 2 ** 31:
            raise ValueError("more than 2^31 nearfield blocks")
        self.indptr = device.to_dev(pstart.astype(np.int32))
        self.indices = device.to_dev(idx)
        self.data = data if data is not None else device.zeros(81 * self.stride, self.float_type)

    def slots(self, k):
        """Slots of the blocks with CSR positions k (host int64 array)."""
        return np.asarray(k, dtype=np.int64) if self.pos is None else self.pos[k]

    @property
    def nbytes(self):
        return int(self.data.numel() * self.data.element_size()
                   + 4 * (self.stride + self.n_row_blocks + 1))

    def matvec(self, x, y, accumulate=False, extra=None, stream=None):
        """y (+)= A x on device tensors (A + extra when `extra` is another
        block array with the same structure)."""
        _lib.check(_lib.lib.tct_bsr9_matvec(
            _lib.prec_of(self.float_type), self.n_row_blocks, _lib.tptr(self.indptr),
            _lib.tptr(self.indices), _lib.tptr(self.data),
            _lib.tptr(extra) if extra is not None else None, self.stride,
            _lib.tptr(x), _lib.tptr(y), int(bool(accumulate)), _lib.stream_ptr(stream)),
            "tct_bsr9_matvec")
        return y

    def matvec_panel(self, X, Y, accumulate=False, stream=None):
        """Y[v] (+)= A X[v] for device tensors X (R, n_cols), Y (R, n_rows)
        (row strides may exceed the lengths); one launch, each block read
        from HBM once."""
        R = X.shape[0]
        if Y.shape[0] != R:
            raise ValueError("matvec_panel: %d input vs %d output vectors" % (R, Y.shape[0]))
        if X.stride(1) != 1 or Y.stride(1) != 1:
            raise ValueError("matvec_panel: rows must be contiguous")
        _lib.check(_lib.lib.tct_bsr9_matvec_panel(
            _lib.prec_of(self.float_type), self.n_row_blocks, _lib.tptr(self.indptr),
            _lib.tptr(self.indices), _lib.tptr(self.data), self.stride, _lib.tptr(X),
            X.stride(0), _lib.tptr(Y), Y.stride(0), R, int(bool(accumulate)),
            _lib.stream_ptr(stream)), "tct_bsr9_matvec_panel")
        return Y

    def blocks_host(self, data=None):
        """(nnzb, 9, 9) host array of the blocks in BSR order."""
        d = (self.data if data is None else data)[:81 * self.stride].reshape(81, self.stride)
        if self.pos is None:
            d = d[:, :self.nnzb]
        else:
            d = d[:, device.to_dev(self.pos, np.int64)]
        return d.t().reshape(self.nnzb, 9, 9).cpu().numpy()

    def rows_host(self):
        return np.repeat(np.arange(self.n_row_blocks, dtype=np.int64), np.diff(self.indptr_host))


class BCOOMatrix:
    """Block-COO matrix (util/sparse.py:14-42); ``dot`` runs on the device."""

    def __init__(self, rows, cols, data, shape):
        self.rows = rows
        self.cols = cols
        self.data = data
        self.shape = shape

    @property
    def dtype(self):
        return self.data.dtype

    @property
    def blocksize(self):
        return self.data.shape[1]

    def dot(self, v):
        return self.to_bsr().dot(v)

    def to_bsr(self):
        n_row_blocks = self.shape[0] // self.blocksize
        indptr, indices, slot = make_bsr_index(n_row_blocks, self.rows, self.cols)
        data = np.empty_like(self.data)
        data[slot] = self.data
        return BSRMatrix(indptr, indices, data, self.shape)

    def to_dense(self):
        return self.to_bsr().to_scipy().todense()


class BSRMatrix:
    """Block-CSR matrix (util/sparse.py:44-70); ``dot`` runs on the device for
    9x9 blocks.  The reference allocates the output with shape[1] (only right
    for square matrices, util/sparse.py:61); this one uses shape[0]."""

    def __init__(self, indptr, indices, data, shape):
        assert data.shape[1] == data.shape[2]
        self.indptr = indptr
        self.indices = indices
        self.data = data
        self.shape = shape

    @property
    def dtype(self):
        return self.data.dtype

    @property
    def blocksize(self):
        return self.data.shape[1]

    def dot(self, v):
        if self.blocksize != 9:
            return self.to_scipy().dot(v).astype(self.dtype)
        ft = self.dtype
        nnzb = self.data.shape[0]
        m = DeviceBSR9(self.shape, self.indptr, self.indices, ft)
        if nnzb:
            soa = np.ascontiguousarray(self.data.reshape(nnzb, 81).T, dtype=ft)
            m.data = device.to_dev(soa.reshape(-1))
        x = device.to_dev(np.asarray(v), ft)
        y = device.empty(self.shape[0], ft)
        m.matvec(x, y)
        return y.cpu().numpy()

    def to_scipy(self):
        return scipy.sparse.bsr_matrix((self.data, self.indices, self.indptr), self.shape)

    def to_dense(self):
        return self.to_scipy().todense()


def from_scipy_bsr(A):
    return BSRMatrix(A.indptr, A.indices, A.data, A.shape)
