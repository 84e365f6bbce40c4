// 9x9 block-sparse (BSR) nearfield matvec, HBM-bandwidth bound.
//
// Replaces the reference's host BCOO/BSR matvecs (bcoomv9 / bsrmv9,
// tectosaur/util/fast_sparse.cpp:71-163; OpenMP with atomic scatter) with a
// row-owned device kernel: one warp per block row, no atomics.
//
// Blocks are stored structure-of-arrays: element e = i*9 + j of block s at
// data[e * stride + s].  The lanes of a warp take consecutive blocks of the
// row, so each of the 81 element loads of a step is one contiguous 128-byte
// (FP32) or 256-byte (FP64) transaction; x is gathered through L1/L2 (it is
// 9 Reals per triangle and stays cache resident).  Each lane keeps 9 row
// partial sums, reduced across the warp with shuffles at the end of the row.
//
// Slots with a negative column index are padding: the operator's matrix
// starts every block row on a 128-byte line of the element planes, so a
// row's loads never share a line with another row or with another step of
// the same row.  Unpadded, each such shared line is fetched from DRAM once
// per reader (1.35x the algorithmic bytes at ~90 blocks per row, 1.06x
// padded).
#include <algorithm>

#include "common.cuh"

namespace tct {
namespace {

// Long rows (16 or 32 lanes per row): at most 80 registers per thread (3
// blocks of 256 threads per SM) and streaming loads of the blocks; short
// rows (8 lanes or fewer): 64 registers (4 blocks) and L2-retaining loads.
// Left unconstrained the compiler hoists all 81 block loads into registers
// (222 registers, 1 block per SM) and the per-row shuffle reduction then
// leaves the SM with no loads in flight; with 64 registers fewer loads are
// in flight per warp (C2 matrix, ~90 blocks per row: 0.363 ms at 64
// registers, 0.355 ms at 80, 0.339 ms at 80 with streaming loads; 128
// registers spill).  On rows of one or two blocks, where the rows a warp
// serves share lines, the long-row form is slower (0.104 against 0.093 ms
// for 400k blocks).
//
// LPR lanes serve one block row (LPR = 32: a warp per row, the shape for
// the operator's ~90 blocks per row; 16 down to 1: a warp serves 32 / LPR
// rows at once, the shapes for rows of a few blocks).  The row loop is
// warp-uniform -- every lane runs the same number of iterations, lanes past
// the last row carry zeros -- so the shuffles always have the full warp.
template <typename R, bool TWO, int LPR>
__global__ void __launch_bounds__(256, LPR >= 16 ? 3 : 4)
bsr9_kernel(int64_t n_rows, const int32_t* __restrict__ indptr,
            const int32_t* __restrict__ indices, const R* __restrict__ data,
            const R* __restrict__ data2, int64_t stride, const R* __restrict__ x,
            R* __restrict__ y, int accumulate) {
    constexpr int G = 32 / LPR;  // rows per warp
    const int lane = threadIdx.x & 31;
    const int sub = lane % LPR;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    // each warp takes a contiguous range of row groups, in order
    const int64_t n_groups = (n_rows + G - 1) / G;
    const int64_t per_warp = (n_groups + n_warps - 1) / n_warps;
    const int64_t g_end = min(n_groups, (warp + 1) * per_warp);
    for (int64_t gi = warp * per_warp; gi < g_end; gi++) {
        const int64_t base = gi * G;
        const int64_t row = base + lane / LPR;
        int32_t start = 0, end = 0;
        if (row < n_rows) {
            start = __ldg(indptr + row);
            end = __ldg(indptr + row + 1);
        }
        R acc[9];
#pragma unroll
        for (int i = 0; i < 9; i++) acc[i] = 0;
        for (int32_t s = start + sub; s < end; s += LPR) {
            const int64_t col = __ldg(indices + s);
            if (col < 0) continue;  // padding slot
            R xv[9];
#pragma unroll
            for (int j = 0; j < 9; j++) xv[j] = __ldg(x + col * 9 + j);
#pragma unroll
            for (int i = 0; i < 9; i++)
#pragma unroll
                for (int j = 0; j < 9; j++) {
                    // long rows: streaming loads (evict first): every block
                    // is read once per apply, and with rows starting on
                    // lines no line is shared with another warp
                    const int64_t e = (int64_t)(i * 9 + j) * stride + s;
                    R a = LPR >= 16 ? __ldcs(data + e) : __ldg(data + e);
                    if (TWO) a += LPR >= 16 ? __ldcs(data2 + e) : __ldg(data2 + e);
                    acc[i] += a * xv[j];
                }
        }
#pragma unroll
        for (int i = 0; i < 9; i++) {
#pragma unroll
            for (int off = LPR / 2; off > 0; off >>= 1)
                acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
        }
        if (row < n_rows) {
#pragma unroll
            for (int i = 0; i < 9; i++) {
                if (i % LPR == sub) {
                    R* yp = y + row * 9 + i;
                    *yp = accumulate ? *yp + acc[i] : acc[i];
                }
            }
        }
    }
}

// Launch shape of tct_bsr9_matvec: lanes per row and CTAs per SM, from the
// shape cache (key: block rows, blocks per row) or the defaults (32, 8).
void bsr_shape(int prec, int64_t n_rows, int64_t stride, int* lpr, int* cps) {
    *lpr = 32;
    *cps = 8;
    int v0 = 0, v1 = 0;
    const int64_t per_row = n_rows > 0 ? std::max<int64_t>(1, stride / n_rows) : 1;
    if (tune_lookup(kTuneBsr9, -1, prec, 0, 1, n_rows, per_row, &v0, &v1)) {
        if (v0 == 32 || v0 == 16 || v0 == 8 || v0 == 4 || v0 == 2 || v0 == 1) *lpr = v0;
        if (v1 >= 1 && v1 <= 64) *cps = v1;
    }
}

template <typename R, int LPR>
void launch_bsr(int64_t blocks, int64_t n_rows, const int32_t* indptr, const int32_t* indices,
                const void* data, const void* data2, int64_t stride, const void* x, void* y,
                int accumulate, cudaStream_t st) {
    if (data2)
        bsr9_kernel<R, true, LPR><<<(unsigned)blocks, 256, 0, st>>>(
            n_rows, indptr, indices, (const R*)data, (const R*)data2, stride, (const R*)x, (R*)y,
            accumulate);
    else
        bsr9_kernel<R, false, LPR><<<(unsigned)blocks, 256, 0, st>>>(
            n_rows, indptr, indices, (const R*)data, nullptr, stride, (const R*)x, (R*)y,
            accumulate);
}

template <typename R>
int run_bsr(int64_t n_rows, const int32_t* indptr, const int32_t* indices, const void* data,
            const void* data2, int64_t stride, const void* x, void* y, int accumulate,
            cudaStream_t st) {
    const int threads = 256;
    int lpr = 32, cps = 8;
    bsr_shape(sizeof(R) == 8 ? TCT_F64 : TCT_F32, n_rows, stride, &lpr, &cps);
    const int64_t warps_needed = (n_rows + (32 / lpr) - 1) / (32 / lpr);
    const int64_t max_blocks = (int64_t)sm_count() * cps;
    int64_t blocks = (warps_needed * 32 + threads - 1) / threads;
    if (blocks > max_blocks) blocks = max_blocks;
    if (blocks < 1) blocks = 1;
    switch (lpr) {
        case 16: launch_bsr<R, 16>(blocks, n_rows, indptr, indices, data, data2, stride, x, y,
                                   accumulate, st); break;
        case 8: launch_bsr<R, 8>(blocks, n_rows, indptr, indices, data, data2, stride, x, y,
                                 accumulate, st); break;
        case 4: launch_bsr<R, 4>(blocks, n_rows, indptr, indices, data, data2, stride, x, y,
                                 accumulate, st); break;
        case 2: launch_bsr<R, 2>(blocks, n_rows, indptr, indices, data, data2, stride, x, y,
                                 accumulate, st); break;
        case 1: launch_bsr<R, 1>(blocks, n_rows, indptr, indices, data, data2, stride, x, y,
                                 accumulate, st); break;
        default: launch_bsr<R, 32>(blocks, n_rows, indptr, indices, data, data2, stride, x, y,
                                   accumulate, st);
    }
    return launch_status("tct_bsr9_matvec");
}


// Panel form: y_v (+)= A x_v for n_vec vectors (x_v at x + v * x_stride,
// y_v at y + v * y_stride).  Each block is read once per group of NV
// vectors: a lane loads column j of its block (9 values) and updates the
// NV x 9 row sums with x_v[col*9 + j].  The flattened grid puts the NV-vector
// groups of a row range in consecutive blocks, which run together, so a
// block row is fetched from HBM once and re-read from L2 by the other groups.
template <typename R, int NV>
__global__ void __launch_bounds__(256, 2)
bsr9_panel_kernel(int64_t n_rows, const int32_t* __restrict__ indptr,
                  const int32_t* __restrict__ indices, const R* __restrict__ data,
                  int64_t stride, const R* __restrict__ x, int64_t x_stride,
                  R* __restrict__ y, int64_t y_stride, int n_vec, int n_groups,
                  int accumulate) {
    const int lane = threadIdx.x & 31;
    const int group = (int)(blockIdx.x % (unsigned)n_groups);
    const int64_t xb = blockIdx.x / (unsigned)n_groups;
    const int64_t n_xb = gridDim.x / (unsigned)n_groups;
    const int v0 = group * NV;
    const int nv = min(NV, n_vec - v0);
    const int wpb = blockDim.x >> 5;
    const int64_t warp = xb * wpb + (threadIdx.x >> 5);
    const int64_t n_warps = n_xb * wpb;
    const R* xg = x + (int64_t)v0 * x_stride;
    for (int64_t row = warp; row < n_rows; row += n_warps) {
        const int32_t start = __ldg(indptr + row), end = __ldg(indptr + row + 1);
        R acc[NV][9];
#pragma unroll
        for (int v = 0; v < NV; v++)
#pragma unroll
            for (int i = 0; i < 9; i++) acc[v][i] = 0;
        for (int32_t s = start + lane; s < end; s += 32) {
            const int64_t col9 = (int64_t)__ldg(indices + s) * 9;
            if (col9 < 0) continue;  // padding slot
#pragma unroll 1
            for (int j = 0; j < 9; j++) {
                R a[9];
#pragma unroll
                for (int i = 0; i < 9; i++) a[i] = __ldg(data + (int64_t)(i * 9 + j) * stride + s);
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    if (v < nv) {
                        const R xs = __ldg(xg + v * x_stride + col9 + j);
#pragma unroll
                        for (int i = 0; i < 9; i++) acc[v][i] += a[i] * xs;
                    }
                }
            }
        }
#pragma unroll
        for (int v = 0; v < NV; v++) {
#pragma unroll
            for (int i = 0; i < 9; i++)
#pragma unroll
                for (int off = 16; off > 0; off >>= 1)
                    acc[v][i] += __shfl_xor_sync(0xffffffffu, acc[v][i], off);
            if (lane < 9 && v < nv) {
                R val = acc[v][0];
#pragma unroll
                for (int i = 1; i < 9; i++)
                    if (lane == i) val = acc[v][i];
                R* yp = y + (int64_t)(v0 + v) * y_stride + row * 9 + lane;
                *yp = accumulate ? *yp + val : val;
            }
        }
    }
}

template <typename R, int NV>
int run_bsr_panel(int64_t n_rows, const int32_t* indptr, const int32_t* indices,
                  const void* data, int64_t stride, const void* x, int64_t x_stride, void* y,
                  int64_t y_stride, int n_vec, int accumulate, cudaStream_t st) {
    const int threads = 256;
    const int n_groups = (n_vec + NV - 1) / NV;
    const int64_t max_xb = std::max<int64_t>(1, (int64_t)sm_count() * 4 / n_groups);
    int64_t xb = (n_rows * 32 + threads - 1) / threads;
    if (xb > max_xb) xb = max_xb;
    if (xb < 1) xb = 1;
    bsr9_panel_kernel<R, NV><<<(unsigned)(xb * n_groups), threads, 0, st>>>(
        n_rows, indptr, indices, (const R*)data, stride, (const R*)x, x_stride, (R*)y, y_stride,
        n_vec, n_groups, accumulate);
    return launch_status("tct_bsr9_matvec_panel");
}

}  // namespace
}  // namespace tct

extern "C" int tct_bsr9_matvec(int prec, int64_t n_row_blocks, const int32_t* indptr,
                               const int32_t* indices, const void* data, const void* data2,
                               int64_t data_stride, const void* x, void* y, int accumulate,
                               void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(n_row_blocks >= 0 && data_stride >= 0, "tct_bsr9_matvec: negative size");
    if (n_row_blocks == 0) return TCT_OK;
    TCT_CHECK_ARG(indptr && y, "tct_bsr9_matvec: null pointer");
    TCT_CHECK_ARG(data_stride < (int64_t(1) << 31), "tct_bsr9_matvec: more than 2^31 blocks");
    if (prec == TCT_F32)
        return run_bsr<float>(n_row_blocks, indptr, indices, data, data2, data_stride, x, y,
                              accumulate, as_stream(stream));
    if (prec == TCT_F64)
        return run_bsr<double>(n_row_blocks, indptr, indices, data, data2, data_stride, x, y,
                               accumulate, as_stream(stream));
    set_error("tct_bsr9_matvec: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}

// Candidate shapes (lanes per row x CTAs per SM), each timed as one untimed
// launch then the mean of eight under CUDA events; the fastest stays in the
// shape cache.  (On the 5.5 M-block C2 matrix, 32 lanes: 4 / 6 / 8 / 12 / 16
// CTAs per SM took 0.398 / 0.342 / 0.345 / 0.343 / 0.355 ms, and 3 -- one
// resident wave -- 0.409 ms: warps that finish early leave their SM idle
// until the whole CTA exits; with three timed launches the 3 % between 8
// and 16 was within the noise of the pick.)  Lane counts below a quarter
// of min(32, slots per row) are skipped: on rows of ~90 blocks the 1-, 2-
// and 4-lane shapes take 2 to 8 ms a launch against 0.35 ms, and timing
// them was most of the tuning time.
extern "C" int tct_bsr9_autotune(int prec, int64_t n_row_blocks, const int32_t* indptr,
                                 const int32_t* indices, const void* data, int64_t data_stride,
                                 const void* x, void* y, void* stream, int* lanes,
                                 int* ctas_per_sm) {
    using namespace tct;
    TCT_CHECK_ARG(lanes && ctas_per_sm, "tct_bsr9_autotune: null result pointer");
    TCT_CHECK_ARG(n_row_blocks > 0, "tct_bsr9_autotune: empty matrix");
    const int64_t per_row = std::max<int64_t>(1, data_stride / n_row_blocks);
    static const int kLanes[] = {32, 16, 8, 4, 2, 1};
    static const int kCtas[] = {4, 6, 8, 12, 16};
    cudaStream_t st = as_stream(stream);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return launch_status("tct_bsr9_autotune events");
    int had0 = 0, had1 = 0;
    const bool had = tune_lookup(kTuneBsr9, -1, prec, 0, 1, n_row_blocks, per_row, &had0, &had1);
    int rc = TCT_OK, bl = 0, bc = 0;
    float best_ms = 0.f;
    for (int l : kLanes) {
        if (4 * (int64_t)l < std::min<int64_t>(32, per_row)) continue;
        for (int c : kCtas) {
            tune_store(kTuneBsr9, -1, prec, 0, 1, n_row_blocks, per_row, l, c);
            for (int rep = 0; rep < 9 && rc == TCT_OK; rep++) {
                if (rep == 1) cudaEventRecord(e0, st);
                rc = tct_bsr9_matvec(prec, n_row_blocks, indptr, indices, data, nullptr,
                                     data_stride, x, y, 0, stream);
            }
            if (rc != TCT_OK) break;
            float ms = 0.f;
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                rc = launch_status("tct_bsr9_autotune timing");
                break;
            }
            if (bl == 0 || ms < best_ms) {
                bl = l;
                bc = c;
                best_ms = ms;
            }
        }
        if (rc != TCT_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != TCT_OK || bl == 0) {
        if (had) tune_store(kTuneBsr9, -1, prec, 0, 1, n_row_blocks, per_row, had0, had1);
        else tune_erase(kTuneBsr9, -1, prec, 0, 1, n_row_blocks, per_row);
        return rc != TCT_OK ? rc : TCT_ERR_ARG;
    }
    tune_store(kTuneBsr9, -1, prec, 0, 1, n_row_blocks, per_row, bl, bc);
    *lanes = bl;
    *ctas_per_sm = bc;
    return TCT_OK;
}

extern "C" int tct_bsr9_matvec_panel(int prec, int64_t n_row_blocks, const int32_t* indptr,
                                     const int32_t* indices, const void* data,
                                     int64_t data_stride, const void* x, int64_t x_stride,
                                     void* y, int64_t y_stride, int n_vec, int accumulate,
                                     void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(n_row_blocks >= 0 && data_stride >= 0 && n_vec >= 0,
                  "tct_bsr9_matvec_panel: negative size");
    if (n_row_blocks == 0 || n_vec == 0) return TCT_OK;
    TCT_CHECK_ARG(indptr && y && x, "tct_bsr9_matvec_panel: null pointer");
    TCT_CHECK_ARG(data_stride < (int64_t(1) << 31), "tct_bsr9_matvec_panel: more than 2^31 blocks");
    TCT_CHECK_ARG(n_vec == 1 || (x_stride >= 0 && y_stride >= 9 * n_row_blocks),
                  "tct_bsr9_matvec_panel: vector strides overlap");
    if (prec == TCT_F32)
        return run_bsr_panel<float, 8>(n_row_blocks, indptr, indices, data, data_stride, x,
                                       x_stride, y, y_stride, n_vec, accumulate,
                                       as_stream(stream));
    if (prec == TCT_F64)
        return run_bsr_panel<double, 4>(n_row_blocks, indptr, indices, data, data_stride, x,
                                        x_stride, y, y_stride, n_vec, accumulate,
                                        as_stream(stream));
    set_error("tct_bsr9_matvec_panel: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}
