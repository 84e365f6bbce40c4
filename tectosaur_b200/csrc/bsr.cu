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
#include "common.cuh"

namespace tct {
namespace {

// At most 64 registers per thread (4 blocks of 256 threads per SM): left
// unconstrained the compiler hoists all 81 block loads into registers (222
// registers, 1 block per SM) and the per-row shuffle reduction then leaves
// the SM with no loads in flight.
template <typename R, bool TWO>
__global__ void __launch_bounds__(256, 4)
bsr9_kernel(int64_t n_rows, const int32_t* __restrict__ indptr,
            const int32_t* __restrict__ indices, const R* __restrict__ data,
            const R* __restrict__ data2, int64_t stride, const R* __restrict__ x,
            R* __restrict__ y, int accumulate) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t row = warp; row < n_rows; row += n_warps) {
        const int32_t start = __ldg(indptr + row), end = __ldg(indptr + row + 1);
        R acc[9];
#pragma unroll
        for (int i = 0; i < 9; i++) acc[i] = 0;
        for (int32_t s = start + lane; s < end; s += 32) {
            const int64_t col = __ldg(indices + s);
            R xv[9];
#pragma unroll
            for (int j = 0; j < 9; j++) xv[j] = __ldg(x + col * 9 + j);
#pragma unroll
            for (int i = 0; i < 9; i++)
#pragma unroll
                for (int j = 0; j < 9; j++) {
                    // default (L2-retaining) loads: a row's segment of each
                    // element plane shares its first and last 128-byte lines
                    // with the neighbouring rows, read by nearby warps
                    R a = __ldg(data + (int64_t)(i * 9 + j) * stride + s);
                    if (TWO) a += __ldg(data2 + (int64_t)(i * 9 + j) * stride + s);
                    acc[i] += a * xv[j];
                }
        }
#pragma unroll
        for (int i = 0; i < 9; i++) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
        }
        if (lane < 9) {
            R v = acc[0];
#pragma unroll
            for (int i = 1; i < 9; i++)
                if (lane == i) v = acc[i];
            R* yp = y + row * 9 + lane;
            *yp = accumulate ? *yp + v : v;
        }
    }
}

template <typename R>
int run_bsr(int64_t n_rows, const int32_t* indptr, const int32_t* indices, const void* data,
            const void* data2, int64_t stride, const void* x, void* y, int accumulate,
            cudaStream_t st) {
    const int threads = 256;
    const int64_t warps_needed = n_rows;
    const int64_t max_blocks = (int64_t)sm_count() * 8;
    int64_t blocks = (warps_needed * 32 + threads - 1) / threads;
    if (blocks > max_blocks) blocks = max_blocks;
    if (blocks < 1) blocks = 1;
    if (data2)
        bsr9_kernel<R, true><<<(unsigned)blocks, threads, 0, st>>>(
            n_rows, indptr, indices, (const R*)data, (const R*)data2, stride, (const R*)x, (R*)y,
            accumulate);
    else
        bsr9_kernel<R, false><<<(unsigned)blocks, threads, 0, st>>>(
            n_rows, indptr, indices, (const R*)data, nullptr, stride, (const R*)x, (R*)y,
            accumulate);
    return launch_status("tct_bsr9_matvec");
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
