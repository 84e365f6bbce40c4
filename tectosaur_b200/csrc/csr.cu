// CSR sparse matrix-vector product for the constraint matrices of the
// constrained solve: y (+)= A x with A = cm or cm^T (examples/solve.py:44-49,
// simple_solver.py:14-33, where scipy's csr_matrix.dot does it on the host).
// Constraint matrices have a handful of entries per row, so a thread owns a
// row; values are stored in double (constraint coefficients), x / y in Real.
#include "common.cuh"

namespace tct {
namespace {

template <typename R>
__global__ void __launch_bounds__(256)
csr_kernel(int64_t n_rows, const int64_t* __restrict__ indptr,
           const int64_t* __restrict__ indices, const double* __restrict__ data,
           const R* __restrict__ x, R* __restrict__ y, int accumulate, int64_t x_stride,
           int64_t y_stride) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rows) return;
    x += blockIdx.y * x_stride;  // vector blockIdx.y of a panel
    y += blockIdx.y * y_stride;
    double s = 0;
    for (int64_t k = indptr[i]; k < indptr[i + 1]; k++) s += data[k] * (double)x[indices[k]];
    y[i] = accumulate ? (R)((double)y[i] + s) : (R)s;
}

}  // namespace
}  // namespace tct

using namespace tct;

extern "C" int tct_csr_matvec_panel(int prec, int64_t n_rows, const int64_t* indptr,
                                    const int64_t* indices, const double* data, const void* x,
                                    int64_t x_stride, void* y, int64_t y_stride, int n_vec,
                                    int accumulate, void* stream) {
    TCT_CHECK_ARG(n_rows >= 0 && n_vec >= 0 && n_vec < 65536,
                  "tct_csr_matvec: bad row or vector count");
    if (n_rows == 0 || n_vec == 0) return TCT_OK;
    TCT_CHECK_ARG(indptr && x && y, "tct_csr_matvec: null pointer");
    cudaStream_t st = as_stream(stream);
    const dim3 grid((unsigned)((n_rows + 255) / 256), (unsigned)n_vec);
    if (prec == TCT_F64) {
        csr_kernel<double><<<grid, 256, 0, st>>>(n_rows, indptr, indices, data, (const double*)x,
                                                 (double*)y, accumulate, x_stride, y_stride);
    } else if (prec == TCT_F32) {
        csr_kernel<float><<<grid, 256, 0, st>>>(n_rows, indptr, indices, data, (const float*)x,
                                                (float*)y, accumulate, x_stride, y_stride);
    } else {
        set_error("tct_csr_matvec: unsupported precision %d", prec);
        return TCT_ERR_PREC;
    }
    return launch_status("csr matvec");
}

extern "C" int tct_csr_matvec(int prec, int64_t n_rows, const int64_t* indptr,
                              const int64_t* indices, const double* data, const void* x, void* y,
                              int accumulate, void* stream) {
    return tct_csr_matvec_panel(prec, n_rows, indptr, indices, data, x, 0, y, 0, 1, accumulate,
                                stream);
}
