// Fused element-wise pieces of the batched (served) quasidynamic step: the
// slip deficit that drives the traction solve, the derivative's assembly
// with the reference's rejection of non-finite or out-of-range states, the
// RK23 stage combinations and the error norm, each one launch over all
// states instead of a chain of element-wise tensor operations (the
// reference evaluates them with numpy on the host: qd/full_model.py:178-200
// for the derivative, scipy's RK23 step for the combinations).
//
// Every value is rounded in the order of the element-wise expressions they
// replace, one IEEE operation at a time (no fused multiply-add), so the
// results are bit-identical to them; only the error norm's sum of squares
// is a block reduction (a different summation order).
#include <cmath>

#include "common.cuh"

namespace tct {
namespace {

// out[r][i] = interior[i] * ((ts[r] * plate_rate) * inslipdir[i] - Y[r][i])
template <typename O>
__global__ void __launch_bounds__(256)
qd_deficit_kernel(int64_t n9, int n_sys, const double* __restrict__ ts, double plate_rate,
                  const double* __restrict__ dir, const double* __restrict__ interior,
                  const double* __restrict__ Y, int64_t y_stride, O* __restrict__ out,
                  int64_t out_stride) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n9 * n_sys) return;
    const int r = (int)(g / n9);
    const int64_t i = g % n9;
    const double tr = __dmul_rn(ts[r], plate_rate);
    const double plate = __dmul_rn(tr, dir[i]);
    const double d = __dmul_rn(interior[i], __dsub_rn(plate, Y[r * y_stride + i]));
    out[r * out_stride + i] = (O)d;
}

// One CTA per state: the state is rejected (its derivative is Y * inf) when
// Y has a non-finite entry, a state variable below 0 or above state_max, or
// the velocity a non-finite entry; else the derivative is (V, dstate).
__global__ void __launch_bounds__(256)
qd_finish_kernel(int64_t n9, int64_t n_state, const double* __restrict__ Y, int64_t y_stride,
                 const double* __restrict__ V, int64_t v_stride, const double* __restrict__ dstate,
                 int64_t ds_stride, double state_max, double* __restrict__ out,
                 int64_t out_stride) {
    const int r = blockIdx.x;
    const double* y = Y + r * y_stride;
    const double* v = V + r * v_stride;
    const double* ds = dstate + r * ds_stride;
    double* o = out + r * out_stride;
    const int64_t n_y = n9 + n_state;
    int bad = 0;
    for (int64_t i = threadIdx.x; i < n_y; i += blockDim.x) {
        const double a = y[i];
        if (!isfinite(a)) bad = 1;
        if (i >= n9 && (a < 0.0 || a > state_max)) bad = 1;
        if (i < n9 && !isfinite(v[i])) bad = 1;
    }
    bad = __syncthreads_or(bad);
    if (bad) {
        for (int64_t i = threadIdx.x; i < n_y; i += blockDim.x)
            o[i] = __dmul_rn(y[i], (double)INFINITY);
    } else {
        for (int64_t i = threadIdx.x; i < n_y; i += blockDim.x) o[i] = i < n9 ? v[i] : ds[i - n9];
    }
}

struct Terms {
    const double* k[4];
    int64_t stride[4];
    double c[4];
    int n;
};

// s = ((K0 c0 + K1 c1) + K2 c2) + K3 c3 for the first n terms, left to right
__device__ __forceinline__ double combine(const Terms& T, int r, int64_t i) {
    double s = __dmul_rn(T.k[0][r * T.stride[0] + i], T.c[0]);
#pragma unroll
    for (int j = 1; j < 4; j++)
        if (j < T.n) s = __dadd_rn(s, __dmul_rn(T.k[j][r * T.stride[j] + i], T.c[j]));
    return s;
}

// out[r][i] = y[r][i] + s * h[r]   (y may be null: out = s * h[r])
__global__ void __launch_bounds__(256)
qd_combine_kernel(int64_t n, int n_sys, Terms T, const double* __restrict__ h,
                  const double* __restrict__ y, int64_t y_stride, double* __restrict__ out,
                  int64_t out_stride) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n * n_sys) return;
    const int r = (int)(g / n);
    const int64_t i = g % n;
    const double sh = __dmul_rn(combine(T, r, i), h[r]);
    out[r * out_stride + i] = y ? __dadd_rn(y[r * y_stride + i], sh) : sh;
}

// One CTA per state: norms[r] = || (s h[r]) / (tol + max(|y|, |y_new|) tol) ||_2
__global__ void __launch_bounds__(256)
qd_error_norm_kernel(int64_t n, Terms T, const double* __restrict__ h,
                     const double* __restrict__ y, int64_t y_stride,
                     const double* __restrict__ y_new, int64_t yn_stride, double tol,
                     double* __restrict__ norms) {
    __shared__ double red[256];
    const int r = blockIdx.x;
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double err = __dmul_rn(combine(T, r, i), h[r]);
        const double m = fmax(fabs(y[r * y_stride + i]), fabs(y_new[r * yn_stride + i]));
        const double scale = __dadd_rn(tol, __dmul_rn(m, tol));
        const double q = __ddiv_rn(err, scale);
        acc = __dadd_rn(acc, __dmul_rn(q, q));
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) norms[r] = sqrt(red[0]);
}

int make_terms(Terms& T, int n_terms, const double* const* k, const int64_t* strides,
               const double* coeffs) {
    TCT_CHECK_ARG(n_terms >= 1 && n_terms <= 4 && k && strides && coeffs,
                  "qd combination: 1 to 4 terms with their arrays");
    T.n = n_terms;
    for (int j = 0; j < 4; j++) {
        T.k[j] = j < n_terms ? k[j] : nullptr;
        T.stride[j] = j < n_terms ? strides[j] : 0;
        T.c[j] = j < n_terms ? coeffs[j] : 0.0;
        if (j < n_terms) TCT_CHECK_ARG(k[j], "qd combination: null term %d", j);
    }
    return TCT_OK;
}

}  // namespace
}  // namespace tct

using namespace tct;

extern "C" int tct_qd_deficit_batch(int64_t n9, int n_sys, const double* ts, double plate_rate,
                                    const double* inslipdir, const double* interior,
                                    const double* Y, int64_t y_stride, int out_prec, void* out,
                                    int64_t out_stride, void* stream) {
    TCT_CHECK_ARG(n9 >= 0 && n_sys >= 0, "tct_qd_deficit_batch: negative size");
    if (n9 == 0 || n_sys == 0) return TCT_OK;
    TCT_CHECK_ARG(ts && inslipdir && interior && Y && out, "tct_qd_deficit_batch: null pointer");
    const unsigned nb = (unsigned)((n9 * n_sys + 255) / 256);
    cudaStream_t st = as_stream(stream);
    if (out_prec == TCT_F64)
        qd_deficit_kernel<double><<<nb, 256, 0, st>>>(n9, n_sys, ts, plate_rate, inslipdir,
                                                      interior, Y, y_stride, (double*)out,
                                                      out_stride);
    else if (out_prec == TCT_F32)
        qd_deficit_kernel<float><<<nb, 256, 0, st>>>(n9, n_sys, ts, plate_rate, inslipdir,
                                                     interior, Y, y_stride, (float*)out,
                                                     out_stride);
    else
        TCT_CHECK_ARG(false, "tct_qd_deficit_batch: unsupported precision %d", out_prec);
    return launch_status("tct_qd_deficit_batch");
}

extern "C" int tct_qd_finish_batch(int64_t n9, int64_t n_state, int n_sys, const double* Y,
                                   int64_t y_stride, const double* V, int64_t v_stride,
                                   const double* dstate, int64_t ds_stride, double state_max,
                                   double* out, int64_t out_stride, void* stream) {
    TCT_CHECK_ARG(n9 >= 0 && n_state >= 0 && n_sys >= 0, "tct_qd_finish_batch: negative size");
    if (n_sys == 0 || n9 + n_state == 0) return TCT_OK;
    TCT_CHECK_ARG(Y && V && dstate && out, "tct_qd_finish_batch: null pointer");
    qd_finish_kernel<<<(unsigned)n_sys, 256, 0, as_stream(stream)>>>(
        n9, n_state, Y, y_stride, V, v_stride, dstate, ds_stride, state_max, out, out_stride);
    return launch_status("tct_qd_finish_batch");
}

extern "C" int tct_qd_combine_batch(int64_t n, int n_sys, int n_terms, const double* const* k,
                                    const int64_t* k_strides, const double* coeffs,
                                    const double* h, const double* y, int64_t y_stride,
                                    double* out, int64_t out_stride, void* stream) {
    TCT_CHECK_ARG(n >= 0 && n_sys >= 0, "tct_qd_combine_batch: negative size");
    if (n == 0 || n_sys == 0) return TCT_OK;
    TCT_CHECK_ARG(h && out, "tct_qd_combine_batch: null pointer");
    Terms T;
    int rc = make_terms(T, n_terms, k, k_strides, coeffs);
    if (rc) return rc;
    qd_combine_kernel<<<(unsigned)((n * n_sys + 255) / 256), 256, 0, as_stream(stream)>>>(
        n, n_sys, T, h, y, y_stride, out, out_stride);
    return launch_status("tct_qd_combine_batch");
}

extern "C" int tct_qd_error_norm_batch(int64_t n, int n_sys, int n_terms, const double* const* k,
                                       const int64_t* k_strides, const double* coeffs,
                                       const double* h, const double* y, int64_t y_stride,
                                       const double* y_new, int64_t yn_stride, double tol,
                                       double* norms, void* stream) {
    TCT_CHECK_ARG(n >= 0 && n_sys >= 0, "tct_qd_error_norm_batch: negative size");
    if (n_sys == 0) return TCT_OK;
    TCT_CHECK_ARG(h && y && y_new && norms, "tct_qd_error_norm_batch: null pointer");
    Terms T;
    int rc = make_terms(T, n_terms, k, k_strides, coeffs);
    if (rc) return rc;
    qd_error_norm_kernel<<<(unsigned)n_sys, 256, 0, as_stream(stream)>>>(
        n, T, h, y, y_stride, y_new, yn_stride, tol, norms);
    return launch_status("tct_qd_error_norm_batch");
}
