// Triangle-pair quadrature: the 81-entry (3x3x3x3) interaction block of each
// (observation, source) triangle pair under a 4-D quadrature rule.
//
// Restates single_pairs{Z,N} and single_pairs{N}_adj of the reference
// (tectosaur/assemble.cl:24-103, integrate_pair of
// tectosaur/integral_primitives.cl:174-213 and the tensor forms of
// tectosaur/kernels/__init__.py and tectosaur/kernels/kernels.cl:29-98).
//
// One thread integrates one pair: the rule is shared by every pair of a
// launch, so the warp reads each quadrature point once (broadcast) and the
// work per thread is uniform.  FP32 keeps the reference's Kahan-compensated
// accumulation for the U/T/A/H tensor forms; FP64 accumulates directly (its
// rounding error is far below the 1e-10 parity bar).
#include "pair_math.cuh"

namespace tct {
namespace {

template <typename R, int K, bool ADJ>
__global__ void __launch_bounds__(128)
pairs_kernel(Consts<R> c, int check0, R* __restrict__ out,
             const int32_t* __restrict__ out_slot, int64_t slot_stride, R sign,
             int accumulate, int n_q, const R* __restrict__ qp, const R* __restrict__ qw,
             const R* __restrict__ pts, const int32_t* __restrict__ tris,
             const int32_t* __restrict__ pairs, int64_t n_pairs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pairs) return;
    constexpr int rec = ADJ ? 5 : 2;
    const int oi = pairs[i * rec], si = pairs[i * rec + 1];
    const int oc = ADJ ? pairs[i * rec + 2] : 0;
    const int scl = ADJ ? pairs[i * rec + 3] : 0;
    const bool flip = ADJ ? (pairs[i * rec + 4] != 0) : false;
    constexpr bool need_osc = (K == kRA || K == kRH);
    constexpr bool need_ssc = (K == kRT || K == kRH);
    TriGeom<R> o, s;
    load_tri(o, pts, tris, oi, oc, false, need_osc);
    load_tri(s, pts, tris, si, scl, flip, need_ssc);
    R res[81];
    constexpr bool kahan = (sizeof(R) == 4) && (K <= kH);
    // adjacent pairs always skip r^2 == 0 points (assemble.cl:67)
    integrate_pair<R, K, kahan>(c, o, s, n_q, qp, qw, ADJ ? true : (check0 != 0), res);
    const R scale = o.J * s.J;
    int od[3] = {0, 1, 2}, sd[3] = {0, 1, 2};
    if (ADJ) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            od[k] = positive_mod(-oc + k, 3);
            sd[k] = positive_mod(-scl + k, 3);
        }
        if (flip) {
            int t = sd[0];
            sd[0] = sd[1];
            sd[1] = t;
        }
    }
    const int64_t slot = out_slot ? (int64_t)out_slot[i] : i;
#pragma unroll
    for (int b1 = 0; b1 < 3; b1++)
#pragma unroll
        for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
            for (int b2 = 0; b2 < 3; b2++)
#pragma unroll
                for (int d2 = 0; d2 < 3; d2++) {
                    const int out_idx = b1 * 27 + d1 * 9 + b2 * 3 + d2;
                    R val;
                    if (ADJ) {
                        // de-rotation of the outputs (assemble.cl:77-101); selected
                        // with compile-time indices so res[] stays in registers
                        val = 0;
#pragma unroll
                        for (int a = 0; a < 3; a++)
#pragma unroll
                            for (int b = 0; b < 3; b++)
                                if (od[b1] == a && sd[b2] == b) val = res[a * 27 + d1 * 9 + b * 3 + d2];
                    } else {
                        val = res[out_idx];
                    }
                    val = sign * (scale * val);
                    R* dst = out_slot ? (out + (int64_t)out_idx * slot_stride + slot)
                                      : (out + slot * 81 + out_idx);
                    if (accumulate) *dst += val;
                    else *dst = val;
                }
}

template <typename R>
int launch_pairs(int kernel, int adj, int check0, void* out, const int32_t* out_slot,
                 int64_t slot_stride, int sign, int accumulate, int n_quad,
                 const void* qp, const void* qw, const void* pts, const int32_t* tris,
                 const int32_t* pairs, int64_t n_pairs, const double* params,
                 cudaStream_t st) {
    Consts<R> c = make_consts<R>(params);
    const int threads = 128;
    const int64_t blocks = (n_pairs + threads - 1) / threads;
    const R sg = sign < 0 ? R(-1) : R(1);
#define TCT_PAIRS_CASE(KID)                                                                   \
    case KID:                                                                                 \
        if (adj)                                                                              \
            pairs_kernel<R, KID, true><<<(unsigned)blocks, threads, 0, st>>>(                \
                c, check0, (R*)out, out_slot, slot_stride, sg, accumulate, n_quad,          \
                (const R*)qp, (const R*)qw, (const R*)pts, tris, pairs, n_pairs);          \
        else                                                                                  \
            pairs_kernel<R, KID, false><<<(unsigned)blocks, threads, 0, st>>>(               \
                c, check0, (R*)out, out_slot, slot_stride, sg, accumulate, n_quad,          \
                (const R*)qp, (const R*)qw, (const R*)pts, tris, pairs, n_pairs);          \
        break;
    switch (kernel) {
        TCT_PAIRS_CASE(kU)
        TCT_PAIRS_CASE(kT)
        TCT_PAIRS_CASE(kA)
        TCT_PAIRS_CASE(kH)
        TCT_PAIRS_CASE(kRT)
        TCT_PAIRS_CASE(kRA)
        TCT_PAIRS_CASE(kRH)
        default:
            set_error("tct_pairs_integrate: unsupported kernel id %d", kernel);
            return TCT_ERR_KERNEL;
    }
#undef TCT_PAIRS_CASE
    return launch_status("tct_pairs_integrate");
}

}  // namespace
}  // namespace tct

extern "C" int tct_pairs_integrate(int kernel, int prec, int adj, int check0, void* out,
                                   const int32_t* out_slot, int64_t slot_stride, int sign,
                                   int accumulate, int n_quad, const void* quad_pts,
                                   const void* quad_wts, const void* pts, const int32_t* tris,
                                   const int32_t* pairs, int64_t n_pairs, const double* params,
                                   void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(n_pairs >= 0, "tct_pairs_integrate: n_pairs < 0");
    if (n_pairs == 0) return TCT_OK;
    TCT_CHECK_ARG(n_pairs < (int64_t(1) << 31) * 128, "tct_pairs_integrate: too many pairs");
    TCT_CHECK_ARG(out && pts && tris && pairs && params, "tct_pairs_integrate: null pointer");
    TCT_CHECK_ARG(n_quad > 0 && quad_pts && quad_wts, "tct_pairs_integrate: empty rule");
    TCT_CHECK_ARG(!out_slot || slot_stride > 0, "tct_pairs_integrate: slot_stride must be > 0");
    TCT_CHECK_ARG(adj == 0 || adj == 1, "tct_pairs_integrate: adj must be 0 or 1");
    if (prec == TCT_F32)
        return launch_pairs<float>(kernel, adj, check0, out, out_slot, slot_stride, sign,
                                   accumulate, n_quad, quad_pts, quad_wts, pts, tris, pairs,
                                   n_pairs, params, as_stream(stream));
    if (prec == TCT_F64)
        return launch_pairs<double>(kernel, adj, check0, out, out_slot, slot_stride, sign,
                                    accumulate, n_quad, quad_pts, quad_wts, pts, tris, pairs,
                                    n_pairs, params, as_stream(stream));
    set_error("tct_pairs_integrate: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}
