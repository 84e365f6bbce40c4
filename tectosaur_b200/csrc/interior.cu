// Interior evaluation: the displacement/traction of a boundary field at
// observation points off (or on the vertices of) the surface
// (tectosaur/interior.py InteriorOp).
//
//   interior_pairs   one thread per (observation point, source triangle,
//                    clicks) pair: the 27 entries [d_obs][b_src][d_src] =
//                    J_s sum_q w_q phi_b(q) K(x, y_q) of a U/T/A/H tensor
//                    kernel over a triangle rule, Kahan-summed, de-rotated
//                    (assemble.cl:140-186 with integrate_pt_tri,
//                    integral_primitives.cl:216-258);
//   interior_corners one thread per pair whose observation point is source
//                    vertex `clicks`: elasticH3 with the radial integral
//                    from the vertex in closed form and a Gauss rule over
//                    the angle (interior_corners.cl).  The reference kernel
//                    scales its log-term tensor I4 by the integer quotient
//                    1/3, which is 0, so only the 1/r^3 tensor I3 and the
//                    scalar terms I1, I2 contribute; restated as is.
#include "common.cuh"
#include "pair_math.cuh"

namespace tct {
namespace {

template <typename R, int K>
__global__ void __launch_bounds__(128)
interior_pairs_kernel(Consts<R> c, R* __restrict__ result, int n_q, const R* __restrict__ qp,
                      const R* __restrict__ qw, const R* __restrict__ obs_pts,
                      const R* __restrict__ obs_ns, const R* __restrict__ pts,
                      const int32_t* __restrict__ tris, const int32_t* __restrict__ pairs,
                      int64_t n_pairs, int finite_part) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pairs) return;
    const int obs = pairs[3 * i], src = pairs[3 * i + 1], clicks = pairs[3 * i + 2];
    TriGeom<R> s;
    load_tri(s, pts, tris, src, clicks, false, false);
    const R x[3] = {obs_pts[3 * (int64_t)obs], obs_pts[3 * (int64_t)obs + 1],
                    obs_pts[3 * (int64_t)obs + 2]};
    const R no[3] = {obs_ns[3 * (int64_t)obs], obs_ns[3 * (int64_t)obs + 1],
                     obs_ns[3 * (int64_t)obs + 2]};
    R rt[27], kc[27];
#pragma unroll
    for (int k = 0; k < 27; k++) rt[k] = kc[k] = 0;
    for (int iq = 0; iq < n_q; iq++) {
        const R sx = __ldg(qp + 2 * iq), sy = __ldg(qp + 2 * iq + 1), w = __ldg(qw + iq);
        const R sb[3] = {1 - sx - sy, sx, sy};
        R D[3];
#pragma unroll
        for (int d = 0; d < 3; d++) D[d] = bary_point(s, sb, d) - x[d];
        const R r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
        R Karr[9];
        karr_utah<R, K>(c, D, r2, no, s.n, Karr);
        const R ob = R(1) * w;
#pragma unroll
        for (int dob = 0; dob < 3; dob++)
#pragma unroll
            for (int bs = 0; bs < 3; bs++)
#pragma unroll
                for (int ds = 0; ds < 3; ds++) {
                    const int idx = dob * 9 + bs * 3 + ds;
                    const R val = ob * sb[bs] * Karr[dob * 3 + ds];
                    const R yk = val - kc[idx];
                    const R t = rt[idx] + yk;
                    kc[idx] = (t - rt[idx]) - yk;
                    rt[idx] = t;
                }
    }
    int derot[3];
#pragma unroll
    for (int b = 0; b < 3; b++) derot[b] = positive_mod(-clicks + b, 3);
    R* out = result + i * 27;
#pragma unroll
    for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
        for (int b2 = 0; b2 < 3; b2++)
#pragma unroll
            for (int d2 = 0; d2 < 3; d2++) {
                R v = s.J * rt[d1 * 9 + derot[b2] * 3 + d2];
                if (finite_part && b2 != clicks) v = 0;
                out[d1 * 9 + b2 * 3 + d2] = v;
            }
}

template <typename R>
__global__ void __launch_bounds__(128)
interior_corners_kernel(Consts<R> c, R* __restrict__ result, int n_q, const R* __restrict__ qt,
                        const R* __restrict__ qw, const R* __restrict__ obs_ns,
                        const R* __restrict__ pts, const int32_t* __restrict__ tris,
                        const int32_t* __restrict__ pairs, int64_t n_pairs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pairs) return;
    const int obs = pairs[3 * i], src = pairs[3 * i + 1], clicks = pairs[3 * i + 2];
    TriGeom<R> s;
    load_tri(s, pts, tris, src, clicks, false, false);
    const R no[3] = {obs_ns[3 * (int64_t)obs], obs_ns[3 * (int64_t)obs + 1],
                     obs_ns[3 * (int64_t)obs + 2]};
    const R mn = no[0] * s.n[0] + no[1] * s.n[1] + no[2] * s.n[2];
    R v1[3], v2[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        v1[d] = s.v[1][d] - s.v[0][d];
        v2[d] = s.v[2][d] - s.v[0][d];
    }
    R rt[27], kc[27];
#pragma unroll
    for (int k = 0; k < 27; k++) rt[k] = kc[k] = 0;
    const R CH03 = c.CsH0 * c.CsH3, CH01 = c.CsH0 * c.CsH1;
    for (int iq = 0; iq < n_q; iq++) {
        const R t = __ldg(qt + iq), w = __ldg(qw + iq);
        const R ct = cos(t), st = sin(t);
        const R rhomax = R(1.0) / (ct + st);
        R a[3];
#pragma unroll
        for (int d = 0; d < 3; d++) a[d] = v1[d] * ct + v2[d] * st;
        const R A2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
        const R A = sqrt(A2);
        const R A3 = A2 * A;
        const R A5 = (A3 * A) * A;
        const R I1 = R(-1) / (A3 * rhomax);
        const R I2 = (log(R(2.0)) + log(A) + log(rhomax) - 1) / A3;
        const R T0[3] = {-I2 * ct - I2 * st + I1, I2 * ct, I2 * st};
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int dob = 0; dob < 3; dob++)
#pragma unroll
                for (int ds = 0; ds < 3; ds++) {
                    // the 1/r^3 tensor enters through basis 0 only
                    const R T1 = b == 0 ? (-a[dob]) * a[ds] / (A5 * rhomax) : R(0);
                    R Kval = 0;
                    Kval += CH03 * T1 * mn;
                    if (dob == ds) Kval += CH01 * mn * T0[b];
                    const int idx = dob * 9 + b * 3 + ds;
                    const R val = w * Kval;
                    const R yk = val - kc[idx];
                    const R tt = rt[idx] + yk;
                    kc[idx] = (tt - rt[idx]) - yk;
                    rt[idx] = tt;
                }
    }
    int derot[3];
#pragma unroll
    for (int b = 0; b < 3; b++) derot[b] = positive_mod(-clicks + b, 3);
    R* out = result + i * 27;
#pragma unroll
    for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
        for (int b2 = 0; b2 < 3; b2++)
#pragma unroll
            for (int d2 = 0; d2 < 3; d2++)
                out[d1 * 9 + b2 * 3 + d2] = s.J * rt[d1 * 9 + derot[b2] * 3 + d2];
}

template <typename R>
int run_interior_pairs(int kernel, const double* params, void* result, int n_q, const void* qp,
                       const void* qw, const void* obs_pts, const void* obs_ns, const void* pts,
                       const int32_t* tris, const int32_t* pairs, int64_t n_pairs,
                       int finite_part, cudaStream_t st) {
    const Consts<R> c = make_consts<R>(params);
    const unsigned blocks = (unsigned)((n_pairs + 127) / 128);
#define TCT_INT_CASE(KID)                                                                   \
    case KID:                                                                               \
        interior_pairs_kernel<R, KID><<<blocks, 128, 0, st>>>(                              \
            c, (R*)result, n_q, (const R*)qp, (const R*)qw, (const R*)obs_pts,              \
            (const R*)obs_ns, (const R*)pts, tris, pairs, n_pairs, finite_part);            \
        break;
    switch (kernel) {
        TCT_INT_CASE(kU)
        TCT_INT_CASE(kT)
        TCT_INT_CASE(kA)
        TCT_INT_CASE(kH)
        default:
            set_error("tct_interior_pairs: kernel id %d has no point-observation form", kernel);
            return TCT_ERR_KERNEL;
    }
#undef TCT_INT_CASE
    return launch_status("tct_interior_pairs");
}

}  // namespace
}  // namespace tct

using namespace tct;

extern "C" int tct_interior_pairs(int kernel, int prec, void* result, int n_q, const void* qp,
                                  const void* qw, const void* obs_pts, const void* obs_ns,
                                  const void* pts, const int32_t* tris, const int32_t* pairs,
                                  int64_t n_pairs, const double* params, int finite_part,
                                  void* stream) {
    TCT_CHECK_ARG(n_pairs >= 0 && n_q >= 0, "tct_interior_pairs: negative size");
    if (n_pairs == 0) return TCT_OK;
    TCT_CHECK_ARG(result && qp && qw && obs_pts && obs_ns && pts && tris && pairs && params,
                  "tct_interior_pairs: null pointer");
    if (prec == TCT_F32)
        return run_interior_pairs<float>(kernel, params, result, n_q, qp, qw, obs_pts, obs_ns,
                                         pts, tris, pairs, n_pairs, finite_part,
                                         as_stream(stream));
    if (prec == TCT_F64)
        return run_interior_pairs<double>(kernel, params, result, n_q, qp, qw, obs_pts, obs_ns,
                                          pts, tris, pairs, n_pairs, finite_part,
                                          as_stream(stream));
    set_error("tct_interior_pairs: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}

extern "C" int tct_interior_corners(int prec, void* result, int n_q, const void* qt,
                                    const void* qw, const void* obs_ns, const void* pts,
                                    const int32_t* tris, const int32_t* pairs, int64_t n_pairs,
                                    const double* params, void* stream) {
    TCT_CHECK_ARG(n_pairs >= 0 && n_q >= 0, "tct_interior_corners: negative size");
    if (n_pairs == 0) return TCT_OK;
    TCT_CHECK_ARG(result && qt && qw && obs_ns && pts && tris && pairs && params,
                  "tct_interior_corners: null pointer");
    const unsigned blocks = (unsigned)((n_pairs + 127) / 128);
    cudaStream_t st = as_stream(stream);
    if (prec == TCT_F32) {
        interior_corners_kernel<float><<<blocks, 128, 0, st>>>(
            make_consts<float>(params), (float*)result, n_q, (const float*)qt,
            (const float*)qw, (const float*)obs_ns, (const float*)pts, tris, pairs, n_pairs);
    } else if (prec == TCT_F64) {
        interior_corners_kernel<double><<<blocks, 128, 0, st>>>(
            make_consts<double>(params), (double*)result, n_q, (const double*)qt,
            (const double*)qw, (const double*)obs_ns, (const double*)pts, tris, pairs, n_pairs);
    } else {
        set_error("tct_interior_corners: unsupported precision %d", prec);
        return TCT_ERR_PREC;
    }
    return launch_status("tct_interior_corners");
}
