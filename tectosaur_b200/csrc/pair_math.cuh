// Pair-integration math shared by the pair-quadrature kernel (pairs.cu) and
// the dense farfield-block kernel (farfield.cu).
//
// integrate_pair restates integrate_pair of tectosaur/integral_primitives.cl:174-213
// with the tensor forms of tectosaur/kernels/__init__.py (U :37-50, T/A :101-125,
// H :174-214) and tectosaur/kernels/kernels.cl:29-98 (RT/RA/RH).
#pragma once
#include "common.cuh"

namespace tct {

// Tensor form for U/T/A/H: Karr[d_obs*3 + d_src] (kernels/__init__.py:37-50,
// 101-125, 174-214).
template <typename R, int K>
__device__ __forceinline__ void karr_utah(const Consts<R>& c, const R D[3], R r2,
                                          const R no[3], const R ns[3], R Karr[9]) {
    const R Dx = D[0], Dy = D[1], Dz = D[2];
    if (K == kU) {
        R invr = rsqrt_r(r2);
        R Q1 = c.CsU0 * invr;
        R Q2 = c.CsU1 * invr / r2;
        Karr[0] = Q2 * Dx * Dx + Q1;
        Karr[1] = Q2 * Dx * Dy;
        Karr[2] = Q2 * Dx * Dz;
        Karr[3] = Q2 * Dy * Dx;
        Karr[4] = Q2 * Dy * Dy + Q1;
        Karr[5] = Q2 * Dy * Dz;
        Karr[6] = Q2 * Dz * Dx;
        Karr[7] = Q2 * Dz * Dy;
        Karr[8] = Q2 * Dz * Dz + Q1;
    } else if (K == kT || K == kA) {
        const R mp = (K == kT) ? R(-1) : R(1);
        const R pm = (K == kT) ? R(1) : R(-1);
        const R* n = (K == kT) ? ns : no;
        R invr = rsqrt_r(r2);
        R invr2 = invr * invr;
        R invr3 = invr2 * invr;
        R rn = n[0] * Dx + n[1] * Dy + n[2] * Dz;
        R A = pm * c.CsT0 * invr3;
        R C = mp * c.CsT1 * invr3 * invr2;
        R nxdy = n[0] * Dy - n[1] * Dx;
        R nzdx = n[2] * Dx - n[0] * Dz;
        R nzdy = n[2] * Dy - n[1] * Dz;
        Karr[0] = A * -rn + C * Dx * rn * Dx;
        Karr[1] = A * (mp * nxdy) + C * Dx * rn * Dy;
        Karr[2] = A * (pm * nzdx) + C * Dx * rn * Dz;
        Karr[3] = A * (pm * nxdy) + C * Dy * rn * Dx;
        Karr[4] = A * -rn + C * Dy * rn * Dy;
        Karr[5] = A * (pm * nzdy) + C * Dy * rn * Dz;
        Karr[6] = A * (mp * nzdx) + C * Dz * rn * Dx;
        Karr[7] = A * (mp * nzdy) + C * Dz * rn * Dy;
        Karr[8] = A * -rn + C * Dz * rn * Dz;
    } else {
        R invr = rsqrt_r(r2);
        R invr2 = invr * invr;
        R invr3 = invr2 * invr;
        R Dor[3] = {invr * Dx, invr * Dy, invr * Dz};
        R rn = ns[0] * Dor[0] + ns[1] * Dor[1] + ns[2] * Dor[2];
        R rm = no[0] * Dor[0] + no[1] * Dor[1] + no[2] * Dor[2];
        R mn = no[0] * ns[0] + no[1] * ns[1] + no[2] * ns[2];
        R Q = c.CsH0 * invr3;
        R A = Q * 3 * rn;
        R B = Q * c.CsH1;
        R C = Q * c.CsH3;
        R MT[3], NT[3], DT[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            MT[d] = Q * c.CsH2 * ns[d] + A * c.CsH1 * Dor[d];
            NT[d] = B * no[d] + C * Dor[d] * rm;
            DT[d] = B * 3 * ns[d] * rm + C * Dor[d] * mn + A * (c.nu * no[d] - 5 * Dor[d] * rm);
        }
        R ST = A * c.nu * rm + B * mn;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                Karr[i * 3 + j] = ns[i] * NT[j] + no[i] * MT[j] + Dor[i] * DT[j] + (i == j ? ST : R(0));
    }
}

template <typename R, int K>
__device__ __forceinline__ R gimk(int p, int m, int j, R Q1, R Q2, const R D[3]) {
    R A = Q1 * (R)levi(m, p, j);
    R B = 0;
#pragma unroll
    for (int It = 0; It < 3; It++) B += (R)levi(m, It, j) * D[It];
    return A + Q2 * D[p] * B;
}

// Per-pair accumulator of the tensor-form integrand.
//
// U/T/A/H and RT/RA keep the 81 outputs per point (U/T/A/H Kahan-compensated
// in FP32, as the reference).  RH is separable: its tensor form
// (kernels/kernels.cl:70-98) multiplies the constant surface curls of the two
// triangles, so
//   sum_q K_q[dob][ds][It][Im] osc[bo][It] ssc[bs][Im]
//     = A (CsRH1 osc[bo][dob] ssc[bs][ds] + CsRH2 osc[bo][ds] ssc[bs][dob]
//          - 2 delta(dob, ds) G[bo][bs]) - 2 S[dob][ds] G[bo][bs]
// with A = sum_q w CsRH0 / r, S = sum_q w CsRH0 D D^T / r^3 and
// G[bo][bs] = osc[bo] . ssc[bs]: seven running sums instead of 81.
template <typename R, int K, bool KAHAN>
struct PairAcc {
    static constexpr int N = (K == kRH) ? 7 : 81;
    R v[N];
    R kc[(KAHAN && K != kRH) ? 81 : 1];

    __device__ __forceinline__ void init() {
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = 0;
        if (KAHAN && K != kRH) {
#pragma unroll
            for (int i = 0; i < 81; i++) kc[i] = 0;
        }
    }

    __device__ __forceinline__ void add(const Consts<R>& c, const TriGeom<R>& o,
                                        const TriGeom<R>& s, R ox, R oy, R sx, R sy, R w,
                                        bool check0) {
        R ob[3] = {1 - ox - oy, ox, oy};
        R sb[3] = {1 - sx - sy, sx, sy};
        R D[3];
#pragma unroll
        for (int d = 0; d < 3; d++) D[d] = bary_point(s, sb, d) - bary_point(o, ob, d);
        R r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
        if (check0 && r2 == R(0)) return;
        if (K <= kH) {
            R Karr[9];
            karr_utah<R, K>(c, D, r2, o.n, s.n, Karr);
#pragma unroll
            for (int d = 0; d < 3; d++) ob[d] *= w;
#pragma unroll
            for (int bo = 0; bo < 3; bo++)
#pragma unroll
                for (int dob = 0; dob < 3; dob++)
#pragma unroll
                    for (int bs = 0; bs < 3; bs++)
#pragma unroll
                        for (int ds = 0; ds < 3; ds++) {
                            const int idx = bo * 27 + dob * 9 + bs * 3 + ds;
                            R val = ob[bo] * sb[bs] * Karr[dob * 3 + ds];
                            if (KAHAN) {
                                R yk = val - kc[idx];
                                R t = v[idx] + yk;
                                kc[idx] = (t - v[idx]) - yk;
                                v[idx] = t;
                            } else {
                                v[idx] += val;
                            }
                        }
        } else if (K == kRT || K == kRA) {
            // elasticRTA3_setup / elasticRTA3_tensor (kernels/kernels.cl:11-68)
            constexpr bool RT = (K == kRT);
            const R* nn = RT ? s.n : o.n;
            R invr = rsqrt_r(r2);
            R invr3 = invr * invr * invr;
            R Q1 = c.CsRT1 * invr;
            R Q2 = c.CsRT0 * invr3;
            R Q3 = c.CsRT2 * invr3;
            R Q3nD = Q3 * (nn[0] * D[0] + nn[1] * D[1] + nn[2] * D[2]);
#pragma unroll
            for (int dob = 0; dob < 3; dob++)
#pragma unroll
                for (int ds = 0; ds < 3; ds++) {
                    const int Ld = RT ? dob : ds;
                    const int Rd = RT ? ds : dob;
#pragma unroll
                    for (int bR = 0; bR < 3; bR++) {
                        R Kval = 0;
#pragma unroll
                        for (int Ij = 0; Ij < 3; Ij++) {
                            R g = gimk<R, K>(Ld, Ij, Rd, Q1, Q2, D);
                            Kval += g * (RT ? s.sc[bR][Ij] : o.sc[bR][Ij]);
                        }
                        if (dob == ds) Kval += Q3nD * (RT ? sb[bR] : ob[bR]) * (RT ? R(1) : R(-1));
#pragma unroll
                        for (int bL = 0; bL < 3; bL++) {
                            R val = w * (RT ? ob[bL] : sb[bL]) * Kval;
                            const int b_obs = RT ? bL : bR;
                            const int b_src = RT ? bR : bL;
                            v[b_obs * 27 + dob * 9 + b_src * 3 + ds] += val;
                        }
                    }
                }
        } else {
            const R invr = rsqrt_r(r2);
            const R a = w * c.CsRH0 * invr;
            const R b = a * (invr * invr);
            v[0] += a;
            const R b0 = b * D[0], b1 = b * D[1], b2 = b * D[2];
            v[1] += b0 * D[0];
            v[2] += b0 * D[1];
            v[3] += b0 * D[2];
            v[4] += b1 * D[1];
            v[5] += b1 * D[2];
            v[6] += b2 * D[2];
        }
    }

    // Sum the accumulators of a warp's 32 lanes (every lane gets the total).
    __device__ __forceinline__ void warp_reduce() {
        if (KAHAN && K != kRH) {
#pragma unroll
            for (int i = 0; i < 81; i++) v[i] -= kc[i];
        }
#pragma unroll
        for (int i = 0; i < N; i++) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], off);
        }
    }

    // The 81 outputs b_obs*27 + d_obs*9 + b_src*3 + d_src (before J_o J_s).
    __device__ __forceinline__ void finish(const Consts<R>& c, const TriGeom<R>& o,
                                           const TriGeom<R>& s, R res[81]) const {
        if (K != kRH) {
#pragma unroll
            for (int i = 0; i < 81; i++) res[i] = v[i];
            return;
        }
        const R A = v[0];
        const R S[3][3] = {{v[1], v[2], v[3]}, {v[2], v[4], v[5]}, {v[3], v[5], v[6]}};
#pragma unroll
        for (int bo = 0; bo < 3; bo++)
#pragma unroll
            for (int bs = 0; bs < 3; bs++) {
                const R G = o.sc[bo][0] * s.sc[bs][0] + o.sc[bo][1] * s.sc[bs][1] +
                            o.sc[bo][2] * s.sc[bs][2];
#pragma unroll
                for (int dob = 0; dob < 3; dob++)
#pragma unroll
                    for (int ds = 0; ds < 3; ds++)
                        res[bo * 27 + dob * 9 + bs * 3 + ds] =
                            A * (c.CsRH1 * o.sc[bo][dob] * s.sc[bs][ds] +
                                 c.CsRH2 * o.sc[bo][ds] * s.sc[bs][dob] -
                                 (dob == ds ? 2 * G : R(0))) -
                            2 * S[dob][ds] * G;
            }
    }
};

template <typename R, int K, bool KAHAN>
__device__ void integrate_pair(const Consts<R>& c, const TriGeom<R>& o, const TriGeom<R>& s,
                               int n_q, const R* __restrict__ qp, const R* __restrict__ qw,
                               bool check0, R res[81]) {
    PairAcc<R, K, KAHAN> acc;
    acc.init();
    for (int iq = 0; iq < n_q; iq++) {
        acc.add(c, o, s, __ldg(qp + 4 * iq + 0), __ldg(qp + 4 * iq + 1), __ldg(qp + 4 * iq + 2),
                __ldg(qp + 4 * iq + 3), __ldg(qw + iq), check0);
    }
    acc.finish(c, o, s, res);
}

}  // namespace tct
