// Shared pieces of the direct tri-to-tri farfield (farfield.cu) and the
// treecode's P2P (fmm.cu): the 2-D rule, the per-source-triangle record and
// its prep kernel, the per-kernel vector forms, the per-record pair sums and
// the obs-side epilogue (tectosaur/matrix_free.cl:19-107,
// kernels/kernels.cl:100-206).
#pragma once

#include "pair_math.cuh"

namespace tct {
namespace {

constexpr int MAXQ = 13;

// Packed FP32 pairs (add/mul/fma.rn.f32x2: two lanes of work per instruction).
typedef unsigned long long f2_t;

__device__ __forceinline__ f2_t pk(float x, float y) {
    f2_t d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(x), "f"(y));
    return d;
}
__device__ __forceinline__ void upk(f2_t d, float& x, float& y) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(d));
}
__device__ __forceinline__ f2_t add2(f2_t a, f2_t b) {
    f2_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2_t mul2(f2_t a, f2_t b) {
    f2_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2_t fma2(f2_t a, f2_t b, f2_t c) {
    f2_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}


template <typename R>
struct Rule2D {
    R x[MAXQ], y[MAXQ], w[MAXQ];
};

// Record layout per source triangle (units of Real).
template <int K, int NQ>
struct Rec {
    static constexpr int Y = 0;               // y[NQ][3]
    static constexpr int SW = 3 * NQ;         // J_s * w_j (RH: times CsRH0)
    static constexpr int N = 4 * NQ;          // source normal (T, H, RT)
    static constexpr int C = 4 * NQ + 3;      // RT: curl c[3] of the input
    static constexpr int INV = (K == kT || K == kH) ? 4 * NQ + 3
                             : (K == kRT)          ? 4 * NQ + 6
                                                   : 4 * NQ;  // interpolated input [NQ][3]
    static constexpr int SSC = 4 * NQ;        // RH: -2 * ssc[3][3]
    static constexpr int P = 4 * NQ + 9;      // RH: P[3][3]
    static constexpr int RAW = (K == kRH) ? 4 * NQ + 18 : INV + 3 * NQ;
    static constexpr int LEN = (RAW + 3) / 4 * 4;
};

template <int K, int NQ>
struct NAcc {
    static constexpr int n = (K == kRH) ? 9 : (K == kRA ? 3 * NQ + 3 : 3 * NQ);
};

template <typename R, int K, int NQ>
__global__ void __launch_bounds__(128)
far_prep(Consts<R> c, Rule2D<R> rule, const R* __restrict__ pts,
         const int32_t* __restrict__ src_tris, int64_t n_src, const R* __restrict__ in,
         const int64_t* __restrict__ src_orig, R* __restrict__ rec) {
    using L = Rec<K, NQ>;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_src) return;
    TriGeom<R> s;
    load_tri(s, pts, src_tris, i, 0, false, K == kRT || K == kRH);
    const int64_t ii = src_orig ? src_orig[i] : i;
    R in9[9];
#pragma unroll
    for (int k = 0; k < 9; k++) in9[k] = in[ii * 9 + k];
    R* r = rec + i * L::LEN;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        const R sx = rule.x[q], sy = rule.y[q];
        const R sb[3] = {1 - sx - sy, sx, sy};
#pragma unroll
        for (int d = 0; d < 3; d++) r[L::Y + 3 * q + d] = bary_point(s, sb, d);
        R sw = s.J * rule.w[q];
        if (K == kRH) sw = sw * c.CsRH0;
        r[L::SW + q] = sw;
        if (K != kRH) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                R a = 0;
                a += in9[0 * 3 + d] * sb[0];
                a += in9[1 * 3 + d] * sb[1];
                a += in9[2 * 3 + d] * sb[2];
                r[L::INV + 3 * q + d] = a;
            }
        }
    }
    if (K == kT || K == kH || K == kRT) {
#pragma unroll
        for (int d = 0; d < 3; d++) r[L::N + d] = s.n[d];
    }
    if (K == kRT || K == kRH) {
        // src_surf_curl[d][Ij] = sum_b bsrc_surf_curl[b][Ij] * in[b*3 + d]
        R ssc[3][3];
#pragma unroll
        for (int Ij = 0; Ij < 3; Ij++)
#pragma unroll
            for (int d = 0; d < 3; d++) {
                R a = 0;
#pragma unroll
                for (int b = 0; b < 3; b++) a += s.sc[b][Ij] * in9[b * 3 + d];
                ssc[d][Ij] = a;
            }
        if (K == kRT) {
            // c[p] = sum_{m,j} e[m][p][j] ssc[j][m]
#pragma unroll
            for (int p = 0; p < 3; p++) {
                R a = 0;
#pragma unroll
                for (int m = 0; m < 3; m++)
#pragma unroll
                    for (int j = 0; j < 3; j++)
                        if (levi(m, p, j) != 0) a += (R)levi(m, p, j) * ssc[j][m];
                r[L::C + p] = a;
            }
        } else {
            R B = (ssc[0][0] + ssc[1][1] + ssc[2][2]) * c.CsRH1;
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    r[L::SSC + 3 * d + j] = R(-2) * ssc[d][j];
                    r[L::P + 3 * d + j] = (d == j ? B : R(0)) + c.CsRH2 * ssc[j][d] - 2 * ssc[d][j];
                }
        }
    }
#pragma unroll
    for (int k = L::RAW; k < L::LEN; k++) r[k] = 0;
}

// Vector forms of U/T/A/H at one point pair (kernels/__init__.py:28-36, 67-99,
// 147-173): returns the 3-vector the reference adds to sum{x,y,z}.
template <typename R, int K>
__device__ __forceinline__ void vec_utah(const Consts<R>& c, const R D[3], R r2, const R no[3],
                                         const R ns[3], const R a[3], R v[3]) {
    if (K == kU) {
        R invr = rsqrt_r(r2);
        R Q1 = c.CsU0 * invr;
        R Q2 = c.CsU1 * invr / r2;
        R ddi = D[0] * a[0] + D[1] * a[1] + D[2] * a[2];
#pragma unroll
        for (int d = 0; d < 3; d++) v[d] = Q1 * a[d] + Q2 * D[d] * ddi;
    } else if (K == kT || K == kA) {
        const R mp = (K == kT) ? R(-1) : R(1);
        const R pm = (K == kT) ? R(1) : R(-1);
        const R* n = (K == kT) ? ns : no;
        R invr = rsqrt_r(r2);
        R invr2 = invr * invr;
        R invr3 = invr2 * invr;
        R rn = n[0] * D[0] + n[1] * D[1] + n[2] * D[2];
        R A = pm * c.CsT0 * invr3;
        R C = mp * c.CsT1 * invr3 * invr2;
        R rnddi = C * rn * (D[0] * a[0] + D[1] * a[1] + D[2] * a[2]);
        R nxdy = n[0] * D[1] - n[1] * D[0];
        R nzdx = n[2] * D[0] - n[0] * D[2];
        R nzdy = n[2] * D[1] - n[1] * D[2];
        v[0] = A * (-rn * a[0] + mp * nxdy * a[1] + pm * nzdx * a[2]) + D[0] * rnddi;
        v[1] = A * (pm * nxdy * a[0] - rn * a[1] + pm * nzdy * a[2]) + D[1] * rnddi;
        v[2] = A * (mp * nzdx * a[0] + mp * nzdy * a[1] - rn * a[2]) + D[2] * rnddi;
    } else {
        R invr = rsqrt_r(r2);
        R invr2 = invr * invr;
        R invr3 = invr2 * invr;
        R rn = invr * (ns[0] * D[0] + ns[1] * D[1] + ns[2] * D[2]);
        R rm = invr * (no[0] * D[0] + no[1] * D[1] + no[2] * D[2]);
        R mn = no[0] * ns[0] + no[1] * ns[1] + no[2] * ns[2];
        R sn = a[0] * ns[0] + a[1] * ns[1] + a[2] * ns[2];
        R sd = invr * (a[0] * D[0] + a[1] * D[1] + a[2] * D[2]);
        R sm = a[0] * no[0] + a[1] * no[1] + a[2] * no[2];
        R Q = c.CsH0 * invr3;
        R A = Q * 3 * rn;
        R B = Q * c.CsH1;
        R C = Q * c.CsH3;
        R MT = Q * c.CsH2 * sn + A * c.CsH1 * sd;
        R NT = B * sm + C * sd * rm;
        R DT = invr * (B * 3 * sn * rm + C * sd * mn + A * (c.nu * sm - 5 * sd * rm));
        R ST = A * c.nu * rm + B * mn;
#pragma unroll
        for (int d = 0; d < 3; d++) v[d] = ns[d] * NT + no[d] * MT + D[d] * DT + ST * a[d];
    }
}

template <typename R, bool KAHAN>
__device__ __forceinline__ void fold(R& tot, R& cmp, R tile) {
    if (KAHAN) {
        R y = tile - cmp;
        R t = tot + y;
        cmp = (t - tot) - y;
        tot = t;
    } else {
        tot += tile;
    }
}

// One source record against one obs triangle: adds the kernel's sums over the
// NQ x NQ point pairs to acc (the layout of NAcc).  Shared by the direct
// matvec and the treecode's P2P.
template <typename R, int K, int NQ>
__device__ __forceinline__ void far_pair(const Consts<R>& c, const Rule2D<R>& rule,
                                         const TriGeom<R>& o, const R (&x)[NQ][3],
                                         const R* __restrict__ r, R (&acc)[NAcc<K, NQ>::n]) {
    using L = Rec<K, NQ>;
    if (K == kRH) {
        R S0 = 0, T00 = 0, T01 = 0, T02 = 0, T11 = 0, T12 = 0, T22 = 0;
#pragma unroll
        for (int q1 = 0; q1 < NQ; q1++)
#pragma unroll
            for (int q2 = 0; q2 < NQ; q2++) {
                R D0 = r[L::Y + 3 * q2 + 0] - x[q1][0];
                R D1 = r[L::Y + 3 * q2 + 1] - x[q1][1];
                R D2 = r[L::Y + 3 * q2 + 2] - x[q1][2];
                R r2 = D0 * D0 + D1 * D1 + D2 * D2;
                R invr = (r2 != R(0)) ? rsqrt_r(r2) : R(0);
                R f = (rule.w[q1] * r[L::SW + q2]) * invr;
                R g = f * (invr * invr);
                S0 += f;
                R g0 = g * D0, g1 = g * D1, g2 = g * D2;
                T00 += g0 * D0;
                T01 += g0 * D1;
                T02 += g0 * D2;
                T11 += g1 * D1;
                T12 += g1 * D2;
                T22 += g2 * D2;
            }
        const R T[3][3] = {{T00, T01, T02}, {T01, T11, T12}, {T02, T12, T22}};
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int jj = 0; jj < 3; jj++) {
                R w = S0 * r[L::P + 3 * d + jj];
                w += T[d][0] * r[L::SSC + 0 * 3 + jj];
                w += T[d][1] * r[L::SSC + 1 * 3 + jj];
                w += T[d][2] * r[L::SSC + 2 * 3 + jj];
                acc[3 * d + jj] += w;
            }
    } else {
#pragma unroll
        for (int q1 = 0; q1 < NQ; q1++)
#pragma unroll
            for (int q2 = 0; q2 < NQ; q2++) {
                R D[3];
                D[0] = r[L::Y + 3 * q2 + 0] - x[q1][0];
                D[1] = r[L::Y + 3 * q2 + 1] - x[q1][1];
                D[2] = r[L::Y + 3 * q2 + 2] - x[q1][2];
                R r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
                if (r2 == R(0)) continue;
                const R sw = r[L::SW + q2];
                const R a[3] = {r[L::INV + 3 * q2 + 0], r[L::INV + 3 * q2 + 1],
                                r[L::INV + 3 * q2 + 2]};
                if (K <= kH) {
                    R ns[3] = {0, 0, 0};
                    if (K == kT || K == kH) {
                        ns[0] = r[L::N + 0];
                        ns[1] = r[L::N + 1];
                        ns[2] = r[L::N + 2];
                    }
                    R v[3];
                    vec_utah<R, K>(c, D, r2, o.n, ns, a, v);
#pragma unroll
                    for (int d = 0; d < 3; d++) acc[3 * q1 + d] += sw * v[d];
                } else if (K == kRT) {
                    // sum_d = Q1 c_d + Q2 D_d (D.c) + Q3 (n_s.D) a_d
                    R invr = rsqrt_r(r2);
                    R invr3 = invr * invr * invr;
                    R Q1 = c.CsRT1 * invr, Q2 = c.CsRT0 * invr3, Q3 = c.CsRT2 * invr3;
                    const R cc[3] = {r[L::C + 0], r[L::C + 1], r[L::C + 2]};
                    R Dc = D[0] * cc[0] + D[1] * cc[1] + D[2] * cc[2];
                    R nD = r[L::N + 0] * D[0] + r[L::N + 1] * D[1] + r[L::N + 2] * D[2];
                    R Q3nD = Q3 * nD;
#pragma unroll
                    for (int d = 0; d < 3; d++)
                        acc[3 * q1 + d] += sw * (Q1 * cc[d] + Q2 * D[d] * Dc + Q3nD * a[d]);
                } else {  // kRA
                    // U_k += w1 sw (Q1 a_k + Q2 (D.a) D_k);
                    // acc[q1] += sw * (-Q3 (n_o.D)) a
                    R invr = rsqrt_r(r2);
                    R invr3 = invr * invr * invr;
                    R Q1 = c.CsRT1 * invr, Q2 = c.CsRT0 * invr3, Q3 = c.CsRT2 * invr3;
                    R Da = D[0] * a[0] + D[1] * a[1] + D[2] * a[2];
                    R nD = o.n[0] * D[0] + o.n[1] * D[1] + o.n[2] * D[2];
                    R ww = rule.w[q1] * sw;
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        acc[3 * NQ + d] += ww * (Q1 * a[d] + Q2 * Da * D[d]);
                        acc[3 * q1 + d] -= sw * (Q3 * nD * a[d]);
                    }
                }
            }
    }
}

// Obs-side contraction of the accumulated sums into the 9 outputs out[b][d]
// (basis b of the obs triangle, component d), times J_o.
template <typename R, int K, int NQ>
__device__ __forceinline__ void far_epilogue(const Rule2D<R>& rule, const TriGeom<R>& o,
                                             const R (&tot)[NAcc<K, NQ>::n], R (&out9)[9]) {
    if (K == kRH) {
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int d = 0; d < 3; d++)
                out9[b * 3 + d] = o.J * (o.sc[b][0] * tot[3 * d + 0] + o.sc[b][1] * tot[3 * d + 1] +
                                         o.sc[b][2] * tot[3 * d + 2]);
    } else {
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int d = 0; d < 3; d++) {
                R s = 0;
#pragma unroll
                for (int q = 0; q < NQ; q++) {
                    const R ox = rule.x[q], oy = rule.y[q];
                    const R ob = (b == 0) ? (1 - ox - oy) : (b == 1 ? ox : oy);
                    s += (rule.w[q] * ob) * tot[3 * q + d];
                }
                if (K == kRA) {
                    // + sum_Ij sc_o[b][Ij] V[Ij][d],  V[m][j] = -sum_k e[m][j][k] U_k
#pragma unroll
                    for (int m = 0; m < 3; m++)
#pragma unroll
                        for (int k = 0; k < 3; k++)
                            if (levi(m, d, k) != 0)
                                s -= (R)levi(m, d, k) * o.sc[b][m] * tot[3 * NQ + k];
                }
                out9[b * 3 + d] = o.J * s;
            }
    }
}

}  // namespace
}  // namespace tct
