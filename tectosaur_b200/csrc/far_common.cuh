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

// ---- packed-FP32 elasticRH3 pair sums (direct farfield and treecode P2P) -----
// Two observation triangles per thread, one in each half of an f32x2 register
// pair, so every point-pair operation is one fma/mul/add.rn.f32x2 instruction
// for both.  Per point pair (both halves): D = y - x, r2e = |D|^2 + EPS,
// invr = rsqrt(r2e) (two MUFU ops), g = invr^3, T += g D D^T; per triangle
// pair S0 = trace(T) (= sum of 1/r, since trace(D D^T) / r^3 = 1/r) and
// W += S0 P + T (-2 ssc).  EPS = 1e-24 keeps invr^3 finite at r2 == 0, where
// D == 0 makes the point pair contribute exactly nothing -- the reference's
// "skip r^2 == 0" (matrix_free.cl:79-81) without a per-pair select.  EPS is
// below the FP32 rounding of any r2 above ~1e-17 (point separations above
// ~3e-9 in mesh units).  J_s * CsRH0 (and, for equal-weight rules, w^2) are
// folded into P and -2 ssc by the prep kernel.
constexpr float RH2_EPS = 1e-24f;

// Record of one source triangle for the packed kernel, every value stored
// twice (an f32x2 operand): y[q][d] (3 NQ pairs), P (9), M = -2 ssc (9).
template <int NQ>
struct RecRH2 {
    static constexpr int Y = 0;
    static constexpr int P = 3 * NQ;
    static constexpr int M = 3 * NQ + 9;
    static constexpr int PAIRS = 3 * NQ + 18;
    static constexpr int LEN = (2 * PAIRS + 3) / 4 * 4;  // floats
};

template <int NQ, bool UNIFORM>
__global__ void __launch_bounds__(128)
far_prep_rh2(Consts<float> c, Rule2D<float> rule, const float* __restrict__ pts,
             const int32_t* __restrict__ src_tris, int64_t n_src, const float* __restrict__ in,
             const int64_t* __restrict__ src_orig, float* __restrict__ rec) {
    using L = RecRH2<NQ>;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_src) return;
    TriGeom<float> s;
    load_tri(s, pts, src_tris, i, 0, false, true);
    const int64_t ii = src_orig ? src_orig[i] : i;  // input row of tree-ordered sources
    float in9[9];
#pragma unroll
    for (int k = 0; k < 9; k++) in9[k] = in[ii * 9 + k];
    float* r = rec + i * L::LEN;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        const float sx = rule.x[q], sy = rule.y[q];
        const float sb[3] = {1 - sx - sy, sx, sy};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const float y = bary_point(s, sb, d);
            r[2 * (L::Y + 3 * q + d)] = y;
            r[2 * (L::Y + 3 * q + d) + 1] = y;
        }
    }
    float ssc[3][3];
#pragma unroll
    for (int Ij = 0; Ij < 3; Ij++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            float a = 0;
#pragma unroll
            for (int b = 0; b < 3; b++) a += s.sc[b][Ij] * in9[b * 3 + d];
            ssc[d][Ij] = a;
        }
    float scale = s.J * c.CsRH0;
    if (UNIFORM) scale *= rule.w[0] * rule.w[0];
    const float B = (ssc[0][0] + ssc[1][1] + ssc[2][2]) * c.CsRH1;
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const float p = scale * ((d == j ? B : 0.f) + c.CsRH2 * ssc[j][d] - 2 * ssc[d][j]);
            const float m = scale * (-2.f * ssc[d][j]);
            r[2 * (L::P + 3 * d + j)] = p;
            r[2 * (L::P + 3 * d + j) + 1] = p;
            r[2 * (L::M + 3 * d + j)] = m;
            r[2 * (L::M + 3 * d + j) + 1] = m;
        }
#pragma unroll
    for (int k = 2 * L::PAIRS; k < L::LEN; k++) r[k] = 0;
}

// One packed source record r against this thread's two observation
// triangles (negated target points negx, pair weights wq for unequal-weight
// rules): W[3 d + j] += S0 P[d][j] + sum_k T[d][k] M[k][j], both halves.
template <int NQ, bool UNIFORM, bool VEC = false>
__device__ __forceinline__ void rh2_pair(const f2_t* __restrict__ r, const f2_t (&negx)[NQ][3],
                                         const f2_t (&wq)[UNIFORM ? 1 : NQ * NQ], f2_t eps,
                                         f2_t (&W)[9]) {
    using L = RecRH2<NQ>;
    // VEC: the record (16-byte aligned: LEN is a multiple of 4 floats) is read
    // with 16-byte loads, two packed values each -- the points before the
    // pair loop, P and M after it: half the shared-memory load instructions,
    // for ~30 more registers (the direct farfield kernel with the 3-point
    // rule, which has them: 5.6 % faster at 60k triangles; the FMM P2P keeps
    // its 128-register cap)
    constexpr int NYV = (3 * NQ + 1) / 2;
    f2_t yv[VEC ? 2 * NYV : 1];
    if constexpr (VEC) {
        const ulonglong2* r2 = reinterpret_cast<const ulonglong2*>(r);
#pragma unroll
        for (int k = 0; k < NYV; k++) {
            const ulonglong2 u = r2[k];
            yv[2 * k] = u.x;
            yv[2 * k + 1] = u.y;
        }
    }
    f2_t T00 = 0ull, T01 = 0ull, T02 = 0ull, T11 = 0ull, T12 = 0ull, T22 = 0ull;
#pragma unroll
    for (int q2 = 0; q2 < NQ; q2++) {
        f2_t y0, y1, y2;
        if constexpr (VEC) {
            y0 = yv[L::Y + 3 * q2 + 0];
            y1 = yv[L::Y + 3 * q2 + 1];
            y2 = yv[L::Y + 3 * q2 + 2];
        } else {
            y0 = r[L::Y + 3 * q2 + 0];
            y1 = r[L::Y + 3 * q2 + 1];
            y2 = r[L::Y + 3 * q2 + 2];
        }
#pragma unroll
        for (int q1 = 0; q1 < NQ; q1++) {
            const f2_t D0 = add2(y0, negx[q1][0]);
            const f2_t D1 = add2(y1, negx[q1][1]);
            const f2_t D2 = add2(y2, negx[q1][2]);
            f2_t r2 = fma2(D0, D0, eps);
            r2 = fma2(D1, D1, r2);
            r2 = fma2(D2, D2, r2);
            float ra, rb;
            upk(r2, ra, rb);
            const f2_t invr = pk(rsqrtf(ra), rsqrtf(rb));
            f2_t g = mul2(mul2(invr, invr), invr);
            if (!UNIFORM) g = mul2(g, wq[q1 * NQ + q2]);
            const f2_t g0 = mul2(g, D0), g1 = mul2(g, D1), g2 = mul2(g, D2);
            T00 = fma2(g0, D0, T00);
            T01 = fma2(g0, D1, T01);
            T02 = fma2(g0, D2, T02);
            T11 = fma2(g1, D1, T11);
            T12 = fma2(g1, D2, T12);
            T22 = fma2(g2, D2, T22);
        }
    }
    const f2_t S0 = add2(add2(T00, T11), T22);
    const f2_t T[3][3] = {{T00, T01, T02}, {T01, T11, T12}, {T02, T12, T22}};
    // P[k] at packed index P + k, M[k] at M + k = P + 9 + k
    constexpr int K0 = L::P / 2, K1 = (L::PAIRS + 1) / 2, OFF = L::P % 2;
    f2_t pm[VEC ? 2 * (K1 - K0) : 1];
    if constexpr (VEC) {
        const ulonglong2* r2 = reinterpret_cast<const ulonglong2*>(r);
#pragma unroll
        for (int k = K0; k < K1; k++) {
            const ulonglong2 u = r2[k];
            pm[2 * (k - K0)] = u.x;
            pm[2 * (k - K0) + 1] = u.y;
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
            f2_t p, m0, m1, m2;
            if constexpr (VEC) {
                p = pm[OFF + 3 * d + jj];
                m0 = pm[OFF + 9 + 0 * 3 + jj];
                m1 = pm[OFF + 9 + 1 * 3 + jj];
                m2 = pm[OFF + 9 + 2 * 3 + jj];
            } else {
                p = r[L::P + 3 * d + jj];
                m0 = r[L::M + 0 * 3 + jj];
                m1 = r[L::M + 1 * 3 + jj];
                m2 = r[L::M + 2 * 3 + jj];
            }
            f2_t w = fma2(S0, p, W[3 * d + jj]);
            w = fma2(T[d][0], m0, w);
            w = fma2(T[d][1], m1, w);
            w = fma2(T[d][2], m2, w);
            W[3 * d + jj] = w;
        }
}

}  // namespace
}  // namespace tct
