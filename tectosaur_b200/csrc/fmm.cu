// Treecode farfield (P2P, P2M, M2M, M2P) for elasticU3, elasticRT3,
// elasticRA3 and elasticRH3 -- the kernels the reference's treecode supports
// (fmm/tsfmm.py, fmm/ts_kernels.cl:428-1003).
//
// Formulation.  In the hoisted vector form every supported kernel sends,
// from a source quadrature point y to a target point x (D = y - x, r = |D|),
//   F[d][j] = c[d][j] / r + sum_k D_d D_k m[k][j] / r^3 + sum_k v[d][k] D_k / r^3
// where c, m, v are per-point "charges" (J = 3 output columns for RH, 1 for U
// and RT; v only for RT).  Since D_k / r^3 = d/dx_k (1/r) and
// D_d = Y_d - X_d with Y = y - C, X = x - C about an expansion centre C:
//   F[d][j] = Phi[c_dj] + Phi_dip[Y_d m_.j] - X_d Phi_dip[m_.j] + Phi_dip[v_d.]
// -- Laplace potentials of monopoles and dipoles only (7, 10 and 21 channels
// for U, RT and RH, the reference's multipole_dim counts).
// Cartesian multipoles about C: N_a = sum q Y^a (monopole), and for a dipole
// v at Y: N_g += -sum_k g_k v_k Y^(g - e_k); the far potential is
//   Phi(x) = sum_{|a| <= p} (-1)^|a| N_a D_a(X),  D_a = (1/a!) d^a (1/|X|),
// with D from the recurrence
//   n |X|^2 D_g = -(2n - 1) sum_i X_i D_(g - e_i) - (n - 1) sum_i D_(g - 2e_i).
// M2M shifts monomials: N^P_a = sum_{b <= a} C(a, b) N^C_b (C_C - C_P)^(a - b);
// the centre-dependent channels Y_d m shift by (C_C - C_P)_d times the m channel.
//
// Multi-indices a = (a0, a1, a2), |a| = n <= p, are stored graded:
// idx(a) = n(n+1)(n+2)/6 + (n - a0)(n - a0 + 1)/2 + a2.
#include <algorithm>

#include "common.cuh"

namespace tct {
namespace {

constexpr int FMM_MAXP = 12;
constexpr int FMM_MAXN = (FMM_MAXP + 1) * (FMM_MAXP + 2) * (FMM_MAXP + 3) / 6;  // 455

__host__ __device__ constexpr int n_terms(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }
__device__ __forceinline__ int midx(int a0, int a1, int a2) {
    const int n = a0 + a1 + a2;
    return n * (n + 1) * (n + 2) / 6 + (n - a0) * (n - a0 + 1) / 2 + a2;
}

// Per-kernel channel layout.
//   U, RT, RH: F[d][j] as above (NOU = 3J outputs per target point).
//   RA: F = (Fu[3], Fv[3]): Fu is a U-type field (constants CsRT1, CsRT0) that
//   the finish kernel contracts with the obs surface curl; Fv[d] =
//   -sum_k n_o[k] D_k / r^3 a'_d, a dipole field per (d, k) channel (9 channels
//   of vector a'_d e_k) contracted with the obs normal at the target.
template <int K>
struct Chan {
    static constexpr int J = (K == kRH) ? 3 : 1;
    static constexpr int NOU = 3 * J;
    static constexpr int NO = NOU + (K == kRA ? 3 : 0);  // F entries per target point
    static constexpr bool HAS_V = (K == kRT);
    static constexpr bool HAS_A = (K == kRA);
    // point record: y(3), c(NOU), m(3J: m[k][j] at 3 + NOU + k*J + j),
    // then v(9) for RT or a'(3) for RA
    static constexpr int XT = 3 + NOU + 3 * J;
    static constexpr int REC = XT + (HAS_V ? 9 : 0) + (HAS_A ? 3 : 0);
    static constexpr int NV = HAS_V ? 3 : (HAS_A ? 9 : 0);
    // multipole channels: mono (NOU), Ydip (NOU), Mdip (J), V/A dipoles (NV)
    static constexpr int NCH = 2 * NOU + J + NV;
    static constexpr int CH_MONO = 0, CH_Y = NOU, CH_M = 2 * NOU, CH_V = 2 * NOU + J;
};

// ---- point charges ---------------------------------------------------------
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_charges(Consts<R> c, int nq, const R* __restrict__ qx, const R* __restrict__ qw,
            const R* __restrict__ pts, const int32_t* __restrict__ src_tris, int64_t n_src,
            const int64_t* __restrict__ src_orig, const R* __restrict__ in,
            R* __restrict__ rec) {
    using C = Chan<K>;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_src) return;
    TriGeom<R> s;
    load_tri(s, pts, src_tris, i, 0, false, K == kRT || K == kRH);
    R in9[9];
#pragma unroll
    for (int k = 0; k < 9; k++) in9[k] = in[src_orig[i] * 9 + k];
    R ssc[3][3];  // ssc[d][Ij] = sum_b sc[b][Ij] in[b*3 + d]
#pragma unroll
    for (int Ij = 0; Ij < 3; Ij++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            R a = 0;
#pragma unroll
            for (int b = 0; b < 3; b++) a += s.sc[b][Ij] * in9[b * 3 + d];
            ssc[d][Ij] = (K == kRT || K == kRH) ? a : R(0);
        }
    for (int q = 0; q < nq; q++) {
        const R sx = qx[2 * q], sy = qx[2 * q + 1];
        const R sb[3] = {1 - sx - sy, sx, sy};
        R* r = rec + ((int64_t)i * nq + q) * C::REC;
#pragma unroll
        for (int d = 0; d < 3; d++) r[d] = bary_point(s, sb, d);
        const R sw = s.J * qw[q];
        R a[3];
#pragma unroll
        for (int d = 0; d < 3; d++) a[d] = in9[d] * sb[0] + in9[3 + d] * sb[1] + in9[6 + d] * sb[2];
        if (K == kU) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                r[3 + d] = sw * c.CsU0 * a[d];
                r[3 + C::NOU + d] = sw * c.CsU1 * a[d];
            }
        } else if (K == kRA) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                r[3 + d] = sw * c.CsRT1 * a[d];
                r[3 + C::NOU + d] = sw * c.CsRT0 * a[d];
                r[C::XT + d] = sw * c.CsRT2 * a[d];
            }
        } else if (K == kRT) {
            // curl vector cc[p] = sum_{m,j} e[m][p][j] ssc[j][m]
            R cc[3];
#pragma unroll
            for (int p = 0; p < 3; p++) {
                R acc = 0;
#pragma unroll
                for (int m = 0; m < 3; m++)
#pragma unroll
                    for (int j = 0; j < 3; j++)
                        if (levi(m, p, j) != 0) acc += (R)levi(m, p, j) * ssc[j][m];
                cc[p] = acc;
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                r[3 + d] = sw * c.CsRT1 * cc[d];
                r[3 + C::NOU + d] = sw * c.CsRT0 * cc[d];
#pragma unroll
                for (int k = 0; k < 3; k++) r[C::XT + 3 * d + k] = sw * c.CsRT2 * s.n[k] * a[d];
            }
        } else {  // kRH: c = sw CsRH0 P, m = sw CsRH0 (-2 ssc)
            const R B = (ssc[0][0] + ssc[1][1] + ssc[2][2]) * c.CsRH1;
            const R f = sw * c.CsRH0;
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    r[3 + d * 3 + j] =
                        f * ((d == j ? B : R(0)) + c.CsRH2 * ssc[j][d] - 2 * ssc[d][j]);
                    r[3 + C::NOU + d * 3 + j] = f * (R(-2) * ssc[d][j]);  // m[k=d][j]
                }
        }
    }
}

// ---- P2M -------------------------------------------------------------------
// One block per source leaf; thread t owns moment entries (ch, a).
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_p2m(int p, int nq, const int64_t* __restrict__ leaves, const int64_t* __restrict__ nstart,
        const int64_t* __restrict__ nend, const R* __restrict__ ncent,
        const R* __restrict__ rec, R* __restrict__ mom) {
    using C = Chan<K>;
    const int NT = n_terms(p);
    const int64_t node = leaves[blockIdx.x];
    const R c0 = ncent[3 * node], c1 = ncent[3 * node + 1], c2 = ncent[3 * node + 2];
    const int64_t p0 = nstart[node] * nq, p1 = nend[node] * nq;
    R* M = mom + node * (int64_t)C::NCH * NT;
    for (int e = threadIdx.x; e < C::NCH * NT; e += blockDim.x) {
        const int ch = e / NT, a = e % NT;
        // decode a -> (a0, a1, a2)
        int n = 0;
        while (n_terms(n) <= a) n++;
        int rem = n > 0 ? a - n_terms(n - 1) : 0;
        int a0 = n, off = 0;
        while (off + (n - a0 + 1) <= rem) {
            off += n - a0 + 1;
            a0--;
        }
        const int a2 = rem - off, a1 = n - a0 - a2;
        R acc = 0;
        for (int64_t pt = p0; pt < p1; pt++) {
            const R* r = rec + pt * C::REC;
            const R Y[3] = {r[0] - c0, r[1] - c1, r[2] - c2};
            auto mono = [&](int b0, int b1, int b2) -> R {
                if (b0 < 0 || b1 < 0 || b2 < 0) return R(0);
                R v = 1;
                for (int k = 0; k < b0; k++) v *= Y[0];
                for (int k = 0; k < b1; k++) v *= Y[1];
                for (int k = 0; k < b2; k++) v *= Y[2];
                return v;
            };
            // dipole of vector w at Y: N_a += -sum_k a_k w_k Y^(a - e_k)
            auto dip = [&](R w0, R w1, R w2) -> R {
                return -((R)a0 * w0 * mono(a0 - 1, a1, a2) + (R)a1 * w1 * mono(a0, a1 - 1, a2) +
                         (R)a2 * w2 * mono(a0, a1, a2 - 1));
            };
            R val;
            if (ch < C::CH_Y) {
                val = r[3 + ch] * mono(a0, a1, a2);
            } else if (ch < C::CH_M) {
                const int o = ch - C::CH_Y, d = o / C::J, j = o % C::J;
                const R* m = r + 3 + C::NOU;
                val = dip(Y[d] * m[0 * C::J + j], Y[d] * m[1 * C::J + j], Y[d] * m[2 * C::J + j]);
            } else if (ch < C::CH_V) {
                const int j = ch - C::CH_M;
                const R* m = r + 3 + C::NOU;
                val = dip(m[0 * C::J + j], m[1 * C::J + j], m[2 * C::J + j]);
            } else if (C::HAS_V) {
                const int d = ch - C::CH_V;
                const R* v = r + C::XT + 3 * d;
                val = dip(v[0], v[1], v[2]);
            } else {  // RA: channel (d, k) is the dipole a'_d e_k
                const int o = ch - C::CH_V, d = o / 3, k = o % 3;
                const R ad = r[C::XT + d];
                val = dip(k == 0 ? ad : R(0), k == 1 ? ad : R(0), k == 2 ? ad : R(0));
            }
            acc += val;
        }
        M[e] = acc;
    }
}

// ---- M2M -------------------------------------------------------------------
// One block per parent node of the given height; children are final.
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_m2m(int p, const int64_t* __restrict__ parents, const int64_t* __restrict__ children,
        const R* __restrict__ ncent, R* __restrict__ mom) {
    using C = Chan<K>;
    const int NT = n_terms(p);
    const int64_t P = parents[blockIdx.x];
    R* MP = mom + P * (int64_t)C::NCH * NT;
    for (int e = threadIdx.x; e < C::NCH * NT; e += blockDim.x) {
        const int ch = e / NT, a = e % NT;
        int n = 0;
        while (n_terms(n) <= a) n++;
        int rem = n > 0 ? a - n_terms(n - 1) : 0;
        int a0 = n, off = 0;
        while (off + (n - a0 + 1) <= rem) {
            off += n - a0 + 1;
            a0--;
        }
        const int a2 = rem - off, a1 = n - a0 - a2;
        R acc = 0;
        for (int c = 0; c < 8; c++) {
            const int64_t ch_node = children[8 * P + c];
            const R* MC = mom + ch_node * (int64_t)C::NCH * NT;
            const R del[3] = {ncent[3 * ch_node] - ncent[3 * P],
                              ncent[3 * ch_node + 1] - ncent[3 * P + 1],
                              ncent[3 * ch_node + 2] - ncent[3 * P + 2]};
            // shift: sum_{b <= a} C(a, b) N_b del^(a - b)
            auto shift = [&](const R* N) -> R {
                R s = 0;
                R p0 = 1, binom0 = 1;
                for (int b0 = a0; b0 >= 0; b0--) {
                    R p1 = 1, binom1 = 1;
                    for (int b1 = a1; b1 >= 0; b1--) {
                        R p2 = 1, binom2 = 1;
                        for (int b2 = a2; b2 >= 0; b2--) {
                            s += binom0 * binom1 * binom2 * p0 * p1 * p2 * N[midx(b0, b1, b2)];
                            // next b2 - 1: del2^(a2 - b2 + 1), C(a2, b2 - 1)
                            p2 *= del[2];
                            binom2 = binom2 * (R)b2 / (R)(a2 - b2 + 1);
                        }
                        p1 *= del[1];
                        binom1 = binom1 * (R)b1 / (R)(a1 - b1 + 1);
                    }
                    p0 *= del[0];
                    binom0 = binom0 * (R)b0 / (R)(a0 - b0 + 1);
                }
                return s;
            };
            R v = shift(MC + (int64_t)ch * NT);
            if (ch >= C::CH_Y && ch < C::CH_M) {
                // Y_d m channel: + del_d * (m channel) shifted
                const int o = ch - C::CH_Y, d = o / C::J, j = o % C::J;
                v += del[d] * shift(MC + (int64_t)(C::CH_M + j) * NT);
            }
            acc += v;
        }
        MP[e] = acc;
    }
}

// ---- target points ---------------------------------------------------------
template <typename R>
__device__ __forceinline__ void target_point(const TriGeom<R>& o, int q, const R* qx, R x[3]) {
    const R ox = qx[2 * q], oy = qx[2 * q + 1];
    const R ob[3] = {1 - ox - oy, ox, oy};
#pragma unroll
    for (int d = 0; d < 3; d++) x[d] = bary_point(o, ob, d);
}

// ---- P2P -------------------------------------------------------------------
// One block per obs leaf with a non-empty P2P list; a thread per target point.
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_p2p(int nq, const R* __restrict__ qx, const int64_t* __restrict__ obs_nodes,
        const int64_t* __restrict__ starts, const int64_t* __restrict__ srcs,
        const int64_t* __restrict__ o_start, const int64_t* __restrict__ o_end,
        const int64_t* __restrict__ s_start, const int64_t* __restrict__ s_end,
        const R* __restrict__ pts, const int32_t* __restrict__ obs_tris,
        const R* __restrict__ rec, R* __restrict__ F) {
    using C = Chan<K>;
    const int64_t node = obs_nodes[blockIdx.x];
    const int64_t t0 = o_start[node] * nq, t1 = o_end[node] * nq;
    for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
        TriGeom<R> o;
        load_tri(o, pts, obs_tris, t / nq, 0, false, false);
        R x[3];
        target_point(o, (int)(t % nq), qx, x);
        R acc[C::NO];
#pragma unroll
        for (int k = 0; k < C::NO; k++) acc[k] = 0;
        for (int64_t l = starts[blockIdx.x]; l < starts[blockIdx.x + 1]; l++) {
            const int64_t sn = srcs[l];
            for (int64_t sp = s_start[sn] * nq; sp < s_end[sn] * nq; sp++) {
                const R* r = rec + sp * C::REC;
                const R D[3] = {r[0] - x[0], r[1] - x[1], r[2] - x[2]};
                const R r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
                if (r2 == R(0)) continue;
                const R invr = rsqrt_r(r2);
                const R invr3 = invr * invr * invr;
#pragma unroll
                for (int d = 0; d < 3; d++)
#pragma unroll
                    for (int j = 0; j < C::J; j++) {
                        const R* m = r + 3 + C::NOU;
                        const R Dm = D[0] * m[0 * C::J + j] + D[1] * m[1 * C::J + j] +
                                     D[2] * m[2 * C::J + j];
                        acc[d * C::J + j] += r[3 + d * C::J + j] * invr + D[d] * Dm * invr3;
                    }
                if (C::HAS_V) {
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        const R* v = r + C::XT + 3 * d;
                        acc[d] += (v[0] * D[0] + v[1] * D[1] + v[2] * D[2]) * invr3;
                    }
                }
                if (C::HAS_A) {
                    const R nD = (o.n[0] * D[0] + o.n[1] * D[1] + o.n[2] * D[2]) * invr3;
#pragma unroll
                    for (int d = 0; d < 3; d++) acc[C::NOU + d] -= nD * r[C::XT + d];
                }
            }
        }
        R* f = F + t * C::NO;
#pragma unroll
        for (int k = 0; k < C::NO; k++) f[k] += acc[k];
    }
}

// ---- M2P -------------------------------------------------------------------
// One block per obs leaf with a non-empty M2P list; moments of each listed
// source node are staged in shared memory; a thread per target point.
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_m2p(int p, int nq, const R* __restrict__ qx, const int64_t* __restrict__ obs_nodes,
        const int64_t* __restrict__ starts, const int64_t* __restrict__ srcs,
        const int64_t* __restrict__ o_start, const int64_t* __restrict__ o_end,
        const R* __restrict__ ncent, const R* __restrict__ pts,
        const int32_t* __restrict__ obs_tris, const R* __restrict__ mom, R* __restrict__ F) {
    using C = Chan<K>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
    const int NT = n_terms(p);
    const int64_t node = obs_nodes[blockIdx.x];
    const int64_t t0 = o_start[node] * nq, t1 = o_end[node] * nq;
    R Dv[FMM_MAXN];
    for (int64_t tb = t0; tb < t1; tb += blockDim.x) {
        const int64_t t = tb + threadIdx.x;
        const bool valid = t < t1;
        R x[3] = {0, 0, 0}, nrm[3] = {0, 0, 0};
        if (valid) {
            TriGeom<R> o;
            load_tri(o, pts, obs_tris, t / nq, 0, false, false);
            target_point(o, (int)(t % nq), qx, x);
#pragma unroll
            for (int d = 0; d < 3; d++) nrm[d] = o.n[d];
        }
        R acc[C::NO];
#pragma unroll
        for (int k = 0; k < C::NO; k++) acc[k] = 0;
        for (int64_t l = starts[blockIdx.x]; l < starts[blockIdx.x + 1]; l++) {
            const int64_t sn = srcs[l];
            __syncthreads();
            for (int e = threadIdx.x; e < C::NCH * NT; e += blockDim.x)
                sm[e] = mom[sn * (int64_t)C::NCH * NT + e];
            __syncthreads();
            if (!valid) continue;
            const R X[3] = {x[0] - ncent[3 * sn], x[1] - ncent[3 * sn + 1], x[2] - ncent[3 * sn + 2]};
            const R r2 = X[0] * X[0] + X[1] * X[1] + X[2] * X[2];
            const R inv_r2 = R(1) / r2;
            R phi[C::NCH];
#pragma unroll
            for (int ch = 0; ch < C::NCH; ch++) phi[ch] = 0;
            // D_0 = 1/r; level by level, D_g from D_(g-e_i), D_(g-2e_i)
            Dv[0] = sqrt(inv_r2);
#pragma unroll
            for (int ch = 0; ch < C::NCH; ch++) phi[ch] += sm[ch * NT] * Dv[0];
            for (int n = 1; n <= p; n++) {
                const R cA = -(R)(2 * n - 1) / (R)n * inv_r2;
                const R cB = -(R)(n - 1) / (R)n * inv_r2;
                const R sgn = (n & 1) ? R(-1) : R(1);
                for (int a0 = n; a0 >= 0; a0--)
                    for (int a2 = 0; a2 <= n - a0; a2++) {
                        const int a1 = n - a0 - a2;
                        R s1 = 0, s2 = 0;
                        if (a0 > 0) s1 += X[0] * Dv[midx(a0 - 1, a1, a2)];
                        if (a1 > 0) s1 += X[1] * Dv[midx(a0, a1 - 1, a2)];
                        if (a2 > 0) s1 += X[2] * Dv[midx(a0, a1, a2 - 1)];
                        if (a0 > 1) s2 += Dv[midx(a0 - 2, a1, a2)];
                        if (a1 > 1) s2 += Dv[midx(a0, a1 - 2, a2)];
                        if (a2 > 1) s2 += Dv[midx(a0, a1, a2 - 2)];
                        const int g = midx(a0, a1, a2);
                        const R Dg = cA * s1 + cB * s2;
                        Dv[g] = Dg;
                        const R sD = sgn * Dg;
#pragma unroll
                        for (int ch = 0; ch < C::NCH; ch++) phi[ch] += sm[ch * NT + g] * sD;
                    }
            }
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int j = 0; j < C::J; j++) {
                    const int oc = d * C::J + j;
                    acc[oc] += phi[C::CH_MONO + oc] + phi[C::CH_Y + oc] - X[d] * phi[C::CH_M + j];
                }
            if (C::HAS_V) {
#pragma unroll
                for (int d = 0; d < 3; d++) acc[d] += phi[C::CH_V + d];
            }
            if (C::HAS_A) {
#pragma unroll
                for (int d = 0; d < 3; d++)
                    acc[C::NOU + d] -= nrm[0] * phi[C::CH_V + 3 * d] +
                                       nrm[1] * phi[C::CH_V + 3 * d + 1] +
                                       nrm[2] * phi[C::CH_V + 3 * d + 2];
            }
        }
        if (valid) {
            R* f = F + t * C::NO;
#pragma unroll
            for (int k = 0; k < C::NO; k++) f[k] += acc[k];
        }
    }
}

// ---- final contraction -----------------------------------------------------
// out[orig(o)][b][d] (+)= L * J_o * (RH: sum_j sc[b][j] sum_q w_q F_q[d][j];
//                                    U/RT: sum_q w_q phi_b(x_q) F_q[d])
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_finish(int nq, const R* __restrict__ qx, const R* __restrict__ qw,
           const R* __restrict__ pts, const int32_t* __restrict__ obs_tris, int64_t n_obs,
           const int64_t* __restrict__ obs_orig, const R* __restrict__ F, R scale,
           R* __restrict__ out, int accumulate) {
    using C = Chan<K>;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_obs) return;
    TriGeom<R> o;
    load_tri(o, pts, obs_tris, i, 0, false, K == kRH || K == kRA);
    R o9[9], U[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 9; k++) o9[k] = 0;
    for (int q = 0; q < nq; q++) {
        const R* f = F + (i * nq + q) * C::NO;
        const R w = qw[q];
        if (K == kRH) {
#pragma unroll
            for (int b = 0; b < 3; b++)
#pragma unroll
                for (int d = 0; d < 3; d++)
                    o9[b * 3 + d] += w * (o.sc[b][0] * f[d * 3 + 0] + o.sc[b][1] * f[d * 3 + 1] +
                                          o.sc[b][2] * f[d * 3 + 2]);
        } else if (K == kRA) {
            // Fv with the basis functions; Fu summed for the curl contraction
            const R ox = qx[2 * q], oy = qx[2 * q + 1];
            const R ob[3] = {1 - ox - oy, ox, oy};
#pragma unroll
            for (int b = 0; b < 3; b++)
#pragma unroll
                for (int d = 0; d < 3; d++) o9[b * 3 + d] += w * ob[b] * f[3 + d];
#pragma unroll
            for (int k = 0; k < 3; k++) U[k] += w * f[k];
        } else {
            const R ox = qx[2 * q], oy = qx[2 * q + 1];
            const R ob[3] = {1 - ox - oy, ox, oy};
#pragma unroll
            for (int b = 0; b < 3; b++)
#pragma unroll
                for (int d = 0; d < 3; d++) o9[b * 3 + d] += w * ob[b] * f[d];
        }
    }
    if (K == kRA) {
        // + sum_m sc_o[b][m] V[m][d],  V[m][d] = -sum_k e[m][d][k] U_k
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int m = 0; m < 3; m++)
#pragma unroll
                    for (int k = 0; k < 3; k++)
                        if (levi(m, d, k) != 0)
                            o9[b * 3 + d] -= (R)levi(m, d, k) * o.sc[b][m] * U[k];
    }
    R* op = out + obs_orig[i] * 9;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const R v = scale * o.J * o9[k];
        op[k] = accumulate ? op[k] + v : v;
    }
}

struct FmmArgs {
    int p, nq;
    const void *qx, *qw;               // device rule (Real): nq x 2, nq
    const void *obs_pts, *src_pts;     // scaled points (Real)
    const int32_t *obs_tris, *src_tris;  // tree order
    int64_t n_obs, n_src;
    const int64_t* obs_orig;           // tree position -> original obs index
    const int64_t* src_orig;           // tree position -> original src index
    const int64_t *o_start, *o_end, *s_start, *s_end;
    const void* s_cent;                // src node centres (Real, 3 per node)
    int64_t n_src_nodes;
    const int64_t* src_leaves;
    int64_t n_src_leaves;
    const int64_t* m2m_parents;        // parents grouped by height (ascending)
    int n_heights;
    const int64_t* s_children;
    const int64_t *p2p_obs, *p2p_start, *p2p_src;
    int64_t n_p2p_obs;
    const int64_t *m2p_obs, *m2p_start, *m2p_src;
    int64_t n_m2p_obs;
};

template <typename R, int K>
int run_fmm(const FmmArgs& a, const double* params, double scale, const void* in, void* out,
            int accumulate, unsigned char* ws, const int64_t* height_counts_host,
            cudaStream_t st) {
    using C = Chan<K>;
    Consts<R> c = make_consts<R>(params);
    const int NT = n_terms(a.p);
    R* rec = reinterpret_cast<R*>(ws);
    const size_t rec_bytes = (sizeof(R) * C::REC * a.n_src * a.nq + 255) / 256 * 256;
    R* mom = reinterpret_cast<R*>(ws + rec_bytes);
    const size_t mom_bytes = (sizeof(R) * (size_t)C::NCH * NT * a.n_src_nodes + 255) / 256 * 256;
    R* F = reinterpret_cast<R*>(ws + rec_bytes + mom_bytes);
    const R* qx = (const R*)a.qx;
    const R* qw = (const R*)a.qw;
    fmm_charges<R, K><<<(unsigned)((a.n_src + 127) / 128), 128, 0, st>>>(
        c, a.nq, qx, qw, (const R*)a.src_pts, a.src_tris, a.n_src, a.src_orig, (const R*)in, rec);
    int rc = launch_status("fmm charges");
    if (rc) return rc;
    cudaMemsetAsync(F, 0, sizeof(R) * C::NO * a.n_obs * a.nq, st);
    if (a.n_src_leaves > 0) {
        fmm_p2m<R, K><<<(unsigned)a.n_src_leaves, 128, 0, st>>>(
            a.p, a.nq, a.src_leaves, a.s_start, a.s_end, (const R*)a.s_cent, rec, mom);
        if ((rc = launch_status("fmm p2m"))) return rc;
    }
    for (int h = 0; h < a.n_heights; h++) {
        const int64_t cnt = height_counts_host[h + 1] - height_counts_host[h];
        if (cnt == 0) continue;
        fmm_m2m<R, K><<<(unsigned)cnt, 128, 0, st>>>(a.p, a.m2m_parents + height_counts_host[h],
                                                     a.s_children, (const R*)a.s_cent, mom);
        if ((rc = launch_status("fmm m2m"))) return rc;
    }
    if (a.n_p2p_obs > 0) {
        fmm_p2p<R, K><<<(unsigned)a.n_p2p_obs, 128, 0, st>>>(
            a.nq, qx, a.p2p_obs, a.p2p_start, a.p2p_src, a.o_start, a.o_end, a.s_start, a.s_end,
            (const R*)a.obs_pts, a.obs_tris, rec, F);
        if ((rc = launch_status("fmm p2p"))) return rc;
    }
    if (a.n_m2p_obs > 0) {
        const size_t smem = sizeof(R) * (size_t)C::NCH * NT;
        auto kfn = fmm_m2p<R, K>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kfn<<<(unsigned)a.n_m2p_obs, 128, smem, st>>>(
            a.p, a.nq, qx, a.m2p_obs, a.m2p_start, a.m2p_src, a.o_start, a.o_end,
            (const R*)a.s_cent, (const R*)a.obs_pts, a.obs_tris, mom, F);
        if ((rc = launch_status("fmm m2p"))) return rc;
    }
    fmm_finish<R, K><<<(unsigned)((a.n_obs + 127) / 128), 128, 0, st>>>(
        a.nq, qx, qw, (const R*)a.obs_pts, a.obs_tris, a.n_obs, a.obs_orig, F, (R)scale, (R*)out,
        accumulate);
    return launch_status("fmm finish");
}

inline int nch_of(int kernel) {
    switch (kernel) {
        case kU: return Chan<kU>::NCH;
        case kRT: return Chan<kRT>::NCH;
        case kRA: return Chan<kRA>::NCH;
        case kRH: return Chan<kRH>::NCH;
        default: return -1;
    }
}
inline int rec_of(int kernel) {
    switch (kernel) {
        case kU: return Chan<kU>::REC;
        case kRT: return Chan<kRT>::REC;
        case kRA: return Chan<kRA>::REC;
        case kRH: return Chan<kRH>::REC;
        default: return -1;
    }
}
inline int no_of(int kernel) {
    switch (kernel) {
        case kU: return Chan<kU>::NO;
        case kRT: return Chan<kRT>::NO;
        case kRA: return Chan<kRA>::NO;
        case kRH: return Chan<kRH>::NO;
        default: return -1;
    }
}

}  // namespace
}  // namespace tct

using namespace tct;

extern "C" size_t tct_treecode_workspace_bytes(int kernel, int prec, int order, int64_t n_obs,
                                               int64_t n_src, int64_t n_src_nodes, int n_q) {
    if (nch_of(kernel) < 0 || order < 0 || order > FMM_MAXP || n_q < 1) return 0;
    const size_t rs = prec == TCT_F64 ? 8 : 4;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    return al(rs * rec_of(kernel) * (size_t)n_src * n_q) +
           al(rs * (size_t)nch_of(kernel) * n_terms(order) * (size_t)n_src_nodes) +
           al(rs * (size_t)no_of(kernel) * (size_t)n_obs * n_q);
}

extern "C" int tct_treecode_matvec(
    int kernel, int prec, int order, int n_q, const void* quad_pts, const void* quad_wts,
    const double* params, double out_scale, const void* obs_pts, const int32_t* obs_tris,
    int64_t n_obs, const int64_t* obs_orig, const int64_t* o_start, const int64_t* o_end,
    const void* src_pts, const int32_t* src_tris, int64_t n_src, const int64_t* src_orig,
    const int64_t* s_start, const int64_t* s_end, const void* s_centers, const int64_t* s_children,
    int64_t n_src_nodes, const int64_t* src_leaves, int64_t n_src_leaves,
    const int64_t* m2m_parents, const int64_t* m2m_height_counts_host, int n_heights,
    const int64_t* p2p_obs, const int64_t* p2p_start, const int64_t* p2p_src, int64_t n_p2p_obs,
    const int64_t* m2p_obs, const int64_t* m2p_start, const int64_t* m2p_src, int64_t n_m2p_obs,
    const void* in, void* out, int accumulate, void* workspace, size_t workspace_bytes,
    void* stream) {
    TCT_CHECK_ARG(order >= 0 && order <= FMM_MAXP, "tct_treecode_matvec: order must be 0..%d",
                  FMM_MAXP);
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_treecode_matvec: negative size");
    if (n_obs == 0) return TCT_OK;
    const size_t need = tct_treecode_workspace_bytes(kernel, prec, order, n_obs, n_src,
                                                     n_src_nodes, n_q);
    if (need == 0) {
        set_error("tct_treecode_matvec: kernel %d has no treecode (supported: elasticU3, "
                  "elasticRT3, elasticRA3, elasticRH3)", kernel);
        return TCT_ERR_KERNEL;
    }
    TCT_CHECK_ARG(workspace && workspace_bytes >= need && aligned(workspace, 256),
                  "tct_treecode_matvec: workspace of %zu bytes (256-aligned) required", need);
    FmmArgs a;
    a.p = order;
    a.nq = n_q;
    a.qx = quad_pts;
    a.qw = quad_wts;
    a.obs_pts = obs_pts;
    a.src_pts = src_pts;
    a.obs_tris = obs_tris;
    a.src_tris = src_tris;
    a.n_obs = n_obs;
    a.n_src = n_src;
    a.obs_orig = obs_orig;
    a.src_orig = src_orig;
    a.o_start = o_start;
    a.o_end = o_end;
    a.s_start = s_start;
    a.s_end = s_end;
    a.s_cent = s_centers;
    a.n_src_nodes = n_src_nodes;
    a.src_leaves = src_leaves;
    a.n_src_leaves = n_src_leaves;
    a.m2m_parents = m2m_parents;
    a.n_heights = n_heights;
    a.s_children = s_children;
    a.p2p_obs = p2p_obs;
    a.p2p_start = p2p_start;
    a.p2p_src = p2p_src;
    a.n_p2p_obs = n_p2p_obs;
    a.m2p_obs = m2p_obs;
    a.m2p_start = m2p_start;
    a.m2p_src = m2p_src;
    a.n_m2p_obs = n_m2p_obs;
    unsigned char* ws = reinterpret_cast<unsigned char*>(workspace);
    cudaStream_t st = as_stream(stream);
#define TCT_FMM(R, KID) \
    return run_fmm<R, KID>(a, params, out_scale, in, out, accumulate, ws, m2m_height_counts_host, st);
    if (prec == TCT_F64) {
        switch (kernel) {
            case kU: TCT_FMM(double, kU)
            case kRT: TCT_FMM(double, kRT)
            case kRA: TCT_FMM(double, kRA)
            case kRH: TCT_FMM(double, kRH)
        }
    } else if (prec == TCT_F32) {
        switch (kernel) {
            case kU: TCT_FMM(float, kU)
            case kRT: TCT_FMM(float, kRT)
            case kRA: TCT_FMM(float, kRA)
            case kRH: TCT_FMM(float, kRH)
        }
    }
#undef TCT_FMM
    set_error("tct_treecode_matvec: unsupported precision %d or kernel %d", prec, kernel);
    return TCT_ERR_ARG;
}
