// Treecode and FMM farfield for elasticU3, elasticRT3, elasticRA3 and
// elasticRH3 -- the kernels the reference's treecode supports
// (fmm/tsfmm.py, fmm/ts_kernels.cl:428-1003).
//
// Formulation.  In the hoisted vector form every supported kernel sends,
// from a source quadrature point y to a target point x (D = y - x, r = |D|),
//   F[d][j] = c[d][j] / r + sum_k D_d D_k m[k][j] / r^3 + sum_k v[d][k] D_k / r^3
// where c, m, v are per-point "charges" (J = 3 output columns for RH, 1 for U,
// RT and RA; v only for RT; RA adds an obs-normal dipole field, see Chan).
// Since D_k / r^3 = d/dx_k (1/r) and D_d = Y_d - X_d with Y = y - C,
// X = x - C about an expansion centre C:
//   F[d][j] = Phi[c_dj] + Phi_dip[Y_d m_.j] - X_d Phi_dip[m_.j] + Phi_dip[v_d.]
// -- Laplace potentials of monopoles and dipoles only.
//
// Multipoles (Cartesian, scaled by the node radius s): N_a = sum q Yh^a for a
// monopole q at Y (Yh = Y / s) and N_a += -(1/s) sum_k a_k w_k Yh^(a - e_k)
// for a dipole w; the potential at X is
//   Phi(X) = (1/s) sum_{|a| <= p} (-1)^|a| N_a D_a(X / s),  D_a = (1/a!) d^a (1/|X|),
// with D from the recurrence
//   n |X|^2 D_g = -(2n - 1) sum_i X_i D_(g - e_i) - (n - 1) sum_i D_(g - 2e_i).
// M2M: N^P_a = sum_{b <= a} C(a, b) (s_C / s_P)^|b| (del / s_P)^(a - b) N^C_b,
// del = C_C - C_P; the centre-dependent channels Y_d m gain del_d times the
// shifted m channel.
//
// Local expansions (FMM mode) about an obs node centre C_o, xi = x - C_o,
// scaled by the obs node radius: Phi(x) = sum_b L_b (xi / s_o)^b with
//   M2L: L_b = (1/rho) (s_o/rho)^|b| sum_a (-1)^|a| (s_s/rho)^|a| C(a+b, b)
//              D_(a+b)(R0 / rho) N_a,   R0 = C_o - C_s, rho = |R0|, |a|+|b| <= p;
//   L2L: L^C_b = (s_C/s_P)^|b| sum_{c >= b} C(c, b) (del / s_P)^(c - b) L^P_c;
// the Y_d m channel becomes Yl = Phi[Y_d m] - R0_d Phi[m] (applied to each
// pair's sums), so that at the target
//   F[d][j] = L[c_dj](xi) + L[Yl_dj](xi) - xi_d L[m_.j](xi).
//
// Multi-indices a = (a0, a1, a2), |a| = n <= p, are stored graded:
// idx(a) = n(n+1)(n+2)/6 + (n - a0)(n - a0 + 1)/2 + a2.
//
// P2P runs the direct farfield's triangle-level pair loop (far_common.cuh) on
// the listed leaf pairs, from the same per-source records the P2M reads.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "far_common.cuh"

namespace tct {
namespace {

constexpr int FMM_MAXP = 12;
constexpr int FMM_LVL = (FMM_MAXP + 1) * (FMM_MAXP + 2) / 2;  // 91 terms in the top level

__host__ __device__ constexpr int n_terms(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }
// number of (a, b) pairs with |a| + |b| <= p: C(p + 6, 6)
__host__ __device__ constexpr int n_terms6(int p) {
    return (p + 1) * (p + 2) * (p + 3) * (p + 4) * (p + 5) * (p + 6) / 720;
}
__host__ __device__ __forceinline__ int midx(int a0, int a1, int a2) {
    const int n = a0 + a1 + a2;
    return n * (n + 1) * (n + 2) / 6 + (n - a0) * (n - a0 + 1) / 2 + a2;
}
// position of (a0, ., a2) within level n
__device__ __forceinline__ int lidx(int n, int a0, int a2) { return (n - a0) * (n - a0 + 1) / 2 + a2; }

__host__ __device__ __forceinline__ void decode(int g, int& a0, int& a1, int& a2) {
    int n = 0;
    while (n_terms(n) <= g) n++;
    int rem = n > 0 ? g - n_terms(n - 1) : 0;
    a0 = n;
    int off = 0;
    while (off + (n - a0 + 1) <= rem) {
        off += n - a0 + 1;
        a0--;
    }
    a2 = rem - off;
    a1 = n - a0 - a2;
}

template <typename R>
__device__ __forceinline__ R ipow(R x, int n) {
    R v = 1;
    for (int k = 0; k < n; k++) v *= x;
    return v;
}

// binomial table C(n, k), n, k <= FMM_MAXP, built in shared memory
template <typename R>
__device__ __forceinline__ void fill_binom(R* bin) {
    if (threadIdx.x <= FMM_MAXP) {
        const int n = threadIdx.x;
        R v = 1;
        for (int k = 0; k <= FMM_MAXP; k++) {
            bin[n * (FMM_MAXP + 1) + k] = (k <= n) ? v : R(0);
            v = v * (R)(n - k) / (R)(k + 1);
        }
    }
}
#define BIN(n, k) bin[(n) * (FMM_MAXP + 1) + (k)]

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
    // point charges: y(3), c(NOU), m(3J: m[k][j] at 3 + NOU + k*J + j),
    // then v(9) for RT or a'(3) for RA
    static constexpr int XT = 3 + NOU + 3 * J;
    static constexpr int REC = XT + (HAS_V ? 9 : 0) + (HAS_A ? 3 : 0);
    static constexpr int NV = HAS_V ? 3 : (HAS_A ? 9 : 0);
    // expansion channels: mono (NOU), Y (NOU), M (J), V / A dipoles (NV)
    static constexpr int NCH = 2 * NOU + J + NV;
    static constexpr int NCHP = (NCH + 3) / 4 * 4;  // padded row of one term
    static constexpr int CH_MONO = 0, CH_Y = NOU, CH_M = 2 * NOU, CH_V = 2 * NOU + J;
};

// Charges of source quadrature point q from the far_prep record r.
template <typename R, int K, int NQ>
__device__ __forceinline__ void point_charges(const Consts<R>& c, const R* __restrict__ r, int q,
                                              R (&ch)[Chan<K>::REC]) {
    using L = Rec<K, NQ>;
    using C = Chan<K>;
#pragma unroll
    for (int d = 0; d < 3; d++) ch[d] = r[L::Y + 3 * q + d];
    const R sw = r[L::SW + q];
    if (K == kRH) {
        // SW carries J_s w CsRH0: c = sw P, m[k][j] = sw (-2 ssc[k][j])
#pragma unroll
        for (int k = 0; k < 9; k++) {
            ch[3 + k] = sw * r[L::P + k];
            ch[3 + C::NOU + k] = sw * r[L::SSC + k];
        }
    } else {
        R a[3];
#pragma unroll
        for (int d = 0; d < 3; d++) a[d] = r[L::INV + 3 * q + d];
        if (K == kU) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                ch[3 + d] = sw * c.CsU0 * a[d];
                ch[3 + C::NOU + d] = sw * c.CsU1 * a[d];
            }
        } else if (K == kRA) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                ch[3 + d] = sw * c.CsRT1 * a[d];
                ch[3 + C::NOU + d] = sw * c.CsRT0 * a[d];
                ch[C::XT + d] = sw * c.CsRT2 * a[d];
            }
        } else {  // kRT: curl c of the input, normal n
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const R cc = r[L::C + d];
                ch[3 + d] = sw * c.CsRT1 * cc;
                ch[3 + C::NOU + d] = sw * c.CsRT0 * cc;
#pragma unroll
                for (int k = 0; k < 3; k++) ch[C::XT + 3 * d + k] = sw * c.CsRT2 * r[L::N + k] * a[d];
            }
        }
    }
}

// Combine the expansion channels at a target into F (the M2P/L2P epilogue).
// X is the target relative to the centre the Y channel refers to.
template <typename R, int K>
__device__ __forceinline__ void combine(const R (&phi)[Chan<K>::NCH], const R X[3], const R nrm[3],
                                        R (&acc)[Chan<K>::NO]) {
    using C = Chan<K>;
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
            acc[C::NOU + d] -= nrm[0] * phi[C::CH_V + 3 * d] + nrm[1] * phi[C::CH_V + 3 * d + 1] +
                               nrm[2] * phi[C::CH_V + 3 * d + 2];
    }
}

// Vectorised copy of n Reals (n a multiple of 4) into shared memory.
template <typename R>
__device__ __forceinline__ void stage(R* __restrict__ dst, const R* __restrict__ src, int n) {
    if (sizeof(R) == 4) {
        const float4* s = reinterpret_cast<const float4*>(src);
        float4* d = reinterpret_cast<float4*>(dst);
        for (int k = threadIdx.x; k < n / 4; k += blockDim.x) d[k] = __ldg(s + k);
    } else {
        const double2* s = reinterpret_cast<const double2*>(src);
        double2* d = reinterpret_cast<double2*>(dst);
        for (int k = threadIdx.x; k < n / 2; k += blockDim.x) d[k] = __ldg(s + k);
    }
}

template <typename R>
__device__ __forceinline__ void target_point(const TriGeom<R>& o, const Rule2D<R>& rule, int q,
                                             R x[3]) {
    const R ob[3] = {1 - rule.x[q] - rule.y[q], rule.x[q], rule.y[q]};
#pragma unroll
    for (int d = 0; d < 3; d++) x[d] = bary_point(o, ob, d);
}

// ---- P2M -------------------------------------------------------------------
// One block per source leaf; thread g owns term g of every channel.
template <typename R, int K, int NQ>
__global__ void __launch_bounds__(128)
fmm_p2m(Consts<R> c, int p, const int64_t* __restrict__ leaves, const int64_t* __restrict__ nstart,
        const int64_t* __restrict__ nend, const R* __restrict__ ncent, const R* __restrict__ nrad,
        const R* __restrict__ rec, R* __restrict__ mom) {
    using C = Chan<K>;
    using L = Rec<K, NQ>;
    const int NT = n_terms(p);
    const int64_t node = leaves[blockIdx.x];
    const R c0 = ncent[3 * node], c1 = ncent[3 * node + 1], c2 = ncent[3 * node + 2];
    const R inv_s = R(1) / nrad[node];
    const int64_t t0 = nstart[node], t1 = nend[node];
    R* M = mom + node * (int64_t)C::NCHP * NT;
    for (int g = threadIdx.x; g < NT; g += blockDim.x) {
        int a0, a1, a2;
        decode(g, a0, a1, a2);
        R acc[C::NCH];
#pragma unroll
        for (int k = 0; k < C::NCH; k++) acc[k] = 0;
        for (int64_t t = t0; t < t1; t++) {
            for (int q = 0; q < NQ; q++) {
                R ch[C::REC];
                point_charges<R, K, NQ>(c, rec + t * L::LEN, q, ch);
                const R Y[3] = {ch[0] - c0, ch[1] - c1, ch[2] - c2};
                const R Yh[3] = {Y[0] * inv_s, Y[1] * inv_s, Y[2] * inv_s};
                const R p0 = ipow(Yh[0], a0 > 0 ? a0 - 1 : 0);
                const R p1 = ipow(Yh[1], a1 > 0 ? a1 - 1 : 0);
                const R p2 = ipow(Yh[2], a2 > 0 ? a2 - 1 : 0);
                const R f0 = a0 > 0 ? p0 * Yh[0] : R(1);
                const R f1 = a1 > 0 ? p1 * Yh[1] : R(1);
                const R f2 = a2 > 0 ? p2 * Yh[2] : R(1);
                const R mono = f0 * f1 * f2;
                // dipole factors: -(1/s) a_k Yh^(a - e_k)
                const R e0 = a0 > 0 ? -inv_s * (R)a0 * p0 * f1 * f2 : R(0);
                const R e1 = a1 > 0 ? -inv_s * (R)a1 * f0 * p1 * f2 : R(0);
                const R e2 = a2 > 0 ? -inv_s * (R)a2 * f0 * f1 * p2 : R(0);
#pragma unroll
                for (int o = 0; o < C::NOU; o++) acc[C::CH_MONO + o] += ch[3 + o] * mono;
#pragma unroll
                for (int j = 0; j < C::J; j++) {
                    const R mk0 = ch[3 + C::NOU + 0 * C::J + j], mk1 = ch[3 + C::NOU + 1 * C::J + j],
                            mk2 = ch[3 + C::NOU + 2 * C::J + j];
                    const R dm = e0 * mk0 + e1 * mk1 + e2 * mk2;
                    acc[C::CH_M + j] += dm;
#pragma unroll
                    for (int d = 0; d < 3; d++) acc[C::CH_Y + d * C::J + j] += Y[d] * dm;
                }
                if (C::HAS_V) {
#pragma unroll
                    for (int d = 0; d < 3; d++)
                        acc[C::CH_V + d] += e0 * ch[C::XT + 3 * d] + e1 * ch[C::XT + 3 * d + 1] +
                                            e2 * ch[C::XT + 3 * d + 2];
                }
                if (C::HAS_A) {
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        const R ad = ch[C::XT + d];
                        acc[C::CH_V + 3 * d + 0] += e0 * ad;
                        acc[C::CH_V + 3 * d + 1] += e1 * ad;
                        acc[C::CH_V + 3 * d + 2] += e2 * ad;
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < C::NCHP; k++) M[g * C::NCHP + k] = k < C::NCH ? acc[k] : R(0);
    }
}

// ---- M2M -------------------------------------------------------------------
// One block per parent node of one height; children are final.
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_m2m(int p, const int64_t* __restrict__ parents, const int64_t* __restrict__ children,
        const R* __restrict__ ncent, const R* __restrict__ nrad, R* __restrict__ mom) {
    using C = Chan<K>;
    __shared__ R bin[(FMM_MAXP + 1) * (FMM_MAXP + 1)];
    fill_binom(bin);
    __syncthreads();
    const int NT = n_terms(p);
    const int64_t P = parents[blockIdx.x];
    const R sP = nrad[P];
    R* MP = mom + P * (int64_t)C::NCHP * NT;
    for (int g = threadIdx.x; g < NT; g += blockDim.x) {
        int a0, a1, a2;
        decode(g, a0, a1, a2);
        R acc[C::NCH];
#pragma unroll
        for (int k = 0; k < C::NCH; k++) acc[k] = 0;
        for (int cidx = 0; cidx < 8; cidx++) {
            const int64_t cn = children[8 * P + cidx];
            const R* MC = mom + cn * (int64_t)C::NCHP * NT;
            const R del[3] = {ncent[3 * cn] - ncent[3 * P], ncent[3 * cn + 1] - ncent[3 * P + 1],
                              ncent[3 * cn + 2] - ncent[3 * P + 2]};
            const R dh[3] = {del[0] / sP, del[1] / sP, del[2] / sP};
            const R ratio = nrad[cn] / sP;
            R sm[C::NCH];  // shifted child moments
#pragma unroll
            for (int k = 0; k < C::NCH; k++) sm[k] = 0;
            R q0 = 1;
            for (int b0 = a0; b0 >= 0; b0--) {
                R q1 = 1;
                for (int b1 = a1; b1 >= 0; b1--) {
                    R q2 = 1;
                    for (int b2 = a2; b2 >= 0; b2--) {
                        const R coef = BIN(a0, b0) * BIN(a1, b1) * BIN(a2, b2) * q0 * q1 * q2 *
                                       ipow(ratio, b0 + b1 + b2);
                        const R* nb = MC + midx(b0, b1, b2) * C::NCHP;
#pragma unroll
                        for (int k = 0; k < C::NCH; k++) sm[k] += coef * nb[k];
                        q2 *= dh[2];
                    }
                    q1 *= dh[1];
                }
                q0 *= dh[0];
            }
#pragma unroll
            for (int k = 0; k < C::NCH; k++) acc[k] += sm[k];
            // Y_d m channel: + del_d times the shifted m channel
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int j = 0; j < C::J; j++) acc[C::CH_Y + d * C::J + j] += del[d] * sm[C::CH_M + j];
        }
#pragma unroll
        for (int k = 0; k < C::NCHP; k++) MP[g * C::NCHP + k] = k < C::NCH ? acc[k] : R(0);
    }
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem_dst)),
                 "l"(gsrc)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---- P2P -------------------------------------------------------------------
// One block per obs leaf with a non-empty P2P list.  The leaf's m obs
// triangles take m threads; the block's 128 threads form G = 128 / m groups,
// and group g takes the g-th of G equal slices of the list's source
// triangles (concatenated in list order), each thread running the direct
// farfield's pair loop over its group's source triangles (records read
// through L1 as broadcasts within a group).  Group sums are added in a fixed
// order, so the result is deterministic.  W[t] = per-obs-triangle sums in the
// NAcc layout (overwritten).
template <typename R, int K, int NQ>
__global__ void __launch_bounds__(128)
fmm_p2p(Consts<R> c, Rule2D<R> rule, const R* __restrict__ pts,
        const int32_t* __restrict__ obs_tris, const int64_t* __restrict__ obs_nodes,
        const int64_t* __restrict__ starts, const int64_t* __restrict__ srcs,
        const int64_t* __restrict__ o_start, const int64_t* __restrict__ o_end,
        const int64_t* __restrict__ s_start, const int64_t* __restrict__ s_end,
        const R* __restrict__ rec, R* __restrict__ W) {
    using L = Rec<K, NQ>;
    constexpr int NA = NAcc<K, NQ>::n;
    constexpr bool KAHAN = sizeof(R) == 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* red = reinterpret_cast<R*>(smem_raw);  // blockDim x NA
    const int64_t node = obs_nodes[blockIdx.x];
    const int64_t l0 = starts[blockIdx.x], l1 = starts[blockIdx.x + 1];
    const int64_t ob0 = o_start[node], n_o = o_end[node] - ob0;
    int64_t n_s = 0;  // source triangles over the whole list
    for (int64_t l = l0; l < l1; l++) {
        const int64_t sn = srcs[l];
        n_s += s_end[sn] - s_start[sn];
    }
    for (int64_t cb = 0; cb < n_o; cb += blockDim.x) {
        const int m = (int)min((int64_t)blockDim.x, n_o - cb);
        const int G = blockDim.x / m;
        const int grp = threadIdx.x / m, li = threadIdx.x % m;
        const bool active = grp < G;
        R tot[NA], cmp[NA];
#pragma unroll
        for (int k = 0; k < NA; k++) {
            tot[k] = 0;
            cmp[k] = 0;
        }
        if (active) {
            TriGeom<R> o;
            load_tri(o, pts, obs_tris, ob0 + cb + li, 0, false, K == kRA || K == kRH);
            R x[NQ][3];
#pragma unroll
            for (int q = 0; q < NQ; q++) target_point(o, rule, q, x[q]);
            // group grp takes source positions [p0, p1) of the list's
            // concatenated source triangles
            const int p0 = (int)(n_s * grp / G), p1 = (int)(n_s * (grp + 1) / G);
            int cpos = 0;
            for (int64_t l = l0; l < l1 && cpos < p1; l++) {
                const int64_t sn = srcs[l];
                const int64_t a = s_start[sn];
                const int n = (int)(s_end[sn] - a);
                const int lo = max(p0, cpos), hi = min(p1, cpos + n);
                const R* rp = rec + (a + (lo - cpos)) * L::LEN;
                cpos += n;
                if (lo >= hi) continue;
                R acc[NA];
#pragma unroll
                for (int k = 0; k < NA; k++) acc[k] = 0;
                for (int j = lo; j < hi; j++, rp += L::LEN)
                    far_pair<R, K, NQ>(c, rule, o, x, rp, acc);
#pragma unroll
                for (int k = 0; k < NA; k++) fold<R, KAHAN>(tot[k], cmp[k], acc[k]);
            }
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int k = 0; k < NA; k++) red[threadIdx.x * NA + k] = tot[k];
        }
        __syncthreads();
        if (threadIdx.x < m) {
            R* w = W + (ob0 + cb + threadIdx.x) * NA;
            for (int k = 0; k < NA; k++) {
                R sacc = 0;
                for (int g = 0; g < G; g++) sacc += red[(g * m + threadIdx.x) * NA + k];
                w[k] = sacc;
            }
        }
    }
}

// ---- P2P, packed elasticRH3 in FP32 ------------------------------------------
// fmm_p2p with the direct farfield's packed pair sums (rh2_pair).  A chunk of
// m <= 128 obs triangles of the leaf is split into T >= ceil(m / 64) teams of
// mt = ceil(m / T) triangles (T chosen for the fewest idle lanes); a group of h = ceil(mt / 2) lanes covers a team
// (a lane takes triangles li and li + h, one in each f32x2 half), a warp holds
// Gw = 32 / h groups (at most P2P_CHW), and the block's 4 Gw groups are team
// g % T and slice g / T of S = 4 Gw / T equal slices of the list's source
// triangles (concatenated in list order), so that small leaves still fill
// the lanes.  A group streams its slice through its own two shared-memory
// buffers of CHg = min(P2P_CHW / Gw, h) packed records (cp.async, the next
// chunk in flight while the current one is summed; records read as
// broadcasts within the group), and Kahan-folds its packed sums into its
// totals every 16 or more records.  Slice totals are added in a fixed order.
// W[t] = the 9 sums of obs triangle t in the NAcc layout (overwritten).
constexpr int P2P_CHW = 24;  // staged records per warp and buffer

template <int NQ>
constexpr size_t p2p_rh2_smem() {
    return sizeof(float) * (128 * 18 + 4 * 2 * P2P_CHW * RecRH2<NQ>::LEN);
}

template <int NQ, bool UNIFORM>
__global__ void __launch_bounds__(128, NQ == 3 ? 4 : 3)
fmm_p2p_rh2(Rule2D<float> rule, const float* __restrict__ pts,
            const int32_t* __restrict__ obs_tris, const int64_t* __restrict__ obs_nodes,
            const int64_t* __restrict__ starts, const int64_t* __restrict__ srcs,
            const int64_t* __restrict__ o_start, const int64_t* __restrict__ o_end,
            const int64_t* __restrict__ s_start, const int64_t* __restrict__ s_end,
            const float* __restrict__ rec, float* __restrict__ W) {
    using L = RecRH2<NQ>;
    constexpr int V4 = L::LEN / 4;  // float4s per record
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* red = reinterpret_cast<float*>(smem_raw);  // 128 x 18 slice totals
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* wbuf = red + 128 * 18 + warp * 2 * P2P_CHW * L::LEN;  // this warp's staging
    const int64_t node = obs_nodes[blockIdx.x];
    const int64_t l0 = starts[blockIdx.x], l1 = starts[blockIdx.x + 1];
    const int64_t ob0 = o_start[node], n_o = o_end[node] - ob0;
    f2_t wq[UNIFORM ? 1 : NQ * NQ];
    wq[0] = 0ull;
    if (!UNIFORM) {
#pragma unroll
        for (int q1 = 0; q1 < NQ; q1++)
#pragma unroll
            for (int q2 = 0; q2 < NQ; q2++) {
                const float w = rule.w[q1] * rule.w[q2];
                wq[q1 * NQ + q2] = pk(w, w);
            }
    }
    const f2_t eps = pk(RH2_EPS, RH2_EPS);
    int n_s = 0;  // source triangles over the whole list (warp reduction)
    for (int64_t l = l0 + lane; l < l1; l += 32) {
        const int64_t sn = srcs[l];
        n_s += (int)(s_end[sn] - s_start[sn]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_s += __shfl_xor_sync(0xffffffffu, n_s, o);

    for (int64_t cb = 0; cb < n_o; cb += 128) {
        const int m = (int)min((int64_t)128, n_o - cb);
        // teams: the count (from ceil(m / 64) up to 8) with the most slices per
        // obs triangle, m S, i.e. the fewest idle lanes and halves
        int T = (m + 63) / 64;
        {
            int best = 0, bt = T;
            for (int t = T; t <= 8; t++) {
                const int mtt = (m + t - 1) / t, ht = (mtt + 1) / 2;
                const int st = 4 * min(32 / ht, P2P_CHW) / t;
                if (m * st > best) {
                    best = m * st;
                    bt = t;
                }
            }
            T = bt;
        }
        const int mt = (m + T - 1) / T;
        const int h = (mt + 1) / 2;
        const int Gw = min(32 / h, P2P_CHW);
        const int S = 4 * Gw / T;
        const int gl = lane / h, li = lane - gl * h;
        const int gi = warp * Gw + gl;
        const int team = gi % T, slice = gi / T;
        const bool active = gl < Gw && slice < S;
        const int tb = team * mt, mteam = min(mt, m - tb);
        const bool va = active && li < mteam, vb = active && li + h < mteam;
        const int CHg = min(P2P_CHW / Gw, h);
        const int gbase = gl * h;
        const unsigned gmask = (h == 32 ? 0xffffffffu : ((1u << h) - 1u)) << (gbase & 31);
        float* buf = wbuf + (gl < Gw ? gl : 0) * 2 * CHg * L::LEN;
        float tot[2][9], cmp[2][9];
#pragma unroll
        for (int k = 0; k < 9; k++) {
            tot[0][k] = tot[1][k] = 0.f;
            cmp[0][k] = cmp[1][k] = 0.f;
        }
        if (active) {
            f2_t negx[NQ][3];
            {
                TriGeom<float> oa, ob;
                if (va) load_tri(oa, pts, obs_tris, ob0 + cb + tb + li, 0, false, true);
                if (vb) load_tri(ob, pts, obs_tris, ob0 + cb + tb + li + h, 0, false, true);
#pragma unroll
                for (int q = 0; q < NQ; q++) {
                    const float ox = rule.x[q], oy = rule.y[q];
                    const float bq[3] = {1 - ox - oy, ox, oy};
#pragma unroll
                    for (int d = 0; d < 3; d++)
                        negx[q][d] = pk(va ? -bary_point(oa, bq, d) : 0.f,
                                        vb ? -bary_point(ob, bq, d) : 0.f);
                }
            }
            // the slice [p0, p1) of the concatenated sources; the stream
            // cursor (list entry l, its first record a, offset off, records
            // left rem), the same in every lane of the group
            const int p0 = (int)((int64_t)n_s * slice / S);
            const int p1 = (int)((int64_t)n_s * (slice + 1) / S);
            int64_t l = l0, a = 0;
            int off = 0, rem = 0, skip = p0;
            while (l < l1) {  // find the entry holding position p0
                const int64_t sn = srcs[l];
                a = s_start[sn];
                rem = (int)(s_end[sn] - a);
                if (skip < rem) break;
                skip -= rem;
                l++;
            }
            off = skip;
            rem -= skip;
            // copy the next `need` (<= CHg <= h) stream records into buffer b
            auto issue = [&](int need, int b) {
                int64_t gidx = 0;
                int r_base = 0;
                while (r_base < need) {
                    while (rem == 0 && l + 1 < l1) {
                        l++;
                        const int64_t sn = srcs[l];
                        a = s_start[sn];
                        rem = (int)(s_end[sn] - a);
                        off = 0;
                    }
                    const int take = min(rem, need - r_base);
                    if (take <= 0) break;  // unreachable: the slice never outruns the list
                    if (li >= r_base && li < r_base + take) gidx = a + off + (li - r_base);
                    r_base += take;
                    off += take;
                    rem -= take;
                }
                float* dst = buf + b * CHg * L::LEN;
                for (int e0 = 0; e0 < need * V4; e0 += h) {  // uniform within the group
                    const int e = e0 + li;
                    const int r = min(e / V4, need - 1), part = e - r * V4;
                    const int64_t g = __shfl_sync(gmask, gidx, gbase + r);
                    if (e < need * V4)
                        cp_async16(dst + r * L::LEN + part * 4, rec + g * L::LEN + part * 4);
                }
                cp_async_commit();
            };
            const int n_mine = p1 - p0;
            f2_t Wp[9];
#pragma unroll
            for (int k = 0; k < 9; k++) Wp[k] = 0ull;
            int since = 0;
            if (n_mine > 0) issue(min(CHg, n_mine), 0);
            for (int c0 = 0; c0 < n_mine; c0 += CHg) {
                const int cur = (c0 / CHg) & 1;
                const int need = min(CHg, n_mine - c0);
                if (c0 + CHg < n_mine) {
                    issue(min(CHg, n_mine - c0 - CHg), cur ^ 1);
                    cp_async_wait_group<1>();
                } else {
                    cp_async_wait_group<0>();
                }
                __syncwarp(gmask);
                const float* rb = buf + cur * CHg * L::LEN;
#pragma unroll 2
                for (int j = 0; j < need; j++)
                    rh2_pair<NQ, UNIFORM>(reinterpret_cast<const f2_t*>(rb + j * L::LEN), negx,
                                          wq, eps, Wp);
                since += need;
                if (since >= 16 || c0 + CHg >= n_mine) {
#pragma unroll
                    for (int k = 0; k < 9; k++) {
                        float wa, wb;
                        upk(Wp[k], wa, wb);
                        fold<float, true>(tot[0][k], cmp[0][k], wa);
                        fold<float, true>(tot[1][k], cmp[1][k], wb);
                        Wp[k] = 0ull;
                    }
                    since = 0;
                }
                __syncwarp(gmask);  // buffer cur is free for the chunk after next
            }
        }
        __syncthreads();  // the previous chunk's reads of red are done
#pragma unroll
        for (int k = 0; k < 9; k++) {
            red[threadIdx.x * 18 + k] = tot[0][k];
            red[threadIdx.x * 18 + 9 + k] = tot[1][k];
        }
        __syncthreads();
        for (int t = threadIdx.x; t < m; t += blockDim.x) {
            const int tm = t / mt, within = t - tm * mt;
            const int half = within / h, ln = within - half * h;
            float* w = W + (ob0 + cb + t) * 9;
            for (int k = 0; k < 9; k++) {
                float sacc = 0.f;
                for (int sl = 0; sl < S; sl++) {
                    const int g = sl * T + tm, wg = g / Gw, lg = g - wg * Gw;
                    sacc += red[(wg * 32 + lg * h + ln) * 18 + half * 9 + k];
                }
                w[k] = sacc;
            }
        }
    }
}

// ---- M2P (treecode) --------------------------------------------------------
// One block per obs leaf with a non-empty M2P list; the moments of each listed
// source node are staged in shared memory; a thread per target point; the D
// recurrence keeps its last three levels in a per-thread ring.
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_m2p(int p, Rule2D<R> rule, int nq, const int64_t* __restrict__ obs_nodes,
        const int64_t* __restrict__ starts, const int64_t* __restrict__ srcs,
        const int64_t* __restrict__ o_start, const int64_t* __restrict__ o_end,
        const R* __restrict__ scent, const R* __restrict__ srad, const R* __restrict__ pts,
        const int32_t* __restrict__ obs_tris, const R* __restrict__ mom, R* __restrict__ F) {
    using C = Chan<K>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
    const int NT = n_terms(p);
    const int64_t node = obs_nodes[blockIdx.x];
    const int64_t t0 = o_start[node] * nq, t1 = o_end[node] * nq;
    R Dr[3][FMM_LVL];
    for (int64_t tb = t0; tb < t1; tb += blockDim.x) {
        const int64_t t = tb + threadIdx.x;
        const bool valid = t < t1;
        R x[3] = {0, 0, 0}, nrm[3] = {0, 0, 0};
        if (valid) {
            TriGeom<R> o;
            load_tri(o, pts, obs_tris, t / nq, 0, false, false);
            target_point(o, rule, (int)(t % nq), x);
#pragma unroll
            for (int d = 0; d < 3; d++) nrm[d] = o.n[d];
        }
        R acc[C::NO];
#pragma unroll
        for (int k = 0; k < C::NO; k++) acc[k] = 0;
        for (int64_t l = starts[blockIdx.x]; l < starts[blockIdx.x + 1]; l++) {
            const int64_t sn = srcs[l];
            __syncthreads();
            stage(sm, mom + sn * (int64_t)C::NCHP * NT, C::NCHP * NT);
            __syncthreads();
            if (!valid) continue;
            const R inv_s = R(1) / srad[sn];
            const R X[3] = {x[0] - scent[3 * sn], x[1] - scent[3 * sn + 1], x[2] - scent[3 * sn + 2]};
            const R Xh[3] = {X[0] * inv_s, X[1] * inv_s, X[2] * inv_s};
            const R inv_r2 = R(1) / (Xh[0] * Xh[0] + Xh[1] * Xh[1] + Xh[2] * Xh[2]);
            R phi[C::NCH];
            Dr[0][0] = sqrt(inv_r2);
#pragma unroll
            for (int k = 0; k < C::NCH; k++) phi[k] = sm[k] * Dr[0][0];
            int g = 1;
            for (int n = 1; n <= p; n++) {
                const R cA = -(R)(2 * n - 1) / (R)n * inv_r2;
                const R cB = -(R)(n - 1) / (R)n * inv_r2;
                const R sgn = (n & 1) ? R(-1) : R(1);
                R* cur = Dr[n % 3];
                const R* prv = Dr[(n - 1) % 3];
                const R* pp = Dr[(n + 1) % 3];  // level n - 2
                for (int a0 = n; a0 >= 0; a0--)
                    for (int a2 = 0; a2 <= n - a0; a2++, g++) {
                        const int a1 = n - a0 - a2;
                        R s1 = 0, s2 = 0;
                        if (a0 > 0) s1 += Xh[0] * prv[lidx(n - 1, a0 - 1, a2)];
                        if (a1 > 0) s1 += Xh[1] * prv[lidx(n - 1, a0, a2)];
                        if (a2 > 0) s1 += Xh[2] * prv[lidx(n - 1, a0, a2 - 1)];
                        if (a0 > 1) s2 += pp[lidx(n - 2, a0 - 2, a2)];
                        if (a1 > 1) s2 += pp[lidx(n - 2, a0, a2)];
                        if (a2 > 1) s2 += pp[lidx(n - 2, a0, a2 - 2)];
                        const R Dg = cA * s1 + cB * s2;
                        cur[lidx(n, a0, a2)] = Dg;
                        const R sD = sgn * Dg;
                        const R* nrow = sm + g * C::NCHP;
#pragma unroll
                        for (int k = 0; k < C::NCH; k++) phi[k] += nrow[k] * sD;
                    }
            }
#pragma unroll
            for (int k = 0; k < C::NCH; k++) phi[k] *= inv_s;
            combine<R, K>(phi, X, nrm, acc);
        }
        if (valid) {
            R* f = F + t * C::NO;
#pragma unroll
            for (int k = 0; k < C::NO; k++) f[k] += acc[k];
        }
    }
}

// ---- M2L (FMM) -------------------------------------------------------------
// Written as L_b = (s_o/rho)^|b| / (rho b!) sum_a f_|a| Dc_(a+b) Nt_a with
// Dc_c = c! D_c(R0 / rho), f_n = (-1)^n (s_s/rho)^n and Nt_a = N_a / a! (the
// moments are divided by a! once, after M2M, by fmm_moment_factorials), so a
// pair's source moments are used as stored; the Yl correction (- R0_d times
// the m channel) is linear in the moments and applied to each source row.
template <typename R>
__global__ void __launch_bounds__(128)
fmm_moment_factorials(int p, int nchp, int64_t n_nodes, R* __restrict__ mom) {
    const int NT = n_terms(p);
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_nodes * NT * nchp) return;
    int a0, a1, a2;
    decode((int)((e / nchp) % NT), a0, a1, a2);
    R f = 1;
    for (int k = 2; k <= a0; k++) f *= (R)k;
    for (int k = 2; k <= a1; k++) f *= (R)k;
    for (int k = 2; k <= a2; k++) f *= (R)k;
    mom[e] /= f;
}

template <typename R>
__device__ __forceinline__ R mfact(int b0, int b1, int b2) {
    R f = 1;
    for (int k = 2; k <= b0; k++) f *= (R)k;
    for (int k = 2; k <= b1; k++) f *= (R)k;
    for (int k = 2; k <= b2; k++) f *= (R)k;
    return f;
}

// ---- M2L, one CTA per observation node ------------------------------------
// L_b = 1/b! sum over the node's M2L list of (s_o/rho)^|b| / rho *
// sum_a f_|a| Dc_(a+b) (N_a with the Yl correction Y_dj - R0_d m_j), |a| + |b|
// <= p (ts_kernels.cl's m2l restated as a contraction over the pair's Dc
// tensor).  Organised for throughput:
//  * warps 0 and 1 (warp 0 alone for one-pair stages) are producers: for
//    the next stage's source nodes (one each) they compute rho, f_n,
//    (s_o/rho)^n / rho and Dc level by level, and scatter Dc into a dense
//    cube, so that Dc_(a+b) = cube[lin(a) + lin(b)] is one indexed load;
//    every thread copies its share of the next stage's moments into the
//    second row buffers with cp.async while the current stage is
//    contracted (the recurrence is latency-bound: one producer warp per
//    pair keeps it off the critical path);
//  * each contraction lane (192 with two-pair stages, 224 with one-pair
//    stages) owns a fixed tuple of NB consecutive
//    local terms b (all channels, accumulated in registers across the whole
//    list) and a contiguous chunk of source terms a, the same chunk for the
//    tuples that share it, so lanes of a warp mostly read the same source
//    row (shared-memory broadcasts); pairs with |a| + |b| > p are masked;
//  * at the end the lanes' partial sums go through shared memory in rounds
//    and each b sums its chunks in a fixed lane order and scales by 1 / b!.
// The plan (tuples, chunk length, lane tables) depends only on p and NB.
constexpr int M2L3_THREADS = 256;
// producer warps: one per pair of a two-pair stage, one for a one-pair stage
// (at the large orders that need one-pair stages the contraction dominates)
__host__ __device__ constexpr int m2l3_nprod(int B) { return B == 2 ? 2 : 1; }
__host__ __device__ constexpr int m2l3_lanes(int B) { return M2L3_THREADS - 32 * m2l3_nprod(B); }
constexpr int M2L3_LANES = M2L3_THREADS - 32;  // table capacity (the most lanes)
constexpr int FMM_NTMAX = (FMM_MAXP + 1) * (FMM_MAXP + 2) * (FMM_MAXP + 3) / 6;
constexpr int M2L3_PLAN_TAG = 0x4d324c33;  // "M2L3": the plan below is complete
struct M2LPlan3 {
    int tag;  // M2L3_PLAN_TAG once built (written last)
    int p, nb, lanes, L, n_lanes, n_k;
    int lane_k[M2L3_LANES];    // tuple of the lane (b = k NB + j), -1 for none
    int lane_a0[M2L3_LANES];   // first source term (graded) and chunk length
    int lane_cnt[M2L3_LANES];
    int warp_steps[M2L3_LANES / 32];
    int kstart[FMM_NTMAX + 1];  // lanes of tuple k: klane[kstart[k] .. kstart[k + 1])
    int klane[M2L3_LANES];
    int ainfo[FMM_NTMAX];      // lin(a) | |a| << 16
    // Dc recurrence per graded c (level n): the graded indices of c - e_0,
    // c - e_1, c - e_2 and lin(c); of c - 2 e_0, c - 2 e_1, c - 2 e_2 and 0;
    // then as float bits cA c_d (3) and 0, cB c_d (c_d - 1) (3) and 0, with
    // cA = -(2n - 1) / n, cB = -(n - 1) / n (absent neighbours: index 0,
    // coefficient 0)
    alignas(16) int rec[FMM_NTMAX][16];
};

// Cube index of a multi-index: lin(c) = c0 S0 + c1 S1 + c2, additive and
// injective on |c| <= p (S1 > p, S0 > p S1 + p); the strides are padded past
// the minimum so that the lanes of a warp, reading Dh[lin(a) + lin(b)] for
// their different b, spread over the shared-memory banks (p = 8: 10 and 91
// instead of 9 and 81 cut a warp step's wavefronts from ~30 to ~24).
__host__ __device__ inline int cube_s1(int p) { return p + 2; }
__host__ __device__ inline int cube_s0(int p) { return p * cube_s1(p) + p + 3; }
__host__ __device__ inline int cube_lin(int p, int a0, int a1, int a2) {
    return a0 * cube_s0(p) + a1 * cube_s1(p) + a2;
}
// cube entries read: lin(a) + lin(b) for |a|, |b| <= p (masked pairs included)
__host__ __device__ inline int cube_size(int p) {
    return 2 * p * (cube_s0(p) + cube_s1(p) + 1) + 1;
}

// Builds the plan; returns 0, or 1 when the tuples do not fit the lanes.
// Tuples k = 0 .. ceil(NT / nb) - 1 take the b's k nb .. k nb + nb - 1; tuple
// k's source range is [0, A_k), A_k = n_terms(p - |k nb|) (its lowest b), cut
// into chunks of L terms, L the smallest length whose chunks fit the lanes;
// lanes are dealt chunk-major (every tuple's first chunk, then every second
// chunk, ...), so the lanes of one chunk index are adjacent.
__host__ __device__ inline int m2l3_make_plan(int p, int nb, int lanes, M2LPlan3* plan) {
    const int NT = n_terms(p);
    const int nk = (NT + nb - 1) / nb;
    if (lanes < 32 || lanes > M2L3_LANES || lanes % 32) return 1;
    plan->p = p;
    plan->nb = nb;
    plan->lanes = lanes;
    plan->n_k = nk;
    auto A = [&](int k) {
        int b0, b1, b2;
        decode(k * nb, b0, b1, b2);
        return n_terms(p - (b0 + b1 + b2));
    };
    int total = 0;
    for (int k = 0; k < nk; k++) total += A(k);
    int L = (total + lanes - 1) / lanes;
    if (L < 1) L = 1;
    for (;; L++) {
        int cnt = 0;
        for (int k = 0; k < nk; k++) cnt += (A(k) + L - 1) / L;
        if (cnt <= lanes) break;
        if (L > NT) return 1;
    }
    plan->L = L;
    int lane = 0;
    for (int c = 0;; c++) {
        bool any = false;
        for (int k = 0; k < nk; k++) {
            const int ak = A(k);
            if (c * L >= ak) continue;
            plan->lane_k[lane] = k;
            plan->lane_a0[lane] = c * L;
            plan->lane_cnt[lane] = (ak - c * L < L) ? ak - c * L : L;
            lane++;
            any = true;
        }
        if (!any) break;
    }
    plan->n_lanes = lane;
    for (int l = lane; l < M2L3_LANES; l++) {
        plan->lane_k[l] = -1;
        plan->lane_a0[l] = 0;
        plan->lane_cnt[l] = 0;
    }
    for (int w = 0; w < lanes / 32; w++) {
        int m = 0;
        for (int l = 32 * w; l < 32 * w + 32; l++) m = plan->lane_cnt[l] > m ? plan->lane_cnt[l] : m;
        plan->warp_steps[w] = m;
    }
    int pos = 0;
    for (int k = 0; k < nk; k++) {
        plan->kstart[k] = pos;
        for (int l = 0; l < lane; l++)
            if (plan->lane_k[l] == k) plan->klane[pos++] = l;
    }
    plan->kstart[nk] = pos;
    for (int g = 0; g < NT; g++) {
        int a0, a1, a2;
        decode(g, a0, a1, a2);
        plan->ainfo[g] = cube_lin(p, a0, a1, a2) | ((a0 + a1 + a2) << 16);
        const int n = a0 + a1 + a2;
        const float cA = n > 0 ? -(float)(2 * n - 1) / (float)n : 0.f;
        const float cB = n > 0 ? -(float)(n - 1) / (float)n : 0.f;
        int* r = plan->rec[g];
        r[0] = a0 > 0 ? midx(a0 - 1, a1, a2) : 0;
        r[1] = a1 > 0 ? midx(a0, a1 - 1, a2) : 0;
        r[2] = a2 > 0 ? midx(a0, a1, a2 - 1) : 0;
        r[3] = cube_lin(p, a0, a1, a2);
        r[4] = a0 > 1 ? midx(a0 - 2, a1, a2) : 0;
        r[5] = a1 > 1 ? midx(a0, a1 - 2, a2) : 0;
        r[6] = a2 > 1 ? midx(a0, a1, a2 - 2) : 0;
        r[7] = 0;
        const float cf[8] = {cA * (float)a0, cA * (float)a1, cA * (float)a2, 0.f,
                             cB * (float)(a0 * (a0 - 1)), cB * (float)(a1 * (a1 - 1)),
                             cB * (float)(a2 * (a2 - 1)), 0.f};
        for (int t = 0; t < 8; t++) {
            float f = cf[t];
            int bits;
            memcpy(&bits, &f, sizeof(int));
            r[8 + t] = bits;
        }
    }
    return 0;
}

// Builds the plan in the operator's workspace once: a plan tagged complete
// for this (p, nb) -- it depends on nothing else -- is reused.
__global__ void __launch_bounds__(32) fmm_m2l3_plan(int p, int nb, int lanes,
                                                    M2LPlan3* __restrict__ plan, int* err) {
    if (threadIdx.x != 0) return;
    volatile int* tag = &plan->tag;
    if (*tag == M2L3_PLAN_TAG && plan->p == p && plan->nb == nb && plan->lanes == lanes) return;
    *tag = 0;
    if (m2l3_make_plan(p, nb, lanes, plan)) {
        *err = 1;
        return;
    }
    __threadfence();
    *tag = M2L3_PLAN_TAG;
}

// Terms b per lane (FP32): the accumulators (NB x NCH values) stay near 64
// registers.
template <int K>
struct M2L3Cfg {
    static constexpr int NCH = Chan<K>::NCH;
    static constexpr int NB = K == kRH ? 3 : 64 / NCH;
};

// Shared-memory layout (floats), B pairs per pipeline stage: row buffers
// 2 B x NT x NCHP, cubes 2 B x CUBEP (CUBEP >= cube_size(p), so lin(a) +
// lin(b) needs no clamp; these two regions double as the reduction area, at least
// 32 lanes' slots), graded Dc scratch B x NTP, 2 B x 40 scalars, 4 x
// M2L3_CAP pair geometry, then ainfo (NTP ints), M2L3_CAP source node ids and
// the recurrence table (NT x 16 ints).
constexpr int M2L3_CAP = 512;  // pairs whose source node and geometry are staged
struct M2L3Smem {
    int NT, NTP, CUBEP, area, dg, sb, pg, ai, total_bytes;
};
template <int K>
__host__ __device__ inline M2L3Smem m2l3_smem(int p, int B) {
    using C = Chan<K>;
    M2L3Smem m;
    m.NT = n_terms(p);
    m.NTP = (m.NT + 3) / 4 * 4;
    m.CUBEP = (cube_size(p) + 3) / 4 * 4;
    const int need = 2 * B * (m.NT * C::NCHP + m.CUBEP);
    const int slots32 = 32 * M2L3Cfg<K>::NB * C::NCH;
    m.area = need > slots32 ? need : (slots32 + 3) / 4 * 4;
    m.dg = m.area;
    m.sb = m.dg + B * m.NTP;
    m.pg = m.sb + 2 * B * 40;
    m.ai = m.pg + 4 * M2L3_CAP;
    m.total_bytes = (int)(sizeof(float) * m.ai + sizeof(int) * (m.NTP + M2L3_CAP) +
                          sizeof(int) * 16 * m.NT);
    return m;
}

template <int K, int B>
__global__ void __launch_bounds__(M2L3_THREADS, 2)
fmm_m2l3(int p, const int64_t* __restrict__ obs_nodes, int64_t n_obs_nodes,
         const int64_t* __restrict__ starts, const int64_t* __restrict__ srcs,
         const float* __restrict__ ocent, const float* __restrict__ orad,
         const float* __restrict__ scent, const float* __restrict__ srad,
         const float* __restrict__ mom, const M2LPlan3* __restrict__ plan,
         float* __restrict__ loc) {
    using C = Chan<K>;
    constexpr int NB = M2L3Cfg<K>::NB;
    constexpr int NCH = C::NCH;
    constexpr int NP = (NCH + 1) / 2;  // channel pairs (f32x2)
    constexpr int NPROD = m2l3_nprod(B), LANES = m2l3_lanes(B);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const M2L3Smem sm = m2l3_smem<K>(p, B);
    const int NT = sm.NT;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t oi = blockIdx.x;
    if (oi >= n_obs_nodes) return;
    const int rowsz = NT * C::NCHP;
    float* base = reinterpret_cast<float*>(smem_raw);
    float* Nb = base;                     // 2 B x NT x NCHP source rows
    float* Cb = base + 2 * B * rowsz;     // 2 B x CUBEP scaled Dc cubes
    float* Dg = base + sm.dg;             // B x NTP graded Dc (producer scratch)
    float* Sb = base + sm.sb;             // 2 B x 40: (-s_s/s_o)^n [0, 16), R0 [32, 35)
    float* pgeo = base + sm.pg;           // first M2L3_CAP pairs: source center and radius
    int* ainfo = reinterpret_cast<int*>(base + sm.ai);
    int* psrc = ainfo + sm.NTP;           // first M2L3_CAP pairs: source node
    int* rtab = psrc + M2L3_CAP;          // recurrence table
    for (int g = tid; g < NT; g += M2L3_THREADS) ainfo[g] = plan->ainfo[g];
    for (int e = tid; e < NT * 4; e += M2L3_THREADS)
        reinterpret_cast<int4*>(rtab)[e] = reinterpret_cast<const int4*>(plan->rec)[e];

    const int64_t node = obs_nodes[oi];
    const float co[3] = {ocent[3 * node], ocent[3 * node + 1], ocent[3 * node + 2]};
    const float so = orad[node];
    const float inv_so = 1.f / so;  // node radii are positive
    const int64_t l0 = starts[oi], l1 = starts[oi + 1];
    const int64_t npair = l1 - l0;
    // the list's source nodes and geometry, staged once (the pipeline below
    // would otherwise wait on dependent global loads every pair)
    for (int64_t i = tid; i < npair && i < M2L3_CAP; i += M2L3_THREADS) {
        const int64_t sn = srcs[l0 + i];
        psrc[i] = (int)sn;
        pgeo[4 * i] = scent[3 * sn];
        pgeo[4 * i + 1] = scent[3 * sn + 1];
        pgeo[4 * i + 2] = scent[3 * sn + 2];
        pgeo[4 * i + 3] = srad[sn];
    }
    __syncthreads();

    // pairs [k0, k0 + B) of the list (those below npair) into stage st
    auto issue_copy = [&](int64_t k0, int st) {
#pragma unroll
        for (int u = 0; u < B; u++) {
            const int64_t k = k0 + u;
            if (k >= npair) break;
            const int64_t sn = k < M2L3_CAP ? (int64_t)psrc[k] : srcs[l0 + k];
            const float* src = mom + sn * (int64_t)rowsz;
            float* dst = Nb + (st * B + u) * rowsz;
            for (int e = tid; e < rowsz / 4; e += M2L3_THREADS) cp_async16(dst + e * 4, src + e * 4);
        }
        cp_async_commit();
    };
    // coef(a, b) = f_|a| (s_o/rho)^|b| / rho Dc_(a+b) = S_|a| Dh_(a+b) with
    // Dh_c = Dc_c (s_o/rho)^|c| / rho (the cube) and S_n = (-s_s/s_o)^n; the
    // B pairs' recurrences run interleaved (independent chains)
    // producer warp w handles the stage's pairs u0 .. u0 + PB - 1
    constexpr int PB = B / NPROD;
    auto produce = [&](int64_t k0, int st) {  // warps 0 .. NPROD - 1
        const int u0 = warp * PB;
        float Rh[B][3], q[B], pwn[B];
        bool on[B];
#pragma unroll
        for (int uu = 0; uu < PB; uu++) {
            const int u = u0 + uu;
            const int64_t k = k0 + u;
            on[u] = k < npair;
            float cs[3] = {co[0] + 1.f, co[1], co[2]}, rs = 0.f;  // any distinct point if off
            if (on[u] && k < M2L3_CAP) {
                const float* g = pgeo + 4 * k;
                cs[0] = g[0]; cs[1] = g[1]; cs[2] = g[2]; rs = g[3];
            } else if (on[u]) {
                const int64_t sn = srcs[l0 + k];
                cs[0] = scent[3 * sn]; cs[1] = scent[3 * sn + 1]; cs[2] = scent[3 * sn + 2];
                rs = srad[sn];
            }
            const float R0[3] = {co[0] - cs[0], co[1] - cs[1], co[2] - cs[2]};
            const float rho = sqrtf(R0[0] * R0[0] + R0[1] * R0[1] + R0[2] * R0[2]);
            const float inv_rho = 1.f / rho;
            Rh[u][0] = R0[0] * inv_rho; Rh[u][1] = R0[1] * inv_rho; Rh[u][2] = R0[2] * inv_rho;
            q[u] = so * inv_rho;  // pw_n = q^n / rho
            pwn[u] = inv_rho;
            float* S = Sb + (st * B + u) * 40;
            if (lane <= p) S[lane] = ipow(-rs * inv_so, lane);
            if (lane < 3) S[32 + lane] = R0[lane];
            if (lane == 0) {
                Dg[u * sm.NTP] = 1.f;
                Cb[(st * B + u) * sm.CUBEP] = inv_rho;
            }
        }
        __syncwarp();
        // level n from levels n - 1 and n - 2; a lane takes entries lane and
        // lane + 32 of the level for each pair, loads first so the chains overlap
        for (int n = 1; n <= p; n++) {
            const int lsz = (n + 1) * (n + 2) / 2, b0 = n_terms(n - 1);
            float v[B][2];
            int dst[2], cl[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int w = lane + 32 * h;
                dst[h] = -1;
                cl[h] = 0;
                if (w >= lsz) continue;
                const int4* rt = reinterpret_cast<const int4*>(rtab + 16 * (b0 + w));
                const int4 i0 = rt[0], i1 = rt[1], f0 = rt[2], f1 = rt[3];
#pragma unroll
                for (int uu = 0; uu < PB; uu++) {
                    const int u = u0 + uu;
                    const float* D = Dg + u * sm.NTP;
                    v[u][h] = __int_as_float(f0.x) * Rh[u][0] * D[i0.x] +
                              __int_as_float(f0.y) * Rh[u][1] * D[i0.y] +
                              __int_as_float(f0.z) * Rh[u][2] * D[i0.z] +
                              __int_as_float(f1.x) * D[i1.x] + __int_as_float(f1.y) * D[i1.y] +
                              __int_as_float(f1.z) * D[i1.z];
                }
                dst[h] = b0 + w;
                cl[h] = i0.w;
            }
#pragma unroll
            for (int uu = 0; uu < PB; uu++) {
                const int u = u0 + uu;
                pwn[u] *= q[u];
#pragma unroll
                for (int h = 0; h < 2; h++)
                    if (dst[h] >= 0) {
                        Dg[u * sm.NTP + dst[h]] = v[u][h];
                        Cb[(st * B + u) * sm.CUBEP + cl[h]] = v[u][h] * pwn[u];
                    }
            }
            __syncwarp();
        }
    };

    // this lane's tuple and source chunk
    const int ct = tid - 32 * NPROD;
    int kk = -1, a_first = 0, cnt = 0, wsteps = 0;
    int blin[NB], thr[NB];
    if (warp >= NPROD) {
        kk = plan->lane_k[ct];
        a_first = plan->lane_a0[ct];
        cnt = plan->lane_cnt[ct];
        wsteps = plan->warp_steps[warp - NPROD];
    }
#pragma unroll
    for (int j = 0; j < NB; j++) {
        const int b = kk * NB + j;
        if (kk >= 0 && b < NT) {
            int b0, b1, b2;
            decode(b, b0, b1, b2);
            blin[j] = cube_lin(p, b0, b1, b2);
            thr[j] = p - (b0 + b1 + b2);  // a valid while |a| <= thr
        } else {
            blin[j] = 0;
            thr[j] = -1;  // never valid
        }
    }
    f2_t acc[NB][NP];
#pragma unroll
    for (int j = 0; j < NB; j++)
#pragma unroll
        for (int i = 0; i < NP; i++) acc[j][i] = 0ull;

    const int64_t nst = (npair + B - 1) / B;  // pipeline stages of B pairs
    if (nst > 0) {
        issue_copy(0, 0);
        if (warp < NPROD) produce(0, 0);
    }
    for (int64_t st = 0; st < nst; st++) {
        const int buf = (int)(st & 1);
        cp_async_wait_all();
        __syncthreads();  // stage st's rows, cubes and scalars are complete; st - 1 is done
        if (st + 1 < nst) {
            issue_copy((st + 1) * B, buf ^ 1);
            if (warp < NPROD) produce((st + 1) * B, buf ^ 1);
        }
        if (warp < NPROD) continue;
#pragma unroll 1
        for (int u = 0; u < B; u++) {
            if (st * B + u >= npair) break;
            const float* S = Sb + (buf * B + u) * 40;
            const float* Dc = Cb + (buf * B + u) * sm.CUBEP;
            const float* N = Nb + (buf * B + u) * rowsz;
            const float R0[3] = {S[32], S[33], S[34]};
#pragma unroll 1
            for (int s = 0; s < wsteps; s++) {
                const bool on = s < cnt;
                const int a = a_first + (on ? s : 0);
                const int e = ainfo[a];
                const int alin = e & 0xffff, la = e >> 16;
                const float fa = on ? S[la] : 0.f;
                f2_t cf[NB];
#pragma unroll
                for (int j = 0; j < NB; j++) {
                    const float c = la <= thr[j] ? Dc[alin + blin[j]] * fa : 0.f;
                    cf[j] = pk(c, c);
                }
                const float4* row = reinterpret_cast<const float4*>(N + a * C::NCHP);
                float v[C::NCHP];
#pragma unroll
                for (int k4 = 0; k4 < C::NCHP / 4; k4++) {
                    const float4 q4 = row[k4];
                    v[4 * k4] = q4.x; v[4 * k4 + 1] = q4.y; v[4 * k4 + 2] = q4.z;
                    v[4 * k4 + 3] = q4.w;
                }
#pragma unroll
                for (int d = 0; d < 3; d++)
#pragma unroll
                    for (int j = 0; j < C::J; j++)
                        v[C::CH_Y + d * C::J + j] -= R0[d] * v[C::CH_M + j];
#pragma unroll
                for (int i = 0; i < NP; i++) {
                    const f2_t vi = pk(v[2 * i], v[2 * i + 1]);
#pragma unroll
                    for (int j = 0; j < NB; j++) acc[j][i] = fma2(cf[j], vi, acc[j][i]);
                }
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();

    // reduction in rounds through the row/cube area
    constexpr int PER = NB * NCH;
    const int lpr = sm.area / PER;
    float* Lg = loc + node * (int64_t)rowsz;
    for (int lo = 0; lo < LANES; lo += lpr) {
        const int hi = lo + lpr < LANES ? lo + lpr : LANES;
        if (warp >= NPROD && ct >= lo && ct < hi) {
            float* sl = base + (ct - lo) * PER;
#pragma unroll
            for (int j = 0; j < NB; j++)
#pragma unroll
                for (int i = 0; i < NP; i++) {
                    float x, y;
                    upk(acc[j][i], x, y);
                    sl[j * NCH + 2 * i] = x;
                    if (2 * i + 1 < NCH) sl[j * NCH + 2 * i + 1] = y;
                }
        }
        __syncthreads();
        for (int b = tid; b < NT; b += M2L3_THREADS) {
            const int k = b / NB, j = b - k * NB;
            float sum[NCH];
#pragma unroll
            for (int c = 0; c < NCH; c++) sum[c] = 0.f;
            for (int i = plan->kstart[k]; i < plan->kstart[k + 1]; i++) {
                const int l = plan->klane[i];
                if (l < lo || l >= hi) continue;
                const float* sl = base + (l - lo) * PER + j * NCH;
#pragma unroll
                for (int c = 0; c < NCH; c++) sum[c] += sl[c];
            }
            int b0, b1, b2;
            decode(b, b0, b1, b2);
            const float inv = 1.f / mfact<float>(b0, b1, b2);
            float* out = Lg + b * C::NCHP;
            if (lo == 0) {
#pragma unroll
                for (int c = 0; c < C::NCHP; c++) out[c] = c < NCH ? sum[c] * inv : 0.f;
            } else {
#pragma unroll
                for (int c = 0; c < NCH; c++) out[c] += sum[c] * inv;
            }
        }
        __syncthreads();
    }
}


// ---- M2L, item form (FP64, and FP32 when the lane plan does not fit) -------
// The same L_b as fmm_m2l3 above.  Warp 0 is the producer:
// for source node k + 1 it computes rho, f_n, (s_o/rho)^n / rho and Dc level
// by level into the second of two shared-memory buffers, while the other
// seven warps contract source node k; every thread copies its share of node
// k + 1's moments into the second moment buffer with cp.async.  A
// contraction thread owns up to M2L2_MAXIT work items (local term b, a range
// of source terms a in graded order), the same items for every pair; per
// pair an item's sum (coef = (s_o/rho)^|b| / rho * f_|a| * Dc_(a+b) times
// the source row with the Yl correction folded in, Y_dj - R0_d m_j) is
// accumulated in registers and added to the item's slot in shared memory,
// which only that thread touches.  At the end the slots of each b are summed
// in a fixed order and scaled by 1 / b!.  One barrier per pair; registers
// stay under 80 so that three CTAs share an SM.
constexpr int M2L2_THREADS = 256;
constexpr int M2L2_TC = M2L2_THREADS - 32;  // contraction threads
constexpr int M2L2_MAXIT = 3;
constexpr int M2L2_MAXITEMS = M2L2_TC * M2L2_MAXIT;
struct M2LPlan2 {
    int n_items;
    int item[M2L2_MAXITEMS][8];   // b, g0, g1, a0, a2, |a| at g0, b0, b2
    int bstart[FMM_NTMAX + 1];    // items of term b: [bstart[b], bstart[b + 1])
    int tcnt[M2L2_TC];
    int titem[M2L2_TC][M2L2_MAXIT];
    int rec[FMM_NTMAX][8];        // Dc recurrence: a0, a1, a2 and the 5 used indices
};

// The plan: items cut term b's n_terms(p - |b|) source terms into near-equal
// chunks of at most CH = ceil(total / M2L2_TC) terms; the items, largest
// first, are dealt to the contraction threads in snake order.  One thread,
// written to the workspace each call.
__global__ void __launch_bounds__(32) fmm_m2l2_plan(int p, M2LPlan2* __restrict__ plan, int* err) {
    if (threadIdx.x != 0) return;
    const int NT = n_terms(p);
    const int total = n_terms6(p);
    const int CH = (total + M2L2_TC - 1) / M2L2_TC;
    int n = 0;
    for (int b = 0; b < NT; b++) {
        int b0, b1, b2;
        decode(b, b0, b1, b2);
        const int t = n_terms(p - (b0 + b1 + b2));
        const int nch = (t + CH - 1) / CH;
        plan->bstart[b] = n;
        for (int c = 0; c < nch; c++) {
            if (n >= M2L2_MAXITEMS) {
                *err = 1;
                return;
            }
            const int g0 = (int)((int64_t)t * c / nch), g1 = (int)((int64_t)t * (c + 1) / nch);
            int a0, a1, a2;
            decode(g0, a0, a1, a2);
            int* it = plan->item[n];
            it[0] = b; it[1] = g0; it[2] = g1; it[3] = a0; it[4] = a2; it[5] = a0 + a1 + a2;
            it[6] = b0; it[7] = b2;
            n++;
        }
    }
    plan->bstart[NT] = n;
    plan->n_items = n;
    // deal items by size, largest first (counting sort on sizes 1..CH), snake order
    for (int t = 0; t < M2L2_TC; t++) plan->tcnt[t] = 0;
    int dealt = 0;
    for (int sz = CH; sz >= 1; sz--)
        for (int i = 0; i < n; i++) {
            if (plan->item[i][2] - plan->item[i][1] != sz) continue;
            const int round = dealt / M2L2_TC, pos = dealt % M2L2_TC;
            const int th = (round & 1) ? M2L2_TC - 1 - pos : pos;
            if (plan->tcnt[th] >= M2L2_MAXIT) {
                *err = 1;
                return;
            }
            plan->titem[th][plan->tcnt[th]++] = i;
            dealt++;
        }
    // the Dc recurrence table
    for (int g = 0; g < NT; g++) {
        int a0, a1, a2;
        decode(g, a0, a1, a2);
        int* r = plan->rec[g];
        r[0] = a0; r[1] = a1; r[2] = a2;
        r[3] = a0 > 0 ? midx(a0 - 1, a1, a2) : 0;
        r[4] = a1 > 0 ? midx(a0, a1 - 1, a2) : 0;
        r[5] = a2 > 0 ? midx(a0, a1, a2 - 1) : 0;
        r[6] = a0 > 1 ? midx(a0 - 2, a1, a2) : 0;
        r[7] = 0;  // the a1 - 2 and a2 - 2 indices are recomputed (rare)
    }
}

// Number of plan items for order p (host mirror of fmm_m2l2_plan's cut).
inline int m2l2_items(int p) {
    const int total = n_terms6(p), CH = (total + M2L2_TC - 1) / M2L2_TC;
    int n = 0;
    for (int m = 0; m <= p; m++) {
        const int t = n_terms(p - m), cnt = (m + 1) * (m + 2) / 2;
        n += cnt * ((t + CH - 1) / CH);
    }
    return n;
}


template <typename R, int K>
__global__ void __launch_bounds__(M2L2_THREADS, 3)
fmm_m2l2(int p, const int64_t* __restrict__ obs_nodes, int64_t n_obs_nodes,
         const int64_t* __restrict__ starts, const int64_t* __restrict__ srcs,
         const R* __restrict__ ocent, const R* __restrict__ orad, const R* __restrict__ scent,
         const R* __restrict__ srad, const R* __restrict__ mom, const M2LPlan2* __restrict__ plan,
         R* __restrict__ loc) {
    using C = Chan<K>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NT = n_terms(p);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t oi = blockIdx.x;
    if (oi >= n_obs_nodes) return;
    const int rowsz = NT * C::NCHP;
    R* Nb = reinterpret_cast<R*>(smem_raw);  // 2 x NT x NCHP moments
    R* Db = Nb + 2 * rowsz;                  // 2 x NT Dc
    R* Sb = Db + 2 * ((NT + 3) / 4 * 4);     // 2 x 40: f_n [0, 16), pw_n [16, 32), R0 [32, 35)
    R* slots = Sb + 80;                      // n_items x NCHP item sums
    const int64_t node = obs_nodes[oi];
    const R co[3] = {ocent[3 * node], ocent[3 * node + 1], ocent[3 * node + 2]};
    const R so = orad[node];
    const int64_t l0 = starts[oi], l1 = starts[oi + 1];
    const int64_t npair = l1 - l0;

    auto issue_copy = [&](int64_t l, int buf) {
        const R* src = mom + srcs[l] * (int64_t)rowsz;
        R* dst = Nb + buf * rowsz;
        constexpr int PER = 16 / sizeof(R);
        for (int k = tid; k < rowsz / PER; k += M2L2_THREADS)
            cp_async16(dst + k * PER, src + k * PER);
        cp_async_commit();
    };
    auto produce = [&](int64_t l, int buf) {  // warp 0
        const int64_t sn = srcs[l];
        const R R0[3] = {co[0] - scent[3 * sn], co[1] - scent[3 * sn + 1],
                         co[2] - scent[3 * sn + 2]};
        const R rho = sqrt(R0[0] * R0[0] + R0[1] * R0[1] + R0[2] * R0[2]);
        const R inv_rho = R(1) / rho;
        const R Rh[3] = {R0[0] * inv_rho, R0[1] * inv_rho, R0[2] * inv_rho};
        R* S = Sb + buf * 40;
        R* D = Db + buf * ((NT + 3) / 4 * 4);
        if (lane <= p) {
            S[lane] = ((lane & 1) ? R(-1) : R(1)) * ipow(srad[sn] * inv_rho, lane);
            S[16 + lane] = ipow(so * inv_rho, lane) * inv_rho;
        }
        if (lane < 3) S[32 + lane] = R0[lane];
        if (lane == 0) D[0] = 1;
        __syncwarp();
        for (int n = 1; n <= p; n++) {
            const int lsz = (n + 1) * (n + 2) / 2, base = n_terms(n - 1);
            const R cA = -(R)(2 * n - 1) / (R)n, cB = -(R)(n - 1) / (R)n;
            for (int w = lane; w < lsz; w += 32) {
                const int* rr = plan->rec[base + w];
                const int a0 = rr[0], a1 = rr[1], a2 = rr[2];
                R s1 = 0, s2 = 0;
                if (a0 > 0) s1 += Rh[0] * (R)a0 * D[rr[3]];
                if (a1 > 0) s1 += Rh[1] * (R)a1 * D[rr[4]];
                if (a2 > 0) s1 += Rh[2] * (R)a2 * D[rr[5]];
                if (a0 > 1) s2 += (R)(a0 * (a0 - 1)) * D[rr[6]];
                if (a1 > 1) s2 += (R)(a1 * (a1 - 1)) * D[midx(a0, a1 - 2, a2)];
                if (a2 > 1) s2 += (R)(a2 * (a2 - 1)) * D[midx(a0, a1, a2 - 2)];
                D[base + w] = cA * s1 + cB * s2;
            }
            __syncwarp();
        }
    };

    // this thread's work items
    const int ct = tid - 32;
    int my_n = 0;
    int itid[M2L2_MAXIT], itg0[M2L2_MAXIT], itg1[M2L2_MAXIT], ita0[M2L2_MAXIT],
        ita2[M2L2_MAXIT], itna[M2L2_MAXIT], itb0[M2L2_MAXIT], itb2[M2L2_MAXIT],
        itnb[M2L2_MAXIT];
    if (warp > 0) {
        my_n = plan->tcnt[ct];
#pragma unroll
        for (int i = 0; i < M2L2_MAXIT; i++) {
            itid[i] = i < my_n ? plan->titem[ct][i] : 0;
            const int* it = plan->item[itid[i]];
            itg0[i] = it[1]; itg1[i] = it[2]; ita0[i] = it[3];
            ita2[i] = it[4]; itna[i] = it[5]; itb0[i] = it[6]; itb2[i] = it[7];
            int b0, b1, b2;
            decode(it[0], b0, b1, b2);
            itnb[i] = b0 + b1 + b2;
        }
    }
    const int n_items = plan->n_items;
    for (int e = tid; e < n_items * C::NCHP; e += M2L2_THREADS) slots[e] = 0;

    if (npair > 0) {
        issue_copy(l0, 0);
        if (warp == 0) produce(l0, 0);
    }
    for (int64_t k = 0; k < npair; k++) {
        const int buf = (int)(k & 1);
        cp_async_wait_all();
        __syncthreads();  // pair k's moments and Dc are complete; pair k - 1 is done
        if (k + 1 < npair) {
            issue_copy(l0 + k + 1, buf ^ 1);
            if (warp == 0) produce(l0 + k + 1, buf ^ 1);
        }
        if (warp == 0) continue;
        const R* S = Sb + buf * 40;
        const R* D = Db + buf * ((NT + 3) / 4 * 4);
        const R* N = Nb + buf * rowsz;
        const R R0[3] = {S[32], S[33], S[34]};
#pragma unroll 1
        for (int i = 0; i < M2L2_MAXIT; i++) {
            if (i >= my_n) break;
            R acc[C::NCH];
#pragma unroll
            for (int c = 0; c < C::NCH; c++) acc[c] = 0;
            const R sb = S[16 + itnb[i]];
            const int b0 = itb0[i], b2 = itb2[i];
            int a0 = ita0[i], a2 = ita2[i], na = itna[i];
            int nn = na + itnb[i];
            int rowbase = n_terms(nn - 1) + (nn - a0 - b0) * (nn - a0 - b0 + 1) / 2 + b2;
            R f = sb * S[na];
            for (int g = itg0[i]; g < itg1[i]; g++) {
                const R coef = f * D[rowbase + a2];
                const R* row = N + g * C::NCHP;
                R v[C::NCHP];
                if (sizeof(R) == 4) {
#pragma unroll
                    for (int k4 = 0; k4 < C::NCHP / 4; k4++) {
                        const float4 q = reinterpret_cast<const float4*>(row)[k4];
                        v[4 * k4] = (R)q.x; v[4 * k4 + 1] = (R)q.y;
                        v[4 * k4 + 2] = (R)q.z; v[4 * k4 + 3] = (R)q.w;
                    }
                } else {
#pragma unroll
                    for (int k2 = 0; k2 < C::NCHP / 2; k2++) {
                        const double2 q = reinterpret_cast<const double2*>(row)[k2];
                        v[2 * k2] = (R)q.x; v[2 * k2 + 1] = (R)q.y;
                    }
                }
#pragma unroll
                for (int d = 0; d < 3; d++)
#pragma unroll
                    for (int j = 0; j < C::J; j++)
                        v[C::CH_Y + d * C::J + j] -= R0[d] * v[C::CH_M + j];
#pragma unroll
                for (int c = 0; c < C::NCH; c++) acc[c] += coef * v[c];
                // next source term in graded order
                a2++;
                if (a2 > na - a0) {
                    a2 = 0;
                    a0--;
                    if (a0 < 0) {
                        na++;
                        a0 = na;
                        nn++;
                        f = sb * S[na];
                    }
                    rowbase = n_terms(nn - 1) + (nn - a0 - b0) * (nn - a0 - b0 + 1) / 2 + b2;
                }
            }
            R* sl = slots + itid[i] * C::NCHP;
#pragma unroll
            for (int c = 0; c < C::NCH; c++) sl[c] += acc[c];
        }
    }
    cp_async_wait_all();
    __syncthreads();
    R* Lg = loc + node * (int64_t)rowsz;
    for (int b = tid; b < NT; b += M2L2_THREADS) {
        int b0, b1, b2;
        decode(b, b0, b1, b2);
        const R inv = R(1) / mfact<R>(b0, b1, b2);
        R sum[C::NCH];
#pragma unroll
        for (int c = 0; c < C::NCH; c++) sum[c] = 0;
        for (int it = plan->bstart[b]; it < plan->bstart[b + 1]; it++)
#pragma unroll
            for (int c = 0; c < C::NCH; c++) sum[c] += slots[it * C::NCHP + c];
#pragma unroll
        for (int c = 0; c < C::NCHP; c++) Lg[b * C::NCHP + c] = c < C::NCH ? sum[c] * inv : R(0);
    }
}


// ---- L2L (FMM) -------------------------------------------------------------
// One block per obs node of one depth (parents final): loc[child] += shift of
// the parent's local expansion (with the Yl transform).
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_l2l(int p, const int64_t* __restrict__ nodes, const int64_t* __restrict__ parent,
        const R* __restrict__ ocent, const R* __restrict__ orad, R* __restrict__ loc) {
    using C = Chan<K>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NT = n_terms(p);
    R* Lp = reinterpret_cast<R*>(smem_raw);  // NT x NCHP
    R* bin = Lp + NT * C::NCHP;
    fill_binom(bin);
    const int64_t cn = nodes[blockIdx.x];
    const int64_t pn = parent[cn];
    const R del[3] = {ocent[3 * cn] - ocent[3 * pn], ocent[3 * cn + 1] - ocent[3 * pn + 1],
                      ocent[3 * cn + 2] - ocent[3 * pn + 2]};
    const R sp = orad[pn];
    const R dh[3] = {del[0] / sp, del[1] / sp, del[2] / sp};
    const R ratio = orad[cn] / sp;
    const R* src = loc + pn * (int64_t)C::NCHP * NT;
    for (int e = threadIdx.x; e < NT * C::NCHP; e += blockDim.x) {
        const int k = e % C::NCHP;
        R v = src[e];
        if (k >= C::CH_Y && k < C::CH_M) {
            const int o = k - C::CH_Y, d = o / C::J, j = o % C::J;
            v -= del[d] * src[(e - k) + C::CH_M + j];
        }
        Lp[e] = v;
    }
    __syncthreads();
    R* dst = loc + cn * (int64_t)C::NCHP * NT;
    for (int b = threadIdx.x; b < NT; b += blockDim.x) {
        int b0, b1, b2;
        decode(b, b0, b1, b2);
        const int nb = b0 + b1 + b2;
        R acc[C::NCH];
#pragma unroll
        for (int k = 0; k < C::NCH; k++) acc[k] = 0;
        R q0 = 1;
        for (int c0 = b0; c0 <= p; c0++) {
            R q1 = 1;
            for (int c1 = b1; c0 + c1 <= p; c1++) {
                R q2 = 1;
                for (int c2 = b2; c0 + c1 + c2 <= p; c2++) {
                    const R coef = BIN(c0, b0) * BIN(c1, b1) * BIN(c2, b2) * q0 * q1 * q2;
                    const R* lrow = Lp + midx(c0, c1, c2) * C::NCHP;
#pragma unroll
                    for (int k = 0; k < C::NCH; k++) acc[k] += coef * lrow[k];
                    q2 *= dh[2];
                }
                q1 *= dh[1];
            }
            q0 *= dh[0];
        }
        const R sc = ipow(ratio, nb);
#pragma unroll
        for (int k = 0; k < C::NCH; k++) dst[b * C::NCHP + k] += sc * acc[k];
    }
}

// ---- L2P (FMM) -------------------------------------------------------------
// One block per obs leaf; its local expansion staged in shared memory; a
// thread per target point.
template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_l2p(int p, Rule2D<R> rule, int nq, const int64_t* __restrict__ leaves,
        const int64_t* __restrict__ o_start, const int64_t* __restrict__ o_end,
        const R* __restrict__ ocent, const R* __restrict__ orad, const R* __restrict__ pts,
        const int32_t* __restrict__ obs_tris, const R* __restrict__ loc, R* __restrict__ F) {
    using C = Chan<K>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
    const int NT = n_terms(p);
    const int64_t node = leaves[blockIdx.x];
    const int64_t t0 = o_start[node] * nq, t1 = o_end[node] * nq;
    if (t0 == t1) return;
    stage(sm, loc + node * (int64_t)C::NCHP * NT, C::NCHP * NT);
    __syncthreads();
    const R inv_s = R(1) / orad[node];
    const R co[3] = {ocent[3 * node], ocent[3 * node + 1], ocent[3 * node + 2]};
    for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
        TriGeom<R> o;
        load_tri(o, pts, obs_tris, t / nq, 0, false, false);
        R x[3];
        target_point(o, rule, (int)(t % nq), x);
        const R xi[3] = {x[0] - co[0], x[1] - co[1], x[2] - co[2]};
        R pw[3][FMM_MAXP + 1];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            pw[d][0] = 1;
            for (int k = 1; k <= p; k++) pw[d][k] = pw[d][k - 1] * (xi[d] * inv_s);
        }
        R phi[C::NCH];
#pragma unroll
        for (int k = 0; k < C::NCH; k++) phi[k] = 0;
        int g = 0;
        for (int n = 0; n <= p; n++)
            for (int a0 = n; a0 >= 0; a0--)
                for (int a2 = 0; a2 <= n - a0; a2++, g++) {
                    const R mono = pw[0][a0] * pw[1][n - a0 - a2] * pw[2][a2];
                    const R* lrow = sm + g * C::NCHP;
#pragma unroll
                    for (int k = 0; k < C::NCH; k++) phi[k] += mono * lrow[k];
                }
        R acc[C::NO];
#pragma unroll
        for (int k = 0; k < C::NO; k++) acc[k] = 0;
        combine<R, K>(phi, xi, o.n, acc);
        R* f = F + t * C::NO;
#pragma unroll
        for (int k = 0; k < C::NO; k++) f[k] += acc[k];
    }
}

// ---- finish ------------------------------------------------------------------
// Per obs triangle (tree order): the P2P sums W plus the per-point far fields
// F brought to the same layout, then the direct farfield's obs-side epilogue;
// written to the triangle's original row, times scale.
template <typename R, int K, int NQ>
__global__ void __launch_bounds__(128)
fmm_finish(Rule2D<R> rule, const R* __restrict__ pts, const int32_t* __restrict__ obs_tris,
           int64_t n_obs, const int64_t* __restrict__ obs_orig, const R* __restrict__ W,
           const R* __restrict__ F, R scale, R* __restrict__ out, int accumulate) {
    using C = Chan<K>;
    constexpr int NA = NAcc<K, NQ>::n;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_obs) return;
    TriGeom<R> o;
    load_tri(o, pts, obs_tris, i, 0, false, K == kRH || K == kRA);
    R tot[NA];
#pragma unroll
    for (int k = 0; k < NA; k++) tot[k] = W[i * NA + k];
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        const R* f = F + (i * NQ + q) * C::NO;
        if (K == kRH) {
#pragma unroll
            for (int k = 0; k < 9; k++) tot[k] += rule.w[q] * f[k];
        } else if (K == kRA) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                tot[3 * q + d] += f[3 + d];
                tot[3 * NQ + d] += rule.w[q] * f[d];
            }
        } else {
#pragma unroll
            for (int d = 0; d < 3; d++) tot[3 * q + d] += f[d];
        }
    }
    R out9[9];
    far_epilogue<R, K, NQ>(rule, o, tot, out9);
    R* op = out + obs_orig[i] * 9;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const R v = scale * out9[k];
        op[k] = accumulate ? op[k] + v : v;
    }
}

// ---- host ------------------------------------------------------------------

inline size_t al256(size_t b) { return (b + 255) / 256 * 256; }

struct Sizes {
    size_t rec, mom, loc, plan, W, F, rec2;
};

// Whether the lane plan fits for (p, nb, lanes), decided on the host once.
inline bool m2l3_plan_fits(int p, int nb, int lanes) {
    static std::atomic<int> fits[FMM_MAXP + 1][16][8];  // 0 unknown, 1 yes, 2 no
    if (p < 0 || p > FMM_MAXP || nb < 1 || nb > 15 || lanes < 32 || lanes > M2L3_LANES ||
        lanes % 32)
        return false;
    std::atomic<int>& f = fits[p][nb][lanes / 32];
    int v = f.load(std::memory_order_relaxed);
    if (v == 0) {
        std::vector<unsigned char> buf(sizeof(M2LPlan3));
        v = m2l3_make_plan(p, nb, lanes, reinterpret_cast<M2LPlan3*>(buf.data())) == 0 ? 1 : 2;
        f.store(v, std::memory_order_relaxed);
    }
    return v == 1;
}

inline size_t m2l_plan_bytes() {
    return sizeof(M2LPlan2) > sizeof(M2LPlan3) ? sizeof(M2LPlan2) : sizeof(M2LPlan3);
}

// The packed P2P runs for elasticRH3 in FP32 with the 3-, 4- and 7-point rules.
template <typename R, int K, int NQ>
constexpr bool p2p_packed() {
    return sizeof(R) == 4 && K == kRH && (NQ == 3 || NQ == 4 || NQ == 7);
}

template <int K, int NQ>
Sizes sizes_for(size_t rs, int mode, int order, int64_t n_obs, int64_t n_src, int64_t n_obs_nodes,
                int64_t n_src_nodes) {
    using C = Chan<K>;
    Sizes s;
    s.rec = al256(rs * Rec<K, NQ>::LEN * (size_t)n_src);
    s.mom = al256(rs * C::NCHP * (size_t)n_terms(order) * n_src_nodes);
    s.loc = mode == 1 ? al256(rs * C::NCHP * (size_t)n_terms(order) * n_obs_nodes) : 0;
    s.plan = mode == 1 ? al256(m2l_plan_bytes()) + 256 : 0;
    s.W = al256(rs * NAcc<K, NQ>::n * (size_t)n_obs);
    s.F = al256(rs * C::NO * (size_t)NQ * n_obs);
    s.rec2 = (rs == 4 && K == kRH && (NQ == 3 || NQ == 4 || NQ == 7))
                 ? al256(4 * (size_t)RecRH2<NQ>::LEN * n_src)
                 : 0;
    return s;
}

bool supported_kernel(int k) { return k == kU || k == kRT || k == kRA || k == kRH; }
bool supported_nq(int nq) { return nq == 3 || nq == 4 || nq == 7 || nq == 13; }

Sizes sizes_dispatch(int kernel, int prec, int mode, int order, int nq, int64_t n_obs,
                     int64_t n_src, int64_t n_obs_nodes, int64_t n_src_nodes) {
    const size_t rs = prec == TCT_F64 ? 8 : 4;
#define TCT_SZ_NQ(KID, NQV) \
    if (nq == NQV) return sizes_for<KID, NQV>(rs, mode, order, n_obs, n_src, n_obs_nodes, n_src_nodes);
#define TCT_SZ_K(KID)      \
    if (kernel == KID) {   \
        TCT_SZ_NQ(KID, 3)  \
        TCT_SZ_NQ(KID, 4)  \
        TCT_SZ_NQ(KID, 7)  \
        TCT_SZ_NQ(KID, 13) \
    }
    TCT_SZ_K(kU)
    TCT_SZ_K(kRT)
    TCT_SZ_K(kRA)
    TCT_SZ_K(kRH)
#undef TCT_SZ_K
#undef TCT_SZ_NQ
    return Sizes{0, 0, 0, 0, 0, 0, 0};
}

template <typename KF>
int set_smem(KF kfn, size_t smem) {
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
        return launch_status("fmm shared-memory attribute");
    return TCT_OK;
}

// Per host thread and device: the high-priority stream that runs the
// expansion stages next to P2P, and the fork / join events (created once,
// kept for the process).
struct SideStream {
    int dev = -1;
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
inline SideStream* side_stream() {
    static thread_local SideStream tab[16];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 16) return nullptr;
    SideStream& e = tab[dev];
    if (e.dev != dev) {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
            cudaStreamCreateWithPriority(&e.s, cudaStreamNonBlocking, greatest) != cudaSuccess ||
            cudaEventCreateWithFlags(&e.fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&e.join, cudaEventDisableTiming) != cudaSuccess)
            return nullptr;
        e.dev = dev;
    }
    return &e;
}

template <typename R, int K, int NQ>
int run_fmm(int mode, int p, const Rule2D<R>& rule, const double* params, double scale,
            const R* obs_pts, const int32_t* obs_tris, int64_t n_obs, const tct_fmm_tree& ot,
            const R* src_pts, const int32_t* src_tris, int64_t n_src, const tct_fmm_tree& stt,
            const tct_fmm_list& near, const tct_fmm_list& far, const R* in, R* out,
            int accumulate, unsigned char* ws, cudaStream_t st) {
    using C = Chan<K>;
    constexpr int NA = NAcc<K, NQ>::n;
    const Consts<R> c = make_consts<R>(params);
    const int NT = n_terms(p);
    const Sizes sz = sizes_for<K, NQ>(sizeof(R), mode, p, n_obs, n_src, ot.n_nodes, stt.n_nodes);
    R* rec = reinterpret_cast<R*>(ws);
    R* mom = reinterpret_cast<R*>(ws + sz.rec);
    R* loc = reinterpret_cast<R*>(ws + sz.rec + sz.mom);
    unsigned char* plan = ws + sz.rec + sz.mom + sz.loc;
    R* W = reinterpret_cast<R*>(ws + sz.rec + sz.mom + sz.loc + sz.plan);
    R* F = reinterpret_cast<R*>(ws + sz.rec + sz.mom + sz.loc + sz.plan + sz.W);
    float* rec2 = reinterpret_cast<float*>(ws + sz.rec + sz.mom + sz.loc + sz.plan + sz.W + sz.F);
    bool uniform = true;
    for (int q = 1; q < NQ; q++) uniform = uniform && (rule.w[q] == rule.w[0]);
    const R* scent = (const R*)stt.centers;
    const R* srad = (const R*)stt.radii;
    const R* ocent = (const R*)ot.centers;
    const R* orad = (const R*)ot.radii;
    int rc;
    if (n_src > 0) {
        far_prep<R, K, NQ><<<(unsigned)((n_src + 127) / 128), 128, 0, st>>>(
            c, rule, src_pts, src_tris, n_src, in, stt.orig, rec);
        if ((rc = launch_status("fmm prep"))) return rc;
    }
    if (cudaMemsetAsync(W, 0, sizeof(R) * NA * (size_t)n_obs, st) != cudaSuccess ||
        cudaMemsetAsync(F, 0, sizeof(R) * C::NO * (size_t)NQ * n_obs, st) != cudaSuccess)
        return launch_status("fmm memset");
    // The expansion stages (P2M .. L2P) run on a second, high-priority
    // stream next to P2P: as P2P blocks retire the scheduler hands their SMs
    // to M2L blocks first, so the FMA-bound P2P and the shared-memory-bound
    // M2L share SMs instead of running back to back; joined before fmm_finish
    SideStream* side = side_stream();
    if (!side) return launch_status("fmm side stream");
    const cudaStream_t sp = st;       // P2P
    const cudaStream_t se = side->s;  // expansions
    if (cudaEventRecord(side->fork, st) != cudaSuccess ||
        cudaStreamWaitEvent(se, side->fork, 0) != cudaSuccess)
        return launch_status("fmm fork");
    if (near.n_obs > 0) {
        if constexpr (p2p_packed<R, K, NQ>()) {
            const Rule2D<float>& rf = rule;
            const unsigned pb = (unsigned)((n_src + 127) / 128);
            const size_t smem = p2p_rh2_smem<NQ>();
            if ((rc = set_smem(fmm_p2p_rh2<NQ, true>, smem)) ||
                (rc = set_smem(fmm_p2p_rh2<NQ, false>, smem)))
                return rc;
            if (uniform) {
                far_prep_rh2<NQ, true><<<pb, 128, 0, sp>>>(c, rf, (const float*)src_pts,
                                                            src_tris, n_src, (const float*)in,
                                                            stt.orig, rec2);
                if ((rc = launch_status("fmm prep (packed)"))) return rc;
                fmm_p2p_rh2<NQ, true><<<(unsigned)near.n_obs, 128, smem, sp>>>(
                    rf, (const float*)obs_pts, obs_tris, near.obs, near.start, near.src, ot.start,
                    ot.end, stt.start, stt.end, rec2, (float*)W);
            } else {
                far_prep_rh2<NQ, false><<<pb, 128, 0, sp>>>(c, rf, (const float*)src_pts,
                                                             src_tris, n_src, (const float*)in,
                                                             stt.orig, rec2);
                if ((rc = launch_status("fmm prep (packed)"))) return rc;
                fmm_p2p_rh2<NQ, false><<<(unsigned)near.n_obs, 128, smem, sp>>>(
                    rf, (const float*)obs_pts, obs_tris, near.obs, near.start, near.src, ot.start,
                    ot.end, stt.start, stt.end, rec2, (float*)W);
            }
            if ((rc = launch_status("fmm p2p (packed)"))) return rc;
        } else {
            const size_t smem = sizeof(R) * 128 * NA;
            if ((rc = set_smem(fmm_p2p<R, K, NQ>, smem))) return rc;
            fmm_p2p<R, K, NQ><<<(unsigned)near.n_obs, 128, smem, sp>>>(
                c, rule, obs_pts, obs_tris, near.obs, near.start, near.src, ot.start, ot.end,
                stt.start, stt.end, rec, W);
            if ((rc = launch_status("fmm p2p"))) return rc;
        }
    }
    if (stt.n_leaves > 0) {
        fmm_p2m<R, K, NQ><<<(unsigned)stt.n_leaves, 128, 0, se>>>(
            c, p, stt.leaves, stt.start, stt.end, scent, srad, rec, mom);
        if ((rc = launch_status("fmm p2m"))) return rc;
    }
    for (int h = 0; h < stt.n_levels; h++) {
        const int64_t cnt = stt.level_offsets[h + 1] - stt.level_offsets[h];
        if (cnt == 0) continue;
        fmm_m2m<R, K><<<(unsigned)cnt, 128, 0, se>>>(p, stt.levels + stt.level_offsets[h],
                                                     stt.children, scent, srad, mom);
        if ((rc = launch_status("fmm m2m"))) return rc;
    }
    if (mode == 0) {
        if (far.n_obs > 0) {
            const size_t smem = sizeof(R) * (size_t)C::NCHP * NT;
            if ((rc = set_smem(fmm_m2p<R, K>, smem))) return rc;
            fmm_m2p<R, K><<<(unsigned)far.n_obs, 128, smem, se>>>(
                p, rule, NQ, far.obs, far.start, far.src, ot.start, ot.end, scent, srad, obs_pts,
                obs_tris, mom, F);
            if ((rc = launch_status("fmm m2p"))) return rc;
        }
    } else {
        if (cudaMemsetAsync(loc, 0, sz.loc, se) != cudaSuccess) return launch_status("fmm memset");
        if (far.n_obs > 0) {
            const int64_t n_el = stt.n_nodes * (int64_t)NT * C::NCHP;
            fmm_moment_factorials<R><<<(unsigned)((n_el + 127) / 128), 128, 0, se>>>(
                p, C::NCHP, stt.n_nodes, mom);
            if ((rc = launch_status("fmm moment factorials"))) return rc;
            bool lanes = false;  // the lane plan (fmm_m2l3) for FP32
            int* plan_err = reinterpret_cast<int*>(plan + al256(m2l_plan_bytes()));
            if constexpr (sizeof(R) == 4) {
                const int smem1 = m2l3_smem<K>(p, 1).total_bytes;
                const int smem2 = m2l3_smem<K>(p, 2).total_bytes;
                // two pairs per stage while two CTAs still fit an SM
                const bool two = smem2 + 1024 <= 113 * 1024;
                const int nl = two ? m2l3_lanes(2) : m2l3_lanes(1);
                lanes = m2l3_plan_fits(p, M2L3Cfg<K>::NB, nl) && smem1 <= 227 * 1024;
                if (lanes) {
                    M2LPlan3* plan3 = reinterpret_cast<M2LPlan3*>(plan);
                    fmm_m2l3_plan<<<1, 32, 0, se>>>(p, M2L3Cfg<K>::NB, nl, plan3, plan_err);
                    if ((rc = launch_status("fmm m2l plan"))) return rc;
                    if (two) {
                        if ((rc = set_smem(fmm_m2l3<K, 2>, (size_t)smem2))) return rc;
                        fmm_m2l3<K, 2><<<(unsigned)far.n_obs, M2L3_THREADS, smem2, se>>>(
                            p, far.obs, far.n_obs, far.start, far.src, ocent, orad, scent, srad,
                            mom, plan3, loc);
                    } else {
                        if ((rc = set_smem(fmm_m2l3<K, 1>, (size_t)smem1))) return rc;
                        fmm_m2l3<K, 1><<<(unsigned)far.n_obs, M2L3_THREADS, smem1, se>>>(
                            p, far.obs, far.n_obs, far.start, far.src, ocent, orad, scent, srad,
                            mom, plan3, loc);
                    }
                }
            }
            if (!lanes) {
                if (m2l2_items(p) > M2L2_MAXITEMS) {
                    set_error("tct_fmm_matvec: FMM order %d exceeds the M2L plan's capacity", p);
                    return TCT_ERR_ARG;
                }
                M2LPlan2* plan2 = reinterpret_cast<M2LPlan2*>(plan);
                fmm_m2l2_plan<<<1, 32, 0, se>>>(p, plan2, plan_err);
                if ((rc = launch_status("fmm m2l plan"))) return rc;
                const size_t smem_all = sizeof(R) * (2 * (size_t)NT * C::NCHP +
                                                     2 * (size_t)((NT + 3) / 4 * 4) + 80 +
                                                     (size_t)m2l2_items(p) * C::NCHP);
                if (smem_all > 227 * 1024) {
                    // FP64 at p = 12 needs 286 KB (p = 10: 190 KB)
                    set_error("tct_fmm_matvec: the item-form M2L at order %d needs %zu bytes of "
                              "shared memory (the limit is 227 KB; FP64 runs orders up to 10)",
                              p, smem_all);
                    return TCT_ERR_ARG;
                }
                if ((rc = set_smem(fmm_m2l2<R, K>, smem_all))) return rc;
                fmm_m2l2<R, K><<<(unsigned)far.n_obs, M2L2_THREADS, smem_all, se>>>(
                    p, far.obs, far.n_obs, far.start, far.src, ocent, orad, scent, srad, mom,
                    plan2, loc);
            }
            if ((rc = launch_status("fmm m2l"))) return rc;
        }
        const size_t smem_l2l =
            sizeof(R) * ((size_t)C::NCHP * NT + (FMM_MAXP + 1) * (FMM_MAXP + 1));
        if ((rc = set_smem(fmm_l2l<R, K>, smem_l2l))) return rc;
        for (int d = 0; d < ot.n_levels; d++) {
            const int64_t cnt = ot.level_offsets[d + 1] - ot.level_offsets[d];
            if (cnt == 0) continue;
            fmm_l2l<R, K><<<(unsigned)cnt, 128, smem_l2l, se>>>(
                p, ot.levels + ot.level_offsets[d], ot.parent, ocent, orad, loc);
            if ((rc = launch_status("fmm l2l"))) return rc;
        }
        if (ot.n_leaves > 0) {
            const size_t smem = sizeof(R) * (size_t)C::NCHP * NT;
            if ((rc = set_smem(fmm_l2p<R, K>, smem))) return rc;
            fmm_l2p<R, K><<<(unsigned)ot.n_leaves, 128, smem, se>>>(
                p, rule, NQ, ot.leaves, ot.start, ot.end, ocent, orad, obs_pts, obs_tris, loc, F);
            if ((rc = launch_status("fmm l2p"))) return rc;
        }
    }
    if (cudaEventRecord(side->join, se) != cudaSuccess ||
        cudaStreamWaitEvent(st, side->join, 0) != cudaSuccess)
        return launch_status("fmm join");
    fmm_finish<R, K, NQ><<<(unsigned)((n_obs + 127) / 128), 128, 0, st>>>(
        rule, obs_pts, obs_tris, n_obs, ot.orig, W, F, (R)scale, out, accumulate);
    return launch_status("fmm finish");
}

}  // namespace
}  // namespace tct

using namespace tct;

extern "C" size_t tct_fmm_workspace_bytes(int kernel, int prec, int mode, int order, int n_q,
                                          int64_t n_obs, int64_t n_src, int64_t n_obs_nodes,
                                          int64_t n_src_nodes) {
    if (!supported_kernel(kernel) || !supported_nq(n_q) || order < 0 || order > FMM_MAXP ||
        (mode != 0 && mode != 1) || (prec != TCT_F32 && prec != TCT_F64))
        return 0;
    const Sizes s = sizes_dispatch(kernel, prec, mode, order, n_q, n_obs, n_src, n_obs_nodes,
                                   n_src_nodes);
    return s.rec + s.mom + s.loc + s.plan + s.W + s.F + s.rec2;
}

extern "C" int tct_fmm_matvec(int kernel, int prec, int mode, int order, int n_q,
                              const double* quad_pts, const double* quad_wts,
                              const double* params, double out_scale, const void* obs_pts,
                              const int32_t* obs_tris, int64_t n_obs,
                              const tct_fmm_tree* obs_tree, const void* src_pts,
                              const int32_t* src_tris, int64_t n_src,
                              const tct_fmm_tree* src_tree, const tct_fmm_list* p2p,
                              const tct_fmm_list* far, const void* in, void* out, int accumulate,
                              void* workspace, size_t workspace_bytes, void* stream) {
    TCT_CHECK_ARG(order >= 0 && order <= FMM_MAXP, "tct_fmm_matvec: order must be 0..%d",
                  FMM_MAXP);
    TCT_CHECK_ARG(mode == 0 || mode == 1, "tct_fmm_matvec: mode must be 0 (treecode) or 1 (fmm)");
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_fmm_matvec: negative size");
    TCT_CHECK_ARG(obs_tree && src_tree && p2p && far && params && quad_pts && quad_wts,
                  "tct_fmm_matvec: null argument");
    if (!supported_kernel(kernel)) {
        set_error("tct_fmm_matvec: kernel %d has no treecode (supported: elasticU3, "
                  "elasticRT3, elasticRA3, elasticRH3)",
                  kernel);
        return TCT_ERR_KERNEL;
    }
    if (prec != TCT_F32 && prec != TCT_F64) {
        set_error("tct_fmm_matvec: unsupported precision %d", prec);
        return TCT_ERR_PREC;
    }
    TCT_CHECK_ARG(supported_nq(n_q), "tct_fmm_matvec: n_q must be 3, 4, 7 or 13 (got %d)", n_q);
    if (n_obs == 0) return TCT_OK;
    const size_t need = tct_fmm_workspace_bytes(kernel, prec, mode, order, n_q, n_obs, n_src,
                                                obs_tree->n_nodes, src_tree->n_nodes);
    TCT_CHECK_ARG(workspace && workspace_bytes >= need && aligned(workspace, 256),
                  "tct_fmm_matvec: workspace of %zu bytes (256-aligned) required", need);
    unsigned char* ws = reinterpret_cast<unsigned char*>(workspace);
    cudaStream_t st = as_stream(stream);
#define TCT_FMM_NQ(R, KID, NQV)                                                                \
    if (n_q == NQV) {                                                                         \
        Rule2D<R> rule;                                                                       \
        for (int q = 0; q < MAXQ; q++) {                                                      \
            rule.x[q] = q < NQV ? (R)quad_pts[2 * q] : R(0);                                  \
            rule.y[q] = q < NQV ? (R)quad_pts[2 * q + 1] : R(0);                              \
            rule.w[q] = q < NQV ? (R)quad_wts[q] : R(0);                                      \
        }                                                                                     \
        return run_fmm<R, KID, NQV>(mode, order, rule, params, out_scale, (const R*)obs_pts, \
                                    obs_tris, n_obs, *obs_tree, (const R*)src_pts, src_tris,  \
                                    n_src, *src_tree, *p2p, *far, (const R*)in, (R*)out,      \
                                    accumulate, ws, st);                                      \
    }
#define TCT_FMM_K(R, KID)      \
    if (kernel == KID) {       \
        TCT_FMM_NQ(R, KID, 3)  \
        TCT_FMM_NQ(R, KID, 4)  \
        TCT_FMM_NQ(R, KID, 7)  \
        TCT_FMM_NQ(R, KID, 13) \
    }
    if (prec == TCT_F64) {
        TCT_FMM_K(double, kU)
        TCT_FMM_K(double, kRT)
        TCT_FMM_K(double, kRA)
        TCT_FMM_K(double, kRH)
    } else {
        TCT_FMM_K(float, kU)
        TCT_FMM_K(float, kRT)
        TCT_FMM_K(float, kRA)
        TCT_FMM_K(float, kRH)
    }
#undef TCT_FMM_K
#undef TCT_FMM_NQ
    set_error("tct_fmm_matvec: unsupported kernel %d / n_q %d", kernel, n_q);
    return TCT_ERR_ARG;
}

// Host-side check of the M2L work plan for order p, nb terms b per lane and
// `lanes` contraction lanes (192 with two-pair stages, 224 with one-pair ones):
// out[0] = valid (a, b) pairs covered, out[1] = pairs covered more than once
// or invalid and unmasked, out[2] = the chunk length L, out[3] = lanes used,
// out[4] = the sum over warps of their step counts.  Returns 0, or 1 when the
// plan does not fit.
extern "C" int tct_fmm_m2l_plan_stats(int order, int nb, int lanes, int64_t* out) {
    if (order < 0 || order > FMM_MAXP || nb < 1 || !out) return TCT_ERR_ARG;
    M2LPlan3* plan = new M2LPlan3();
    const int rc = m2l3_make_plan(order, nb, lanes, plan);
    if (rc) {
        delete plan;
        return 1;
    }
    const int NT = n_terms(order);
    std::vector<int> seen((size_t)NT * NT, 0);
    int64_t covered = 0, bad = 0;
    for (int l = 0; l < M2L3_LANES; l++) {
        const int k = plan->lane_k[l];
        if (k < 0) continue;
        for (int s = 0; s < plan->lane_cnt[l]; s++) {
            const int a = plan->lane_a0[l] + s;
            const int la = plan->ainfo[a] >> 16;
            for (int j = 0; j < nb; j++) {
                const int b = k * nb + j;
                if (b >= NT) continue;
                int b0, b1, b2;
                decode(b, b0, b1, b2);
                if (la + b0 + b1 + b2 > order) continue;  // masked in the kernel
                if (seen[(size_t)a * NT + b]++) bad++;
                else covered++;
            }
        }
    }
    // a lane's steps may not exceed its warp's count
    int64_t steps = 0;
    for (int w = 0; w < lanes / 32; w++) {
        steps += plan->warp_steps[w];
        for (int l = 32 * w; l < 32 * w + 32; l++)
            if (plan->lane_cnt[l] > plan->warp_steps[w]) bad++;
    }
    out[0] = covered;
    out[1] = bad;
    out[2] = plan->L;
    out[3] = plan->n_lanes;
    out[4] = steps;
    delete plan;
    return 0;
}

