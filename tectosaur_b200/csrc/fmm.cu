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
__device__ __forceinline__ int midx(int a0, int a1, int a2) {
    const int n = a0 + a1 + a2;
    return n * (n + 1) * (n + 2) / 6 + (n - a0) * (n - a0 + 1) / 2 + a2;
}
// position of (a0, ., a2) within level n
__device__ __forceinline__ int lidx(int n, int a0, int a2) { return (n - a0) * (n - a0 + 1) / 2 + a2; }

__device__ __forceinline__ void decode(int g, int& a0, int& a1, int& a2) {
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

// ---- P2P -------------------------------------------------------------------
// One block per obs leaf with a non-empty P2P list.  The leaf's m obs
// triangles take m threads; the block's 128 threads form 128 / m groups that
// take the listed source leaves round-robin, each thread running the direct
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
            for (int64_t l = l0 + grp; l < l1; l += G) {
                const int64_t sn = srcs[l];
                R acc[NA];
#pragma unroll
                for (int k = 0; k < NA; k++) acc[k] = 0;
                const int64_t e = s_end[sn];
                for (int64_t s = s_start[sn]; s < e; s++)
                    far_pair<R, K, NQ>(c, rule, o, x, rec + s * L::LEN, acc);
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
// pair's source moments are used as stored.  One warp per obs node walks its
// M2L list; per pair the lanes copy the source node's moments into the warp's
// shared memory and build Dc level by level there (warp syncs only), then
// lane l contracts the local terms b dealt to it in snake order (b = 32k + l,
// 32k + 31 - l, ... balances the trip counts, which fall with |b|), reading
// the moment rows as shared-memory broadcasts.  The
// pair's sums get the Yl correction (- R0_d times the m channel) and the b
// scaling, and are added to the warp's local expansion in shared memory.
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

// Lane plan of the M2L contraction for order p (one warp, written to the
// workspace each call).  The work of local term b is n_terms(p - |b|)
// source terms; terms are cut into chunks of at most CH = ceil(total / 32)
// iterations and the chunks are dealt, in order, to the lane with the least
// work so far (ties to the lowest lane), so every lane runs about CH
// iterations.  A term cut into several chunks gets consecutive partial slots,
// summed in a fixed order after the contraction (deterministic results).
constexpr int M2L_MAXI = 32;   // chunks per lane (15 at most for p <= 12)
constexpr int M2L_SLOTS = 32;  // partial slots (31 at most for p <= 12)
struct M2LPlan {
    int item[32][M2L_MAXI][4];  // b, first, end (graded source-term range), slot or -1
    int cnt[32];
    int split[M2L_SLOTS][3];    // b, first slot, end slot
    int nsplit;
};

__global__ void __launch_bounds__(32) fmm_m2l_plan(int p, M2LPlan* __restrict__ plan) {
    const int lane = threadIdx.x;
    const int NT = n_terms(p);
    const int CH = (n_terms6(p) + 31) / 32;
    int load = 0, cnt = 0, slot = 0, nsplit = 0;
    for (int b = 0; b < NT; b++) {
        int b0, b1, b2;
        decode(b, b0, b1, b2);
        const int t = n_terms(p - (b0 + b1 + b2));
        const int nch = (t + CH - 1) / CH;
        const bool split = nch > 1 && slot + nch <= M2L_SLOTS;
        const int step = split ? CH : t;
        for (int c = 0, g0 = 0; g0 < t; c++, g0 += step) {
            const int g1 = min(t, g0 + step);
            const unsigned key = ((unsigned)load << 5) | (unsigned)lane;
            const unsigned win = __reduce_min_sync(0xffffffffu, key) & 31u;
            if ((unsigned)lane == win && cnt < M2L_MAXI) {
                plan->item[lane][cnt][0] = b;
                plan->item[lane][cnt][1] = g0;
                plan->item[lane][cnt][2] = g1;
                plan->item[lane][cnt][3] = split ? slot + c : -1;
                cnt++;
                load += g1 - g0;
            }
        }
        if (split) {
            if (lane == 0) {
                plan->split[nsplit][0] = b;
                plan->split[nsplit][1] = slot;
                plan->split[nsplit][2] = slot + nch;
            }
            slot += nch;
            nsplit++;
        }
    }
    plan->cnt[lane] = cnt;
    if (lane == 0) plan->nsplit = nsplit;
}

template <typename R, int K>
__device__ __forceinline__ void m2l_flush(R (&acc)[Chan<K>::NCH], const R R0[3], R sc, R* lrow) {
    using C = Chan<K>;
    // Yl = Y - R0_d m; scaled add into the warp's local expansion
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
        for (int j = 0; j < C::J; j++) acc[C::CH_Y + d * C::J + j] -= R0[d] * acc[C::CH_M + j];
#pragma unroll
    for (int k = 0; k < C::NCH; k++) lrow[k] += sc * acc[k];
}

template <typename R>
__device__ __forceinline__ R mfact(int b0, int b1, int b2) {
    R f = 1;
    for (int k = 2; k <= b0; k++) f *= (R)k;
    for (int k = 2; k <= b1; k++) f *= (R)k;
    for (int k = 2; k <= b2; k++) f *= (R)k;
    return f;
}

template <typename R, int K>
__global__ void __launch_bounds__(128)
fmm_m2l(int p, int wpb, const int64_t* __restrict__ obs_nodes, int64_t n_obs_nodes,
        const int64_t* __restrict__ starts, const int64_t* __restrict__ srcs,
        const R* __restrict__ ocent, const R* __restrict__ orad, const R* __restrict__ scent,
        const R* __restrict__ srad, const R* __restrict__ mom, const M2LPlan* __restrict__ plan,
        R* __restrict__ loc) {
    using C = Chan<K>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NT = n_terms(p);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t oi = (int64_t)blockIdx.x * wpb + warp;
    if (warp >= wpb || oi >= n_obs_nodes) return;  // whole warps only: no block barriers below
    // per-warp segment: Lw, Ns (NT x NCHP each), partial slots, Dc, fw, pw;
    // padded to 4 Reals so that every warp's Ns stays 16-byte aligned
    const int seg = (2 * NT + M2L_SLOTS) * C::NCHP + (NT + 32 + 3) / 4 * 4;
    R* Lw = reinterpret_cast<R*>(smem_raw) + (size_t)warp * seg;
    R* Ns = Lw + NT * C::NCHP;        // the current source node's moments
    R* Ps = Ns + NT * C::NCHP;        // partial sums of split terms
    R* Dc = Ps + M2L_SLOTS * C::NCHP;  // NT
    R* fw = Dc + NT;                  // f_n, n <= p
    R* pw = fw + 16;                  // (s_o/rho)^n / rho
    for (int e = lane; e < NT * C::NCHP; e += 32) Lw[e] = 0;
    const int mycnt = plan->cnt[lane];
    const int nsplit = plan->nsplit;
    const int64_t node = obs_nodes[oi];
    const R co[3] = {ocent[3 * node], ocent[3 * node + 1], ocent[3 * node + 2]};
    const R so = orad[node];
    for (int64_t l = starts[oi]; l < starts[oi + 1]; l++) {
        const int64_t sn = srcs[l];
        const R R0[3] = {co[0] - scent[3 * sn], co[1] - scent[3 * sn + 1], co[2] - scent[3 * sn + 2]};
        const R rho = sqrt(R0[0] * R0[0] + R0[1] * R0[1] + R0[2] * R0[2]);
        const R inv_rho = R(1) / rho;
        const R Rh[3] = {R0[0] * inv_rho, R0[1] * inv_rho, R0[2] * inv_rho};
        __syncwarp();  // the previous pair's readers are done
        if (lane <= p) {
            fw[lane] = ((lane & 1) ? R(-1) : R(1)) * ipow(srad[sn] * inv_rho, lane);
            pw[lane] = ipow(so * inv_rho, lane) * inv_rho;
        } else if (lane < 16) {
            fw[lane] = 0;
            pw[lane] = 0;
        }
        if (lane == 0) Dc[0] = 1;
        {
            const R* Ms = mom + sn * (int64_t)C::NCHP * NT;
            if (sizeof(R) == 4) {
                const float4* sv = reinterpret_cast<const float4*>(Ms);
                float4* dv = reinterpret_cast<float4*>(Ns);
                for (int k = lane; k < NT * C::NCHP / 4; k += 32) dv[k] = __ldg(sv + k);
            } else {
                const double2* sv = reinterpret_cast<const double2*>(Ms);
                double2* dv = reinterpret_cast<double2*>(Ns);
                for (int k = lane; k < NT * C::NCHP / 2; k += 32) dv[k] = __ldg(sv + k);
            }
        }
        __syncwarp();
        for (int n = 1; n <= p; n++) {
            const int lsz = (n + 1) * (n + 2) / 2;
            const R cA = -(R)(2 * n - 1) / (R)n, cB = -(R)(n - 1) / (R)n;
            for (int w = lane; w < lsz; w += 32) {
                int a0 = n, off = 0;
                while (off + (n - a0 + 1) <= w) {
                    off += n - a0 + 1;
                    a0--;
                }
                const int a2 = w - off, a1 = n - a0 - a2;
                R s1 = 0, s2 = 0;
                if (a0 > 0) s1 += Rh[0] * (R)a0 * Dc[midx(a0 - 1, a1, a2)];
                if (a1 > 0) s1 += Rh[1] * (R)a1 * Dc[midx(a0, a1 - 1, a2)];
                if (a2 > 0) s1 += Rh[2] * (R)a2 * Dc[midx(a0, a1, a2 - 1)];
                if (a0 > 1) s2 += (R)(a0 * (a0 - 1)) * Dc[midx(a0 - 2, a1, a2)];
                if (a1 > 1) s2 += (R)(a1 * (a1 - 1)) * Dc[midx(a0, a1 - 2, a2)];
                if (a2 > 1) s2 += (R)(a2 * (a2 - 1)) * Dc[midx(a0, a1, a2 - 2)];
                Dc[n_terms(n - 1) + w] = cA * s1 + cB * s2;
            }
            __syncwarp();
        }
        // flat loop over this lane's chunks: every lane runs ~CH iterations
        int k = 0;
        int b = 0, b0 = 0, b1 = 0, b2 = 0, g = 0, g1 = 0, slot = -1, na = 0, a0 = 0, a2 = 0,
            n = 0, rowbase = 0;
        R f = 0;
        R acc[C::NCH];
        while (k < mycnt) {
            if (g == g1) {  // start chunk k
                b = plan->item[lane][k][0];
                g = plan->item[lane][k][1];
                g1 = plan->item[lane][k][2];
                slot = plan->item[lane][k][3];
                decode(b, b0, b1, b2);
                int a1;
                decode(g, a0, a1, a2);
                na = a0 + a1 + a2;
                n = na + b0 + b1 + b2;
                rowbase = n_terms(n - 1) + (n - a0 - b0) * (n - a0 - b0 + 1) / 2 + b2;
                f = fw[na];
#pragma unroll
                for (int c = 0; c < C::NCH; c++) acc[c] = 0;
            }
            const R coef = f * Dc[rowbase + a2];
            const R* nrow = Ns + g * C::NCHP;
            if (sizeof(R) == 4) {
#pragma unroll
                for (int k4 = 0; k4 < C::NCHP / 4; k4++) {
                    const float4 v = reinterpret_cast<const float4*>(nrow)[k4];
                    const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        if (4 * k4 + u < C::NCH) acc[4 * k4 + u] += coef * (R)vv[u];
                }
            } else {
#pragma unroll
                for (int k2 = 0; k2 < C::NCHP / 2; k2++) {
                    const double2 v = reinterpret_cast<const double2*>(nrow)[k2];
                    if (2 * k2 < C::NCH) acc[2 * k2] += coef * (R)v.x;
                    if (2 * k2 + 1 < C::NCH) acc[2 * k2 + 1] += coef * (R)v.y;
                }
            }
            // next source term in graded order
            g++;
            a2++;
            if (a2 > na - a0) {
                a2 = 0;
                a0--;
                if (a0 < 0) {
                    na++;
                    a0 = na;
                    n++;
                    f = fw[na];
                }
                rowbase = n_terms(n - 1) + (n - a0 - b0) * (n - a0 - b0 + 1) / 2 + b2;
            }
            if (g == g1) {  // end of chunk k
                if (slot < 0) {
                    m2l_flush<R, K>(acc, R0, pw[b0 + b1 + b2] / mfact<R>(b0, b1, b2),
                                    Lw + b * C::NCHP);
                } else {
#pragma unroll
                    for (int c = 0; c < C::NCH; c++) Ps[slot * C::NCHP + c] = acc[c];
                }
                k++;
            }
        }
        __syncwarp();
        for (int j = lane; j < nsplit; j += 32) {
            const int bs = plan->split[j][0];
            int c0, c1, c2;
            decode(bs, c0, c1, c2);
            R sacc[C::NCH];
#pragma unroll
            for (int c = 0; c < C::NCH; c++) sacc[c] = 0;
            for (int sl = plan->split[j][1]; sl < plan->split[j][2]; sl++)
#pragma unroll
                for (int c = 0; c < C::NCH; c++) sacc[c] += Ps[sl * C::NCHP + c];
            m2l_flush<R, K>(sacc, R0, pw[c0 + c1 + c2] / mfact<R>(c0, c1, c2), Lw + bs * C::NCHP);
        }
    }
    __syncwarp();
    R* Lg = loc + node * (int64_t)C::NCHP * NT;
    for (int e = lane; e < NT * C::NCHP; e += 32) Lg[e] = Lw[e];
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
    size_t rec, mom, loc, plan, W, F;
};

template <int K, int NQ>
Sizes sizes_for(size_t rs, int mode, int order, int64_t n_obs, int64_t n_src, int64_t n_obs_nodes,
                int64_t n_src_nodes) {
    using C = Chan<K>;
    Sizes s;
    s.rec = al256(rs * Rec<K, NQ>::LEN * (size_t)n_src);
    s.mom = al256(rs * C::NCHP * (size_t)n_terms(order) * n_src_nodes);
    s.loc = mode == 1 ? al256(rs * C::NCHP * (size_t)n_terms(order) * n_obs_nodes) : 0;
    s.plan = mode == 1 ? al256(sizeof(M2LPlan)) : 0;
    s.W = al256(rs * NAcc<K, NQ>::n * (size_t)n_obs);
    s.F = al256(rs * C::NO * (size_t)NQ * n_obs);
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
    return Sizes{0, 0, 0, 0, 0, 0};
}

template <typename KF>
int set_smem(KF kfn, size_t smem) {
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
        return launch_status("fmm shared-memory attribute");
    return TCT_OK;
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
    M2LPlan* plan = reinterpret_cast<M2LPlan*>(ws + sz.rec + sz.mom + sz.loc);
    R* W = reinterpret_cast<R*>(ws + sz.rec + sz.mom + sz.loc + sz.plan);
    R* F = reinterpret_cast<R*>(ws + sz.rec + sz.mom + sz.loc + sz.plan + sz.W);
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
    if (stt.n_leaves > 0) {
        fmm_p2m<R, K, NQ><<<(unsigned)stt.n_leaves, 128, 0, st>>>(
            c, p, stt.leaves, stt.start, stt.end, scent, srad, rec, mom);
        if ((rc = launch_status("fmm p2m"))) return rc;
    }
    for (int h = 0; h < stt.n_levels; h++) {
        const int64_t cnt = stt.level_offsets[h + 1] - stt.level_offsets[h];
        if (cnt == 0) continue;
        fmm_m2m<R, K><<<(unsigned)cnt, 128, 0, st>>>(p, stt.levels + stt.level_offsets[h],
                                                     stt.children, scent, srad, mom);
        if ((rc = launch_status("fmm m2m"))) return rc;
    }
    if (near.n_obs > 0) {
        const size_t smem = sizeof(R) * 128 * NA;
        if ((rc = set_smem(fmm_p2p<R, K, NQ>, smem))) return rc;
        fmm_p2p<R, K, NQ><<<(unsigned)near.n_obs, 128, smem, st>>>(
            c, rule, obs_pts, obs_tris, near.obs, near.start, near.src, ot.start, ot.end,
            stt.start, stt.end, rec, W);
        if ((rc = launch_status("fmm p2p"))) return rc;
    }
    if (mode == 0) {
        if (far.n_obs > 0) {
            const size_t smem = sizeof(R) * (size_t)C::NCHP * NT;
            if ((rc = set_smem(fmm_m2p<R, K>, smem))) return rc;
            fmm_m2p<R, K><<<(unsigned)far.n_obs, 128, smem, st>>>(
                p, rule, NQ, far.obs, far.start, far.src, ot.start, ot.end, scent, srad, obs_pts,
                obs_tris, mom, F);
            if ((rc = launch_status("fmm m2p"))) return rc;
        }
    } else {
        if (cudaMemsetAsync(loc, 0, sz.loc, st) != cudaSuccess) return launch_status("fmm memset");
        if (far.n_obs > 0) {
            const int64_t n_el = stt.n_nodes * (int64_t)NT * C::NCHP;
            fmm_moment_factorials<R><<<(unsigned)((n_el + 127) / 128), 128, 0, st>>>(
                p, C::NCHP, stt.n_nodes, mom);
            if ((rc = launch_status("fmm moment factorials"))) return rc;
            fmm_m2l_plan<<<1, 32, 0, st>>>(p, plan);
            if ((rc = launch_status("fmm m2l plan"))) return rc;
            const size_t per_warp =
                sizeof(R) * ((2 * (size_t)NT + M2L_SLOTS) * C::NCHP + (NT + 32 + 3) / 4 * 4);
            const int wpb = (int)std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / per_warp));
            const size_t smem = per_warp * wpb;
            if ((rc = set_smem(fmm_m2l<R, K>, smem))) return rc;
            fmm_m2l<R, K><<<(unsigned)((far.n_obs + wpb - 1) / wpb), 32 * wpb, smem, st>>>(
                p, wpb, far.obs, far.n_obs, far.start, far.src, ocent, orad, scent, srad, mom,
                plan, loc);
            if ((rc = launch_status("fmm m2l"))) return rc;
        }
        const size_t smem_l2l =
            sizeof(R) * ((size_t)C::NCHP * NT + (FMM_MAXP + 1) * (FMM_MAXP + 1));
        if ((rc = set_smem(fmm_l2l<R, K>, smem_l2l))) return rc;
        for (int d = 0; d < ot.n_levels; d++) {
            const int64_t cnt = ot.level_offsets[d + 1] - ot.level_offsets[d];
            if (cnt == 0) continue;
            fmm_l2l<R, K><<<(unsigned)cnt, 128, smem_l2l, st>>>(
                p, ot.levels + ot.level_offsets[d], ot.parent, ocent, orad, loc);
            if ((rc = launch_status("fmm l2l"))) return rc;
        }
        if (ot.n_leaves > 0) {
            const size_t smem = sizeof(R) * (size_t)C::NCHP * NT;
            if ((rc = set_smem(fmm_l2p<R, K>, smem))) return rc;
            fmm_l2p<R, K><<<(unsigned)ot.n_leaves, 128, smem, st>>>(
                p, rule, NQ, ot.leaves, ot.start, ot.end, ocent, orad, obs_pts, obs_tris, loc, F);
            if ((rc = launch_status("fmm l2p"))) return rc;
        }
    }
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
    return s.rec + s.mom + s.loc + s.plan + s.W + s.F;
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
