// Multi-RHS direct farfield for elasticRT3 (FP32, 3-point rule) on the
// 5th-generation tensor cores: y_r = Far x_r for a panel of 16 right-hand
// sides (the reference applies farfield_tris_to_tris once per vector,
// tectosaur/matrix_free.cl:19-107, with the RT vector form of
// kernels/kernels.cl).
//
// Per observation point x (point q1 of observation triangle o) and source
// point y (point q2 of source triangle s), D = y - x, the RT kernel adds
//   J_s w_q2 (CsRT1 / r c_d + CsRT0 / r^3 D_d (D . c) + CsRT2 / r^3 (n_s . D) a_q2,d)
// where c is the source triangle's curl of the input and a_q2 the input
// interpolated at y.  Summed over the source points of one source triangle
// this is linear in (c, a) with coefficients that do not depend on the input:
//   A[x, s] = (S0, T00, T01, T02, T11, T12, T22, V0, V1, V2),
//   T_kl = sum_q2 g D_k D_l,  S0 = T00 + T11 + T22 = sum_q2 1/r,
//   V_q2 = g (n_s . D),  g = w_q2 / r^3 (w_q2 folded into B for equal weights),
// and with R inputs the farfield is the GEMM
//   W[x, (d, r)] = sum_{s, c} A[x, (s, c)] B[(s, c), (d, r)]
// with B (CsRT1 c_d; CsRT0 ((d == k) c_l + (d == l, k != l) c_k); CsRT2 a_q2,d)
// times J_s, built once per apply from the input panel.  The observation-side
// contraction out[b][d] = J_o sum_q1 w_q1 phi_b(q1) W[(o, q1), d] follows in
// the reduce kernel.
//
// A CTA owns 128 observation points (the MMA's M rows: lane = point); per
// tile of 8 source triangles (K = 80) each thread generates its row of A in
// registers and stores it straight into tensor memory (tcgen05.st, hi and
// lo TF32 parts), so the MMAs read A from tensor memory and only B (N = 48
// columns) streams through shared memory -- with A in shared memory too the
// M = 128, N = 48 MMA would be bound by shared-memory bandwidth (~5.5 KB of
// operands per MMA).  Split TF32 (Ah Bh + Ah Bl + Al Bh), the accumulator
// folded into a Kahan pair every RT_FLUSH tiles, source chunks summed in a
// fixed order (deterministic), bounded mbarrier waits with the error word
// and clean-up of far_mrhs.cu.  The D = 0 point pair (a source point on the
// observation point) contributes exactly nothing, as in the reference's
// "skip r^2 == 0": r^2 is offset by 1e-24 and S0 is formed as the trace of
// T, so every A entry carries a factor of D.
#include <algorithm>

#include "far_common.cuh"
#include "tc_common.cuh"

namespace tct {
namespace {

constexpr int RT_M = TC_M;            // observation points per CTA (MMA M)
constexpr int RT_NQ = 3;              // points of the rule (both sides)
constexpr int RT_R = 16;              // right-hand sides per panel
constexpr int RT_N = 3 * RT_R;        // 48: GEMM N, column n = d * R + r
constexpr int RT_C = 7 + RT_NQ;       // 10 A columns per source triangle
constexpr int RT_S = 8;               // source triangles per tile
constexpr int RT_K = RT_C * RT_S;     // 80: GEMM K per tile
constexpr int RT_KSTEPS = RT_K / 8;   // tf32 MMA K = 8
constexpr int RT_G = 2;               // A-generating warp groups (2 packed pairs each)
constexpr int RT_FLUSH = 8;           // tiles per tensor-memory accumulation
constexpr float RT_EPS = 1e-24f;
constexpr int RT_COPIES = 4;          // bulk copies per B tile
constexpr uint32_t RT_B_BYTES = 2u * RT_N * RT_K * 4;  // hi + lo
// tensor-memory columns: D [0, 48), Kahan S [48, 96), C [96, 144); A of
// tile buffer b: hi at RT_COL_A + 2 RT_K b, lo RT_K columns further
constexpr int RT_COL_A = 160;
constexpr int RT_NCOL = 512;
// source record: per pair of consecutive source triangles, the 12 values
// y[q][d] (9) and n[d] (3) of each, interleaved (one 8-byte load = the pair)
constexpr int RT_REC = 3 * RT_NQ + 3;

static_assert(RT_K % 8 == 0 && RT_S % (2 * RT_G) == 0, "tile split");
static_assert(RT_B_BYTES % (16 * RT_COPIES) == 0, "bulk copies must be 16-byte multiples");
static_assert(RT_COL_A + 4 * RT_K <= RT_NCOL, "tensor-memory columns");

__device__ __forceinline__ void tmem_st4(uint32_t taddr, float a, float b, float c, float d) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr),
                 "r"(__float_as_uint(a)), "r"(__float_as_uint(b)), "r"(__float_as_uint(c)),
                 "r"(__float_as_uint(d)));
}

// tcgen05.mma with A in tensor memory, B by shared-memory descriptor
__device__ __forceinline__ void mma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b,
                                            uint32_t idesc, uint32_t accumulate) {
    uint32_t mask[4] = {0, 0, 0, 0};
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(d_tmem), "r"(a_tmem), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask[0]),
          "r"(mask[1]), "r"(mask[2]), "r"(mask[3]));
}

// ---- source points and normals, padded with far-away points ------------------
__global__ void __launch_bounds__(128)
rt_points(Rule2D<float> rule, const float* __restrict__ pts, const int32_t* __restrict__ src_tris,
          int64_t n_src, int64_t n_src_pad, float* __restrict__ srcy) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_src_pad) return;
    float* y = srcy + (s / 2) * (2 * RT_REC) + (s % 2);
    if (s >= n_src) {
#pragma unroll
        for (int k = 0; k < 3 * RT_NQ; k++) y[2 * k] = 1e18f;
#pragma unroll
        for (int k = 3 * RT_NQ; k < RT_REC; k++) y[2 * k] = 0.f;
        return;
    }
    TriGeom<float> t;
    load_tri(t, pts, src_tris, s, 0, false, false);
#pragma unroll
    for (int q = 0; q < RT_NQ; q++) {
        const float bq[3] = {1.f - rule.x[q] - rule.y[q], rule.x[q], rule.y[q]};
#pragma unroll
        for (int d = 0; d < 3; d++) y[2 * (3 * q + d)] = bary_point(t, bq, d);
    }
#pragma unroll
    for (int d = 0; d < 3; d++) y[2 * (3 * RT_NQ + d)] = t.n[d];
}

// ---- B panel: per source triangle and RHS, the 10 x 48 GEMM rows ------------
// One thread per (padded source triangle, r); rows k = 10 sl + c of tile
// s / RT_S, hi block then lo block, in the canonical K-major layout.
__global__ void __launch_bounds__(128)
rt_prep(Consts<float> c, Rule2D<float> rule, float wbar, const float* __restrict__ pts,
        const int32_t* __restrict__ src_tris, int64_t n_src, int64_t n_src_pad,
        const float* __restrict__ in, float* __restrict__ Bg) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_src_pad * RT_R) return;
    const int64_t s = g / RT_R;
    const int r = (int)(g % RT_R);
    float cv[3] = {0.f, 0.f, 0.f}, av[RT_NQ][3] = {};
    float scale = 0.f;
    if (s < n_src) {
        TriGeom<float> t;
        load_tri(t, pts, src_tris, s, 0, false, true);
        const float* x = in + (int64_t)r * n_src * 9 + s * 9;
        float in9[9];
#pragma unroll
        for (int k = 0; k < 9; k++) in9[k] = x[k];
        // src_surf_curl[d][Ij] = sum_b sc[b][Ij] in[b][d]; c[p] = e[m][p][j] ssc[j][m]
        float ssc[3][3];
#pragma unroll
        for (int Ij = 0; Ij < 3; Ij++)
#pragma unroll
            for (int d = 0; d < 3; d++) {
                float a = 0.f;
#pragma unroll
                for (int b = 0; b < 3; b++) a += t.sc[b][Ij] * in9[b * 3 + d];
                ssc[d][Ij] = a;
            }
#pragma unroll
        for (int p = 0; p < 3; p++) {
            float a = 0.f;
#pragma unroll
            for (int m = 0; m < 3; m++)
#pragma unroll
                for (int j = 0; j < 3; j++)
                    if (levi(m, p, j) != 0) a += (float)levi(m, p, j) * ssc[j][m];
            cv[p] = a;
        }
#pragma unroll
        for (int q = 0; q < RT_NQ; q++) {
            const float sb[3] = {1.f - rule.x[q] - rule.y[q], rule.x[q], rule.y[q]};
#pragma unroll
            for (int d = 0; d < 3; d++)
                av[q][d] = in9[0 * 3 + d] * sb[0] + in9[1 * 3 + d] * sb[1] + in9[2 * 3 + d] * sb[2];
        }
        scale = t.J * wbar;
    }
    const int64_t tile = s / RT_S;
    const int sl = (int)(s % RT_S);
    unsigned char* base = reinterpret_cast<unsigned char*>(Bg) + tile * (int64_t)RT_B_BYTES;
    const int ab[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
#pragma unroll
    for (int cc = 0; cc < RT_C; cc++) {
        const int k = RT_C * sl + cc;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            float v;
            if (cc == 0) {
                v = c.CsRT1 * cv[d];
            } else if (cc < 7) {
                const int a = ab[cc - 1][0], b = ab[cc - 1][1];
                v = c.CsRT0 * ((d == a ? cv[b] : 0.f) + ((d == b && a != b) ? cv[a] : 0.f));
            } else {
                v = c.CsRT2 * av[cc - 7][d];
            }
            v *= scale;
            const int n = d * RT_R + r;
            const float hi = tf32_round(v);
            const float lo = tf32_round(v - hi);
            const uint32_t off = mr_off(n, k, RT_N);
            *reinterpret_cast<float*>(base + off) = hi;
            *reinterpret_cast<float*>(base + (int64_t)RT_N * RT_K * 4 + off) = lo;
        }
    }
}

// ---- main: generate A into tensor memory, copy B, tcgen05.mma --------------
// grid (point blocks of 128, source chunks); RT_G x 128 threads generate A
// (thread (row, group): observation point `row`, the group's 4 of the tile's
// 8 source triangles as two packed pairs, their records loaded while the
// previous tile is stored), one more warp issues the B copies and the MMAs.
// Per tile t: A(t) is generated in registers while the MMAs of t - 1 run;
// each thread waits (itself, on the mbarrier) for the MMAs of t - 2, which
// read A buffer t & 1, and stores A(t) there; the B tile of t + 1 goes into
// the B buffer those MMAs read (three B buffers); after one CTA barrier the
// MMAs of t are issued behind those of t - 1.  At the end of each group of
// RT_FLUSH tiles all MMAs complete and D is folded into the Kahan pair.
// Measured on the 60k-triangle surface (16 vectors, 152 ms): timing copies
// without the MMAs take 98 ms, without the A arithmetic 126 ms -- the
// per-tile B traffic from L2 (every CTA of 128 points re-reads the 230 MB B
// operand) and the per-tile barrier, not the arithmetic, set the pace.
template <bool UNIFORM>
__global__ void __launch_bounds__(128 * RT_G + 32, 1)
rt_main(Rule2D<float> rule, const float* __restrict__ pts, const int32_t* __restrict__ obs_tris,
        int64_t n_pts, const float* __restrict__ srcy, int64_t n_tiles, int64_t tiles_per_chunk,
        const float* __restrict__ Bg, float* __restrict__ partial, int* __restrict__ err) {
    constexpr int SG = RT_S / RT_G;  // source triangles per thread group
    constexpr int NP = SG / 2;       // packed source pairs per thread
    constexpr int KG = RT_C * SG;    // A values per thread and tile
    static_assert(SG % 2 == 0 && KG % 4 == 0, "whole packed pairs, 4-column stores");
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* Bs0 = smem;  // three B buffers, each hi then lo
    __shared__ __align__(8) uint64_t bar_m[2];
    __shared__ __align__(8) uint64_t bar_b[3];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int tid = threadIdx.x;
    if (tid == 0) abort_flag = *reinterpret_cast<volatile int*>(err);
    __syncthreads();
    if (abort_flag) return;  // an earlier CTA timed out: no tensor memory taken yet
    const int warp = tid >> 5;
    const int row = tid & (RT_M - 1);
    const int grp = tid >> 7;
    const bool mma_warp = warp == 4 * RT_G;
    const bool mma_lead = tid == 128 * RT_G;
    const int64_t p = (int64_t)blockIdx.x * RT_M + row;  // observation point
    const bool valid = p < n_pts;
    const int64_t t0 = (int64_t)blockIdx.y * tiles_per_chunk;
    const int64_t t1 = min(n_tiles, t0 + tiles_per_chunk);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(RT_NCOL));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int i = 0; i < 2; i++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar_m[i])),
                         "r"(1));
        for (int i = 0; i < 3; i++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar_b[i])),
                         "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;
    const uint32_t barm0 = smem_u32(&bar_m[0]), barm1 = smem_u32(&bar_m[1]);
    const uint32_t barb0 = smem_u32(&bar_b[0]), barb1 = smem_u32(&bar_b[1]),
                   barb2 = smem_u32(&bar_b[2]);

    // this thread's observation point (packed, negated: D = y_pair + negx);
    // a row past the last point sits 1e18 away, where every A entry
    // underflows to 0 (r^-3 < 1e-54; or D = 0 against a padding source)
    f2_t negx[3];
    {
        float x[3] = {1e18f, 1e18f, 1e18f};
        if (valid) {
            TriGeom<float> ot;
            load_tri(ot, pts, obs_tris, p / RT_NQ, 0, false, false);
            const int q1 = (int)(p % RT_NQ);
            const float bq[3] = {1.f - rule.x[q1] - rule.y[q1], rule.x[q1], rule.y[q1]};
#pragma unroll
            for (int d = 0; d < 3; d++) x[d] = bary_point(ot, bq, d);
        }
#pragma unroll
        for (int d = 0; d < 3; d++) negx[d] = pk(-x[d], -x[d]);
    }
    f2_t wq2[UNIFORM ? 1 : RT_NQ];
    if constexpr (!UNIFORM) {
#pragma unroll
        for (int q = 0; q < RT_NQ; q++) wq2[q] = pk(rule.w[q], rule.w[q]);
    }
    const f2_t eps2 = pk(RT_EPS, RT_EPS);

    // Pipeline state, the same in every thread (each thread runs every wait
    // itself): MMAs of tile t commit to bar_m[t & 1]; B tiles rotate through
    // three buffers, so the copy of tile t + 1 needs only the MMAs of t - 2
    // to have completed, and the MMAs of t queue behind those of t - 1.
    uint32_t ph_m0 = 0, ph_m1 = 0, ph_b0 = 0, ph_b1 = 0, ph_b2 = 0;
    bool pm0 = false, pm1 = false;              // MMA commit not yet observed
    bool pb0 = false, pb1 = false, pb2 = false;  // B copy not yet observed
    bool ok = true;                             // CTA-uniform after each barrier
    const uint32_t idesc = mr_instr_desc(RT_N);
    const uint32_t lane_off = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t lane_base = tmem + lane_off;
    // this warp's accumulator columns in the fold and the epilogue
    const int col0 = (grp * (RT_N / 8) / RT_G) * 8, col1 = ((grp + 1) * (RT_N / 8) / RT_G) * 8;
    auto wait_m = [&](int i, bool& good) {
        if (i == 0 && pm0) {
            good = mbar_wait(barm0, ph_m0) && good;
            ph_m0 ^= 1;
            pm0 = false;
        } else if (i == 1 && pm1) {
            good = mbar_wait(barm1, ph_m1) && good;
            ph_m1 ^= 1;
            pm1 = false;
        }
    };
    auto issue_b = [&](int64_t tile, int buf) {
        const uint32_t bar = buf == 0 ? barb0 : (buf == 1 ? barb1 : barb2);
        if (mma_lead) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                         "r"(RT_B_BYTES)
                         : "memory");
            const unsigned char* src =
                reinterpret_cast<const unsigned char*>(Bg) + tile * (int64_t)RT_B_BYTES;
            const uint32_t dst = smem_u32(Bs0) + (uint32_t)buf * RT_B_BYTES;
#pragma unroll
            for (int cpy = 0; cpy < RT_COPIES; cpy++)
                bulk_g2s(dst + cpy * (RT_B_BYTES / RT_COPIES),
                         src + cpy * (RT_B_BYTES / RT_COPIES), RT_B_BYTES / RT_COPIES, bar);
        }
        if (buf == 0) pb0 = true;
        else if (buf == 1) pb1 = true;
        else pb2 = true;
    };
    // this thread's source pair record of tile t
    const f2_t* recs = reinterpret_cast<const f2_t*>(srcy) + grp * NP * RT_REC;
    constexpr int64_t REC_STRIDE = (RT_S / 2) * RT_REC;  // f2 values per tile
    f2_t yc[NP][RT_REC];
    if (!mma_warp && t0 < t1) {
#pragma unroll
        for (int sp = 0; sp < NP; sp++)
#pragma unroll
            for (int k = 0; k < RT_REC; k++)
                yc[sp][k] = __ldg(recs + t0 * REC_STRIDE + sp * RT_REC + k);
    }
    if (t0 < t1) issue_b(t0, 0);
    for (int64_t t = t0; t < t1; t++) {
        const int64_t k = t - t0;
        const int abuf = (int)(k & 1), bbuf = (int)(k % 3);
        bool good = true;
        if (k > 0 && k % RT_FLUSH == 0) {
            // an accumulation group ends: its MMAs (up to those of t - 1)
            // complete, then D is folded into the Kahan pair before the
            // MMAs of t restart it
            wait_m(0, good);
            wait_m(1, good);
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (!mma_warp) tmem_fold<RT_N>(lane_base, col0, col1, k == RT_FLUSH);
        }
        float av[KG];
        if (!mma_warp) {
#pragma unroll
            for (int sp = 0; sp < NP; sp++) {
                // A of one packed source pair for this point: 10 values per source
                const f2_t* yr = yc[sp];
                const f2_t n0 = yr[3 * RT_NQ], n1 = yr[3 * RT_NQ + 1], n2 = yr[3 * RT_NQ + 2];
                f2_t T00 = 0ull, T01 = 0ull, T02 = 0ull, T11 = 0ull, T12 = 0ull, T22 = 0ull;
                f2_t V[RT_NQ];
#pragma unroll
                for (int q2 = 0; q2 < RT_NQ; q2++) {
                    const f2_t D0 = add2(yr[3 * q2], negx[0]);
                    const f2_t D1 = add2(yr[3 * q2 + 1], negx[1]);
                    const f2_t D2 = add2(yr[3 * q2 + 2], negx[2]);
                    f2_t r2 = fma2(D0, D0, eps2);
                    r2 = fma2(D1, D1, r2);
                    r2 = fma2(D2, D2, r2);
                    float ra, rb;
                    upk(r2, ra, rb);
                    const f2_t ir = pk(rsqrtf(ra), rsqrtf(rb));
                    f2_t gg = mul2(mul2(ir, ir), ir);
                    if constexpr (!UNIFORM) gg = mul2(gg, wq2[q2]);
                    const f2_t g0 = mul2(gg, D0), g1 = mul2(gg, D1), g2 = mul2(gg, D2);
                    T00 = fma2(g0, D0, T00);
                    T01 = fma2(g0, D1, T01);
                    T02 = fma2(g0, D2, T02);
                    T11 = fma2(g1, D1, T11);
                    T12 = fma2(g1, D2, T12);
                    T22 = fma2(g2, D2, T22);
                    V[q2] = fma2(g2, n2, fma2(g1, n1, mul2(g0, n0)));
                }
                const f2_t S0 = add2(add2(T00, T11), T22);
                const f2_t Tc[RT_C] = {S0, T00, T01, T02, T11, T12, T22, V[0], V[1], V[2]};
#pragma unroll
                for (int cc = 0; cc < RT_C; cc++) {
                    float va, vb;
                    upk(Tc[cc], va, vb);
                    av[2 * RT_C * sp + cc] = va;
                    av[2 * RT_C * sp + RT_C + cc] = vb;
                }
            }
            // the next tile's records: in flight while A is stored and the
            // CTA waits for the B tile
            if (t + 1 < t1) {
#pragma unroll
                for (int sp = 0; sp < NP; sp++)
#pragma unroll
                    for (int q = 0; q < RT_REC; q++)
                        yc[sp][q] = __ldg(recs + (t + 1) * REC_STRIDE + sp * RT_REC + q);
            }
        }
        // the MMAs of t - 2 read A buffer abuf and B buffer (k + 1) % 3
        wait_m(abuf, good);
        if (!mma_warp) {
            // hi / lo parts into A buffer abuf, columns [KG grp, KG (grp + 1));
            // lo is left in FP32: the MMA reads the top 19 bits of a TF32
            // operand, so it is truncated there (|lo| <= 2^-11 |v|, its
            // truncation <= 2^-21 |v|)
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t ahi = lane_base + RT_COL_A + 2 * RT_K * abuf + KG * grp;
#pragma unroll
            for (int ch = 0; ch < KG / 4; ch++) {
                float h[4], l[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    h[u] = tf32_round(av[4 * ch + u]);
                    l[u] = av[4 * ch + u] - h[u];
                }
                tmem_st4(ahi + 4 * ch, h[0], h[1], h[2], h[3]);
                tmem_st4(ahi + RT_K + 4 * ch, l[0], l[1], l[2], l[3]);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        }
        if (good && t + 1 < t1) issue_b(t + 1, (int)((k + 1) % 3));
        asm volatile("tcgen05.fence::before_thread_sync;");
        {
            bool wb = true;
            if (mma_warp) {
                const uint32_t bar = bbuf == 0 ? barb0 : (bbuf == 1 ? barb1 : barb2);
                const uint32_t ph = bbuf == 0 ? ph_b0 : (bbuf == 1 ? ph_b1 : ph_b2);
                wb = mbar_wait(bar, ph);
            }
            if (bbuf == 0) {
                ph_b0 ^= 1;
                pb0 = false;
            } else if (bbuf == 1) {
                ph_b1 ^= 1;
                pb1 = false;
            } else {
                ph_b2 ^= 1;
                pb2 = false;
            }
            if (!__syncthreads_and(good && wb)) {
                ok = false;  // a bounded wait gave up
                break;
            }
        }
        if (mma_lead) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t lboB = RT_N / 8 * 128;
            const uint32_t bH = smem_u32(Bs0) + (uint32_t)bbuf * RT_B_BYTES,
                           bL = bH + RT_N * RT_K * 4;
            const uint32_t aH = tmem + RT_COL_A + 2 * RT_K * abuf, aL = aH + RT_K;
#pragma unroll
            for (int ks = 0; ks < RT_KSTEPS; ks++) {
                // D restarts at the first tile of every RT_FLUSH group
                const uint32_t first = (k % RT_FLUSH == 0 && ks == 0) ? 0u : 1u;
                const uint64_t dBh = mr_smem_desc(bH + 2 * ks * lboB, lboB, 128);
                const uint64_t dBl = mr_smem_desc(bL + 2 * ks * lboB, lboB, 128);
                mma_tf32_ts(tmem, aH + 8 * ks, dBh, idesc, first);
                mma_tf32_ts(tmem, aH + 8 * ks, dBl, idesc, 1u);
                mma_tf32_ts(tmem, aL + 8 * ks, dBh, idesc, 1u);
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    abuf ? barm1 : barm0)
                : "memory");
        }
        if (abuf) pm1 = true;
        else pm0 = true;
    }
    if (ok) {
        bool good = true;
        wait_m(0, good);
        wait_m(1, good);
        if (!__syncthreads_and(good)) ok = false;
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        // one more bounded wait for whatever is still in flight
        if (pm0) mbar_wait(barm0, ph_m0);
        if (pm1) mbar_wait(barm1, ph_m1);
        if (pb0) mbar_wait(barb0, ph_b0);
        if (pb1) mbar_wait(barb1, ph_b1);
        if (pb2) mbar_wait(barb2, ph_b2);
    }
    asm volatile("tcgen05.fence::after_thread_sync;");

    // epilogue: fold the last group, then S - C of this thread's point and
    // column range -> partial[chunk][r][point][d]
    if (ok && t1 > t0 && !mma_warp) {
        tmem_fold<RT_N>(lane_base, col0, col1, t1 - t0 <= RT_FLUSH);
#pragma unroll 1
        for (int c0 = col0; c0 < col1; c0 += 8) {
            float sv[8], cv[8];
            tmem_ld8(lane_base + RT_N + c0, sv);
            tmem_ld8(lane_base + 2 * RT_N + c0, cv);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (valid) {
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int n = c0 + u;
                    const int d = n / RT_R, r = n % RT_R;
                    partial[(((int64_t)blockIdx.y * RT_R + r) * n_pts + p) * 3 + d] = sv[u] - cv[u];
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(RT_NCOL));
    }
}

// Sum the chunk partials in a fixed order (compensated) and contract the
// observation points: out[r][o][b][d] (+)= J_o sum_q1 w_q1 phi_b(q1) W[r][(o, q1)][d].
__global__ void __launch_bounds__(128)
rt_reduce(Rule2D<float> rule, const float* __restrict__ pts, const int32_t* __restrict__ obs_tris,
          int64_t n_obs, int n_chunks, const float* __restrict__ partial,
          float* __restrict__ out, int accumulate) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_obs * RT_R) return;
    const int64_t o = g % n_obs;
    const int r = (int)(g / n_obs);
    const int64_t n_pts = RT_NQ * n_obs;
    float W[RT_NQ][3];
#pragma unroll
    for (int q = 0; q < RT_NQ; q++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            float s = 0.f, cmp = 0.f;
            for (int c = 0; c < n_chunks; c++) {
                const float y =
                    partial[(((int64_t)c * RT_R + r) * n_pts + RT_NQ * o + q) * 3 + d] - cmp;
                const float t = s + y;
                cmp = (t - s) - y;
                s = t;
            }
            W[q][d] = s;
        }
    TriGeom<float> ot;
    load_tri(ot, pts, obs_tris, o, 0, false, false);
    float* op = out + ((int64_t)r * n_obs + o) * 9;
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            float s = 0.f;
#pragma unroll
            for (int q = 0; q < RT_NQ; q++) {
                const float ob = (b == 0) ? (1.f - rule.x[q] - rule.y[q])
                                          : (b == 1 ? rule.x[q] : rule.y[q]);
                s += (rule.w[q] * ob) * W[q][d];
            }
            const float v = ot.J * s;
            op[b * 3 + d] = accumulate ? op[b * 3 + d] + v : v;
        }
}

inline size_t rt_al256(size_t b) { return (b + 255) / 256 * 256; }

int64_t rt_chunks(int64_t n_pts, int64_t n_tiles) {
    const int64_t blocks = (n_pts + RT_M - 1) / RT_M;
    // a few waves over the 148 SMs, at most 1024 tiles (4096 sources) per
    // accumulator, at least 8 tiles per chunk, at most 64 chunks
    int64_t want = (148 * 2 + blocks - 1) / std::max<int64_t>(blocks, 1);
    want = std::max<int64_t>(want, (n_tiles + 1023) / 1024);
    return std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(want, n_tiles / 8 + 1), 64));
}

struct RtSizes {
    size_t B, y, partial, err;
};

RtSizes rt_sizes(int64_t n_obs, int64_t n_src) {
    const int64_t n_pad = (n_src + RT_S - 1) / RT_S * RT_S;
    const int64_t n_tiles = n_pad / RT_S;
    const int64_t n_pts = RT_NQ * n_obs;
    RtSizes s;
    s.B = rt_al256((size_t)n_tiles * RT_B_BYTES);
    s.y = rt_al256((size_t)(n_pad / 2) * 2 * RT_REC * 4);
    s.partial = rt_al256((size_t)rt_chunks(n_pts, n_tiles) * RT_R * n_pts * 3 * 4);
    s.err = 256;
    return s;
}

template <bool UNIFORM>
int run_rt(const Consts<float>& c, const Rule2D<float>& rule, float* out, const float* in,
           const float* pts, const int32_t* obs_tris, int64_t n_obs, const int32_t* src_tris,
           int64_t n_src, int accumulate, unsigned char* ws, cudaStream_t st) {
    const int64_t n_pad = (n_src + RT_S - 1) / RT_S * RT_S;
    const int64_t n_tiles = n_pad / RT_S;
    const int64_t n_pts = RT_NQ * n_obs;
    const RtSizes sz = rt_sizes(n_obs, n_src);
    float* Bg = reinterpret_cast<float*>(ws);
    float* srcy = reinterpret_cast<float*>(ws + sz.B);
    float* partial = reinterpret_cast<float*>(ws + sz.B + sz.y);
    int* err = reinterpret_cast<int*>(ws + sz.B + sz.y + sz.partial);
    if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return launch_status("rt memset");
    rt_points<<<(unsigned)((n_pad + 127) / 128), 128, 0, st>>>(rule, pts, src_tris, n_src, n_pad,
                                                               srcy);
    int rc = launch_status("rt points");
    if (rc) return rc;
    const float wbar = UNIFORM ? rule.w[0] : 1.f;
    rt_prep<<<(unsigned)((n_pad * RT_R + 127) / 128), 128, 0, st>>>(c, rule, wbar, pts, src_tris,
                                                                    n_src, n_pad, in, Bg);
    if ((rc = launch_status("rt prep"))) return rc;
    const int64_t chunks = rt_chunks(n_pts, n_tiles);
    const int64_t per = (n_tiles + chunks - 1) / chunks;
    const int64_t real = (n_tiles + per - 1) / per;
    const size_t smem = (size_t)3 * RT_B_BYTES;
    auto kfn = rt_main<UNIFORM>;
    if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return launch_status("rt smem attribute");
    dim3 grid((unsigned)((n_pts + RT_M - 1) / RT_M), (unsigned)real);
    kfn<<<grid, 128 * RT_G + 32, smem, st>>>(rule, pts, obs_tris, n_pts, srcy, n_tiles, per, Bg,
                                            partial, err);
    if ((rc = launch_status("rt main"))) return rc;
    rt_reduce<<<(unsigned)((n_obs * RT_R + 127) / 128), 128, 0, st>>>(
        rule, pts, obs_tris, n_obs, (int)real, partial, out, accumulate);
    return launch_status("rt reduce");
}

}  // namespace
}  // namespace tct

using namespace tct;

extern "C" size_t tct_farfield_rt_panel_workspace_bytes(int64_t n_obs, int64_t n_src, int R,
                                                        int n_q) {
    if (R != RT_R || n_q != RT_NQ || n_obs < 0 || n_src < 0) return 0;
    const RtSizes s = rt_sizes(n_obs, n_src);
    return s.B + s.y + s.partial + s.err;
}

extern "C" int tct_farfield_rt_panel_error(const void* workspace, int64_t n_obs, int64_t n_src,
                                           int R, int n_q, void* stream, int* host_flag) {
    TCT_CHECK_ARG(workspace && host_flag && R == RT_R && n_q == RT_NQ,
                  "tct_farfield_rt_panel_error: bad arguments");
    const RtSizes s = rt_sizes(n_obs, n_src);
    cudaStream_t st = as_stream(stream);
    if (cudaMemcpyAsync(host_flag, reinterpret_cast<const unsigned char*>(workspace) + s.B + s.y +
                                       s.partial,
                        sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return launch_status("tct_farfield_rt_panel_error");
    return TCT_OK;
}

extern "C" int tct_farfield_rt_panel_matvec(void* out, const void* in, const void* pts,
                                            const int32_t* obs_tris, int64_t n_obs,
                                            const int32_t* src_tris, int64_t n_src, int R,
                                            int n_q, const double* quad_pts,
                                            const double* quad_wts, const double* params,
                                            int accumulate, void* workspace,
                                            size_t workspace_bytes, void* stream) {
    TCT_CHECK_ARG(R == RT_R, "tct_farfield_rt_panel_matvec: R must be 16 (got %d)", R);
    TCT_CHECK_ARG(n_q == RT_NQ,
                  "tct_farfield_rt_panel_matvec: %d-point rule (supported: 3)", n_q);
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_farfield_rt_panel_matvec: negative size");
    TCT_CHECK_ARG(params && quad_pts && quad_wts,
                  "tct_farfield_rt_panel_matvec: null params or rule");
    if (n_obs == 0) return TCT_OK;
    TCT_CHECK_ARG(n_obs < (int64_t(1) << 40) && n_src < (int64_t(1) << 40),
                  "tct_farfield_rt_panel_matvec: size out of range");
    const size_t need = tct_farfield_rt_panel_workspace_bytes(n_obs, n_src, R, n_q);
    TCT_CHECK_ARG(workspace && workspace_bytes >= need && aligned(workspace, 256),
                  "tct_farfield_rt_panel_matvec: workspace of %zu bytes (256-aligned) required",
                  need);
    const Consts<float> c = make_consts<float>(params);
    Rule2D<float> rule;
    bool uniform = true;
    for (int q = 0; q < MAXQ; q++) {
        rule.x[q] = q < n_q ? (float)quad_pts[2 * q] : 0.f;
        rule.y[q] = q < n_q ? (float)quad_pts[2 * q + 1] : 0.f;
        rule.w[q] = q < n_q ? (float)quad_wts[q] : 0.f;
        if (q < n_q) uniform = uniform && quad_wts[q] == quad_wts[0];
    }
    unsigned char* ws = reinterpret_cast<unsigned char*>(workspace);
    cudaStream_t st = as_stream(stream);
    if (n_src == 0) {
        if (!accumulate && cudaMemsetAsync(out, 0, sizeof(float) * 9 * n_obs * R, st) != cudaSuccess)
            return launch_status("tct_farfield_rt_panel_matvec memset");
        return TCT_OK;
    }
    float* o = (float*)out;
    const float* x = (const float*)in;
    const float* p = (const float*)pts;
    return uniform ? run_rt<true>(c, rule, o, x, p, obs_tris, n_obs, src_tris, n_src, accumulate,
                                  ws, st)
                   : run_rt<false>(c, rule, o, x, p, obs_tris, n_obs, src_tris, n_src, accumulate,
                                   ws, st);
}
