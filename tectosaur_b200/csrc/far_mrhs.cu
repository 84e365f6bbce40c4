// Multi-RHS direct farfield for elasticRH3 (FP32; 3-, 4- and 7-point rules) on the
// 5th-generation tensor cores: y_r = Far x_r for a panel of R right-hand
// sides (the reference applies farfield_tris_to_tris once per vector,
// tectosaur/matrix_free.cl:19-107).
//
// For elasticRH3 the NQ x NQ point pairs of a triangle pair reduce to the
// scalar S0 and the symmetric 3x3 T (the direct kernel's factorisation:
// T = sum_q1,q2 w_q1 w_q2 D D^T / r^3 over the point pairs), and the
// input enters only through per-source 3x3 matrices P and M = -2 ssc:
//   W_o[d][j] += S0 P_s[d][j] + sum_k T[d][k] M_s[k][j].
// With R inputs this is a GEMM:
//   W[o, (dj, r)] = sum_{s, c} A[o, (s, c)] B[(s, c), (dj, r)]
// with A = (S0, T00, T01, T02, T11, T12, T22) per triangle pair -- generated
// on the fly by the CUDA cores, never stored in HBM -- and B built once per
// apply from the input panel.  Per tile of 128 observation and 8 source
// triangles: the 128 threads compute A (K = 56) into shared memory, the tile
// of B is copied in, and one thread issues tcgen05.mma (kind::tf32, M = 128,
// N = 9R) accumulating in tensor memory.  Split TF32: A = Ah + Al and
// B = Bh + Bl with every part rounded to TF32; Ah Bh + Ah Bl + Al Bh are
// accumulated in FP32 (the dropped Al Bl term is below 2^-22 relative).
// Compensated accumulation: the tensor-memory accumulator D takes only
// MR_FLUSH tiles; it is then folded into a Kahan pair (S, C) kept in spare
// tensor-memory columns (tcgen05.ld / st, 8 columns at a time), and the next
// tile overwrites D.  (Plain FP32 accumulation over a whole source chunk
// loses ~2e-4 relative on the 60k-triangle surface, where near pairs add
// large, partly cancelling terms; the single-vector kernel keeps Kahan per
// tile for the same reason.)  The source range is split into chunks (grid.y)
// whose partial results are summed in a fixed order (deterministic).
//
// Operand layout in shared memory (K-major, no swizzle, the canonical UMMA
// layout): 8-row x 16-byte core matrices; element (row, k) of an operand with
// `rows` rows at byte (k / 4) * LBO + (row / 8) * 128 + (row % 8) * 16 +
// (k % 4) * 4 with LBO = rows / 8 * 128.  B is stored in HBM already in this
// layout, tile by tile (hi block, then lo block), so a tile is one contiguous
// copy.
//
// Waits on the MMA completion barrier are bounded in time (TC_WAIT_NS, by
// %globaltimer) and their outcome is made CTA-uniform with
// __syncthreads_and, so no thread is left at a barrier; on timeout the kernel
// records an error word in the workspace, waits once more (bounded), frees
// its tensor memory and returns; CTAs that start after an error exit before
// allocating tensor memory.
#include <algorithm>

#include "far_common.cuh"
#include "tc_common.cuh"

namespace tct {
namespace {

constexpr int MR_M = TC_M;           // observation triangles per CTA (MMA M)
constexpr int MR_S = 8;              // source triangles per tile
constexpr int MR_K = 7 * MR_S;       // 56: GEMM K per tile
constexpr int MR_KSTEPS = MR_K / 8;  // tf32 MMA K = 8
constexpr float MR_EPS = 1e-24f;     // r^2 offset (see far_main_rh2)
constexpr int MR_FLUSH = 8;          // tiles per tensor-memory accumulation

// ---- B panel: per source triangle and RHS, the 7 x 9 GEMM rows --------------
// B[(s, c), (dj, r)]: c = 0 (S0): P_r[d][j]; c = T_ab: (d == a) M_r[b][j] +
// (d == b, a != b) M_r[a][j].  One thread per (padded source triangle, r).
__global__ void __launch_bounds__(128)
mrhs_prep(Consts<float> c, float w2, const float* __restrict__ pts,
          const int32_t* __restrict__ src_tris, int64_t n_src, int64_t n_src_pad,
          const float* __restrict__ in, int R, float* __restrict__ Bg) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_src_pad * R) return;
    const int64_t s = g / R;
    const int r = (int)(g % R);
    const int N = 9 * R;
    float P[3][3] = {}, M[3][3] = {};
    if (s < n_src) {
        TriGeom<float> t;
        load_tri(t, pts, src_tris, s, 0, false, true);
        const float* x = in + (int64_t)r * n_src * 9 + s * 9;
        float ssc[3][3];
#pragma unroll
        for (int Ij = 0; Ij < 3; Ij++)
#pragma unroll
            for (int d = 0; d < 3; d++) {
                float a = 0.f;
#pragma unroll
                for (int b = 0; b < 3; b++) a += t.sc[b][Ij] * x[b * 3 + d];
                ssc[d][Ij] = a;
            }
        const float scale = t.J * c.CsRH0 * w2;
        const float Bt = (ssc[0][0] + ssc[1][1] + ssc[2][2]) * c.CsRH1;
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                P[d][j] = scale * ((d == j ? Bt : 0.f) + c.CsRH2 * ssc[j][d] - 2.f * ssc[d][j]);
                M[d][j] = scale * (-2.f * ssc[d][j]);
            }
    }
    const int64_t tile = s / MR_S;
    const int sl = (int)(s % MR_S);
    unsigned char* base = reinterpret_cast<unsigned char*>(Bg) + tile * (int64_t)2 * N * MR_K * 4;
    const int ab[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
#pragma unroll
    for (int cc = 0; cc < 7; cc++) {
        const int k = 7 * sl + cc;
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                float v;
                if (cc == 0) {
                    v = P[d][j];
                } else {
                    const int a = ab[cc - 1][0], b = ab[cc - 1][1];
                    v = (d == a ? M[b][j] : 0.f) + ((d == b && a != b) ? M[a][j] : 0.f);
                }
                const int n = (d * 3 + j) * R + r;
                const float hi = tf32_round(v);
                const float lo = tf32_round(v - hi);
                const uint32_t off = mr_off(n, k, N);
                *reinterpret_cast<float*>(base + off) = hi;
                *reinterpret_cast<float*>(base + (int64_t)N * MR_K * 4 + off) = lo;
            }
    }
}

// ---- main: generate A, copy B, tcgen05.mma into TMEM ------------------------
// Observation quadrature points of the rule (barycentric 1 - x - y, x, y).
// grid (obs blocks of 128, source chunks); G x 128 threads: thread
// (row, group) generates row `row` of A for the group's 8 / G of the tile's 8
// source triangles (G = 4 keeps 16 warps in flight where the registers allow,
// G = 2 for the 7-point rule); one thread issues the B tiles as bulk async
// copies (completing on bar_b[buffer]) and the MMAs (completing on
// bar_mma).  The G warp groups split the tensor-memory columns of the fold
// and the epilogue.  Dynamic smem: A hi/lo (2 x 128 x 56 x 4), two B
// buffers of hi/lo (2 x 2 x N x 56 x 4).
constexpr int MR_COPIES = 4;  // bulk copies per B tile

template <int R, int NQ, bool UNIFORM, int G>
__global__ void __launch_bounds__(128 * G + 32, 1)
mrhs_main(Rule2D<float> rule, const float* __restrict__ pts, const int32_t* __restrict__ obs_tris,
          int64_t n_obs,
          const float* __restrict__ srcy, int64_t n_tiles, int64_t tiles_per_chunk,
          const float* __restrict__ Bg, float* __restrict__ partial, int* __restrict__ err) {
    constexpr int N = 9 * R;
    constexpr int SG = MR_S / G;  // source triangles per thread group
    constexpr int KG = 7 * SG;    // A values per thread and tile
    static_assert(3 * N <= 512, "D, S and C must fit the 512 tensor-memory columns");
    static_assert(N % 8 == 0 && MR_S % G == 0 && KG % 2 == 0, "tile split");
    constexpr int NCOL = 512;
    constexpr uint32_t B_BYTES = 2u * N * MR_K * 4;
    static_assert(B_BYTES % (16 * MR_COPIES) == 0, "bulk copies must be 16-byte multiples");
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* Ah = smem;
    unsigned char* Al = Ah + MR_M * MR_K * 4;
    // two B buffers (tile t and t + 1), each hi then lo, 2 * N * MR_K * 4
    unsigned char* Bs0 = Al + MR_M * MR_K * 4;
    __shared__ __align__(8) uint64_t bar_mma;
    __shared__ __align__(8) uint64_t bar_b[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int tid = threadIdx.x;
    if (tid == 0) abort_flag = *reinterpret_cast<volatile int*>(err);
    __syncthreads();
    if (abort_flag) return;  // an earlier CTA timed out: no tensor memory taken yet
    const int warp = tid >> 5;
    const int row = tid & (MR_M - 1);
    const int grp = tid >> 7;  // thread group: A sources and tensor-memory columns
    // The last warp issues the B copies and the MMAs and polls their
    // barriers, so that the A generators never stall behind the tensor
    // core's instruction queue.
    const bool mma_warp = warp == 4 * G;
    const bool mma_lead = tid == 128 * G;
    const int64_t o = (int64_t)blockIdx.x * MR_M + row;
    const bool valid = o < n_obs;
    const int64_t t0 = (int64_t)blockIdx.y * tiles_per_chunk;
    const int64_t t1 = min(n_tiles, t0 + tiles_per_chunk);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(NCOL));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar_mma)), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar_b[0])), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar_b[1])), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;
    const uint32_t barm = smem_u32(&bar_mma);
    const uint32_t barb0 = smem_u32(&bar_b[0]), barb1 = smem_u32(&bar_b[1]);

    // obs quadrature points of the rule; weight products for non-uniform rules
    // (a uniform rule's w^2 is folded into B by mrhs_prep)
    float x[NQ][3];
    {
        TriGeom<float> ot;
        if (valid) {
            load_tri(ot, pts, obs_tris, o, 0, false, false);
        } else {
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int d = 0; d < 3; d++) ot.v[a][d] = 0.f;
        }
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            const float bq[3] = {1.f - rule.x[q] - rule.y[q], rule.x[q], rule.y[q]};
#pragma unroll
            for (int d = 0; d < 3; d++) x[q][d] = bary_point(ot, bq, d);
        }
    }
    // packed (the same point in both lanes, negated): D = y_pair + negx
    f2_t negx[NQ][3];
#pragma unroll
    for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int d = 0; d < 3; d++) negx[q][d] = pk(-x[q][d], -x[q][d]);
    // weight products of a non-uniform rule (packed where the registers allow)
    constexpr bool WPACK = !UNIFORM && NQ <= 4;
    f2_t wq2[WPACK ? NQ * NQ : 1];
    float wq[(!UNIFORM && !WPACK) ? NQ * NQ : 1];
#pragma unroll
    for (int q1 = 0; q1 < NQ; q1++)
#pragma unroll
        for (int q2 = 0; q2 < NQ; q2++) {
            const float w = rule.w[q1] * rule.w[q2];
            if constexpr (WPACK) wq2[q1 * NQ + q2] = pk(w, w);
            else if constexpr (!UNIFORM) wq[q1 * NQ + q2] = w;
        }
    const f2_t eps2 = pk(MR_EPS, MR_EPS);

    // Pipeline per tile t: the A values of tile t are generated in registers
    // while the MMAs of tile t - 1 run on the tensor cores and the B tile of t
    // (issued one tile ahead) is in flight; then, once the MMAs of t - 1 have
    // completed, A is stored to shared memory, the B tile of t + 1 is issued
    // into the buffer the MMAs of t - 1 read, and the MMAs of t are issued.
    // (per-buffer state in scalars: a runtime-indexed array would live in local memory)
    uint32_t phase_m = 0, phase_b0 = 0, phase_b1 = 0;
    bool pend0 = false, pend1 = false;  // CTA-uniform: B copies issued, not waited for
    bool ok = true;            // CTA-uniform
    bool mma_pending = false;  // CTA-uniform: a commit not yet waited for
    const uint32_t idesc = mr_instr_desc(N);
    const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    // this warp's tensor-memory columns: whole 8-column groups, split over G
    const int col0 = (grp * (N / 8) / G) * 8, col1 = ((grp + 1) * (N / 8) / G) * 8;
    auto issue_b = [&](int64_t tile, int buf) {
        const uint32_t bar = buf ? barb1 : barb0;
        if (mma_lead) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                         "r"(B_BYTES)
                         : "memory");
            const unsigned char* src =
                reinterpret_cast<const unsigned char*>(Bg) + tile * (int64_t)B_BYTES;
            const uint32_t dst = smem_u32(Bs0) + (uint32_t)buf * B_BYTES;
#pragma unroll
            for (int cpy = 0; cpy < MR_COPIES; cpy++)
                bulk_g2s(dst + cpy * (B_BYTES / MR_COPIES), src + cpy * (B_BYTES / MR_COPIES),
                         B_BYTES / MR_COPIES, bar);
        }
        if (buf) pend1 = true;
        else pend0 = true;
    };
    if (t0 < t1) issue_b(t0, 0);
    for (int64_t t = t0; t < t1; t++) {
        const int buf = (int)((t - t0) & 1);
        // A: this thread's SG source triangles of the tile, KG values, two
        // source triangles per packed instruction (the MMA warp has no rows)
        float av[KG];
#pragma unroll
        for (int sp = 0; sp < (mma_warp ? 0 : SG / 2); sp++) {
            const f2_t* y = reinterpret_cast<const f2_t*>(srcy) +
                            ((t * MR_S + grp * SG) / 2 + sp) * (3 * NQ);
            f2_t T00 = 0ull, T01 = 0ull, T02 = 0ull, T11 = 0ull, T12 = 0ull, T22 = 0ull;
#pragma unroll
            for (int q2 = 0; q2 < NQ; q2++) {
                const f2_t y0 = __ldg(y + 3 * q2), y1 = __ldg(y + 3 * q2 + 1),
                           y2 = __ldg(y + 3 * q2 + 2);
#pragma unroll
                for (int q1 = 0; q1 < NQ; q1++) {
                    const f2_t D0 = add2(y0, negx[q1][0]);
                    const f2_t D1 = add2(y1, negx[q1][1]);
                    const f2_t D2 = add2(y2, negx[q1][2]);
                    f2_t r2 = fma2(D0, D0, eps2);
                    r2 = fma2(D1, D1, r2);
                    r2 = fma2(D2, D2, r2);
                    float ra, rb;
                    upk(r2, ra, rb);
                    const f2_t ir = pk(rsqrtf(ra), rsqrtf(rb));
                    f2_t g = mul2(mul2(ir, ir), ir);
                    if constexpr (WPACK) g = mul2(g, wq2[q1 * NQ + q2]);
                    else if constexpr (!UNIFORM)
                        g = mul2(g, pk(wq[q1 * NQ + q2], wq[q1 * NQ + q2]));
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
            const f2_t Tc[7] = {S0, T00, T01, T02, T11, T12, T22};
#pragma unroll
            for (int c = 0; c < 7; c++) {
                float va, vb;
                upk(Tc[c], va, vb);
                av[7 * (2 * sp) + c] = valid ? va : 0.f;
                av[7 * (2 * sp + 1) + c] = valid ? vb : 0.f;
            }
        }
        // the MMAs of tile t - 1 have read A and B buffer buf ^ 1
        if (mma_pending) {
            // the MMA warp polls; the others wait at the CTA barrier
            const bool w = mma_warp ? mbar_wait(barm, phase_m) : true;
            if (!__syncthreads_and(w)) {
                ok = false;  // the MMAs of the previous tile did not complete in time
                break;
            }
            phase_m ^= 1;
            mma_pending = false;
            if ((t - t0) % MR_FLUSH == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;");
                if (!mma_warp) tmem_fold<N>(lane_base, col0, col1, t - t0 == MR_FLUSH);
                asm volatile("tcgen05.fence::before_thread_sync;");
            }
        }
        if (t + 1 < t1) issue_b(t + 1, buf ^ 1);
        if (mma_warp) {
        } else if constexpr (KG % 4 == 0) {
#pragma unroll
            for (int ch = 0; ch < KG / 4; ch++) {
                float4 h, l;
                h.x = tf32_round(av[4 * ch + 0]);
                h.y = tf32_round(av[4 * ch + 1]);
                h.z = tf32_round(av[4 * ch + 2]);
                h.w = tf32_round(av[4 * ch + 3]);
                l.x = tf32_round(av[4 * ch + 0] - h.x);
                l.y = tf32_round(av[4 * ch + 1] - h.y);
                l.z = tf32_round(av[4 * ch + 2] - h.z);
                l.w = tf32_round(av[4 * ch + 3] - h.w);
                const uint32_t off = mr_off(row, grp * KG + 4 * ch, MR_M);
                *reinterpret_cast<float4*>(Ah + off) = h;
                *reinterpret_cast<float4*>(Al + off) = l;
            }
        } else {  // KG = 14: the group's k range starts at an even k
#pragma unroll
            for (int ch = 0; ch < KG / 2; ch++) {
                float2 h, l;
                h.x = tf32_round(av[2 * ch + 0]);
                h.y = tf32_round(av[2 * ch + 1]);
                l.x = tf32_round(av[2 * ch + 0] - h.x);
                l.y = tf32_round(av[2 * ch + 1] - h.y);
                const uint32_t off = mr_off(row, grp * KG + 2 * ch, MR_M);
                *reinterpret_cast<float2*>(Ah + off) = h;
                *reinterpret_cast<float2*>(Al + off) = l;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        {
            const bool wb = mma_warp ? mbar_wait(buf ? barb1 : barb0, buf ? phase_b1 : phase_b0)
                                     : true;
            if (!__syncthreads_and(wb)) {
                ok = false;
                break;
            }
            if (buf) {
                phase_b1 ^= 1;
                pend1 = false;
            } else {
                phase_b0 ^= 1;
                pend0 = false;
            }
        }
        if (mma_lead) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t lboA = MR_M / 8 * 128, lboB = N / 8 * 128;
            const uint32_t aH = smem_u32(Ah), aL = smem_u32(Al),
                           bH = smem_u32(Bs0) + (uint32_t)buf * B_BYTES,
                           bL = bH + N * MR_K * 4;
#pragma unroll
            for (int ks = 0; ks < MR_KSTEPS; ks++) {
                const uint64_t dAh = mr_smem_desc(aH + 2 * ks * lboA, lboA, 128);
                const uint64_t dAl = mr_smem_desc(aL + 2 * ks * lboA, lboA, 128);
                // D restarts at the first tile of every MR_FLUSH group
                const uint32_t first = ((t - t0) % MR_FLUSH == 0 && ks == 0) ? 0u : 1u;
                const uint64_t dBh = mr_smem_desc(bH + 2 * ks * lboB, lboB, 128);
                const uint64_t dBl = mr_smem_desc(bL + 2 * ks * lboB, lboB, 128);
                mma_tf32(tmem, dAh, dBh, idesc, first);
                mma_tf32(tmem, dAh, dBl, idesc, 1u);
                mma_tf32(tmem, dAl, dBh, idesc, 1u);
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    barm)
                : "memory");
        }
        mma_pending = true;
    }
    if (ok && mma_pending) {
        const bool w = mma_warp ? mbar_wait(barm, phase_m) : true;
        if (!__syncthreads_and(w)) ok = false;
        else mma_pending = false;
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        // one more bounded wait for whatever is still in flight
        if (mma_pending) mbar_wait(barm, phase_m);
        if (pend0) mbar_wait(barb0, phase_b0);
        if (pend1) mbar_wait(barb1, phase_b1);
    }
    asm volatile("tcgen05.fence::after_thread_sync;");

    // epilogue: fold the last group, then S - C of this thread's row and
    // column half -> partial[chunk][r][o][9] (the obs-side contraction
    // out[b][d] = J_o sum_j sc_o[b][j] W[d][j] is done by the reduce kernel)
    if (ok && t1 > t0 && !mma_warp) {
        tmem_fold<N>(lane_base, col0, col1, t1 - t0 <= MR_FLUSH);
#pragma unroll 1
        for (int c0 = col0; c0 < col1; c0 += 8) {
            float sv[8], cv[8];
            tmem_ld8(lane_base + N + c0, sv);
            tmem_ld8(lane_base + 2 * N + c0, cv);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (valid) {
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int n = c0 + u;
                    const int dj = n / R, r = n % R;
                    partial[(((int64_t)blockIdx.y * R + r) * n_obs + o) * 9 + dj] = sv[u] - cv[u];
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(NCOL));
    }
}

// Source quadrature points, padded with far-away points that contribute
// nothing (their A entries are multiplied by zero rows of B).  Layout: pairs
// of consecutive source triangles interleaved, value (q, d) of triangle s at
// srcy[(s / 2) * 6 NQ + 2 (3 q + d) + s % 2], so that one 8-byte load gives
// the packed pair.
template <int NQ>
__global__ void __launch_bounds__(128)
mrhs_points(Rule2D<float> rule, const float* __restrict__ pts,
            const int32_t* __restrict__ src_tris, int64_t n_src, int64_t n_src_pad,
            float* __restrict__ srcy) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_src_pad) return;
    float* y = srcy + (s / 2) * (6 * NQ) + (s % 2);
    if (s >= n_src) {
#pragma unroll
        for (int k = 0; k < 3 * NQ; k++) y[2 * k] = 1e18f;
        return;
    }
    TriGeom<float> t;
    load_tri(t, pts, src_tris, s, 0, false, false);
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        const float bq[3] = {1.f - rule.x[q] - rule.y[q], rule.x[q], rule.y[q]};
#pragma unroll
        for (int d = 0; d < 3; d++) y[2 * (3 * q + d)] = bary_point(t, bq, d);
    }
}

// Sum the chunk partials in a fixed order and apply the obs-side contraction:
// out[r][o][b][d] (+)= J_o sum_j sc_o[b][j] W[r][o][d][j].
__global__ void __launch_bounds__(128)
mrhs_reduce(const float* __restrict__ pts, const int32_t* __restrict__ obs_tris, int64_t n_obs,
            int R, int n_chunks, const float* __restrict__ partial, float* __restrict__ out,
            int accumulate) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_obs * R) return;
    const int64_t o = g % n_obs;
    const int r = (int)(g / n_obs);
    float W[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        float s = 0.f, cmp = 0.f;
        for (int c = 0; c < n_chunks; c++) {
            const float y = partial[(((int64_t)c * R + r) * n_obs + o) * 9 + k] - cmp;
            const float t = s + y;
            cmp = (t - s) - y;
            s = t;
        }
        W[k] = s;
    }
    TriGeom<float> ot;
    load_tri(ot, pts, obs_tris, o, 0, false, true);
    float* op = out + ((int64_t)r * n_obs + o) * 9;
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const float v = ot.J * (ot.sc[b][0] * W[3 * d + 0] + ot.sc[b][1] * W[3 * d + 1] +
                                    ot.sc[b][2] * W[3 * d + 2]);
            op[b * 3 + d] = accumulate ? op[b * 3 + d] + v : v;
        }
}

inline size_t al256(size_t b) { return (b + 255) / 256 * 256; }

int64_t mrhs_chunks(int64_t n_obs, int64_t n_tiles) {
    const int64_t obs_blocks = (n_obs + MR_M - 1) / MR_M;
    // a few waves over the 148 SMs, at least 8 tiles per chunk, at most 64
    int64_t want = (148 * 4 + obs_blocks - 1) / std::max<int64_t>(obs_blocks, 1);
    want = std::max<int64_t>(want, (n_tiles + 511) / 512);  // <= 512 tiles per accumulator
    return std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(want, n_tiles / 8 + 1), 64));
}

struct MrhsSizes {
    size_t B, y, partial, err;
};

MrhsSizes mrhs_sizes(int64_t n_obs, int64_t n_src, int R, int nq) {
    const int64_t n_pad = (n_src + MR_S - 1) / MR_S * MR_S;
    const int64_t n_tiles = n_pad / MR_S;
    MrhsSizes s;
    s.B = al256((size_t)n_tiles * 2 * 9 * R * MR_K * 4);
    s.y = al256((size_t)n_pad * 3 * nq * 4);
    s.partial = al256((size_t)mrhs_chunks(n_obs, n_tiles) * R * n_obs * 9 * 4);
    s.err = 256;
    return s;
}

template <int R, int NQ, bool UNIFORM>
int run_mrhs(const Consts<float>& c, const Rule2D<float>& rule, float* out, const float* in,
             const float* pts, const int32_t* obs_tris, int64_t n_obs, const int32_t* src_tris,
             int64_t n_src, int accumulate, unsigned char* ws, cudaStream_t st) {
    constexpr int N = 9 * R;
    const int64_t n_pad = (n_src + MR_S - 1) / MR_S * MR_S;
    const int64_t n_tiles = n_pad / MR_S;
    const MrhsSizes sz = mrhs_sizes(n_obs, n_src, R, NQ);
    const float w2 = UNIFORM ? rule.w[0] * rule.w[0] : 1.f;
    float* Bg = reinterpret_cast<float*>(ws);
    float* srcy = reinterpret_cast<float*>(ws + sz.B);
    float* partial = reinterpret_cast<float*>(ws + sz.B + sz.y);
    int* err = reinterpret_cast<int*>(ws + sz.B + sz.y + sz.partial);
    if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return launch_status("mrhs memset");
    mrhs_points<NQ><<<(unsigned)((n_pad + 127) / 128), 128, 0, st>>>(rule, pts, src_tris, n_src,
                                                                     n_pad, srcy);
    int rc = launch_status("mrhs points");
    if (rc) return rc;
    mrhs_prep<<<(unsigned)((n_pad * R + 127) / 128), 128, 0, st>>>(c, w2, pts, src_tris, n_src,
                                                                   n_pad, in, R, Bg);
    if ((rc = launch_status("mrhs prep"))) return rc;
    const int64_t chunks = mrhs_chunks(n_obs, n_tiles);
    const int64_t per = (n_tiles + chunks - 1) / chunks;
    const int64_t real = (n_tiles + per - 1) / per;
    const size_t smem = (size_t)2 * MR_M * MR_K * 4 + (size_t)2 * 2 * N * MR_K * 4;
    constexpr int G = 2;  // 8 A-generating warps (16 measured slower: 266 vs 277 applies/s)
    auto kfn = mrhs_main<R, NQ, UNIFORM, G>;
    if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return launch_status("mrhs smem attribute");
    dim3 grid((unsigned)((n_obs + MR_M - 1) / MR_M), (unsigned)real);
    kfn<<<grid, 128 * G + 32, smem, st>>>(rule, pts, obs_tris, n_obs, srcy, n_tiles, per, Bg,
                                        partial, err);
    if ((rc = launch_status("mrhs main"))) return rc;
    mrhs_reduce<<<(unsigned)((n_obs * R + 127) / 128), 128, 0, st>>>(
        pts, obs_tris, n_obs, R, (int)real, partial, out, accumulate);
    return launch_status("mrhs reduce");
}

}  // namespace
}  // namespace tct

using namespace tct;

inline bool mrhs_rule_ok(int nq) { return nq == 3 || nq == 4 || nq == 7; }

extern "C" size_t tct_farfield_rh_panel_workspace_bytes(int64_t n_obs, int64_t n_src, int R,
                                                        int n_q) {
    if (R != 16 || !mrhs_rule_ok(n_q) || n_obs < 0 || n_src < 0) return 0;
    const MrhsSizes s = mrhs_sizes(n_obs, n_src, R, n_q);
    return s.B + s.y + s.partial + s.err;
}

extern "C" int tct_farfield_rh_panel_error(const void* workspace, int64_t n_obs, int64_t n_src,
                                           int R, int n_q, void* stream, int* host_flag) {
    TCT_CHECK_ARG(workspace && host_flag && R == 16 && mrhs_rule_ok(n_q),
                  "tct_farfield_rh_panel_error: bad arguments");
    const MrhsSizes s = mrhs_sizes(n_obs, n_src, R, n_q);
    cudaStream_t st = as_stream(stream);
    if (cudaMemcpyAsync(host_flag, reinterpret_cast<const unsigned char*>(workspace) + s.B + s.y +
                                       s.partial,
                        sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return launch_status("tct_farfield_rh_panel_error");
    return TCT_OK;
}

extern "C" int tct_farfield_rh_panel_matvec(void* out, const void* in, const void* pts,
                                            const int32_t* obs_tris, int64_t n_obs,
                                            const int32_t* src_tris, int64_t n_src, int R,
                                            int n_q, const double* quad_pts,
                                            const double* quad_wts, const double* params,
                                            int accumulate, void* workspace,
                                            size_t workspace_bytes, void* stream) {
    TCT_CHECK_ARG(R == 16, "tct_farfield_rh_panel_matvec: R must be 16 (got %d)", R);
    TCT_CHECK_ARG(mrhs_rule_ok(n_q),
                  "tct_farfield_rh_panel_matvec: %d-point rule (supported: 3, 4, 7)", n_q);
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_farfield_rh_panel_matvec: negative size");
    TCT_CHECK_ARG(params && quad_pts && quad_wts,
                  "tct_farfield_rh_panel_matvec: null params or rule");
    if (n_obs == 0) return TCT_OK;
    const size_t need = tct_farfield_rh_panel_workspace_bytes(n_obs, n_src, R, n_q);
    TCT_CHECK_ARG(workspace && workspace_bytes >= need && aligned(workspace, 256),
                  "tct_farfield_rh_panel_matvec: workspace of %zu bytes (256-aligned) required",
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
            return launch_status("tct_farfield_rh_panel_matvec memset");
        return TCT_OK;
    }
    float* o = (float*)out;
    const float* x = (const float*)in;
    const float* p = (const float*)pts;
#define TCT_MRHS(NQV)                                                                        \
    return uniform ? run_mrhs<16, NQV, true>(c, rule, o, x, p, obs_tris, n_obs, src_tris, n_src, \
                                             accumulate, ws, st)                               \
                   : run_mrhs<16, NQV, false>(c, rule, o, x, p, obs_tris, n_obs, src_tris,       \
                                              n_src, accumulate, ws, st);
    switch (n_q) {
        case 3: TCT_MRHS(3)
        case 4: TCT_MRHS(4)
        default: TCT_MRHS(7)
    }
#undef TCT_MRHS
}
