// Multi-RHS point-to-point farfield (elasticU3 / T3 / A3 / H3, FP32) on the
// 5th-generation tensor cores: y_r = K w_r for a panel of R = 16 source
// weight vectors (the reference applies farfield_pts{K} once per vector,
// tectosaur/farfield_direct.cl:15-113, farfield.py:15-38).
//
// Each kernel's vector form is linear in the source weight a
// (kernels/__init__.py:28-36, 67-99, 147-173): v = M(x_i, y_j, n_i, n_j) a
// with a 3x3 matrix M per point pair.  With R weight vectors this is a GEMM
//   Y[i, (d, r)] = sum_{(j, c)} A[i, (j, c)] B[(j, c), (d, r)],
//   A[i, (j, 3d' + k)] = M_{d'k}(i, j),  B[(j, 3d' + k), (d, r)] = [d == d'] w_r[j][k],
// with A generated on the fly by the CUDA cores (never stored in HBM) and B
// built once per apply from the weights (one third of it zeros: N = 3R
// keeps every output component of a row in one accumulator).  Point pairs
// at distance zero contribute nothing (the reference skips r^2 == 0).
// Per CTA: 128 observation points (MMA M) and tiles of 8 source points
// (K = 72); the A-generating warps, the MMA/copy warp, the split-TF32
// products (Ah Bh + Ah Bl + Al Bh), the bounded mbarrier waits, the
// compensated TMEM folds every PM_FLUSH tiles and the fixed-order chunk
// reduction are those of the elasticRH3 triangle panel (far_mrhs.cu);
// see there for the pipeline.
#include <algorithm>

#include "far_common.cuh"
#include "tc_common.cuh"

namespace tct {
namespace {

constexpr int PM_M = TC_M;            // observation points per CTA
constexpr int PM_S = 8;               // source points per tile
constexpr int PM_KC = 9;              // A values per (obs, source) pair
constexpr int PM_K = PM_KC * PM_S;    // 72: GEMM K per tile
constexpr int PM_KSTEPS = PM_K / 8;   // tf32 MMA K = 8
constexpr int PM_R = 16;              // right-hand sides per panel
constexpr int PM_N = 3 * PM_R;        // 48: MMA N
constexpr int PM_FLUSH = 8;           // tiles per tensor-memory accumulation
constexpr int PM_COPIES = 2;          // bulk copies per B tile

// The 3x3 matrix of kernel K at one point pair: v_d = sum_k M[d][k] a_k is
// vec_utah<K> (far_common.cuh) regrouped by the components of a.
template <int K>
__device__ __forceinline__ void kernel_matrix(const Consts<float>& c, const float D[3], float r2,
                                              const float no[3], const float ns[3],
                                              float M[3][3]) {
    const float invr = rsqrtf(r2);
    if (K == kU) {
        const float Q1 = c.CsU0 * invr;
        const float Q2 = c.CsU1 * invr / r2;
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int k = 0; k < 3; k++) M[d][k] = (d == k ? Q1 : 0.f) + Q2 * D[d] * D[k];
    } else if (K == kT || K == kA) {
        const float mp = (K == kT) ? -1.f : 1.f;
        const float pm = (K == kT) ? 1.f : -1.f;
        const float* n = (K == kT) ? ns : no;
        const float invr2 = invr * invr;
        const float invr3 = invr2 * invr;
        const float rn = n[0] * D[0] + n[1] * D[1] + n[2] * D[2];
        const float A = pm * c.CsT0 * invr3;
        const float Cr = mp * c.CsT1 * invr3 * invr2 * rn;
        const float nxdy = n[0] * D[1] - n[1] * D[0];
        const float nzdx = n[2] * D[0] - n[0] * D[2];
        const float nzdy = n[2] * D[1] - n[1] * D[2];
        const float Am[3][3] = {{-rn, mp * nxdy, pm * nzdx},
                                {pm * nxdy, -rn, pm * nzdy},
                                {mp * nzdx, mp * nzdy, -rn}};
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int k = 0; k < 3; k++) M[d][k] = A * Am[d][k] + Cr * D[d] * D[k];
    } else {  // kH
        const float invr2 = invr * invr;
        const float invr3 = invr2 * invr;
        const float rn = invr * (ns[0] * D[0] + ns[1] * D[1] + ns[2] * D[2]);
        const float rm = invr * (no[0] * D[0] + no[1] * D[1] + no[2] * D[2]);
        const float mn = no[0] * ns[0] + no[1] * ns[1] + no[2] * ns[2];
        const float Q = c.CsH0 * invr3;
        const float A = Q * 3 * rn;
        const float B = Q * c.CsH1;
        const float C = Q * c.CsH3;
        const float ST = A * c.nu * rm + B * mn;
        // NT = NTv . a, MT = MTv . a, DT = DTv . a (sn = a.ns, sd = invr a.D, sm = a.no)
        float NTv[3], MTv[3], DTv[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float dk = invr * D[k];
            NTv[k] = B * no[k] + C * rm * dk;
            MTv[k] = Q * c.CsH2 * ns[k] + A * c.CsH1 * dk;
            DTv[k] = invr * (B * 3 * rm * ns[k] + A * c.nu * no[k] + (C * mn - A * 5 * rm) * dk);
        }
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int k = 0; k < 3; k++)
                M[d][k] = ns[d] * NTv[k] + no[d] * MTv[k] + D[d] * DTv[k] + (d == k ? ST : 0.f);
    }
}

// B panel: per source point and RHS, the 9 x 48 GEMM rows (hi and lo TF32
// parts, canonical K-major layout, tile after tile).  One thread per
// (padded source point, r).
__global__ void __launch_bounds__(128)
pts_panel_prep(const float* __restrict__ w, int64_t n_src, int64_t n_pad, float* __restrict__ Bg) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_pad * PM_R) return;
    const int64_t j = g / PM_R;
    const int r = (int)(g % PM_R);
    float a[3] = {0.f, 0.f, 0.f};
    if (j < n_src) {
#pragma unroll
        for (int k = 0; k < 3; k++) a[k] = w[((int64_t)r * n_src + j) * 3 + k];
    }
    const int64_t tile = j / PM_S;
    const int jl = (int)(j % PM_S);
    unsigned char* base =
        reinterpret_cast<unsigned char*>(Bg) + tile * (int64_t)2 * PM_N * PM_K * 4;
#pragma unroll
    for (int dd = 0; dd < 3; dd++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int kk = PM_KC * jl + 3 * dd + k;
            const float hi = tf32_round(a[k]);
            const float lo = tf32_round(a[k] - hi);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const int n = d * PM_R + r;
                const uint32_t off = mr_off(n, kk, PM_N);
                *reinterpret_cast<float*>(base + off) = d == dd ? hi : 0.f;
                *reinterpret_cast<float*>(base + (int64_t)PM_N * PM_K * 4 + off) =
                    d == dd ? lo : 0.f;
            }
        }
}

// Source points and normals packed 6 floats per point, padded with points
// far away (their B rows are zero).
__global__ void __launch_bounds__(128)
pts_panel_points(const float* __restrict__ pts, const float* __restrict__ ns, int64_t n_src,
                 int64_t n_pad, float* __restrict__ sp) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_pad) return;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        sp[6 * j + d] = j < n_src ? pts[3 * j + d] : 1e18f;
        sp[6 * j + 3 + d] = j < n_src ? ns[3 * j + d] : 0.f;
    }
}

template <int K, int G>
__global__ void __launch_bounds__(128 * G + 32, 1)
pts_panel_main(Consts<float> c, const float* __restrict__ obs_pts,
               const float* __restrict__ obs_ns, int64_t n_obs, const float* __restrict__ sp,
               int64_t n_tiles, int64_t tiles_per_chunk, const float* __restrict__ Bg,
               float* __restrict__ partial, int* __restrict__ err) {
    constexpr int N = PM_N;
    constexpr int SG = PM_S / G;   // source points per thread group
    constexpr int KG = PM_KC * SG; // A values per thread and tile
    static_assert(3 * N <= 512, "D, S and C must fit the 512 tensor-memory columns");
    static_assert(PM_S % G == 0 && KG % 4 == 0, "tile split");
    constexpr int NCOL = 256;
    constexpr uint32_t B_BYTES = 2u * N * PM_K * 4;
    static_assert(B_BYTES % (16 * PM_COPIES) == 0, "bulk copies must be 16-byte multiples");
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* Ah = smem;
    unsigned char* Al = Ah + PM_M * PM_K * 4;
    unsigned char* Bs0 = Al + PM_M * PM_K * 4;
    __shared__ __align__(8) uint64_t bar_mma;
    __shared__ __align__(8) uint64_t bar_b[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int tid = threadIdx.x;
    if (tid == 0) abort_flag = *reinterpret_cast<volatile int*>(err);
    __syncthreads();
    if (abort_flag) return;
    const int warp = tid >> 5;
    const int row = tid & (PM_M - 1);
    const int grp = tid >> 7;
    const bool mma_warp = warp == 4 * G;
    const bool mma_lead = tid == 128 * G;
    const int64_t i = (int64_t)blockIdx.x * PM_M + row;
    const bool valid = i < n_obs;
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

    float xo[3] = {0.f, 0.f, 0.f}, no[3] = {0.f, 0.f, 0.f};
    if (valid) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            xo[d] = obs_pts[3 * i + d];
            no[d] = obs_ns[3 * i + d];
        }
    }

    uint32_t phase_m = 0, phase_b0 = 0, phase_b1 = 0;
    bool pend0 = false, pend1 = false;
    bool ok = true;
    bool mma_pending = false;
    const uint32_t idesc = mr_instr_desc(N);
    const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
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
            for (int cpy = 0; cpy < PM_COPIES; cpy++)
                bulk_g2s(dst + cpy * (B_BYTES / PM_COPIES), src + cpy * (B_BYTES / PM_COPIES),
                         B_BYTES / PM_COPIES, bar);
        }
        if (buf) pend1 = true;
        else pend0 = true;
    };
    if (t0 < t1) issue_b(t0, 0);
    for (int64_t t = t0; t < t1; t++) {
        const int buf = (int)((t - t0) & 1);
        // A: this thread's SG source points of the tile, 9 values each
        float av[KG];
#pragma unroll
        for (int p = 0; p < (mma_warp ? 0 : SG); p++) {
            const float* s = sp + 6 * (t * PM_S + grp * SG + p);
            const float D[3] = {__ldg(s) - xo[0], __ldg(s + 1) - xo[1], __ldg(s + 2) - xo[2]};
            const float ns[3] = {__ldg(s + 3), __ldg(s + 4), __ldg(s + 5)};
            float r2 = D[0] * D[0];
            r2 += D[1] * D[1];
            r2 += D[2] * D[2];
            float M[3][3];
            kernel_matrix<K>(c, D, r2, no, ns, M);
            const bool use = valid && r2 != 0.f;
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int k = 0; k < 3; k++) av[PM_KC * p + 3 * d + k] = use ? M[d][k] : 0.f;
        }
        if (mma_pending) {
            const bool w = mma_warp ? mbar_wait(barm, phase_m) : true;
            if (!__syncthreads_and(w)) {
                ok = false;
                break;
            }
            phase_m ^= 1;
            mma_pending = false;
            if ((t - t0) % PM_FLUSH == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;");
                if (!mma_warp) tmem_fold<N>(lane_base, col0, col1, t - t0 == PM_FLUSH);
                asm volatile("tcgen05.fence::before_thread_sync;");
            }
        }
        if (t + 1 < t1) issue_b(t + 1, buf ^ 1);
        if (!mma_warp) {
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
                const uint32_t off = mr_off(row, grp * KG + 4 * ch, PM_M);
                *reinterpret_cast<float4*>(Ah + off) = h;
                *reinterpret_cast<float4*>(Al + off) = l;
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
            const uint32_t lboA = PM_M / 8 * 128, lboB = N / 8 * 128;
            const uint32_t aH = smem_u32(Ah), aL = smem_u32(Al),
                           bH = smem_u32(Bs0) + (uint32_t)buf * B_BYTES,
                           bL = bH + N * PM_K * 4;
#pragma unroll
            for (int ks = 0; ks < PM_KSTEPS; ks++) {
                const uint64_t dAh = mr_smem_desc(aH + 2 * ks * lboA, lboA, 128);
                const uint64_t dAl = mr_smem_desc(aL + 2 * ks * lboA, lboA, 128);
                const uint32_t first = ((t - t0) % PM_FLUSH == 0 && ks == 0) ? 0u : 1u;
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
        if (mma_pending) mbar_wait(barm, phase_m);
        if (pend0) mbar_wait(barb0, phase_b0);
        if (pend1) mbar_wait(barb1, phase_b1);
    }
    asm volatile("tcgen05.fence::after_thread_sync;");

    // epilogue: fold the last group, then S - C of this row -> partial[chunk][r][i][d]
    if (ok && t1 > t0 && !mma_warp) {
        tmem_fold<N>(lane_base, col0, col1, t1 - t0 <= PM_FLUSH);
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
                    const int d = n / PM_R, r = n % PM_R;
                    partial[(((int64_t)blockIdx.y * PM_R + r) * n_obs + i) * 3 + d] =
                        sv[u] - cv[u];
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

// Chunk partials summed in a fixed order (compensated): out[r][i][d] (+)=.
__global__ void __launch_bounds__(128)
pts_panel_reduce(int64_t n_obs, int n_chunks, const float* __restrict__ partial,
                 float* __restrict__ out, int accumulate) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_obs * PM_R * 3) return;
    float s = 0.f, cmp = 0.f;
    for (int c = 0; c < n_chunks; c++) {
        const float y = partial[(int64_t)c * PM_R * n_obs * 3 + g] - cmp;
        const float t = s + y;
        cmp = (t - s) - y;
        s = t;
    }
    out[g] = accumulate ? out[g] + s : s;
}

inline size_t al256(size_t b) { return (b + 255) / 256 * 256; }

int64_t pts_panel_chunks(int64_t n_obs, int64_t n_tiles) {
    const int64_t obs_blocks = (n_obs + PM_M - 1) / PM_M;
    int64_t want = (148 * 4 + obs_blocks - 1) / std::max<int64_t>(obs_blocks, 1);
    want = std::max<int64_t>(want, (n_tiles + 511) / 512);  // <= 512 tiles per accumulator
    return std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(want, n_tiles / 8 + 1), 64));
}

struct PtsPanelSizes {
    size_t B, sp, partial, err;
};

PtsPanelSizes pts_panel_sizes(int64_t n_obs, int64_t n_src) {
    const int64_t n_pad = (n_src + PM_S - 1) / PM_S * PM_S;
    const int64_t n_tiles = n_pad / PM_S;
    PtsPanelSizes s;
    s.B = al256((size_t)n_tiles * 2 * PM_N * PM_K * 4);
    s.sp = al256((size_t)n_pad * 6 * 4);
    s.partial = al256((size_t)pts_panel_chunks(n_obs, n_tiles) * PM_R * n_obs * 3 * 4);
    s.err = 256;
    return s;
}

template <int K>
int run_pts_panel(const Consts<float>& c, float* out, const float* w, const float* obs_pts,
                  const float* obs_ns, int64_t n_obs, const float* src_pts, const float* src_ns,
                  int64_t n_src, int accumulate, unsigned char* ws, cudaStream_t st) {
    const int64_t n_pad = (n_src + PM_S - 1) / PM_S * PM_S;
    const int64_t n_tiles = n_pad / PM_S;
    const PtsPanelSizes sz = pts_panel_sizes(n_obs, n_src);
    float* Bg = reinterpret_cast<float*>(ws);
    float* sp = reinterpret_cast<float*>(ws + sz.B);
    float* partial = reinterpret_cast<float*>(ws + sz.B + sz.sp);
    int* err = reinterpret_cast<int*>(ws + sz.B + sz.sp + sz.partial);
    if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess)
        return launch_status("pts panel memset");
    pts_panel_points<<<(unsigned)((n_pad + 127) / 128), 128, 0, st>>>(src_pts, src_ns, n_src,
                                                                       n_pad, sp);
    int rc = launch_status("pts panel points");
    if (rc) return rc;
    pts_panel_prep<<<(unsigned)((n_pad * PM_R + 127) / 128), 128, 0, st>>>(w, n_src, n_pad, Bg);
    if ((rc = launch_status("pts panel prep"))) return rc;
    const int64_t chunks = pts_panel_chunks(n_obs, n_tiles);
    const int64_t per = (n_tiles + chunks - 1) / chunks;
    const int64_t real = (n_tiles + per - 1) / per;
    const size_t smem = (size_t)2 * PM_M * PM_K * 4 + (size_t)2 * 2 * PM_N * PM_K * 4;
    constexpr int G = 2;
    auto kfn = pts_panel_main<K, G>;
    if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return launch_status("pts panel smem attribute");
    dim3 grid((unsigned)((n_obs + PM_M - 1) / PM_M), (unsigned)real);
    kfn<<<grid, 128 * G + 32, smem, st>>>(c, obs_pts, obs_ns, n_obs, sp, n_tiles, per, Bg, partial,
                                        err);
    if ((rc = launch_status("pts panel main"))) return rc;
    const int64_t n_out = n_obs * PM_R * 3;
    pts_panel_reduce<<<(unsigned)((n_out + 127) / 128), 128, 0, st>>>(n_obs, (int)real, partial,
                                                                      out, accumulate);
    return launch_status("pts panel reduce");
}

}  // namespace
}  // namespace tct

using namespace tct;

extern "C" size_t tct_farfield_pts_panel_workspace_bytes(int64_t n_obs, int64_t n_src, int R) {
    if (R != PM_R || n_obs < 0 || n_src < 0) return 0;
    const PtsPanelSizes s = pts_panel_sizes(n_obs, n_src);
    return s.B + s.sp + s.partial + s.err;
}

extern "C" int tct_farfield_pts_panel_error(const void* workspace, int64_t n_obs, int64_t n_src,
                                            int R, void* stream, int* host_flag) {
    TCT_CHECK_ARG(workspace && host_flag && R == PM_R, "tct_farfield_pts_panel_error: bad arguments");
    const PtsPanelSizes s = pts_panel_sizes(n_obs, n_src);
    cudaStream_t st = as_stream(stream);
    if (cudaMemcpyAsync(host_flag,
                        reinterpret_cast<const unsigned char*>(workspace) + s.B + s.sp + s.partial,
                        sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return launch_status("tct_farfield_pts_panel_error");
    return TCT_OK;
}

extern "C" int tct_farfield_pts_panel(int kernel, void* out, const void* in, const void* obs_pts,
                                      const void* obs_ns, int64_t n_obs, const void* src_pts,
                                      const void* src_ns, int64_t n_src, int R,
                                      const double* params, int accumulate, void* workspace,
                                      size_t workspace_bytes, void* stream) {
    TCT_CHECK_ARG(R == PM_R, "tct_farfield_pts_panel: R must be %d (got %d)", PM_R, R);
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_farfield_pts_panel: negative size");
    TCT_CHECK_ARG(n_obs < (int64_t(1) << 31) && n_src < (int64_t(1) << 31),
                  "tct_farfield_pts_panel: more than 2^31 points");
    TCT_CHECK_ARG(params, "tct_farfield_pts_panel: null params");
    if (n_obs == 0) return TCT_OK;
    TCT_CHECK_ARG(out && obs_pts && obs_ns, "tct_farfield_pts_panel: null pointer");
    cudaStream_t st = as_stream(stream);
    if (n_src == 0) {
        if (!accumulate &&
            cudaMemsetAsync(out, 0, sizeof(float) * 3 * n_obs * PM_R, st) != cudaSuccess)
            return launch_status("tct_farfield_pts_panel memset");
        return TCT_OK;
    }
    TCT_CHECK_ARG(in && src_pts && src_ns, "tct_farfield_pts_panel: null pointer");
    const size_t need = tct_farfield_pts_panel_workspace_bytes(n_obs, n_src, R);
    TCT_CHECK_ARG(workspace && workspace_bytes >= need && aligned(workspace, 256),
                  "tct_farfield_pts_panel: workspace of %zu bytes (256-aligned) required", need);
    const Consts<float> c = make_consts<float>(params);
    unsigned char* ws = reinterpret_cast<unsigned char*>(workspace);
    float* o = (float*)out;
    const float *w = (const float*)in, *op = (const float*)obs_pts, *on = (const float*)obs_ns,
                *sp = (const float*)src_pts, *sn = (const float*)src_ns;
    switch (kernel) {
        case kU: return run_pts_panel<kU>(c, o, w, op, on, n_obs, sp, sn, n_src, accumulate, ws, st);
        case kT: return run_pts_panel<kT>(c, o, w, op, on, n_obs, sp, sn, n_src, accumulate, ws, st);
        case kA: return run_pts_panel<kA>(c, o, w, op, on, n_obs, sp, sn, n_src, accumulate, ws, st);
        case kH: return run_pts_panel<kH>(c, o, w, op, on, n_obs, sp, sn, n_src, accumulate, ws, st);
        default:
            set_error("tct_farfield_pts_panel: kernel id %d has no point form", kernel);
            return TCT_ERR_KERNEL;
    }
}
