// Direct farfield: matrix-free tri-to-tri matvec, point-to-point matvec and
// dense farfield blocks.
//
// Tri-to-tri matvec (replaces farfield_tris_to_tris{K}, tectosaur/matrix_free.cl:19-107):
//   out[o, b, d] = sum_s sum_{i,j} J_o J_s w_i w_j phi_b(x_i) v_d(x_i, y_j)
// where v is the kernel's vector form (kernels/__init__.py, kernels/kernels.cl:100-206)
// applied to the source input interpolated at y_j, point pairs with r^2 == 0 skipped.
//
// B200 design:
//  * a prep pass writes one fixed-length record per source triangle: its
//    quadrature points y_j, J_s w_j, and the input-dependent terms the
//    kernel's vector form needs (interpolated input, normal, or the
//    surface-curl contractions of RT/RH), so the point-pair loop reads no
//    geometry and re-derives nothing;
//  * the obs-side basis, weight and Jacobian are factored out of the pair
//    loop: per obs triangle the loop accumulates one small set of sums
//    (3 per obs quadrature point, or the 3x3 W of RH) and the 9 outputs are
//    formed once at the end;
//  * source records are staged through shared memory in tiles and read as
//    warp-wide broadcasts; each tile's sum is added to the running total with
//    Kahan compensation in FP32 ("compensated per-tile sums");
//  * the source range is split into chunks (grid.y) so the grid covers all
//    148 SMs several times over; chunk partials are summed in a fixed order
//    by a second kernel, so results are deterministic.
#include <algorithm>

#include "far_common.cuh"

namespace tct {
namespace {

template <typename R, int K, int NQ, int TS>
__global__ void __launch_bounds__(128)
far_main(Consts<R> c, Rule2D<R> rule, const R* __restrict__ pts,
         const int32_t* __restrict__ obs_tris, int64_t n_obs, const R* __restrict__ rec,
         int64_t n_src, int64_t src_per_chunk, R* __restrict__ dst, int direct,
         int accumulate) {
    using L = Rec<K, NQ>;
    constexpr int NA = NAcc<K, NQ>::n;
    constexpr bool KAHAN = sizeof(R) == 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);

    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n_obs;
    const int64_t s_begin = (int64_t)blockIdx.y * src_per_chunk;
    const int64_t s_end = min(n_src, s_begin + src_per_chunk);

    constexpr bool need_sc = (K == kRA || K == kRH);
    TriGeom<R> o;
    if (valid) {
        load_tri(o, pts, obs_tris, i, 0, false, need_sc);
    } else {
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int d = 0; d < 3; d++) {
                o.v[a][d] = 0;
                o.sc[a][d] = 0;
            }
        o.n[0] = o.n[1] = o.n[2] = 0;
        o.J = 0;
    }
    R x[NQ][3];
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        const R ox = rule.x[q], oy = rule.y[q];
        const R ob[3] = {1 - ox - oy, ox, oy};
#pragma unroll
        for (int d = 0; d < 3; d++) x[q][d] = bary_point(o, ob, d);
    }
    R tot[NA], cmp[NA];
#pragma unroll
    for (int k = 0; k < NA; k++) {
        tot[k] = 0;
        cmp[k] = 0;
    }

    for (int64_t t0 = s_begin; t0 < s_end; t0 += TS) {
        const int n_tile = (int)min((int64_t)TS, s_end - t0);
        __syncthreads();
        {
            // cooperative, vectorised copy of n_tile records into shared memory
            const int n_vec = n_tile * L::LEN / 4;
            if (sizeof(R) == 4) {
                const float4* srcv = reinterpret_cast<const float4*>(rec + t0 * L::LEN);
                float4* dstv = reinterpret_cast<float4*>(sm);
                for (int k = threadIdx.x; k < n_vec; k += blockDim.x) dstv[k] = __ldg(srcv + k);
            } else {
                const double2* srcv = reinterpret_cast<const double2*>(rec + t0 * L::LEN);
                double2* dstv = reinterpret_cast<double2*>(sm);
                for (int k = threadIdx.x; k < 2 * n_vec; k += blockDim.x) dstv[k] = __ldg(srcv + k);
            }
        }
        __syncthreads();
        if (!valid) continue;
        R acc[NA];
#pragma unroll
        for (int k = 0; k < NA; k++) acc[k] = 0;
        for (int j = 0; j < n_tile; j++) {
            far_pair<R, K, NQ>(c, rule, o, x, sm + j * L::LEN, acc);
        }
#pragma unroll
        for (int k = 0; k < NA; k++) fold<R, KAHAN>(tot[k], cmp[k], acc[k]);
    }
    if (!valid) return;

    R out9[9];
    far_epilogue<R, K, NQ>(rule, o, tot, out9);
    if (direct) {
        R* op = dst + i * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) op[k] = accumulate ? op[k] + out9[k] : out9[k];
    } else {
        R* op = dst + ((int64_t)blockIdx.y * n_obs + i) * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) op[k] = out9[k];
    }
}

template <int NQ, bool UNIFORM>
__global__ void __launch_bounds__(128)
far_main_rh2(Consts<float> c, Rule2D<float> rule, const float* __restrict__ pts,
             const int32_t* __restrict__ obs_tris, int64_t n_obs, const float* __restrict__ rec,
             int64_t n_src, int64_t src_per_chunk, float* __restrict__ dst, int direct,
             int accumulate) {
    using L = RecRH2<NQ>;
    constexpr int TS = 128;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sm = reinterpret_cast<float*>(smem_raw);

    // obs triangles a and b of this thread (coalesced: a block covers 256)
    const int64_t ia = (int64_t)blockIdx.x * 256 + threadIdx.x;
    const int64_t ib = ia + 128;
    const bool va = ia < n_obs, vb = ib < n_obs;
    const int64_t s_begin = (int64_t)blockIdx.y * src_per_chunk;
    const int64_t s_end = min(n_src, s_begin + src_per_chunk);

    TriGeom<float> oa, ob;
    if (va) load_tri(oa, pts, obs_tris, ia, 0, false, true);
    if (vb) load_tri(ob, pts, obs_tris, ib, 0, false, true);
    f2_t negx[NQ][3];
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        const float ox = rule.x[q], oy = rule.y[q];
        const float bq[3] = {1 - ox - oy, ox, oy};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const float xa = va ? bary_point(oa, bq, d) : 0.f;
            const float xb = vb ? bary_point(ob, bq, d) : 0.f;
            negx[q][d] = pk(-xa, -xb);
        }
    }
    f2_t wq[UNIFORM ? 1 : NQ * NQ];
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
    float tot[2][9], cmp[2][9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        tot[0][k] = tot[1][k] = 0.f;
        cmp[0][k] = cmp[1][k] = 0.f;
    }

    for (int64_t t0 = s_begin; t0 < s_end; t0 += TS) {
        const int n_tile = (int)min((int64_t)TS, s_end - t0);
        __syncthreads();
        {
            const int n_vec = n_tile * L::LEN / 4;
            const float4* srcv = reinterpret_cast<const float4*>(rec + t0 * L::LEN);
            float4* dstv = reinterpret_cast<float4*>(sm);
            for (int k = threadIdx.x; k < n_vec; k += blockDim.x) dstv[k] = __ldg(srcv + k);
        }
        __syncthreads();
        f2_t W[9];
#pragma unroll
        for (int k = 0; k < 9; k++) W[k] = 0ull;
#pragma unroll 2
        for (int j = 0; j < n_tile; j++) {
            // 16-byte record loads for the 3-point rule (measured faster;
            // the 4- and 7-point forms would need 164-244 registers)
            rh2_pair<NQ, UNIFORM, NQ == 3>(reinterpret_cast<const f2_t*>(sm + j * L::LEN), negx,
                                           wq, eps, W);
        }
#pragma unroll
        for (int k = 0; k < 9; k++) {
            float wa, wb;
            upk(W[k], wa, wb);
            fold<float, true>(tot[0][k], cmp[0][k], wa);
            fold<float, true>(tot[1][k], cmp[1][k], wb);
        }
    }

    // out[b][d] = J_o sum_j sc_o[b][j] W[d][j]
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const bool v = h == 0 ? va : vb;
        if (!v) continue;
        const TriGeom<float>& o = h == 0 ? oa : ob;
        const int64_t i = h == 0 ? ia : ib;
        float out9[9];
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int d = 0; d < 3; d++)
                out9[b * 3 + d] = o.J * (o.sc[b][0] * tot[h][3 * d + 0] + o.sc[b][1] * tot[h][3 * d + 1] +
                                         o.sc[b][2] * tot[h][3 * d + 2]);
        if (direct) {
            float* op = dst + i * 9;
#pragma unroll
            for (int k = 0; k < 9; k++) op[k] = accumulate ? op[k] + out9[k] : out9[k];
        } else {
            float* op = dst + ((int64_t)blockIdx.y * n_obs + i) * 9;
#pragma unroll
            for (int k = 0; k < 9; k++) op[k] = out9[k];
        }
    }
}

template <typename R>
__global__ void chunk_reduce(const R* __restrict__ partial, int n_chunks, int64_t n,
                             R* __restrict__ out, int accumulate) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    R s = accumulate ? out[i] : R(0);
    for (int c = 0; c < n_chunks; c++) s += partial[(int64_t)c * n + i];
    out[i] = s;
}

inline size_t align256(size_t b) { return (b + 255) / 256 * 256; }

int rec_len(int kernel, int nq) {
#define TCT_LEN_CASE(KID)                                                  \
    case KID:                                                              \
        switch (nq) {                                                      \
            case 3: return Rec<KID, 3>::LEN;                               \
            case 4: return Rec<KID, 4>::LEN;                               \
            case 7: return Rec<KID, 7>::LEN;                               \
            case 13: return Rec<KID, 13>::LEN;                             \
            default: return -1;                                            \
        }
    switch (kernel) {
        TCT_LEN_CASE(kU)
        TCT_LEN_CASE(kT)
        TCT_LEN_CASE(kA)
        TCT_LEN_CASE(kH)
        TCT_LEN_CASE(kRT)
        TCT_LEN_CASE(kRA)
        TCT_LEN_CASE(kRH)
        default: return -1;
    }
#undef TCT_LEN_CASE
}

// Number of source chunks: enough (obs-block, chunk) tiles to cover the 148
// SMs about eight times, at least CHUNK_GRAIN sources per chunk (chunks need
// not be whole shared-memory tiles: the main kernels handle a partial last
// tile), at most 32.  Depends only on the problem size, so the workspace size
// is device-independent.
constexpr int64_t CHUNK_GRAIN = 16;
int64_t n_chunks_for(int64_t n_obs, int64_t n_src, int /*ts*/) {
    const int64_t obs_blocks = (n_obs + 127) / 128;
    int64_t want = (148 * 8 + obs_blocks - 1) / std::max<int64_t>(obs_blocks, 1);
    int64_t max_by_src = std::max<int64_t>(1, n_src / CHUNK_GRAIN);
    return std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(want, max_by_src), 32));
}

inline int tile_for(int nq) { return nq <= 4 ? 128 : 32; }

// Largest source-chunk count a launch may use (tuned or not).
constexpr int64_t MAX_CHUNKS = 64;

// Source chunks of a direct-farfield launch: the tuned value of this
// problem's key when the shape cache has one (tune.cu), else the heuristic;
// at most one chunk per CHUNK_GRAIN sources, at most MAX_CHUNKS, and no more
// than the workspace's partial-sum space (after rec_bytes of records) holds.
int64_t choose_chunks(int kernel, int prec, int nq, int64_t n_obs, int64_t n_src,
                      int64_t heuristic, size_t rec_bytes, size_t real_bytes, size_t ws_bytes) {
    int64_t chunks = heuristic;
    int v0 = 0, v1 = 0;
    if (tune_lookup(kTuneFar, kernel, prec, nq, 1, n_obs, n_src, &v0, &v1)) chunks = v0;
    chunks = std::min<int64_t>(chunks, std::max<int64_t>(1, n_src / CHUNK_GRAIN));
    chunks = std::min<int64_t>(chunks, MAX_CHUNKS);
    while (chunks > 1 && rec_bytes + align256(real_bytes * 9 * (size_t)n_obs * chunks) > ws_bytes)
        chunks--;
    return std::max<int64_t>(1, chunks);
}

template <typename R, int K, int NQ>
int run_far(const Consts<R>& c, const Rule2D<R>& rule, R* out, const R* in, const R* pts,
            const int32_t* obs_tris, int64_t n_obs, const int32_t* src_tris, int64_t n_src,
            int accumulate, unsigned char* ws, size_t ws_bytes, cudaStream_t st) {
    using L = Rec<K, NQ>;
    constexpr int TS = NQ <= 4 ? 128 : 32;
    R* rec = reinterpret_cast<R*>(ws);
    const size_t rec_bytes = align256(sizeof(R) * L::LEN * (size_t)n_src);
    far_prep<R, K, NQ><<<(unsigned)((n_src + 127) / 128), 128, 0, st>>>(c, rule, pts, src_tris,
                                                                      n_src, in, nullptr, rec);
    int rc = launch_status("farfield prep");
    if (rc) return rc;
    const int64_t chunks =
        choose_chunks(K, sizeof(R) == 8 ? TCT_F64 : TCT_F32, NQ, n_obs, n_src,
                      n_chunks_for(n_obs, n_src, TS), rec_bytes, sizeof(R), ws_bytes);
    const int64_t per_chunk =
        ((n_src + chunks - 1) / chunks + CHUNK_GRAIN - 1) / CHUNK_GRAIN * CHUNK_GRAIN;
    const int64_t real_chunks = (n_src + per_chunk - 1) / per_chunk;
    const size_t smem = sizeof(R) * L::LEN * TS;
    auto kfn = far_main<R, K, NQ, TS>;
    if (smem > 48 * 1024) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    dim3 grid((unsigned)((n_obs + 127) / 128), (unsigned)real_chunks);
    if (real_chunks == 1) {
        kfn<<<grid, 128, smem, st>>>(c, rule, pts, obs_tris, n_obs, rec, n_src, per_chunk, out, 1,
                                      accumulate);
        return launch_status("farfield main");
    }
    R* partial = reinterpret_cast<R*>(ws + rec_bytes);
    kfn<<<grid, 128, smem, st>>>(c, rule, pts, obs_tris, n_obs, rec, n_src, per_chunk, partial, 0,
                                  0);
    rc = launch_status("farfield main");
    if (rc) return rc;
    const int64_t n = n_obs * 9;
    chunk_reduce<R><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(partial, (int)real_chunks, n, out,
                                                                accumulate);
    return launch_status("farfield chunk reduce");
}

// Source chunks for the packed RH kernel (256 observation triangles per block).
int64_t n_chunks_rh2(int64_t n_obs, int64_t n_src) {
    const int64_t obs_blocks = (n_obs + 255) / 256;
    int64_t want = (148 * 8 + obs_blocks - 1) / std::max<int64_t>(obs_blocks, 1);
    int64_t max_by_src = std::max<int64_t>(1, n_src / CHUNK_GRAIN);
    return std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(want, max_by_src), 32));
}

int rec_len_rh2(int nq) {
    switch (nq) {
        case 3: return RecRH2<3>::LEN;
        case 4: return RecRH2<4>::LEN;
        case 7: return RecRH2<7>::LEN;
        default: return -1;
    }
}

template <int NQ, bool UNIFORM>
int run_far_rh2(const Consts<float>& c, const Rule2D<float>& rule, float* out, const float* in,
                const float* pts, const int32_t* obs_tris, int64_t n_obs,
                const int32_t* src_tris, int64_t n_src, int accumulate, unsigned char* ws,
                size_t ws_bytes, cudaStream_t st) {
    using L = RecRH2<NQ>;
    float* rec = reinterpret_cast<float*>(ws);
    const size_t rec_bytes = align256(sizeof(float) * L::LEN * (size_t)n_src);
    far_prep_rh2<NQ, UNIFORM><<<(unsigned)((n_src + 127) / 128), 128, 0, st>>>(
        c, rule, pts, src_tris, n_src, in, nullptr, rec);
    int rc = launch_status("farfield prep (RH, packed)");
    if (rc) return rc;
    const int64_t chunks = choose_chunks(kRH, TCT_F32, NQ, n_obs, n_src,
                                         n_chunks_rh2(n_obs, n_src), rec_bytes, 4, ws_bytes);
    const int64_t per_chunk =
        ((n_src + chunks - 1) / chunks + CHUNK_GRAIN - 1) / CHUNK_GRAIN * CHUNK_GRAIN;
    const int64_t real_chunks = (n_src + per_chunk - 1) / per_chunk;
    const size_t smem = sizeof(float) * L::LEN * 128;
    auto kfn = far_main_rh2<NQ, UNIFORM>;
    if (smem > 48 * 1024) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    dim3 grid((unsigned)((n_obs + 255) / 256), (unsigned)real_chunks);
    if (real_chunks == 1) {
        kfn<<<grid, 128, smem, st>>>(c, rule, pts, obs_tris, n_obs, rec, n_src, per_chunk, out, 1,
                                      accumulate);
        return launch_status("farfield main (RH, packed)");
    }
    float* partial = reinterpret_cast<float*>(ws + rec_bytes);
    kfn<<<grid, 128, smem, st>>>(c, rule, pts, obs_tris, n_obs, rec, n_src, per_chunk, partial, 0,
                                  0);
    rc = launch_status("farfield main (RH, packed)");
    if (rc) return rc;
    const int64_t n = n_obs * 9;
    chunk_reduce<float><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(partial, (int)real_chunks, n,
                                                                    out, accumulate);
    return launch_status("farfield chunk reduce");
}

int run_far_rh2_nq(int nq, bool uniform, const Consts<float>& c, const Rule2D<float>& rule,
                   float* out, const float* in, const float* pts, const int32_t* ot,
                   int64_t n_obs, const int32_t* stris, int64_t n_src, int acc,
                   unsigned char* ws, size_t ws_bytes, cudaStream_t st) {
#define TCT_RH2(NQV)                                                                          \
    return uniform ? run_far_rh2<NQV, true>(c, rule, out, in, pts, ot, n_obs, stris, n_src, acc, \
                                            ws, ws_bytes, st)                                 \
                   : run_far_rh2<NQV, false>(c, rule, out, in, pts, ot, n_obs, stris, n_src, acc, \
                                             ws, ws_bytes, st);
    switch (nq) {
        case 3: TCT_RH2(3)
        case 4: TCT_RH2(4)
        case 7: TCT_RH2(7)
        default:
            set_error("tct_farfield_tris_matvec: %d-point rule not supported by the packed RH path",
                      nq);
            return TCT_ERR_ARG;
    }
#undef TCT_RH2
}

// The packed FP32 elasticRH3 path serves 3-, 4- and 7-point rules.
inline bool use_rh2(int kernel, int prec, int nq) {
    return kernel == kRH && prec == TCT_F32 && (nq == 3 || nq == 4 || nq == 7);
}

template <typename R, int K>
int run_far_nq(int nq, const Consts<R>& c, const Rule2D<R>& rule, R* out, const R* in,
               const R* pts, const int32_t* ot, int64_t n_obs, const int32_t* stris,
               int64_t n_src, int acc, unsigned char* ws, size_t wsb, cudaStream_t st) {
    switch (nq) {
        case 3: return run_far<R, K, 3>(c, rule, out, in, pts, ot, n_obs, stris, n_src, acc, ws, wsb, st);
        case 4: return run_far<R, K, 4>(c, rule, out, in, pts, ot, n_obs, stris, n_src, acc, ws, wsb, st);
        case 7: return run_far<R, K, 7>(c, rule, out, in, pts, ot, n_obs, stris, n_src, acc, ws, wsb, st);
        case 13: return run_far<R, K, 13>(c, rule, out, in, pts, ot, n_obs, stris, n_src, acc, ws, wsb, st);
        default:
            set_error("tct_farfield_tris_matvec: %d-point triangle rules are not supported "
                      "(supported: 3, 4, 7, 13 = gauss2d_tri(1..4))", nq);
            return TCT_ERR_ARG;
    }
}

template <typename R>
int far_dispatch(int kernel, int nq, const double* qp, const double* qw, const double* params,
                 void* out, const void* in, const void* pts, const int32_t* ot, int64_t n_obs,
                 const int32_t* stris, int64_t n_src, int acc, void* ws, size_t wsb,
                 cudaStream_t st) {
    Consts<R> c = make_consts<R>(params);
    Rule2D<R> rule;
    for (int q = 0; q < MAXQ; q++) {
        rule.x[q] = q < nq ? (R)qp[2 * q] : R(0);
        rule.y[q] = q < nq ? (R)qp[2 * q + 1] : R(0);
        rule.w[q] = q < nq ? (R)qw[q] : R(0);
    }
    unsigned char* w = reinterpret_cast<unsigned char*>(ws);
    if constexpr (sizeof(R) == 4) {
        if (use_rh2(kernel, TCT_F32, nq)) {
            bool uniform = true;
            for (int q = 1; q < nq; q++) uniform = uniform && (qw[q] == qw[0]);
            return run_far_rh2_nq(nq, uniform, c, rule, (float*)out, (const float*)in,
                                  (const float*)pts, ot, n_obs, stris, n_src, acc, w, wsb, st);
        }
    }
#define TCT_FAR_CASE(KID)                                                                 \
    case KID:                                                                               \
        return run_far_nq<R, KID>(nq, c, rule, (R*)out, (const R*)in, (const R*)pts, ot,   \
                                  n_obs, stris, n_src, acc, w, wsb, st);
    switch (kernel) {
        TCT_FAR_CASE(kU)
        TCT_FAR_CASE(kT)
        TCT_FAR_CASE(kA)
        TCT_FAR_CASE(kH)
        TCT_FAR_CASE(kRT)
        TCT_FAR_CASE(kRA)
        TCT_FAR_CASE(kRH)
        default:
            set_error("tct_farfield_tris_matvec: unsupported kernel id %d", kernel);
            return TCT_ERR_KERNEL;
    }
#undef TCT_FAR_CASE
}

// ---- point-to-point farfield (farfield_direct.cl:15-113) --------------------
template <typename R, int K>
__global__ void __launch_bounds__(128)
pts_kernel(Consts<R> c, R* __restrict__ out, const R* __restrict__ obs_pts,
           const R* __restrict__ obs_ns, int64_t n_obs, const R* __restrict__ src_pts,
           const R* __restrict__ src_ns, int64_t n_src, const R* __restrict__ in,
           int64_t src_per_chunk) {
    // grid.y splits the sources into chunks; chunk c writes out + c n_obs 3
    __shared__ R sh[128 * 9];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t s_begin = (int64_t)blockIdx.y * src_per_chunk;
    const int64_t s_end = min(n_src, s_begin + src_per_chunk);
    out += (int64_t)blockIdx.y * n_obs * 3;
    const bool valid = i < n_obs;
    R xo[3] = {0, 0, 0}, no[3] = {0, 0, 0};
    if (valid) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            xo[d] = obs_pts[i * 3 + d];
            no[d] = obs_ns[i * 3 + d];
        }
    }
    R sum[3] = {0, 0, 0};
    for (int64_t t0 = s_begin; t0 < s_end; t0 += 128) {
        const int n_tile = (int)min((int64_t)128, s_end - t0);
        __syncthreads();
        if (threadIdx.x < n_tile) {
            const int64_t j = t0 + threadIdx.x;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                sh[threadIdx.x * 9 + d] = src_pts[j * 3 + d];
                sh[threadIdx.x * 9 + 3 + d] = src_ns[j * 3 + d];
                sh[threadIdx.x * 9 + 6 + d] = in[j * 3 + d];
            }
        }
        __syncthreads();
        if (!valid) continue;
        for (int k = 0; k < n_tile; k++) {
            const R* r = sh + k * 9;
            R D[3] = {r[0] - xo[0], r[1] - xo[1], r[2] - xo[2]};
            R r2 = D[0] * D[0];
            r2 += D[1] * D[1];
            r2 += D[2] * D[2];
            if (r2 == R(0)) continue;
            R v[3];
            vec_utah<R, K>(c, D, r2, no, r + 3, r + 6, v);
            sum[0] += v[0];
            sum[1] += v[1];
            sum[2] += v[2];
        }
    }
    if (valid) {
#pragma unroll
        for (int d = 0; d < 3; d++) out[i * 3 + d] = sum[d];
    }
}

// Source records of the triangle-to-point farfield (matrix_free.cl:109-194):
// per (source triangle, quadrature point) the point y_q, the normal and the
// interpolated input scaled by J_s w_q; the point-to-point kernel then sums
// them in (triangle, point) order, skipping r2 == 0 as the reference does.
template <typename R>
__global__ void __launch_bounds__(128)
tris_to_pts_prep(Rule2D<R> rule, int n_q, const R* __restrict__ pts,
                 const int32_t* __restrict__ tris, int64_t n_src, const R* __restrict__ in,
                 R* __restrict__ yq, R* __restrict__ nq, R* __restrict__ vq) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_src * n_q) return;
    const int64_t j = g / n_q;
    const int q = (int)(g - j * n_q);
    TriGeom<R> t;
    load_tri(t, pts, tris, j, 0, false, false);
    const R x = rule.x[q], y = rule.y[q];
    const R b[3] = {1 - x - y, x, y};
    const R f = t.J * rule.w[q];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        yq[g * 3 + d] = bary_point(t, b, d);
        nq[g * 3 + d] = t.n[d];
        R v = 0;
#pragma unroll
        for (int k = 0; k < 3; k++) v += in[j * 9 + k * 3 + d] * b[k];
        vq[g * 3 + d] = f * v;
    }
}

template <typename R>
int pts_dispatch(int kernel, const double* params, void* out, const void* op, const void* on,
                 int64_t n_obs, const void* sp, const void* sn, int64_t n_src, const void* in,
                 cudaStream_t st, int64_t n_chunks = 1) {
    Consts<R> c = make_consts<R>(params);
    const int64_t per = n_chunks > 1 ? (n_src + n_chunks - 1) / n_chunks : n_src;
    dim3 blocks((unsigned)((n_obs + 127) / 128), (unsigned)std::max<int64_t>(n_chunks, 1));
#define TCT_PTS_CASE(KID)                                                                 \
    case KID:                                                                             \
        pts_kernel<R, KID><<<blocks, 128, 0, st>>>(c, (R*)out, (const R*)op, (const R*)on, \
                                                   n_obs, (const R*)sp, (const R*)sn,     \
                                                   n_src, (const R*)in, per);             \
        break;
    switch (kernel) {
        TCT_PTS_CASE(kU)
        TCT_PTS_CASE(kT)
        TCT_PTS_CASE(kA)
        TCT_PTS_CASE(kH)
        default:
            set_error("tct_farfield_pts: kernel id %d has no point form (surface-curl "
                      "kernels need whole triangles)", kernel);
            return TCT_ERR_KERNEL;
    }
#undef TCT_PTS_CASE
    return launch_status("tct_farfield_pts");
}

// ---- dense farfield blocks (assemble.cl:105-138) ------------------------------
template <typename R, int K>
__global__ void __launch_bounds__(128)
dense_kernel(Consts<R> c, R* __restrict__ out, int n_q, const R* __restrict__ qp,
             const R* __restrict__ qw, const R* __restrict__ pts,
             const int32_t* __restrict__ obs_tris, int64_t n_obs,
             const int32_t* __restrict__ src_tris, int64_t n_src) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_obs * n_src) return;
    const int64_t oi = p / n_src, si = p % n_src;
    TriGeom<R> o, s;
    load_tri(o, pts, obs_tris, oi, 0, false, K == kRA || K == kRH);
    load_tri(s, pts, src_tris, si, 0, false, K == kRT || K == kRH);
    R res[81];
    integrate_pair<R, K, (sizeof(R) == 4) && (K <= kH)>(c, o, s, n_q, qp, qw, false, res);
    const R scale = o.J * s.J;
#pragma unroll
    for (int bo = 0; bo < 3; bo++)
#pragma unroll
        for (int dob = 0; dob < 3; dob++)
#pragma unroll
            for (int bs = 0; bs < 3; bs++)
#pragma unroll
                for (int ds = 0; ds < 3; ds++)
                    out[(oi * 9 + bo * 3 + dob) * n_src * 9 + (si * 9 + bs * 3 + ds)] =
                        scale * res[bo * 27 + dob * 9 + bs * 3 + ds];
}

template <typename R>
int dense_dispatch(int kernel, const double* params, void* out, int n_q, const void* qp,
                   const void* qw, const void* pts, const int32_t* ot, int64_t n_obs,
                   const int32_t* stris, int64_t n_src, cudaStream_t st) {
    Consts<R> c = make_consts<R>(params);
    const int64_t n = n_obs * n_src;
    unsigned blocks = (unsigned)((n + 127) / 128);
#define TCT_DENSE_CASE(KID)                                                               \
    case KID:                                                                             \
        dense_kernel<R, KID><<<blocks, 128, 0, st>>>(c, (R*)out, n_q, (const R*)qp,       \
                                                     (const R*)qw, (const R*)pts, ot,     \
                                                     n_obs, stris, n_src);                \
        break;
    switch (kernel) {
        TCT_DENSE_CASE(kU)
        TCT_DENSE_CASE(kT)
        TCT_DENSE_CASE(kA)
        TCT_DENSE_CASE(kH)
        TCT_DENSE_CASE(kRT)
        TCT_DENSE_CASE(kRA)
        TCT_DENSE_CASE(kRH)
        default:
            set_error("tct_farfield_tris_dense: unsupported kernel id %d", kernel);
            return TCT_ERR_KERNEL;
    }
#undef TCT_DENSE_CASE
    return launch_status("tct_farfield_tris_dense");
}

}  // namespace

// Workspace of a direct-farfield launch: the source records plus the
// partial sums of `max_chunks` source chunks (<= 0: the heuristic count).
size_t farfield_workspace_bytes_chunks(int kernel, int prec, int64_t n_obs, int64_t n_src,
                                       int n_q, int64_t max_chunks) {
    if (n_src < 0 || n_obs < 0) return 0;
    if (use_rh2(kernel, prec, n_q)) {
        const size_t rec_bytes = align256(4 * (size_t)rec_len_rh2(n_q) * (size_t)n_src);
        const int64_t chunks = max_chunks > 0 ? std::min(max_chunks, MAX_CHUNKS)
                                              : n_chunks_rh2(n_obs, n_src);
        const size_t part = chunks > 1 ? align256(4 * 9 * (size_t)n_obs * chunks) : 0;
        return rec_bytes + part;
    }
    const int len = rec_len(kernel, n_q);
    if (len < 0 || n_src < 0 || n_obs < 0) return 0;
    const size_t rs = prec == TCT_F64 ? 8 : 4;
    const size_t rec_bytes = align256(rs * len * (size_t)n_src);
    const int64_t chunks = max_chunks > 0 ? std::min(max_chunks, MAX_CHUNKS)
                                          : n_chunks_for(n_obs, n_src, tile_for(n_q));
    const size_t part = chunks > 1 ? align256(rs * 9 * (size_t)n_obs * chunks) : 0;
    return rec_bytes + part;
}

size_t farfield_workspace_bytes(int kernel, int prec, int64_t n_obs, int64_t n_src, int n_q) {
    return farfield_workspace_bytes_chunks(kernel, prec, n_obs, n_src, n_q, 0);
}

}  // namespace tct

extern "C" size_t tct_farfield_workspace_bytes(int kernel, int prec, int64_t n_obs,
                                               int64_t n_src, int n_q) {
    return tct::farfield_workspace_bytes(kernel, prec, n_obs, n_src, n_q);
}

extern "C" int tct_farfield_tris_matvec(int kernel, int prec, void* out, const void* in,
                                        const void* pts, const int32_t* obs_tris, int64_t n_obs,
                                        const int32_t* src_tris, int64_t n_src, int n_q,
                                        const double* quad_pts, const double* quad_wts,
                                        const double* params, int accumulate, void* workspace,
                                        size_t workspace_bytes, void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_farfield_tris_matvec: negative size");
    TCT_CHECK_ARG(n_obs < (int64_t(1) << 31) && n_src < (int64_t(1) << 31),
                  "tct_farfield_tris_matvec: more than 2^31 triangles");
    TCT_CHECK_ARG(n_q >= 1 && n_q <= 13 && quad_pts && quad_wts && params,
                  "tct_farfield_tris_matvec: bad quadrature rule or params");
    if (n_obs == 0) return TCT_OK;
    TCT_CHECK_ARG(out && pts && obs_tris, "tct_farfield_tris_matvec: null pointer");
    if (n_src == 0) {
        if (!accumulate) {
            cudaMemsetAsync(out, 0, (prec == TCT_F64 ? 8 : 4) * 9 * (size_t)n_obs, as_stream(stream));
            return launch_status("tct_farfield_tris_matvec memset");
        }
        return TCT_OK;
    }
    TCT_CHECK_ARG(in && src_tris && workspace, "tct_farfield_tris_matvec: null pointer");
    TCT_CHECK_ARG(aligned(workspace, 256), "tct_farfield_tris_matvec: workspace not 256-byte aligned");
    const size_t need = farfield_workspace_bytes(kernel, prec, n_obs, n_src, n_q);
    if (need == 0) {
        set_error("tct_farfield_tris_matvec: unsupported kernel %d or %d-point rule", kernel, n_q);
        return TCT_ERR_ARG;
    }
    if (workspace_bytes < need) {
        set_error("tct_farfield_tris_matvec: workspace %zu bytes < required %zu", workspace_bytes, need);
        return TCT_ERR_OOM;
    }
    if (prec == TCT_F32)
        return far_dispatch<float>(kernel, n_q, quad_pts, quad_wts, params, out, in, pts, obs_tris,
                                   n_obs, src_tris, n_src, accumulate, workspace, workspace_bytes,
                                   as_stream(stream));
    if (prec == TCT_F64)
        return far_dispatch<double>(kernel, n_q, quad_pts, quad_wts, params, out, in, pts, obs_tris,
                                    n_obs, src_tris, n_src, accumulate, workspace, workspace_bytes,
                                    as_stream(stream));
    set_error("tct_farfield_tris_matvec: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}

extern "C" int tct_farfield_pts(int kernel, int prec, void* out, const void* obs_pts,
                                const void* obs_ns, int64_t n_obs, const void* src_pts,
                                const void* src_ns, int64_t n_src, const void* in,
                                const double* params, void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_farfield_pts: negative size");
    if (n_obs == 0) return TCT_OK;
    TCT_CHECK_ARG(out && obs_pts && obs_ns && params, "tct_farfield_pts: null pointer");
    TCT_CHECK_ARG(n_src == 0 || (src_pts && src_ns && in), "tct_farfield_pts: null pointer");
    if (prec == TCT_F32)
        return pts_dispatch<float>(kernel, params, out, obs_pts, obs_ns, n_obs, src_pts, src_ns,
                                   n_src, in, as_stream(stream));
    if (prec == TCT_F64)
        return pts_dispatch<double>(kernel, params, out, obs_pts, obs_ns, n_obs, src_pts, src_ns,
                                    n_src, in, as_stream(stream));
    set_error("tct_farfield_pts: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}

namespace tct {
namespace {
// Source chunks of the triangle-to-point farfield: about two blocks per SM
// over the observation blocks, at least 512 source points per chunk, at
// most 64 chunks.
int64_t t2p_chunks(int64_t n_obs, int64_t n_src_pts) {
    const int64_t obs_blocks = std::max<int64_t>((n_obs + 127) / 128, 1);
    int64_t want = (2 * 148 + obs_blocks - 1) / obs_blocks;
    want = std::min<int64_t>(want, std::max<int64_t>(n_src_pts / 512, 1));
    return std::max<int64_t>(1, std::min<int64_t>(want, 64));
}
}  // namespace
}  // namespace tct

extern "C" size_t tct_farfield_tris_to_pts_workspace_bytes(int prec, int64_t n_obs,
                                                           int64_t n_src, int n_q) {
    const size_t r = prec == TCT_F32 ? 4 : 8;
    const int64_t chunks = tct::t2p_chunks(n_obs, n_src * n_q);
    const size_t recs = ((size_t)n_src * n_q * 9 * r + 255) / 256 * 256;
    const size_t part = chunks > 1 ? ((size_t)chunks * n_obs * 3 * r + 255) / 256 * 256 : 0;
    return recs + part + 256;
}

extern "C" int tct_farfield_tris_to_pts(int kernel, int prec, void* out, const void* in,
                                        const void* obs_pts, const void* obs_ns, int64_t n_obs,
                                        const void* pts, const int32_t* src_tris, int64_t n_src,
                                        int n_q, const double* quad_pts, const double* quad_wts,
                                        const double* params, void* workspace,
                                        size_t workspace_bytes, void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_farfield_tris_to_pts: negative size");
    TCT_CHECK_ARG(n_q >= 1 && n_q <= MAXQ, "tct_farfield_tris_to_pts: %d-point rule (1..%d)",
                  n_q, MAXQ);
    if (n_obs == 0) return TCT_OK;
    TCT_CHECK_ARG(out && obs_pts && obs_ns && params && quad_pts && quad_wts,
                  "tct_farfield_tris_to_pts: null pointer");
    const size_t need = tct_farfield_tris_to_pts_workspace_bytes(prec, n_obs, n_src, n_q);
    TCT_CHECK_ARG(n_src == 0 || (workspace && workspace_bytes >= need && aligned(workspace, 256)),
                  "tct_farfield_tris_to_pts: workspace of %zu bytes (256-aligned) required", need);
    cudaStream_t st = as_stream(stream);
    const int64_t m = n_src * n_q;
    const unsigned blocks = (unsigned)((m + 127) / 128);
#define TCT_T2P(R, PREC)                                                                    \
    if (prec == PREC) {                                                                     \
        Rule2D<R> rule;                                                                     \
        for (int q = 0; q < MAXQ; q++) {                                                    \
            rule.x[q] = q < n_q ? (R)quad_pts[2 * q] : R(0);                                \
            rule.y[q] = q < n_q ? (R)quad_pts[2 * q + 1] : R(0);                            \
            rule.w[q] = q < n_q ? (R)quad_wts[q] : R(0);                                    \
        }                                                                                   \
        R* yq = reinterpret_cast<R*>(workspace);                                            \
        R* nq = yq + 3 * m;                                                                 \
        R* vq = nq + 3 * m;                                                                 \
        if (m > 0) {                                                                        \
            tris_to_pts_prep<R><<<blocks, 128, 0, st>>>(rule, n_q, (const R*)pts, src_tris, \
                                                        n_src, (const R*)in, yq, nq, vq);   \
            int rc = launch_status("tct_farfield_tris_to_pts prep");                        \
            if (rc) return rc;                                                              \
        }                                                                                   \
        const int64_t chunks = t2p_chunks(n_obs, m);                                        \
        if (chunks <= 1)                                                                    \
            return pts_dispatch<R>(kernel, params, out, obs_pts, obs_ns, n_obs, yq, nq, m,  \
                                   vq, st);                                                 \
        R* part = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(workspace) +      \
                                       ((size_t)m * 9 * sizeof(R) + 255) / 256 * 256);       \
        int rc = pts_dispatch<R>(kernel, params, part, obs_pts, obs_ns, n_obs, yq, nq, m,   \
                                 vq, st, chunks);                                           \
        if (rc) return rc;                                                                  \
        const int64_t n3 = n_obs * 3;                                                       \
        chunk_reduce<R><<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(part, (int)chunks, n3, \
                                                                     (R*)out, 0);           \
        return launch_status("tct_farfield_tris_to_pts reduce");                            \
    }
    TCT_T2P(float, TCT_F32)
    TCT_T2P(double, TCT_F64)
#undef TCT_T2P
    set_error("tct_farfield_tris_to_pts: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}

extern "C" int tct_farfield_tris_dense(int kernel, int prec, void* out, int n_quad,
                                       const void* quad_pts, const void* quad_wts,
                                       const void* pts, const int32_t* obs_tris, int64_t n_obs,
                                       const int32_t* src_tris, int64_t n_src,
                                       const double* params, void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_farfield_tris_dense: negative size");
    if (n_obs == 0 || n_src == 0) return TCT_OK;
    TCT_CHECK_ARG(n_obs * n_src < (int64_t(1) << 31) * 128, "tct_farfield_tris_dense: too large");
    TCT_CHECK_ARG(out && quad_pts && quad_wts && pts && obs_tris && src_tris && params && n_quad > 0,
                  "tct_farfield_tris_dense: null pointer or empty rule");
    if (prec == TCT_F32)
        return dense_dispatch<float>(kernel, params, out, n_quad, quad_pts, quad_wts, pts, obs_tris,
                                     n_obs, src_tris, n_src, as_stream(stream));
    if (prec == TCT_F64)
        return dense_dispatch<double>(kernel, params, out, n_quad, quad_pts, quad_wts, pts,
                                      obs_tris, n_obs, src_tris, n_src, as_stream(stream));
    set_error("tct_farfield_tris_dense: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}

extern "C" size_t tct_farfield_workspace_bytes_chunks(int kernel, int prec, int64_t n_obs,
                                                      int64_t n_src, int n_q, int max_chunks) {
    return tct::farfield_workspace_bytes_chunks(kernel, prec, n_obs, n_src, n_q, max_chunks);
}

// Candidate source-chunk counts: each is timed (one untimed launch, then the
// mean of three under CUDA events) with the chunk count forced through the
// shape cache; the fastest stays in the cache.
extern "C" int tct_farfield_autotune(int kernel, int prec, void* out, const void* in,
                                     const void* pts, const int32_t* obs_tris, int64_t n_obs,
                                     const int32_t* src_tris, int64_t n_src, int n_q,
                                     const double* quad_pts, const double* quad_wts,
                                     const double* params, void* workspace,
                                     size_t workspace_bytes, void* stream, int* chunks) {
    using namespace tct;
    TCT_CHECK_ARG(chunks, "tct_farfield_autotune: null result pointer");
    TCT_CHECK_ARG(n_obs > 0 && n_src > 0, "tct_farfield_autotune: empty problem");
    static const int kCand[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 48, 64};
    cudaStream_t st = as_stream(stream);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return launch_status("tct_farfield_autotune events");
    int rc = TCT_OK, best = 0;
    float best_ms = 0.f;
    int had0 = 0, had1 = 0;
    const bool had = tune_lookup(kTuneFar, kernel, prec, n_q, 1, n_obs, n_src, &had0, &had1);
    for (int c : kCand) {
        if (c > 1 && c > n_src / CHUNK_GRAIN) break;
        if (c > 1 && farfield_workspace_bytes_chunks(kernel, prec, n_obs, n_src, n_q, c) >
                         workspace_bytes)
            break;  // the workspace holds no more chunk partials
        tune_store(kTuneFar, kernel, prec, n_q, 1, n_obs, n_src, c, 1);
        float ms = 0.f;
        for (int rep = 0; rep < 4 && rc == TCT_OK; rep++) {
            if (rep == 1) cudaEventRecord(e0, st);
            rc = tct_farfield_tris_matvec(kernel, prec, out, in, pts, obs_tris, n_obs, src_tris,
                                          n_src, n_q, quad_pts, quad_wts, params, 0, workspace,
                                          workspace_bytes, stream);
        }
        if (rc != TCT_OK) break;
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = launch_status("tct_farfield_autotune timing");
            break;
        }
        if (best == 0 || ms < best_ms) {
            best = c;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != TCT_OK || best == 0) {
        // leave the cache as it was
        if (had) tune_store(kTuneFar, kernel, prec, n_q, 1, n_obs, n_src, had0, had1);
        else tune_erase(kTuneFar, kernel, prec, n_q, 1, n_obs, n_src);
        return rc != TCT_OK ? rc : TCT_ERR_ARG;
    }
    tune_store(kTuneFar, kernel, prec, n_q, 1, n_obs, n_src, best, 1);
    *chunks = best;
    return TCT_OK;
}
