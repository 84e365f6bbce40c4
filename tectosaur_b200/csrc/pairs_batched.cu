// Batched pair quadrature: pairs of every class (coincident, edge-adjacent,
// vertex-adjacent, near) and every quadrature order in ONE persistent launch.
//
// The reference integrates one class at a time with one thread per pair and
// a single rule per launch (nearfield/pairs_integrator.py:43-68), so a launch
// of mixed orders 3..20 would be bound by its largest rule (960,000 points for
// a coincident pair at order 20) on one thread.  Here the host cuts every pair
// into work items of at most `chunk` quadrature points and sorts them by size;
// a persistent grid (a few CTAs per SM) drains two queues with atomic
// counters:
//   * warp items (large rules): the 32 lanes of a warp stride over the item's
//     points, accumulate privately, reduce with shuffles and store (or, when
//     the pair was split over several items, atomically add) the block;
//   * thread items (small rules, whole pairs): one pair per lane, 32 at a time.
// Per-rule flags select the adjacent-pair handling (vertex rotation, source
// flip, output de-rotation; assemble.cl:49-103) and the r^2 == 0 skip.
#include "pair_math.cuh"

namespace tct {
namespace {

constexpr int MAX_PSETS = 8;

template <typename R>
struct ConstSets {
    Consts<R> c[MAX_PSETS];
};

struct BatchArgs {
    const int32_t* pairs;     // n_pairs x 7: obs, src, obs_clicks, src_clicks, flip, rule, pset
    const int64_t* rule_off;  // n_rules + 1 (points)
    const int32_t* rule_flags;  // bit 0: adjacent record, bit 1: skip r^2 == 0
    const int32_t* items;     // n_items x 4: pair, first point, end point, split flag
    int64_t n_warp_items;
    int64_t n_thread_items;
    int* counters;            // 2 ints, zero at launch
    // destination: slot == nullptr -> block of pair p at out + 81 p; else
    // element e of pair p at out[e * slot_stride + slot[p]] (the nearfield
    // BSR's structure-of-arrays blocks)
    const int32_t* slot;
    int64_t slot_stride;
    int add;                  // whole-pair stores add to the destination
    double sign;              // factor on every stored value
};

template <typename R, int K>
__device__ __forceinline__ void load_pair(const BatchArgs& a, const R* pts, const int32_t* tris,
                                          int32_t pair, TriGeom<R>& o, TriGeom<R>& s, int& flags,
                                          int64_t& rule_start, int& pset, int od[3], int sd[3]) {
    const int32_t* rec = a.pairs + 7 * (int64_t)pair;
    const int oi = rec[0], si = rec[1], oc = rec[2], sc = rec[3];
    const bool flip = rec[4] != 0;
    const int rule = rec[5];
    pset = rec[6];
    flags = a.rule_flags[rule];
    rule_start = a.rule_off[rule];
    const bool adj = flags & 1;
    load_tri(o, pts, tris, oi, adj ? oc : 0, false, K == kRA || K == kRH);
    load_tri(s, pts, tris, si, adj ? sc : 0, adj && flip, K == kRT || K == kRH);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        od[k] = adj ? positive_mod(-oc + k, 3) : k;
        sd[k] = adj ? positive_mod(-sc + k, 3) : k;
    }
    if (adj && flip) {
        int t = sd[0];
        sd[0] = sd[1];
        sd[1] = t;
    }
}

// Write (or atomically add) the de-rotated, Jacobian-scaled block; when
// `lane_mask` >= 0 only the outputs idx with idx % 32 == lane_mask are written.
template <typename R>
__device__ __forceinline__ void store_block(const BatchArgs& a, R* out, int32_t pair,
                                            const R res[81], R scale, const int od[3],
                                            const int sd[3], bool atomic, int lane_mask) {
    const int64_t base = a.slot ? (int64_t)__ldg(a.slot + pair) : (int64_t)pair * 81;
    const int64_t step = a.slot ? a.slot_stride : 1;
    scale *= (R)a.sign;
#pragma unroll
    for (int b1 = 0; b1 < 3; b1++)
#pragma unroll
        for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
            for (int b2 = 0; b2 < 3; b2++)
#pragma unroll
                for (int d2 = 0; d2 < 3; d2++) {
                    const int out_idx = b1 * 27 + d1 * 9 + b2 * 3 + d2;
                    if (lane_mask >= 0 && (out_idx & 31) != lane_mask) continue;
                    R val = 0;
#pragma unroll
                    for (int x = 0; x < 3; x++)
#pragma unroll
                        for (int y = 0; y < 3; y++)
                            if (od[b1] == x && sd[b2] == y) val = res[x * 27 + d1 * 9 + y * 3 + d2];
                    R* dst = out + base + (int64_t)out_idx * step;
                    if (atomic) atomicAdd(dst, scale * val);
                    else *dst = a.add ? *dst + scale * val : scale * val;
                }
}

template <typename R, int K>
__global__ void __launch_bounds__(128)
pairs_batched_kernel(const Consts<R>* __restrict__ cs, BatchArgs a, R* __restrict__ out,
                     const R* __restrict__ pts, const int32_t* __restrict__ tris,
                     const R* __restrict__ rule_pts, const R* __restrict__ rule_wts) {
    constexpr bool KAHAN = (sizeof(R) == 4) && (K <= kH);
    const int lane = threadIdx.x & 31;
    // ---- warp items ----
    for (;;) {
        int64_t it = 0;
        if (lane == 0) it = atomicAdd(&a.counters[0], 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= a.n_warp_items) break;
        const int32_t* item = a.items + 4 * it;
        const int32_t pair = item[0];
        const int32_t p0 = item[1], p1 = item[2];
        const bool split = item[3] != 0;
        TriGeom<R> o, s;
        int flags, pset, od[3], sd[3];
        int64_t rs;
        load_pair<R, K>(a, pts, tris, pair, o, s, flags, rs, pset, od, sd);
        const Consts<R> c = cs[pset];
        const bool check0 = (flags & 2) != 0;
        PairAcc<R, K, KAHAN> acc;
        acc.init();
        for (int p = p0 + lane; p < p1; p += 32) {
            const int64_t q = rs + p;
            acc.add(c, o, s, __ldg(rule_pts + 4 * q + 0), __ldg(rule_pts + 4 * q + 1),
                    __ldg(rule_pts + 4 * q + 2), __ldg(rule_pts + 4 * q + 3), __ldg(rule_wts + q),
                    check0);
        }
        acc.warp_reduce();
        R res[81];
        acc.finish(c, o, s, res);
        store_block(a, out, pair, res, o.J * s.J, od, sd, split, lane);
    }
    // ---- thread items: one whole pair per lane ----
    for (;;) {
        int64_t base = 0;
        if (lane == 0) base = atomicAdd(&a.counters[1], 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= a.n_thread_items) break;
        if (base + lane < a.n_thread_items) {
            const int32_t* item = a.items + 4 * (a.n_warp_items + base + lane);
            const int32_t pair = item[0];
            const int32_t p0 = item[1], p1 = item[2];
            TriGeom<R> o, s;
            int flags, pset, od[3], sd[3];
            int64_t rs;
            load_pair<R, K>(a, pts, tris, pair, o, s, flags, rs, pset, od, sd);
            const Consts<R> c = cs[pset];
            const bool check0 = (flags & 2) != 0;
            PairAcc<R, K, KAHAN> acc;
            acc.init();
            for (int p = p0; p < p1; p++) {
                const int64_t q = rs + p;
                acc.add(c, o, s, __ldg(rule_pts + 4 * q + 0), __ldg(rule_pts + 4 * q + 1),
                        __ldg(rule_pts + 4 * q + 2), __ldg(rule_pts + 4 * q + 3),
                        __ldg(rule_wts + q), check0);
            }
            R res[81];
            acc.finish(c, o, s, res);
            store_block(a, out, pair, res, o.J * s.J, od, sd, false, -1);
        }
        __syncwarp();
    }
}

template <typename R>
int launch_batched(int kernel, const double* params, int n_psets, void* out, int64_t n_pairs,
                   const void* pts, const int32_t* tris, const BatchArgs& a, const void* rule_pts,
                   const void* rule_wts, int accumulate, cudaStream_t st) {
    // the kernel constants of each parameter set go to the workspace (after
    // the two queue counters) so the kernel can index them per pair
    ConstSets<R> cs;
    for (int k = 0; k < MAX_PSETS; k++) cs.c[k] = make_consts<R>(params + 2 * (k < n_psets ? k : 0));
    Consts<R>* dcs = reinterpret_cast<Consts<R>*>(reinterpret_cast<unsigned char*>(a.counters) + 256);
    {
        cudaError_t e = cudaMemcpyAsync(dcs, &cs, sizeof(cs), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            set_error("tct_pairs_integrate_batched: constants upload: %s", cudaGetErrorString(e));
            return TCT_ERR_CUDA;
        }
    }
    if (!accumulate && !a.slot) {
        cudaError_t e = cudaMemsetAsync(out, 0, sizeof(R) * 81 * (size_t)n_pairs, st);
        if (e != cudaSuccess) {
            set_error("tct_pairs_integrate_batched: memset: %s", cudaGetErrorString(e));
            return TCT_ERR_CUDA;
        }
    }
    cudaError_t e = cudaMemsetAsync(a.counters, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) {
        set_error("tct_pairs_integrate_batched: memset: %s", cudaGetErrorString(e));
        return TCT_ERR_CUDA;
    }
    const int blocks = sm_count() * 4;
#define TCT_BATCH_CASE(KID)                                                                 \
    case KID:                                                                               \
        pairs_batched_kernel<R, KID><<<blocks, 128, 0, st>>>(dcs, a, (R*)out, (const R*)pts, \
                                                             tris, (const R*)rule_pts,      \
                                                             (const R*)rule_wts);          \
        break;
    switch (kernel) {
        TCT_BATCH_CASE(kU)
        TCT_BATCH_CASE(kT)
        TCT_BATCH_CASE(kA)
        TCT_BATCH_CASE(kH)
        TCT_BATCH_CASE(kRT)
        TCT_BATCH_CASE(kRA)
        TCT_BATCH_CASE(kRH)
        default:
            set_error("tct_pairs_integrate_batched: unsupported kernel id %d", kernel);
            return TCT_ERR_KERNEL;
    }
#undef TCT_BATCH_CASE
    return launch_status("tct_pairs_integrate_batched");
}

}  // namespace
}  // namespace tct

extern "C" int tct_pairs_integrate_batched(int kernel, int prec, void* out, int64_t n_pairs,
                                           const void* pts, const int32_t* tris,
                                           const int32_t* pairs, const int64_t* rule_off,
                                           const int32_t* rule_flags, const void* rule_pts,
                                           const void* rule_wts, const int32_t* items,
                                           int64_t n_warp_items, int64_t n_thread_items,
                                           const double* params, int n_param_sets,
                                           int accumulate, void* workspace,
                                           size_t workspace_bytes, void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(n_pairs >= 0 && n_warp_items >= 0 && n_thread_items >= 0,
                  "tct_pairs_integrate_batched: negative size");
    if (n_pairs == 0) return TCT_OK;
    TCT_CHECK_ARG(n_pairs < (int64_t(1) << 31), "tct_pairs_integrate_batched: too many pairs");
    TCT_CHECK_ARG(out && pts && tris && pairs && rule_off && rule_flags && rule_pts && rule_wts &&
                      params && (items || n_warp_items + n_thread_items == 0),
                  "tct_pairs_integrate_batched: null pointer");
    TCT_CHECK_ARG(n_param_sets >= 1 && n_param_sets <= MAX_PSETS,
                  "tct_pairs_integrate_batched: 1 to %d parameter sets", MAX_PSETS);
    TCT_CHECK_ARG(workspace && workspace_bytes >= 2048 && aligned(workspace, 256),
                  "tct_pairs_integrate_batched: workspace of >= 2048 bytes, 256-byte aligned, "
                  "required");
    BatchArgs a{pairs, rule_off, rule_flags, items, n_warp_items, n_thread_items,
                reinterpret_cast<int*>(workspace), nullptr, 0, 0, 1.0};
    if (prec == TCT_F32)
        return launch_batched<float>(kernel, params, n_param_sets, out, n_pairs, pts, tris, a,
                                     rule_pts, rule_wts, accumulate, as_stream(stream));
    if (prec == TCT_F64)
        return launch_batched<double>(kernel, params, n_param_sets, out, n_pairs, pts, tris, a,
                                      rule_pts, rule_wts, accumulate, as_stream(stream));
    set_error("tct_pairs_integrate_batched: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}

// Slot form (an addition, for the operator build): the same work queues,
// blocks written into a structure-of-arrays block array through a slot map:
// element e of pair p at out[e * slot_stride + slot[p]], times `sign`, added
// to what is there when `add`.  Pairs cut into several warp items (split
// flag) are added atomically, so a plan with split items needs its
// destination slots zeroed (or `add`); a plan without split items is
// deterministic.
extern "C" int tct_pairs_integrate_batched_slots(
    int kernel, int prec, void* out, const int32_t* slot, int64_t slot_stride, double sign,
    int add, int64_t n_pairs, const void* pts, const int32_t* tris, const int32_t* pairs,
    const int64_t* rule_off, const int32_t* rule_flags, const void* rule_pts,
    const void* rule_wts, const int32_t* items, int64_t n_warp_items, int64_t n_thread_items,
    const double* params, int n_param_sets, void* workspace, size_t workspace_bytes,
    void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(n_pairs >= 0 && n_warp_items >= 0 && n_thread_items >= 0 && slot_stride >= 0,
                  "tct_pairs_integrate_batched_slots: negative size");
    if (n_pairs == 0) return TCT_OK;
    TCT_CHECK_ARG(n_pairs < (int64_t(1) << 31) && slot_stride < (int64_t(1) << 31),
                  "tct_pairs_integrate_batched_slots: too many pairs");
    TCT_CHECK_ARG(out && slot && pts && tris && pairs && rule_off && rule_flags && rule_pts &&
                      rule_wts && params && (items || n_warp_items + n_thread_items == 0),
                  "tct_pairs_integrate_batched_slots: null pointer");
    TCT_CHECK_ARG(slot_stride > 0, "tct_pairs_integrate_batched_slots: bad slot stride");
    TCT_CHECK_ARG(n_param_sets >= 1 && n_param_sets <= MAX_PSETS,
                  "tct_pairs_integrate_batched_slots: 1 to %d parameter sets", MAX_PSETS);
    TCT_CHECK_ARG(workspace && workspace_bytes >= 2048 && aligned(workspace, 256),
                  "tct_pairs_integrate_batched_slots: workspace of >= 2048 bytes, 256-byte "
                  "aligned, required");
    BatchArgs a{pairs, rule_off, rule_flags, items, n_warp_items, n_thread_items,
                reinterpret_cast<int*>(workspace), slot, slot_stride, add ? 1 : 0, sign};
    if (prec == TCT_F32)
        return launch_batched<float>(kernel, params, n_param_sets, out, n_pairs, pts, tris, a,
                                     rule_pts, rule_wts, 1, as_stream(stream));
    if (prec == TCT_F64)
        return launch_batched<double>(kernel, params, n_param_sets, out, n_pairs, pts, tris, a,
                                      rule_pts, rule_wts, 1, as_stream(stream));
    set_error("tct_pairs_integrate_batched_slots: unsupported precision %d", prec);
    return TCT_ERR_PREC;
}
