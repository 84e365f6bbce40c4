// Device half of the near-pair search (mesh/fast_find_nearfield.cpp:22-74,
// 96-141; get_nearfield :255-285).  The host builds the reference's octrees
// and runs its dual traversal down to leaf pairs (tct_near_plan_build,
// host.cpp); here every ball of an obs leaf is tested against the balls of
// its source leaves with the reference's leaf test, in the same double
// arithmetic (no contraction: dist2 is ((dx^2 + dy^2) + dz^2), the limit is
// ((r_i + r_j) thr)^2, a pair is kept unless dist2 > limit), and the radius
// read at the balls' TREE positions, as the reference's leaf loop does.
//
//   near_count   a block per obs leaf, a thread per obs ball: how many
//                sources pass, stored at the ball's original index;
//   (scan)       row offsets over original obs indices;
//   near_fill    the same loops again, writing the passing sources' original
//                indices into the ball's row in test order;
//   (sort)       each row sorted by source index (segmented sort);
//   near_expand  rows written out as (obs, src) pairs.
// The result is the pair set of tct_find_near_pairs in the same canonical
// (obs, src) order, so the two agree bit for bit.
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include "common.cuh"
#include "near_plan.h"

namespace tct {
namespace {

__device__ __forceinline__ bool near_test(const double* __restrict__ ci, double ri,
                                          const double* __restrict__ cj, double rj,
                                          double thr) {
    const double v0 = __dsub_rn(ci[0], cj[0]);
    const double v1 = __dsub_rn(ci[1], cj[1]);
    const double v2 = __dsub_rn(ci[2], cj[2]);
    const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2));
    const double x = __dmul_rn(__dadd_rn(ri, rj), thr);
    return !(d2 > __dmul_rn(x, x));
}

struct NearDev {
    const double *oc, *orq, *sc, *srq;
    const int64_t *oorig, *sorig, *leaf_start, *leaf_end, *lp_start, *lp_s, *lp_e;
};

__global__ void __launch_bounds__(64)
near_count(NearDev d, double thr, int64_t* __restrict__ counts) {
    const int64_t lf = blockIdx.x;
    const int64_t p0 = d.lp_start[lf], p1 = d.lp_start[lf + 1];
    for (int64_t i = d.leaf_start[lf] + threadIdx.x; i < d.leaf_end[lf]; i += blockDim.x) {
        const double ci[3] = {d.oc[3 * i], d.oc[3 * i + 1], d.oc[3 * i + 2]};
        const double ri = d.orq[i];
        int64_t n = 0;
        for (int64_t p = p0; p < p1; p++)
            for (int64_t j = d.lp_s[p]; j < d.lp_e[p]; j++) n += near_test(ci, ri, d.sc + 3 * j, d.srq[j], thr);
        counts[d.oorig[i]] = n;
    }
}

__global__ void __launch_bounds__(64)
near_fill(NearDev d, double thr, const int64_t* __restrict__ offs, int32_t* __restrict__ keys) {
    const int64_t lf = blockIdx.x;
    const int64_t p0 = d.lp_start[lf], p1 = d.lp_start[lf + 1];
    for (int64_t i = d.leaf_start[lf] + threadIdx.x; i < d.leaf_end[lf]; i += blockDim.x) {
        const double ci[3] = {d.oc[3 * i], d.oc[3 * i + 1], d.oc[3 * i + 2]};
        const double ri = d.orq[i];
        int64_t w = offs[d.oorig[i]];
        for (int64_t p = p0; p < p1; p++)
            for (int64_t j = d.lp_s[p]; j < d.lp_e[p]; j++)
                if (near_test(ci, ri, d.sc + 3 * j, d.srq[j], thr)) keys[w++] = (int32_t)d.sorig[j];
    }
}

// a warp per obs row: (obs, src) pairs in row order
__global__ void __launch_bounds__(256)
near_expand(int64_t n_obs, const int64_t* __restrict__ offs, const int32_t* __restrict__ keys,
            int64_t* __restrict__ pairs) {
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n_obs) return;
    for (int64_t k = offs[r] + lane; k < offs[r + 1]; k += 32) {
        pairs[2 * k] = r;
        pairs[2 * k + 1] = keys[k];
    }
}

inline size_t al256(size_t b) { return (b + 255) / 256 * 256; }

template <typename T>
T* carve(unsigned char*& p, size_t count) {
    T* out = reinterpret_cast<T*>(p);
    p += al256(sizeof(T) * count);
    return out;
}

size_t n_leaves(const tct_near_plan* pl) {
    return pl->dev_built ? (size_t)pl->nl_dev : pl->leaf_start.size();
}
size_t n_leaf_pairs(const tct_near_plan* pl) {
    return pl->dev_built ? (size_t)pl->nlp_dev : pl->lp_s.size();
}

NearDev device_view(tct_near_plan* pl) {
    unsigned char* p = static_cast<unsigned char*>(pl->dev);
    NearDev d;
    const size_t nl = n_leaves(pl), nlp = n_leaf_pairs(pl);
    d.oc = carve<double>(p, 3 * pl->n_obs);
    d.orq = carve<double>(p, pl->n_obs);
    d.sc = carve<double>(p, 3 * pl->n_src);
    d.srq = carve<double>(p, pl->n_src);
    d.oorig = carve<int64_t>(p, pl->n_obs);
    d.sorig = carve<int64_t>(p, pl->n_src);
    d.leaf_start = carve<int64_t>(p, nl);
    d.leaf_end = carve<int64_t>(p, nl);
    d.lp_start = carve<int64_t>(p, nl + 1);
    d.lp_s = carve<int64_t>(p, nlp);
    d.lp_e = carve<int64_t>(p, nlp);
    pl->d_counts = carve<int64_t>(p, pl->n_obs + 1);
    return d;
}

size_t device_bytes(const tct_near_plan* pl) {
    const size_t nl = n_leaves(pl), nlp = n_leaf_pairs(pl);
    return al256(8 * 3 * pl->n_obs) + al256(8 * pl->n_obs) + al256(8 * 3 * pl->n_src) +
           al256(8 * pl->n_src) + al256(8 * pl->n_obs) + al256(8 * pl->n_src) + 2 * al256(8 * nl) +
           al256(8 * (nl + 1)) + 2 * al256(8 * nlp) + al256(8 * (pl->n_obs + 1));
}

template <typename T>
int upload(const T* dst, const std::vector<T>& src, cudaStream_t st) {
    if (src.empty()) return TCT_OK;
    if (cudaMemcpyAsync(const_cast<T*>(dst), src.data(), sizeof(T) * src.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess)
        return launch_status("near upload");
    return TCT_OK;
}

}  // namespace

int near_plan_alloc_device(tct_near_plan* plan) {
    if (plan->dev) return TCT_OK;
    plan->dev_bytes = device_bytes(plan);
    if (cudaMalloc(&plan->dev, plan->dev_bytes) != cudaSuccess) {
        plan->dev = nullptr;
        cudaGetLastError();
        set_error("near plan: out of device memory (%zu bytes)", plan->dev_bytes);
        return TCT_ERR_OOM;
    }
    return TCT_OK;
}

NearDevPtrs near_plan_device_ptrs(tct_near_plan* plan) {
    NearDev d = device_view(plan);
    return NearDevPtrs{const_cast<double*>(d.oc), const_cast<double*>(d.orq),
                       const_cast<double*>(d.sc), const_cast<double*>(d.srq),
                       const_cast<int64_t*>(d.oorig), const_cast<int64_t*>(d.sorig),
                       const_cast<int64_t*>(d.leaf_start), const_cast<int64_t*>(d.leaf_end),
                       const_cast<int64_t*>(d.lp_start), const_cast<int64_t*>(d.lp_s),
                       const_cast<int64_t*>(d.lp_e)};
}

}  // namespace tct

using namespace tct;

// Device counting pass: uploads the plan, tests every ball pair of every
// listed leaf pair and forms the row offsets; *total = number of near pairs
// (synchronises the stream).
extern "C" int tct_near_device_count(tct_near_plan* plan, void* stream, int64_t* total) {
    TCT_CHECK_ARG(plan && total, "tct_near_device_count: null pointer");
    cudaStream_t st = as_stream(stream);
    *total = 0;
    plan->total = 0;
    if (plan->n_obs == 0 || plan->n_src == 0) return TCT_OK;
    // source indices are sorted as int32 keys; the scan and sort count in int
    TCT_CHECK_ARG(plan->n_obs < 0x7fffffff && plan->n_src < 0x7fffffff,
                  "tct_near_device_count: more than 2^31 - 2 balls on a side");
    int rc;
    if ((rc = near_plan_alloc_device(plan))) return rc;
    NearDev d = device_view(plan);
    if (!plan->dev_built &&
        ((rc = upload(d.oc, plan->oc, st)) || (rc = upload(d.orq, plan->orq, st)) ||
        (rc = upload(d.sc, plan->sc, st)) || (rc = upload(d.srq, plan->srq, st)) ||
        (rc = upload(d.oorig, plan->oorig, st)) || (rc = upload(d.sorig, plan->sorig, st)) ||
        (rc = upload(d.leaf_start, plan->leaf_start, st)) ||
        (rc = upload(d.leaf_end, plan->leaf_end, st)) ||
        (rc = upload(d.lp_start, plan->lp_start, st)) || (rc = upload(d.lp_s, plan->lp_s, st)) ||
        (rc = upload(d.lp_e, plan->lp_e, st))))
        return rc;
    int64_t* counts = plan->d_counts;
    if (cudaMemsetAsync(counts, 0, sizeof(int64_t) * (plan->n_obs + 1), st) != cudaSuccess)
        return launch_status("near memset");
    const int64_t nl = (int64_t)n_leaves(plan);
    if (nl > 0) {
        near_count<<<(unsigned)nl, 64, 0, st>>>(d, plan->threshold, counts);
        if ((rc = launch_status("near_count"))) return rc;
    }
    // exclusive scan in place over n_obs + 1 entries (the last is 0 -> total)
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts, counts, (int)(plan->n_obs + 1), st);
    void* tmp = nullptr;
    if (cudaMallocAsync(&tmp, tmp_bytes, st) != cudaSuccess) return launch_status("near scan alloc");
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, counts, (int)(plan->n_obs + 1), st);
    rc = launch_status("near scan");
    cudaFreeAsync(tmp, st);
    if (rc) return rc;
    int64_t t = 0;
    if (cudaMemcpyAsync(&t, counts + plan->n_obs, sizeof(int64_t), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return launch_status("near total");
    if (t > (int64_t)0x7fffffff) {
        set_error("tct_near_device_count: %lld pairs exceed the segmented sort's 2^31 limit",
                  (long long)t);
        return TCT_ERR_ARG;
    }
    plan->total = t;
    *total = t;
    return TCT_OK;
}

// Fill pass: pairs (total x 2 int64, device, caller-owned) = the near pairs
// in (obs, src) order.  Requires tct_near_device_count first.
extern "C" int tct_near_device_fill(tct_near_plan* plan, int64_t* pairs, void* stream) {
    TCT_CHECK_ARG(plan, "tct_near_device_fill: null plan");
    TCT_CHECK_ARG(plan->total >= 0, "tct_near_device_fill: run tct_near_device_count first");
    if (plan->total == 0) return TCT_OK;
    TCT_CHECK_ARG(pairs, "tct_near_device_fill: null output");
    cudaStream_t st = as_stream(stream);
    NearDev d = device_view(plan);
    const int64_t total = plan->total;
    const int64_t* offs = plan->d_counts;
    int32_t *keys = nullptr, *sorted = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    cub::DeviceSegmentedSort::SortKeys(nullptr, tmp_bytes, (const int32_t*)nullptr,
                                       (int32_t*)nullptr, (int)total, (int)plan->n_obs, offs,
                                       offs + 1, st);
    if (cudaMallocAsync(&keys, sizeof(int32_t) * total, st) != cudaSuccess ||
        cudaMallocAsync(&sorted, sizeof(int32_t) * total, st) != cudaSuccess ||
        cudaMallocAsync(&tmp, tmp_bytes, st) != cudaSuccess) {
        if (keys) cudaFreeAsync(keys, st);
        if (sorted) cudaFreeAsync(sorted, st);
        cudaGetLastError();
        set_error("tct_near_device_fill: out of device memory");
        return TCT_ERR_OOM;
    }
    int rc = TCT_OK;
    const int64_t nl = (int64_t)n_leaves(plan);
    near_fill<<<(unsigned)nl, 64, 0, st>>>(d, plan->threshold, offs, keys);
    rc = launch_status("near_fill");
    if (!rc) {
        cub::DeviceSegmentedSort::SortKeys(tmp, tmp_bytes, keys, sorted, (int)total,
                                           (int)plan->n_obs, offs, offs + 1, st);
        rc = launch_status("near sort");
    }
    if (!rc) {
        const int64_t threads = plan->n_obs * 32;
        near_expand<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(plan->n_obs, offs, sorted,
                                                                      pairs);
        rc = launch_status("near_expand");
    }
    cudaFreeAsync(tmp, st);
    cudaFreeAsync(sorted, st);
    cudaFreeAsync(keys, st);
    return rc;
}

extern "C" void tct_near_plan_free(tct_near_plan* plan) {
    if (!plan) return;
    if (plan->dev) cudaFree(plan->dev);
    delete plan;
}
