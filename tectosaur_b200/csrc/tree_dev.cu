// The near-pair search's octrees and dual traversal on the device.
//
// The reference builds its ball octree recursively on the host
// (fmm/octree.cpp:27-76, with the bounds of fmm/tree_helpers.hpp) and runs
// the dual-tree ball query there (mesh/fast_find_nearfield.cpp:22-74, 96-141);
// host.cpp restates both step for step.  Here the same tree is built level by
// level on the device and is equal to the host tree node for node:
//
//  * a node's bounds are the centre of mass of its ball centres -- summed in
//    tree order by one thread, in the host's order and rounding (no
//    contraction: adds, one division) -- and the radius max(|c - com| + r);
//    an empty child takes (parent centre, parent R / 50), a one-ball child
//    the ball itself; the root's bounds are computed on the host;
//  * a node with more than `leaf` balls (and depth < 60) splits into 8
//    octants (x bit 2, y bit 1, z bit 0, "greater than" = 1), stably: a
//    block per splitting node counts the octants, then scatters its range
//    chunk by chunk with ballot ranks, in order;
//  * nodes are numbered breadth first on the device; tct_tree_build_device
//    renumbers them depth-first (the host tree's order) when it exports.
//
// The dual traversal runs breadth first over (obs node, src node) pairs with
// the reference's node test (expanded radii, ((r1 + r2) thr)^2 against the
// squared centre distance, the same split rule), in a count pass and a write
// pass per level, down to leaf pairs, which are grouped by obs leaf; the
// ball tests, row fill and row sort that follow are near.cu's.  The set of
// leaf pairs is the host traversal's, so the pairs are the same, in the same
// canonical (obs, src) order.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "near_plan.h"
#include "octree.h"

namespace tct {
namespace {

constexpr int TREE_MAX_DEPTH = 60;

__device__ __forceinline__ double ddist2(const double* a, const double* b) {
    const double v0 = __dsub_rn(a[0], b[0]);
    const double v1 = __dsub_rn(a[1], b[1]);
    const double v2 = __dsub_rn(a[2], b[2]);
    return __dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2));
}

__device__ __forceinline__ int octant_of(const double* p, const double* c) {
    int o = 0;
    o = (o | (p[0] > c[0] ? 1 : 0)) << 1;
    o = (o | (p[1] > c[1] ? 1 : 0)) << 1;
    o = o | (p[2] > c[2] ? 1 : 0);
    return o;
}

// Device arrays of one tree under construction (nodes breadth first).
struct DTree {
    int64_t n = 0, n_nodes = 0, cap = 0;
    double *c = nullptr, *r = nullptr;   // balls, tree order (3 / 1 per ball)
    int64_t* orig = nullptr;
    double *c2 = nullptr, *r2 = nullptr;  // partition targets
    int64_t* orig2 = nullptr;
    int64_t *ns = nullptr, *ne = nullptr, *child0 = nullptr;
    double *nc = nullptr, *nR = nullptr, *er = nullptr;
    int32_t *depth = nullptr, *leaf = nullptr;
};

template <typename T>
int dalloc(T** p, size_t count, cudaStream_t st) {
    *p = nullptr;
    if (count == 0) count = 1;
    if (cudaMallocAsync(reinterpret_cast<void**>(p), sizeof(T) * count, st) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        set_error("device octree: out of device memory (%zu bytes)", sizeof(T) * count);
        return TCT_ERR_OOM;
    }
    return TCT_OK;
}

template <typename T>
void dfree(T*& p, cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
}

void free_tree(DTree& t, cudaStream_t st) {
    dfree(t.c, st); dfree(t.r, st); dfree(t.orig, st);
    dfree(t.c2, st); dfree(t.r2, st); dfree(t.orig2, st);
    dfree(t.ns, st); dfree(t.ne, st); dfree(t.child0, st);
    dfree(t.nc, st); dfree(t.nR, st); dfree(t.er, st);
    dfree(t.depth, st); dfree(t.leaf, st);
}

int alloc_nodes(DTree& t, int64_t cap, cudaStream_t st) {
    int rc;
    if ((rc = dalloc(&t.ns, cap, st)) || (rc = dalloc(&t.ne, cap, st)) ||
        (rc = dalloc(&t.child0, cap, st)) || (rc = dalloc(&t.nc, 3 * cap, st)) ||
        (rc = dalloc(&t.nR, cap, st)) || (rc = dalloc(&t.depth, cap, st)) ||
        (rc = dalloc(&t.leaf, cap, st)))
        return rc;
    t.cap = cap;
    return TCT_OK;
}

// grow the node arrays to `cap` (copying the first n_nodes)
int grow_nodes(DTree& t, int64_t cap, cudaStream_t st) {
    DTree o = t;
    int rc = alloc_nodes(t, cap, st);
    if (rc) return rc;
    const size_t k = (size_t)t.n_nodes;
    cudaMemcpyAsync(t.ns, o.ns, 8 * k, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(t.ne, o.ne, 8 * k, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(t.child0, o.child0, 8 * k, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(t.nc, o.nc, 24 * k, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(t.nR, o.nR, 8 * k, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(t.depth, o.depth, 4 * k, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(t.leaf, o.leaf, 4 * k, cudaMemcpyDeviceToDevice, st);
    dfree(o.ns, st); dfree(o.ne, st); dfree(o.child0, st); dfree(o.nc, st);
    dfree(o.nR, st); dfree(o.depth, st); dfree(o.leaf, st);
    return launch_status("device octree grow");
}

// leaf flags of nodes [lo, hi) and their split flags (for the scan)
__global__ void level_flags(int64_t lo, int64_t hi, int64_t leaf_size,
                            const int64_t* __restrict__ ns, const int64_t* __restrict__ ne,
                            const int32_t* __restrict__ depth, int32_t* __restrict__ leaf,
                            int64_t* __restrict__ child0, int32_t* __restrict__ split) {
    const int64_t k = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= hi) return;
    const bool lf = (ne[k] - ns[k] <= leaf_size) || depth[k] >= TREE_MAX_DEPTH;
    leaf[k] = lf ? 1 : 0;
    child0[k] = -1;
    split[k - lo] = lf ? 0 : 1;
}

// splitting node of each rank
__global__ void split_nodes(int64_t lo, int64_t m, const int32_t* __restrict__ split,
                            const int32_t* __restrict__ rank, int64_t* __restrict__ node_of) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && split[i]) node_of[rank[i]] = lo + i;
}

// a block per splitting node: ball counts per octant
__global__ void __launch_bounds__(256)
octant_count(const int64_t* __restrict__ node_of, const int64_t* __restrict__ ns,
             const int64_t* __restrict__ ne, const double* __restrict__ nc,
             const double* __restrict__ c, int64_t* __restrict__ cnt) {
    __shared__ unsigned long long sc[8];
    const int64_t k = node_of[blockIdx.x];
    if (threadIdx.x < 8) sc[threadIdx.x] = 0;
    __syncthreads();
    const double cc[3] = {nc[3 * k], nc[3 * k + 1], nc[3 * k + 2]};
    unsigned long long loc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t i = ns[k] + threadIdx.x; i < ne[k]; i += blockDim.x) loc[octant_of(c + 3 * i, cc)]++;
#pragma unroll
    for (int o = 0; o < 8; o++)
        if (loc[o]) atomicAdd(&sc[o], loc[o]);
    __syncthreads();
    if (threadIdx.x < 8) cnt[8 * (int64_t)blockIdx.x + threadIdx.x] = (int64_t)sc[threadIdx.x];
}

// a block per splitting node: the stable octant partition of its range,
// chunk by chunk in order (rank of a ball = balls of its octant before it)
__global__ void __launch_bounds__(256)
octant_scatter(const int64_t* __restrict__ node_of, const int64_t* __restrict__ ns,
               const int64_t* __restrict__ ne, const double* __restrict__ nc,
               const int64_t* __restrict__ cnt, const double* __restrict__ c,
               const double* __restrict__ r, const int64_t* __restrict__ orig,
               double* __restrict__ c2, double* __restrict__ r2, int64_t* __restrict__ orig2) {
    __shared__ int64_t base[8];
    __shared__ int wcnt[8][8];  // [warp][octant]
    const int64_t k = node_of[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        int64_t s = ns[k];
        for (int o = 0; o < 8; o++) {
            base[o] = s;
            s += cnt[8 * (int64_t)blockIdx.x + o];
        }
    }
    const double cc[3] = {nc[3 * k], nc[3 * k + 1], nc[3 * k + 2]};
    const int64_t s0 = ns[k], e0 = ne[k];
    __syncthreads();
    for (int64_t ch = s0; ch < e0; ch += blockDim.x) {
        const int64_t i = ch + threadIdx.x;
        const bool valid = i < e0;
        const int o = valid ? octant_of(c + 3 * i, cc) : -1;
        int my_rank = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const unsigned m = __ballot_sync(0xffffffffu, o == q);
            if (o == q) my_rank = __popc(m & ((1u << lane) - 1u));
            if (lane == 0) wcnt[warp][q] = __popc(m);
        }
        __syncthreads();
        if (valid) {
            int64_t dst = base[o] + my_rank;
            for (int w = 0; w < warp; w++) dst += wcnt[w][o];
            c2[3 * dst] = c[3 * i];
            c2[3 * dst + 1] = c[3 * i + 1];
            c2[3 * dst + 2] = c[3 * i + 2];
            r2[dst] = r[i];
            orig2[dst] = orig[i];
        }
        __syncthreads();
        if (threadIdx.x < 8) {
            int64_t t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += wcnt[w][threadIdx.x];
            base[threadIdx.x] += t;
        }
        __syncthreads();
    }
}

// a thread per child (rank, octant): its range and bounds (the balls are
// already in the partitioned order)
__global__ void make_children(int64_t n_split, int64_t first_child,
                              const int64_t* __restrict__ node_of, const int64_t* __restrict__ cnt,
                              const double* __restrict__ c, const double* __restrict__ r,
                              int64_t* __restrict__ ns, int64_t* __restrict__ ne,
                              int64_t* __restrict__ child0, double* __restrict__ nc,
                              double* __restrict__ nR, int32_t* __restrict__ depth) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= 8 * n_split) return;
    const int64_t j = g >> 3;
    const int o = (int)(g & 7);
    const int64_t k = node_of[j];
    int64_t cs = ns[k];
    for (int q = 0; q < o; q++) cs += cnt[8 * j + q];
    const int64_t ce = cs + cnt[8 * j + o];
    const int64_t ch = first_child + 8 * j + o;
    if (o == 0) child0[k] = first_child + 8 * j;
    ns[ch] = cs;
    ne[ch] = ce;
    depth[ch] = depth[k] + 1;
    double cc[3], cr;
    if (ce == cs) {
        cc[0] = nc[3 * k]; cc[1] = nc[3 * k + 1]; cc[2] = nc[3 * k + 2];
        cr = __ddiv_rn(nR[k], 50.0);
    } else if (ce - cs == 1) {
        cc[0] = c[3 * cs]; cc[1] = c[3 * cs + 1]; cc[2] = c[3 * cs + 2];
        cr = r[cs];
    } else {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int64_t i = cs; i < ce; i++) {
            s0 = __dadd_rn(s0, c[3 * i]);
            s1 = __dadd_rn(s1, c[3 * i + 1]);
            s2 = __dadd_rn(s2, c[3 * i + 2]);
        }
        const double cnt_d = (double)(ce - cs);
        cc[0] = __ddiv_rn(s0, cnt_d);
        cc[1] = __ddiv_rn(s1, cnt_d);
        cc[2] = __ddiv_rn(s2, cnt_d);
        double m = 0.0;
        for (int64_t i = cs; i < ce; i++) {
            const double v = __dadd_rn(__dsqrt_rn(ddist2(c + 3 * i, cc)), r[i]);
            m = fmax(m, v);
        }
        cr = m;
    }
    nc[3 * ch] = cc[0];
    nc[3 * ch + 1] = cc[1];
    nc[3 * ch + 2] = cc[2];
    nR[ch] = cr;
}

// a block per node: the radius that covers every member ball
// (fast_find_nearfield.cpp:77-94)
__global__ void __launch_bounds__(256)
expanded_radii(const int64_t* __restrict__ ns, const int64_t* __restrict__ ne,
               const double* __restrict__ nc, const double* __restrict__ nR,
               const double* __restrict__ c, const double* __restrict__ r,
               double* __restrict__ er) {
    __shared__ double red[256];
    const int64_t k = blockIdx.x;
    const double cc[3] = {nc[3 * k], nc[3 * k + 1], nc[3 * k + 2]};
    double m = nR[k];
    for (int64_t i = ns[k] + threadIdx.x; i < ne[k]; i += blockDim.x)
        m = fmax(m, __dadd_rn(__dsqrt_rn(ddist2(c + 3 * i, cc)), r[i]));
    red[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) er[k] = red[0];
}

// Host bounds of all n balls (the root), in the host builder's arithmetic.
void root_bounds(const double* c, const double* r, int64_t n, double* cc, double* R) {
    if (n == 0) {
        cc[0] = cc[1] = cc[2] = 0.0;
        *R = 1.0;
        return;
    }
    if (n == 1) {
        cc[0] = c[0]; cc[1] = c[1]; cc[2] = c[2];
        *R = r[0];
        return;
    }
    double com[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) com[d] += c[3 * i + d];
    for (int d = 0; d < 3; d++) com[d] /= (double)n;
    double m = 0.0;
    for (int64_t i = 0; i < n; i++) {
        double d2 = 0;
        for (int d = 0; d < 3; d++) {
            const double v = c[3 * i + d] - com[d];
            d2 += v * v;
        }
        m = std::max(m, std::sqrt(d2) + r[i]);
    }
    for (int d = 0; d < 3; d++) cc[d] = com[d];
    *R = m;
}

template <typename T>
int scan_exclusive(const T* in, T* out, int64_t m, cudaStream_t st) {
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, in, out, (int)m, st);
    void* tmp = nullptr;
    if (cudaMallocAsync(&tmp, std::max<size_t>(tmp_bytes, 1), st) != cudaSuccess) {
        cudaGetLastError();
        set_error("device octree: out of device memory (scan)");
        return TCT_ERR_OOM;
    }
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, (int)m, st);
    cudaFreeAsync(tmp, st);
    return launch_status("device octree scan");
}

template <typename T>
int read_back(const T* dev, T* host, cudaStream_t st) {
    if (cudaMemcpyAsync(host, dev, sizeof(T), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return launch_status("device octree read-back");
    return TCT_OK;
}

// Build the tree of n balls (host arrays) on the device, nodes breadth
// first, plus the expanded node radii.
int build_dtree(const double* h_c, const double* h_r, int64_t n, int64_t leaf_size,
                cudaStream_t st, DTree& t) {
    int rc;
    t.n = n;
    if ((rc = dalloc(&t.c, 3 * n, st)) || (rc = dalloc(&t.r, n, st)) ||
        (rc = dalloc(&t.orig, n, st)) || (rc = dalloc(&t.c2, 3 * n, st)) ||
        (rc = dalloc(&t.r2, n, st)) || (rc = dalloc(&t.orig2, n, st)))
        return rc;
    if (n > 0) {
        std::vector<int64_t> iota(n);
        for (int64_t i = 0; i < n; i++) iota[i] = i;
        if (cudaMemcpyAsync(t.c, h_c, 24 * (size_t)n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(t.r, h_r, 8 * (size_t)n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(t.orig, iota.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return launch_status("device octree upload");
    }
    if ((rc = alloc_nodes(t, std::max<int64_t>(1024, 1 + 8 * (n / 16)), st))) return rc;
    {
        double cc[3], R;
        root_bounds(h_c, h_r, n, cc, &R);
        const int64_t s = 0, e = n;
        const int32_t d = 0;
        cudaMemcpyAsync(t.ns, &s, 8, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(t.ne, &e, 8, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(t.nc, cc, 24, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(t.nR, &R, 8, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(t.depth, &d, 4, cudaMemcpyHostToDevice, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return launch_status("device octree root");
    }
    t.n_nodes = 1;
    int64_t lo = 0, hi = 1;
    while (hi > lo) {
        const int64_t m = hi - lo;
        int32_t *split = nullptr, *rank = nullptr;
        int64_t *node_of = nullptr, *cnt = nullptr;
        if ((rc = dalloc(&split, m, st)) || (rc = dalloc(&rank, m, st))) return rc;
        const unsigned nb = (unsigned)((m + 255) / 256);
        level_flags<<<nb, 256, 0, st>>>(lo, hi, leaf_size, t.ns, t.ne, t.depth, t.leaf, t.child0,
                                        split);
        if ((rc = launch_status("level_flags"))) return rc;
        if ((rc = scan_exclusive(split, rank, m, st))) return rc;
        int32_t last_rank = 0, last_split = 0;
        if ((rc = read_back(rank + m - 1, &last_rank, st)) ||
            (rc = read_back(split + m - 1, &last_split, st)))
            return rc;
        const int64_t n_split = (int64_t)last_rank + last_split;
        if (n_split == 0) {
            dfree(split, st);
            dfree(rank, st);
            break;
        }
        if (hi + 8 * n_split > t.cap &&
            (rc = grow_nodes(t, std::max<int64_t>(2 * t.cap, hi + 8 * n_split), st)))
            return rc;
        if ((rc = dalloc(&node_of, n_split, st)) || (rc = dalloc(&cnt, 8 * n_split, st)))
            return rc;
        split_nodes<<<nb, 256, 0, st>>>(lo, m, split, rank, node_of);
        if ((rc = launch_status("split_nodes"))) return rc;
        octant_count<<<(unsigned)n_split, 256, 0, st>>>(node_of, t.ns, t.ne, t.nc, t.c, cnt);
        if ((rc = launch_status("octant_count"))) return rc;
        // balls of nodes that do not split keep their places
        cudaMemcpyAsync(t.c2, t.c, 24 * (size_t)n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(t.r2, t.r, 8 * (size_t)n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(t.orig2, t.orig, 8 * (size_t)n, cudaMemcpyDeviceToDevice, st);
        octant_scatter<<<(unsigned)n_split, 256, 0, st>>>(node_of, t.ns, t.ne, t.nc, cnt, t.c, t.r,
                                                          t.orig, t.c2, t.r2, t.orig2);
        if ((rc = launch_status("octant_scatter"))) return rc;
        std::swap(t.c, t.c2);
        std::swap(t.r, t.r2);
        std::swap(t.orig, t.orig2);
        make_children<<<(unsigned)((8 * n_split + 127) / 128), 128, 0, st>>>(
            n_split, hi, node_of, cnt, t.c, t.r, t.ns, t.ne, t.child0, t.nc, t.nR, t.depth);
        if ((rc = launch_status("make_children"))) return rc;
        dfree(split, st);
        dfree(rank, st);
        dfree(node_of, st);
        dfree(cnt, st);
        lo = hi;
        hi = hi + 8 * n_split;
        t.n_nodes = hi;
    }
    if ((rc = dalloc(&t.er, t.n_nodes, st))) return rc;
    expanded_radii<<<(unsigned)t.n_nodes, 256, 0, st>>>(t.ns, t.ne, t.nc, t.nR, t.c, t.r, t.er);
    return launch_status("expanded_radii");
}

// ---- dual traversal to leaf pairs ----------------------------------------------
struct TravArgs {
    const int64_t *ons, *one, *oc0, *sns, *sne, *sc0;
    const double *onc, *oer, *snc, *ser;
    const int32_t *oleaf, *sleaf;
    double thr;
};

// what pair i becomes: 0 pruned, 1 a leaf pair, 2 eight child pairs
__device__ __forceinline__ int trav_decide(const TravArgs& a, int32_t on, int32_t sn,
                                          bool* split_src) {
    const double r1 = a.oer[on], r2 = a.ser[sn];
    const double x = __dmul_rn(__dadd_rn(r1, r2), a.thr);
    if (ddist2(a.onc + 3 * (int64_t)on, a.snc + 3 * (int64_t)sn) > __dmul_rn(x, x)) return 0;
    const bool ol = a.oleaf[on] != 0, sl = a.sleaf[sn] != 0;
    if (ol && sl) return 1;
    *split_src = ((r1 < r2) && !sl) || ol;
    return 2;
}

__global__ void trav_count(TravArgs a, const int32_t* __restrict__ fr, int64_t m,
                           int32_t* __restrict__ n_leaf, int32_t* __restrict__ n_next) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    bool ss = false;
    const int d = trav_decide(a, fr[2 * i], fr[2 * i + 1], &ss);
    n_leaf[i] = d == 1 ? 1 : 0;
    n_next[i] = d == 2 ? 8 : 0;
}

__global__ void trav_write(TravArgs a, const int32_t* __restrict__ fr, int64_t m,
                           const int32_t* __restrict__ off_leaf,
                           const int32_t* __restrict__ off_next, int32_t* __restrict__ leaf_out,
                           int32_t* __restrict__ next) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int32_t on = fr[2 * i], sn = fr[2 * i + 1];
    bool ss = false;
    const int d = trav_decide(a, on, sn, &ss);
    if (d == 1) {
        leaf_out[2 * (int64_t)off_leaf[i]] = on;
        leaf_out[2 * (int64_t)off_leaf[i] + 1] = sn;
    } else if (d == 2) {
        int32_t* p = next + 2 * (int64_t)off_next[i];
        for (int k = 0; k < 8; k++) {
            p[2 * k] = ss ? on : (int32_t)(a.oc0[on] + k);
            p[2 * k + 1] = ss ? (int32_t)(a.sc0[sn] + k) : sn;
        }
    }
}

// grouped leaf pairs -> the plan's obs-leaf and source-leaf ranges
__global__ void group_leaf_pairs(int64_t nlp, const int32_t* __restrict__ okey,
                                 const int32_t* __restrict__ sval,
                                 const int32_t* __restrict__ seg,
                                 const int64_t* __restrict__ ons, const int64_t* __restrict__ one,
                                 const int64_t* __restrict__ sns, const int64_t* __restrict__ sne,
                                 int64_t* __restrict__ leaf_start, int64_t* __restrict__ leaf_end,
                                 int64_t* __restrict__ lp_start, int64_t* __restrict__ lp_s,
                                 int64_t* __restrict__ lp_e) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nlp) return;
    const int32_t o = okey[i];
    if (i == 0 || okey[i - 1] != o) {
        const int32_t g = seg[i];
        leaf_start[g] = ons[o];
        leaf_end[g] = one[o];
        lp_start[g] = i;
    }
    lp_s[i] = sns[sval[i]];
    lp_e[i] = sne[sval[i]];
}

__global__ void new_segment_flags(int64_t nlp, const int32_t* __restrict__ okey,
                                  int32_t* __restrict__ flag) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nlp) flag[i] = (i == 0 || okey[i - 1] != okey[i]) ? 1 : 0;
}

int traverse_leaf_pairs(const DTree& ot, const DTree& stt, double thr, cudaStream_t st,
                        int32_t** out_pairs, int64_t* out_n) {
    *out_pairs = nullptr;
    *out_n = 0;
    TravArgs a{ot.ns, ot.ne, ot.child0, stt.ns, stt.ne, stt.child0, ot.nc, ot.er,
               stt.nc, stt.er, ot.leaf, stt.leaf, thr};
    int rc;
    int32_t* fr = nullptr;
    int64_t m = 1;
    if ((rc = dalloc(&fr, 2, st))) return rc;
    const int32_t root[2] = {0, 0};
    cudaMemcpyAsync(fr, root, 8, cudaMemcpyHostToDevice, st);
    std::vector<int32_t*> parts;
    std::vector<int64_t> part_n;
    int64_t total = 0;
    while (m > 0) {
        if (m > 0x7fffffff / 8) {
            set_error("near traversal: frontier of %lld pairs too large", (long long)m);
            rc = TCT_ERR_ARG;
            break;
        }
        int32_t *nl = nullptr, *nn = nullptr, *ol = nullptr, *on = nullptr;
        if ((rc = dalloc(&nl, m, st)) || (rc = dalloc(&nn, m, st)) || (rc = dalloc(&ol, m, st)) ||
            (rc = dalloc(&on, m, st)))
            break;
        const unsigned nb = (unsigned)((m + 255) / 256);
        trav_count<<<nb, 256, 0, st>>>(a, fr, m, nl, nn);
        if ((rc = launch_status("trav_count"))) break;
        if ((rc = scan_exclusive(nl, ol, m, st)) || (rc = scan_exclusive(nn, on, m, st))) break;
        int32_t lo_l = 0, lo_n = 0, la_l = 0, la_n = 0;
        if ((rc = read_back(ol + m - 1, &lo_l, st)) || (rc = read_back(on + m - 1, &lo_n, st)) ||
            (rc = read_back(nl + m - 1, &la_l, st)) || (rc = read_back(nn + m - 1, &la_n, st)))
            break;
        const int64_t n_leaf = (int64_t)lo_l + la_l, n_next = ((int64_t)lo_n + la_n) / 8;
        int32_t *lout = nullptr, *next = nullptr;
        if ((rc = dalloc(&lout, 2 * n_leaf, st)) || (rc = dalloc(&next, 16 * n_next, st))) break;
        trav_write<<<nb, 256, 0, st>>>(a, fr, m, ol, on, lout, next);
        if ((rc = launch_status("trav_write"))) break;
        dfree(nl, st); dfree(nn, st); dfree(ol, st); dfree(on, st);
        dfree(fr, st);
        fr = next;
        m = 8 * n_next;
        if (n_leaf > 0) {
            parts.push_back(lout);
            part_n.push_back(n_leaf);
            total += n_leaf;
        } else {
            dfree(lout, st);
        }
    }
    dfree(fr, st);
    if (rc == TCT_OK && total > 0x7fffffff) {
        set_error("near traversal: %lld leaf pairs exceed 2^31", (long long)total);
        rc = TCT_ERR_ARG;
    }
    int32_t* all = nullptr;
    if (rc == TCT_OK && (rc = dalloc(&all, 2 * std::max<int64_t>(total, 1), st)) == TCT_OK) {
        int64_t at = 0;
        for (size_t k = 0; k < parts.size(); k++) {
            cudaMemcpyAsync(all + 2 * at, parts[k], 8 * (size_t)part_n[k],
                            cudaMemcpyDeviceToDevice, st);
            at += part_n[k];
        }
        rc = launch_status("near traversal gather");
    }
    for (auto* p : parts) dfree(p, st);
    if (rc != TCT_OK) {
        dfree(all, st);
        return rc;
    }
    *out_pairs = all;
    *out_n = total;
    return TCT_OK;
}

__global__ void split_pairs(int64_t n, const int32_t* __restrict__ p, int32_t* __restrict__ o,
                            int32_t* __restrict__ s) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        o[i] = p[2 * i];
        s[i] = p[2 * i + 1];
    }
}

}  // namespace

// The plan's device arrays from device-built trees (near.cu's layout).
int near_plan_fill_device(tct_near_plan* plan, const DTree& ot, const DTree& stt,
                          const double* obs_r, const double* src_r, cudaStream_t st);

}  // namespace tct

using namespace tct;

namespace {

// Depth-first renumbering of a breadth-first device tree into the host
// builder's Octree (same node order, same arrays).
int export_dtree(const DTree& t, cudaStream_t st, Octree& out) {
    const int64_t nn = t.n_nodes, n = t.n;
    std::vector<int64_t> ns(nn), ne(nn), c0(nn);
    std::vector<double> nc(3 * nn), nR(nn);
    std::vector<int32_t> depth(nn), leaf(nn);
    out.centers.resize(3 * n);
    out.radii.resize(n);
    out.orig.resize(n);
    cudaMemcpyAsync(ns.data(), t.ns, 8 * nn, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(ne.data(), t.ne, 8 * nn, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(c0.data(), t.child0, 8 * nn, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(nc.data(), t.nc, 24 * nn, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(nR.data(), t.nR, 8 * nn, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(depth.data(), t.depth, 4 * nn, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(leaf.data(), t.leaf, 4 * nn, cudaMemcpyDeviceToHost, st);
    if (n > 0) {
        cudaMemcpyAsync(out.centers.data(), t.c, 24 * n, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(out.radii.data(), t.r, 8 * n, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(out.orig.data(), t.orig, 8 * n, cudaMemcpyDeviceToHost, st);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return launch_status("device octree export");
    // subtree sizes (children after their parent in breadth-first order)
    std::vector<int64_t> sz(nn, 1), pre(nn, 0);
    for (int64_t k = nn - 1; k >= 0; k--)
        if (!leaf[k])
            for (int q = 0; q < 8; q++) sz[k] += sz[c0[k] + q];
    for (int64_t k = 0; k < nn; k++)
        if (!leaf[k]) {
            int64_t at = pre[k] + 1;
            for (int q = 0; q < 8; q++) {
                pre[c0[k] + q] = at;
                at += sz[c0[k] + q];
            }
        }
    out.nodes.assign(nn, OctNode{});
    for (int64_t k = 0; k < nn; k++) {
        OctNode& d = out.nodes[pre[k]];
        d.start = ns[k];
        d.end = ne[k];
        for (int q = 0; q < 3; q++) d.c[q] = nc[3 * k + q];
        d.R = nR[k];
        d.leaf = leaf[k] != 0;
        d.depth = depth[k];
        for (int q = 0; q < 8; q++) d.child[q] = d.leaf ? -1 : pre[c0[k] + q];
    }
    return TCT_OK;
}

int node_height_of(tct_tree& tr, int64_t k) {
    const OctNode& n = tr.t.nodes[k];
    if (n.leaf) return tr.height[k] = 0;
    int h = 0;
    for (int c = 0; c < 8; c++) h = std::max(h, node_height_of(tr, n.child[c]));
    return tr.height[k] = h + 1;
}

}  // namespace

// Device build of the ball octree (the tree of tct_tree_build, node for
// node), exported to a host tct_tree.
extern "C" int tct_tree_build_device(const double* centers, const double* radii, int64_t n,
                                     int64_t leaf_size, void* stream, tct_tree** out) {
    if (!out || n < 0 || leaf_size < 1 || (n > 0 && (!centers || !radii))) {
        set_error("tct_tree_build_device: bad arguments");
        return TCT_ERR_ARG;
    }
    *out = nullptr;
    cudaStream_t st = as_stream(stream);
    DTree t;
    int rc = build_dtree(centers, radii, n, leaf_size, st, t);
    auto* tr = new tct_tree();
    if (rc == TCT_OK) rc = export_dtree(t, st, tr->t);
    free_tree(t, st);
    cudaStreamSynchronize(st);
    if (rc != TCT_OK) {
        delete tr;
        return rc;
    }
    tr->height.assign(tr->t.nodes.size(), 0);
    tr->max_height = node_height_of(*tr, 0);
    *out = tr;
    return TCT_OK;
}

// The near-pair search plan built entirely on the device: octrees, expanded
// radii, dual traversal to leaf pairs and their grouping; then
// tct_near_device_count / _fill as for a host-built plan.
extern "C" int tct_near_plan_build_device(const double* obs_c, const double* obs_r, int64_t n_obs,
                                          const double* src_c, const double* src_r,
                                          int64_t n_src, double threshold, void* stream,
                                          tct_near_plan** out) {
    if (!out) {
        set_error("tct_near_plan_build_device: null output handle");
        return TCT_ERR_ARG;
    }
    *out = nullptr;
    if (n_obs < 0 || n_src < 0 || !(threshold >= 0)) {
        set_error("tct_near_plan_build_device: bad size or threshold");
        return TCT_ERR_ARG;
    }
    if (n_obs >= 0x7fffffff || n_src >= 0x7fffffff) {
        set_error("tct_near_plan_build_device: more than 2^31 - 2 balls on a side");
        return TCT_ERR_ARG;
    }
    auto* plan = new tct_near_plan();
    plan->n_obs = n_obs;
    plan->n_src = n_src;
    plan->threshold = threshold;
    plan->lp_start.push_back(0);
    if (n_obs == 0 || n_src == 0) {
        *out = plan;
        return TCT_OK;
    }
    if (!obs_c || !obs_r || !src_c || !src_r) {
        delete plan;
        set_error("tct_near_plan_build_device: null pointer");
        return TCT_ERR_ARG;
    }
    cudaStream_t st = as_stream(stream);
    const bool same = obs_c == src_c && obs_r == src_r && n_obs == n_src;
    DTree ot, stt;
    int rc = build_dtree(obs_c, obs_r, n_obs, 50, st, ot);
    if (rc == TCT_OK && !same) rc = build_dtree(src_c, src_r, n_src, 50, st, stt);
    if (rc == TCT_OK) rc = near_plan_fill_device(plan, ot, same ? ot : stt, obs_r, src_r, st);
    free_tree(ot, st);
    if (!same) free_tree(stt, st);
    cudaStreamSynchronize(st);
    if (rc != TCT_OK) {
        tct_near_plan_free(plan);
        return rc;
    }
    *out = plan;
    return TCT_OK;
}

namespace tct {

int near_plan_fill_device(tct_near_plan* plan, const DTree& ot, const DTree& stt,
                          const double* obs_r, const double* src_r, cudaStream_t st) {
    int32_t* lp = nullptr;
    int64_t nlp = 0;
    int rc = traverse_leaf_pairs(ot, stt, plan->threshold, st, &lp, &nlp);
    if (rc) return rc;
    // sort the leaf pairs by obs node (radix sort, stable) and find segments
    int32_t *ok = nullptr, *sv = nullptr, *ok2 = nullptr, *sv2 = nullptr, *flag = nullptr,
            *seg = nullptr;
    void* tmp = nullptr;
    auto cleanup = [&]() {
        dfree(lp, st); dfree(ok, st); dfree(sv, st); dfree(ok2, st); dfree(sv2, st);
        dfree(flag, st); dfree(seg, st);
        if (tmp) cudaFreeAsync(tmp, st);
    };
    const int64_t m = std::max<int64_t>(nlp, 1);
    if ((rc = dalloc(&ok, m, st)) || (rc = dalloc(&sv, m, st)) || (rc = dalloc(&ok2, m, st)) ||
        (rc = dalloc(&sv2, m, st)) || (rc = dalloc(&flag, m, st)) || (rc = dalloc(&seg, m, st))) {
        cleanup();
        return rc;
    }
    int64_t nl = 0;
    if (nlp > 0) {
        const unsigned nb = (unsigned)((nlp + 255) / 256);
        split_pairs<<<nb, 256, 0, st>>>(nlp, lp, ok, sv);
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, ok, ok2, sv, sv2, (int)nlp, 0, 32, st);
        if (cudaMallocAsync(&tmp, std::max<size_t>(tb, 1), st) != cudaSuccess) {
            tmp = nullptr;
            cudaGetLastError();
            cleanup();
            set_error("near plan: out of device memory (sort)");
            return TCT_ERR_OOM;
        }
        cub::DeviceRadixSort::SortPairs(tmp, tb, ok, ok2, sv, sv2, (int)nlp, 0, 32, st);
        if ((rc = launch_status("near plan sort"))) {
            cleanup();
            return rc;
        }
        new_segment_flags<<<nb, 256, 0, st>>>(nlp, ok2, flag);
        if ((rc = scan_exclusive(flag, seg, nlp, st))) {
            cleanup();
            return rc;
        }
        int32_t a = 0, b = 0;
        if ((rc = read_back(seg + nlp - 1, &a, st)) || (rc = read_back(flag + nlp - 1, &b, st))) {
            cleanup();
            return rc;
        }
        nl = (int64_t)a + b;
    }
    plan->nl_dev = nl;
    plan->nlp_dev = nlp;
    plan->dev_built = true;
    rc = near_plan_alloc_device(plan);
    if (rc) {
        cleanup();
        return rc;
    }
    NearDevPtrs d = near_plan_device_ptrs(plan);
    cudaMemcpyAsync(d.oc, ot.c, 24 * (size_t)plan->n_obs, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d.orq, obs_r, 8 * (size_t)plan->n_obs, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d.sc, stt.c, 24 * (size_t)plan->n_src, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d.srq, src_r, 8 * (size_t)plan->n_src, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d.oorig, ot.orig, 8 * (size_t)plan->n_obs, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d.sorig, stt.orig, 8 * (size_t)plan->n_src, cudaMemcpyDeviceToDevice, st);
    if (nlp > 0) {
        group_leaf_pairs<<<(unsigned)((nlp + 255) / 256), 256, 0, st>>>(
            nlp, ok2, sv2, seg, ot.ns, ot.ne, stt.ns, stt.ne, d.leaf_start, d.leaf_end,
            d.lp_start, d.lp_s, d.lp_e);
        rc = launch_status("near plan group");
    }
    const int64_t tail = nlp;
    cudaMemcpyAsync(d.lp_start + nl, &tail, 8, cudaMemcpyHostToDevice, st);
    if (rc == TCT_OK && cudaStreamSynchronize(st) != cudaSuccess)
        rc = launch_status("near plan fill");
    cleanup();
    return rc;
}

}  // namespace tct
