// Host-side structure builders of the nearfield: near-pair search, adjacency
// split, edge-adjacent orientation and the BSR index; plus the library's
// error/version plumbing.  Compiled with -ffp-contract=off so the distance
// tests round exactly like the reference's C++ (no fused multiply-add).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "tct_b200.h"
#include "near_plan.h"
#include "octree.h"

namespace tct {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

}  // namespace tct

struct tct_pair_list {
    std::vector<int64_t> pairs;  // flattened (obs, src)
};

namespace {

// |a - b|^2 accumulated as ((0 + d0^2) + d1^2) + d2^2, the order of
// fmm/geometry.hpp dist2 (dot of sub(a, b) with itself).
inline double dist2(const double* a, const double* b) {
    double out = 0;
    for (int d = 0; d < 3; d++) {
        double v = a[d] - b[d];
        out += v * v;
    }
    return out;
}

// ---- ball octree (the reference's fmm/octree.cpp + fmm/tree_helpers.hpp) ----
// Balls = triangle bounding spheres.  A node's bounds are the centre of mass
// of its ball centres and the radius max(|c - com| + R); a node with more
// than `leaf` balls splits into 8 octants by comparing each centre with the
// node centre (x bit 2, y bit 1, z bit 0, "greater than" = 1), stably; an
// empty child gets (parent centre, parent R / 50), a single-ball child the
// ball itself.  Nodes are stored in depth-first preorder.
using Node = tct::OctNode;
using tct::Octree;

inline double dist(const double* a, const double* b) { return std::sqrt(dist2(a, b)); }

void com_bounds(const Octree& t, int64_t s, int64_t e, double* c, double* R) {
    double com[3] = {0, 0, 0};
    for (int64_t i = s; i < e; i++)
        for (int d = 0; d < 3; d++) com[d] += t.centers[3 * i + d];
    for (int d = 0; d < 3; d++) com[d] /= (double)(e - s);
    double max_r = 0.0;
    for (int64_t i = s; i < e; i++) max_r = std::max(max_r, dist(&t.centers[3 * i], com) + t.radii[i]);
    for (int d = 0; d < 3; d++) c[d] = com[d];
    *R = max_r;
}

int64_t add_node(Octree& t, int64_t s, int64_t e, int64_t leaf, int depth, const double* c,
                 double R, std::vector<int64_t>& scratch) {
    const int64_t idx = (int64_t)t.nodes.size();
    Node n;
    n.start = s;
    n.end = e;
    for (int d = 0; d < 3; d++) n.c[d] = c[d];
    n.R = R;
    // depth cap: more than `leaf` balls at one identical centre would never split
    n.leaf = (e - s <= leaf) || depth >= 60;
    n.depth = depth;
    for (int k = 0; k < 8; k++) n.child[k] = -1;
    t.nodes.push_back(n);
    if (n.leaf) return idx;
    // stable partition into octants
    int64_t counts[9] = {0};
    std::vector<int> oct(e - s);
    for (int64_t i = s; i < e; i++) {
        int o = 0;
        for (int d = 0; d < 3; d++) {
            if (t.centers[3 * i + d] > c[d]) o++;
            if (d < 2) o <<= 1;
        }
        oct[i - s] = o;
        counts[o + 1]++;
    }
    for (int k = 0; k < 8; k++) counts[k + 1] += counts[k];
    {
        std::vector<int64_t> fill(counts, counts + 8);
        scratch.resize(e - s);
        for (int64_t i = s; i < e; i++) scratch[fill[oct[i - s]]++] = i;
        std::vector<double> cc(3 * (e - s)), rr(e - s);
        std::vector<int64_t> oo(e - s);
        for (int64_t k = 0; k < e - s; k++) {
            const int64_t i = scratch[k];
            for (int d = 0; d < 3; d++) cc[3 * k + d] = t.centers[3 * i + d];
            rr[k] = t.radii[i];
            oo[k] = t.orig[i];
        }
        std::copy(cc.begin(), cc.end(), t.centers.begin() + 3 * s);
        std::copy(rr.begin(), rr.end(), t.radii.begin() + s);
        std::copy(oo.begin(), oo.end(), t.orig.begin() + s);
    }
    for (int k = 0; k < 8; k++) {
        const int64_t cs = s + counts[k], ce = s + counts[k + 1];
        double cc[3], cr;
        if (ce - cs == 0) {
            for (int d = 0; d < 3; d++) cc[d] = c[d];
            cr = R / 50.0;
        } else if (ce - cs == 1) {
            for (int d = 0; d < 3; d++) cc[d] = t.centers[3 * cs + d];
            cr = t.radii[cs];
        } else {
            com_bounds(t, cs, ce, cc, &cr);
        }
        const int64_t ch = add_node(t, cs, ce, leaf, depth + 1, cc, cr, scratch);
        t.nodes[idx].child[k] = ch;
    }
    return idx;
}

Octree build_octree(const double* centers, const double* radii, int64_t n, int64_t leaf) {
    Octree t;
    t.centers.assign(centers, centers + 3 * n);
    t.radii.assign(radii, radii + n);
    t.orig.resize(n);
    for (int64_t i = 0; i < n; i++) t.orig[i] = i;
    double c[3] = {0, 0, 0}, R = 1.0;
    if (n == 1) {
        for (int d = 0; d < 3; d++) c[d] = centers[d];
        R = radii[0];
    } else if (n > 1) {
        com_bounds(t, 0, n, c, &R);
    }
    std::vector<int64_t> scratch;
    add_node(t, 0, n, leaf, 0, c, R, scratch);
    return t;
}

// Node radius enlarged to cover every member ball (fast_find_nearfield.cpp:77-94).
std::vector<double> expanded_r(const Octree& t, const double* orig_radii) {
    std::vector<double> out(t.nodes.size());
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t k = 0; k < (int64_t)t.nodes.size(); k++) {
        const Node& n = t.nodes[k];
        double m = n.R;
        for (int64_t j = n.start; j < n.end; j++) {
            double md = dist(&t.centers[3 * j], n.c) + orig_radii[t.orig[j]];
            if (md > m) m = md;
        }
        out[k] = m;
    }
    return out;
}

// The two trees and expanded radii of a search.  A self search (the same
// arrays on both sides) builds one tree; otherwise the two build side by side.
struct TreePair {
    Octree ot, st_own;
    std::vector<double> oer, ser_own;
    bool same = false;
    const Octree& st() const { return same ? ot : st_own; }
    const std::vector<double>& ser() const { return same ? oer : ser_own; }
};

void build_tree_pair(const double* obs_c, const double* obs_r, int64_t n_obs, const double* src_c,
                     const double* src_r, int64_t n_src, int64_t leaf, TreePair& tp) {
    tp.same = obs_c == src_c && obs_r == src_r && n_obs == n_src;
    if (tp.same) {
        tp.ot = build_octree(obs_c, obs_r, n_obs, leaf);
    } else {
#pragma omp parallel sections num_threads(2)
        {
#pragma omp section
            tp.ot = build_octree(obs_c, obs_r, n_obs, leaf);
#pragma omp section
            tp.st_own = build_octree(src_c, src_r, n_src, leaf);
        }
    }
    tp.oer = expanded_r(tp.ot, obs_r);
    if (!tp.same) tp.ser_own = expanded_r(tp.st_own, src_r);
}

struct Query {
    const Octree& ot;
    const Octree& st;
    const std::vector<double>& oer;
    const std::vector<double>& ser;
    const double* orad;  // original-order radii, indexed by TREE position (see below)
    const double* srad;
    double thr;
};

// Dual-tree ball query (fast_find_nearfield.cpp:22-74).  The leaf test reads
// the radius arrays at the balls' tree positions i, j -- not at their
// original indices -- exactly as the reference does; with near-uniform
// triangle sizes this only moves pairs within rounding of the threshold, but
// it is the reference's pair set, so it is kept.
void query(const Query& q, int64_t on, int64_t sn, std::vector<int64_t>& out) {
    const Node& o = q.ot.nodes[on];
    const Node& s = q.st.nodes[sn];
    const double r1 = q.oer[on], r2 = q.ser[sn];
    const double limit = std::pow((r1 + r2) * q.thr, 2);
    if (dist2(o.c, s.c) > limit) return;
    if (o.leaf && s.leaf) {
        for (int64_t i = o.start; i < o.end; i++) {
            const int64_t oi = q.ot.orig[i];
            for (int64_t j = s.start; j < s.end; j++) {
                const double sep = q.orad[i] + q.srad[j];
                const double pt_limit = std::pow(sep * q.thr, 2);
                if (dist2(&q.ot.centers[3 * i], &q.st.centers[3 * j]) > pt_limit) continue;
                out.push_back(oi);
                out.push_back(q.st.orig[j]);
            }
        }
        return;
    }
    const bool split_src = ((r1 < r2) && !s.leaf) || o.leaf;
    if (split_src) {
        for (int k = 0; k < 8; k++) query(q, on, s.child[k], out);
    } else {
        for (int k = 0; k < 8; k++) query(q, o.child[k], sn, out);
    }
}

// The same traversal, stopping at leaf pairs: (obs node, src node) pairs
// whose balls the leaf test above would examine.
void query_leaves(const Query& q, int64_t on, int64_t sn, std::vector<int64_t>& out) {
    const Node& o = q.ot.nodes[on];
    const Node& s = q.st.nodes[sn];
    const double r1 = q.oer[on], r2 = q.ser[sn];
    const double limit = std::pow((r1 + r2) * q.thr, 2);
    if (dist2(o.c, s.c) > limit) return;
    if (o.leaf && s.leaf) {
        out.push_back(on);
        out.push_back(sn);
        return;
    }
    const bool split_src = ((r1 < r2) && !s.leaf) || o.leaf;
    if (split_src) {
        for (int k = 0; k < 8; k++) query_leaves(q, on, s.child[k], out);
    } else {
        for (int k = 0; k < 8; k++) query_leaves(q, o.child[k], sn, out);
    }
}

}  // namespace

extern "C" {

const char* tct_version(void) { return "tct_b200 0.1 (sm_100a)"; }

const char* tct_last_error(void) { return tct::g_err; }

int tct_kernel_id(const char* name) {
    static const char* names[] = {"elasticU3",  "elasticT3",  "elasticA3", "elasticH3",
                                  "elasticRT3", "elasticRA3", "elasticRH3"};
    if (!name) return -1;
    for (int i = 0; i < 7; i++)
        if (std::strcmp(name, names[i]) == 0) return i;
    return -1;
}

// Near pairs (fast_find_nearfield.cpp:96-141, get_nearfield :255-285): octrees
// with 50 balls per leaf on both sides, then one dual-tree query per obs node
// at depth 2 (or shallower leaf), run in parallel.  The pair set is the
// reference's; the output is ordered by (obs, src) with a counting sort.
int tct_find_near_pairs(const double* obs_c, const double* obs_r, int64_t n_obs,
                        const double* src_c, const double* src_r, int64_t n_src,
                        double threshold, int n_threads, tct_pair_list** out) {
    using namespace tct;
    if (!out) {
        set_error("tct_find_near_pairs: null output handle");
        return TCT_ERR_ARG;
    }
    *out = nullptr;
    if (n_obs < 0 || n_src < 0 || !(threshold >= 0)) {
        set_error("tct_find_near_pairs: bad size or threshold");
        return TCT_ERR_ARG;
    }
    auto* list = new tct_pair_list();
    if (n_obs == 0 || n_src == 0) {
        *out = list;
        return TCT_OK;
    }
    if (!obs_c || !obs_r || !src_c || !src_r) {
        delete list;
        set_error("tct_find_near_pairs: null pointer");
        return TCT_ERR_ARG;
    }
    if (n_threads <= 0) n_threads = omp_get_max_threads();
    const int64_t leaf = 50;
    TreePair tp;
    build_tree_pair(obs_c, obs_r, n_obs, src_c, src_r, n_src, leaf, tp);
    const Octree& ot = tp.ot;
    const Octree& st = tp.st();
    Query q{ot, st, tp.oer, tp.ser(), obs_r, src_r, threshold};
    std::vector<int64_t> starts;
    for (size_t k = 0; k < ot.nodes.size(); k++) {
        const Node& n = ot.nodes[k];
        if (n.depth > 2) continue;
        if (n.depth != 2 && !n.leaf) continue;
        starts.push_back((int64_t)k);
    }
    std::vector<std::vector<int64_t>> parts(starts.size());
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 1)
    for (int64_t k = 0; k < (int64_t)starts.size(); k++) query(q, starts[k], 0, parts[k]);
    // counting sort by obs index, then sort each obs's sources
    std::vector<int64_t> offs(n_obs + 1, 0);
    int64_t total = 0;
    for (auto& p : parts) {
        for (size_t m = 0; m < p.size(); m += 2) offs[p[m] + 1]++;
        total += (int64_t)p.size() / 2;
    }
    for (int64_t i = 0; i < n_obs; i++) offs[i + 1] += offs[i];
    std::vector<int64_t> src_sorted(total);
    {
        std::vector<int64_t> fill(offs.begin(), offs.end() - 1);
        for (auto& p : parts)
            for (size_t m = 0; m < p.size(); m += 2) src_sorted[fill[p[m]]++] = p[m + 1];
    }
    list->pairs.resize(2 * total);
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 256)
    for (int64_t i = 0; i < n_obs; i++) {
        std::sort(src_sorted.begin() + offs[i], src_sorted.begin() + offs[i + 1]);
        for (int64_t k = offs[i]; k < offs[i + 1]; k++) {
            list->pairs[2 * k] = i;
            list->pairs[2 * k + 1] = src_sorted[k];
        }
    }
    *out = list;
    return TCT_OK;
}

// Host half of the device near-pair search (tct_near_device_count/_fill,
// csrc/near.cu): the same octrees and traversal as tct_find_near_pairs, down
// to leaf pairs, grouped by obs leaf.
int tct_near_plan_build(const double* obs_c, const double* obs_r, int64_t n_obs,
                        const double* src_c, const double* src_r, int64_t n_src,
                        double threshold, int n_threads, tct_near_plan** out) {
    using namespace tct;
    if (!out) {
        set_error("tct_near_plan_build: null output handle");
        return TCT_ERR_ARG;
    }
    *out = nullptr;
    if (n_obs < 0 || n_src < 0 || !(threshold >= 0)) {
        set_error("tct_near_plan_build: bad size or threshold");
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
        set_error("tct_near_plan_build: null pointer");
        return TCT_ERR_ARG;
    }
    if (n_threads <= 0) n_threads = omp_get_max_threads();
    const int64_t leaf = 50;
    TreePair tp;
    build_tree_pair(obs_c, obs_r, n_obs, src_c, src_r, n_src, leaf, tp);
    const Octree& ot = tp.ot;
    const Octree& st = tp.st();
    Query q{ot, st, tp.oer, tp.ser(), obs_r, src_r, threshold};
    std::vector<int64_t> starts;
    for (size_t k = 0; k < ot.nodes.size(); k++) {
        const Node& n = ot.nodes[k];
        if (n.depth > 2) continue;
        if (n.depth != 2 && !n.leaf) continue;
        starts.push_back((int64_t)k);
    }
    std::vector<std::vector<int64_t>> parts(starts.size());
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 1)
    for (int64_t k = 0; k < (int64_t)starts.size(); k++) query_leaves(q, starts[k], 0, parts[k]);
    // group the leaf pairs by obs leaf (counting sort on the node id, stable)
    std::vector<int64_t> cnt(ot.nodes.size() + 1, 0);
    for (auto& p : parts)
        for (size_t m = 0; m < p.size(); m += 2) cnt[p[m] + 1]++;
    for (size_t k = 0; k < ot.nodes.size(); k++) cnt[k + 1] += cnt[k];
    const int64_t n_lp = cnt[ot.nodes.size()];
    std::vector<int64_t> srcn(n_lp);
    {
        std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
        for (auto& p : parts)
            for (size_t m = 0; m < p.size(); m += 2) srcn[fill[p[m]]++] = p[m + 1];
    }
    for (size_t k = 0; k < ot.nodes.size(); k++) {
        if (cnt[k + 1] == cnt[k]) continue;
        plan->leaf_start.push_back(ot.nodes[k].start);
        plan->leaf_end.push_back(ot.nodes[k].end);
        for (int64_t m = cnt[k]; m < cnt[k + 1]; m++) {
            plan->lp_s.push_back(st.nodes[srcn[m]].start);
            plan->lp_e.push_back(st.nodes[srcn[m]].end);
        }
        plan->lp_start.push_back((int64_t)plan->lp_s.size());
    }
    plan->oc = ot.centers;
    plan->sc = st.centers;
    plan->orq.assign(obs_r, obs_r + n_obs);
    plan->srq.assign(src_r, src_r + n_src);
    plan->oorig = ot.orig;
    plan->sorig = st.orig;
    *out = plan;
    return TCT_OK;
}

int64_t tct_near_plan_leaf_pairs(const tct_near_plan* plan) {
    return plan ? (int64_t)plan->lp_s.size() : -1;
}

// ---- treecode trees and interaction lists (fmm/tsfmm.py:22-28, 66-70) --------
}  // extern "C"


struct tct_lists {
    // compressed lists (fmm/traversal.cpp:20-53): obs nodes with a non-empty
    // list, CSR starts, source node indices; 0 p2p, 1 m2p, 2 p2l, 3 m2l
    std::vector<int64_t> obs[4], start[4], src[4];
};

namespace {

int node_height(tct_tree& tr, int64_t k) {
    const Node& n = tr.t.nodes[k];
    if (n.leaf) return tr.height[k] = 0;
    int h = 0;
    for (int c = 0; c < 8; c++) h = std::max(h, node_height(tr, n.child[c]));
    return tr.height[k] = h + 1;
}

template <typename F>
void for_all_leaves(const Octree& t, int64_t k, const F& f) {
    const Node& n = t.nodes[k];
    if (n.leaf) {
        f(k);
        return;
    }
    for (int c = 0; c < 8; c++) for_all_leaves(t, n.child[c], f);
}

// Dual-tree traversal with the multipole acceptance criterion
// outer_r * R_src + inner_r * R_obs < 0.98 * |c_obs - c_src| (fmm/traversal.cpp:119-192).
typedef std::vector<std::vector<int64_t>> NodeLists;

void traverse(const Octree& ot, const Octree& st, int64_t on, int64_t sn, double inner_r,
              double outer_r, int64_t order, bool treecode, NodeLists& p2p, NodeLists& m2p,
              NodeLists& p2l, NodeLists& m2l) {
    const Node& o = ot.nodes[on];
    const Node& s = st.nodes[sn];
    const double r_src = s.R, r_obs = o.R;
    double d0 = o.c[0] - s.c[0], d1 = o.c[1] - s.c[1], d2 = o.c[2] - s.c[2];
    const double sep = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    if (outer_r * r_src + inner_r * r_obs < 0.98 * sep) {
        const int64_t n_src = s.end - s.start, n_obs = o.end - o.start;
        if (n_src == 0 || n_obs == 0) return;
        const bool small_src = n_src < order, small_obs = n_obs < order;
        if (small_src && small_obs) {
            for_all_leaves(ot, on, [&](int64_t leaf) { p2p[leaf].push_back(sn); });
        } else if (small_obs || treecode) {
            for_all_leaves(ot, on, [&](int64_t leaf) { m2p[leaf].push_back(sn); });
        } else if (small_src) {
            p2l[on].push_back(sn);
        } else {
            m2l[on].push_back(sn);
        }
        return;
    }
    if (s.leaf && o.leaf) {
        p2p[on].push_back(sn);
        return;
    }
    const bool split_src = ((r_obs < r_src) && !s.leaf) || o.leaf;
    if (split_src) {
        for (int c = 0; c < 8; c++)
            traverse(ot, st, on, s.child[c], inner_r, outer_r, order, treecode, p2p, m2p, p2l,
                     m2l);
    } else {
        for (int c = 0; c < 8; c++)
            traverse(ot, st, o.child[c], sn, inner_r, outer_r, order, treecode, p2p, m2p, p2l,
                     m2l);
    }
}

void compress(const std::vector<std::vector<int64_t>>& list, std::vector<int64_t>& obs,
              std::vector<int64_t>& start, std::vector<int64_t>& src) {
    obs.clear();
    start.assign(1, 0);
    src.clear();
    for (size_t i = 0; i < list.size(); i++) {
        if (list[i].empty()) continue;
        obs.push_back((int64_t)i);
        src.insert(src.end(), list[i].begin(), list[i].end());
        start.push_back((int64_t)src.size());
    }
}

}  // namespace

extern "C" {

// Ball octree on triangle centres and radii (fmm/octree.cpp via the treecode's
// make_tree, fmm/tsfmm.py:22-28): the same tree as the near-pair search.
int tct_tree_build(const double* centers, const double* radii, int64_t n, int64_t leaf_size,
                   tct_tree** out) {
    if (!out || n < 0 || leaf_size < 1 || (n > 0 && (!centers || !radii))) {
        tct::set_error("tct_tree_build: bad arguments");
        return TCT_ERR_ARG;
    }
    auto* tr = new tct_tree();
    tr->t = build_octree(centers, radii, n, leaf_size);
    tr->height.assign(tr->t.nodes.size(), 0);
    tr->max_height = node_height(*tr, 0);
    *out = tr;
    return TCT_OK;
}

int64_t tct_tree_n_nodes(const tct_tree* tr) { return tr ? (int64_t)tr->t.nodes.size() : 0; }

int tct_tree_max_height(const tct_tree* tr) { return tr ? tr->max_height : -1; }

// Node arrays: start, end (int64), centre (3 doubles), R, leaf flag, depth,
// height (int32) and the 8 children (int64, -1 for leaves); orig_idx[i] is the
// original index of the ball at tree position i.  Any pointer may be NULL.
int tct_tree_export(const tct_tree* tr, int64_t* orig_idx, int64_t* start, int64_t* end,
                    double* center, double* R, int32_t* leaf, int32_t* depth, int32_t* height,
                    int64_t* children) {
    if (!tr) {
        tct::set_error("tct_tree_export: null tree");
        return TCT_ERR_ARG;
    }
    const Octree& t = tr->t;
    if (orig_idx) std::copy(t.orig.begin(), t.orig.end(), orig_idx);
    for (size_t k = 0; k < t.nodes.size(); k++) {
        const Node& n = t.nodes[k];
        if (start) start[k] = n.start;
        if (end) end[k] = n.end;
        if (center)
            for (int d = 0; d < 3; d++) center[3 * k + d] = n.c[d];
        if (R) R[k] = n.R;
        if (leaf) leaf[k] = n.leaf ? 1 : 0;
        if (depth) depth[k] = n.depth;
        if (height) height[k] = tr->height[k];
        if (children)
            for (int c = 0; c < 8; c++) children[8 * k + c] = n.leaf ? -1 : n.child[c];
    }
    return TCT_OK;
}

void tct_tree_free(tct_tree* tr) { delete tr; }

// P2P and M2P lists of the dual traversal (fmm/traversal.cpp:227-242 with
// order and treecode as the reference's treecode passes them: 0 and true).
int tct_treecode_lists(const tct_tree* obs, const tct_tree* src, double inner_r, double outer_r,
                       int64_t order, int treecode, tct_lists** out) {
    if (!obs || !src || !out) {
        tct::set_error("tct_treecode_lists: null argument");
        return TCT_ERR_ARG;
    }
    const size_t nn = obs->t.nodes.size();
    NodeLists lists[4] = {NodeLists(nn), NodeLists(nn), NodeLists(nn), NodeLists(nn)};
    traverse(obs->t, src->t, 0, 0, inner_r, outer_r, order, treecode != 0, lists[0], lists[1],
             lists[2], lists[3]);
    auto* l = new tct_lists();
    for (int k = 0; k < 4; k++) compress(lists[k], l->obs[k], l->start[k], l->src[k]);
    *out = l;
    return TCT_OK;
}

int tct_lists_sizes(const tct_lists* l, int64_t* sizes) {
    if (!l || !sizes) return TCT_ERR_ARG;
    for (int k = 0; k < 4; k++) {
        sizes[2 * k] = (int64_t)l->obs[k].size();
        sizes[2 * k + 1] = (int64_t)l->src[k].size();
    }
    return TCT_OK;
}

int tct_lists_export(const tct_lists* l, int which, int64_t* obs, int64_t* start, int64_t* src) {
    if (!l || which < 0 || which > 3) {
        tct::set_error("tct_lists_export: bad list handle or index %d", which);
        return TCT_ERR_ARG;
    }
    auto cp = [](const std::vector<int64_t>& v, int64_t* d) {
        if (d && !v.empty()) std::memcpy(d, v.data(), v.size() * sizeof(int64_t));
    };
    cp(l->obs[which], obs);
    cp(l->start[which], start);
    cp(l->src[which], src);
    return TCT_OK;
}

void tct_lists_free(tct_lists* l) { delete l; }

int64_t tct_pairs_count(const tct_pair_list* list) {
    return list ? (int64_t)(list->pairs.size() / 2) : 0;
}

int tct_pairs_copy(const tct_pair_list* list, int64_t* dst) {
    if (!list || (!dst && !list->pairs.empty())) {
        tct::set_error("tct_pairs_copy: null pointer");
        return TCT_ERR_ARG;
    }
    if (!list->pairs.empty()) std::memcpy(dst, list->pairs.data(), list->pairs.size() * sizeof(int64_t));
    return TCT_OK;
}

void tct_pairs_free(tct_pair_list* list) { delete list; }

// Classify each close pair by shared vertex count (fast_find_nearfield.cpp:143-182).
int tct_split_adjacent_close(const int64_t* pairs, int64_t n_pairs, const int64_t* tris_a,
                             const int64_t* tris_b, int64_t* near_out, int64_t* n_near,
                             int64_t* va_out, int64_t* n_va, int64_t* ea_out, int64_t* n_ea) {
    using namespace tct;
    if (n_pairs < 0 || !n_near || !n_va || !n_ea) {
        set_error("tct_split_adjacent_close: bad arguments");
        return TCT_ERR_ARG;
    }
    int64_t nn = 0, nv = 0, ne = 0;
    for (int64_t p = 0; p < n_pairs; p++) {
        const int64_t a = pairs[2 * p], b = pairs[2 * p + 1];
        int first[2] = {-1, -1}, second[2] = {-1, -1};
        bool coincident = false;
        for (int d1 = 0; d1 < 3; d1++)
            for (int d2 = 0; d2 < 3; d2++) {
                if (tris_a[3 * a + d1] != tris_b[3 * b + d2]) continue;
                if (first[0] == -1) {
                    first[0] = d1;
                    first[1] = d2;
                } else if (second[0] == -1) {
                    second[0] = d1;
                    second[1] = d2;
                } else {
                    coincident = true;
                }
            }
        if (coincident) continue;
        if (first[0] == -1) {
            near_out[2 * nn] = a;
            near_out[2 * nn + 1] = b;
            nn++;
        } else if (second[0] == -1) {
            int64_t* r = va_out + 4 * nv;
            r[0] = a;
            r[1] = b;
            r[2] = first[0];
            r[3] = first[1];
            nv++;
        } else {
            int64_t* r = ea_out + 6 * ne;
            r[0] = a;
            r[1] = b;
            r[2] = first[0];
            r[3] = first[1];
            r[4] = second[0];
            r[5] = second[1];
            ne++;
        }
    }
    *n_near = nn;
    *n_va = nv;
    *n_ea = ne;
    return TCT_OK;
}

// Rotation that brings the shared edge to corners (0, 1): sorted corner
// pair (0,1) -> 0 clicks, (1,2) -> 1, (0,2) -> 2 (nearfield_op.py:44-50);
// the source is flipped when its rotated corners 1, 0 do not match the
// observer's 0, 1 (nearfield_op.py:52-62).
static int edge_clicks(int64_t u, int64_t v) {
    int64_t a = std::min(u, v), b = std::max(u, v);
    if (a == 0) return b == 2 ? 2 : 0;
    return 1;
}

int tct_resolve_ea_rotation(const int64_t* tris, const int64_t* ea, int64_t n, int64_t* out) {
    if (n < 0 || (n > 0 && (!tris || !ea || !out))) {
        tct::set_error("tct_resolve_ea_rotation: bad arguments");
        return TCT_ERR_ARG;
    }
    for (int64_t i = 0; i < n; i++) {
        const int64_t* r = ea + 6 * i;
        const int oc = edge_clicks(r[2], r[4]);
        const int sc = edge_clicks(r[3], r[5]);
        const int64_t o = r[0], s = r[1];
        const bool flip = tris[3 * o + (0 + oc) % 3] != tris[3 * s + (1 + sc) % 3] ||
                          tris[3 * o + (1 + oc) % 3] != tris[3 * s + (0 + sc) % 3];
        int64_t* w = out + 5 * i;
        w[0] = o;
        w[1] = s;
        w[2] = oc;
        w[3] = sc;
        w[4] = flip ? 1 : 0;
    }
    return TCT_OK;
}

// Stable counting sort by block row (fast_sparse.cpp:14-68).
int tct_make_bsr_index(int64_t n_row_blocks, int64_t n_blocks, const int64_t* rows,
                       const int64_t* cols, int64_t* indptr, int64_t* indices, int64_t* slot) {
    if (n_row_blocks < 0 || n_blocks < 0 || !indptr ||
        (n_blocks > 0 && (!rows || !cols || !indices || !slot))) {
        tct::set_error("tct_make_bsr_index: bad arguments");
        return TCT_ERR_ARG;
    }
    std::fill(indptr, indptr + n_row_blocks + 1, 0);
    for (int64_t i = 0; i < n_blocks; i++) {
        if (rows[i] < 0 || rows[i] >= n_row_blocks) {
            tct::set_error("tct_make_bsr_index: row %lld out of range", (long long)rows[i]);
            return TCT_ERR_ARG;
        }
        indptr[rows[i] + 1]++;
    }
    for (int64_t r = 0; r < n_row_blocks; r++) indptr[r + 1] += indptr[r];
    std::vector<int64_t> fill(indptr, indptr + n_row_blocks);
    for (int64_t i = 0; i < n_blocks; i++) {
        const int64_t dest = fill[rows[i]]++;
        indices[dest] = cols[i];
        slot[i] = dest;
    }
    return TCT_OK;
}


// One Arnoldi step's host update for a set of GMRES systems (the Givens
// QR of the Hessenberg matrix, as in the reference's solver, scipy's gmres
// driven by examples/solve.py:25-61).  System s = sys[i] takes its new
// column cols[i * col_stride + 0 .. j[s] + 1] (h_0..h_j, ||w||) into column
// j[s] of H_s ((m + 1) x m, column-major per system), applies its previous
// rotations, forms rotation j[s], updates g_s and writes |g_s[j + 1]| to
// res[i].
int tct_gmres_givens(int64_t n_active, const int64_t* sys, const int64_t* j, int64_t m,
                     const double* cols, int64_t col_stride, double* H, double* cs, double* sn,
                     double* g, double* res) {
    if (n_active < 0 || m < 1 || (n_active > 0 && (!sys || !j || !cols || !H || !cs || !sn ||
                                                   !g || !res))) {
        tct::set_error("tct_gmres_givens: bad arguments");
        return TCT_ERR_ARG;
    }
    for (int64_t i = 0; i < n_active; i++) {
        const int64_t s = sys[i], js = j[s];
        if (s < 0 || js < 0 || js >= m || js + 2 > col_stride) {
            tct::set_error("tct_gmres_givens: step %lld of system %lld out of range",
                           (long long)js, (long long)s);
            return TCT_ERR_ARG;
        }
        double* h = H + s * (m + 1) * m + js * (m + 1);
        double* c = cs + s * m;
        double* sv = sn + s * m;
        double* gs = g + s * (m + 1);
        const double* col = cols + i * col_stride;
        for (int64_t k = 0; k < js + 2; k++) h[k] = col[k];
        for (int64_t k = js + 2; k < m + 1; k++) h[k] = 0.0;
        for (int64_t k = 0; k < js; k++) {
            const double a = h[k], b = h[k + 1];
            h[k] = c[k] * a + sv[k] * b;
            h[k + 1] = -sv[k] * a + c[k] * b;
        }
        const double den = std::hypot(h[js], h[js + 1]);
        c[js] = den > 0 ? h[js] / den : 1.0;
        sv[js] = den > 0 ? h[js + 1] / den : 0.0;
        h[js] = den;
        h[js + 1] = 0.0;
        gs[js + 1] = -sv[js] * gs[js];
        gs[js] = c[js] * gs[js];
        res[i] = std::fabs(gs[js + 1]);
    }
    return TCT_OK;
}

}  // extern "C"
