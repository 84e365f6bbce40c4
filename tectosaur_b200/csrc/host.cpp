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

struct Grid {
    double origin[3];
    double h;
    int64_t n[3];
    std::vector<int64_t> cell_start;  // size n0*n1*n2 + 1
    std::vector<int64_t> order;       // src indices sorted by cell

    int64_t cell_coord(double v, int d) const {
        double t = std::floor((v - origin[d]) / h);
        if (t < 0) return 0;
        if (t > (double)(n[d] - 1)) return n[d] - 1;
        return (int64_t)t;
    }
};

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

// Ball query of every obs ball against every src ball:
// pair (i, j) iff |c_i - c_j|^2 <= ((r_i + r_j) * threshold)^2 (the leaf test
// of mesh/fast_find_nearfield.cpp:72-84).  A uniform grid of cell width
// >= 2 * threshold * max(r_src) (grown if the grid would be huge) bins the
// src centres; each obs ball visits the cells within (r_i + max r_src) *
// threshold of its centre, widened by a relative 1e-9, so every qualifying
// pair is tested with the exact double-precision predicate.  Output order:
// by obs index, then src index.
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

    double lo[3], hi[3], rmax = 0;
    for (int d = 0; d < 3; d++) {
        lo[d] = src_c[d];
        hi[d] = src_c[d];
    }
    for (int64_t j = 0; j < n_src; j++) {
        for (int d = 0; d < 3; d++) {
            lo[d] = std::min(lo[d], src_c[3 * j + d]);
            hi[d] = std::max(hi[d], src_c[3 * j + d]);
        }
        rmax = std::max(rmax, src_r[j]);
    }
    Grid g;
    double extent = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-300});
    g.h = std::max(2.0 * threshold * rmax, extent * 1e-6);
    if (!(g.h > 0)) g.h = 1.0;
    for (;;) {
        int64_t cells = 1;
        for (int d = 0; d < 3; d++) {
            g.n[d] = (int64_t)std::floor((hi[d] - lo[d]) / g.h) + 1;
            cells *= g.n[d];
        }
        if (cells <= 4 * n_src + 4096) break;
        g.h *= 1.5;
    }
    for (int d = 0; d < 3; d++) g.origin[d] = lo[d];
    const int64_t n_cells = g.n[0] * g.n[1] * g.n[2];
    std::vector<int64_t> cell_of(n_src);
    g.cell_start.assign(n_cells + 1, 0);
    for (int64_t j = 0; j < n_src; j++) {
        int64_t cx = g.cell_coord(src_c[3 * j], 0), cy = g.cell_coord(src_c[3 * j + 1], 1),
                cz = g.cell_coord(src_c[3 * j + 2], 2);
        cell_of[j] = (cz * g.n[1] + cy) * g.n[0] + cx;
        g.cell_start[cell_of[j] + 1]++;
    }
    for (int64_t c = 0; c < n_cells; c++) g.cell_start[c + 1] += g.cell_start[c];
    g.order.resize(n_src);
    {
        std::vector<int64_t> fill(g.cell_start.begin(), g.cell_start.end() - 1);
        for (int64_t j = 0; j < n_src; j++) g.order[fill[cell_of[j]]++] = j;
    }

    const int64_t chunk = 256;
    const int64_t n_chunks = (n_obs + chunk - 1) / chunk;
    std::vector<std::vector<int64_t>> parts(n_chunks);
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 1)
    for (int64_t ch = 0; ch < n_chunks; ch++) {
        std::vector<int64_t>& part = parts[ch];
        std::vector<int64_t> hits;
        const int64_t i_end = std::min(n_obs, (ch + 1) * chunk);
        for (int64_t i = ch * chunk; i < i_end; i++) {
            const double* ci = obs_c + 3 * i;
            const double reach = (obs_r[i] + rmax) * threshold * (1.0 + 1e-9) + 1e-300;
            int64_t c0[3], c1[3];
            for (int d = 0; d < 3; d++) {
                c0[d] = g.cell_coord(ci[d] - reach, d);
                c1[d] = g.cell_coord(ci[d] + reach, d);
            }
            hits.clear();
            for (int64_t cz = c0[2]; cz <= c1[2]; cz++)
                for (int64_t cy = c0[1]; cy <= c1[1]; cy++)
                    for (int64_t cx = c0[0]; cx <= c1[0]; cx++) {
                        const int64_t cell = (cz * g.n[1] + cy) * g.n[0] + cx;
                        for (int64_t k = g.cell_start[cell]; k < g.cell_start[cell + 1]; k++) {
                            const int64_t j = g.order[k];
                            const double sep = obs_r[i] + src_r[j];
                            const double lim = std::pow(sep * threshold, 2);
                            if (dist2(ci, src_c + 3 * j) > lim) continue;
                            hits.push_back(j);
                        }
                    }
            std::sort(hits.begin(), hits.end());
            for (int64_t j : hits) {
                part.push_back(i);
                part.push_back(j);
            }
        }
    }
    size_t total = 0;
    for (auto& p : parts) total += p.size();
    list->pairs.reserve(total);
    for (auto& p : parts) list->pairs.insert(list->pairs.end(), p.begin(), p.end());
    *out = list;
    return TCT_OK;
}

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

}  // extern "C"
