// Tuned launch shapes: the library's one piece of shared mutable state
// besides the per-thread error strings.
//
// The reference instantiates its kernels per template argument and caches
// the compiled modules (util/gpu.py:63-77); its launch shapes are fixed.
// Here the kernels are compiled once for sm_100a and the shape of a launch
// -- how the work is cut into CTAs -- is a run-time choice looked up in this
// cache, keyed by (operation, kernel, precision, rule points, right-hand
// sides, size buckets).  An entry is written by the autotune entry points
// (tct_farfield_autotune, tct_bsr9_autotune), which time the candidate shapes
// on the caller's own buffers with CUDA events, or restored from a saved
// cache (tct_tune_put_entry).  Launches whose key has no entry use the
// built-in heuristics, so an empty cache gives the library's default shapes.
//
// Sizes are bucketed by rounded log2 (bucket = round(log2 n) + 1, 0 for
// n <= 0: a factor of about 1.4 either way), so one tuned entry serves
// meshes of similar size.
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"

namespace tct {
namespace {

using Key = std::tuple<int, int, int, int, int, int, int>;

std::mutex g_tune_mutex;
std::map<Key, std::pair<int, int>> g_tune;

Key make_key(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1) {
    return Key(op, kernel, prec, nq, rhs, tune_bucket(n0), tune_bucket(n1));
}

}  // namespace

int tune_bucket(int64_t n) {
    if (n <= 0) return 0;
    // round(log2(n)) + 1: floor(log2(n)) + 1, plus one when n >= 2^k sqrt(2)
    int k = 63 - __builtin_clzll((unsigned long long)n);
    const double lo = (double)(1ull << k);
    return (double)n >= lo * 1.4142135623730951 ? k + 2 : k + 1;
}

bool tune_lookup(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1, int* v0,
                 int* v1) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    if (g_tune.empty()) return false;
    auto it = g_tune.find(make_key(op, kernel, prec, nq, rhs, n0, n1));
    if (it == g_tune.end()) return false;
    *v0 = it->second.first;
    *v1 = it->second.second;
    return true;
}

void tune_store(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1, int v0,
                int v1) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune[make_key(op, kernel, prec, nq, rhs, n0, n1)] = {v0, v1};
}

void tune_erase(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune.erase(make_key(op, kernel, prec, nq, rhs, n0, n1));
}

}  // namespace tct

extern "C" int tct_tune_set(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1,
                            int v0, int v1) {
    TCT_CHECK_ARG(op >= 1 && op <= 3, "tct_tune_set: unknown operation %d", op);
    TCT_CHECK_ARG(v0 >= 1 && v1 >= 1, "tct_tune_set: shape values must be positive");
    tct::tune_store(op, kernel, prec, nq, rhs, n0, n1, v0, v1);
    return TCT_OK;
}

extern "C" int tct_tune_get(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1,
                            int* v0, int* v1) {
    if (!v0 || !v1) return 0;
    return tct::tune_lookup(op, kernel, prec, nq, rhs, n0, n1, v0, v1) ? 1 : 0;
}

extern "C" int tct_tune_bucket(int64_t n) { return tct::tune_bucket(n); }

extern "C" int64_t tct_tune_size(void) {
    std::lock_guard<std::mutex> lock(tct::g_tune_mutex);
    return (int64_t)tct::g_tune.size();
}

extern "C" int tct_tune_entry(int64_t i, int* key7, int* v0, int* v1) {
    std::lock_guard<std::mutex> lock(tct::g_tune_mutex);
    TCT_CHECK_ARG(i >= 0 && i < (int64_t)tct::g_tune.size() && key7 && v0 && v1,
                  "tct_tune_entry: index %lld out of range", (long long)i);
    auto it = tct::g_tune.begin();
    std::advance(it, i);
    const tct::Key& k = it->first;
    key7[0] = std::get<0>(k); key7[1] = std::get<1>(k); key7[2] = std::get<2>(k);
    key7[3] = std::get<3>(k); key7[4] = std::get<4>(k); key7[5] = std::get<5>(k);
    key7[6] = std::get<6>(k);
    *v0 = it->second.first;
    *v1 = it->second.second;
    return TCT_OK;
}

extern "C" int tct_tune_put_entry(const int* key7, int v0, int v1) {
    TCT_CHECK_ARG(key7 && key7[0] >= 1 && key7[0] <= 3 && v0 >= 1 && v1 >= 1,
                  "tct_tune_put_entry: bad entry");
    std::lock_guard<std::mutex> lock(tct::g_tune_mutex);
    tct::g_tune[tct::Key(key7[0], key7[1], key7[2], key7[3], key7[4], key7[5], key7[6])] = {v0,
                                                                                          v1};
    return TCT_OK;
}

extern "C" void tct_tune_clear(void) {
    std::lock_guard<std::mutex> lock(tct::g_tune_mutex);
    tct::g_tune.clear();
}
