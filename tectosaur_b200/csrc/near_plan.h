// Shared between host.cpp (builds it) and near.cu (runs it): the near-pair
// search split into the host part -- the reference's two octrees and its
// dual-tree traversal down to pairs of leaves (fast_find_nearfield.cpp:22-74,
// 96-141) -- and the device part, the ball tests inside each leaf pair, the
// per-row fill and the per-row sort into (obs, src) order.
#pragma once

#include <cstdint>
#include <vector>

struct tct_near_plan {
    int64_t n_obs = 0, n_src = 0;
    double threshold = 0;
    // balls in tree order: centres, and the radius the reference's leaf test
    // reads, the original-order radius array indexed by TREE position
    std::vector<double> oc, orq, sc, srq;
    std::vector<int64_t> oorig, sorig;  // tree position -> original index
    // obs leaves reached by the traversal: ball range, and their source
    // leaves (CSR: lp_start[k] .. lp_start[k + 1] into lp_s / lp_e)
    std::vector<int64_t> leaf_start, leaf_end, lp_start, lp_s, lp_e;
    // device side (owned)
    void* dev = nullptr;        // one allocation holding the arrays below
    size_t dev_bytes = 0;
    int64_t* d_counts = nullptr;  // n_obs + 1 (row offsets after the scan)
    int64_t total = -1;
    // a plan built on the device (tct_near_plan_build_device) has its arrays
    // in `dev` already and its leaf counts here; the host vectors stay empty
    bool dev_built = false;
    int64_t nl_dev = 0, nlp_dev = 0;
};

namespace tct {
// The plan's device arrays (carved from plan->dev in this order).
struct NearDevPtrs {
    double *oc, *orq, *sc, *srq;
    int64_t *oorig, *sorig, *leaf_start, *leaf_end, *lp_start, *lp_s, *lp_e;
};
// Allocate plan->dev for the plan's sizes (near.cu).
int near_plan_alloc_device(tct_near_plan* plan);
NearDevPtrs near_plan_device_ptrs(tct_near_plan* plan);
}  // namespace tct
