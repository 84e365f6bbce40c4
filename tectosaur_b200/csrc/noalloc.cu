// Allocation-free farfield matvec.
//
// Some callers of this library cannot allocate device memory at the moment
// they apply the operator: code running inside a CUDA stream capture that
// must not add memory nodes, embedders whose device memory is owned by
// another allocator or pool (cudaMalloc would fragment or bypass it), and
// environments where cudaMalloc may synchronise the device or is disallowed
// on the hot path.  tct_farfield_tris_matvec needs a scratch workspace the
// caller normally allocates; this entry point instead uses a fixed scratch
// array compiled into the library, so the caller passes only its inputs and
// outputs and nothing is allocated.
//
// The scratch is a file-scope __device__ array of TCT_NOALLOC_SCRATCH_BYTES
// (32 MiB).  Every GPU that loads the library holds it until the process
// exits.  Host code cannot use the array's name as a device address, so the
// first call on each device looks the address up with cudaGetSymbolAddress
// (with that device current) and caches it; make that first call before any
// stream capture.  All calls share the one array and it keeps the last call's
// contents: nothing in it has to start at zero (every byte a call reads was
// written earlier in the same call), but two calls that run at the same time
// on the GPU -- on different streams, or from different host threads --
// overwrite each other's scratch and race.  The cached address belongs to the
// device's primary context: do not call cudaDeviceReset between calls (the
// context it creates afterwards holds the array at a new address).
#include <mutex>

#include "common.cuh"

namespace tct {
namespace {

constexpr size_t kScratchBytes = TCT_NOALLOC_SCRATCH_BYTES;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_scratch_mutex;
void* g_scratch_ptr[64] = {nullptr};

int scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error("tct_farfield_tris_matvec_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
        return TCT_ERR_CUDA;
    }
    if (dev < 0 || dev >= 64) {
        set_error("tct_farfield_tris_matvec_noalloc: device ordinal %d out of range", dev);
        return TCT_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("tct_farfield_tris_matvec_noalloc: cudaGetSymbolAddress: %s",
                      cudaGetErrorString(e));
            return TCT_ERR_CUDA;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return TCT_OK;
}

}  // namespace
}  // namespace tct

extern "C" size_t tct_farfield_noalloc_capacity(void) { return tct::kScratchBytes; }

extern "C" int tct_farfield_tris_matvec_noalloc(int kernel, int prec, void* out, const void* in,
                                                const void* pts, const int32_t* obs_tris,
                                                int64_t n_obs, const int32_t* src_tris,
                                                int64_t n_src, int n_q, const double* quad_pts,
                                                const double* quad_wts, const double* params,
                                                int accumulate, void* stream) {
    using namespace tct;
    // Same order of argument checks as tct_farfield_tris_matvec: sizes first,
    // then the cases with nothing to integrate (no scratch needed), then the
    // scratch capacity.
    TCT_CHECK_ARG(n_obs >= 0 && n_src >= 0, "tct_farfield_tris_matvec_noalloc: negative size");
    if (n_obs == 0) return TCT_OK;
    if (n_src == 0)
        return tct_farfield_tris_matvec(kernel, prec, out, in, pts, obs_tris, n_obs, src_tris,
                                        n_src, n_q, quad_pts, quad_wts, params, accumulate,
                                        nullptr, 0, stream);
    const size_t need = tct_farfield_workspace_bytes(kernel, prec, n_obs, n_src, n_q);
    if (need == 0) {
        set_error("tct_farfield_tris_matvec_noalloc: unsupported kernel %d, precision %d or "
                  "%d-point rule", kernel, prec, n_q);
        return TCT_ERR_ARG;
    }
    if (need > kScratchBytes) {
        set_error("tct_farfield_tris_matvec_noalloc: this problem (%lld obs x %lld src "
                  "triangles) needs %zu bytes of scratch; the built-in scratch holds %zu bytes "
                  "-- use tct_farfield_tris_matvec with a caller-provided workspace",
                  (long long)n_obs, (long long)n_src, need, kScratchBytes);
        return TCT_ERR_ARG;
    }
    void* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    return tct_farfield_tris_matvec(kernel, prec, out, in, pts, obs_tris, n_obs, src_tris, n_src,
                                    n_q, quad_pts, quad_wts, params, accumulate, scratch,
                                    kScratchBytes, stream);
}
