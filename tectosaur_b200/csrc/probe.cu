// FP32 FMA-throughput probe: the denominator of the farfield kernel's
// roofline (an FP32 CUDA-core kernel; no library peak covers that pipe).
// Each thread runs 8 independent FMA chains so the pipe, not latency, bounds it.
#include "common.cuh"

namespace tct {
namespace {

__global__ void __launch_bounds__(256) fma_probe(float* out, int iters, float seed) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + 0.001f * (threadIdx.x + k);
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fmaf(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chains live
}

}  // namespace
}  // namespace tct

extern "C" int tct_fp32_fma_probe(void* out, int64_t n_blocks, int iters, void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(out && n_blocks > 0 && n_blocks < (1 << 30) && iters > 0,
                  "tct_fp32_fma_probe: bad arguments");
    fma_probe<<<(unsigned)n_blocks, 256, 0, as_stream(stream)>>>((float*)out, iters, 1.0f);
    return launch_status("tct_fp32_fma_probe");
}
