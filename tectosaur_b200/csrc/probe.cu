// FMA-throughput probes: the denominators of the CUDA-core kernels'
// rooflines (FP32 farfield, FP64 pair quadrature; no library peak covers
// those pipes).
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

// Packed variant: 8 independent chains of fma.rn.f32x2 (two FP32 FMAs per
// instruction, sm_100a).
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b,
                                                    unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

__device__ __forceinline__ unsigned long long pack2(float x, float y) {
    return (unsigned long long)__float_as_uint(x) | ((unsigned long long)__float_as_uint(y) << 32);
}

__global__ void __launch_bounds__(256) fma2_probe(float* out, int iters, float seed) {
    unsigned long long a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = pack2(seed + 0.001f * threadIdx.x, seed + 0.002f * k);
    const unsigned long long m = pack2(0.999999f, 0.999999f), c = pack2(1e-7f, 1e-7f);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = ffma2(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++)
        s += __uint_as_float((unsigned)(a[k] & 0xffffffffu)) + __uint_as_float((unsigned)(a[k] >> 32));
    if (s == 12345.678f) out[threadIdx.x] = s;
}

// FP64 variant: the denominator of the FP64 pair-quadrature roofline.
__global__ void __launch_bounds__(256) dfma_probe(double* out, int iters, double seed) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + 0.001 * (threadIdx.x + k);
    const double m = 0.999999999, c = 1e-12;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fma(a[k], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == 12345.678) out[threadIdx.x] = s;
}

}  // namespace
}  // namespace tct

extern "C" int tct_fp64_fma_probe(void* out, int64_t n_blocks, int iters, void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(out && n_blocks > 0 && n_blocks < (1 << 30) && iters > 0,
                  "tct_fp64_fma_probe: bad arguments");
    dfma_probe<<<(unsigned)n_blocks, 256, 0, as_stream(stream)>>>((double*)out, iters, 1.0);
    return launch_status("tct_fp64_fma_probe");
}

extern "C" int tct_fp32_fma_probe(void* out, int64_t n_blocks, int iters, void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(out && n_blocks > 0 && n_blocks < (1 << 30) && iters > 0,
                  "tct_fp32_fma_probe: bad arguments");
    fma_probe<<<(unsigned)n_blocks, 256, 0, as_stream(stream)>>>((float*)out, iters, 1.0f);
    return launch_status("tct_fp32_fma_probe");
}

extern "C" int tct_fp32x2_fma_probe(void* out, int64_t n_blocks, int iters, void* stream) {
    using namespace tct;
    TCT_CHECK_ARG(out && n_blocks > 0 && n_blocks < (1 << 30) && iters > 0,
                  "tct_fp32x2_fma_probe: bad arguments");
    fma2_probe<<<(unsigned)n_blocks, 256, 0, as_stream(stream)>>>((float*)out, iters, 1.0f);
    return launch_status("tct_fp32x2_fma_probe");
}

namespace tct {
std::atomic<unsigned long long> g_launches{0};
}

extern "C" uint64_t tct_launch_count(void) {
    return tct::g_launches.load(std::memory_order_relaxed);
}
