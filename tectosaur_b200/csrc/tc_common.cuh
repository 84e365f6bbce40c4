// tcgen05 helpers shared by the multi-RHS farfield panels (far_mrhs.cu,
// pts_mrhs.cu): shared-memory and instruction descriptors of the canonical
// K-major no-swizzle TF32 layout, bounded mbarrier waits, the split-TF32
// MMA, tensor-memory loads/stores and the compensated (Kahan) fold of the
// accumulator, bulk async copies (no multicast).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tct {

constexpr int TC_M = 128;                                   // MMA M (rows per CTA)
constexpr unsigned long long TC_WAIT_NS = 200000000ull;      // 0.2 s per bounded wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ float tf32_round(float x) {
    uint32_t y;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(y) : "f"(x));
    return __uint_as_float(y);
}

// shared-memory matrix descriptor, K-major, no swizzle (version 1)
__host__ __device__ __forceinline__ uint64_t mr_smem_desc(uint32_t saddr, uint32_t lbo_bytes,
                                                          uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3fff);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3fff) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3fff) << 32;
    d |= (uint64_t)1 << 46;  // version
    // base offset 0, lbo mode 0, layout type 0 (no swizzle)
    return d;
}

// instruction descriptor: D F32, A/B TF32, both K-major, M = 128, N
__host__ __device__ __forceinline__ uint32_t mr_instr_desc(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(TC_M >> 4) << 24);
}

// byte offset of element (row, k) in a K-major no-swizzle operand tile
__host__ __device__ __forceinline__ uint32_t mr_off(int row, int k, int rows) {
    return (uint32_t)((k >> 2) * (rows / 8) * 128 + (row >> 3) * 128 + (row & 7) * 16 +
                      (k & 3) * 4);
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for phase `phase` of an mbarrier (the MMA completion).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    const unsigned long long start = gtimer();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
        if (gtimer() - start > TC_WAIT_NS) return false;
    }
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
    uint32_t mask[4] = {0, 0, 0, 0};
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask[0]), "r"(mask[1]),
          "r"(mask[2]), "r"(mask[3]));
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t u[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]),
          "=r"(u[7])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = __uint_as_float(u[k]);
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float (&v)[8]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(
            taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])));
}

// Fold columns [c_begin, c_end) of the accumulator D (columns [0, N)) into
// the Kahan pair S = [N, 2N), C = [2N, 3N) of this warp's lanes; `first`
// initialises S = D, C = 0.
template <int N>
__device__ __forceinline__ void tmem_fold(uint32_t lane_base, int c_begin, int c_end, bool first) {
#pragma unroll 1
    for (int c0 = c_begin; c0 < c_end; c0 += 8) {
        float d[8], sv[8], cv[8];
        tmem_ld8(lane_base + c0, d);
        if (!first) {
            tmem_ld8(lane_base + N + c0, sv);
            tmem_ld8(lane_base + 2 * N + c0, cv);
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (first) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                sv[k] = d[k];
                cv[k] = 0.f;
            }
        } else {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const float y = d[k] - cv[k];
                const float t = sv[k] + y;
                cv[k] = (t - sv[k]) - y;
                sv[k] = t;
            }
        }
        tmem_st8(lane_base + N + c0, sv);
        tmem_st8(lane_base + 2 * N + c0, cv);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

}  // namespace tct
