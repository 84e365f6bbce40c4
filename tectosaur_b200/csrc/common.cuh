// Shared device/host helpers for the tct_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <string>

#include "tct_b200.h"

namespace tct {

// Last-error message of the calling host thread (tct_last_error()).
void set_error(const char* fmt, ...);

#define TCT_CHECK_ARG(cond, ...)            \
    do {                                    \
        if (!(cond)) {                      \
            ::tct::set_error(__VA_ARGS__);  \
            return TCT_ERR_ARG;             \
        }                                   \
    } while (0)

// Kernels launched by the library (every launch is followed by
// launch_status; read by tct_launch_count).
extern std::atomic<unsigned long long> g_launches;

inline int launch_status(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return TCT_ERR_CUDA;
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return TCT_OK;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline bool aligned(const void* p, size_t a) {
    return (reinterpret_cast<uintptr_t>(p) % a) == 0;
}

// Number of SMs of the current device (cached per device).
int sm_count();

// ---- tuned launch shapes (tune.cu) -------------------------------------------
// Operations whose launch shape is looked up: the direct farfield (value:
// source chunk count), the BSR matvec (values: lanes per block row, CTAs per
// SM), the multi-RHS farfield panel (reserved).
enum TuneOp { kTuneFar = TCT_TUNE_FARFIELD, kTuneBsr9 = TCT_TUNE_BSR9,
              kTuneFarPanel = TCT_TUNE_FAR_PANEL };
int tune_bucket(int64_t n);
bool tune_lookup(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1, int* v0,
                 int* v1);
void tune_store(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1, int v0,
                int v1);
void tune_erase(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1);

// ---- kernel catalogue (ids match tct_kernel_id) -----------------------------
enum KernelId { kU = 0, kT = 1, kA = 2, kH = 3, kRT = 4, kRA = 5, kRH = 6 };

// Elastic constants of tectosaur/kernels/__init__.py:20-258, formed in double
// then rounded to Real (the reference's constants_code evaluates the double
// literals and stores into `const Real`).
template <typename R>
struct Consts {
    R nu;
    R CsU0, CsU1;
    R CsT0, CsT1;
    R CsH0, CsH1, CsH2, CsH3;
    R CsRT0, CsRT1, CsRT2;
    R CsRH0, CsRH1, CsRH2;
};

template <typename R>
inline Consts<R> make_consts(const double* params) {
    const double PI = 3.14159265358979323846;
    // params are rounded to Real first, as the reference uploads them in float_type
    const double G = (double)(R)params[0];
    const double nu = (double)(R)params[1];
    Consts<R> c;
    c.nu = (R)nu;
    c.CsU0 = (R)((3.0 - 4.0 * nu) / (G * 16.0 * PI * (1.0 - nu)));
    c.CsU1 = (R)(1.0 / (G * 16.0 * PI * (1.0 - nu)));
    c.CsT0 = (R)((1 - 2.0 * nu) / (8.0 * PI * (1.0 - nu)));
    c.CsT1 = (R)(3.0 / (8.0 * PI * (1.0 - nu)));
    c.CsH0 = (R)(G / (4 * PI * (1 - nu)));
    c.CsH1 = (R)(1 - 2 * nu);
    c.CsH2 = (R)(-1 + 4 * nu);
    c.CsH3 = (R)(3 * nu);
    c.CsRT0 = (R)(-1.0 / (8.0 * PI * (1.0 - nu)));
    c.CsRT1 = (R)(-(1 - 2 * nu) / (8.0 * PI * (1.0 - nu)));
    c.CsRT2 = (R)(-1.0 / (4 * PI));
    c.CsRH0 = (R)(G / (8.0 * PI * (1 - nu)));
    c.CsRH1 = (R)(2 * (1 - nu));
    c.CsRH2 = (R)(4 * nu);
    return c;
}

// Levi-Civita symbol, usable in constant expressions.
__host__ __device__ constexpr int levi(int i, int j, int k) {
    return (i - j) * (j - k) * (k - i) / 2;
}

__host__ __device__ inline int positive_mod(int i, int n) { return (i % n + n) % n; }

template <typename R>
__device__ __forceinline__ R rsqrt_r(R x);
template <>
__device__ __forceinline__ float rsqrt_r<float>(float x) { return rsqrtf(x); }
template <>
__device__ __forceinline__ double rsqrt_r<double>(double x) { return rsqrt(x); }

// Triangle geometry of integral_primitives.cl:8-112: vertices (optionally
// rotated by `clicks` and with vertices 0/1 swapped by `flip`), unit normal
// of (v2 - v0) x (v2 - v1) (negated when flipped), Jacobian = |normal|, and
// the surface-curl basis (grad_b[0] * (v2 - v0) - grad_b[1] * (v1 - v0)) / J.
template <typename R>
struct TriGeom {
    R v[3][3];
    R n[3];
    R J;
    R sc[3][3];  // [basis][component]
};

template <typename R>
__device__ __forceinline__ void load_tri(TriGeom<R>& t, const R* __restrict__ pts,
                                         const int32_t* __restrict__ tris, int64_t idx,
                                         int clicks, bool flip, bool need_sc) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        int fc = c;
        if (flip) fc = (c == 0) ? 1 : ((c == 1) ? 0 : c);
        int p = tris[3 * idx + positive_mod(fc + clicks, 3)];
#pragma unroll
        for (int d = 0; d < 3; d++) t.v[c][d] = pts[3 * (int64_t)p + d];
    }
    R s20[3], s21[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        s20[d] = t.v[2][d] - t.v[0][d];
        s21[d] = t.v[2][d] - t.v[1][d];
    }
    R un[3];
    un[0] = s20[1] * s21[2] - s20[2] * s21[1];
    un[1] = s20[2] * s21[0] - s20[0] * s21[2];
    un[2] = s20[0] * s21[1] - s20[1] * s21[0];
    if (flip) {
#pragma unroll
        for (int d = 0; d < 3; d++) un[d] = -un[d];
    }
    R len = sqrt(un[0] * un[0] + un[1] * un[1] + un[2] * un[2]);
    t.J = len;
#pragma unroll
    for (int d = 0; d < 3; d++) t.n[d] = un[d] / len;
    if (need_sc) {
        // basis gradients (-1,-1), (1,0), (0,1)
        R g1[3], g2[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            g1[d] = t.v[1][d] - t.v[0][d];
            g2[d] = t.v[2][d] - t.v[0][d];
        }
#pragma unroll
        for (int s = 0; s < 3; s++) {
            t.sc[0][s] = (-g2[s] + g1[s]) / len;
            t.sc[1][s] = g2[s] / len;
            t.sc[2][s] = -g1[s] / len;
        }
    }
}

// Point of a triangle at basis values b (pts_from_basis of
// integral_primitives.cl:121-128: v = 0; v += b0 t0; v += b1 t1; v += b2 t2).
// Every kernel forms observation and source quadrature points through this one
// function, so a triangle's own points agree bit for bit wherever they are
// computed (coincident points then give r^2 == 0 exactly, as in the reference).
template <typename R>
__device__ __forceinline__ R bary_point(const TriGeom<R>& t, const R b[3], int d) {
    R v = 0;
    v += b[0] * t.v[0][d];
    v += b[1] * t.v[1][d];
    v += b[2] * t.v[2][d];
    return v;
}

}  // namespace tct
