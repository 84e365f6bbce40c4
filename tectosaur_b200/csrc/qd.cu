// Quasidynamic rate-and-state stepper pieces, FP64 (the reference runs them
// on the host: qd/newton.cpp, qd/pt_average.cpp, qd/model_helpers.py, and the
// scipy conjugate-gradient mass solve of qd/full_model.py:160-176).
//
//   qd_rate_state    one thread per DOF: the Newton solve of
//                    tau_qs - eta V = a sigma_n asinh(V / (2 V0) e^(state/a)) - C
//                    for the slip speed along the shear traction
//                    (newton.cpp:18-131), started at V = 0, stopping when
//                    |V1 - V0| <= tol |V0|; DOFs that do not converge are
//                    counted and keep their last iterate (the reference's
//                    convergence assert is compiled out under NDEBUG);
//   qd_velocity      one thread per DOF: the vertex average of the Newton
//                    velocity (summed over the vertex's corners in DOF order,
//                    divided by their count: pt_average.cpp:10-35), the
//                    optional no-backslip filter, plus the plate-rate field
//                    on the free edges (model_helpers.py:96-116), and the
//                    aging-law state derivative (model_helpers.py:122-130);
//   cg_csr_block     one CTA: conjugate gradients on a CSR matrix with x0 = 0,
//                    stopping when ||r|| < max(atol, rtol ||b||), the
//                    iteration of scipy.sparse.linalg.cg, with the vector
//                    updates rounded as scipy's (no fused multiply-add); a
//                    non-finite right-hand side or residual returns the NaN
//                    solution at once (iterations -1), where scipy's
//                    iteration runs out its maxiter first.
#include "common.cuh"

namespace tct {
namespace {

__device__ __forceinline__ double rs_F(double V, double sn, double st, double a, double V0,
                                       double C) {
    return a * sn * asinh(V / (2 * V0) * exp(st / a)) - C;
}

__device__ __forceinline__ double rs_dFdV(double V, double sn, double st, double a, double V0) {
    const double expsa = exp(st / a);
    const double Q = (V * expsa) / (2 * V0);
    return a * expsa * sn / (2 * V0 * sqrt(1 + (Q * Q)));
}

__device__ double newton_rs(double tau, double eta, double sn, double st, double a, double V0,
                            double C, double tol, int maxiter, bool& ok) {
    double x0 = 0.0;
    for (int i = 0; i < maxiter; i++) {
        const double y = tau - eta * x0 - rs_F(x0, sn, st, a, V0, C);
        const double yp = -eta - rs_dFdV(x0, sn, st, a, V0);
        const double x1 = x0 - y / yp;
        if (fabs(x1 - x0) <= tol * fabs(x0)) {
            ok = true;
            return x1;
        }
        x0 = x1;
    }
    ok = false;
    return x0;
}

__global__ void __launch_bounds__(128)
qd_rate_state(int64_t n_dofs, int n_sys, int basis_dim, const double* __restrict__ normals,
              const double* __restrict__ traction, int64_t traction_stride,
              const double* __restrict__ state, int64_t state_stride,
              const double* __restrict__ a, double eta, double V0, double C,
              const double* __restrict__ normal_stress, double tol, int maxiter, int separate,
              double* __restrict__ velocity, int64_t velocity_stride,
              int* __restrict__ n_failed) {
    // one thread per (system, DOF); the mesh fields are shared by the systems
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_dofs * n_sys) return;
    const int64_t sys = g / n_dofs, dof = g - sys * n_dofs;
    const double* t = traction + sys * traction_stride + dof * 3;
    double* v = velocity + sys * velocity_stride + dof * 3;
    const double st = state[sys * state_stride + dof], ad = a[dof], extra = normal_stress[dof];
    bool ok = true;
    if (separate) {
        for (int k = 0; k < 3; k++) {
            bool okk;
            const double m = newton_rs(fabs(t[k]), eta, 0.0 + extra, st, ad, V0, C, tol, maxiter,
                                       okk);
            ok = ok && okk;
            v[k] = m * (double)((t[k] > 0) - (t[k] < 0));
        }
    } else {
        const double* n = normals + (dof / basis_dim) * 3;
        const double nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
        const double f = (t[0] * n[0] + t[1] * n[1] + t[2] * n[2]) / nn;
        const double nv[3] = {n[0] * f, n[1] * f, n[2] * f};
        const double sh[3] = {t[0] - nv[0], t[1] - nv[1], t[2] - nv[2]};
        const double nmag = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
        const double smag = sqrt(sh[0] * sh[0] + sh[1] * sh[1] + sh[2] * sh[2]);
        if (smag < 1e-14) {
            v[0] = v[1] = v[2] = 0.0;
        } else {
            const double m = newton_rs(smag, eta, nmag + extra, st, ad, V0, C, tol, maxiter, ok);
            const double inv = 1.0 / smag;
            for (int k = 0; k < 3; k++) v[k] = sh[k] * inv * m;
        }
    }
    if (!ok) atomicAdd(n_failed, 1);
}

__global__ void __launch_bounds__(128)
qd_velocity(int64_t n_dofs, int n_sys, const int32_t* __restrict__ vert_start,
            const int32_t* __restrict__ vert_dofs, const int32_t* __restrict__ dof_vert,
            const double* __restrict__ v_newton, int64_t vn_stride,
            const double* __restrict__ field_edges, const double* __restrict__ field_interior,
            double plate_rate, int no_backslip, const double* __restrict__ state,
            int64_t state_stride, const double* __restrict__ b, double V0, double Dc, double f0,
            double* __restrict__ velocity, int64_t velocity_stride, double* __restrict__ dstatedt,
            int64_t dstate_stride) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_dofs * n_sys) return;
    const int64_t sys = g / n_dofs, dof = g - sys * n_dofs;
    v_newton += sys * vn_stride;
    state += sys * state_stride;
    velocity += sys * velocity_stride;
    dstatedt += sys * dstate_stride;
    const int32_t p = dof_vert[dof];
    const int32_t s = vert_start[p], e = vert_start[p + 1];
    double avg[3];
    for (int k = 0; k < 3; k++) {
        double sum = 0.0;
        for (int32_t j = s; j < e; j++) sum += v_newton[(int64_t)vert_dofs[j] * 3 + k];
        avg[k] = sum / (double)(e - s);
    }
    if (no_backslip) {
        const double* fi = field_interior + dof * 3;
        const double nf = sqrt(fi[0] * fi[0] + fi[1] * fi[1] + fi[2] * fi[2]);
        const double speed = (avg[0] * fi[0] + avg[1] * fi[1] + avg[2] * fi[2]) / nf;
        if (speed < 0 || isnan(speed)) avg[0] = avg[1] = avg[2] = 0.0;
    }
    double* v = velocity + dof * 3;
    const double* fe = field_edges + dof * 3;
    for (int k = 0; k < 3; k++) v[k] = fe[k] * plate_rate + avg[k];
    const double vmag = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double bd = b[dof];
    dstatedt[dof] = (bd * V0 / Dc) * (exp((f0 - state[dof]) / bd) - (vmag / V0));
}

constexpr int CG_THREADS = 1024;

// Sum of v over the block (every thread gets the result).
__device__ double block_sum(double v, double* red) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
    return t;
}

__global__ void __launch_bounds__(CG_THREADS)
cg_csr_block(int64_t n, const int64_t* __restrict__ indptr, const int64_t* __restrict__ indices,
             const double* __restrict__ data, const double* __restrict__ bvec, int64_t b_stride,
             double* __restrict__ x, int64_t x_stride, double* __restrict__ work, double rtol,
             double atol_in, int maxiter, int* __restrict__ iters) {
    // one CTA per system (blockIdx.x), all with the same matrix
    __shared__ double red[32];
    const int tid = threadIdx.x;
    bvec += blockIdx.x * b_stride;
    x += blockIdx.x * x_stride;
    double* __restrict__ r = work + (int64_t)blockIdx.x * 3 * n;
    double* __restrict__ p = r + n;
    double* __restrict__ q = p + n;
    iters += blockIdx.x;
    double bb = 0.0;
    for (int64_t i = tid; i < n; i += blockDim.x) bb += bvec[i] * bvec[i];
    const double bnrm2 = sqrt(block_sum(bb, red));
    if (bnrm2 == 0.0) {
        for (int64_t i = tid; i < n; i += blockDim.x) x[i] = bvec[i];
        if (tid == 0) *iters = 0;
        return;
    }
    if (!isfinite(bnrm2)) {
        // a non-finite right-hand side (a state the stepper will reject):
        // scipy's cg never meets its stopping test then and returns a NaN
        // solution after maxiter iterations; return that solution at once
        for (int64_t i = tid; i < n; i += blockDim.x) x[i] = nan("");
        if (tid == 0) *iters = -1;
        return;
    }
    const double atol = fmax(atol_in, rtol * bnrm2);
    for (int64_t i = tid; i < n; i += blockDim.x) {
        x[i] = 0.0;
        r[i] = bvec[i];
    }
    double rho_prev = 0.0;
    int it = 0;
    for (; it < maxiter; it++) {
        __syncthreads();
        double rr = 0.0;
        for (int64_t i = tid; i < n; i += blockDim.x) rr += r[i] * r[i];
        const double rho = block_sum(rr, red);  // r . z with z = r
        if (sqrt(rho) < atol) break;
        if (!isfinite(rho)) {  // the iteration broke down: the NaN solution, at once
            for (int64_t i = tid; i < n; i += blockDim.x) x[i] = nan("");
            it = -1;
            break;
        }
        const double beta = it > 0 ? rho / rho_prev : 0.0;
        for (int64_t i = tid; i < n; i += blockDim.x)
            p[i] = it > 0 ? __dadd_rn(__dmul_rn(p[i], beta), r[i]) : r[i];
        __syncthreads();
        double pq = 0.0;
        for (int64_t i = tid; i < n; i += blockDim.x) {
            double acc = 0.0;
            for (int64_t k = indptr[i]; k < indptr[i + 1]; k++) acc += data[k] * p[indices[k]];
            q[i] = acc;
            pq += p[i] * acc;
        }
        const double alpha = rho / block_sum(pq, red);
        for (int64_t i = tid; i < n; i += blockDim.x) {
            x[i] = __dadd_rn(x[i], __dmul_rn(alpha, p[i]));
            r[i] = __dsub_rn(r[i], __dmul_rn(alpha, q[i]));
        }
        rho_prev = rho;
    }
    if (tid == 0) *iters = it;
}

}  // namespace
}  // namespace tct

using namespace tct;

extern "C" int tct_qd_rate_state_batch(int64_t n_tris, int basis_dim, int n_sys,
                                       const double* tri_normals, const double* traction,
                                       int64_t traction_stride, const double* state,
                                       int64_t state_stride, const double* a, double eta,
                                       double V0, double C, const double* normal_stress,
                                       double tol, int maxiter, int separate_dims,
                                       double* velocity, int64_t velocity_stride, int* n_failed,
                                       void* stream) {
    TCT_CHECK_ARG(n_tris >= 0 && basis_dim >= 1 && maxiter >= 0 && n_sys >= 0,
                  "tct_qd_rate_state: bad sizes");
    const int64_t n = n_tris * basis_dim;
    if (n == 0 || n_sys == 0) return TCT_OK;
    TCT_CHECK_ARG(tri_normals && traction && state && a && normal_stress && velocity && n_failed,
                  "tct_qd_rate_state: null pointer");
    const int64_t m = n * n_sys;
    qd_rate_state<<<(unsigned)((m + 127) / 128), 128, 0, as_stream(stream)>>>(
        n, n_sys, basis_dim, tri_normals, traction, traction_stride, state, state_stride, a, eta,
        V0, C, normal_stress, tol, maxiter, separate_dims, velocity, velocity_stride, n_failed);
    return launch_status("tct_qd_rate_state");
}

extern "C" int tct_qd_rate_state(int64_t n_tris, int basis_dim, const double* tri_normals,
                                 const double* traction, const double* state, const double* a,
                                 double eta, double V0, double C, const double* normal_stress,
                                 double tol, int maxiter, int separate_dims, double* velocity,
                                 int* n_failed, void* stream) {
    return tct_qd_rate_state_batch(n_tris, basis_dim, 1, tri_normals, traction, 0, state, 0, a,
                                   eta, V0, C, normal_stress, tol, maxiter, separate_dims,
                                   velocity, 0, n_failed, stream);
}

extern "C" int tct_qd_velocity_state_batch(int64_t n_dofs, int n_sys, const int32_t* vert_start,
                                           const int32_t* vert_dofs, const int32_t* dof_vert,
                                           const double* v_newton, int64_t vn_stride,
                                           const double* field_edges,
                                           const double* field_interior, double plate_rate,
                                           int no_backslip, const double* state,
                                           int64_t state_stride, const double* b, double V0,
                                           double Dc, double f0, double* velocity,
                                           int64_t velocity_stride, double* dstatedt,
                                           int64_t dstate_stride, void* stream) {
    TCT_CHECK_ARG(n_dofs >= 0 && n_sys >= 0, "tct_qd_velocity_state: negative size");
    if (n_dofs == 0 || n_sys == 0) return TCT_OK;
    TCT_CHECK_ARG(vert_start && vert_dofs && dof_vert && v_newton && field_edges &&
                      field_interior && state && b && velocity && dstatedt,
                  "tct_qd_velocity_state: null pointer");
    const int64_t m = n_dofs * n_sys;
    qd_velocity<<<(unsigned)((m + 127) / 128), 128, 0, as_stream(stream)>>>(
        n_dofs, n_sys, vert_start, vert_dofs, dof_vert, v_newton, vn_stride, field_edges,
        field_interior, plate_rate, no_backslip, state, state_stride, b, V0, Dc, f0, velocity,
        velocity_stride, dstatedt, dstate_stride);
    return launch_status("tct_qd_velocity_state");
}

extern "C" int tct_qd_velocity_state(int64_t n_dofs, const int32_t* vert_start,
                                     const int32_t* vert_dofs, const int32_t* dof_vert,
                                     const double* v_newton, const double* field_edges,
                                     const double* field_interior, double plate_rate,
                                     int no_backslip, const double* state, const double* b,
                                     double V0, double Dc, double f0, double* velocity,
                                     double* dstatedt, void* stream) {
    return tct_qd_velocity_state_batch(n_dofs, 1, vert_start, vert_dofs, dof_vert, v_newton, 0,
                                       field_edges, field_interior, plate_rate, no_backslip,
                                       state, 0, b, V0, Dc, f0, velocity, 0, dstatedt, 0, stream);
}

extern "C" int tct_cg_csr_batch(int64_t n, int n_sys, const int64_t* indptr,
                                const int64_t* indices, const double* data, const double* b,
                                int64_t b_stride, double* x, int64_t x_stride, double* work,
                                double rtol, double atol, int maxiter, int* iters, void* stream) {
    TCT_CHECK_ARG(n >= 0 && maxiter >= 0 && n_sys >= 0, "tct_cg_csr: bad sizes");
    if (n == 0 || n_sys == 0) return TCT_OK;
    TCT_CHECK_ARG(indptr && indices && data && b && x && work && iters,
                  "tct_cg_csr: null pointer");
    cg_csr_block<<<(unsigned)n_sys, CG_THREADS, 0, as_stream(stream)>>>(
        n, indptr, indices, data, b, b_stride, x, x_stride, work, rtol, atol, maxiter, iters);
    return launch_status("tct_cg_csr");
}

extern "C" int tct_cg_csr(int64_t n, const int64_t* indptr, const int64_t* indices,
                          const double* data, const double* b, double* x, double* work,
                          double rtol, double atol, int maxiter, int* iters, void* stream) {
    return tct_cg_csr_batch(n, 1, indptr, indices, data, b, 0, x, 0, work, rtol, atol, maxiter,
                            iters, stream);
}
