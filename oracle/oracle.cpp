// Test infrastructure: CPU restatement of the reference's elastic-BEM kernels.
// Checker for the CUDA product and bench.py's CPU baseline; never shipped.
// Each function cites the reference file:line it restates.  Expression order
// follows the reference templates so the FP64 results agree to rounding.
#include "oracle.h"

#include <cmath>
#include <algorithm>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

constexpr double PI = 3.14159265358979323846;

// Levi-Civita symbol e[i][j][k] = (i-j)(j-k)(k-i)/2 (kernels/kernels.cl:4-5).
inline int levi(int i, int j, int k) { return (i - j) * (j - k) * (k - i) / 2; }
inline int kron(int i, int j) { return i == j ? 1 : 0; }

inline int positive_mod(int i, int n) { return (i % n + n) % n; }

// Triangle geometry: integral_primitives.cl:8-112.
template <typename R>
struct TriInfo {
    R tri[3][3];
    R unscaled_normal[3];
    R jacobian;
    R n[3];           // unit normal
    R surf_curl[3][3];  // [basis][component]
};

template <typename R>
void tri_info(TriInfo<R>& t, const R* pts, const int* tris, int tri_idx,
              int clicks, bool flip) {
    for (int c = 0; c < 3; c++) {
        int fc = c;
        if (flip) {
            if (c == 0) fc = 1;
            else if (c == 1) fc = 0;
        }
        int pt_idx = tris[3 * tri_idx + positive_mod(fc + clicks, 3)];
        for (int d = 0; d < 3; d++) t.tri[c][d] = pts[pt_idx * 3 + d];
    }
    R s20[3], s21[3];
    for (int d = 0; d < 3; d++) {
        s20[d] = t.tri[2][d] - t.tri[0][d];
        s21[d] = t.tri[2][d] - t.tri[1][d];
    }
    t.unscaled_normal[0] = s20[1] * s21[2] - s20[2] * s21[1];
    t.unscaled_normal[1] = s20[2] * s21[0] - s20[0] * s21[2];
    t.unscaled_normal[2] = s20[0] * s21[1] - s20[1] * s21[0];
    if (flip) {
        for (int d = 0; d < 3; d++) t.unscaled_normal[d] *= -1;
    }
    R len = std::sqrt(t.unscaled_normal[0] * t.unscaled_normal[0] +
                      t.unscaled_normal[1] * t.unscaled_normal[1] +
                      t.unscaled_normal[2] * t.unscaled_normal[2]);
    t.jacobian = len;
    for (int d = 0; d < 3; d++) t.n[d] = t.unscaled_normal[d] / len;
    const R grad[3][2] = {{-1.0, -1.0}, {1.0, 0.0}, {0.0, 1.0}};
    R g1[3], g2[3];
    for (int d = 0; d < 3; d++) {
        g1[d] = t.tri[1][d] - t.tri[0][d];
        g2[d] = t.tri[2][d] - t.tri[0][d];
    }
    for (int b = 0; b < 3; b++)
        for (int s = 0; s < 3; s++)
            t.surf_curl[b][s] = (+grad[b][0] * g2[s] - grad[b][1] * g1[s]) / t.jacobian;
}

// Kernel constants: kernels/__init__.py:20-258 (constants_code strings).
template <typename R>
struct Consts {
    R G, nu;
    R CsU0, CsU1;
    R CsT0, CsT1;
    R CsH0, CsH1, CsH2, CsH3;
    R CsRT0, CsRT1, CsRT2;
    R CsRH0, CsRH1, CsRH2;
    explicit Consts(const R* params) {
        G = params[0];
        nu = params[1];
        CsU0 = (3.0 - 4.0 * nu) / (G * 16.0 * PI * (1.0 - nu));
        CsU1 = 1.0 / (G * 16.0 * PI * (1.0 - nu));
        CsT0 = (1 - 2.0 * nu) / (8.0 * PI * (1.0 - nu));
        CsT1 = 3.0 / (8.0 * PI * (1.0 - nu));
        CsH0 = G / (4 * PI * (1 - nu));
        CsH1 = 1 - 2 * nu;
        CsH2 = -1 + 4 * nu;
        CsH3 = 3 * nu;
        CsRT0 = -1.0 / (8.0 * PI * (1.0 - nu));
        CsRT1 = -(1 - 2 * nu) / (8.0 * PI * (1.0 - nu));
        CsRT2 = -1.0 / (4 * PI);
        CsRH0 = G / (8.0 * PI * (1 - nu));
        CsRH1 = 2 * (1 - nu);
        CsRH2 = 4 * nu;
    }
};

template <typename R>
inline R rsqrt_(R x) { return R(1) / std::sqrt(x); }

// 3x3 tensor kernels U/T/A/H: kernels/__init__.py:37-50 (U), :101-125 (T/A),
// :174-214 (H).  Karr is row-major [d_obs][d_src].
template <typename R>
void tensor_UTAH(int kernel, const Consts<R>& c, R Dx, R Dy, R Dz, R r2,
                 const R* nobs, const R* nsrc, R* Karr) {
    if (kernel == 0) {
        R invr = rsqrt_(r2);
        R Q1 = c.CsU0 * invr;
        R Q2 = c.CsU1 * invr / r2;
        Karr[0] = Q2 * Dx * Dx + Q1;
        Karr[1] = Q2 * Dx * Dy;
        Karr[2] = Q2 * Dx * Dz;
        Karr[3] = Q2 * Dy * Dx;
        Karr[4] = Q2 * Dy * Dy + Q1;
        Karr[5] = Q2 * Dy * Dz;
        Karr[6] = Q2 * Dz * Dx;
        Karr[7] = Q2 * Dz * Dy;
        Karr[8] = Q2 * Dz * Dz + Q1;
    } else if (kernel == 1 || kernel == 2) {
        // T: minus_or_plus = -, plus_or_minus = +, n = nsrc; A: +, -, nobs.
        const bool T = kernel == 1;
        const R mp = T ? R(-1) : R(1);
        const R pm = T ? R(1) : R(-1);
        const R* n = T ? nsrc : nobs;
        R invr = rsqrt_(r2);
        R invr2 = invr * invr;
        R invr3 = invr2 * invr;
        R rn = n[0] * Dx + n[1] * Dy + n[2] * Dz;
        R A = pm * c.CsT0 * invr3;
        R C = mp * c.CsT1 * invr3 * invr2;
        R nxdy = n[0] * Dy - n[1] * Dx;
        R nzdx = n[2] * Dx - n[0] * Dz;
        R nzdy = n[2] * Dy - n[1] * Dz;
        Karr[0] = A * -rn + C * Dx * rn * Dx;
        Karr[1] = A * (mp * nxdy) + C * Dx * rn * Dy;
        Karr[2] = A * (pm * nzdx) + C * Dx * rn * Dz;
        Karr[3] = A * (pm * nxdy) + C * Dy * rn * Dx;
        Karr[4] = A * -rn + C * Dy * rn * Dy;
        Karr[5] = A * (pm * nzdy) + C * Dy * rn * Dz;
        Karr[6] = A * (mp * nzdx) + C * Dz * rn * Dx;
        Karr[7] = A * (mp * nzdy) + C * Dz * rn * Dy;
        Karr[8] = A * -rn + C * Dz * rn * Dz;
    } else {
        R invr = rsqrt_(r2);
        R invr2 = invr * invr;
        R invr3 = invr2 * invr;
        R Dor[3] = {invr * Dx, invr * Dy, invr * Dz};
        R rn = nsrc[0] * Dor[0] + nsrc[1] * Dor[1] + nsrc[2] * Dor[2];
        R rm = nobs[0] * Dor[0] + nobs[1] * Dor[1] + nobs[2] * Dor[2];
        R mn = nobs[0] * nsrc[0] + nobs[1] * nsrc[1] + nobs[2] * nsrc[2];
        R Q = c.CsH0 * invr3;
        R A = Q * 3 * rn;
        R B = Q * c.CsH1;
        R C = Q * c.CsH3;
        R MT[3], NT[3], DT[3];
        for (int d = 0; d < 3; d++) {
            MT[d] = Q * c.CsH2 * nsrc[d] + A * c.CsH1 * Dor[d];
            NT[d] = B * nobs[d] + C * Dor[d] * rm;
            DT[d] = B * 3 * nsrc[d] * rm + C * Dor[d] * mn + A * (c.nu * nobs[d] - 5 * Dor[d] * rm);
        }
        R ST = A * c.nu * rm + B * mn;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                Karr[i * 3 + j] = nsrc[i] * NT[j] + nobs[i] * MT[j] + Dor[i] * DT[j] + (i == j ? ST : R(0));
    }
}

// Gimk of kernels/kernels.cl:20-27.
template <typename R>
inline R gimk(int p, int m, int j, R Q1, R Q2, const R* D) {
    R A = Q1 * levi(m, p, j);
    R B = 0.0;
    for (int It = 0; It < 3; It++) B += levi(m, It, j) * D[It];
    return A + Q2 * D[p] * B;
}

// Pair integration with the tensor kernels: integral_primitives.cl:146-213,
// kernels/kernels.cl:29-98 (RT/RA/RH tensor forms, no Kahan).
template <typename R>
void integrate_pair(int kernel, const Consts<R>& c, const TriInfo<R>& o,
                    const TriInfo<R>& s, int n_q, const R* qp, const R* qw,
                    bool check0, R* result_temp) {
    R kahanC[81];
    for (int i = 0; i < 81; i++) {
        result_temp[i] = 0;
        kahanC[i] = 0;
    }
    for (int iq = 0; iq < n_q; iq++) {
        R obsxhat = qp[iq * 4 + 0], obsyhat = qp[iq * 4 + 1];
        R srcxhat = qp[iq * 4 + 2], srcyhat = qp[iq * 4 + 3];
        R quadw = qw[iq];
        R obsb[3] = {1 - obsxhat - obsyhat, obsxhat, obsyhat};
        R srcb[3] = {1 - srcxhat - srcyhat, srcxhat, srcyhat};
        R x[3], y[3];
        for (int d = 0; d < 3; d++) {
            x[d] = 0;
            y[d] = 0;
            for (int b = 0; b < 3; b++) {
                x[d] += obsb[b] * o.tri[b][d];
            }
            for (int b = 0; b < 3; b++) {
                y[d] += srcb[b] * s.tri[b][d];
            }
        }
        R D[3] = {y[0] - x[0], y[1] - x[1], y[2] - x[2]};
        R r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
        if (check0 && r2 == 0.0) continue;

        if (kernel <= 3) {
            R Karr[9];
            tensor_UTAH(kernel, c, D[0], D[1], D[2], r2, o.n, s.n, Karr);
            for (int d = 0; d < 3; d++) obsb[d] *= quadw;
            int idx = 0;
            for (int bo = 0; bo < 3; bo++)
                for (int dob = 0; dob < 3; dob++)
                    for (int bs = 0; bs < 3; bs++)
                        for (int ds = 0; ds < 3; ds++, idx++) {
                            R val = obsb[bo] * srcb[bs] * Karr[dob * 3 + ds];
                            R yk = val - kahanC[idx];
                            R t = result_temp[idx] + yk;
                            kahanC[idx] = (t - result_temp[idx]) - yk;
                            result_temp[idx] = t;
                        }
        } else if (kernel == 4 || kernel == 5) {
            // elasticRTA3_setup + elasticRTA3_tensor (kernels.cl:11-68).
            const bool RT = kernel == 4;
            const R* nn = RT ? s.n : o.n;
            R invr = rsqrt_(r2);
            R invr3 = invr * invr * invr;
            R Q1 = c.CsRT1 * invr;
            R Q2 = c.CsRT0 * invr3;
            R Q3 = c.CsRT2 * invr3;
            R Q3nD = Q3 * (nn[0] * D[0] + nn[1] * D[1] + nn[2] * D[2]);
            for (int dob = 0; dob < 3; dob++)
                for (int ds = 0; ds < 3; ds++) {
                    int L_d = RT ? dob : ds;
                    int R_d = RT ? ds : dob;
                    for (int bR = 0; bR < 3; bR++) {
                        R Kval = 0.0;
                        for (int Ij = 0; Ij < 3; Ij++) {
                            R g = gimk<R>(L_d, Ij, R_d, Q1, Q2, D);
                            Kval += g * (RT ? s.surf_curl[bR][Ij] : o.surf_curl[bR][Ij]);
                        }
                        if (dob == ds) {
                            Kval += Q3nD * (RT ? srcb[bR] : obsb[bR]) * (RT ? 1 : -1);
                        }
                        for (int bL = 0; bL < 3; bL++) {
                            R val = quadw * (RT ? obsb[bL] : srcb[bL]) * Kval;
                            int b_obs = RT ? bL : bR;
                            int b_src = RT ? bR : bL;
                            int idx = b_obs * 27 + dob * 9 + b_src * 3 + ds;
                            result_temp[idx] += val;
                        }
                    }
                }
        } else {
            // elasticRH3_tensor (kernels.cl:70-98).
            const R invr2 = 1.0 / r2;
            const R invr = std::sqrt(invr2);
            for (int dob = 0; dob < 3; dob++)
                for (int ds = 0; ds < 3; ds++)
                    for (int It = 0; It < 3; It++)
                        for (int Im = 0; Im < 3; Im++) {
                            R Kval = quadw * c.CsRH0 * invr *
                                     (-2 * D[dob] * D[ds] * invr2 * kron(It, Im) +
                                      c.CsRH1 * (kron(dob, It) * kron(ds, Im)) +
                                      c.CsRH2 * (kron(dob, Im) * kron(ds, It)) -
                                      2 * (kron(dob, ds) * kron(It, Im)));
                            for (int bs = 0; bs < 3; bs++)
                                for (int bo = 0; bo < 3; bo++) {
                                    int idx = bo * 27 + dob * 9 + bs * 3 + ds;
                                    result_temp[idx] += Kval * o.surf_curl[bo][It] * s.surf_curl[bs][Im];
                                }
                        }
        }
    }
}

template <typename R>
std::vector<R> cast(const double* p, size_t n) {
    std::vector<R> out(n);
    for (size_t i = 0; i < n; i++) out[i] = static_cast<R>(p[i]);
    return out;
}

inline int max_index(const int* tris, long n) {
    int m = -1;
    for (long i = 0; i < n; i++) m = tris[i] > m ? tris[i] : m;
    return m;
}

template <typename R>
int pairs_impl(int kernel, int adj, int check0, double* result, int n_q,
               const double* qp_d, const double* qw_d, const double* pts_d,
               const int* tris, const int* pairs, int n_pairs,
               const double* params_d, int n_threads) {
    if (n_pairs <= 0) return 0;
    int rec = adj ? 5 : 2;
    int max_tri = 0;
    for (int i = 0; i < n_pairs; i++) {
        max_tri = std::max(max_tri, std::max(pairs[i * rec], pairs[i * rec + 1]));
    }
    int n_pts = max_index(tris, 3L * (max_tri + 1)) + 1;
    auto qp = cast<R>(qp_d, 4 * (size_t)n_q);
    auto qw = cast<R>(qw_d, n_q);
    auto pts = cast<R>(pts_d, 3 * (size_t)n_pts);
    R params[2] = {R(params_d[0]), R(params_d[1])};
    Consts<R> c(params);
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 16)
    for (int i = 0; i < n_pairs; i++) {
        int oi = pairs[i * rec], si = pairs[i * rec + 1];
        int oc = adj ? pairs[i * rec + 2] : 0;
        int sc = adj ? pairs[i * rec + 3] : 0;
        bool flip = adj ? pairs[i * rec + 4] != 0 : false;
        TriInfo<R> o, s;
        tri_info(o, pts.data(), tris, oi, oc, false);
        tri_info(s, pts.data(), tris, si, sc, flip);
        R rt[81];
        integrate_pair<R>(kernel, c, o, s, n_q, qp.data(), qw.data(),
                          adj ? true : check0 != 0, rt);
        if (!adj) {
            for (int k = 0; k < 81; k++) result[(size_t)i * 81 + k] = o.jacobian * s.jacobian * rt[k];
        } else {
            // de-rotation of the outputs (assemble.cl:77-101)
            int od[3], sd[3];
            for (int k = 0; k < 3; k++) {
                od[k] = positive_mod(-oc + k, 3);
                sd[k] = positive_mod(-sc + k, 3);
            }
            if (flip) std::swap(sd[0], sd[1]);
            for (int b1 = 0; b1 < 3; b1++)
                for (int d1 = 0; d1 < 3; d1++)
                    for (int b2 = 0; b2 < 3; b2++)
                        for (int d2 = 0; d2 < 3; d2++) {
                            int out_idx = b1 * 27 + d1 * 9 + b2 * 3 + d2;
                            int in_idx = od[b1] * 27 + d1 * 9 + sd[b2] * 3 + d2;
                            R val = o.jacobian * s.jacobian * rt[in_idx];
                            result[(size_t)i * 81 + out_idx] = val;
                        }
        }
    }
    return 0;
}

// Vector (matvec) forms: kernels/__init__.py:28-36,67-99,147-173 and
// kernels/kernels.cl:100-206.  `in9` = raw 9 source dofs, `inv` = the input
// interpolated at the source point; sum3 = the per-point 3-vector, sum9 = the
// per-basis accumulator written directly by RA/RH (matrix_free.cl:237-292).
template <typename R>
void vector_code(int kernel, const Consts<R>& c, const R* D, R r2, const R* nobs,
                 const R* nsrc, const R* inv, const R* in9, const R (*obs_sc)[3],
                 const R (*src_sc)[3], R factor, R* sum3, R* sum9) {
    R Dx = D[0], Dy = D[1], Dz = D[2];
    R inx = inv[0], iny = inv[1], inz = inv[2];
    if (kernel == 0) {
        R invr = rsqrt_(r2);
        R Q1 = c.CsU0 * invr;
        R Q2 = c.CsU1 * invr / r2;
        R ddi = Dx * inx + Dy * iny + Dz * inz;
        sum3[0] += Q1 * inx + Q2 * Dx * ddi;
        sum3[1] += Q1 * iny + Q2 * Dy * ddi;
        sum3[2] += Q1 * inz + Q2 * Dz * ddi;
    } else if (kernel == 1 || kernel == 2) {
        const bool T = kernel == 1;
        const R mp = T ? R(-1) : R(1);
        const R pm = T ? R(1) : R(-1);
        const R* n = T ? nsrc : nobs;
        R invr = rsqrt_(r2);
        R invr2 = invr * invr;
        R invr3 = invr2 * invr;
        R rn = n[0] * Dx + n[1] * Dy + n[2] * Dz;
        R A = pm * c.CsT0 * invr3;
        R C = mp * c.CsT1 * invr3 * invr2;
        R rnddi = C * rn * (Dx * inx + Dy * iny + Dz * inz);
        R nxdy = n[0] * Dy - n[1] * Dx;
        R nzdx = n[2] * Dx - n[0] * Dz;
        R nzdy = n[2] * Dy - n[1] * Dz;
        sum3[0] += A * (-rn * inx + mp * nxdy * iny + pm * nzdx * inz) + Dx * rnddi;
        sum3[1] += A * (pm * nxdy * inx - rn * iny + pm * nzdy * inz) + Dy * rnddi;
        sum3[2] += A * (mp * nzdx * inx + mp * nzdy * iny - rn * inz) + Dz * rnddi;
    } else if (kernel == 3) {
        R invr = rsqrt_(r2);
        R invr2 = invr * invr;
        R invr3 = invr2 * invr;
        R rn = invr * (nsrc[0] * Dx + nsrc[1] * Dy + nsrc[2] * Dz);
        R rm = invr * (nobs[0] * Dx + nobs[1] * Dy + nobs[2] * Dz);
        R mn = nobs[0] * nsrc[0] + nobs[1] * nsrc[1] + nobs[2] * nsrc[2];
        R sn = inx * nsrc[0] + iny * nsrc[1] + inz * nsrc[2];
        R sd = invr * (inx * Dx + iny * Dy + inz * Dz);
        R sm = inx * nobs[0] + iny * nobs[1] + inz * nobs[2];
        R Q = c.CsH0 * invr3;
        R A = Q * 3 * rn;
        R B = Q * c.CsH1;
        R C = Q * c.CsH3;
        R MT = Q * c.CsH2 * sn + A * c.CsH1 * sd;
        R NT = B * sm + C * sd * rm;
        R DT = invr * (B * 3 * sn * rm + C * sd * mn + A * (c.nu * sm - 5 * sd * rm));
        R ST = A * c.nu * rm + B * mn;
        for (int d = 0; d < 3; d++)
            sum3[d] += nsrc[d] * NT + nobs[d] * MT + D[d] * DT + ST * inv[d];
    } else if (kernel == 4) {
        R ssc[3][3];
        for (int Ij = 0; Ij < 3; Ij++)
            for (int d = 0; d < 3; d++) {
                ssc[d][Ij] = 0.0;
                for (int b = 0; b < 3; b++) ssc[d][Ij] += src_sc[b][Ij] * in9[b * 3 + d];
            }
        R invr = rsqrt_(r2);
        R invr3 = invr * invr * invr;
        R Q1 = c.CsRT1 * invr, Q2 = c.CsRT0 * invr3, Q3 = c.CsRT2 * invr3;
        R Q3nD = Q3 * (nsrc[0] * Dx + nsrc[1] * Dy + nsrc[2] * Dz);
        for (int dob = 0; dob < 3; dob++)
            for (int ds = 0; ds < 3; ds++)
                for (int Ij = 0; Ij < 3; Ij++) {
                    R g = gimk<R>(dob, Ij, ds, Q1, Q2, D);
                    sum3[dob] += g * ssc[ds][Ij];
                }
        for (int d = 0; d < 3; d++) sum3[d] += Q3nD * inv[d];
    } else if (kernel == 5) {
        R invr = rsqrt_(r2);
        R invr3 = invr * invr * invr;
        R Q1 = c.CsRT1 * invr, Q2 = c.CsRT0 * invr3, Q3 = c.CsRT2 * invr3;
        R Q3nD = Q3 * (nobs[0] * Dx + nobs[1] * Dy + nobs[2] * Dz);
        for (int dob = 0; dob < 3; dob++)
            for (int ds = 0; ds < 3; ds++)
                for (int Ij = 0; Ij < 3; Ij++) {
                    R g = gimk<R>(ds, Ij, dob, Q1, Q2, D);
                    R Kval = factor * g * inv[ds];
                    for (int bo = 0; bo < 3; bo++) sum9[bo * 3 + dob] += Kval * obs_sc[bo][Ij];
                }
        for (int d = 0; d < 3; d++) sum3[d] -= Q3nD * inv[d];
    } else {
        const R invr2 = 1.0 / r2;
        const R invr = std::sqrt(invr2);
        R F = factor * c.CsRH0 * invr;
        R ssc[3][3];
        for (int Ij = 0; Ij < 3; Ij++)
            for (int d = 0; d < 3; d++) {
                ssc[d][Ij] = 0.0;
                for (int b = 0; b < 3; b++) ssc[d][Ij] += src_sc[b][Ij] * in9[b * 3 + d];
            }
        R B = 0.0;
        for (int d = 0; d < 3; d++) B += ssc[d][d];
        B *= c.CsRH1;
        for (int bo = 0; bo < 3; bo++) {
            R A = 0.0;
            for (int ds = 0; ds < 3; ds++)
                A += D[ds] * (ssc[ds][0] * obs_sc[bo][0] + ssc[ds][1] * obs_sc[bo][1] +
                              ssc[ds][2] * obs_sc[bo][2]);
            for (int dob = 0; dob < 3; dob++) {
                R C = ssc[0][dob] * obs_sc[bo][0] + ssc[1][dob] * obs_sc[bo][1] +
                      ssc[2][dob] * obs_sc[bo][2];
                R Dd = ssc[dob][0] * obs_sc[bo][0] + ssc[dob][1] * obs_sc[bo][1] +
                       ssc[dob][2] * obs_sc[bo][2];
                sum9[bo * 3 + dob] += F * (-2 * D[dob] * invr2 * A + obs_sc[bo][dob] * B +
                                           c.CsRH2 * C - 2 * Dd);
            }
        }
    }
}

template <typename R>
int farfield_tris_impl(int kernel, double* out, const double* in_d,
                       const double* pts_d, const int* obs_tris, int n_obs,
                       const int* src_tris, int n_src, int n_q,
                       const double* qp_d, const double* qw_d,
                       const double* params_d, int n_threads) {
    int n_pts = std::max(max_index(obs_tris, 3L * n_obs), max_index(src_tris, 3L * n_src)) + 1;
    auto pts = cast<R>(pts_d, 3 * (size_t)n_pts);
    auto input = cast<R>(in_d, 9 * (size_t)n_src);
    auto qp = cast<R>(qp_d, 2 * (size_t)n_q);
    auto qw = cast<R>(qw_d, n_q);
    R params[2] = {R(params_d[0]), R(params_d[1])};
    Consts<R> c(params);
    std::vector<TriInfo<R>> src(n_src);
    for (int j = 0; j < n_src; j++) tri_info(src[j], pts.data(), src_tris, j, 0, false);
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 4)
    for (int i = 0; i < n_obs; i++) {
        TriInfo<R> o;
        tri_info(o, pts.data(), obs_tris, i, 0, false);
        R sum[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < n_src; j++) {
            const TriInfo<R>& s = src[j];
            const R* in9 = &input[(size_t)j * 9];
            for (int iq1 = 0; iq1 < n_q; iq1++) {
                R obsxhat = qp[iq1 * 2], obsyhat = qp[iq1 * 2 + 1];
                for (int iq2 = 0; iq2 < n_q; iq2++) {
                    R srcxhat = qp[iq2 * 2], srcyhat = qp[iq2 * 2 + 1];
                    R quadw = qw[iq1] * qw[iq2];
                    R obsb[3] = {1 - obsxhat - obsyhat, obsxhat, obsyhat};
                    R srcb[3] = {1 - srcxhat - srcyhat, srcxhat, srcyhat};
                    R x[3], y[3];
                    for (int d = 0; d < 3; d++) {
                        x[d] = 0;
                        y[d] = 0;
                        for (int b = 0; b < 3; b++) x[d] += obsb[b] * o.tri[b][d];
                        for (int b = 0; b < 3; b++) y[d] += srcb[b] * s.tri[b][d];
                    }
                    R D[3] = {y[0] - x[0], y[1] - x[1], y[2] - x[2]};
                    R r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
                    if (r2 == 0.0) continue;
                    R factor = o.jacobian * s.jacobian * quadw;
                    R sum3[3] = {0, 0, 0};
                    R inv[3] = {0, 0, 0};
                    for (int d = 0; d < 3; d++)
                        for (int b = 0; b < 3; b++) inv[d] += in9[b * 3 + d] * srcb[b];
                    vector_code<R>(kernel, c, D, r2, o.n, s.n, inv, in9, o.surf_curl,
                                   s.surf_curl, factor, sum3, sum);
                    for (int bo = 0; bo < 3; bo++)
                        for (int d = 0; d < 3; d++) sum[bo * 3 + d] += factor * obsb[bo] * sum3[d];
                }
            }
        }
        for (int k = 0; k < 9; k++) out[(size_t)i * 9 + k] = sum[k];
    }
    return 0;
}

template <typename R>
int farfield_pts_impl(int kernel, double* out, const double* obs_pts_d,
                      const double* obs_ns_d, int n_obs, const double* src_pts_d,
                      const double* src_ns_d, int n_src, const double* in_d,
                      const double* params_d, int n_threads) {
    auto op = cast<R>(obs_pts_d, 3 * (size_t)n_obs);
    auto on = cast<R>(obs_ns_d, 3 * (size_t)n_obs);
    auto sp = cast<R>(src_pts_d, 3 * (size_t)n_src);
    auto sn = cast<R>(src_ns_d, 3 * (size_t)n_src);
    auto input = cast<R>(in_d, 3 * (size_t)n_src);
    R params[2] = {R(params_d[0]), R(params_d[1])};
    Consts<R> c(params);
#pragma omp parallel for num_threads(n_threads) schedule(static)
    for (int i = 0; i < n_obs; i++) {
        R sum3[3] = {0, 0, 0};
        for (int j = 0; j < n_src; j++) {
            R D[3];
            for (int d = 0; d < 3; d++) D[d] = sp[j * 3 + d] - op[i * 3 + d];
            R r2 = D[0] * D[0];
            r2 += D[1] * D[1];
            r2 += D[2] * D[2];
            if (r2 == 0.0) continue;
            vector_code<R>(kernel, c, D, r2, &on[i * 3], &sn[j * 3], &input[j * 3],
                           nullptr, nullptr, nullptr, R(1), sum3, nullptr);
        }
        for (int d = 0; d < 3; d++) out[(size_t)i * 3 + d] = sum3[d];
    }
    return 0;
}

template <typename R>
int farfield_dense_impl(int kernel, double* out, int n_q, const double* qp_d,
                        const double* qw_d, const double* pts_d,
                        const int* obs_tris, int n_obs, const int* src_tris,
                        int n_src, const double* params_d, int n_threads) {
    int n_pts = std::max(max_index(obs_tris, 3L * n_obs), max_index(src_tris, 3L * n_src)) + 1;
    auto pts = cast<R>(pts_d, 3 * (size_t)n_pts);
    auto qp = cast<R>(qp_d, 4 * (size_t)n_q);
    auto qw = cast<R>(qw_d, n_q);
    R params[2] = {R(params_d[0]), R(params_d[1])};
    Consts<R> c(params);
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 1)
    for (int i = 0; i < n_obs; i++) {
        TriInfo<R> o;
        tri_info(o, pts.data(), obs_tris, i, 0, false);
        for (int j = 0; j < n_src; j++) {
            TriInfo<R> s;
            tri_info(s, pts.data(), src_tris, j, 0, false);
            R rt[81];
            integrate_pair<R>(kernel, c, o, s, n_q, qp.data(), qw.data(), false, rt);
            for (int bo = 0; bo < 3; bo++)
                for (int dob = 0; dob < 3; dob++)
                    for (int bs = 0; bs < 3; bs++)
                        for (int ds = 0; ds < 3; ds++) {
                            size_t idx = ((size_t)i * 9 + bo * 3 + dob) * (size_t)n_src * 9 +
                                         ((size_t)j * 9 + bs * 3 + ds);
                            out[idx] = o.jacobian * s.jacobian * rt[bo * 27 + dob * 9 + bs * 3 + ds];
                        }
        }
    }
    return 0;
}

template <typename R>
int bsr_impl(long mb, int bs, const long* indptr, const long* indices,
             const double* data, const double* x, double* y) {
    for (long r = 0; r < mb; r++) {
        R sum[16] = {0};
        for (long p = indptr[r]; p < indptr[r + 1]; p++) {
            long col = indices[p];
            const double* A = data + (size_t)bs * bs * p;
            for (int i = 0; i < bs; i++) {
                R acc = 0;
                for (int j = 0; j < bs; j++) acc = acc + R(A[i * bs + j]) * R(x[bs * col + j]);
                sum[i] += acc;
            }
        }
        for (int i = 0; i < bs; i++) y[bs * r + i] = sum[i];
    }
    return 0;
}

// bcoomv: one block per iteration, atomic scatter into y
// (util/fast_sparse.cpp:128-163); serial when n_threads == 1.
template <typename R>
int bcoo_impl(long nb, int bs, const long* rows, const long* cols,
              const double* data, const double* x, double* y, int n_threads) {
    std::vector<R> yr(std::max(0L, 0L));
    long n_rows = 0;
    for (long b = 0; b < nb; b++) n_rows = std::max(n_rows, rows[b] + 1);
    yr.assign((size_t)n_rows * bs, R(0));
    std::vector<R> xr;
    long n_cols = 0;
    for (long b = 0; b < nb; b++) n_cols = std::max(n_cols, cols[b] + 1);
    xr.resize((size_t)n_cols * bs);
    for (long k = 0; k < n_cols * bs; k++) xr[k] = R(x[k]);
    std::vector<R> Ar((size_t)nb * bs * bs);
    for (size_t k = 0; k < Ar.size(); k++) Ar[k] = R(data[k]);
    for (long k = 0; k < n_rows * bs; k++) yr[k] = R(y[k]);
#pragma omp parallel for num_threads(n_threads) schedule(static)
    for (long b = 0; b < nb; b++) {
        const R* A = Ar.data() + (size_t)bs * bs * b;
        const R* xs = xr.data() + (size_t)bs * cols[b];
        R* ys = yr.data() + (size_t)bs * rows[b];
        for (int i = 0; i < bs; i++) {
            R acc = 0;
            for (int j = 0; j < bs; j++) acc = acc + A[i * bs + j] * xs[j];
#pragma omp atomic
            ys[i] += acc;
        }
    }
    for (long k = 0; k < n_rows * bs; k++) y[k] = yr[k];
    return 0;
}

}  // namespace

// ---- interior evaluation (interior.py, assemble.cl:140-186,
// matrix_free.cl:109-194, interior_corners.cl) --------------------------------

// Point-triangle integrals (interior_pairs + integrate_pt_tri,
// integral_primitives.cl:216-258): per pair (obs point, src tri, clicks) the
// 27 entries [d_obs][b_src][d_src] = J_s sum_q w_q phi_b(q) K(x, y_q)
// (Kahan-summed, no r2 == 0 skip), de-rotated by the clicks.
template <typename R>
int interior_pairs_impl(int kernel, double* result, int n_q, const double* qp_d,
                        const double* qw_d, const double* obs_pts_d, const double* obs_ns_d,
                        int n_obs, const double* pts_d, int n_pts, const int* tris,
                        const int* pairs, long n_pairs, const double* params_d,
                        int finite_part, int n_threads) {
    auto op = cast<R>(obs_pts_d, 3 * (size_t)n_obs);
    auto on = cast<R>(obs_ns_d, 3 * (size_t)n_obs);
    auto pts = cast<R>(pts_d, 3 * (size_t)n_pts);
    auto qp = cast<R>(qp_d, 2 * (size_t)n_q);
    auto qw = cast<R>(qw_d, n_q);
    R params[2] = {R(params_d[0]), R(params_d[1])};
    Consts<R> c(params);
#pragma omp parallel for num_threads(n_threads) schedule(static)
    for (long i = 0; i < n_pairs; i++) {
        const int obs = pairs[3 * i], src = pairs[3 * i + 1], clicks = pairs[3 * i + 2];
        TriInfo<R> s;
        tri_info(s, pts.data(), tris, src, clicks, false);
        const R* x = &op[(size_t)obs * 3];
        const R* nobs = &on[(size_t)obs * 3];
        R rt[27], kc[27];
        for (int k = 0; k < 27; k++) rt[k] = kc[k] = 0;
        for (int iq = 0; iq < n_q; iq++) {
            R sx = qp[iq * 2], sy = qp[iq * 2 + 1], quadw = qw[iq];
            R srcb[3] = {1 - sx - sy, sx, sy};
            R y[3];
            for (int d = 0; d < 3; d++) {
                y[d] = 0;
                for (int b = 0; b < 3; b++) y[d] += srcb[b] * s.tri[b][d];
            }
            R D[3] = {y[0] - x[0], y[1] - x[1], y[2] - x[2]};
            R r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
            R Karr[9];
            tensor_UTAH(kernel, c, D[0], D[1], D[2], r2, nobs, s.n, Karr);
            R obsb0 = R(1) * quadw;
            int idx = 0;
            for (int dob = 0; dob < 3; dob++)
                for (int bs = 0; bs < 3; bs++)
                    for (int ds = 0; ds < 3; ds++, idx++) {
                        R val = obsb0 * srcb[bs] * Karr[dob * 3 + ds];
                        R yk = val - kc[idx];
                        R t = rt[idx] + yk;
                        kc[idx] = (t - rt[idx]) - yk;
                        rt[idx] = t;
                    }
        }
        int derot[3];
        for (int b = 0; b < 3; b++) derot[b] = positive_mod(-clicks + b, 3);
        double* out = result + i * 27;
        for (int d1 = 0; d1 < 3; d1++)
            for (int b2 = 0; b2 < 3; b2++) {
                if (finite_part && b2 != clicks) continue;
                for (int d2 = 0; d2 < 3; d2++)
                    out[d1 * 9 + b2 * 3 + d2] = s.jacobian * rt[d1 * 9 + derot[b2] * 3 + d2];
            }
    }
    return 0;
}

// Observation point at a vertex of the source triangle (interior_corners.cl,
// elasticH3): the radial integral from the vertex done in closed form, a
// Gauss rule over the angle t in [0, pi/2].  In the reference kernel the
// log-term tensor I4 is scaled by the integer quotient 1/3, which is 0, so
// only the 1/r^3 tensor I3 and the scalar terms I1, I2 contribute; that is
// restated as is.
template <typename R>
int interior_corners_impl(double* result, int n_q, const double* qp_d, const double* qw_d,
                          const double* obs_ns_d, int n_obs, const double* pts_d, int n_pts,
                          const int* tris, const int* pairs, long n_pairs,
                          const double* params_d, int n_threads) {
    auto on = cast<R>(obs_ns_d, 3 * (size_t)n_obs);
    auto pts = cast<R>(pts_d, 3 * (size_t)n_pts);
    auto qp = cast<R>(qp_d, n_q);
    auto qw = cast<R>(qw_d, n_q);
    R params[2] = {R(params_d[0]), R(params_d[1])};
    Consts<R> c(params);
#pragma omp parallel for num_threads(n_threads) schedule(static)
    for (long i = 0; i < n_pairs; i++) {
        const int obs = pairs[3 * i], src = pairs[3 * i + 1], clicks = pairs[3 * i + 2];
        TriInfo<R> s;
        tri_info(s, pts.data(), tris, src, clicks, false);
        const R* nobs = &on[(size_t)obs * 3];
        R rt[27], kc[27];
        for (int k = 0; k < 27; k++) rt[k] = kc[k] = 0;
        R v1[3], v2[3];
        for (int d = 0; d < 3; d++) {
            v1[d] = s.tri[1][d] - s.tri[0][d];
            v2[d] = s.tri[2][d] - s.tri[0][d];
        }
        const R mn = nobs[0] * s.n[0] + nobs[1] * s.n[1] + nobs[2] * s.n[2];
        for (int iq = 0; iq < n_q; iq++) {
            const R t = qp[iq], quadw = qw[iq];
            const R ct = std::cos(t), st = std::sin(t);
            const R rhomax = R(1.0) / (ct + st);
            R a[3];
            for (int d = 0; d < 3; d++) a[d] = v1[d] * ct + v2[d] * st;
            const R A2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
            const R A = std::sqrt(A2);
            const R A3 = A2 * A;
            const R A5 = (A3 * A) * A;
            const R I1 = R(-1) / (A3 * rhomax);
            const R I2 = (std::log(R(2.0)) + std::log(A) + std::log(rhomax) - 1) / A3;
            const R T0[3] = {-I2 * ct - I2 * st + I1, I2 * ct, I2 * st};
            for (int b = 0; b < 3; b++)
                for (int dob = 0; dob < 3; dob++)
                    for (int ds = 0; ds < 3; ds++) {
                        // I3 enters through basis 0 only (the I4 terms vanish)
                        const R I3 = (-a[dob]) * a[ds] / (A5 * rhomax);
                        const R T1 = b == 0 ? I3 : R(0);
                        R Kval = 0.0;
                        Kval += c.CsH0 * c.CsH3 * T1 * mn;
                        if (dob == ds) Kval += c.CsH0 * c.CsH1 * mn * T0[b];
                        const int idx = dob * 9 + b * 3 + ds;
                        const R val = quadw * Kval;
                        const R yk = val - kc[idx];
                        const R tt = rt[idx] + yk;
                        kc[idx] = (tt - rt[idx]) - yk;
                        rt[idx] = tt;
                    }
        }
        int derot[3];
        for (int b = 0; b < 3; b++) derot[b] = positive_mod(-clicks + b, 3);
        double* out = result + i * 27;
        for (int d1 = 0; d1 < 3; d1++)
            for (int b2 = 0; b2 < 3; b2++)
                for (int d2 = 0; d2 < 3; d2++)
                    out[d1 * 9 + b2 * 3 + d2] = s.jacobian * rt[d1 * 9 + derot[b2] * 3 + d2];
    }
    return 0;
}

// Triangle sources to observation points (matrix_free.cl:109-194
// farfield_tris_to_pts{K}): per point the sum over all source triangles
// and quadrature points of J_s w_q K(x, y_q) . (sum_b in_b phi_b), r2 == 0
// skipped.
template <typename R>
int farfield_tris_to_pts_impl(int kernel, double* out, const double* in_d,
                              const double* obs_pts_d, const double* obs_ns_d, int n_obs,
                              const double* pts_d, int n_pts, const int* src_tris, int n_src,
                              int n_q, const double* qp_d, const double* qw_d,
                              const double* params_d, int n_threads) {
    auto op = cast<R>(obs_pts_d, 3 * (size_t)n_obs);
    auto on = cast<R>(obs_ns_d, 3 * (size_t)n_obs);
    auto pts = cast<R>(pts_d, 3 * (size_t)n_pts);
    auto input = cast<R>(in_d, 9 * (size_t)n_src);
    auto qp = cast<R>(qp_d, 2 * (size_t)n_q);
    auto qw = cast<R>(qw_d, n_q);
    R params[2] = {R(params_d[0]), R(params_d[1])};
    Consts<R> c(params);
    std::vector<TriInfo<R>> src(n_src);
    for (int j = 0; j < n_src; j++) tri_info(src[j], pts.data(), src_tris, j, 0, false);
#pragma omp parallel for num_threads(n_threads) schedule(static)
    for (int i = 0; i < n_obs; i++) {
        const R* x = &op[(size_t)i * 3];
        R sum[3] = {0, 0, 0};
        for (int j = 0; j < n_src; j++) {
            const TriInfo<R>& s = src[j];
            const R* in9 = &input[(size_t)j * 9];
            for (int iq = 0; iq < n_q; iq++) {
                R sx = qp[iq * 2], sy = qp[iq * 2 + 1], quadw = qw[iq];
                R srcb[3] = {1 - sx - sy, sx, sy};
                R y[3];
                for (int d = 0; d < 3; d++) {
                    y[d] = 0;
                    for (int b = 0; b < 3; b++) y[d] += srcb[b] * s.tri[b][d];
                }
                R D[3] = {y[0] - x[0], y[1] - x[1], y[2] - x[2]};
                R r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
                if (r2 == 0.0) continue;
                R factor = s.jacobian * quadw;
                R inv[3] = {0, 0, 0};
                for (int d = 0; d < 3; d++)
                    for (int b = 0; b < 3; b++) inv[d] += in9[b * 3 + d] * srcb[b];
                R sum3[3] = {0, 0, 0};
                vector_code<R>(kernel, c, D, r2, &on[(size_t)i * 3], s.n, inv, in9, nullptr,
                               nullptr, R(1), sum3, nullptr);
                for (int d = 0; d < 3; d++) sum[d] += factor * sum3[d];
            }
        }
        for (int d = 0; d < 3; d++) out[(size_t)i * 3 + d] = sum[d];
    }
    return 0;
}

extern "C" {

int orc_pairs(int kernel, int prec, int adj, int check0, double* result,
              int n_quad, const double* quad_pts, const double* quad_wts,
              const double* pts, const int* tris, const int* pairs, int n_pairs,
              const double* params, int n_threads) {
    if (kernel < 0 || kernel > 6) return 2;
    if (prec == 0)
        return pairs_impl<float>(kernel, adj, check0, result, n_quad, quad_pts, quad_wts,
                                 pts, tris, pairs, n_pairs, params, n_threads);
    return pairs_impl<double>(kernel, adj, check0, result, n_quad, quad_pts, quad_wts,
                              pts, tris, pairs, n_pairs, params, n_threads);
}

int orc_farfield_tris(int kernel, int prec, double* out, const double* in,
                      const double* pts, const int* obs_tris, int n_obs,
                      const int* src_tris, int n_src, int n_q,
                      const double* quad_pts, const double* quad_wts,
                      const double* params, int n_threads) {
    if (kernel < 0 || kernel > 6) return 2;
    if (prec == 0)
        return farfield_tris_impl<float>(kernel, out, in, pts, obs_tris, n_obs, src_tris, n_src,
                                         n_q, quad_pts, quad_wts, params, n_threads);
    return farfield_tris_impl<double>(kernel, out, in, pts, obs_tris, n_obs, src_tris, n_src,
                                      n_q, quad_pts, quad_wts, params, n_threads);
}

int orc_farfield_pts(int kernel, int prec, double* out, const double* obs_pts,
                     const double* obs_ns, int n_obs, const double* src_pts,
                     const double* src_ns, int n_src, const double* in,
                     const double* params, int n_threads) {
    if (kernel < 0 || kernel > 3) return 2;
    if (prec == 0)
        return farfield_pts_impl<float>(kernel, out, obs_pts, obs_ns, n_obs, src_pts, src_ns,
                                        n_src, in, params, n_threads);
    return farfield_pts_impl<double>(kernel, out, obs_pts, obs_ns, n_obs, src_pts, src_ns,
                                     n_src, in, params, n_threads);
}

int orc_farfield_tris_dense(int kernel, int prec, double* out, int n_quad,
                            const double* quad_pts, const double* quad_wts,
                            const double* pts, const int* obs_tris, int n_obs,
                            const int* src_tris, int n_src, const double* params,
                            int n_threads) {
    if (kernel < 0 || kernel > 6) return 2;
    if (prec == 0)
        return farfield_dense_impl<float>(kernel, out, n_quad, quad_pts, quad_wts, pts, obs_tris,
                                          n_obs, src_tris, n_src, params, n_threads);
    return farfield_dense_impl<double>(kernel, out, n_quad, quad_pts, quad_wts, pts, obs_tris,
                                       n_obs, src_tris, n_src, params, n_threads);
}

int orc_interior_pairs(int kernel, int prec, double* result, int n_q, const double* qp,
                       const double* qw, const double* obs_pts, const double* obs_ns, int n_obs,
                       const double* pts, int n_pts, const int* tris, const int* pairs,
                       long n_pairs, const double* params, int finite_part, int n_threads) {
    if (kernel < 0 || kernel > 3) return 2;
    if (prec == 0)
        return interior_pairs_impl<float>(kernel, result, n_q, qp, qw, obs_pts, obs_ns, n_obs,
                                          pts, n_pts, tris, pairs, n_pairs, params, finite_part,
                                          n_threads);
    return interior_pairs_impl<double>(kernel, result, n_q, qp, qw, obs_pts, obs_ns, n_obs, pts,
                                       n_pts, tris, pairs, n_pairs, params, finite_part,
                                       n_threads);
}

int orc_interior_corners(int prec, double* result, int n_q, const double* qp,
                         const double* qw, const double* obs_ns, int n_obs, const double* pts,
                         int n_pts, const int* tris, const int* pairs, long n_pairs,
                         const double* params, int n_threads) {
    if (prec == 0)
        return interior_corners_impl<float>(result, n_q, qp, qw, obs_ns, n_obs, pts, n_pts, tris,
                                            pairs, n_pairs, params, n_threads);
    return interior_corners_impl<double>(result, n_q, qp, qw, obs_ns, n_obs, pts, n_pts, tris,
                                         pairs, n_pairs, params, n_threads);
}

int orc_farfield_tris_to_pts(int kernel, int prec, double* out, const double* in,
                             const double* obs_pts, const double* obs_ns, int n_obs,
                             const double* pts, int n_pts, const int* src_tris, int n_src,
                             int n_q, const double* qp, const double* qw,
                             const double* params, int n_threads) {
    if (kernel < 0 || kernel > 3) return 2;
    if (prec == 0)
        return farfield_tris_to_pts_impl<float>(kernel, out, in, obs_pts, obs_ns, n_obs, pts,
                                                n_pts, src_tris, n_src, n_q, qp, qw, params,
                                                n_threads);
    return farfield_tris_to_pts_impl<double>(kernel, out, in, obs_pts, obs_ns, n_obs, pts, n_pts,
                                             src_tris, n_src, n_q, qp, qw, params, n_threads);
}

int orc_make_bsr(long n_row_blocks, long n_blocks, int bs, const long* rows,
                 const long* cols, const double* data, long* indptr,
                 long* indices, double* data_out) {
    const long blocksize = (long)bs * bs;
    for (long i = 0; i <= n_row_blocks; i++) indptr[i] = 0;
    for (long i = 0; i < n_blocks; i++) indptr[rows[i]]++;
    for (long i = 0, cumsum = 0; i < n_row_blocks; i++) {
        long temp = indptr[i];
        indptr[i] = cumsum;
        cumsum += temp;
    }
    indptr[n_row_blocks] = n_blocks;
    for (long n = 0; n < n_blocks; n++) {
        long row = rows[n];
        long dest = indptr[row];
        indices[dest] = cols[n];
        std::memcpy(data_out + dest * blocksize, data + n * blocksize, sizeof(double) * blocksize);
        indptr[row]++;
    }
    for (long i = 0, last = 0; i <= n_row_blocks; i++) {
        long temp = indptr[i];
        indptr[i] = last;
        last = temp;
    }
    return 0;
}

int orc_bsr_matvec(int prec, long n_row_blocks, int bs, const long* indptr,
                   const long* indices, const double* data, const double* x,
                   double* y) {
    if (bs < 1 || bs > 16) return 1;
    if (prec == 0) return bsr_impl<float>(n_row_blocks, bs, indptr, indices, data, x, y);
    return bsr_impl<double>(n_row_blocks, bs, indptr, indices, data, x, y);
}

int orc_bcoo_matvec(int prec, long n_blocks, int bs, const long* rows,
                    const long* cols, const double* data, const double* x,
                    double* y, int n_threads) {
    if (bs < 1 || bs > 16) return 1;
    if (n_threads < 1) n_threads = 1;
    if (prec == 0) return bcoo_impl<float>(n_blocks, bs, rows, cols, data, x, y, n_threads);
    return bcoo_impl<double>(n_blocks, bs, rows, cols, data, x, y, n_threads);
}

}  // extern "C"
