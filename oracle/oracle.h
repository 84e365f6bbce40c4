/* Test infrastructure: CPU restatement of the reference's elastic-BEM kernel math.
 *
 * This library is the checker for the CUDA product and the timed CPU baseline
 * of bench.py.  It is never linked into, called by or shipped with the
 * product.  Every routine follows the reference file and lines cited beside
 * it; `prec` selects the arithmetic type (0 = float, as the reference's
 * default float_type = np.float32; 1 = double).  Inputs and outputs are double
 * regardless of `prec` (float mode rounds inputs to float first, exactly as the
 * reference's `gpu.to_gpu(x, float_type)` does).
 *
 * Kernel ids: 0 elasticU3, 1 elasticT3, 2 elasticA3, 3 elasticH3,
 *             4 elasticRT3, 5 elasticRA3, 6 elasticRH3.
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

/* single_pairs{Z,N} (adj = 0, record = 2 ints) and single_pairs{N}_adj
 * (adj = 1, record = 5 ints: obs, src, obs_clicks, src_clicks, src_flip):
 * tectosaur/assemble.cl:24-103, tectosaur/integral_primitives.cl:56-213.
 * result: n_pairs x 81, index b_obs*27 + d_obs*9 + b_src*3 + d_src. */
int orc_pairs(int kernel, int prec, int adj, int check0, double* result,
              int n_quad, const double* quad_pts, const double* quad_wts,
              const double* pts, const int* tris, const int* pairs, int n_pairs,
              const double* params, int n_threads);

/* farfield_tris_to_tris{K}: tectosaur/matrix_free.cl:19-107.
 * quad_pts (n_q x 2), quad_wts (n_q): the 2-D triangle rule of gauss2d_tri. */
int orc_farfield_tris(int kernel, int prec, double* out, const double* in,
                      const double* pts, const int* obs_tris, int n_obs,
                      const int* src_tris, int n_src, int n_q,
                      const double* quad_pts, const double* quad_wts,
                      const double* params, int n_threads);

/* farfield_pts{K}: tectosaur/farfield_direct.cl:15-113 (kernels 0-3 only). */
int orc_farfield_pts(int kernel, int prec, double* out, const double* obs_pts,
                     const double* obs_ns, int n_obs, const double* src_pts,
                     const double* src_ns, int n_src, const double* in,
                     const double* params, int n_threads);

/* Interior evaluation (tectosaur/interior.py).  interior_pairs:
 * assemble.cl:140-186 with integrate_pt_tri (integral_primitives.cl:216-258),
 * kernels 0-3; pairs (obs pt, src tri, clicks) int32; result (n, 3, 3, 3)
 * [d_obs][b_src][d_src]. */
int orc_interior_pairs(int kernel, int prec, double* result, int n_q, const double* qp,
                       const double* qw, const double* obs_pts, const double* obs_ns, int n_obs,
                       const double* pts, int n_pts, const int* tris, const int* pairs,
                       long n_pairs, const double* params, int finite_part, int n_threads);
/* interior_corners.cl (elasticH3, observation point at source vertex
 * `clicks`); qp: n_q angles in [0, pi/2]. */
int orc_interior_corners(int prec, double* result, int n_q, const double* qp,
                         const double* qw, const double* obs_ns, int n_obs, const double* pts,
                         int n_pts, const int* tris, const int* pairs, long n_pairs,
                         const double* params, int n_threads);
/* farfield_tris_to_pts{K}: matrix_free.cl:109-194, kernels 0-3. */
int orc_farfield_tris_to_pts(int kernel, int prec, double* out, const double* in,
                             const double* obs_pts, const double* obs_ns, int n_obs,
                             const double* pts, int n_pts, const int* src_tris, int n_src,
                             int n_q, const double* qp, const double* qw,
                             const double* params, int n_threads);

/* farfield_tris (dense 9x9 blocks): tectosaur/assemble.cl:105-138.
 * out layout (n_obs, 3, 3, n_src, 3, 3). */
int orc_farfield_tris_dense(int kernel, int prec, double* out, int n_quad,
                            const double* quad_pts, const double* quad_wts,
                            const double* pts, const int* obs_tris, int n_obs,
                            const int* src_tris, int n_src, const double* params,
                            int n_threads);

/* make_bsr_matrix: tectosaur/util/fast_sparse.cpp:14-68 (stable counting sort
 * by block row; duplicates kept; column order within a row = input order). */
int orc_make_bsr(long n_row_blocks, long n_blocks, int bs, const long* rows,
                 const long* cols, const double* data, long* indptr,
                 long* indices, double* data_out);

/* bsrmv{bs} and bcoomv{bs}: tectosaur/util/fast_sparse.cpp:71-163.  bsr is
 * serial (deterministic order) and overwrites y; bcoo accumulates into y with
 * an atomic scatter over n_threads OpenMP threads, as the reference does. */
int orc_bsr_matvec(int prec, long n_row_blocks, int bs, const long* indptr,
                   const long* indices, const double* data, const double* x,
                   double* y);
int orc_bcoo_matvec(int prec, long n_blocks, int bs, const long* rows,
                    const long* cols, const double* data, const double* x,
                    double* y, int n_threads);

#ifdef __cplusplus
}
#endif
