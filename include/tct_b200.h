/* tct_b200: C ABI of the B200 elastic-BEM operator-apply path.
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (TCT_OK = 0).  Device pointers are CUDA global-memory addresses on the
 * current device; `stream` is a cudaStream_t passed as void* (NULL = legacy
 * default stream).  Host pointers are marked "host".  The library never frees
 * caller memory and keeps no per-call device allocations: scratch space is
 * passed in by the caller (see the *_workspace_bytes queries).
 *
 * Arithmetic type: `prec` = TCT_F32 (float, the reference's default
 * float_type) or TCT_F64 (double).  Real below means float or double
 * according to `prec`.
 *
 * Kernel ids follow the reference's kernel names (tectosaur/kernels/__init__.py):
 *   0 elasticU3  1 elasticT3  2 elasticA3  3 elasticH3
 *   4 elasticRT3 5 elasticRA3 6 elasticRH3
 * params = {mu (shear modulus G), nu} as host doubles.
 */
#ifndef TCT_B200_H
#define TCT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCT_OK 0
#define TCT_ERR_ARG 1        /* bad size, pointer, alignment or index       */
#define TCT_ERR_KERNEL 2     /* kernel id not supported by this entry point */
#define TCT_ERR_CUDA 3       /* CUDA runtime / launch error                  */
#define TCT_ERR_OOM 4        /* workspace too small / allocation failed      */
#define TCT_ERR_TIMEOUT 5    /* a bounded device wait gave up                */
#define TCT_ERR_PREC 6       /* unsupported precision                        */

#define TCT_F32 0
#define TCT_F64 1

/* Library version string and the last error message of the calling thread. */
const char* tct_version(void);
const char* tct_last_error(void);

/* Kernel id of a reference kernel name ("elasticRH3" -> 6), or -1. */
int tct_kernel_id(const char* name);

/* ------------------------------------------------------------------------ */
/* Triangle-pair quadrature (nearfield assembly).                            */
/* Replaces the reference's single_pairsZ / single_pairsN / single_pairsN_adj
 * kernels (tectosaur/assemble.cl:24-103) and PairsIntegrator.pairs_quad
 * (tectosaur/nearfield/pairs_integrator.py:43-68).
 *
 * pairs:   n_pairs records of int32 (device): 2 ints (obs_tri, src_tri) when
 *          adj == 0, 5 ints (obs_tri, src_tri, obs_clicks, src_clicks,
 *          src_flip) when adj == 1 (assemble.cl:58-62).
 * quad:    n_quad 4-D points (obs xhat, obs yhat, src xhat, src yhat) and
 *          weights, Real, device.
 * pts:     n_pts x 3 Real (device); tris: n_tris x 3 int32 (device).
 * check0:  skip quadrature points with r^2 == 0 (the "Z" variant); adjacent
 *          pairs always skip them (assemble.cl:67).
 * out:     81 Real per pair, index b_obs*27 + d_obs*9 + b_src*3 + d_src.
 *          When out_slot is non-NULL, pair i's 81 values go to block
 *          out_slot[i] of a block array with `slot_stride` blocks between
 *          consecutive entries of one block (structure-of-arrays BSR layout:
 *          element e of block s at out[e * slot_stride + s]); otherwise to
 *          out[i * 81 + e].  `sign` (+1 or -1) multiplies the result and
 *          `accumulate` adds into the destination instead of overwriting
 *          (used to subtract the farfield-rule correction in place,
 *          nearfield/nearfield_op.py:135-141).
 */
int tct_pairs_integrate(int kernel, int prec, int adj, int check0,
                        void* out, const int32_t* out_slot, int64_t slot_stride,
                        int sign, int accumulate,
                        int n_quad, const void* quad_pts, const void* quad_wts,
                        const void* pts, const int32_t* tris,
                        const int32_t* pairs, int64_t n_pairs,
                        const double* params, void* stream);

/* Batched form: pairs of every class and quadrature order in one persistent
 * launch (replaces the per-class, one-rule-per-launch calls of
 * nearfield/pairs_integrator.py:70-93).
 * pairs:      n_pairs x 7 int32 (device): obs, src, obs_clicks, src_clicks,
 *             src_flip, rule index, parameter-set index.
 * rule_off:   n_rules + 1 int64 (device): point ranges of the concatenated
 *             rules in rule_pts (n x 4 Real) / rule_wts (n Real).
 * rule_flags: n_rules int32 (device): bit 0 = adjacent record (rotate, flip,
 *             de-rotate), bit 1 = skip r^2 == 0 points.
 * items:      (n_warp_items + n_thread_items) x 4 int32 (device): pair, first
 *             point, end point (relative to the rule), split flag.  Warp items
 *             (first n_warp_items) are integrated by a warp each and, when the
 *             pair is split over several items (flag 1), atomically added;
 *             thread items are whole pairs, one per thread.
 * params:     n_param_sets (1..8) x {mu, nu} host doubles.
 * out:        n_pairs x 81 Real (device), zeroed first unless accumulate.
 * workspace:  >= 2048 bytes, 256-byte aligned (queue counters and the
 *             kernel constants of each parameter set; the constants are
 *             uploaded with cudaMemcpyAsync from host memory). */
int tct_pairs_integrate_batched(int kernel, int prec, void* out, int64_t n_pairs,
                                const void* pts, const int32_t* tris,
                                const int32_t* pairs, const int64_t* rule_off,
                                const int32_t* rule_flags, const void* rule_pts,
                                const void* rule_wts, const int32_t* items,
                                int64_t n_warp_items, int64_t n_thread_items,
                                const double* params, int n_param_sets,
                                int accumulate, void* workspace,
                                size_t workspace_bytes, void* stream);

/* Slot form of tct_pairs_integrate_batched, used by the nearfield operator
 * build (RegularizedNearfieldIntegralOp, nearfield/nearfield_op.py:76-150:
 * its four pair classes and their far-rule corrections, each class
 * integrated there by its own single_pairs launch): element e of pair p's
 * block goes to out[e * slot_stride + slot[p]] (the BSR's structure-of-arrays
 * blocks), times `sign`, added to the destination when `add`.  Pairs cut
 * into several warp items are added atomically, so their slots must start
 * at zero (or `add`); a plan without split items is deterministic. */
int tct_pairs_integrate_batched_slots(int kernel, int prec, void* out, const int32_t* slot,
                                      int64_t slot_stride, double sign, int add, int64_t n_pairs,
                                      const void* pts, const int32_t* tris,
                                      const int32_t* pairs, const int64_t* rule_off,
                                      const int32_t* rule_flags, const void* rule_pts,
                                      const void* rule_wts, const int32_t* items,
                                      int64_t n_warp_items, int64_t n_thread_items,
                                      const double* params, int n_param_sets, void* workspace,
                                      size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Direct tri-to-tri farfield matvec.                                        */
/* Replaces farfield_tris_to_tris{K} (tectosaur/matrix_free.cl:19-107) behind
 * TriToTriDirectFarfieldOp.dot (tectosaur/ops/sparse_farfield_op.py:16-62):
 *   out[obs, b_obs, d] (+)= sum over all src tris and quadrature point pairs of
 *   J_obs J_src w_i w_j phi_b_obs(x_i) K(x_i, y_j) . (sum_b phi_b(y_j) in[src, b, :]),
 * skipping point pairs with r^2 == 0.
 * quad_pts (n_q x 2) and quad_wts (n_q) are the host 2-D triangle rule
 * (gauss2d_tri(nq_far)): n_q in {3, 4, 7, 13} (nq_far = 1..4).
 * in:  n_src x 9 Real, out: n_obs x 9 Real (device).  accumulate != 0 adds to out.
 * workspace: device scratch of at least tct_farfield_workspace_bytes() bytes,
 * 256-byte aligned. */
size_t tct_farfield_workspace_bytes(int kernel, int prec, int64_t n_obs, int64_t n_src,
                                    int n_q);
int tct_farfield_tris_matvec(int kernel, int prec, void* out, const void* in,
                             const void* pts, const int32_t* obs_tris, int64_t n_obs,
                             const int32_t* src_tris, int64_t n_src,
                             int n_q, const double* quad_pts, const double* quad_wts,
                             const double* params, int accumulate,
                             void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Point-to-point farfield.                                                  */
/* Replaces farfield_pts{K} (tectosaur/farfield_direct.cl:15-113) behind
 * farfield_pts_direct (tectosaur/farfield.py:15-38); kernels 0-3 only.
 * obs/src points and normals n x 3 Real, in n_src x 3, out n_obs x 3 (device). */
int tct_farfield_pts(int kernel, int prec, void* out, const void* obs_pts,
                     const void* obs_ns, int64_t n_obs, const void* src_pts,
                     const void* src_ns, int64_t n_src, const void* in,
                     const double* params, void* stream);

/* ------------------------------------------------------------------------ */
/* Dense farfield blocks.                                                    */
/* Replaces farfield_tris (tectosaur/assemble.cl:105-138) behind
 * FarfieldTriMatrix.assemble (tectosaur/ops/dense_integral_op.py:48-90).
 * out: (n_obs, 3, 3, n_src, 3, 3) Real (device). */
int tct_farfield_tris_dense(int kernel, int prec, void* out, int n_quad,
                            const void* quad_pts, const void* quad_wts,
                            const void* pts, const int32_t* obs_tris, int64_t n_obs,
                            const int32_t* src_tris, int64_t n_src,
                            const double* params, void* stream);

/* ------------------------------------------------------------------------ */
/* 9x9 block-sparse (BSR) nearfield matvec.                                  */
/* Replaces bsrmv9 / bcoomv9 (tectosaur/util/fast_sparse.cpp:71-163) behind
 * BCOOMatrix.dot / BSRMatrix.dot (tectosaur/util/sparse.py:29-64) as summed
 * by RegularizedNearfieldIntegralOp.dot (nearfield/nearfield_op.py:158-159).
 * Layout: indptr (n_row_blocks + 1) and indices (one per slot,
 * indptr[n_row_blocks] slots) int32; data in structure-of-arrays order,
 * element e (= i*9 + j) of the block in slot s at data[e * data_stride + s],
 * data_stride >= indptr[n_row_blocks].
 * y[9*r + i] (+)= sum_{s in row r} sum_j A_s[i][j] x[9*indices[s] + j].
 * A slot whose index is negative is padding and is skipped (its data is
 * not read): rows may start on 128-byte lines of the element planes (32
 * FP32 or 16 FP64 slots), so that no line holds the blocks of two rows and
 * none is fetched from DRAM twice.
 * With data2 != NULL the blocks are data + data2 (no-correction form). */
int tct_bsr9_matvec(int prec, int64_t n_row_blocks, const int32_t* indptr,
                    const int32_t* indices, const void* data, const void* data2,
                    int64_t data_stride, const void* x, void* y, int accumulate,
                    void* stream);

/* Panel form of tct_bsr9_matvec (an addition: the reference applies its
 * BSR matrix to one vector at a time, util/sparse.py:44-64): y_v (+)= A x_v
 * for v < n_vec, x_v = x + v * x_stride, y_v = y + v * y_stride (strides in
 * Reals; y_stride >= 9 * n_row_blocks).  Each block is read from HBM once
 * per apply (vector groups of 8 (FP32) / 4 (FP64) re-read it from L2). */
int tct_bsr9_matvec_panel(int prec, int64_t n_row_blocks, const int32_t* indptr,
                          const int32_t* indices, const void* data, int64_t data_stride,
                          const void* x, int64_t x_stride, void* y, int64_t y_stride,
                          int n_vec, int accumulate, void* stream);

/* Number of kernels this library has launched in the process (a measurement
 * aid with no reference counterpart; host). */
uint64_t tct_launch_count(void);

/* ------------------------------------------------------------------------ */
/* Measurement utility (no reference counterpart): FP32 FMA throughput probe.
 * Launches n_blocks x 256 threads, each running `iters` steps of 8 independent
 * fused multiply-adds (16 * iters flops per thread); out: >= 256 floats of
 * device scratch.  Timed by the caller; the FP32 roofline denominator. */
int tct_fp32_fma_probe(void* out, int64_t n_blocks, int iters, void* stream);
/* Same with packed fma.rn.f32x2 (2 FMAs per instruction, 32 * iters flops per
 * thread). */
int tct_fp32x2_fma_probe(void* out, int64_t n_blocks, int iters, void* stream);
/* FP64 FMA throughput probe: n_blocks x 256 threads x iters x 8 fma.rn.f64. */
int tct_fp64_fma_probe(void* out, int64_t n_blocks, int iters, void* stream);

/* ------------------------------------------------------------------------ */
/* Allocation-free farfield matvec (no counterpart in the reference).        */
/* For callers that cannot allocate device memory when they apply the
 * operator -- inside a stream capture that must not add memory nodes, under
 * an embedding application's own memory pool, or where cudaMalloc's implicit
 * synchronisation is not acceptable.  Same arguments and results as
 * tct_farfield_tris_matvec minus the workspace: the scratch is a fixed
 * TCT_NOALLOC_SCRATCH_BYTES array compiled into the library (held on every
 * GPU that loads the library until the process exits).  Problems whose
 * workspace (tct_farfield_workspace_bytes) exceeds it are rejected with
 * TCT_ERR_ARG and a message; nothing is ever allocated.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) -- make
 * it before any stream capture; the address belongs to the device's primary
 * context, so do not call cudaDeviceReset between calls.  All calls share the
 * one array: calls that overlap on the GPU (different streams or host
 * threads) race. */
#define TCT_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
size_t tct_farfield_noalloc_capacity(void);
int tct_farfield_tris_matvec_noalloc(int kernel, int prec, void* out, const void* in,
                                     const void* pts, const int32_t* obs_tris, int64_t n_obs,
                                     const int32_t* src_tris, int64_t n_src,
                                     int n_q, const double* quad_pts, const double* quad_wts,
                                     const double* params, int accumulate, void* stream);

/* ------------------------------------------------------------------------ */
/* Host-side (CPU) structure builders.                                       */

/* Near-pair search: all (i, j) with |c_i - c_j|^2 <= ((r_i + r_j) * threshold)^2
 * evaluated in the same double arithmetic as the reference
 * (mesh/fast_find_nearfield.cpp:22-74, get_nearfield :255-285).  The result
 * set equals the reference's; its order is canonical (lexicographic by
 * (i, j)) rather than the reference's thread-completion order.
 * Two-phase: tct_find_near_pairs returns an opaque handle holding the pairs;
 * read them with tct_pairs_count / tct_pairs_copy and release with
 * tct_pairs_free.  All pointers host. */
typedef struct tct_pair_list tct_pair_list;
int tct_find_near_pairs(const double* obs_centers, const double* obs_radii, int64_t n_obs,
                        const double* src_centers, const double* src_radii, int64_t n_src,
                        double threshold, int n_threads, tct_pair_list** out);
int64_t tct_pairs_count(const tct_pair_list* list);
int tct_pairs_copy(const tct_pair_list* list, int64_t* dst);
void tct_pairs_free(tct_pair_list* list);

/* Device near-pair search: the same pair set and (obs, src) order as
 * tct_find_near_pairs (mesh/fast_find_nearfield.cpp:22-74, 96-141,
 * get_nearfield :255-285), with the ball tests, row fill and row sort on the
 * GPU.  tct_near_plan_build (host) builds the reference's octrees and runs
 * its dual traversal down to leaf pairs; tct_near_device_count uploads the
 * plan, counts the pairs and synchronises `stream` to return the total;
 * tct_near_device_fill writes the pairs (total x 2 int64, caller-owned
 * device memory) in (obs, src) order.  The plan owns its device buffers;
 * tct_near_plan_free releases them.  At most 2^31 - 1 pairs. */
typedef struct tct_near_plan tct_near_plan;
int tct_near_plan_build(const double* obs_centers, const double* obs_radii, int64_t n_obs,
                        const double* src_centers, const double* src_radii, int64_t n_src,
                        double threshold, int n_threads, tct_near_plan** out);
int64_t tct_near_plan_leaf_pairs(const tct_near_plan* plan);
int tct_near_device_count(tct_near_plan* plan, void* stream, int64_t* total);
int tct_near_device_fill(tct_near_plan* plan, int64_t* pairs, void* stream);
void tct_near_plan_free(tct_near_plan* plan);
/* The same plan built entirely on the GPU (the reference builds its octrees
 * and runs the traversal on the host, fmm/octree.cpp:27-76,
 * mesh/fast_find_nearfield.cpp:96-141): the octrees level by level (equal
 * to tct_tree_build's node for node), the expanded node radii, the dual
 * traversal breadth first to leaf pairs, grouped by obs leaf; inputs are host
 * arrays (copied in); synchronises `stream`.  Use with tct_near_device_count
 * / _fill / tct_near_plan_free as a host-built plan; the pairs are the same
 * in the same order.  Fewer than 2^31 - 1 balls per side. */
int tct_near_plan_build_device(const double* obs_centers, const double* obs_radii, int64_t n_obs,
                               const double* src_centers, const double* src_radii, int64_t n_src,
                               double threshold, void* stream, tct_near_plan** out);

/* Split close pairs by the number of shared vertices
 * (mesh/fast_find_nearfield.cpp:143-182): 0 -> near (2 cols), 1 -> vertex
 * adjacent (4 cols: obs, src, obs corner, src corner), 2 -> edge adjacent
 * (6 cols), 3 -> coincident (dropped).  Output capacities: n_pairs rows each.
 * Order = input order.  Host. */
int tct_split_adjacent_close(const int64_t* pairs, int64_t n_pairs,
                             const int64_t* tris_a, const int64_t* tris_b,
                             int64_t* near_out, int64_t* n_near,
                             int64_t* va_out, int64_t* n_va,
                             int64_t* ea_out, int64_t* n_ea);

/* Edge-adjacent orientation records (obs, src, obs_clicks, src_clicks, flip)
 * from the 6-column edge-adjacent rows (nearfield/nearfield_op.py:44-62). Host. */
int tct_resolve_ea_rotation(const int64_t* tris, const int64_t* ea, int64_t n,
                            int64_t* out);

/* Host update of one GMRES step for several systems at once (Givens QR
 * of each system's Hessenberg matrix; the reference runs scipy's gmres,
 * examples/solve.py:25-61): system s = sys[i] puts its new column
 * cols[i * col_stride + 0 .. j[s] + 1] into column j[s] of H_s
 * (H + s (m+1) m, column-major), applies its rotations cs/sn (m per system),
 * adds rotation j[s], updates g (m + 1 per system) and writes the residual
 * estimate |g_s[j[s] + 1]| to res[i].  Host. */
int tct_gmres_givens(int64_t n_active, const int64_t* sys, const int64_t* j, int64_t m,
                     const double* cols, int64_t col_stride, double* H, double* cs, double* sn,
                     double* g, double* res);

/* BSR index build (util/fast_sparse.cpp:14-68 semantics: stable counting
 * sort by block row, duplicates kept).  slot[i] = position of input block i
 * in the BSR order.  Host. */
int tct_make_bsr_index(int64_t n_row_blocks, int64_t n_blocks, const int64_t* rows,
                       const int64_t* cols, int64_t* indptr, int64_t* indices,
                       int64_t* slot);

/* ---- treecode farfield (fmm/tsfmm.py, fmm/traversal.cpp, fmm/octree.cpp) -- */

typedef struct tct_tree tct_tree;
typedef struct tct_lists tct_lists;

/* Ball octree over n balls (centers n x 3, radii n), at most leaf_size balls
 * per leaf; replaces Octree<3>::build (fmm/octree.cpp:28-79, bound through
 * fmm/traversal_wrapper.cpp:31-40).  Node order, orig_idxs, bounds and
 * children match the reference exactly.  Host. */
int tct_tree_build(const double* centers, const double* radii, int64_t n, int64_t leaf_size,
                   tct_tree** out);
/* The same tree built on the GPU (level by level, centres of mass summed in
 * the host builder's order and rounding), exported depth first: node for
 * node equal to tct_tree_build's.  Host inputs; synchronises `stream`. */
int tct_tree_build_device(const double* centers, const double* radii, int64_t n,
                          int64_t leaf_size, void* stream, tct_tree** out);
int64_t tct_tree_n_nodes(const tct_tree* tree);
int tct_tree_max_height(const tct_tree* tree);
/* Per-node arrays (any may be NULL): orig_idx (n balls: tree position ->
 * input index), start/end (ball range), center (x3), R, leaf, depth, height
 * (0 at leaves), children (8 per node, -1 for leaves).  Host. */
int tct_tree_export(const tct_tree* tree, int64_t* orig_idx, int64_t* start, int64_t* end,
                    double* center, double* R, int32_t* leaf, int32_t* depth,
                    int32_t* height, int64_t* children);
void tct_tree_free(tct_tree* tree);

/* Dual traversal producing the compressed P2P, M2P, P2L and M2L lists;
 * replaces fmmmm_interactions (fmm/traversal.cpp:120-243).  treecode = 1 is
 * the mode fmm/tsfmm.py:66-70 uses.  Host. */
int tct_treecode_lists(const tct_tree* obs, const tct_tree* src, double inner_r,
                       double outer_r, int64_t order, int treecode, tct_lists** out);
/* sizes[0..7] = lengths of the obs and src arrays of the p2p, m2p, p2l and
 * m2l lists, in that order (each start array holds one more entry than its
 * obs array).  p2l and m2l are only filled without treecode. */
int tct_lists_sizes(const tct_lists* lists, int64_t* sizes);
/* Copies list `which` (0 p2p, 1 m2p, 2 p2l, 3 m2l) into obs / start / src. */
int tct_lists_export(const tct_lists* lists, int which, int64_t* obs, int64_t* start,
                     int64_t* src);
void tct_lists_free(tct_lists* lists);

/* Device-side description of one tree for tct_fmm_matvec (all pointers
 * device memory unless marked host). */
typedef struct tct_fmm_tree {
    int64_t n_nodes;
    const int64_t* start;         /* first triangle (tree order) of each node */
    const int64_t* end;           /* one past its last triangle */
    const void* centers;          /* Real, 3 per node: ball centre */
    const void* radii;            /* Real: ball radius (> 0) */
    const int64_t* children;      /* 8 per node, -1 at leaves (source tree: M2M) */
    const int64_t* parent;        /* parent node, -1 at the root (obs tree: L2L) */
    const int64_t* orig;          /* tree position -> original triangle index */
    const int64_t* leaves;        /* leaf nodes (source: P2M; obs: L2P) */
    int64_t n_leaves;
    const int64_t* levels;        /* nodes grouped by level: source tree = non-leaf
                                     nodes by height 1, 2, ... (M2M order); obs
                                     tree = nodes by depth 1, 2, ... (L2L order) */
    const int64_t* level_offsets; /* HOST: n_levels + 1 offsets into levels */
    int n_levels;
} tct_fmm_tree;

/* One compressed interaction list (fmm/traversal.cpp:20-53 layout), device. */
typedef struct tct_fmm_list {
    const int64_t* obs;    /* obs nodes with a non-empty list */
    const int64_t* start;  /* n_obs + 1 offsets into src */
    const int64_t* src;    /* source nodes */
    int64_t n_obs;
} tct_fmm_list;

/* Workspace bytes for tct_fmm_matvec (0 for an unsupported kernel, rule,
 * order or mode).  order is the Cartesian expansion order p (0..12). */
size_t tct_fmm_workspace_bytes(int kernel, int prec, int mode, int order, int n_q,
                               int64_t n_obs, int64_t n_src, int64_t n_obs_nodes,
                               int64_t n_src_nodes);

/* Host-side check of the FMM M2L work plan (no GPU): for order p, nb local
 * terms per lane and `lanes` contraction lanes (a multiple of 32, at most
 * 224; the FP32 M2L uses 192 with two source nodes per pipeline stage, 224
 * with one), out[0] = valid (a, b) pairs covered, out[1] = pairs covered
 * twice (or lanes over their warp's step count), out[2] = the chunk length,
 * out[3] = lanes used, out[4] = summed warp step counts.  Returns 0, or 1
 * when the plan does not fit.  Test support for tct_fmm_matvec. */
int tct_fmm_m2l_plan_stats(int order, int nb, int lanes, int64_t* out);

/* Treecode / FMM farfield matvec for elasticU3, elasticRT3, elasticRA3 and
 * elasticRH3; replaces TSFMM.dot (fmm/tsfmm.py:241-256, the p2m, m2m, p2p and
 * m2p kernels of fmm/ts_kernels.cl:428-1003).
 *   mode 0 (treecode, the reference's): far = the M2P list; P2M, M2M by
 *          height, P2P, M2P.
 *   mode 1 (FMM): far = the M2L list (traversal without treecode); P2M, M2M,
 *          M2L, L2L by depth, L2P, P2P.
 * Expansions are Cartesian multipoles / locals of order `order` on
 * monopole and dipole Laplace channels (the reference uses spherical
 * harmonics); which pairs are direct (P2P) is decided by the lists.
 * quad_pts (n_q x 2) and quad_wts are the host 2-D rule (n_q in 3, 4, 7,
 * 13); obs_pts / src_pts Real (device); obs_tris / src_tris in tree order;
 * `in` (n_src x 9) and `out` (n_obs x 9) in original order; out (+)=
 * out_scale * result. */
int tct_fmm_matvec(int kernel, int prec, int mode, int order, int n_q,
                   const double* quad_pts, const double* quad_wts, const double* params,
                   double out_scale, const void* obs_pts, const int32_t* obs_tris,
                   int64_t n_obs, const tct_fmm_tree* obs_tree, const void* src_pts,
                   const int32_t* src_tris, int64_t n_src, const tct_fmm_tree* src_tree,
                   const tct_fmm_list* p2p, const tct_fmm_list* far, const void* in,
                   void* out, int accumulate, void* workspace, size_t workspace_bytes,
                   void* stream);

/* ---- multi-RHS farfield on the tensor cores ------------------------------- */

/* Direct farfield of elasticRH3 (FP32; n_q = 3, 4 or 7 point triangle rule,
 * quad_pts / quad_wts as in tct_farfield_tris_matvec) applied to a panel of
 * R input vectors at once: out[r] (+)= Far in[r] for r < R (R = 16).
 * The reference applies farfield_tris_to_tris{K} (matrix_free.cl:19-107) to
 * one vector per call; here the per-triangle-pair kernel scalars are
 * generated on the CUDA cores and contracted with the input panel by
 * tcgen05.mma (split TF32, FP32 accumulation in tensor memory folded into
 * a Kahan pair every 8 source tiles).
 * in: R x (9 n_src) floats, out: R x (9 n_obs) floats (device, vector after
 * vector); pts / tris as in tct_farfield_tris_matvec.  The workspace size
 * is 0 for an unsupported R or rule. */
size_t tct_farfield_rh_panel_workspace_bytes(int64_t n_obs, int64_t n_src, int R, int n_q);
int tct_farfield_rh_panel_matvec(void* out, const void* in, const void* pts,
                                 const int32_t* obs_tris, int64_t n_obs,
                                 const int32_t* src_tris, int64_t n_src, int R, int n_q,
                                 const double* quad_pts, const double* quad_wts,
                                 const double* params, int accumulate, void* workspace,
                                 size_t workspace_bytes, void* stream);
/* Reads (synchronising the stream) the error word of the last panel apply
 * with this workspace: 0 = ok, 1 = a bounded wait on the tensor cores gave up. */
int tct_farfield_rh_panel_error(const void* workspace, int64_t n_obs, int64_t n_src, int R,
                                int n_q, void* stream, int* host_flag);

/* The same for elasticRT3 (FP32, n_q = 3; R = 16): the RT kernel's sums
 * over the source points of one source triangle are linear in the source
 * triangle's curl of the input and the input at its points, with
 * coefficients (per observation point: sum 1/r, sum D D^T / r^3 and
 * (n_s . D) / r^3 per source point) generated on the CUDA cores straight
 * into tensor memory and contracted with the input panel by tcgen05.mma
 * (A from tensor memory, split TF32, Kahan-folded accumulation).  Replaces
 * R calls of farfield_tris_to_tris{elasticRT3} (matrix_free.cl:19-107).
 * Same arguments, workspace and error word as the RH form. */
size_t tct_farfield_rt_panel_workspace_bytes(int64_t n_obs, int64_t n_src, int R, int n_q);
int tct_farfield_rt_panel_matvec(void* out, const void* in, const void* pts,
                                 const int32_t* obs_tris, int64_t n_obs,
                                 const int32_t* src_tris, int64_t n_src, int R, int n_q,
                                 const double* quad_pts, const double* quad_wts,
                                 const double* params, int accumulate, void* workspace,
                                 size_t workspace_bytes, void* stream);
int tct_farfield_rt_panel_error(const void* workspace, int64_t n_obs, int64_t n_src, int R,
                                int n_q, void* stream, int* host_flag);

/* Point farfield on R = 16 weight vectors at once (FP32 elasticU3/T3/A3/H3;
 * the reference applies farfield_pts{K}, tectosaur/farfield_direct.cl:15-113,
 * one vector per call): out[r][i][d] (+)= sum_j sum_k M_dk(x_i, y_j, n_i, n_j)
 * w[r][j][k] with M the kernel's 3x3 point-pair matrix (r^2 == 0 pairs
 * skipped), generated on the CUDA cores and contracted with the weight panel
 * on the tensor cores (tcgen05.mma kind::tf32, split TF32 hi/lo,
 * compensated folds of the TMEM accumulator, bounded mbarrier waits).
 * in: (R, n_src, 3) float; out: (R, n_obs, 3); points and normals float
 * (n, 3).  Workspace from tct_farfield_pts_panel_workspace_bytes (0 = R
 * unsupported).  tct_farfield_pts_panel_error copies the workspace's timeout
 * flag to host (0 = none; synchronises `stream`). */
size_t tct_farfield_pts_panel_workspace_bytes(int64_t n_obs, int64_t n_src, int R);
int tct_farfield_pts_panel(int kernel, void* out, const void* in, const void* obs_pts,
                           const void* obs_ns, int64_t n_obs, const void* src_pts,
                           const void* src_ns, int64_t n_src, int R, const double* params,
                           int accumulate, void* workspace, size_t workspace_bytes, void* stream);
int tct_farfield_pts_panel_error(const void* workspace, int64_t n_obs, int64_t n_src, int R,
                                 void* stream, int* host_flag);

/* ---- interior evaluation (tectosaur/interior.py InteriorOp) --------------- */

/* Triangle sources to observation points (matrix_free.cl:109-194,
 * farfield_tris_to_pts{K}; kernels U/T/A/H): out[i] (3 per point) = sum over
 * source triangles and rule points of J_s w_q K(x_i, y_q; n_i, n_s) .
 * (sum_b in_b phi_b(q)), r2 == 0 skipped.  in: 9 per source triangle; the
 * rule (n_q <= 13 points) and params on the host; workspace sized by
 * tct_farfield_tris_to_pts_workspace_bytes.  Small point sets split the
 * sources over blocks (partial sums reduced in a fixed order). */
size_t tct_farfield_tris_to_pts_workspace_bytes(int prec, int64_t n_obs, int64_t n_src, int n_q);
int tct_farfield_tris_to_pts(int kernel, int prec, void* out, const void* in,
                             const void* obs_pts, const void* obs_ns, int64_t n_obs,
                             const void* pts, const int32_t* src_tris, int64_t n_src, int n_q,
                             const double* quad_pts, const double* quad_wts,
                             const double* params, void* workspace, size_t workspace_bytes,
                             void* stream);

/* Point-triangle integrals (assemble.cl:140-186 interior_pairs, kernels
 * U/T/A/H): per pair (obs point, src triangle, clicks) (int32 x3) the 27
 * entries [d_obs][b_src][d_src] of J_s sum_q w_q phi_b K, Kahan-summed, the
 * source triangle rotated by clicks and the basis de-rotated.  qp (2 n_q),
 * qw (n_q): device arrays in the working precision.  finite_part keeps only
 * basis b = clicks. */
int tct_interior_pairs(int kernel, int prec, void* result, int n_q, const void* qp,
                       const void* qw, const void* obs_pts, const void* obs_ns, const void* pts,
                       const int32_t* tris, const int32_t* pairs, int64_t n_pairs,
                       const double* params, int finite_part, void* stream);

/* Observation point at vertex `clicks` of the source triangle
 * (interior_corners.cl, elasticH3): 27 entries per pair as above; qt, qw:
 * device arrays of an angle rule on [0, pi/2]. */
int tct_interior_corners(int prec, void* result, int n_q, const void* qt, const void* qw,
                         const void* obs_ns, const void* pts, const int32_t* tris,
                         const int32_t* pairs, int64_t n_pairs, const double* params,
                         void* stream);

/* ---- quasidynamic (rate-and-state) stepper, FP64 --------------------------- */

/* Per DOF: slip velocity from the rate-state Newton solve of
 * qd/newton.cpp:107-150 (rate_state_solver; shear-magnitude form, or
 * per-component with separate_dims).  traction, velocity: (n_tris *
 * basis_dim, 3); tri_normals (n_tris, 3); state, a, normal_stress: per DOF.
 * *n_failed (device int, caller-zeroed) counts DOFs whose Newton iteration
 * did not converge in maxiter steps; they keep the last iterate, as in the
 * reference, whose convergence assert is compiled out (NDEBUG). */
int tct_qd_rate_state(int64_t n_tris, int basis_dim, const double* tri_normals,
                      const double* traction, const double* state, const double* a, double eta,
                      double V0, double C, const double* normal_stress, double tol, int maxiter,
                      int separate_dims, double* velocity, int* n_failed, void* stream);

/* Per DOF: vertex average of v_newton (qd/pt_average.cpp:10-35; vertex p's
 * DOFs are vert_dofs[vert_start[p] .. vert_start[p+1]) in increasing order,
 * dof_vert[dof] = p), the optional no-backslip filter, plus plate_rate x
 * field_edges (qd/model_helpers.py:79-119), and the aging-law derivative
 * dstatedt = (b V0 / Dc)(exp((f0 - state) / b) - |V| / V0)
 * (model_helpers.py:122-130).  velocity: (n_dofs, 3), dstatedt: n_dofs. */
int tct_qd_velocity_state(int64_t n_dofs, const int32_t* vert_start, const int32_t* vert_dofs,
                          const int32_t* dof_vert, const double* v_newton,
                          const double* field_edges, const double* field_interior,
                          double plate_rate, int no_backslip, const double* state,
                          const double* b, double V0, double Dc, double f0, double* velocity,
                          double* dstatedt, void* stream);

/* Batched forms: n_sys systems on the same mesh, system k's traction /
 * state / velocity / Newton velocity / derivative at base + k * stride (in
 * doubles); the mesh fields (normals, a, b, normal_stress, fields, vertex
 * lists) are shared. */
int tct_qd_rate_state_batch(int64_t n_tris, int basis_dim, int n_sys, const double* tri_normals,
                            const double* traction, int64_t traction_stride, const double* state,
                            int64_t state_stride, const double* a, double eta, double V0,
                            double C, const double* normal_stress, double tol, int maxiter,
                            int separate_dims, double* velocity, int64_t velocity_stride,
                            int* n_failed, void* stream);
int tct_qd_velocity_state_batch(int64_t n_dofs, int n_sys, const int32_t* vert_start,
                                const int32_t* vert_dofs, const int32_t* dof_vert,
                                const double* v_newton, int64_t vn_stride,
                                const double* field_edges, const double* field_interior,
                                double plate_rate, int no_backslip, const double* state,
                                int64_t state_stride, const double* b, double V0, double Dc,
                                double f0, double* velocity, int64_t velocity_stride,
                                double* dstatedt, int64_t dstate_stride, void* stream);

/* Fused element-wise steps of the batched derivative and RK23 step (no
 * reference counterpart as kernels: qd/full_model.py:178-200 evaluates them
 * with numpy; scipy's RK23 forms the stages).  Each rounds every value in
 * the order of the element-wise expression it replaces (no fused
 * multiply-add), so the results are bit-identical to it, except the error
 * norm's sum of squares (a block reduction).  Device arrays; strides in
 * elements.
 * Slip deficit, cast to out_prec (TCT_F32 / TCT_F64):
 *   out[r][i] = interior[i] * ((ts[r] * plate_rate) * inslipdir[i] - Y[r][i]),
 *   i < n9 (the slip part of state row r). */
int tct_qd_deficit_batch(int64_t n9, int n_sys, const double* ts, double plate_rate,
                         const double* inslipdir, const double* interior, const double* Y,
                         int64_t y_stride, int out_prec, void* out, int64_t out_stride,
                         void* stream);
/* Derivative rows: out[r] = (V[r], dstate[r]), or Y[r] * inf when Y[r] has a
 * non-finite entry, a state entry (Y[r][n9 ..]) below 0 or above state_max,
 * or V[r] a non-finite entry (full_model.py's rejection of such states). */
int tct_qd_finish_batch(int64_t n9, int64_t n_state, int n_sys, const double* Y, int64_t y_stride,
                        const double* V, int64_t v_stride, const double* dstate,
                        int64_t ds_stride, double state_max, double* out, int64_t out_stride,
                        void* stream);
/* Stage combination: out[r][i] = y[r][i] + (((k0 c0 + k1 c1) + k2 c2) + k3 c3)[r][i] * h[r]
 * for the first n_terms (1..4) terms; y may be NULL (no y term).  k,
 * k_strides, coeffs: host arrays of n_terms (device row pointers). */
int tct_qd_combine_batch(int64_t n, int n_sys, int n_terms, const double* const* k,
                         const int64_t* k_strides, const double* coeffs, const double* h,
                         const double* y, int64_t y_stride, double* out, int64_t out_stride,
                         void* stream);
/* Error norm of an RK23 attempt: norms[r] = || e / (tol + max(|y|, |y_new|) tol) ||_2
 * with e = (combination of the terms) * h[r]. */
int tct_qd_error_norm_batch(int64_t n, int n_sys, int n_terms, const double* const* k,
                            const int64_t* k_strides, const double* coeffs, const double* h,
                            const double* y, int64_t y_stride, const double* y_new,
                            int64_t yn_stride, double tol, double* norms, void* stream);

/* Conjugate gradients on a CSR matrix (int64 indices, double values) in one
 * CTA, x0 = 0, stopping when ||r|| < max(atol, rtol ||b||) or after maxiter
 * iterations: the scipy.sparse.linalg.cg solve of the constrained mass
 * system in qd/full_model.py:160-176.  work: 3 n doubles; *iters (device)
 * receives the iteration count. */
int tct_cg_csr(int64_t n, const int64_t* indptr, const int64_t* indices, const double* data,
               const double* b, double* x, double* work, double rtol, double atol, int maxiter,
               int* iters, void* stream);
/* n_sys systems with the same matrix, one CTA each: b_k = b + k b_stride,
 * x_k = x + k x_stride, work: 3 n n_sys doubles, iters: n_sys ints. */
int tct_cg_csr_batch(int64_t n, int n_sys, const int64_t* indptr, const int64_t* indices,
                     const double* data, const double* b, int64_t b_stride, double* x,
                     int64_t x_stride, double* work, double rtol, double atol, int maxiter,
                     int* iters, void* stream);

/* ---- tuned launch shapes (the autotuner) ---------------------------------- */
/* The reference compiles a kernel per template argument set and caches the
 * module (tectosaur/util/gpu.py:63-77); its launch shapes are fixed.  Here a
 * launch's shape -- how the work is cut into CTAs -- is looked up in an
 * in-library cache keyed by (op, kernel, prec, nq, rhs, bucket(n0),
 * bucket(n1)), bucket(n) = round(log2 n) + 1 (0 for n <= 0); launches
 * without an entry use the built-in heuristics.  Values per op:
 *   TCT_TUNE_FARFIELD  n0 = n_obs, n1 = n_src, rhs = 1: v0 = source chunks
 *                      (grid.y of the direct farfield; clamped to the sources
 *                      and to the partial sums the workspace holds), v1 = 1;
 *   TCT_TUNE_BSR9      kernel = -1, nq = 0, rhs = 1, n0 = block rows,
 *                      n1 = blocks per row (data_stride / n_row_blocks):
 *                      v0 = lanes per block row (32, 16, 8, 4, 2 or 1;
 *                      below 32 a warp serves several short rows), v1 = CTAs
 *                      per SM (1 to 64);
 *   TCT_TUNE_FAR_PANEL reserved.
 * A shape changes the floating-point summation order, not the quantity
 * computed.  Host functions; the cache is shared by all threads. */
#define TCT_TUNE_FARFIELD 1
#define TCT_TUNE_BSR9 2
#define TCT_TUNE_FAR_PANEL 3
int tct_tune_set(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1, int v0,
                 int v1);
/* 1 and the values when the key has an entry, else 0. */
int tct_tune_get(int op, int kernel, int prec, int nq, int rhs, int64_t n0, int64_t n1, int* v0,
                 int* v1);
int tct_tune_bucket(int64_t n);
/* Enumeration and restore of the cache for persistence: key7 = {op, kernel,
 * prec, nq, rhs, bucket0, bucket1}. */
int64_t tct_tune_size(void);
int tct_tune_entry(int64_t i, int* key7, int* v0, int* v1);
int tct_tune_put_entry(const int* key7, int v0, int v1);
void tct_tune_clear(void);

/* Autotune the direct farfield's source chunking for one problem: times the
 * candidate chunk counts with CUDA events (on `stream`, which is
 * synchronised) on the caller's buffers -- the same arguments as
 * tct_farfield_tris_matvec, out is overwritten -- stores the fastest in the
 * cache and returns it in *chunks (host). */
int tct_farfield_autotune(int kernel, int prec, void* out, const void* in, const void* pts,
                          const int32_t* obs_tris, int64_t n_obs, const int32_t* src_tris,
                          int64_t n_src, int n_q, const double* quad_pts,
                          const double* quad_wts, const double* params, void* workspace,
                          size_t workspace_bytes, void* stream, int* chunks);
/* Autotune tct_bsr9_matvec's shape (lanes per block row x CTAs per SM) for
 * one matrix, as above (y is overwritten with A x); data_stride is the
 * matrix's own plane stride (its slot count when rows are padded), as given
 * to tct_bsr9_matvec.  Results in *lanes, *ctas_per_sm. */
int tct_bsr9_autotune(int prec, int64_t n_row_blocks, const int32_t* indptr,
                      const int32_t* indices, const void* data, int64_t data_stride,
                      const void* x, void* y, void* stream, int* lanes, int* ctas_per_sm);
/* Workspace of tct_farfield_tris_matvec that holds the partial sums of up to
 * max_chunks source chunks (>= tct_farfield_workspace_bytes), for operators
 * that let the autotuner raise the chunk count. */
size_t tct_farfield_workspace_bytes_chunks(int kernel, int prec, int64_t n_obs, int64_t n_src,
                                           int n_q, int max_chunks);

/* ---- constrained solve -------------------------------------------------- */

/* y (+)= A x for a CSR matrix with double values (device): the constraint
 * matrix cm or its transpose in the constrained GMRES; replaces the host
 * csr_matrix.dot calls of examples/solve.py:44-49 and
 * simple_solver.py:18-22.  x, y Real according to prec. */
int tct_csr_matvec(int prec, int64_t n_rows, const int64_t* indptr, const int64_t* indices,
                   const double* data, const void* x, void* y, int accumulate, void* stream);
/* The same for a panel of n_vec vectors: x + v * x_stride -> y + v * y_stride
 * (strides in elements), one launch. */
int tct_csr_matvec_panel(int prec, int64_t n_rows, const int64_t* indptr, const int64_t* indices,
                         const double* data, const void* x, int64_t x_stride, void* y,
                         int64_t y_stride, int n_vec, int accumulate, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TCT_B200_H */
