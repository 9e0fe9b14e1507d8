/*
 * Additive API of libhodlr_b200.so (no counterpart in hmat_lib).
 *
 * The hmat_lib entry points (allocators.h, constructors.h, vector_algebra.h,
 * dense_algebra.h, hodlr_algebra.h, utils.h) take host buffers: each call
 * copies its dense inputs to the GPU and its result back.  A tree built by
 * dense_to_tree_hodlr() or multiply_hodlr_hodlr() keeps a device copy that
 * later products reuse; a tree assembled by the caller is uploaded on its
 * first product and reused while its structure, data pointers and sampled
 * values are unchanged (call hodlr_b200_sync_tree() after editing factor
 * values in place).
 *
 * The functions below work on device-resident trees and device buffers
 * directly.  `stream` is a cudaStream_t (NULL: the CUDA default stream);
 * they return an ErrorCode (error.h) and never fall back to the CPU.
 */
#pragma once

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

struct TreeHODLR;
typedef struct hodlr_b200_tree_s *hodlr_b200_tree;

enum HodlrB200Op {
  HODLR_B200_OP_N = 0,   /* Y = H X   */
  HODLR_B200_OP_T = 1,   /* Y = H^T X */
  HODLR_B200_OP_L = 2    /* Y = X H   (X is k x n) */
};

/* Status of the entry points that say so when a CUDA runtime call or a kernel
 * launch fails (hmat_lib's ErrorCode has no such value). */
enum { HODLR_B200_CUDA_ERROR = 100 };

enum HodlrB200Precision {
  HODLR_B200_FP64 = 0,   /* FP64 products (FP64 tensor cores) */
  HODLR_B200_MIXED = 1   /* split-precision tensor-core products with FP64 result */
};

const char *hodlr_b200_version(void);
/* Message describing the last failure on the calling thread. */
const char *hodlr_b200_last_error(void);
/* Runtime knobs (process-wide; read when a call or a cached plan is made).
 * Returns SUCCESS.  Every option the library reads, with its default:
 *   matmat_precision (0): 1 = host-buffer products (multiply_hodlr_dense,
 *       multiply_hodlr_transpose_dense, multiply_dense_hodlr) on the int8
 *       tensor-core path
 *   host_chunks (0): column chunks of host-buffer products; 0 automatic (up to
 *       4 from 128 columns), 1 one piece, n that many
 *   matvec_kernels (1): one right-hand side by the dedicated matvec kernels;
 *       0 = the GEMM engine
 *   pool_keep (1): freed stream-ordered scratch and tree arenas stay mapped in
 *       the device's default memory pool (release threshold unlimited); set
 *       0 before the library's first call on a device to leave that pool alone
 *   learned_ranks (0): size each sketch from the rank model (fallback to
 *       adaptive growth per block)
 *   learned_margin (0.1), learned_extra (40), learned_eta (1.0): one-shot width
 *       ceil((1 + margin) r) + extra; accepted when the residual estimate is
 *       at most eta tol sigma_0
 *   kernel_length (0): kernel length scale given to the rank model (0: the
 *       kernel's own length in a matrix-free build, else unknown)
 *   record_features (0): record per-block features and Frobenius eps-ranks of
 *       the next builds (hodlr_b200_build_features)
 *   sketch_first (64), sketch_step (64): first and later widths of the
 *       adaptive range finder's rounds
 *   sketch_eta (0.01): stopping residual, times tol sigma_0
 *   sketch_start (256): starting sketch scratch width of a block (or an eighth
 *       of its width, or twice its one-shot width, if more); grown 2x in place
 *       when it fills
 *   sketch_cap (0): largest sketch width (a block that needs more ends the
 *       build with SVD_FAILURE); 0 = as wide as memory allows
 *   sketch_mem_frac (0.6): with sketch_cap 0, a block's sketch grows while
 *       each growth of its scratch (plus its core SVD) fits this share of the
 *       device memory free or held unused by the stream-ordered pool
 *   sketch_seed (20240607): seed of the Gaussian test matrices
 *   sketch_clean_rel (1e-13): rounding level below which a new panel is zeroed
 *   exact_max (128): blocks with min(m, n) up to this are compressed by an
 *       exact Jacobi SVD
 *   jacobi_max_sweeps (60): Jacobi sweep bound (SVD_FAILURE past it)
 *   jacobi_norm_stop (0): 1 = in the build's one-CTA / cluster Jacobi SVDs a
 *       column pair also counts as orthogonal when its product is at rounding
 *       level of eps ||A||_F times the larger column norm (fewer sweeps; the
 *       singular vectors of small singular values are then orthogonal only to
 *       about eps ||A|| / sigma)
 *   jacobi_cluster_min_c (192): problems this wide or wider use a cluster of
 *       8 CTAs
 *   bj_inner_sweeps (30): sweeps of the block Jacobi SVD's per-pair eigensolver
 *       at most (fewer: cheaper rounds, possibly more outer sweeps)
 *   jacobi_block_min_c (128): sketch cores this wide or wider are solved by
 *       the block Jacobi SVD (32-column blocks; per round one launch: Gram of
 *       each 64-column pair, its eigenvectors, in-place rotation)
 *   hxh_dense_max (256): H x H blocks up to this many rows are recompressed
 *       from their dense product
 *   hxh_precision (0): 1 = the subtree products of H x H on the int8 tensor
 *       cores (cores, recompression and leaves stay FP64)
 *   build_precision (0): 1 = the sketch products of a dense-input build
 *       (Y = A Omega, B^T = A^T Q) on the int8 tensor cores; orthonormalisation,
 *       core SVDs and truncation stay FP64
 *   autotune (1), batch_shape (-1), use_graphs (1), check_status (0): batched
 *       products time candidate tile shapes / force one (0-3) / replay a CUDA
 *       graph / read the mixed kernels' status word after each call
 *   ozaki_schedule (1): int8 GEMM tile schedule, longest first (0 round-robin)
 *   ozaki_phase1_tiles_per_cta (2): K-split granularity of the projections
 *   ozaki_copy_split (1): bulk copies per int8 operand block
 *   record_phase_times (0): events around each product phase and its main GEMM
 *       (hodlr_b200_phase_times)
 *   gemm_f64_engine (2): FP64 products on the FP64 tensor cores (DMMA) with
 *       32-deep K stages; 1 = the same with 16-deep K stages; 0 = the DFMA
 *       kernel
 *   product_shape1 (-1), product_shape2 (-1): tile shape of the FP64 product's
 *       projection / output phase (0: 128x64, 1: 64x128, 2: 32x128,
 *       3: 32x256; -1: chosen by op and k)
 *   product_graphs (1): a device FP64 product that repeats an earlier call
 *       (same tree, op, sizes, buffers and non-default stream) is captured
 *       once as a CUDA graph and replayed; 0 = always launch directly */
int hodlr_b200_set_option(const char *name, double value);
/* Allocator for every host buffer the library allocates (tree nodes, factor
 * copies, results returned for out == NULL).  Both NULL restores malloc/free. */
void hodlr_b200_set_host_allocator(void *(*alloc_fn)(size_t), void (*free_fn)(void *));
/* Number of kernels launched by this library so far in this process. */
long long hodlr_b200_kernel_launches(void);

/* Build from a device-resident n x n column-major matrix (leading dimension
 * ld), block sizes halved as dense_to_tree_hodlr does (ms == NULL) or given
 * per leaf (2^height entries).  flags: 0.  Like dense_to_tree_hodlr, a build
 * that ends with SVD_FAILURE (a Jacobi SVD out of sweeps, or a rank at the
 * sketch cap) still stores the tree it made in *out: the caller frees it with
 * hodlr_b200_tree_free.  Other errors leave *out untouched. */
int hodlr_b200_build_dev(int height, int n, const int *ms, const double *d_matrix, int ld,
                         double svd_threshold, int flags, void *stream, hodlr_b200_tree *out,
                         int *ierr);
/* Builds `count` trees at once, tree i of height heights[i] from the
 * ns[i] x ns[i] device matrix d_matrices[i] (leading dimension lds[i], block
 * sizes halved as dense_to_tree_hodlr does), all with relative tolerance
 * svd_threshold: the blocks of every tree share the launches of every stage,
 * and each tree comes out as it would from hodlr_b200_build_dev.  The trees
 * go to out[0 .. count-1] (free each with hodlr_b200_tree_free); on
 * SVD_FAILURE (any tree) the trees are still stored, on other errors none.
 * hmat_lib builds one tree per call (dense_to_tree_hodlr,
 * src/constructors.c:629). */
int hodlr_b200_build_batched_dev(int count, const int *heights, const int *ns,
                                 const double *const *d_matrices, const int *lds,
                                 double svd_threshold, void *stream, hodlr_b200_tree *out,
                                 int *ierr);
void hodlr_b200_tree_free(hodlr_b200_tree t);
/* Fills an allocated, empty host tree of the same height with copies of the
 * device factors (library allocator; free with free_tree_data). */
int hodlr_b200_tree_to_host(hodlr_b200_tree t, struct TreeHODLR *hodlr, int *ierr);
/* Device handle of a host tree (uploading it if needed); release with
 * hodlr_b200_tree_free. */
hodlr_b200_tree hodlr_b200_tree_from_host(const struct TreeHODLR *hodlr, int *ierr);
int hodlr_b200_tree_info(hodlr_b200_tree t, int *height, int *n, int *max_rank,
                         long long *storage_doubles, long long *arena_bytes);
/* Ranks in block order b = 2 * (2^d - 1 + j) + (c - 1); returns the count. */
int hodlr_b200_tree_ranks(hodlr_b200_tree t, int *ranks, int capacity);
/* Y = op(H, X) on device buffers (column-major). */
int hodlr_b200_matmat_dev(hodlr_b200_tree t, int op, int precision, const double *d_x, int k,
                          int ldx, double *d_y, int ldy, void *stream);
/* Synchronises with `stream` and returns SUCCESS, or SVD_FAILURE if a
 * mixed-precision kernel on this tree stopped on its bounded barrier wait
 * since the last check (the error word is then reset). */
int hodlr_b200_check(hodlr_b200_tree t, void *stream);
/* H1 * H2 with recompression at svd_threshold, result stays on the device. */
int hodlr_b200_hxh_dev(hodlr_b200_tree a, hodlr_b200_tree b, double svd_threshold,
                       hodlr_b200_tree *out, int *ierr);
/* Build of the kernel matrix A_ij = k(|p_i - p_j|) + diag delta_ij (points
 * and kinds as for hodlr_b200_kernel_matrix_dev below) without forming it:
 * every entry the construction needs is computed on the device where it is
 * used, so memory holds only the points, the tree and the sketches (a dense
 * n = 65536 input would take 34 GB).  The tree equals the one
 * hodlr_b200_build_dev makes from the generated dense matrix.  No
 * counterpart in hmat_lib, whose constructor takes the dense matrix
 * (dense_to_tree_hodlr, src/constructors.c:629).  Ownership and errors as for
 * hodlr_b200_build_dev. */
int hodlr_b200_build_kernel_dev(int height, int n, const int *ms, const double *d_points,
                                int dim, int kind, double length, double diag,
                                double svd_threshold, int flags, void *stream,
                                hodlr_b200_tree *out, int *ierr);
/* Recompression of one low-rank product U V^T (U m x s, V n x s, device,
 * column-major with leading dimensions ldu >= m, ldv >= n) by the routine
 * hodlr_b200_hxh_dev / multiply_hodlr_hodlr applies to every output block.
 * It replaces hmat_lib's internal recompress (src/hodlr_algebra.c:97-211):
 * Householder QR of U and V, SVD of R_U R_V^T, absolute truncation of the
 * singular values at svd_threshold (:160-163), U' = Q_U W Sigma, V' = Q_V Z;
 * with dense != 0 it replaces recompress_large_s (:280-343), the SVD of the
 * dense U V^T.  Writes the rank r to *rank and U' (m x r, ld m), V' (n x r,
 * ld n) to d_u_out / d_v_out, which hold max(s, min(m, n)) columns.
 * Synchronises with `stream`; returns an ErrorCode (SVD_FAILURE when the
 * Jacobi SVD runs out of sweeps). */
int hodlr_b200_recompress_dev(int m, int n, int s, const double *d_u, int ldu, const double *d_v,
                              int ldv, double svd_threshold, int dense, double *d_u_out,
                              double *d_v_out, int *rank, void *stream);
/* Kernel matrix in device memory: out_ij = k(|p_i - p_j|) + diag delta_ij,
 * points column-major n x dim (coordinate a of point i at d_points[i + a n]);
 * kind 0: exp(-r^2 / (2 l^2)), 1: Matern-3/2 (1 + sqrt(3) r / l) exp(-sqrt(3) r / l),
 * 2: exp(-r / l). */
int hodlr_b200_kernel_matrix_dev(const double *d_points, int n, int dim, int kind, double length,
                                 double diag, double *d_out, int ld, void *stream);
/* The rows x cols block of that kernel matrix whose first entry is (r0, c0)
 * (0 <= r0, r0 + rows <= n, likewise for columns), column-major with leading
 * dimension ld >= rows: for products with kernel matrices too large to hold
 * whole.  No counterpart in hmat_lib. */
int hodlr_b200_kernel_block_dev(const double *d_points, int n, int dim, int kind, double length,
                                double diag, int r0, int c0, int rows, int cols, double *d_out,
                                int ld, void *stream);
/* Device time (ms) of the two product phases accumulated since the last call
 * while option "record_phase_times" is non-zero: out[0] projections
 * (W = V^T X), out[1] output bands (Y = D X + sum U W), out[2] number of
 * products, out[3] / out[4] the main GEMM launch of each phase alone (for
 * mixed products the phases also slice their operands; for FP64 products
 * these equal out[0] / out[1]).  Resets the accumulators; returns the
 * number of values. */
int hodlr_b200_phase_times(double *out, int capacity);
/* Statistics of the calling thread's most recent build: exact blocks,
 * sketched blocks, sketch rounds, seconds, cap hit, max Jacobi sweeps (exact,
 * sketched), unconverged Jacobi problems (exact, sketched), largest sketch,
 * then the device milliseconds of the stages: small-block SVDs, sketch
 * rounds, SVDs of the sketched cores, finishing; one-shot sketches that fell
 * back to adaptive growth; milliseconds of the rank-model features and
 * prediction; FP64 GEMM work (flops, 2 M N K summed) and input entries;
 * host milliseconds from the call to the first stage and spent making GEMM
 * and TSQR plans.  Returns the number of values. */
int hodlr_b200_build_stats(double *out, int capacity);
/* y = H x on device buffers, allocating nothing (no counterpart in hmat_lib).
 * For callers that cannot allocate device memory while they run: an
 * iterative solver whose memory pool already holds nearly all of HBM, or
 * latency-critical code that cannot afford cudaMalloc's implicit device
 * synchronisation.  The per-block projections V_b^T x, the product's only
 * scratch, live in a fixed 528 KiB array of device memory inside the library
 * (held on every GPU that loads it, until exit) instead of a per-call
 * allocation.  Limits: the ranks of the tree sum to at most 65536 and it has
 * at most 4096 off-diagonal blocks; larger trees return INPUT_ERROR with a
 * message.  The tree's device must be the current device (INPUT_ERROR
 * otherwise).  The first call on a device looks the array's address up
 * (cudaGetSymbolAddress), so make it before any stream capture.  All calls
 * share the array: calls that overlap on the GPU (unordered streams) race;
 * order them on one stream.  Returns an ErrorCode, or HODLR_B200_CUDA_ERROR
 * when a launch fails or a CUDA error from earlier work was pending (that
 * error is cleared and named in hodlr_b200_last_error()). */
int hodlr_b200_matvec_noalloc_dev(hodlr_b200_tree t, const double *d_x, double *d_y,
                                  void *stream);
/* Re-upload a host tree whose factor values were edited in place. */
int hodlr_b200_sync_tree(const struct TreeHODLR *hodlr);

/* ---- direct solver (no counterpart in hmat_lib) -----------------------------
 * A = D (I + W_{h-1} V_{h-1}^T) ... (I + W_0 V_0^T): leaf inverses, then per
 * depth the level's U blocks solved through the deeper levels and, per node,
 * the inverse of its capacitance matrix (Woodbury).  The factor keeps a
 * reference to the tree.  Factorising returns INPUT_ERROR when a leaf or a
 * capacitance matrix is singular to working precision. */
typedef struct hodlr_b200_factor_s *hodlr_b200_factor;
int hodlr_b200_factorize_dev(hodlr_b200_tree t, void *stream, hodlr_b200_factor *out, int *ierr);
/* X = A^-1 B for k right-hand sides (device, column-major; X and B distinct).
 * The first call for a given (k, ldb, ldx, stream) builds and keeps its launch
 * plans and scratch (synchronously); later calls launch 1 + 3h GEMMs. */
int hodlr_b200_solve_dev(hodlr_b200_factor f, const double *d_b, int k, int ldb, double *d_x,
                         int ldx, void *stream);
void hodlr_b200_factor_free(hodlr_b200_factor f);

/* Writes a device tree to a file: height, n, leaf sizes, ranks, every leaf and
 * factor, and a checksum (layout in hmat_lib_b200/csrc/treefile.cpp).  No
 * counterpart in hmat_lib, which has no serialisation. */
int hodlr_b200_tree_save(hodlr_b200_tree t, const char *path);
/* Reads a file written by hodlr_b200_tree_save into a new device tree
 * (*out, freed with hodlr_b200_tree_free).  A file that is not a tree file,
 * is truncated or fails its checksum gives INPUT_ERROR and leaves *out
 * untouched. */
int hodlr_b200_tree_load(const char *path, hodlr_b200_tree *out);

/* Y_i = op(H_i) X_i for i < count, every tree of the batch (any sizes, ranks
 * and heights) in one launch per phase.  Device pointers, column-major;
 * k[i] columns of X_i / Y_i (rows for op L), leading dimensions ldx[i],
 * ldy[i].  precision HODLR_B200_MIXED needs op N, leaf sizes that are
 * multiples of 32 and each tree at most once in the batch.  No counterpart in
 * hmat_lib, which multiplies one tree at a time (multiply_hodlr_dense,
 * src/dense_algebra.c:361).  The plan for a call signature (trees, pointers,
 * sizes) is made on its first call: an autotuner times the candidate tile
 * configurations on the real operands, and the chosen launches are captured
 * into a CUDA graph that later calls with the same signature replay (option
 * "autotune" = 0 keeps the default configuration, "use_graphs" = 0 launches
 * directly).  Up to four plans are cached; a freed tree invalidates every plan
 * that uses it.  Returns an ErrorCode. */
int hodlr_b200_matmat_batched_dev(int count, const hodlr_b200_tree *trees, int op, int precision,
                                  const double *const *d_x, const int *k, const int *ldx,
                                  double *const *d_y, const int *ldy, void *stream);
/* Configuration the autotuner chose for the latest batched plan, written to
 * buf (NUL-terminated, at most capacity bytes); returns its full length. */
int hodlr_b200_batched_tuning(char *buf, int capacity);
/* SUCCESS, or SVD_FAILURE if a cached mixed-precision batch hit a barrier
 * timeout (read and reset). */
int hodlr_b200_batched_check(void);
/* Drops every cached batched plan (their graphs and scratch). */
void hodlr_b200_batched_release(void);

/* ---- learned rank predictor (no counterpart in hmat_lib) -------------------
 * An MLP 8 -> 64 -> 64 -> 1 (ReLU, FP32) maps an off-diagonal block's
 * features to log2(rank + 1), the rank being the block's Frobenius
 * epsilon-rank at the build tolerance (the sketch width at which the
 * randomized range finder's a-posteriori error estimate meets it).  Features: log2(min(m,
 * n)), depth, ln(kernel length) (option "kernel_length", 0 if unknown),
 * log10(s_i / s_1) for i = 2, 4, 8, 12, 16 of a 16-column Gaussian sketch of
 * the block.  Parameters (hodlr_b200_rank_model_size() floats): feature mean
 * [8], feature scale [8], W1 [8][64], b1 [64], W2 [64][64], b2 [64], W3 [64],
 * b3.  All arrays below are host memory; the arithmetic runs on the GPU with
 * the library's own training and inference kernels. */
int hodlr_b200_rank_model_size(void);
/* Model used by builds with option "learned_ranks" = 1 (count 0 clears it). */
int hodlr_b200_rank_model_set(const float *params, int count);
/* Copies the current model out; returns its size (0: none). */
int hodlr_b200_rank_model_get(float *params, int capacity);
/* Trains from scratch on n samples (features n x 8 row-major, targets
 * log2(rank + 1)) with Adam on mini-batches; writes the parameters and the
 * full-data loss every 100 steps (up to log_capacity values). */
int hodlr_b200_rank_model_train(const float *features, const float *targets, int n, int steps,
                                int batch, double lr, unsigned long long seed, float *params_out,
                                float *loss_log, int log_capacity);
/* out[i] = model(params, features[i]). */
int hodlr_b200_rank_model_predict(const float *params, const float *features, int n,
                                  float *out);
/* Mean squared error of the model on n samples and its gradient with respect
 * to every parameter (the normalisation entries get 0). */
int hodlr_b200_rank_model_gradient(const float *params, const float *features,
                                   const float *targets, int n, float *grad_out,
                                   float *loss_out);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) of step number `step`
 * (1-based) on the trainable parameters; m and v are updated in place. */
int hodlr_b200_rank_model_adam(float *params, const float *grad, float *m, float *v, int step,
                               double lr);
/* Per sketched block of the calling thread's latest build that computed
 * features (option "learned_ranks" or "record_features"): 8 features, the
 * final rank, the predicted rank (-1 without a model), the first sketch
 * width, whether the block fell back to adaptive growth, the final sketch
 * width, the Frobenius epsilon-rank (fewest leading singular values whose
 * discarded tail has Frobenius norm <= tol * s_0; computed only with option
 * "record_features", 0 otherwise).  Rows of 14 floats; returns the number of
 * rows. */
int hodlr_b200_build_features(float *out, int capacity_rows);

#ifdef __cplusplus
}
#endif
