/*
 * hyperalignment_b200.h -- C ABI of the B200 (sm_100a) searchlight alignment backend.
 *
 * The backend is a drop-in for the searchlight calls of the reference C library
 * (neurolabusc/hyperalignment, csrc/).  It adds one value to the reference's
 * backend enum, kHaBackendB200 = 4, and exports:
 *
 *   - the reference's dense entry point under its own name and signature
 *     (csrc/ha_searchlight.h:69-80), accepting backend == kHaBackendB200, so the
 *     reference ctypes wrapper (hyperalignment_c.py:44-60) binds it unchanged;
 *   - a backend function with the signature of the reference's CUDA backend
 *     (csrc/ha_cuda.h:56-66), for the reference dispatcher
 *     (csrc/ha_searchlight.c:1106-1132) to call;
 *   - flat-array (pointer + size) forms of the sparse-output Procrustes and ridge
 *     searchlight calls (csrc/ha_searchlight.h:46-52, :86-90) and of the CSC
 *     pattern builder (csrc/ha_sparse.h, ha_sparse_init);
 *   - lifecycle calls shaped like the CUDA backend's (csrc/ha_cuda.h:32-42).
 *
 * All arguments are plain pointers and sizes.  Unless a function says
 * "device", every pointer is host memory owned by the caller.  Return values
 * are the reference's error codes (csrc/ha_common.h:36-42).  There is no CPU
 * fallback: with no usable GPU or no loaded kernels the calls return
 * kHaErrorInternal and print the reason to stderr.
 *
 * Threading: one host thread at a time (calls are serialised by a mutex).
 * The backend keeps device buffers between calls; ha_b200_cleanup releases them.
 */
#ifndef HYPERALIGNMENT_B200_H
#define HYPERALIGNMENT_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef HA_COMMON_H
/* Same values as csrc/ha_common.h:36-42 and :71-76 of the reference. */
enum {
	kHaSuccess       =  0,
	kHaErrorAlloc    = -1,
	kHaErrorSvd      = -2,
	kHaErrorArg      = -3,
	kHaErrorInternal = -4,
};
typedef enum {
	kHaBackendCPU64 = 0,
	kHaBackendCPU32 = 1,
	kHaBackendMetal = 2,
	kHaBackendCUDA  = 3,
} THaBackend;
#endif

#ifndef HA_HAS_BACKEND_B200
/* New backend value; 0-3 keep their reference meaning. */
#define kHaBackendB200 ((THaBackend)4)
#endif

/* ---- lifecycle (cf. ha_cuda_init / ha_cuda_cleanup / ha_cuda_available, csrc/ha_cuda.h:32-42) ---- */

/* Selects the current CUDA device and checks that it is sm_100.  Idempotent and cheap. */
int ha_b200_init(void);
/* Releases every device buffer, stream and cached plan.  Safe without init. */
void ha_b200_cleanup(void);
/* True once ha_b200_init succeeded. */
bool ha_b200_available(void);

/* Host threads for host-side work (accumulating into caller's dense T), cf. csrc/ha_searchlight.h:14-20. */
void ha_set_num_threads(int n);
int ha_get_num_threads(void);

/* ---- dense searchlight Procrustes ---- */

/*
 * Same contract as the reference's ha_searchlight_procrustes_dense
 * (csrc/ha_searchlight.h:69-80, csrc/ha_searchlight.c:950-1376):
 * X_data, Y_data are nt x nv float64 (column-major when col_major);
 * searchlight s is sl_indices[sl_offsets[s] .. sl_offsets[s+1]); sl_dists NULL
 * means uniform weights, else w = (radius - d) / radius normalised to sum to 1
 * per vertex; T_out is nv x nv row-major float64 and is ACCUMULATED
 * (T_out[sl[i], sl[j]] += w[i] * T_s[i, j]).  isReflection = false forces
 * det(T_s) > 0 and isScaling applies the reference's global scale.
 * backend must be kHaBackendB200; anything else returns kHaErrorArg (this
 * library has no CPU paths).
 */
int ha_searchlight_procrustes_dense(
	const double *X_data, const double *Y_data,
	int32_t nt, int32_t nv,
	const int32_t *sl_indices,
	const int32_t *sl_offsets,
	const double *sl_dists,
	int32_t count,
	double radius,
	double *T_out,
	bool isReflection, bool isScaling,
	THaBackend backend,
	bool col_major);

/*
 * Backend arm with the signature of ha_searchlight_procrustes_cuda
 * (csrc/ha_cuda.h:56-66).  Unlike the reference CUDA arm it honours
 * isScaling and isReflection = false, accepts col_major = false, and
 * accumulates into T_out instead of overwriting it (ha_cuda.cu:445, :457-460).
 */
int ha_searchlight_procrustes_b200(
	const double *X_data, const double *Y_data,
	int32_t nt, int32_t nv,
	const int32_t *sl_indices,
	const int32_t *sl_offsets,
	const double *sl_dists,
	int32_t count,
	double radius,
	double *T_out,
	bool isReflection, bool isScaling,
	bool col_major);

/* ---- CSC pattern and weights ---- */

/*
 * CSC sparsity pattern of the union of sl x sl blocks (nv x nv), bit-exact to
 * the reference's ha_sparse_init (csrc/ha_sparse.c:31-112): rows ascending in
 * each column, indptr of nv + 1 int32.  Built on the GPU without enumerating
 * the sum of n^2 pairs.  Pass indices = NULL to get *nnz only; otherwise
 * capacity must be >= nnz.  Searchlight indices must be unique within a
 * searchlight and in [0, nv).
 */
int ha_sparse_pattern_b200(
	const int32_t *sl_indices, const int32_t *sl_offsets, int32_t count, int32_t nv,
	int32_t *indptr, int32_t *indices, int64_t capacity, int64_t *nnz);

/*
 * Flat searchlight weights (one float64 per sl_indices entry), the rule of
 * ha_searchlight_weights (csrc/ha_searchlight.c:36-92), bit-exact.
 */
int ha_searchlight_weights_b200(
	const int32_t *sl_indices, const int32_t *sl_offsets, const double *sl_dists,
	int32_t count, double radius, int32_t nv, double *weights_out);

/* ---- sparse-output searchlight Procrustes and ridge ---- */

/*
 * Flattened form of ha_searchlight_procrustes (csrc/ha_searchlight.h:46-52,
 * csrc/ha_searchlight.c:147-413) with sls_Y = NULL: accumulates
 * data[k] += w[i] * T_s[i, j] into the CSC matrix (indptr, indices, nnz)
 * whose pattern came from ha_sparse_init or ha_sparse_pattern_b200.
 * weights: one float64 per sl_indices entry (row weights, as
 * ha_sparse_scatter_add, csrc/ha_sparse.c:128-142), or NULL for unweighted.
 */
int ha_searchlight_procrustes_csc_b200(
	const double *X_data, const double *Y_data, int32_t nt, int32_t nv,
	const int32_t *sl_indices, const int32_t *sl_offsets, int32_t count,
	const double *weights,
	const int32_t *indptr, const int32_t *indices, int64_t nnz, double *data,
	bool isReflection, bool isScaling, bool col_major);

/*
 * Flattened form of ha_searchlight_ridge (csrc/ha_searchlight.h:86-90,
 * csrc/ha_searchlight.c:1378-1429; local solve ha_ridge, csrc/ha_ridge.c:13-54):
 * beta_s = V diag(s / (alpha + s^2)) U^T Y_s with X_s = U diag(s) V^T, scattered
 * like the Procrustes call above.  Computed in float64.
 */
int ha_searchlight_ridge_csc_b200(
	const double *X_data, const double *Y_data, int32_t nt, int32_t nv,
	const int32_t *sl_indices, const int32_t *sl_offsets, int32_t count,
	const double *weights,
	const int32_t *indptr, const int32_t *indices, int64_t nnz, double *data,
	double alpha, bool col_major);

/*
 * Searchlight ridge grid search with cross-validated ensembles: the reference's ha_ridge_grid
 * (csrc/ha_ridge.c:97-227) inside ha_ensemble_ridge (csrc/ha_ridge.c:229-345), applied to every
 * searchlight with X_s = X[:, sl] and the n_s targets Y[:, sl].  For every CV model m the grid of
 * betas over alphas x PC counts is fitted on the training rows train_idx_li[m] (train_sizes[m]
 * rows, duplicates kept); every tested row averages the predictions of the models that test it,
 * and the cost of a grid point is the squared prediction error over all rows, SUMMED OVER THE
 * TARGETS of the searchlight, so each searchlight gets one winner: the first grid index
 * g = a * n_npcs + p with the smallest cost (best_out[s], int32 per searchlight).  The winner's
 * model-averaged beta (n_s x n_s) is scattered like ha_searchlight_ridge_csc_b200.  PC chunks
 * follow the reference: [npcs[p-1], npcs[p]) clipped at min(train rows, n_s), summed over p.
 * cost_out (count x n_alphas x n_npcs float64, may be NULL) receives every grid cost.
 * Computed in float64 (eigen decomposition of X_tr^T X_tr by Jacobi rotations).  kHaErrorArg for
 * negative PC counts, non-finite alphas, empty training lists, rows outside [0, nt), a row
 * repeated within one test list, or a searchlight of more than 512 vertices.
 */
int ha_searchlight_ridge_grid_b200(
	const double *X_data, const double *Y_data, int32_t nt, int32_t nv,
	const int32_t *sl_indices, const int32_t *sl_offsets, int32_t count,
	const double *weights,
	const int32_t *indptr, const int32_t *indices, int64_t nnz, double *data,
	const double *alphas, int32_t n_alphas, const int32_t *npcs, int32_t n_npcs,
	const int32_t *const *train_idx_li, const int32_t *const *test_idx_li,
	const int32_t *train_sizes, const int32_t *test_sizes, int32_t n_models,
	int32_t *best_out, double *cost_out, bool col_major);

/*
 * CV split indices, the same draws as ha_ensemble_indices (csrc/ha_ensemble.h,
 * csrc/ha_ensemble.c:58-249: xoshiro256** seeded by splitmix64, shuffled blocks dealt to folds,
 * bootstrap training rows outside the test blocks' buffers, test rows outside the training rows'
 * buffers, optional mask with index remapping), into caller buffers: split k = perm * n_folds +
 * fold has nt training rows at train_out[k * nt] and test_sizes[k] test rows at test_out[k * nt]
 * (both buffers n_perms * n_folds * nt int32).  kHaErrorArg where the reference would read
 * uninitialised memory (a fold without training rows) or divide by zero (blocksize < 1).
 */
int ha_ensemble_indices_b200(
	int32_t nt, int32_t n_perms, int32_t n_folds, int32_t blocksize, int32_t buffersize,
	uint64_t seed, const bool *mask,
	int32_t *train_out, int32_t *test_out, int32_t *test_sizes);

/*
 * Searchlight Procrustes template (the loop of ha_template_procrustes, csrc/ha_template.c:14-114,
 * with every whole-matrix Procrustes replaced by a searchlight solve and aligned = X @ T taken
 * as a sparse product over the searchlight pattern):
 *   common = X_0; for s = 1..n_subj-1: T = SL(X_s -> common), A_s = X_s @ T, [zscore A_s],
 *   common = (common + A_s) / 2, [zscore common];
 *   level2_iter times: sum = sum_s A_s; for s: ref = (sum - A_s) / (n_subj - 1), [zscore ref],
 *   A_s = X_s @ SL(X_s -> ref);
 *   tpl = sum_s A_s, then zscore (isZscoreCommon) or / n_subj.
 * dms: n_subj consecutive nt x nv float64 column-major matrices (host); tpl_out: nt x nv
 * float64 column-major (host, overwritten).  Searchlights, weights and flags as in
 * ha_searchlight_procrustes_dense; z-scores use the one-pass rule of ha_zscore_columns
 * (csrc/ha_linalg.c:263-291).
 */
int ha_searchlight_template_b200(
	const double *dms, int32_t n_subj, int32_t nt, int32_t nv,
	const int32_t *sl_indices, const int32_t *sl_offsets, const double *sl_dists,
	int32_t count, double radius,
	bool isReflection, bool isScaling, bool isZscoreCommon, int32_t level2_iter,
	double *tpl_out);

/*
 * Searchlight PCA template: replaces searchlight_template(..., tpl_kind="pca") of the Python
 * package (src/hyperalignment/searchlight.py:215-236 with compute_template(kind="pca",
 * max_npc=n, common_topography=True, demean=False), src/hyperalignment/local_template.py:224-248,
 * :72-78, :11-53).  Per searchlight (n vertices sl): X = [dms_1[:, sl] .. dms_ns[:, sl]];
 * tmpl = U_n S_n / sqrt(n_subj) from the top n singular pairs of X; R = polar(tmpl^T sum_s
 * dms_s[:, sl]) (reflection allowed, no scaling); tpl_out[:, sl] += (tmpl R) diag(w) with the
 * searchlight weights of sl_dists and radius (ha_compute_weights).  The singular pairs are exact
 * (float64 Gram of the smaller side, eigen decomposition by Jacobi rotations): they agree with the
 * reference's randomized SVD where the top-n singular subspace is separated from the rest.
 * dms: n_subj consecutive nt x nv float64 column-major matrices (host); tpl_out: nt x nv float64
 * column-major (host, overwritten).  kHaErrorArg when a searchlight holds more than nt vertices
 * or min(nt, n_subj * n) exceeds 512.
 */
int ha_searchlight_pca_template_b200(
	const double *dms, int32_t n_subj, int32_t nt, int32_t nv,
	const int32_t *sl_indices, const int32_t *sl_offsets, const double *sl_dists,
	int32_t count, double radius, double *tpl_out);

/* ---- device-resident plan (repeated calls on one searchlight geometry) ---- */

typedef struct HaB200Plan HaB200Plan;

/* Output kinds of a plan run. */
enum {
	kHaB200OutCSR = 0, /* values in row order of the symmetric pattern (row r = dense row r) */
	kHaB200OutCSC = 1, /* values in CSC order (the layout of ha_sparse_init) */
};

/* Solver variants. */
enum {
	kHaB200SolverMixed = 0, /* FP32 Jacobi + FP32 Newton-Schulz refinement, FP64 re-solve of searchlights
	                           with sigma_min / sigma_max < 5e-5 (environment HA_B200_ILL_RATIO overrides) */
	kHaB200SolverFP32  = 1, /* plain FP32 form: FP32 Jacobi only, no refinement, no FP64 re-solve */
	kHaB200SolverFP64  = 2, /* every searchlight in FP64 */
	kHaB200SolverTC    = 3, /* tensor cores: split-BF16 (three parts, six products, FP32 accuracy)
	                           cross-covariance and Newton-Schulz polar iteration; exactly singular A
	                           get their null spaces completed, and searchlights that still do not
	                           converge are re-solved by FP64 Jacobi.  Needs isReflection; without it
	                           the mixed solver runs. */
};

/*
 * Uploads the searchlight geometry and builds on the GPU everything that
 * depends only on it: weights (as ha_searchlight_procrustes_dense when
 * weights == NULL, else the caller's), per-vertex membership lists, the
 * symmetric CSC pattern, size buckets and scratch layout.
 */
int ha_b200_plan_create(
	int32_t nt, int32_t nv,
	const int32_t *sl_indices, const int32_t *sl_offsets, const double *sl_dists,
	int32_t count, double radius, const double *weights,
	HaB200Plan **plan_out);
void ha_b200_plan_destroy(HaB200Plan *plan);
/* Number of stored entries of the pattern, and a host copy of it (indptr: nv + 1 int64). */
int64_t ha_b200_plan_nnz(const HaB200Plan *plan);
int ha_b200_plan_pattern(const HaB200Plan *plan, int64_t *indptr, int32_t *indices);
/* Device pointer to the plan's per-vertex pattern (indptr int64 nv+1, indices int32 nnz). */
int ha_b200_plan_device_pattern(const HaB200Plan *plan, const int64_t **d_indptr, const int32_t **d_indices);
/* Searchlights of the last run that were solved in FP64, and that hit the sweep limit. */
int ha_b200_plan_stats(const HaB200Plan *plan, int32_t *n_fp64, int32_t *n_jacobi_unconverged);
/* Jacobi sweeps of the last run: sum over searchlights (final solve of each) and maximum. */
int ha_b200_plan_sweep_stats(const HaB200Plan *plan, int64_t *sweeps_sum, int32_t *sweeps_max);
/*
 * Per-searchlight solve record of the last run, searchlights [first, first + n) of its last
 * chunk: smallest and largest singular value, flags (1 unconverged, 2 ill-conditioned,
 * 4 reflection removed, 8 solved in FP64, 16 zero singular values completed after the tensor-core
 * iteration) and Jacobi sweeps (tensor-core solver: Newton-Schulz iterations; its sigma_max is
 * the upper bound the iterate was scaled by and sigma_min is not computed, 0).  Any output may
 * be NULL.
 */
int ha_b200_plan_searchlight_stats(const HaB200Plan *plan, int32_t first, int32_t n, double *s_min,
                                   double *s_max, int32_t *flags, int32_t *sweeps);

/*
 * Searchlight Procrustes on device-resident data.  d_X, d_Y: nt x nv float64
 * in DEVICE memory, column-major (vertex j's time series contiguous).
 * d_values: DEVICE float64 array of plan nnz entries, accumulated (+=) in the
 * order given by out_kind.  stream: a cudaStream_t, or NULL for the legacy
 * default stream.  Returns after enqueueing; synchronise the stream to read.
 */
int ha_b200_plan_procrustes_device(
	HaB200Plan *plan, const double *d_X, const double *d_Y,
	bool isReflection, bool isScaling, int solver, int out_kind,
	double *d_values, void *stream);

/* Ridge on device-resident data (same conventions), computed in float64. */
int ha_b200_plan_ridge_device(
	HaB200Plan *plan, const double *d_X, const double *d_Y, double alpha,
	int out_kind, double *d_values, void *stream);

/*
 * Ridge grid search on device-resident data (conventions of ha_b200_plan_ridge_device; grid and
 * CV lists in host memory as ha_searchlight_ridge_grid_b200).  d_best (count int32) and d_cost
 * (count x n_alphas x n_npcs float64, may be NULL) are DEVICE memory, overwritten.
 */
int ha_b200_plan_ridge_grid_device(
	HaB200Plan *plan, const double *d_X, const double *d_Y,
	const double *alphas, int32_t n_alphas, const int32_t *npcs, int32_t n_npcs,
	const int32_t *const *train_idx_li, const int32_t *const *test_idx_li,
	const int32_t *train_sizes, const int32_t *test_sizes, int32_t n_models,
	int out_kind, double *d_values, int32_t *d_best, double *d_cost, void *stream);

/*
 * Arithmetic of this plan's ridge grid search and learned form.  bits 64 (the default) computes
 * every Gram, factor, eigen decomposition, prediction and cost in float64.  bits 32 is the plain
 * FP32 form: float32 Gram and cross-covariance over the rows, pivoted Cholesky, eigenvector-mode
 * Jacobi, per-model products, predictions and costs in ha_b200_plan_ridge_grid_device, and the
 * float32 eigen solve, features, proposal fit and fallback grid in
 * ha_b200_plan_ridge_learned_device and ha_b200_plan_ridge_features_device.  The inputs, the
 * winners' betas and the reduction stay float64.  It is the same composition of ha_ridge_grid and
 * ha_ensemble_ridge (csrc/ha_ridge.c:97-345).  Its costs carry float32 rounding: grid points whose
 * costs differ by less than about 1e-5 relative can pick another winner, and at the smallest
 * alphas of searchlights with more vertices than distinct training rows the cost of a losing grid
 * point can be far off (the rounding of V^T C on near-null components, amplified by 1 / alpha).
 * The host entry ha_searchlight_ridge_grid_b200 stays float64.  Returns kHaErrorArg for other
 * values of bits.
 */
int ha_b200_plan_set_grid_precision(HaB200Plan *plan, int32_t bits);

/*
 * Per-searchlight local transforms of the last device run, for testing:
 * copies T_s (n_s x n_s, float32, unweighted and unscaled; row-major after a
 * CSR-ordered run, column-major after a CSC-ordered one) of searchlights
 * [first, first + n) into host out (sum of n_s^2 floats).
 */
int ha_b200_plan_local_transforms(const HaB200Plan *plan, int32_t first, int32_t n, float *out);

/* ---- local Procrustes without allocation ---- */

/*
 * No counterpart in the reference.  For callers that cannot allocate device memory (their own
 * pool allocator owns the GPU, or their host program forbids new allocations, or the
 * device-wide synchronisation of cudaMalloc/cudaFree is not acceptable in their loop): computes
 * the local transforms T_s (the unscaled, unweighted polar factors of X[:, sl]^T Y[:, sl],
 * reflection allowed, plain FP32 Jacobi) of searchlights of at most kHaB200NoAllocMaxSize vertices
 * and writes them packed, row-major, searchlight after searchlight, to d_T_out (float32, sum of
 * n_s^2 entries).  d_X, d_Y (nt x nv float64, column-major), d_sl_indices and d_T_out are DEVICE
 * memory owned by the caller; sl_offsets (count + 1 entries) is host memory.
 *
 * The only scratch is a static 64 MiB device array inside this library, held by every GPU that
 * loads it until the process exits; the call allocates nothing.  The first call on a device
 * looks up that array's address and raises kernel shared-memory limits; make it before any
 * stream capture.  All calls share the array: calls that overlap on the GPU (from other host
 * threads or other streams) race.  Returns after the work on `stream` is finished;
 * kHaErrorArg for a searchlight size outside 1..kHaB200NoAllocMaxSize (checked before any work)
 * or a vertex index outside [0, nv) (checked on the device).
 */
#define kHaB200NoAllocMaxSize 160
#define kHaB200NoAllocScratchBytes (64u << 20)
int ha_b200_local_procrustes_noalloc(
	const double *d_X, const double *d_Y, int32_t nt, int32_t nv,
	const int32_t *d_sl_indices, const int32_t *sl_offsets, int32_t count,
	float *d_T_out, void *stream);

/* ---- learned (alpha, PC count) proposal ---- */

/*
 * No reference counterpart.  A perceptron 65 -> 128 GELU -> 128 GELU -> n_classes (softmax) that
 * proposes the grid point (g = a * n_npcs + p) of a searchlight from its features (the 64 largest
 * singular values of the searchlight's training block divided by the largest, zero-padded, and
 * log n; ha_b200_plan_ridge_features_device).  Parameters: float32, packed W1[65][128], b1[128],
 * W2[128][128], b2[128], W3[128][C], b3[C], in DEVICE memory.  Features: DEVICE float32 [n][65];
 * labels DEVICE int32 [n] in 0..C-1.  C at most 64.
 */
int64_t ha_b200_mlp_param_count(int32_t n_classes);
/* Uniform(+-1/sqrt(fan_in)) initialisation from a SplitMix64 stream (seed). */
int ha_b200_mlp_init(float *d_params, int32_t n_classes, uint64_t seed);
/* Gradient (d_grad, DEVICE) and value (loss_out, host) of the mean cross-entropy over n samples. */
int ha_b200_mlp_grad(const float *d_params, int32_t n_classes, const float *d_x, const int32_t *d_y, int32_t n,
                     float *d_grad, float *loss_out);
/* Adam (0.9, 0.999, 1e-8) over shuffled mini-batches for epochs passes; final mean loss if asked. */
int ha_b200_mlp_train(float *d_params, int32_t n_classes, const float *d_x, const int32_t *d_y, int32_t n,
                      int32_t epochs, int32_t batch, float lr, uint64_t seed, float *final_loss);
/* bfloat16 inference: most probable class (ties to the lower index) and its probability (DEVICE). */
int ha_b200_mlp_infer(const float *d_params, int32_t n_classes, const float *d_x, int32_t n, int32_t *d_class,
                      float *d_prob, void *stream);

/*
 * Features of every searchlight of the plan for the perceptron: the 64 largest singular values of
 * X[rows, sl] divided by the largest (zero-padded) and log n, d_features DEVICE float32
 * [count][65].  rows: host int32 list (duplicates allowed) of time points in [0, nt).
 */
int ha_b200_plan_ridge_features_device(HaB200Plan *plan, const double *d_X, const int32_t *rows, int32_t n_rows,
                                       float *d_features, void *stream);
/*
 * The learned form of the ridge grid search.  Per searchlight: the features over the fit rows, the
 * perceptron's proposed grid point g and its probability (d_choice, d_prob: DEVICE, count
 * entries); where the probability is at least min_prob, ha_ridge_grid's beta at g fitted on the
 * rows (csrc/ha_ridge.c:97-227 restricted to one grid point, all targets of the searchlight);
 * below it, the full CV grid search of ha_searchlight_ridge_grid_b200 (its winner replaces
 * d_choice).  Betas are scattered into d_values like the other plan runs.
 */
int ha_b200_plan_ridge_learned_device(
	HaB200Plan *plan, const double *d_X, const double *d_Y, const int32_t *rows, int32_t n_rows,
	const double *alphas, int32_t n_alphas, const int32_t *npcs, int32_t n_npcs,
	const float *d_params, float min_prob,
	const int32_t *const *train_idx_li, const int32_t *const *test_idx_li,
	const int32_t *train_sizes, const int32_t *test_sizes, int32_t n_models,
	int out_kind, double *d_values, int32_t *d_choice, float *d_prob, void *stream);

/* ---- evaluation ---- */

/*
 * Vertex-wise correlation of aligned data with a target: the evaluation step of the reference's
 * benchmark (benchmark_neuroboros.py:204-211, the mean over time of zscore(A) * zscore(Y) per
 * vertex with scipy's population z-score; benchmark_neuroboros.py:229-232 forms A = X @ W).
 * A = X @ W for W in CSC form (d_indptr: nv + 1 int64, d_indices: nnz int32 rows, d_values: nnz
 * float64, e.g. a plan's device pattern and the values of a kHaB200OutCSC run), or A = X when
 * d_values is NULL (the unaligned correlation).  d_X, d_Y: nt x nv float64 column-major DEVICE
 * memory.  d_r: nv float64 DEVICE memory, overwritten; a column with zero variance gives NaN, as
 * the z-score does, and so does a column whose pattern entries are out of range (indptr outside
 * [0, nnz] or decreasing, a row outside [0, nv)).  d_aligned (nt x nv float64 DEVICE, may be NULL)
 * receives A.  Returns after enqueueing on stream (a cudaStream_t, or NULL).
 */
int ha_b200_aligned_correlation_device(
	const double *d_X, const double *d_Y, int32_t nt, int32_t nv,
	const int64_t *d_indptr, const int32_t *d_indices, const double *d_values, int64_t nnz,
	double *d_r, double *d_aligned, void *stream);

/* ---- tracing ---- */

/* Kernel kinds reported by ha_b200_kernel_times. */
enum {
	kHaB200KConvert = 0,    /* float64 -> float32 vertex-major restage */
	kHaB200KColVar = 1,     /* per-vertex population variance (scaling) */
	kHaB200KXcov32 = 2,     /* cross-covariance, float32 */
	kHaB200KJacobi32 = 3,   /* Jacobi polar, float32 */
	kHaB200KFormT32 = 4,    /* T = U V^T for blocked float32 searchlights */
	kHaB200KXcov64 = 5,
	kHaB200KJacobi64 = 6,
	kHaB200KFormT64 = 7,
	kHaB200KRefine = 8,     /* Newton-Schulz orthogonality refinement */
	kHaB200KReflect = 9,    /* det(T) < 0 fix */
	kHaB200KScale = 10,     /* per-searchlight scale / bookkeeping */
	kHaB200KReduce = 11,    /* deterministic segmented reduction */
	kHaB200KPattern = 12,   /* CSC pattern builder */
	kHaB200KRidge = 13,     /* ridge solves, pivoted Cholesky factors of the grid */
	kHaB200KGrid = 14,      /* ridge grid: per-model products and grid evaluation */
	kHaB200KMlp = 15,       /* learned proposal: training and inference */
	kHaB200KEval = 16,      /* vertex-wise correlation of aligned data with a target */
	kHaB200KTcXcov = 17,    /* cross-covariance on the tensor cores (split BF16) */
	kHaB200KTcNs = 18,      /* Newton-Schulz polar iteration on the tensor cores */
	kHaB200KPca = 19,       /* searchlight PCA template: Gram, eigen, template, polar, reduction */
	kHaB200NumKernelKinds = 20,
};

/*
 * When on, every kernel launch of this library is bracketed by CUDA events on its
 * stream; ha_b200_kernel_times synchronises those events and returns (and resets), per
 * kind, the device milliseconds during which at least one launch of that kind ran (the
 * union of the launch intervals: launches of independent size buckets run on side streams
 * and overlap) and the launch counts.
 */
void ha_b200_set_kernel_timing(bool on);
int ha_b200_kernel_times(double *ms, int64_t *launches);
/* Kernels launched by this library since it was loaded. */
int64_t ha_b200_launch_count(void);

/*
 * Tile layout of the tensor-core solver's per-phase launches, per size class (tiles of at most 128
 * columns; of 129-256): shared memory per CTA in KB, which sets the CTAs per SM and the pipeline
 * depth.  Class 0 candidates: 110, 72, 53 KB (2, 3, 4 CTAs per SM); class 1: 110, 200 KB (2, 1).
 * The plan's first tensor-core run times one Gram launch per candidate with CUDA events and keeps
 * the fastest (environment HA_B200_AUTOTUNE=0 keeps 110 / 110 instead); every layout gives the same
 * results bit for bit.  cand_ms (6 doubles, may be NULL) receives the measured times (0 = not
 * timed); tuned is 1 once a layout was chosen or pinned.  set_tc_layout pins one.
 */
int ha_b200_plan_tc_layout(const HaB200Plan *plan, int32_t *smem_kb, int32_t *tuned, double *cand_ms);

/*
 * Repeated launch sequences (the tensor-core iteration of a plan chunk, the ridge grid search of a
 * plan) are captured once into CUDA graphs and replayed; off, they are launched one by one.  On by
 * default (environment HA_B200_GRAPHS=0 turns it off); the results are the same bit for bit.
 */
void ha_b200_set_graphs(bool on);
int ha_b200_plan_set_tc_layout(HaB200Plan *plan, const int32_t *smem_kb);

/*
 * Diagnostic: one tensor-core product of the Newton-Schulz solver's kernels on host data, FP32
 * row-major n x n output (n <= 512).  which 0: h_a^T h_a (h_a row-major n x n); which 1:
 * h_a h_b (both row-major n x n); which 2: the cross-covariance h_a h_b^T of two n x nt
 * vertex-major matrices (h_a[j * nt + t], vertex j's series contiguous).  Checks the operand
 * layouts of every product type.
 */
int ha_b200_tc_selftest(int32_t which, int32_t n, int32_t nt, const float *h_a, const float *h_b, float *h_out);

#ifdef __cplusplus
}
#endif

#endif /* HYPERALIGNMENT_B200_H */
