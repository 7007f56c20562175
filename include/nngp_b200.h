/*
 * nngp_b200.h — C ABI of the B200 (sm_100a) NNGP fit/predict hot path.
 *
 * One shared library, libnngp_b200.so, replaces the numerical layers that the
 * reference nngpr (stavoltafunzia/nngpr 0.1.1) runs per batch:
 *
 *   - the kernel-space nearest-neighbour search
 *       NngprWorker.find_nearest_neighbors        nngpr/base_nngpr.py:1613-1686
 *       RbfAccelerator.find_nearest_neighbors     nngpr/cuda_kernel_accelerators.py:196-381
 *       calc_nn (CUDA)                            nngpr/cuda_kernel_accelerators.py:663-743
 *   - the local covariance fill, batched Cholesky, solves and the log-likelihood
 *     reduction with its gradient
 *       Nngpr._log_likelihood_worker              nngpr/base_nngpr.py:453-614
 *       RbfAccelerator.fill_nn_kernel             nngpr/cuda_kernel_accelerators.py:383-518, 748-863
 *       TorchWorker.batched_chofactor/chosolve    nngpr/torch_nngpr.py:294-300
 *   - the predictive mean / standard deviation conditioned on the training set
 *       Nngpr._predict_worker                     nngpr/base_nngpr.py:1032-1135
 *
 * Conventions
 *   - Every array argument is a DEVICE pointer owned by the caller, except the
 *     length_scale arrays and the nngp_kernel struct, which are read on the host
 *     during the call.  Row-major, contiguous.
 *   - Every call is stream ordered on `stream` (a cudaStream_t passed as void*;
 *     NULL = legacy default stream) and returns before the GPU work finishes.
 *     Results and the device status word are valid after the stream reaches them.
 *   - Calls return an nngp_status; nothing traps or aborts.  The text of the last
 *     error of the calling thread is returned by nngp_last_error().
 *   - Scratch memory is caller provided (`workspace`, `workspace_bytes`); the
 *     *_workspace_size functions return the bytes a call needs.  The library
 *     allocates no device memory.
 *   - Conditions that only the GPU can see (a neighbour index out of range, a
 *     non-positive pivot, a wait that ran out of time) are OR-ed into the optional
 *     device int32 `status_flags` (NNGP_FLAG_*), never trapped.
 *   - Calls on different streams may run concurrently if their workspaces differ.
 */
#ifndef NNGP_B200_H
#define NNGP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NNGP_ABI_VERSION 3

typedef enum nngp_status {
    NNGP_OK = 0,
    NNGP_ERR_INVALID_ARGUMENT = 1, /* bad size, null pointer, misaligned buffer */
    NNGP_ERR_UNSUPPORTED = 2,      /* a size this build does not handle (message says which) */
    NNGP_ERR_WORKSPACE = 3,        /* workspace missing or smaller than *_workspace_size */
    NNGP_ERR_CUDA = 4,             /* a CUDA runtime call failed (message carries its text) */
    NNGP_ERR_NO_DEVICE = 5         /* no usable sm_100 device is current */
} nngp_status;

/* Bits OR-ed into the device status word by the kernels. */
#define NNGP_FLAG_BAD_INDEX 1      /* a neighbour index outside [0, n) was treated as missing (-1) */
#define NNGP_FLAG_NOT_PD 2         /* a local system had a non-positive pivot: its terms are NaN */
#define NNGP_FLAG_TIMEOUT 4        /* a bounded wait inside a kernel gave up; results are invalid */
#define NNGP_FLAG_FP64_FALLBACK 8  /* some FP32 systems were re-solved in FP64 (informational) */

/*
 * Kernel  k(a, b) = rbf_level * s(r) + const_value + noise_level * [a is b],
 * r^2 = sum_f (a_f - b_f)^2 / l_f^2, with the stationary part s chosen by `family`:
 * NNGP_FAMILY_RBF s = exp(-r^2 / 2) -- the WhiteKernel + ConstantKernel + ConstantKernel*RBF
 * family that the reference accelerates on CUDA (nngpr/cuda_kernel_accelerators.py:169-194,
 * parameters from get_kernel_params :520-581) -- or the Matern kernels the reference
 * evaluates on its generic path (nngpr/batched_kernels.py:1070-1131): nu = 1/2
 * s = exp(-r); nu = 3/2 s = (1 + sqrt3 r) exp(-sqrt3 r); nu = 5/2
 * s = (1 + sqrt5 r + 5 r^2 / 3) exp(-sqrt5 r).  `alpha` is the GaussianProcessRegressor jitter added to
 * every valid diagonal slot (base_nngpr.py:555-556; training slots only in predict,
 * :1106-1107).  The idx_* fields give the position of each free hyperparameter in
 * kernel.theta (get_kernel_theta_mapping, :583-649), -1 when fixed or absent; the
 * n_ls length-scale positions are idx_ls, idx_ls+1, ...  Gradients are with respect
 * to these log-hyperparameters.
 *
 * dev_params (may be NULL): a DEVICE block that nngp_theta_params filled from a device theta;
 * the log-likelihood calls then take the hyperparameter values from it instead of the fields
 * above (the structure -- idx_*, n_ls, family, alpha -- still comes from this struct), so a fit
 * loop can keep theta on the device.
 */
typedef struct nngp_kernel {
    double rbf_level;
    double const_value;
    double noise_level;
    double alpha;
    const double *length_scale; /* HOST pointer: n_ls values, 1 (isotropic) or d (ARD) */
    int32_t n_ls;               /* 0 = no stationary term (rbf_level must then be 0) */
    int32_t idx_rbf_level;
    int32_t idx_const;
    int32_t idx_noise;
    int32_t idx_ls;
    int32_t n_theta;
    int32_t family;             /* NNGP_FAMILY_* (0 = RBF) */
    const double *dev_params;   /* DEVICE pointer or NULL: see nngp_theta_params */
} nngp_kernel;

#define NNGP_FAMILY_RBF 0
#define NNGP_FAMILY_MATERN12 1
#define NNGP_FAMILY_MATERN32 2
#define NNGP_FAMILY_MATERN52 3

/* ---------------------------------------------------------------------------------------
 * Library information
 * ------------------------------------------------------------------------------------- */
int32_t nngp_abi_version(void);
/* Text of the last failed call on this thread ("" if none). */
const char *nngp_last_error(void);
const char *nngp_status_string(nngp_status status);
/* NNGP_OK if the current device is an sm_100 part this build runs on. */
nngp_status nngp_check_device(void);

/* Failure-path testing (no counterpart in the reference): the time limit, in nanoseconds of the
 * GPU's global timer, of the bounded waits in the tensor-core search's main loop (default 2 s;
 * 0 restores the default).  A wait that runs out raises NNGP_FLAG_TIMEOUT and the kernel returns
 * after draining the copies and MMAs it issued (those drains always use the 2 s default), so a
 * tiny limit turns a search into a clean, flagged failure whose results are invalid, and the next
 * call with the default limit runs normally.  Process-wide; returns the previous limit. */
uint64_t nngp_set_wait_limit_ns(uint64_t ns);

/* ---------------------------------------------------------------------------------------
 * Nearest-neighbour search
 *
 * Replaces NngprWorker.find_nearest_neighbors (base_nngpr.py:1613-1686) and the CUDA
 * calc_nn search (cuda_kernel_accelerators.py:196-381, 663-743).
 *
 * out_idx[q, k] (n_query x num_nn, int32) = index in `ref` of the k-th nearest ref of
 * query q, ascending by squared distance of the scaled points x / length_scale
 * (length_scale == NULL: input-space search, plain Euclidean), equal distances ordered
 * by lower index, -1 for missing slots.  With has_ref_cut != 0 query q only considers
 * refs [0, q + ref_cut_index) (the reference's ref_cut_index; the fit step uses
 * ref = query = X and ref_cut_index = 0, i.e. strictly earlier points in input order);
 * otherwise every ref.  Distances are evaluated in the input precision with one rounding
 * per operation, so the lists equal those of an exact search in that precision.
 *
 * The fit step's search of a set over itself (ref == query, n_ref == n_query, has_ref_cut with
 * ref_cut_index 0, FP32, n >= 8,192) starts every row from a proven bound of its num_nn-th
 * distance (Morton-window seeds) and, for d <= 24 and 65,536 <= n <= 2,000,000, visits per group
 * of rows only the ref tiles bounding boxes cannot exclude; the lists are the same.
 * A search of other queries without a cut (predict: n_ref >= 8,192, n_query >= 16,384) seeds
 * every query from the refs' curve windows around it and, for d <= 24, prunes the same way.
 * NNGP_KNN_SEED_W=0 / NNGP_KNN_PRUNE=0 switch these off (testing).  The workspace covers them.
 * ------------------------------------------------------------------------------------- */
size_t nngp_knn_workspace_size_f32(int64_t n_ref, int64_t n_query, int32_t d, int32_t num_nn);
nngp_status nngp_knn_f32(const float *ref, int64_t n_ref, const float *query, int64_t n_query,
                         int32_t d, const double *length_scale, int32_t n_ls, int32_t num_nn,
                         int32_t has_ref_cut, int64_t ref_cut_index, int32_t *out_idx,
                         int32_t *status_flags, void *workspace, size_t workspace_bytes,
                         void *stream);
/* nngp_knn_f32 / _f64 with the length scale (n_ls values, 1 or d) in DEVICE memory, e.g. the block
 * of nngp_theta_params (a fit loop that keeps theta on the device). */
nngp_status nngp_knn_f32_ls_device(const float *ref, int64_t n_ref, const float *query, int64_t n_query,
                                   int32_t d, const double *length_scale_dev, int32_t n_ls, int32_t num_nn,
                                   int32_t has_ref_cut, int64_t ref_cut_index, int32_t *out_idx,
                                   int32_t *status_flags, void *workspace, size_t workspace_bytes,
                                   void *stream);
nngp_status nngp_knn_f64_ls_device(const double *ref, int64_t n_ref, const double *query, int64_t n_query,
                                   int32_t d, const double *length_scale_dev, int32_t n_ls, int32_t num_nn,
                                   int32_t has_ref_cut, int64_t ref_cut_index, int32_t *out_idx,
                                   int32_t *status_flags, void *workspace, size_t workspace_bytes,
                                   void *stream);
size_t nngp_knn_workspace_size_f64(int64_t n_ref, int64_t n_query, int32_t d, int32_t num_nn);
nngp_status nngp_knn_f64(const double *ref, int64_t n_ref, const double *query, int64_t n_query,
                         int32_t d, const double *length_scale, int32_t n_ls, int32_t num_nn,
                         int32_t has_ref_cut, int64_t ref_cut_index, int32_t *out_idx,
                         int32_t *status_flags, void *workspace, size_t workspace_bytes,
                         void *stream);

/* Neighbour-list reuse across fit steps (isotropic or no length scale, FP32 search): the
 * reference recomputes the fit step's search on every log-likelihood call (base_nngpr.py:532);
 * an isotropic length scale only rescales every distance, so the lists can change only through
 * FP32 rounding.  With n_cand > num_nn candidates per point from one prefix search
 * (nngp_knn_f32, ref_cut_index 0, at length scale l0, ascending), nngp_knn_reuse_prepare_f32
 * stores per point the normalised distance of its last candidate minus twice a rounding bound,
 * 2 (d + 6) 2^-24 (|x_i| + max_norm)^2 (max_norm >= every row's 2-norm); nngp_knn_reuse_rank_f32
 * then ranks the candidates at a new length scale l in the search's exact arithmetic and writes
 * the top num_nn.  A point whose num_nn-th distance l^2 D is not below its threshold is counted
 * in *n_failed (device int, accumulated): only when *n_failed stays 0 are the lists proven equal
 * to nngp_knn_f32's at l; otherwise run the full search.  x: the unscaled FP32 points (n, d);
 * n_cand <= 64, num_nn <= 32. */
nngp_status nngp_knn_reuse_prepare_f32(const float *x, int64_t n, int32_t d, double length_scale,
                                       const int32_t *cand, int32_t n_cand, double max_norm, double *thr,
                                       void *stream);
nngp_status nngp_knn_reuse_rank_f32(const float *x, int64_t n, int32_t d, double length_scale,
                                    const int32_t *cand, int32_t n_cand, const double *thr,
                                    int32_t num_nn, int32_t *out_idx, int32_t *n_failed, void *stream);

/* ---------------------------------------------------------------------------------------
 * Log-likelihood (+ gradient) of the fit step
 *
 * Replaces the per-batch arithmetic of Nngpr._log_likelihood_worker (base_nngpr.py:538-614)
 * together with fill_nn_kernel (cuda_kernel_accelerators.py:383-518) and the batched
 * Cholesky / solves (torch_nngpr.py:294-300, numpy_nngpr.py:140-170).
 *
 * x (n x d), y (n x ydim), nbr (n x m, int32, -1 = missing; the point itself is implicit,
 * it is NOT a column of nbr).  out[0] = sum over points and outputs of
 *   -0.5 (y - mu)^2 / sigma^2 - 0.5 log(2 pi) - log(sigma)       (base_nngpr.py:581)
 * and, if eval_gradient, out[1 + t] = d out[0] / d theta_t for t < kernel->n_theta
 * (base_nngpr.py:586-614).  out is a device double array, written (not accumulated).
 * The f32 entry point computes each local system in FP32 and re-solves it in FP64 when a
 * pivot falls below pivot_tol * (rbf_level + const_value + noise_level + alpha); the
 * per-point terms are summed in FP64.  The f64 entry point computes in FP64 throughout
 * (pivot_tol is ignored).
 * ------------------------------------------------------------------------------------- */
size_t nngp_loglik_workspace_size(int64_t n, int32_t d, int32_t ydim, int32_t m, int32_t n_theta);
nngp_status nngp_loglik_f32(const float *x, const float *y, int64_t n, int32_t d, int32_t ydim,
                            const int32_t *nbr, int32_t m, const nngp_kernel *kernel,
                            int32_t eval_gradient, double pivot_tol, double *out,
                            int32_t *status_flags, void *workspace, size_t workspace_bytes,
                            void *stream);
nngp_status nngp_loglik_f64(const double *x, const double *y, int64_t n, int32_t d, int32_t ydim,
                            const int32_t *nbr, int32_t m, const nngp_kernel *kernel,
                            int32_t eval_gradient, double pivot_tol, double *out,
                            int32_t *status_flags, void *workspace, size_t workspace_bytes,
                            void *stream);

/*
 * How many local systems the last nngp_loglik_f32 / nngp_loglik_rows_f32 call given `workspace`
 * re-solved in FP64 (the count behind NNGP_FLAG_FP64_FALLBACK; 0 after an f64 call): the DEVICE
 * address of an unsigned 64-bit counter inside the workspace, valid once the stream has reached
 * the end of that call and until the workspace is used again.  No counterpart in the reference
 * (its FP32 mode has no FP64 re-solve); a host-only function, no GPU work.
 */
const uint64_t *nngp_loglik_fp64_count(const void *workspace);

/*
 * Hyperparameter values from a DEVICE theta (log-hyperparameters, the layout of kernel.theta)
 * without a host round trip: writes NNGP_THETA_PARAMS_LEN(d) doubles at params_dev (device),
 * [rbf_level, const_value, noise_level, pivot_abs, 1/l_0 .. 1/l_{d-1}, l_0 .. l_{d-1}], each free
 * hyperparameter exp of its theta entry (Kernel.theta's map, get_kernel_theta_mapping,
 * nngpr/base_nngpr.py:583-649; sklearn's clone_with_theta), fixed ones and the structure from
 * *k; pivot_abs = pivot_tol * |rbf_level + const_value + noise_level + alpha| (the FP32 re-solve
 * threshold).  Set k->dev_params = params_dev for nngp_loglik_* and pass params_dev + 4 + d as
 * the DEVICE length scale of nngp_knn_f32_ls_device.  Stream-ordered, one small kernel.
 */
#define NNGP_THETA_PARAMS_LEN(d) (4 + 2 * (d))
nngp_status nngp_theta_params(const nngp_kernel *k, const double *theta_dev, int32_t d, double pivot_tol,
                              double *params_dev, void *stream);

/*
 * Same as nngp_loglik_f32/_f64 restricted to the points [row_begin, row_begin + row_count)
 * (nbr then has row_count rows; neighbour indices still refer to all n rows of x, y).
 * Replaces one task of the reference's row-batched worker loop (base_nngpr.py:440-449,
 * :503-538); summing the outputs of a partition of [0, n) gives the full result.
 */
nngp_status nngp_loglik_rows_f32(const float *x, const float *y, int64_t n, int32_t d, int32_t ydim,
                                 int64_t row_begin, int64_t row_count, const int32_t *nbr, int32_t m,
                                 const nngp_kernel *kernel, int32_t eval_gradient, double pivot_tol,
                                 double *out, int32_t *status_flags, void *workspace,
                                 size_t workspace_bytes, void *stream);
nngp_status nngp_loglik_rows_f64(const double *x, const double *y, int64_t n, int32_t d, int32_t ydim,
                                 int64_t row_begin, int64_t row_count, const int32_t *nbr, int32_t m,
                                 const nngp_kernel *kernel, int32_t eval_gradient, double pivot_tol,
                                 double *out, int32_t *status_flags, void *workspace,
                                 size_t workspace_bytes, void *stream);

/*
 * nngp_loglik_f64 without a workspace: no counterpart in the reference.
 *
 * For callers that cannot allocate device memory — for instance a serving process whose
 * device memory is fixed at start-up, or a foreign-language binding (cgo, JNI, ctypes) that
 * cannot own CUDA allocations — and so cannot pass the workspace nngp_loglik_f64 needs.
 * The per-CTA partial sums go to a fixed device array inside the library (333 KiB, held by
 * every GPU that loads the library until the process exits); the call allocates nothing.
 * Same inputs, outputs and results as nngp_loglik_f64 (which it matches bit for bit on a
 * 148-SM B200); it rejects more than 35 hyperparameters (n_theta > 35 with eval_gradient)
 * with NNGP_ERR_UNSUPPORTED.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it for the life of the process; make that first call before
 * any stream capture, and do not use the library across a cudaDeviceReset.  All calls share
 * the array: calls that overlap on the GPU (other streams or host threads on the same device)
 * race on it and must be serialised by the caller.
 */
nngp_status nngp_loglik_f64_noalloc(const double *x, const double *y, int64_t n, int32_t d, int32_t ydim,
                                    const int32_t *nbr, int32_t m, const nngp_kernel *kernel,
                                    int32_t eval_gradient, double *out, int32_t *status_flags,
                                    void *stream);

/* ---------------------------------------------------------------------------------------
 * Predictive mean / variance conditioned on the training set only
 *
 * Replaces Nngpr._predict_worker (base_nngpr.py:1032-1135) for
 * conditioning_method='only-train'.  Query q's local system is itself plus nbr[q, :]
 * (training indices, -1 = missing); alpha is added to the training slots only.
 * mean (nq x ydim) = K_xn K_nn^-1 y_nn, var (nq) = K_00 - K_xn K_nn^-1 K_xn^T (the
 * reference returns sqrt(var)).  Outputs in the input precision; FP32 systems whose
 * pivots fall below pivot_tol * (kernel diagonal) are re-solved in FP64.
 * ------------------------------------------------------------------------------------- */
nngp_status nngp_predict_f32(const float *x_train, const float *y_train, int64_t n_train,
                             const float *x_query, int64_t n_query, int32_t d, int32_t ydim,
                             const int32_t *nbr, int32_t m, const nngp_kernel *kernel,
                             double pivot_tol, float *mean, float *var, int32_t *status_flags,
                             void *stream);
nngp_status nngp_predict_f64(const double *x_train, const double *y_train, int64_t n_train,
                             const double *x_query, int64_t n_query, int32_t d, int32_t ydim,
                             const int32_t *nbr, int32_t m, const nngp_kernel *kernel,
                             double pivot_tol, double *mean, double *var, int32_t *status_flags,
                             void *stream);

/* ---------------------------------------------------------------------------------------
 * Measurement utility (no counterpart in the reference)
 *
 * Launches `blocks` x 256 threads, each running 8 independent FP32 FMA chains of 8 * iters
 * steps (128 * iters flops per thread), and writes one float per thread to `out`
 * (blocks * 256 floats).  Timing the launch gives the FP32 FMA rate that bounds the SIMT
 * kernels above.
 * ------------------------------------------------------------------------------------- */
nngp_status nngp_fma_probe(float *out, int64_t iters, int32_t blocks, void *stream);
/* FP64 FMA-rate probe (measurement only): blocks x 256 threads, 8 FMA chains of 8 x iters
 * steps each; out receives blocks x 256 doubles. */
nngp_status nngp_fma_probe_f64(double *out, int64_t iters, int32_t blocks, void *stream);

/* Plain FP32 GPU form of the neighbour search: the comparator the optimised search is measured
 * against (no counterpart in the reference's plugin interface; it restates the structure of the
 * reference's `calc_nn`, nngpr/cuda_kernel_accelerators.py:663-743: one thread per query, a
 * serial scan of the eligible refs, a sorted top-m list in shared memory).  Inputs are already
 * divided by the length scale, row-major (n, d) FP32.  Same results as nngp_knn_f32
 * (identical FP32 distance arithmetic, lower index first on ties, -1 padding, ref cut as there).
 * num_nn <= 256.  No workspace, no status flags.
 * ------------------------------------------------------------------------------------- */
nngp_status nngp_plain_knn_f32(const float *ref_scaled, int64_t n_ref, const float *query_scaled,
                               int64_t n_query, int32_t d, int32_t num_nn, int32_t has_ref_cut,
                               int64_t ref_cut_index, int32_t *out_idx, void *stream);

/* Predict with conditioning_method='full' (Nngpr.predict's sequential algorithm,
 * base_nngpr.py:896-1030): query i conditions on the training set and on the queries before it.
 * x_full = [x_train; x_query] (n_train + n_query rows), nbr (n_query, num_nn) indices into
 * x_full from nngp_knn_f64/_f32 with ref = x_full, query = x_query, ref_cut_index = n_train
 * (-1 padded; an index >= n_train + i is flagged and ignored).  Each query's local system gives
 * its conditioning weights in parallel (alpha on training neighbours only, :952-954); one warp
 * then walks the queries in order: the mean uses the predicted means of query neighbours, the
 * variance adds their covariance, which is tracked only between a query and its own query
 * neighbours, as the reference's sparse partial covariance does (:923-930, :1002-1008).  mean:
 * (n_query, ydim); var (n_query) when want_var.  FP64, num_nn <= 64 (for 'full-double-nn' pass
 * the packed lists of the training search and the queries' prefix search, base_nngpr.py:1418-1449,
 * num_nn = their combined width); the recursion is serial in the queries (tens of microseconds
 * per hundred queries). */
size_t nngp_predict_full_workspace_size(int64_t n_query, int32_t num_nn);
nngp_status nngp_predict_full_f64(const double *x_full, const double *y_train, int64_t n_train,
                                  int64_t n_query, int32_t d, int32_t ydim, const int32_t *nbr,
                                  int32_t num_nn, const nngp_kernel *kernel, int32_t want_var,
                                  double *mean, double *var, int32_t *status_flags, void *workspace,
                                  size_t workspace_bytes, void *stream);

/* Predict with conditioning_method='full' and the dense predictive covariance (Nngpr.predict
 * with return_cov, base_nngpr.py:989-1000): as nngp_predict_full_f64, but the covariance of every
 * pair of queries is kept, so each query's variance uses the full covariance of its query
 * neighbours.  cov: (n_query, n_query), symmetric, variances on the diagonal (normalised y
 * units).  One CTA walks the queries in order: O(n_query^2 num_nn) work, n_query^2 doubles. */
nngp_status nngp_predict_cov_full_f64(const double *x_full, const double *y_train, int64_t n_train,
                                      int64_t n_query, int32_t d, int32_t ydim, const int32_t *nbr,
                                      int32_t num_nn, const nngp_kernel *kernel, double *mean, double *cov,
                                      int32_t *status_flags, void *workspace, size_t workspace_bytes,
                                      void *stream);

/* Samples with conditioning_method='full' (Nngpr.sample_y's sequential algorithm,
 * base_nngpr.py:691-750): query i's samples condition on the training y and on the samples
 * already drawn for the queries before it, sample = w . v + max(0, sqrt(s2)) z.  Same inputs and
 * workspace as nngp_predict_full_f64; z: (n_query, ydim, n_samples) standard normals (device), in
 * the order the reference draws them (query by query, then (ydim, n_samples) in C order), so the
 * reference's own samples come back for its random stream; samples: same shape. */
nngp_status nngp_sample_full_f64(const double *x_full, const double *y_train, int64_t n_train,
                                 int64_t n_query, int32_t d, int32_t ydim, const int32_t *nbr,
                                 int32_t num_nn, const nngp_kernel *kernel, int32_t n_samples,
                                 const double *z, double *samples, int32_t *status_flags,
                                 void *workspace, size_t workspace_bytes, void *stream);

/* Self-test of the tensor-core operand layout used by the search (no counterpart in the
 * reference): d (128 x 128) = a (128 x kp) * b (128 x kp)^T in TF32 with FP32 accumulation,
 * a and b row-major device arrays, kp = 8, 16 or 32, through the same shared-memory layout,
 * descriptors, tcgen05.mma and TMEM reads as the search kernel.  One CTA. */
nngp_status nngp_tc_layout_selftest(const float *a, const float *b, int32_t kp, float *d, int32_t *status_flags,
                                    void *stream);
/* The same for the BF16 operands of the search at d >= 12 (tcgen05.mma kind::f16, K = 16 per
 * instruction): a and b hold values exactly representable in BF16 (converted with round to
 * nearest on staging), kp = 16, 32 or 64. */
nngp_status nngp_tc_layout_selftest_bf16(const float *a, const float *b, int32_t kp, float *d,
                                         int32_t *status_flags, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* NNGP_B200_H */
