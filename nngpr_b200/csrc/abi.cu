// C ABI of libnngp_b200: argument checks, error text and dispatch to the kernels.
// Declarations and the reference interface each entry point replaces: include/nngp_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <exception>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include "common.cuh"

namespace nngp {

// implemented in knn.cu / local.cu
size_t knn_workspace_f32(int64_t n_ref, int64_t n_query, int d, int m);
size_t knn_workspace_f64(int64_t n_ref, int64_t n_query, int d, int m);
nngp_status knn_f32(const float *, int64_t, const float *, int64_t, int, const double *, int, int, int, int64_t,
                    int32_t *, int32_t *, void *, size_t, cudaStream_t);
nngp_status knn_f64(const double *, int64_t, const double *, int64_t, int, const double *, int, int, int, int64_t,
                    int32_t *, int32_t *, void *, size_t, cudaStream_t);
nngp_status knn_f32_ls_device(const float *, int64_t, const float *, int64_t, int, const double *, int, int, int,
                              int64_t, int32_t *, int32_t *, void *, size_t, cudaStream_t);
nngp_status knn_f64_ls_device(const double *, int64_t, const double *, int64_t, int, const double *, int, int, int,
                              int64_t, int32_t *, int32_t *, void *, size_t, cudaStream_t);
nngp_status theta_params(const nngp_kernel *, const double *, int, double, double *, cudaStream_t);
size_t loglik_workspace(int64_t n, int d, int ydim, int m, int n_theta);
nngp_status loglik_f32(const float *, const float *, int64_t, int, int, const int32_t *, int, const nngp_kernel *, int,
                       double, double *, int32_t *, void *, size_t, cudaStream_t);
nngp_status loglik_f64(const double *, const double *, int64_t, int, int, const int32_t *, int, const nngp_kernel *,
                       int, double, double *, int32_t *, void *, size_t, cudaStream_t);
nngp_status loglik_rows_f32(const float *, const float *, int64_t, int, int, int64_t, int64_t, const int32_t *, int,
                            const nngp_kernel *, int, double, double *, int32_t *, void *, size_t, cudaStream_t);
nngp_status loglik_rows_f64(const double *, const double *, int64_t, int, int, int64_t, int64_t, const int32_t *, int,
                            const nngp_kernel *, int, double, double *, int32_t *, void *, size_t, cudaStream_t);
nngp_status loglik_f64_noalloc(const double *, const double *, int64_t, int, int, const int32_t *, int,
                               const nngp_kernel *, int, double *, int32_t *, cudaStream_t);
nngp_status plain_knn_f32(const float *, int64_t, const float *, int64_t, int, int, bool, int64_t, int32_t *,
                          cudaStream_t);
size_t predict_full_workspace_size(int64_t, int);
nngp_status predict_full(const double *, const double *, int64_t, int64_t, int, int, const int32_t *, int,
                         const nngp_kernel *, int, double *, double *, int32_t *, void *, size_t, cudaStream_t);
nngp_status predict_cov_full(const double *, const double *, int64_t, int64_t, int, int, const int32_t *, int,
                             const nngp_kernel *, double *, double *, int32_t *, void *, size_t, cudaStream_t);
nngp_status sample_full(const double *, const double *, int64_t, int64_t, int, int, const int32_t *, int,
                        const nngp_kernel *, int, const double *, double *, int32_t *, void *, size_t, cudaStream_t);
nngp_status reuse_prepare_f32(const float *, int64_t, int, double, const int32_t *, int, double, double *,
                              cudaStream_t);
nngp_status reuse_rank_f32(const float *, int64_t, int, double, const int32_t *, int, const double *, int, int32_t *,
                           int32_t *, cudaStream_t);
nngp_status predict_f32(const float *, const float *, int64_t, const float *, int64_t, int, int, const int32_t *, int,
                        const nngp_kernel *, double, float *, float *, int32_t *, cudaStream_t);
nngp_status predict_f64(const double *, const double *, int64_t, const double *, int64_t, int, int, const int32_t *,
                        int, const nngp_kernel *, double, double *, double *, int32_t *, cudaStream_t);

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string &msg) { g_last_error = msg; }

nngp_status fail(nngp_status st, const std::string &msg) {
    g_last_error = msg;
    return st;
}

nngp_status cuda_fail(cudaError_t e, const char *what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return NNGP_ERR_CUDA;
}

const char *last_error_cstr() { return g_last_error.c_str(); }

namespace {
std::atomic<uint64_t> g_wait_limit{kWaitLimitNs};
}

uint64_t wait_limit_ns() { return g_wait_limit.load(std::memory_order_relaxed); }
uint64_t set_wait_limit_ns(uint64_t ns) { return g_wait_limit.exchange(ns == 0 ? kWaitLimitNs : ns); }

cudaError_t ensure_smem_limit(const void *fn, int bytes, int carveout) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, std::pair<int, int>> done;  // (fn, device) -> (bytes, carveout)
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    auto it = done.find({fn, dev});
    if (it != done.end() && it->second.first >= bytes && (carveout < 0 || it->second.second == carveout))
        return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && carveout >= 0) e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, carveout);
    if (e == cudaSuccess) {
        auto &v = done[{fn, dev}];
        v.first = std::max(v.first, bytes);
        if (carveout >= 0) v.second = carveout;
    }
    return e;
}

}  // namespace nngp

using namespace nngp;

namespace {

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Every entry point clears the error text, never lets a C++ exception cross the ABI.
template <typename F> nngp_status guarded(F &&f) {
    set_error("");
    try {
        return f();
    } catch (const std::exception &ex) {
        return fail(NNGP_ERR_INVALID_ARGUMENT, std::string("internal error: ") + ex.what());
    } catch (...) {
        return fail(NNGP_ERR_INVALID_ARGUMENT, "internal error");
    }
}

}  // namespace

extern "C" {

int32_t nngp_abi_version(void) { return NNGP_ABI_VERSION; }

uint64_t nngp_set_wait_limit_ns(uint64_t ns) { return set_wait_limit_ns(ns); }

const char *nngp_last_error(void) { return last_error_cstr(); }

const char *nngp_status_string(nngp_status status) {
    switch (status) {
        case NNGP_OK: return "NNGP_OK";
        case NNGP_ERR_INVALID_ARGUMENT: return "NNGP_ERR_INVALID_ARGUMENT";
        case NNGP_ERR_UNSUPPORTED: return "NNGP_ERR_UNSUPPORTED";
        case NNGP_ERR_WORKSPACE: return "NNGP_ERR_WORKSPACE";
        case NNGP_ERR_CUDA: return "NNGP_ERR_CUDA";
        case NNGP_ERR_NO_DEVICE: return "NNGP_ERR_NO_DEVICE";
    }
    return "NNGP_ERR_UNKNOWN";
}

nngp_status nngp_check_device(void) {
    return guarded([&]() -> nngp_status {
        int dev = -1;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return fail(NNGP_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
        cudaDeviceProp prop;
        e = cudaGetDeviceProperties(&prop, dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
        if (prop.major != 10 || prop.minor != 0)
            return fail(NNGP_ERR_NO_DEVICE, std::string("device ") + prop.name + " is sm_" + std::to_string(prop.major) +
                                                std::to_string(prop.minor) + "; this build runs on sm_100a only");
        return NNGP_OK;
    });
}

size_t nngp_knn_workspace_size_f32(int64_t n_ref, int64_t n_query, int32_t d, int32_t num_nn) {
    return knn_workspace_f32(n_ref, n_query, d, num_nn);
}
size_t nngp_knn_workspace_size_f64(int64_t n_ref, int64_t n_query, int32_t d, int32_t num_nn) {
    return knn_workspace_f64(n_ref, n_query, d, num_nn);
}

nngp_status nngp_knn_f32(const float *ref, int64_t n_ref, const float *query, int64_t n_query, int32_t d,
                         const double *length_scale, int32_t n_ls, int32_t num_nn, int32_t has_ref_cut,
                         int64_t ref_cut_index, int32_t *out_idx, int32_t *status_flags, void *workspace,
                         size_t workspace_bytes, void *stream) {
    return guarded([&] {
        return knn_f32(ref, n_ref, query, n_query, d, length_scale, n_ls, num_nn, has_ref_cut != 0, ref_cut_index,
                       out_idx, status_flags, workspace, workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_knn_f32_ls_device(const float *ref, int64_t n_ref, const float *query, int64_t n_query, int32_t d,
                                   const double *length_scale_dev, int32_t n_ls, int32_t num_nn, int32_t has_ref_cut,
                                   int64_t ref_cut_index, int32_t *out_idx, int32_t *status_flags, void *workspace,
                                   size_t workspace_bytes, void *stream) {
    return guarded([&] {
        return knn_f32_ls_device(ref, n_ref, query, n_query, d, length_scale_dev, n_ls, num_nn, has_ref_cut != 0,
                                 ref_cut_index, out_idx, status_flags, workspace, workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_knn_f64_ls_device(const double *ref, int64_t n_ref, const double *query, int64_t n_query, int32_t d,
                                   const double *length_scale_dev, int32_t n_ls, int32_t num_nn, int32_t has_ref_cut,
                                   int64_t ref_cut_index, int32_t *out_idx, int32_t *status_flags, void *workspace,
                                   size_t workspace_bytes, void *stream) {
    return guarded([&] {
        return knn_f64_ls_device(ref, n_ref, query, n_query, d, length_scale_dev, n_ls, num_nn, has_ref_cut != 0,
                                 ref_cut_index, out_idx, status_flags, workspace, workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_theta_params(const nngp_kernel *k, const double *theta_dev, int32_t d, double pivot_tol,
                              double *params_dev, void *stream) {
    return guarded([&] { return theta_params(k, theta_dev, d, pivot_tol, params_dev, as_stream(stream)); });
}

nngp_status nngp_knn_f64(const double *ref, int64_t n_ref, const double *query, int64_t n_query, int32_t d,
                         const double *length_scale, int32_t n_ls, int32_t num_nn, int32_t has_ref_cut,
                         int64_t ref_cut_index, int32_t *out_idx, int32_t *status_flags, void *workspace,
                         size_t workspace_bytes, void *stream) {
    return guarded([&] {
        return knn_f64(ref, n_ref, query, n_query, d, length_scale, n_ls, num_nn, has_ref_cut != 0, ref_cut_index,
                       out_idx, status_flags, workspace, workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_plain_knn_f32(const float *ref_scaled, int64_t n_ref, const float *query_scaled, int64_t n_query,
                               int32_t d, int32_t num_nn, int32_t has_ref_cut, int64_t ref_cut_index,
                               int32_t *out_idx, void *stream) {
    return guarded([&] {
        return plain_knn_f32(ref_scaled, n_ref, query_scaled, n_query, d, num_nn, has_ref_cut != 0, ref_cut_index,
                             out_idx, as_stream(stream));
    });
}

size_t nngp_predict_full_workspace_size(int64_t n_query, int32_t num_nn) {
    return predict_full_workspace_size(n_query, num_nn);
}

nngp_status nngp_predict_full_f64(const double *x_full, const double *y_train, int64_t n_train, int64_t n_query,
                                  int32_t d, int32_t ydim, const int32_t *nbr, int32_t num_nn,
                                  const nngp_kernel *kernel, int32_t want_var, double *mean, double *var,
                                  int32_t *status_flags, void *workspace, size_t workspace_bytes, void *stream) {
    return guarded([&] {
        return predict_full(x_full, y_train, n_train, n_query, d, ydim, nbr, num_nn, kernel, want_var, mean, var,
                            status_flags, workspace, workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_predict_cov_full_f64(const double *x_full, const double *y_train, int64_t n_train, int64_t n_query,
                                      int32_t d, int32_t ydim, const int32_t *nbr, int32_t num_nn,
                                      const nngp_kernel *kernel, double *mean, double *cov, int32_t *status_flags,
                                      void *workspace, size_t workspace_bytes, void *stream) {
    return guarded([&] {
        return predict_cov_full(x_full, y_train, n_train, n_query, d, ydim, nbr, num_nn, kernel, mean, cov,
                                status_flags, workspace, workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_sample_full_f64(const double *x_full, const double *y_train, int64_t n_train, int64_t n_query,
                                 int32_t d, int32_t ydim, const int32_t *nbr, int32_t num_nn, const nngp_kernel *kernel,
                                 int32_t n_samples, const double *z, double *samples, int32_t *status_flags,
                                 void *workspace, size_t workspace_bytes, void *stream) {
    return guarded([&] {
        return sample_full(x_full, y_train, n_train, n_query, d, ydim, nbr, num_nn, kernel, n_samples, z, samples,
                           status_flags, workspace, workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_knn_reuse_prepare_f32(const float *x, int64_t n, int32_t d, double length_scale,
                                       const int32_t *cand, int32_t n_cand, double max_norm, double *thr,
                                       void *stream) {
    return guarded([&] {
        return reuse_prepare_f32(x, n, d, length_scale, cand, n_cand, max_norm, thr, as_stream(stream));
    });
}

nngp_status nngp_knn_reuse_rank_f32(const float *x, int64_t n, int32_t d, double length_scale, const int32_t *cand,
                                    int32_t n_cand, const double *thr, int32_t num_nn, int32_t *out_idx,
                                    int32_t *n_failed, void *stream) {
    return guarded([&] {
        return reuse_rank_f32(x, n, d, length_scale, cand, n_cand, thr, num_nn, out_idx, n_failed,
                              as_stream(stream));
    });
}

size_t nngp_loglik_workspace_size(int64_t n, int32_t d, int32_t ydim, int32_t m, int32_t n_theta) {
    return loglik_workspace(n, d, ydim, m, n_theta);
}

const uint64_t *nngp_loglik_fp64_count(const void *workspace) {
    if (!workspace) return nullptr;
    return reinterpret_cast<const uint64_t *>(align_up(reinterpret_cast<uintptr_t>(workspace), 256));
}

nngp_status nngp_loglik_f32(const float *x, const float *y, int64_t n, int32_t d, int32_t ydim, const int32_t *nbr,
                            int32_t m, const nngp_kernel *kernel, int32_t eval_gradient, double pivot_tol,
                            double *out, int32_t *status_flags, void *workspace, size_t workspace_bytes,
                            void *stream) {
    return guarded([&] {
        return loglik_f32(x, y, n, d, ydim, nbr, m, kernel, eval_gradient, pivot_tol, out, status_flags, workspace,
                          workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_loglik_f64(const double *x, const double *y, int64_t n, int32_t d, int32_t ydim, const int32_t *nbr,
                            int32_t m, const nngp_kernel *kernel, int32_t eval_gradient, double pivot_tol,
                            double *out, int32_t *status_flags, void *workspace, size_t workspace_bytes,
                            void *stream) {
    return guarded([&] {
        return loglik_f64(x, y, n, d, ydim, nbr, m, kernel, eval_gradient, pivot_tol, out, status_flags, workspace,
                          workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_loglik_rows_f32(const float *x, const float *y, int64_t n, int32_t d, int32_t ydim, int64_t row_begin,
                                 int64_t row_count, const int32_t *nbr, int32_t m, const nngp_kernel *kernel,
                                 int32_t eval_gradient, double pivot_tol, double *out, int32_t *status_flags,
                                 void *workspace, size_t workspace_bytes, void *stream) {
    return guarded([&] {
        return loglik_rows_f32(x, y, n, d, ydim, row_begin, row_count, nbr, m, kernel, eval_gradient, pivot_tol, out,
                               status_flags, workspace, workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_loglik_rows_f64(const double *x, const double *y, int64_t n, int32_t d, int32_t ydim,
                                 int64_t row_begin, int64_t row_count, const int32_t *nbr, int32_t m,
                                 const nngp_kernel *kernel, int32_t eval_gradient, double pivot_tol, double *out,
                                 int32_t *status_flags, void *workspace, size_t workspace_bytes, void *stream) {
    return guarded([&] {
        return loglik_rows_f64(x, y, n, d, ydim, row_begin, row_count, nbr, m, kernel, eval_gradient, pivot_tol, out,
                               status_flags, workspace, workspace_bytes, as_stream(stream));
    });
}

nngp_status nngp_loglik_f64_noalloc(const double *x, const double *y, int64_t n, int32_t d, int32_t ydim,
                                   const int32_t *nbr, int32_t m, const nngp_kernel *kernel, int32_t eval_gradient,
                                   double *out, int32_t *status_flags, void *stream) {
    return guarded([&] {
        return loglik_f64_noalloc(x, y, n, d, ydim, nbr, m, kernel, eval_gradient, out, status_flags,
                                  as_stream(stream));
    });
}

nngp_status nngp_predict_f32(const float *x_train, const float *y_train, int64_t n_train, const float *x_query,
                             int64_t n_query, int32_t d, int32_t ydim, const int32_t *nbr, int32_t m,
                             const nngp_kernel *kernel, double pivot_tol, float *mean, float *var,
                             int32_t *status_flags, void *stream) {
    return guarded([&] {
        return predict_f32(x_train, y_train, n_train, x_query, n_query, d, ydim, nbr, m, kernel, pivot_tol, mean, var,
                           status_flags, as_stream(stream));
    });
}

nngp_status nngp_predict_f64(const double *x_train, const double *y_train, int64_t n_train, const double *x_query,
                             int64_t n_query, int32_t d, int32_t ydim, const int32_t *nbr, int32_t m,
                             const nngp_kernel *kernel, double pivot_tol, double *mean, double *var,
                             int32_t *status_flags, void *stream) {
    return guarded([&] {
        return predict_f64(x_train, y_train, n_train, x_query, n_query, d, ydim, nbr, m, kernel, pivot_tol, mean, var,
                           status_flags, as_stream(stream));
    });
}

}  // extern "C"
