// Neighbour-list reuse across fit steps whose length scale changes (isotropic kernels).
//
// The fit step's search ranks the earlier points j < i of each point i by the FP32 squared
// distance of the scaled coordinates, D_l(i, j) = sum_f (fl(x_jf / l) - fl(x_if / l))^2 in the
// oracle's arithmetic, ties by lower index (nngpr/base_nngpr.py:530-535 with calc_nn's rule,
// nngpr/cuda_kernel_accelerators.py:728).  The reference recomputes the search on every call
// (base_nngpr.py:532).  In exact arithmetic an isotropic l only scales every distance by 1/l^2,
// so the order cannot change; in FP32 it can, but only by the rounding error.  With
// E(i, j) = |x_i - x_j|^2 (exact, unscaled) and u = 2^-24, the oracle's arithmetic gives
//
//     | l^2 D_l(i, j) - E(i, j) | <= b(i, j) = 2 (d + 6) u (|x_i| + |x_j|)^2
//
// for every l (first-order bound of the two divisions, the difference, the square and the
// running sum, doubled for the higher-order terms).  So one search at l0 for C > m candidates
// per point, with tau_i = l0^2 D_l0(i, c_C) the normalised distance of the C-th candidate, proves
// for any later l: every non-candidate j has l^2 D_l(i, j) >= tau_i - 2 b_i, b_i = b with |x_j|
// replaced by max_j |x_j|.  If the m-th smallest candidate distance mu_i at l satisfies
// l^2 mu_i < tau_i - 2 b_i, the exact top-m at l lies among the candidates, and ranking them
// exactly gives the exact list.  Rows that fail the test are counted; the caller then runs the
// full search.
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"

namespace nngp {

constexpr int kReuseMaxCand = 64;
constexpr int kReuseMaxNN = 32;
constexpr int kReuseThreads = 128;
constexpr double kUnitRoundoff = 5.9604644775390625e-08;  // 2^-24

// D_l(i, j) in the oracle's arithmetic: scaled coordinates rounded, then
// ((t0^2 + t1^2) + t2^2) + ..., t_f = s_jf - s_if, every step rounded.
__device__ __forceinline__ float reuse_dist(const float *__restrict__ x, int64_t i, int64_t j, int d, float ls) {
    const float *xi = x + i * d, *xj = x + j * d;
    const float t0 = sub_rn(div_rn(xj[0], ls), div_rn(xi[0], ls));
    float d2 = mul_rn(t0, t0);
    for (int f = 1; f < d; ++f) {
        const float t = sub_rn(div_rn(xj[f], ls), div_rn(xi[f], ls));
        d2 = add_rn(d2, mul_rn(t, t));
    }
    return d2;
}

__device__ __forceinline__ double row_norm(const float *__restrict__ x, int64_t i, int d) {
    double s = 0.0;
    for (int f = 0; f < d; ++f) s += (double)x[i * d + f] * (double)x[i * d + f];
    return sqrt(s);
}

// thr_i = l0^2 D_l0(i, last candidate) - 2 b_i, or +inf when the row holds every earlier point
// (fewer valid candidates than slots).  Candidates are the search's list at l0 (ascending).
__global__ void __launch_bounds__(kReuseThreads) reuse_prepare_kernel(const float *__restrict__ x, int64_t n, int d,
                                                                      float ls, double ls2, const int32_t *__restrict__ cand,
                                                                      int nc, double max_norm, double *__restrict__ thr) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t last = cand[i * nc + nc - 1];
    if (last < 0) {
        thr[i] = pos_inf<double>();
        return;
    }
    const double tau = ls2 * (double)reuse_dist(x, i, last, d, ls);
    const double r = row_norm(x, i, d) * (1.0 + 1e-12) + max_norm;
    thr[i] = tau - 2.0 * (2.0 * (d + 6) * kUnitRoundoff) * r * r;
}

// Exact top-m of the candidates at length scale ls, ascending (distance, index); a row whose
// m-th distance does not clear its threshold is counted in *n_failed (its list is still written).
__global__ void __launch_bounds__(kReuseThreads) reuse_rank_kernel(const float *__restrict__ x, int64_t n, int d,
                                                                   float ls, double ls2,
                                                                   const int32_t *__restrict__ cand, int nc,
                                                                   const double *__restrict__ thr, int m,
                                                                   int32_t *__restrict__ out,
                                                                   int32_t *__restrict__ n_failed) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float bd[kReuseMaxNN];
    int32_t bi[kReuseMaxNN];
    int cnt = 0;
    for (int c = 0; c < nc; ++c) {
        const int32_t j = cand[i * nc + c];
        if (j < 0) continue;
        const float d2 = reuse_dist(x, i, j, d, ls);
        // insertion into the sorted top-m by (distance, index)
        int k = cnt < m ? cnt : m - 1;
        if (cnt >= m && !(d2 < bd[m - 1] || (d2 == bd[m - 1] && j < bi[m - 1]))) continue;
        while (k > 0 && (bd[k - 1] > d2 || (bd[k - 1] == d2 && bi[k - 1] > j))) {
            bd[k] = bd[k - 1];
            bi[k] = bi[k - 1];
            --k;
        }
        bd[k] = d2;
        bi[k] = j;
        if (cnt < m) ++cnt;
    }
    for (int k = 0; k < m; ++k) out[i * m + k] = k < cnt ? bi[k] : -1;
    const double t = thr[i];
    if (cnt == m && !isinf(t) && !(ls2 * (double)bd[m - 1] * (1.0 + 1e-12) < t)) atomicAdd(n_failed, 1);
    if (cnt < m && !isinf(t)) atomicAdd(n_failed, 1);  // fewer candidates than a full list: not proven
}

nngp_status reuse_prepare_f32(const float *x, int64_t n, int d, double ls, const int32_t *cand, int nc,
                              double max_norm, double *thr, cudaStream_t stream) {
    if (n < 0 || d < 1 || nc < 1 || nc > kReuseMaxCand || !(ls > 0.0) || !(max_norm >= 0.0))
        return fail(NNGP_ERR_INVALID_ARGUMENT,
                    "knn_reuse_prepare: need n >= 0, d >= 1, 1 <= n_cand <= 64, length_scale > 0, max_norm >= 0");
    if (n == 0) return NNGP_OK;
    if (!x || !cand || !thr) return fail(NNGP_ERR_INVALID_ARGUMENT, "knn_reuse_prepare: null pointer");
    const float ls32 = (float)ls;
    const double ls2 = (double)ls32 * (double)ls32;
    reuse_prepare_kernel<<<(unsigned)((n + kReuseThreads - 1) / kReuseThreads), kReuseThreads, 0, stream>>>(
        x, n, d, ls32, ls2, cand, nc, max_norm, thr);
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

nngp_status reuse_rank_f32(const float *x, int64_t n, int d, double ls, const int32_t *cand, int nc,
                           const double *thr, int m, int32_t *out, int32_t *n_failed, cudaStream_t stream) {
    if (n < 0 || d < 1 || nc < 1 || nc > kReuseMaxCand || m < 1 || m > kReuseMaxNN || m > nc || !(ls > 0.0))
        return fail(NNGP_ERR_INVALID_ARGUMENT,
                    "knn_reuse_rank: need n >= 0, d >= 1, 1 <= num_nn <= min(32, n_cand), n_cand <= 64, "
                    "length_scale > 0");
    if (n == 0) return NNGP_OK;
    if (!x || !cand || !thr || !out || !n_failed) return fail(NNGP_ERR_INVALID_ARGUMENT, "knn_reuse_rank: null pointer");
    const float ls32 = (float)ls;
    const double ls2 = (double)ls32 * (double)ls32;
    reuse_rank_kernel<<<(unsigned)((n + kReuseThreads - 1) / kReuseThreads), kReuseThreads, 0, stream>>>(
        x, n, d, ls32, ls2, cand, nc, thr, m, out, n_failed);
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

}  // namespace nngp
