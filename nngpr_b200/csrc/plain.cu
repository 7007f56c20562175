// The plain FP32 GPU form of the neighbour search: the comparator the optimised search is
// measured against (one launch per call, one thread per query).
//
// Structure of the reference's CUDA search (`calc_nn`, cuda_kernel_accelerators.py:663-743):
// every thread scans the eligible refs of its query in index order and keeps a sorted top-m
// list in shared memory, inserting by shifting the tail.  Inputs are already divided by the
// length scale (the reference does that before the launch, :237-240).  The distance uses the
// same FP32 arithmetic as the optimised kernels and the oracle (per-feature difference, square
// and running sum, each rounded, no contraction) and ties keep the lower index, so both
// searches return identical lists and the comparison times the same result.
#include <cuda_runtime.h>

#include "common.cuh"

namespace nngp {

constexpr int kPlainThreads = 128;

__global__ void __launch_bounds__(kPlainThreads) plain_knn_kernel(const float *__restrict__ ref, int64_t n_ref,
                                                                  const float *__restrict__ query, int64_t n_query,
                                                                  int d, int m, int has_cut, int64_t cut,
                                                                  int32_t *__restrict__ out) {
    // slot k of this thread's list at [k * blockDim.x + threadIdx.x]: threads of a warp touch
    // consecutive words, no bank conflicts
    extern __shared__ __align__(16) unsigned char plain_smem[];
    float *dist = reinterpret_cast<float *>(plain_smem) + threadIdx.x;
    int32_t *idx = reinterpret_cast<int32_t *>(plain_smem + (size_t)blockDim.x * m * sizeof(float)) + threadIdx.x;
    const int S = blockDim.x;
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= n_query) return;
    for (int k = 0; k < m; ++k) {
        dist[k * S] = pos_inf<float>();
        idx[k * S] = -1;
    }
    int64_t limit = n_ref;
    if (has_cut) {
        limit = q + cut;
        limit = limit < 0 ? 0 : (limit > n_ref ? n_ref : limit);
    }
    const float *qp = query + q * d;
    float worst = pos_inf<float>();
    for (int64_t j = 0; j < limit; ++j) {
        const float *rp = ref + j * d;
        const float t0 = sub_rn(rp[0], qp[0]);
        float d2 = mul_rn(t0, t0);
        for (int f = 1; f < d; ++f) {
            const float t = sub_rn(rp[f], qp[f]);
            d2 = add_rn(d2, mul_rn(t, t));
        }
        if (d2 < worst) {  // strict: an equal distance never displaces a lower index
            int k = m - 1;
            while (k > 0 && dist[(k - 1) * S] > d2) {
                dist[k * S] = dist[(k - 1) * S];
                idx[k * S] = idx[(k - 1) * S];
                --k;
            }
            dist[k * S] = d2;
            idx[k * S] = (int32_t)j;
            worst = dist[(m - 1) * S];
        }
    }
    for (int k = 0; k < m; ++k) out[q * m + k] = idx[k * S];
}

nngp_status plain_knn_f32(const float *ref, int64_t n_ref, const float *query, int64_t n_query, int d, int m,
                          bool has_cut, int64_t cut, int32_t *out, cudaStream_t stream) {
    if (n_ref < 0 || n_query < 0 || d < 1 || m < 1 || m > 256)
        return fail(NNGP_ERR_INVALID_ARGUMENT, "plain_knn: need n >= 0, d >= 1, 1 <= num_nn <= 256");
    if (n_query == 0) return NNGP_OK;
    if (!query || !out || (n_ref > 0 && !ref)) return fail(NNGP_ERR_INVALID_ARGUMENT, "plain_knn: null pointer");
    const size_t smem = (size_t)kPlainThreads * m * (sizeof(float) + sizeof(int32_t));
    NNGP_CUDA_TRY(ensure_smem_limit(reinterpret_cast<const void *>(plain_knn_kernel), (int)smem));
    const int64_t grid = (n_query + kPlainThreads - 1) / kPlainThreads;
    plain_knn_kernel<<<(unsigned)grid, kPlainThreads, smem, stream>>>(ref, n_ref, query, n_query, d, m,
                                                                     has_cut ? 1 : 0, cut, out);
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

}  // namespace nngp
