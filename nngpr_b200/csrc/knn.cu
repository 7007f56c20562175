// Exact k-nearest-neighbour search on B200 (sm_100a).
//
// Semantics (reference: NngprWorker.find_nearest_neighbors, base_nngpr.py:1613-1686, and the
// CUDA calc_nn kernel, cuda_kernel_accelerators.py:663-743): for each query, the num_nn refs
// with the smallest squared distance sum_f (r_f - q_f)^2 of the length-scale-scaled points,
// ascending, equal distances ordered by lower ref index, -1 for missing slots; with a ref cut
// query q only sees refs [0, q + cut).
//
// Design:
//   * a prep kernel writes the scaled points (x / l in the search precision, correctly
//     rounded division) into the workspace, rows padded to DP = round_up(d, 4) floats and the
//     ref array padded with zero rows to whole tiles, so every tile is one aligned TMA copy;
//   * the search kernel gives every thread one query (coordinates in registers) and streams
//     the ref tiles through shared memory with cp.async.bulk (TMA, no multicast) into a
//     4-stage mbarrier ring; every thread reads each ref once from shared memory (broadcast);
//   * each thread keeps its top-M list sorted in registers (M = num_nn rounded up to 8, 16,
//     32 or 64; the unused M - num_nn leading slots hold -inf and never move), inserting with
//     an unrolled compare/select network;
//   * distances use one rounding per operation (__fsub_rn/__fmul_rn/__fadd_rn), the arithmetic
//     of the CPU restatement, so the lists are bit-identical to an exact search;
//   * prefix (fit) searches are triangular: blocks are issued heaviest first.
// A generic kernel (lists in the workspace, any d <= 256, any num_nn, float or double) covers
// the shapes the register kernel does not.
#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>

#include "common.cuh"

namespace nngp {

constexpr int kKnnThreads = 128;
constexpr int kKnnStages = 4;
constexpr int kKnnTileBytes = 4096;
constexpr int kMaxDim = 256;

template <typename T> struct LsParam {
    T v[kMaxDim];
};

// dst (n_pad x dp) = src (n x d) / ls, zero padded (columns d..dp-1 and rows n..n_pad-1).
template <typename T>
__global__ void scale_pad_kernel(const T *__restrict__ src, int64_t n, int d, int dp, int64_t n_pad,
                                 LsParam<T> ls, int use_ls, T *__restrict__ dst) {
    const int64_t total = n_pad * dp;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / dp;
        const int f = (int)(e - i * dp);
        T v = T(0);
        if (i < n && f < d) {
            v = src[i * d + f];
            if (use_ls) v = div_rn(v, ls.v[f]);
        }
        dst[e] = v;
    }
}

// ---------------------------------------------------------------------------------------
// Register top-M search kernel (float)
// ---------------------------------------------------------------------------------------
template <int D, int M>
struct KnnCfg {
    static constexpr int DP = (D + 3) / 4 * 4;
    static constexpr int TJ = kKnnTileBytes / (DP * 4);  // refs per tile
    static constexpr int SMEM = kKnnStages * kKnnTileBytes + 64;
};

template <int D, int M>
__global__ void __launch_bounds__(kKnnThreads) knn_topm_kernel(const float *__restrict__ refs, const float *__restrict__ qs,
                                                               int64_t n_query, int64_t n_ref, int has_cut, int64_t cut,
                                                               int m, int32_t *__restrict__ out,
                                                               int32_t *__restrict__ flags) {
    using Cfg = KnnCfg<D, M>;
    constexpr int DP = Cfg::DP;
    constexpr int TJ = Cfg::TJ;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float4 *tiles = reinterpret_cast<float4 *>(smem_raw);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem_raw + kKnnStages * kKnnTileBytes);

    // heaviest (latest) query blocks first for the triangular prefix search
    const int64_t qblock = has_cut ? (int64_t)(gridDim.x - 1 - blockIdx.x) : (int64_t)blockIdx.x;
    const int64_t q0 = qblock * kKnnThreads;
    const int64_t q = q0 + threadIdx.x;
    const bool active = q < n_query;

    auto limit_of = [&](int64_t qq) -> int64_t {
        if (!has_cut) return n_ref;
        int64_t l = qq + cut;
        return l < 0 ? 0 : (l > n_ref ? n_ref : l);
    };
    const int64_t limit = active ? limit_of(q) : 0;
    const int64_t qlast = min(q0 + kKnnThreads, n_query) - 1;
    const int64_t block_limit = limit_of(qlast);  // non-decreasing in q
    const int64_t ntiles = (block_limit + TJ - 1) / TJ;

    float qv[D];
    {
        const float4 *qp = reinterpret_cast<const float4 *>(qs + (active ? q : 0) * DP);
#pragma unroll
        for (int c = 0; c < DP / 4; ++c) {
            const float4 v = qp[c];
            if (4 * c + 0 < D) qv[4 * c + 0] = v.x;
            if (4 * c + 1 < D) qv[4 * c + 1] = v.y;
            if (4 * c + 2 < D) qv[4 * c + 2] = v.z;
            if (4 * c + 3 < D) qv[4 * c + 3] = v.w;
        }
    }

    float dist[M];
    int32_t idx[M];
#pragma unroll
    for (int k = 0; k < M; ++k) {
        dist[k] = (k < M - m) ? neg_inf<float>() : pos_inf<float>();
        idx[k] = -1;
    }

    if (threadIdx.x == 0) {
        for (int s = 0; s < kKnnStages; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int s = 0; s < kKnnStages && s < ntiles; ++s) {
            mbar_arrive_expect_tx(&full[s], kKnnTileBytes);
            tma_bulk_g2s(tiles + s * (kKnnTileBytes / 16), refs + (int64_t)s * TJ * DP, kKnnTileBytes, &full[s]);
        }
    }

    for (int64_t t = 0; t < ntiles; ++t) {
        const int s = (int)(t % kKnnStages);
        const uint32_t parity = (uint32_t)((t / kKnnStages) & 1);
        const bool ok = mbar_wait_bounded(&full[s], parity);
        if (__syncthreads_or(!ok)) {
            // give up: record it, let the copies already issued land (bounded), then leave
            if (threadIdx.x == 0) {
                flag_or(flags, NNGP_FLAG_TIMEOUT);
                for (int64_t tt = t; tt < ntiles && tt < t + kKnnStages; ++tt)
                    mbar_wait_bounded(&full[tt % kKnnStages], (uint32_t)((tt / kKnnStages) & 1));
            }
            __syncthreads();
            return;
        }
        const float4 *tile = tiles + s * (kKnnTileBytes / 16);
        const int64_t j0 = t * TJ;
        const int64_t jn = limit - j0;  // refs of this tile the thread may use
        if (jn >= TJ) {
#pragma unroll 2
            for (int jj = 0; jj < TJ; ++jj) {
                float rv[DP];
#pragma unroll
                for (int c = 0; c < DP / 4; ++c) {
                    const float4 v = tile[jj * (DP / 4) + c];
                    rv[4 * c + 0] = v.x; rv[4 * c + 1] = v.y; rv[4 * c + 2] = v.z; rv[4 * c + 3] = v.w;
                }
                float d2 = mul_rn(sub_rn(rv[0], qv[0]), sub_rn(rv[0], qv[0]));
#pragma unroll
                for (int f = 1; f < D; ++f) {
                    const float tf = sub_rn(rv[f], qv[f]);
                    d2 = add_rn(d2, mul_rn(tf, tf));
                }
                if (d2 < dist[M - 1]) {
                    const int32_t j = (int32_t)(j0 + jj);
#pragma unroll
                    for (int k = M - 1; k > 0; --k) {
                        const bool sh = d2 < dist[k - 1];
                        const bool here = d2 < dist[k];
                        const float nd = sh ? dist[k - 1] : (here ? d2 : dist[k]);
                        const int32_t ni = sh ? idx[k - 1] : (here ? j : idx[k]);
                        dist[k] = nd;
                        idx[k] = ni;
                    }
                    if (d2 < dist[0]) { dist[0] = d2; idx[0] = j; }
                }
            }
        } else if (jn > 0) {
            for (int jj = 0; jj < (int)jn; ++jj) {
                float rv[DP];
#pragma unroll
                for (int c = 0; c < DP / 4; ++c) {
                    const float4 v = tile[jj * (DP / 4) + c];
                    rv[4 * c + 0] = v.x; rv[4 * c + 1] = v.y; rv[4 * c + 2] = v.z; rv[4 * c + 3] = v.w;
                }
                float d2 = mul_rn(sub_rn(rv[0], qv[0]), sub_rn(rv[0], qv[0]));
#pragma unroll
                for (int f = 1; f < D; ++f) {
                    const float tf = sub_rn(rv[f], qv[f]);
                    d2 = add_rn(d2, mul_rn(tf, tf));
                }
                if (d2 < dist[M - 1]) {
                    const int32_t j = (int32_t)(j0 + jj);
#pragma unroll
                    for (int k = M - 1; k > 0; --k) {
                        const bool sh = d2 < dist[k - 1];
                        const bool here = d2 < dist[k];
                        const float nd = sh ? dist[k - 1] : (here ? d2 : dist[k]);
                        const int32_t ni = sh ? idx[k - 1] : (here ? j : idx[k]);
                        dist[k] = nd;
                        idx[k] = ni;
                    }
                    if (d2 < dist[0]) { dist[0] = d2; idx[0] = j; }
                }
            }
        }
        __syncthreads();  // every thread is done with stage s before it is refilled
        if (threadIdx.x == 0 && t + kKnnStages < ntiles) {
            mbar_arrive_expect_tx(&full[s], kKnnTileBytes);
            tma_bulk_g2s(tiles + s * (kKnnTileBytes / 16), refs + (t + kKnnStages) * TJ * DP, kKnnTileBytes, &full[s]);
        }
    }

    if (active) {
        int32_t *o = out + q * m;
#pragma unroll
        for (int k = 0; k < M; ++k)
            if (k >= M - m) o[k - (M - m)] = idx[k];
    }
}

// ---------------------------------------------------------------------------------------
// Generic search kernel: any d <= kMaxDim, any num_nn, float or double.  Query coordinates
// in shared memory, sorted list in the workspace (list[k * n_query + q]).
// ---------------------------------------------------------------------------------------
constexpr int kGenThreads = 128;
constexpr int kGenTile = 64;

template <typename T>
__global__ void __launch_bounds__(kGenThreads) knn_generic_kernel(const T *__restrict__ refs, const T *__restrict__ qs,
                                                                  int64_t n_query, int64_t n_ref, int dp, int d,
                                                                  int has_cut, int64_t cut, int m,
                                                                  T *__restrict__ ldist, int32_t *__restrict__ lidx,
                                                                  int32_t *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *qsm = reinterpret_cast<T *>(smem_raw);           // d x kGenThreads
    T *tile = qsm + (size_t)d * kGenThreads;            // kGenTile x dp
    const int64_t qblock = has_cut ? (int64_t)(gridDim.x - 1 - blockIdx.x) : (int64_t)blockIdx.x;
    const int64_t q0 = qblock * kGenThreads;
    const int64_t q = q0 + threadIdx.x;
    const bool active = q < n_query;
    auto limit_of = [&](int64_t qq) -> int64_t {
        if (!has_cut) return n_ref;
        int64_t l = qq + cut;
        return l < 0 ? 0 : (l > n_ref ? n_ref : l);
    };
    const int64_t limit = active ? limit_of(q) : 0;
    const int64_t block_limit = limit_of(min(q0 + kGenThreads, n_query) - 1);
    for (int f = 0; f < d; ++f) qsm[f * kGenThreads + threadIdx.x] = active ? qs[q * dp + f] : T(0);
    T *dl = ldist + (active ? q : 0);
    int32_t *il = lidx + (active ? q : 0);
    if (active)
        for (int k = 0; k < m; ++k) { dl[(int64_t)k * n_query] = pos_inf<T>(); il[(int64_t)k * n_query] = -1; }
    T thr = pos_inf<T>();
    for (int64_t j0 = 0; j0 < block_limit; j0 += kGenTile) {
        __syncthreads();
        for (int e = threadIdx.x; e < kGenTile * dp; e += kGenThreads) {
            const int64_t j = j0 + e / dp;
            tile[e] = j < n_ref ? refs[j * dp + (e % dp)] : T(0);
        }
        __syncthreads();
        const int64_t jn = limit - j0;
        const int jmax = jn >= kGenTile ? kGenTile : (jn > 0 ? (int)jn : 0);
        for (int jj = 0; jj < jmax; ++jj) {
            T t0 = sub_rn(tile[jj * dp], qsm[threadIdx.x]);
            T d2 = mul_rn(t0, t0);
            for (int f = 1; f < d; ++f) {
                const T tf = sub_rn(tile[jj * dp + f], qsm[f * kGenThreads + threadIdx.x]);
                d2 = add_rn(d2, mul_rn(tf, tf));
            }
            if (d2 < thr) {
                // insertion sort, ties keep the earlier (lower) index first
                int k = m - 1;
                while (k > 0) {
                    const T prev = dl[(int64_t)(k - 1) * n_query];
                    if (prev <= d2) break;
                    dl[(int64_t)k * n_query] = prev;
                    il[(int64_t)k * n_query] = il[(int64_t)(k - 1) * n_query];
                    --k;
                }
                dl[(int64_t)k * n_query] = d2;
                il[(int64_t)k * n_query] = (int32_t)(j0 + jj);
                thr = dl[(int64_t)(m - 1) * n_query];
            }
        }
    }
    if (active)
        for (int k = 0; k < m; ++k) out[q * m + k] = il[(int64_t)k * n_query];
}

// ---------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------
namespace {

int round_m(int m) {
    if (m <= 8) return 8;
    if (m <= 16) return 16;
    if (m <= 32) return 32;
    if (m <= 64) return 64;
    return 0;
}

int round_d(int d) {
    if (d <= 8) return d;
    if (d <= 32) return (d + 3) / 4 * 4;
    return 0;
}

using TopmFn = void (*)(const float *, const float *, int64_t, int64_t, int, int64_t, int, int32_t *, int32_t *);

template <int D, int M> TopmFn topm_entry() { return knn_topm_kernel<D, M>; }
template <int D, int M> int topm_smem() { return KnnCfg<D, M>::SMEM; }
template <int D, int M> int topm_tj() { return KnnCfg<D, M>::TJ; }

struct TopmVariant {
    TopmFn fn;
    int smem;
    int tj;
};

template <int D> TopmVariant pick_m(int M) {
    switch (M) {
        case 8: return {topm_entry<D, 8>(), topm_smem<D, 8>(), topm_tj<D, 8>()};
        case 16: return {topm_entry<D, 16>(), topm_smem<D, 16>(), topm_tj<D, 16>()};
        case 32: return {topm_entry<D, 32>(), topm_smem<D, 32>(), topm_tj<D, 32>()};
        case 64: return {topm_entry<D, 64>(), topm_smem<D, 64>(), topm_tj<D, 64>()};
    }
    return {nullptr, 0, 0};
}

TopmVariant pick_topm(int D, int M) {
    switch (D) {
        case 1: return pick_m<1>(M);
        case 2: return pick_m<2>(M);
        case 3: return pick_m<3>(M);
        case 4: return pick_m<4>(M);
        case 5: return pick_m<5>(M);
        case 6: return pick_m<6>(M);
        case 7: return pick_m<7>(M);
        case 8: return pick_m<8>(M);
        case 12: return pick_m<12>(M);
        case 16: return pick_m<16>(M);
        case 20: return pick_m<20>(M);
        case 24: return pick_m<24>(M);
        case 28: return pick_m<28>(M);
        case 32: return pick_m<32>(M);
    }
    return {nullptr, 0, 0};
}

struct KnnPlan {
    bool fast = false;
    int dp = 0;        // padded row length of the scaled arrays
    int64_t n_ref_pad = 0;
    size_t off_ref = 0, off_q = 0, off_ldist = 0, off_lidx = 0, total = 0;
    TopmVariant v{};
};

template <typename T>
KnnPlan make_plan(int64_t n_ref, int64_t n_query, int d, int m, bool same) {
    KnnPlan p;
    const int M = round_m(m);
    const int D = round_d(d);
    p.fast = std::is_same<T, float>::value && M != 0 && D != 0 && !(M == 64 && D > 16);
    if (p.fast) {
        p.v = pick_topm(D, M);
        p.fast = p.v.fn != nullptr;
    }
    if (p.fast) {
        p.dp = (D + 3) / 4 * 4;
        p.n_ref_pad = (n_ref + p.v.tj - 1) / p.v.tj * p.v.tj;
    } else {
        p.dp = d;
        p.n_ref_pad = n_ref;
    }
    size_t off = 0;
    p.off_ref = off;
    off = align_up(off + (size_t)p.n_ref_pad * p.dp * sizeof(T), 256);
    p.off_q = same ? p.off_ref : off;
    if (!same) off = align_up(off + (size_t)n_query * p.dp * sizeof(T), 256);
    if (!p.fast) {
        p.off_ldist = off;
        off = align_up(off + (size_t)n_query * m * sizeof(T), 256);
        p.off_lidx = off;
        off = align_up(off + (size_t)n_query * m * sizeof(int32_t), 256);
    }
    p.total = off + 256;  // slack for base alignment
    return p;
}

template <typename T>
nngp_status knn_impl(const T *ref, int64_t n_ref, const T *query, int64_t n_query, int d, const double *ls,
                     int n_ls, int m, int has_cut, int64_t cut, int32_t *out, int32_t *flags, void *ws,
                     size_t ws_bytes, cudaStream_t stream) {
    if (n_ref < 0 || n_query < 0 || d <= 0 || m < 0) return fail(NNGP_ERR_INVALID_ARGUMENT, "knn: negative size or d <= 0");
    if (d > kMaxDim) return fail(NNGP_ERR_UNSUPPORTED, "knn: d > 256 is not supported");
    if (n_ref > INT32_MAX - 1 || n_query > INT32_MAX - 1) return fail(NNGP_ERR_UNSUPPORTED, "knn: more than 2^31-2 points");
    if (n_query == 0 || m == 0) return NNGP_OK;
    if (!query || !out || (n_ref > 0 && !ref)) return fail(NNGP_ERR_INVALID_ARGUMENT, "knn: null pointer");
    if (ls && n_ls != 1 && n_ls != d) return fail(NNGP_ERR_INVALID_ARGUMENT, "knn: n_ls must be 1 or d");
    if (n_ref == 0) {
        NNGP_CUDA_TRY(cudaMemsetAsync(out, 0xff, (size_t)n_query * m * sizeof(int32_t), stream));
        return NNGP_OK;
    }
    const bool same = (ref == query) && (n_ref == n_query);
    KnnPlan p = make_plan<T>(n_ref, n_query, d, m, same);
    if (!ws || ws_bytes < p.total) return fail(NNGP_ERR_WORKSPACE, "knn: workspace missing or too small");
    char *base = reinterpret_cast<char *>(align_up(reinterpret_cast<uintptr_t>(ws), 256));
    T *refs = reinterpret_cast<T *>(base + p.off_ref);
    T *qsc = reinterpret_cast<T *>(base + p.off_q);

    LsParam<T> lp;
    for (int f = 0; f < d; ++f) lp.v[f] = ls ? (T)(n_ls == 1 ? ls[0] : ls[f]) : T(1);
    const int use_ls = ls != nullptr;
    {
        const int64_t tot = p.n_ref_pad * p.dp;
        const int grid = (int)std::min<int64_t>((tot + 255) / 256, 148 * 16);
        scale_pad_kernel<T><<<grid, 256, 0, stream>>>(ref, n_ref, d, p.dp, p.n_ref_pad, lp, use_ls, refs);
        NNGP_CUDA_TRY(cudaGetLastError());
        if (!same) {
            const int64_t totq = n_query * p.dp;
            const int gq = (int)std::min<int64_t>((totq + 255) / 256, 148 * 16);
            scale_pad_kernel<T><<<gq, 256, 0, stream>>>(query, n_query, d, p.dp, n_query, lp, use_ls, qsc);
            NNGP_CUDA_TRY(cudaGetLastError());
        }
    }
    if (p.fast) {
        const int grid = (int)((n_query + kKnnThreads - 1) / kKnnThreads);
        NNGP_CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void *>(p.v.fn),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, p.v.smem));
        void *args[] = {(void *)&refs, (void *)&qsc, (void *)&n_query, (void *)&n_ref, (void *)&has_cut,
                        (void *)&cut, (void *)&m, (void *)&out, (void *)&flags};
        NNGP_CUDA_TRY(cudaLaunchKernel(reinterpret_cast<const void *>(p.v.fn), dim3(grid), dim3(kKnnThreads), args,
                                       (size_t)p.v.smem, stream));
    } else {
        T *ldist = reinterpret_cast<T *>(base + p.off_ldist);
        int32_t *lidx = reinterpret_cast<int32_t *>(base + p.off_lidx);
        const int grid = (int)((n_query + kGenThreads - 1) / kGenThreads);
        const size_t smem = (size_t)d * kGenThreads * sizeof(T) + (size_t)kGenTile * p.dp * sizeof(T);
        NNGP_CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void *>(knn_generic_kernel<T>),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        knn_generic_kernel<T><<<grid, kGenThreads, smem, stream>>>(refs, qsc, n_query, n_ref, p.dp, d, has_cut, cut, m,
                                                                   ldist, lidx, out);
    }
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

}  // namespace

size_t knn_workspace_f32(int64_t n_ref, int64_t n_query, int d, int m) {
    if (n_ref <= 0 || n_query <= 0 || d <= 0 || m <= 0) return 256;
    return make_plan<float>(n_ref, n_query, d, m, false).total;
}
size_t knn_workspace_f64(int64_t n_ref, int64_t n_query, int d, int m) {
    if (n_ref <= 0 || n_query <= 0 || d <= 0 || m <= 0) return 256;
    return make_plan<double>(n_ref, n_query, d, m, false).total;
}

nngp_status knn_f32(const float *ref, int64_t n_ref, const float *query, int64_t n_query, int d, const double *ls,
                    int n_ls, int m, int has_cut, int64_t cut, int32_t *out, int32_t *flags, void *ws, size_t ws_bytes,
                    cudaStream_t stream) {
    return knn_impl<float>(ref, n_ref, query, n_query, d, ls, n_ls, m, has_cut, cut, out, flags, ws, ws_bytes, stream);
}
nngp_status knn_f64(const double *ref, int64_t n_ref, const double *query, int64_t n_query, int d, const double *ls,
                    int n_ls, int m, int has_cut, int64_t cut, int32_t *out, int32_t *flags, void *ws, size_t ws_bytes,
                    cudaStream_t stream) {
    return knn_impl<double>(ref, n_ref, query, n_query, d, ls, n_ls, m, has_cut, cut, out, flags, ws, ws_bytes, stream);
}

}  // namespace nngp
