// Exact k-nearest-neighbour search on B200 (sm_100a).
//
// Semantics (reference: NngprWorker.find_nearest_neighbors, base_nngpr.py:1613-1686, and the
// CUDA calc_nn kernel, cuda_kernel_accelerators.py:663-743): for each query, the num_nn refs
// with the smallest squared distance sum_f (r_f - q_f)^2 of the length-scale-scaled points,
// ascending, equal distances ordered by lower ref index, -1 for missing slots; with a ref cut
// query q only sees refs [0, q + cut).  "Exact" means the distance of the CPU restatement:
// x / l rounded once (correctly rounded division), then per feature one rounding for the
// difference, the square and the running sum, features in order.
//
// Screened kernel (d <= 32, num_nn <= 64, float):
//   * prep kernels write, per ref, a 16-byte-aligned record [ -2 rc, |rc|^2 | r ] where r is
//     the scaled point and rc = r - c its copy centred on the ref mean c; the records are padded
//     to whole tiles so that every tile is one cp.async.bulk (TMA) copy into shared memory,
//     4-stage mbarrier ring, no multicast;
//   * one thread = one query.  Each (query, ref) pair is first SCREENED with
//     s = |rc|^2 - 2 qc.rc (d FMAs; four pairs share one compare through min): with the current
//     M-th best exact distance tau, the ref can only enter the list if
//     s < tau - |qc|^2 + eps, where eps = (4d + 16) u (|qc| + max|rc|)^2 bounds the FP32 error
//     of the screen against the exact distance (u = 2^-24).  Every ref that the exact
//     algorithm would insert passes the screen, so the lists are bit-identical;
//   * refs that pass are appended (tile-local index, one byte) to a per-thread candidate buffer
//     in shared memory and merged into the sorted top-M list in registers (exact distance,
//     unrolled compare/select insertion, strict <) in index order; merges run once per 32-ref
//     sub-block only when a lane's buffer could overflow, and once per tile otherwise.  The
//     threshold only decreases, so a candidate screened with a stale threshold is re-tested
//     exactly at merge time and the insertion sequence equals the exact scan's;
//   * top-M list: M = num_nn rounded up to 8/16/32/64; the M - num_nn leading slots hold -inf
//     and never move; prefix (fit) searches are triangular and issue the heaviest blocks first.
// Generic kernel (any d <= 256, any num_nn, float or double): exact distances, query
// coordinates in shared memory, sorted lists in the workspace.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>

#include "common.cuh"
#include "knn_prune.cuh"
#include "knn_seed.cuh"
#include "knn_tc.cuh"

namespace nngp {

constexpr int kKnnThreads = 128;
constexpr int kKnnStages = 4;
constexpr int kCandCap = 64;  // candidate-buffer entries per thread (bytes)
constexpr int kMaxDim = 256;

template <typename T> struct LsParam {
    T v[kMaxDim];
};

// dst (n_pad x dp) = src (n x d) / ls, zero padded (columns d..dp-1 and rows n..n_pad-1).  The
// length scale comes from ls (by value) or, when ls_dev is set, from device memory (n_ls values,
// each rounded to T as the host does for ls).
template <typename T>
__global__ void scale_pad_kernel(const T *__restrict__ src, int64_t n, int d, int dp, int64_t n_pad,
                                 LsParam<T> ls, int use_ls, const double *__restrict__ ls_dev, int n_ls,
                                 T *__restrict__ dst) {
    const int64_t total = n_pad * dp;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / dp;
        const int f = (int)(e - i * dp);
        T v = T(0);
        if (i < n && f < d) {
            v = src[i * d + f];
            if (use_ls) v = div_rn(v, ls_dev ? (T)ls_dev[n_ls == 1 ? 0 : f] : ls.v[f]);
        }
        dst[e] = v;
    }
}

// ---------------------------------------------------------------------------------------
// Screened kernel
// ---------------------------------------------------------------------------------------
template <int D>
struct ScreenCfg {
    static constexpr int DP = (D + 3) / 4 * 4;  // row length of the scaled arrays
    static constexpr int SP = (D + 1 + 3) / 4;  // float4s of the screening part
    static constexpr int EP = (D + 3) / 4;      // float4s of the exact part
    static constexpr int REC = SP + EP;         // float4s per ref record
    static constexpr int TJ_RAW = 16384 / (REC * 16);
    static constexpr int TJ = TJ_RAW >= 256 ? 256 : (TJ_RAW >= 128 ? 128 : (TJ_RAW >= 64 ? 64 : 32));
    static constexpr int TILE_BYTES = TJ * REC * 16;
    static constexpr int SMEM = kKnnStages * TILE_BYTES + kCandCap * kKnnThreads + 64;
};

// Per-feature sums of the scaled refs (double), for the centre c = sum / n.
__global__ void center_sum_kernel(const float *__restrict__ xs, int64_t n, int dp, int d, double *__restrict__ acc) {
    __shared__ double part[32][8];
    for (int f0 = 0; f0 < d; f0 += 8) {
        double loc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            for (int k = 0; k < 8 && f0 + k < d; ++k) loc[k] += xs[i * dp + f0 + k];
        for (int k = 0; k < 8; ++k) {
            double v = warp_sum(loc[k]);
            if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5][k] = v;
        }
        __syncthreads();
        if (threadIdx.x < 8 && f0 + threadIdx.x < d) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w][threadIdx.x];
            atomicAdd(acc + f0 + threadIdx.x, s);
        }
        __syncthreads();
    }
}

// Records [-2 rc, |rc|^2 | r] of every (padded) ref and the max of |rc|^2 (as float bits).
template <int D>
__global__ void build_records_kernel(const float *__restrict__ xs, int64_t n, int64_t n_pad,
                                     const double *__restrict__ acc, float4 *__restrict__ rec,
                                     unsigned int *__restrict__ r2max_bits) {
    using C = ScreenCfg<D>;
    float c[D];
#pragma unroll
    for (int f = 0; f < D; ++f) c[f] = n > 0 ? (float)(acc[f] / (double)n) : 0.f;
    float mx = 0.f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pad; i += (int64_t)gridDim.x * blockDim.x) {
        float sv[C::SP * 4], ev[C::EP * 4];
#pragma unroll
        for (int k = 0; k < C::SP * 4; ++k) sv[k] = 0.f;
#pragma unroll
        for (int k = 0; k < C::EP * 4; ++k) ev[k] = 0.f;
        if (i < n) {
            float nr = 0.f;
#pragma unroll
            for (int f = 0; f < D; ++f) {
                const float r = xs[i * C::DP + f];
                const float rc = r - c[f];
                ev[f] = r;
                sv[f] = -2.f * rc;
                nr = fmaf(rc, rc, nr);
            }
            sv[D] = nr;
            mx = fmaxf(mx, nr);
        }
        float4 *o = rec + i * C::REC;
#pragma unroll
        for (int k = 0; k < C::SP; ++k) o[k] = make_float4(sv[4 * k], sv[4 * k + 1], sv[4 * k + 2], sv[4 * k + 3]);
#pragma unroll
        for (int k = 0; k < C::EP; ++k) o[C::SP + k] = make_float4(ev[4 * k], ev[4 * k + 1], ev[4 * k + 2], ev[4 * k + 3]);
    }
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 8));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    if ((threadIdx.x & 31) == 0) atomicMax(r2max_bits, __float_as_uint(mx));  // non-negative floats order as uints
}

template <int M>
__device__ __forceinline__ void topm_insert(float (&dist)[M], int32_t (&idx)[M], float d2, int32_t j) {
#pragma unroll
    for (int k = M - 1; k > 0; --k) {
        const bool sh = d2 < dist[k - 1];
        const bool here = d2 < dist[k];
        const float nd = sh ? dist[k - 1] : (here ? d2 : dist[k]);
        const int32_t ni = sh ? idx[k - 1] : (here ? j : idx[k]);
        dist[k] = nd;
        idx[k] = ni;
    }
    if (d2 < dist[0]) {
        dist[0] = d2;
        idx[0] = j;
    }
}

template <int D>
__device__ __forceinline__ float screen_score(const float4 *__restrict__ rec, const float (&qc)[D]) {
    using C = ScreenCfg<D>;
    float sv[C::SP * 4];
#pragma unroll
    for (int k = 0; k < C::SP; ++k) {
        const float4 v = rec[k];
        sv[4 * k] = v.x; sv[4 * k + 1] = v.y; sv[4 * k + 2] = v.z; sv[4 * k + 3] = v.w;
    }
    float s = sv[D];
#pragma unroll
    for (int f = 0; f < D; ++f) s = fmaf(qc[f], sv[f], s);
    return s;
}

template <int D>
__device__ __forceinline__ float exact_d2(const float4 *__restrict__ rec, const float (&qo)[D]) {
    using C = ScreenCfg<D>;
    float ev[C::EP * 4];
#pragma unroll
    for (int k = 0; k < C::EP; ++k) {
        const float4 v = rec[C::SP + k];
        ev[4 * k] = v.x; ev[4 * k + 1] = v.y; ev[4 * k + 2] = v.z; ev[4 * k + 3] = v.w;
    }
    const float t0 = sub_rn(ev[0], qo[0]);
    float d2 = mul_rn(t0, t0);
#pragma unroll
    for (int f = 1; f < D; ++f) {
        const float t = sub_rn(ev[f], qo[f]);
        d2 = add_rn(d2, mul_rn(t, t));
    }
    return d2;
}

template <int D, int M>
__global__ void __launch_bounds__(kKnnThreads) knn_screen_kernel(const float4 *__restrict__ recs,
                                                                 const float *__restrict__ qs,
                                                                 const double *__restrict__ acc,
                                                                 const unsigned int *__restrict__ r2max_bits,
                                                                 int64_t n_query, int64_t n_ref, int has_cut,
                                                                 int64_t cut, int m, int32_t *__restrict__ out,
                                                                 int32_t *__restrict__ flags) {
    using C = ScreenCfg<D>;
    constexpr int TJ = C::TJ;
    constexpr int REC = C::REC;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float4 *tiles = reinterpret_cast<float4 *>(smem_raw);
    uint8_t *cbuf = smem_raw + kKnnStages * C::TILE_BYTES;  // [kCandCap][kKnnThreads]
    uint64_t *full = reinterpret_cast<uint64_t *>(smem_raw + kKnnStages * C::TILE_BYTES + kCandCap * kKnnThreads);

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
    const int64_t block_limit = limit_of(min(q0 + kKnnThreads, n_query) - 1);
    const int64_t ntiles = (block_limit + TJ - 1) / TJ;

    // query: exact scaled coordinates, centred copy, screening threshold offset
    float qo[D], qc[D];
    float nq = 0.f;
    {
        const float4 *qp = reinterpret_cast<const float4 *>(qs + (active ? q : 0) * C::DP);
#pragma unroll
        for (int k = 0; k < C::DP / 4; ++k) {
            const float4 v = qp[k];
            if (4 * k + 0 < D) qo[4 * k + 0] = v.x;
            if (4 * k + 1 < D) qo[4 * k + 1] = v.y;
            if (4 * k + 2 < D) qo[4 * k + 2] = v.z;
            if (4 * k + 3 < D) qo[4 * k + 3] = v.w;
        }
#pragma unroll
        for (int f = 0; f < D; ++f) {
            const float cf = n_ref > 0 ? (float)(acc[f] / (double)n_ref) : 0.f;
            qc[f] = qo[f] - cf;
            nq = fmaf(qc[f], qc[f], nq);
        }
    }
    const float rmax = sqrtf(__uint_as_float(*r2max_bits)) * 1.0001f;
    const float span = sqrtf(nq) * 1.0001f + rmax;
    const float eps = (float)(4 * D + 16) * 5.9604645e-8f * span * span;

    float dist[M];
    int32_t idx[M];
#pragma unroll
    for (int k = 0; k < M; ++k) {
        dist[k] = (k < M - m) ? neg_inf<float>() : pos_inf<float>();
        idx[k] = -1;
    }
    float tq = pos_inf<float>();  // screening threshold: tau - |qc|^2 + eps
    int cnt = 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kKnnStages; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int s = 0; s < kKnnStages && s < ntiles; ++s) {
            mbar_arrive_expect_tx(&full[s], C::TILE_BYTES);
            tma_bulk_g2s(tiles + s * (TJ * REC), recs + (int64_t)s * TJ * REC, C::TILE_BYTES, &full[s]);
        }
    }

    auto merge = [&](const float4 *T, int64_t j0) {
        for (int k = 0; k < cnt; ++k) {
            const int jj = cbuf[k * kKnnThreads + threadIdx.x];
            const float d2 = exact_d2<D>(T + jj * REC, qo);
            if (d2 < dist[M - 1]) topm_insert<M>(dist, idx, d2, (int32_t)(j0 + jj));
        }
        cnt = 0;
        tq = (dist[M - 1] - nq) + eps;
    };

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
        const float4 *T = tiles + s * (TJ * REC);
        const int64_t j0 = t * TJ;
        const int64_t jn64 = limit - j0;
        const int jn = jn64 >= TJ ? TJ : (jn64 > 0 ? (int)jn64 : 0);  // refs of this tile the query may use
        if (__all_sync(FULL, jn == TJ)) {
            // whole tile allowed for every lane of the warp
            for (int sb = 0; sb < TJ; sb += 32) {
#pragma unroll 2
                for (int g = 0; g < 32; g += 4) {
                    const int jj = sb + g;
                    const float s0 = screen_score<D>(T + (jj + 0) * REC, qc);
                    const float s1 = screen_score<D>(T + (jj + 1) * REC, qc);
                    const float s2 = screen_score<D>(T + (jj + 2) * REC, qc);
                    const float s3 = screen_score<D>(T + (jj + 3) * REC, qc);
                    if (fminf(fminf(s0, s1), fminf(s2, s3)) < tq) {
                        if (s0 < tq) cbuf[(cnt++) * kKnnThreads + threadIdx.x] = (uint8_t)(jj + 0);
                        if (s1 < tq) cbuf[(cnt++) * kKnnThreads + threadIdx.x] = (uint8_t)(jj + 1);
                        if (s2 < tq) cbuf[(cnt++) * kKnnThreads + threadIdx.x] = (uint8_t)(jj + 2);
                        if (s3 < tq) cbuf[(cnt++) * kKnnThreads + threadIdx.x] = (uint8_t)(jj + 3);
                    }
                }
                if (__any_sync(FULL, cnt > kCandCap - 32)) merge(T, j0);
            }
        } else {
            // boundary tile of the prefix search: per-lane limit jn
            for (int sb = 0; sb < TJ; sb += 32) {
                for (int g = 0; g < 32; ++g) {
                    const int jj = sb + g;
                    const float s0 = screen_score<D>(T + jj * REC, qc);
                    if (s0 < tq && jj < jn) cbuf[(cnt++) * kKnnThreads + threadIdx.x] = (uint8_t)jj;
                }
                if (__any_sync(FULL, cnt > kCandCap - 32)) merge(T, j0);
            }
        }
        if (__any_sync(FULL, cnt > 0)) merge(T, j0);
        __syncthreads();  // every thread is done with stage s before it is refilled
        if (threadIdx.x == 0 && t + kKnnStages < ntiles) {
            mbar_arrive_expect_tx(&full[s], C::TILE_BYTES);
            tma_bulk_g2s(tiles + s * (TJ * REC), recs + (t + kKnnStages) * TJ * REC, C::TILE_BYTES, &full[s]);
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
    extern __shared__ __align__(128) unsigned char smem_raw[];
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

using ScreenFn = void (*)(const float4 *, const float *, const double *, const unsigned int *, int64_t, int64_t, int,
                          int64_t, int, int32_t *, int32_t *);
using RecordFn = void (*)(const float *, int64_t, int64_t, const double *, float4 *, unsigned int *);

struct ScreenVariant {
    ScreenFn fn = nullptr;
    RecordFn rec = nullptr;
    int smem = 0, tj = 0, rec_f4 = 0, dp = 0;
};

template <int D, int M> ScreenVariant make_variant() {
    using C = ScreenCfg<D>;
    ScreenVariant v;
    v.fn = knn_screen_kernel<D, M>;
    v.rec = build_records_kernel<D>;
    v.smem = C::SMEM;
    v.tj = C::TJ;
    v.rec_f4 = C::REC;
    v.dp = C::DP;
    return v;
}

template <int D> ScreenVariant pick_m(int M) {
    switch (M) {
        case 8: return make_variant<D, 8>();
        case 16: return make_variant<D, 16>();
        case 32: return make_variant<D, 32>();
        case 64: return make_variant<D, 64>();
    }
    return ScreenVariant{};
}

ScreenVariant pick_screen(int D, int M) {
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
    return ScreenVariant{};
}

enum class KnnPath { Tc, Simt, Generic };

// Search kernel: the tensor-core screen where the shape has a variant (FP32, d <= 24 apart
// from 9-11 padded to 12 etc., num_nn <= 32), else the SIMT screen, else the generic kernel.  NNGP_KNN_KERNEL=tc|simt|generic forces a
// kernel where the shape has one (testing and comparisons); unset or any other value selects
// automatically.
KnnPath choose_path(int d, int m, bool is_float) {
    const char *env = std::getenv("NNGP_KNN_KERNEL");
    const std::string want = env ? env : "auto";
    const int M = round_m(m), D = round_d(d);
    const bool tc_ok = is_float && D != 0 && M != 0 && M <= 32 && tc_variant(D, M).fn != nullptr;
    const bool simt_ok = is_float && D != 0 && M != 0 && !(M == 64 && D > 16);
    if (want == "generic") return KnnPath::Generic;
    if (want == "simt") return simt_ok ? KnnPath::Simt : KnnPath::Generic;
    if (want == "tc" && tc_ok) return KnnPath::Tc;
    if (tc_ok) return KnnPath::Tc;  // faster than the SIMT screen at every d measured on B200 (3, 8, 16)
    return simt_ok ? KnnPath::Simt : KnnPath::Generic;
}

struct KnnPlan {
    KnnPath path = KnnPath::Generic;
    int dp = 0;  // padded row length of the scaled arrays
    int64_t n_ref_pad = 0;
    size_t off_ref = 0, off_q = 0, off_rec = 0, off_acc = 0, off_r2 = 0, off_ctr = 0, off_ldist = 0, off_lidx = 0,
           off_seed = 0, off_seed_ws = 0, seed_ws_bytes = 0, off_tiles2 = 0, off_prune_ws = 0, prune_ws_bytes = 0,
           total = 0;
    ScreenVariant v{};
    tc::TcVariant tv{};
};

template <typename T>
KnnPlan make_plan(int64_t n_ref, int64_t n_query, int d, int m, bool same) {
    KnnPlan p;
    const int M = round_m(m);
    const int D = round_d(d);
    p.path = choose_path(d, m, std::is_same<T, float>::value);
    if (p.path == KnnPath::Tc) {
        p.tv = tc_variant(D, M);
        p.dp = p.tv.dp;
        p.n_ref_pad = (n_ref + tc::kTcRefTile - 1) / tc::kTcRefTile * tc::kTcRefTile;
    } else if (p.path == KnnPath::Simt) {
        p.v = pick_screen(D, M);
        p.dp = p.v.dp;
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
    if (p.path != KnnPath::Generic) {
        p.off_rec = off;
        const size_t rec_bytes = p.path == KnnPath::Tc ? (size_t)(p.n_ref_pad / tc::kTcRefTile) * p.tv.stage_bytes
                                                        : (size_t)p.n_ref_pad * p.v.rec_f4 * 16;
        off = align_up(off + rec_bytes, 1024);
        p.off_acc = off;
        off = align_up(off + (size_t)kMaxDim * sizeof(double), 256);
        p.off_r2 = off;
        off = align_up(off + 16, 256);
        p.off_ctr = off;
        off = align_up(off + 16, 256);
        // seeds and pruned lists: of the prefix search (same) or, for other queries, of the query
        // search (the size query plans with same = false and takes the larger of the two)
        const size_t seed_ws = p.path != KnnPath::Tc ? 0
                               : std::max(seed::workspace(n_ref, p.dp),
                                          same ? (size_t)0 : seed::query_workspace_if(n_ref, n_query, p.dp));
        if (seed_ws > 0) {
            p.off_seed = off;
            off = align_up(off + (size_t)std::max(n_ref, n_query) * sizeof(float), 256);
            p.off_seed_ws = off;
            p.seed_ws_bytes = seed_ws;
            off = align_up(off + p.seed_ws_bytes, 256);
            const int G = p.tv.rows_per_item;
            const size_t prune_ws = std::max(prune::workspace(n_ref, d, G),
                                             same ? (size_t)0 : prune::workspace_query(n_ref, n_query, d, G));
            if (prune_ws > 0) {  // pruned search: curve-order tiles + lists
                p.off_tiles2 = align_up(off, 1024);
                off = align_up(p.off_tiles2 + rec_bytes, 1024);
                p.off_prune_ws = off;
                p.prune_ws_bytes = prune_ws;
                off = align_up(off + p.prune_ws_bytes, 256);
            }
        }
    } else {
        p.off_ldist = off;
        off = align_up(off + (size_t)n_query * m * sizeof(T), 256);
        p.off_lidx = off;
        off = align_up(off + (size_t)n_query * m * sizeof(int32_t), 256);
    }
    p.total = off + 1024;  // slack for base alignment
    return p;
}

int num_sms_knn() {
    static int cached = 0;
    if (!cached) {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
            cached = v;
        else
            cached = kNumSMsB200;
    }
    return cached;
}

int grid_for(int64_t work, int per_block = 256) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((work + per_block - 1) / per_block, (int64_t)kNumSMsB200 * 16));
}

// ls_device: ls points to device memory (read by the scaling kernel), else to host memory
template <typename T>
nngp_status knn_impl(const T *ref, int64_t n_ref, const T *query, int64_t n_query, int d, const double *ls,
                     int n_ls, int m, int has_cut, int64_t cut, int32_t *out, int32_t *flags, void *ws,
                     size_t ws_bytes, cudaStream_t stream, bool ls_device = false) {
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
    char *base = reinterpret_cast<char *>(align_up(reinterpret_cast<uintptr_t>(ws), 1024));
    T *refs = reinterpret_cast<T *>(base + p.off_ref);
    T *qsc = reinterpret_cast<T *>(base + p.off_q);

    LsParam<T> lp;
    for (int f = 0; f < d; ++f) lp.v[f] = (ls && !ls_device) ? (T)(n_ls == 1 ? ls[0] : ls[f]) : T(1);
    const int use_ls = ls != nullptr;
    const double *ls_dev = ls_device ? ls : nullptr;
    scale_pad_kernel<T><<<grid_for(p.n_ref_pad * p.dp), 256, 0, stream>>>(ref, n_ref, d, p.dp, p.n_ref_pad, lp, use_ls,
                                                                          ls_dev, n_ls, refs);
    NNGP_CUDA_TRY(cudaGetLastError());
    if (!same) {
        scale_pad_kernel<T><<<grid_for(n_query * p.dp), 256, 0, stream>>>(query, n_query, d, p.dp, n_query, lp,
                                                                          use_ls, ls_dev, n_ls, qsc);
        NNGP_CUDA_TRY(cudaGetLastError());
    }
    if (p.path == KnnPath::Tc) {
        if constexpr (std::is_same<T, float>::value) {
            double *acc = reinterpret_cast<double *>(base + p.off_acc);
            unsigned int *r2 = reinterpret_cast<unsigned int *>(base + p.off_r2);
            int *ctr = reinterpret_cast<int *>(base + p.off_ctr);
            unsigned char *tiles = reinterpret_cast<unsigned char *>(base + p.off_rec);
            NNGP_CUDA_TRY(cudaMemsetAsync(base + p.off_acc, 0, p.off_ctr + 16 - p.off_acc, stream));
            center_sum_kernel<<<grid_for(n_ref), 256, 0, stream>>>(refs, n_ref, p.dp, d, acc);
            NNGP_CUDA_TRY(cudaGetLastError());
            const int32_t *no_perm = nullptr;
            p.tv.build<<<grid_for(p.n_ref_pad), 256, 0, stream>>>(refs, n_ref, p.n_ref_pad, acc, no_perm, tiles, r2);
            NNGP_CUDA_TRY(cudaGetLastError());
            NNGP_CUDA_TRY(ensure_smem_limit(reinterpret_cast<const void *>(p.tv.fn), p.tv.smem, 100));
            // the prefix search of a point set over itself (the fit step) starts every row from a
            // proven bound of its m-th distance: the same lists, far fewer candidates.  A row shard
            // of it (query = rows [cut, cut + n_query) of ref, as a view: the multi-GPU fit step)
            // takes the same path for its rows.
            const bool shard = !same && has_cut && cut >= 0 && cut + n_query <= n_ref &&
                               query == ref + (size_t)cut * (size_t)d;
            const int64_t row_lo = shard ? cut : 0;  // the searched rows are the points [row_lo, row_lo + n_query)
            const bool seeded = ((same && has_cut && cut == 0) || shard) && seed::workspace(n_ref, p.dp) > 0 &&
                                p.seed_ws_bytes >= seed::workspace(n_ref, p.dp) && seed::window() > 0;
            const float *seeds_c = nullptr;
            const int32_t *order0 = nullptr, *pos0 = nullptr;
            const uint64_t *keys0 = nullptr;
            if (seeded) {
                float *sd = reinterpret_cast<float *>(base + p.off_seed);
                nngp_status sst = seed::prefix_seeds(refs, n_ref, d, round_d(d), p.dp, m, base + p.off_seed_ws,
                                                     p.seed_ws_bytes, sd, stream, &order0, &pos0, &keys0, row_lo,
                                                     row_lo + n_query);
                if (sst != NNGP_OK) return sst;
                seeds_c = sd;
            }
            // queries against the set (predict): seeds from the refs' curve windows around each
            // query, and (d <= 24) groups of queries in curve order with their tile lists
            const int G = p.tv.rows_per_item;
            const int32_t *qorder = nullptr;
            const bool qseeded = !same && !has_cut && seed::window() > 0 && seed::query_workspace_if(n_ref, n_query, p.dp) > 0 &&
                                 p.seed_ws_bytes >= seed::workspace_query(n_ref, n_query, p.dp);
            if (qseeded) {
                float *sd = reinterpret_cast<float *>(base + p.off_seed);
                nngp_status sst = seed::query_seeds(refs, n_ref, qsc, n_query, d, round_d(d), p.dp, m,
                                                    base + p.off_seed_ws, p.seed_ws_bytes, sd, stream, &order0, &qorder);
                if (sst != NNGP_OK) return sst;
                seeds_c = sd;
            }
            const size_t qprune_ws = qseeded ? prune::workspace_query(n_ref, n_query, d, G) : 0;
            const bool qpruned = qseeded && qprune_ws > 0 && p.prune_ws_bytes >= qprune_ws && prune::enabled();
            // and, for large sets (d <= 24), visits per group of rows only the ref tiles its seeds
            // allow (rows and refs in curve order; loose and early rows stay in index order, and all
            // rows go back to it on the device when the lists exclude too little)
            const bool pruned = seeded && prune::workspace(n_ref, d, G) > 0 &&
                                p.prune_ws_bytes >= prune::workspace(n_ref, d, G) && prune::enabled();
            prune::Lists lists;
            unsigned char *tiles_curve = reinterpret_cast<unsigned char *>(base + p.off_tiles2);
            if (qpruned) {
                nngp_status pst = prune::build_query(refs, n_ref, qsc, n_query, d, p.dp, G, seeds_c, order0, qorder,
                                                     base + p.off_prune_ws, p.prune_ws_bytes, &lists, stream);
                if (pst != NNGP_OK) return pst;
                p.tv.build<<<grid_for(p.n_ref_pad), 256, 0, stream>>>(refs, n_ref, p.n_ref_pad, acc, order0, tiles_curve,
                                                                      r2);
                NNGP_CUDA_TRY(cudaGetLastError());
            }
            if (pruned) {
                nngp_status pst = prune::build(refs, n_ref, row_lo, row_lo + n_query, d, p.dp, p.tv.rows_per_item,
                                               seed::bits(d), seeds_c, order0, pos0, keys0, base + p.off_prune_ws,
                                               p.prune_ws_bytes, &lists, stream);
                if (pst != NNGP_OK) return pst;
                p.tv.build<<<grid_for(p.n_ref_pad), 256, 0, stream>>>(refs, n_ref, p.n_ref_pad, acc, lists.ref_order,
                                                                      tiles_curve, r2);
                NNGP_CUDA_TRY(cudaGetLastError());
                if (const char *dbg = std::getenv("NNGP_KNN_DEBUG"); dbg && dbg[0] == '1') {
                    prune::DevSizes hs[2];  // diagnostics only (synchronises the stream)
                    int32_t total = 0;
                    NNGP_CUDA_TRY(cudaMemcpyAsync(hs, lists.pruned, sizeof(hs), cudaMemcpyDeviceToHost, stream));
                    NNGP_CUDA_TRY(cudaStreamSynchronize(stream));
                    NNGP_CUDA_TRY(cudaMemcpyAsync(&total, lists.offsets + hs[0].n_groups, sizeof(total),
                                                  cudaMemcpyDeviceToHost, stream));
                    NNGP_CUDA_TRY(cudaStreamSynchronize(stream));
                    std::fprintf(stderr,
                                 "nngp_knn: pruned rows=%lld groups=%lld items=%lld tiles listed=%d (%.1f per group of "
                                 "%lld); index-order rows=%lld items=%lld\n",
                                 (long long)hs[0].n_rows, (long long)hs[0].n_groups, (long long)hs[0].n_items, total,
                                 (double)total / (double)std::max<int64_t>(1, hs[0].n_groups),
                                 (long long)(p.n_ref_pad / tc::kTcRefTile), (long long)hs[1].n_rows,
                                 (long long)hs[1].n_items);
                }
            }
            // persistent grid: the CTAs one SM holds (shared memory and TMEM sized for them) per SM;
            // CTAs that find no SM free start late and pick up no items, nothing waits on them
            const int per_sm = p.tv.ctas_per_sm;
            const float *q_c = qsc;
            const double *acc_c = acc;
            const unsigned int *r2_c = r2;
            const int32_t *none = nullptr;
            const int64_t *no_sizes = nullptr;
            const uint64_t wait_ns = wait_limit_ns();
            // cut_arg / out_base: rows of point indices use cut 0 (limit = the point's index) and
            // write the row of point i at out[(i - out_base) * m]
            auto launch = [&](const unsigned char *tiles_c, int64_t items_bound, const int32_t *rows_perm,
                              const int32_t *row_off, const int64_t *dev_sizes, const tc::TcItems &items,
                              const int32_t *ref_perm, const int32_t *tile_off, const int32_t *tile_list,
                              int *counter, const float *seeds_arg, int64_t cut_arg, int64_t out_base,
                              const float *q_arg) -> nngp_status {
                if (items_bound == 0) return NNGP_OK;
                const int grid = (int)std::min<int64_t>(items_bound, (int64_t)num_sms_knn() * per_sm);
                if (const char *dbg = std::getenv("NNGP_KNN_DEBUG"); dbg && dbg[0] == '1')
                    std::fprintf(stderr,
                                 "nngp_knn: tensor-core path d=%d m=%d items<=%lld ctas/sm=%d grid=%d smem=%d seeded=%d "
                                 "pruned=%d\n",
                                 d, m, (long long)items_bound, per_sm, grid, p.tv.smem, (int)(seeded || qseeded),
                                 (int)(tile_list != nullptr));
                void *args[] = {(void *)&tiles_c,  (void *)&q_arg,     (void *)&acc_c,      (void *)&r2_c,
                                (void *)&seeds_arg, (void *)&rows_perm, (void *)&row_off,  (void *)&dev_sizes,
                                (void *)&items,    (void *)&ref_perm, (void *)&tile_off, (void *)&tile_list,
                                (void *)&counter,  (void *)&n_query,  (void *)&n_ref,      (void *)&has_cut,
                                (void *)&cut_arg,  (void *)&m,        (void *)&out_base,   (void *)&out,
                                (void *)&flags,    (void *)&wait_ns};
                NNGP_CUDA_TRY(cudaLaunchKernel(reinterpret_cast<const void *>(p.tv.fn), dim3(grid), dim3(p.tv.threads),
                                               args, (size_t)p.tv.smem, stream));
                return NNGP_OK;
            };
            nngp_status lst;
            if (pruned) {
                const int64_t *ps = reinterpret_cast<const int64_t *>(lists.pruned);
                const int64_t *is = reinterpret_cast<const int64_t *>(lists.index_order);
                // rows are point indices (the refs' scaled copy holds them), cut 0, shard offset
                const float *pts = refs;
                lst = launch(tiles_curve, lists.max_items[0], lists.rows, lists.row_off, ps, lists.pruned_items,
                             lists.ref_order, lists.offsets, lists.tiles, ctr + 1, seeds_c, 0, row_lo, pts);
                if (lst != NNGP_OK) return lst;
                if ((lst = prune::merge(lists, 0, p.tv.rows_per_item, m, row_lo, out, stream)) != NNGP_OK) return lst;
                lst = launch(tiles, lists.max_items[1], lists.rows, none, is, lists.index_items, none, none, none, ctr,
                             seeds_c, 0, row_lo, pts);
                if (lst != NNGP_OK) return lst;
                lst = prune::merge(lists, 1, p.tv.rows_per_item, m, row_lo, out, stream);
            } else if (qpruned) {
                const int64_t *ps = reinterpret_cast<const int64_t *>(lists.pruned);
                lst = launch(tiles_curve, lists.max_items[0], lists.rows, lists.row_off, ps, lists.pruned_items,
                             lists.ref_order, lists.offsets, lists.tiles, ctr + 1, seeds_c, cut, 0, q_c);
                if (lst != NNGP_OK) return lst;
                lst = prune::merge(lists, 0, G, m, 0, out, stream);
            } else {
                // rows are query rows (limit = row + cut); a seeded shard's seeds are indexed by point
                const int64_t items = (n_query + p.tv.rows_per_item - 1) / p.tv.rows_per_item;
                const tc::TcItems whole{};
                const float *seeds_rows = seeds_c ? seeds_c + row_lo : nullptr;
                lst = launch(tiles, items, none, none, no_sizes, whole, none, none, none, ctr, seeds_rows, cut, 0, q_c);
            }
            if (lst != NNGP_OK) return lst;
        }
    } else if (p.path == KnnPath::Simt) {
        if constexpr (std::is_same<T, float>::value) {
            double *acc = reinterpret_cast<double *>(base + p.off_acc);
            unsigned int *r2 = reinterpret_cast<unsigned int *>(base + p.off_r2);
            float4 *recs = reinterpret_cast<float4 *>(base + p.off_rec);
            NNGP_CUDA_TRY(cudaMemsetAsync(base + p.off_acc, 0, p.off_r2 + 16 - p.off_acc, stream));
            center_sum_kernel<<<grid_for(n_ref), 256, 0, stream>>>(refs, n_ref, p.dp, d, acc);
            NNGP_CUDA_TRY(cudaGetLastError());
            p.v.rec<<<grid_for(p.n_ref_pad), 256, 0, stream>>>(refs, n_ref, p.n_ref_pad, acc, recs, r2);
            NNGP_CUDA_TRY(cudaGetLastError());
            const int grid = (int)((n_query + kKnnThreads - 1) / kKnnThreads);
            NNGP_CUDA_TRY(ensure_smem_limit(reinterpret_cast<const void *>(p.v.fn), p.v.smem));
            const float4 *recs_c = recs;
            const float *q_c = qsc;
            const double *acc_c = acc;
            const unsigned int *r2_c = r2;
            void *args[] = {(void *)&recs_c, (void *)&q_c, (void *)&acc_c, (void *)&r2_c, (void *)&n_query,
                            (void *)&n_ref, (void *)&has_cut, (void *)&cut, (void *)&m, (void *)&out, (void *)&flags};
            NNGP_CUDA_TRY(cudaLaunchKernel(reinterpret_cast<const void *>(p.v.fn), dim3(grid), dim3(kKnnThreads), args,
                                           (size_t)p.v.smem, stream));
        }
    } else {
        T *ldist = reinterpret_cast<T *>(base + p.off_ldist);
        int32_t *lidx = reinterpret_cast<int32_t *>(base + p.off_lidx);
        const int grid = (int)((n_query + kGenThreads - 1) / kGenThreads);
        const size_t smem = (size_t)d * kGenThreads * sizeof(T) + (size_t)kGenTile * p.dp * sizeof(T);
        NNGP_CUDA_TRY(ensure_smem_limit(reinterpret_cast<const void *>(knn_generic_kernel<T>), (int)smem));
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
nngp_status knn_f32_ls_device(const float *ref, int64_t n_ref, const float *query, int64_t n_query, int d,
                              const double *ls_dev, int n_ls, int m, int has_cut, int64_t cut, int32_t *out,
                              int32_t *flags, void *ws, size_t ws_bytes, cudaStream_t stream) {
    if (!ls_dev) return fail(NNGP_ERR_INVALID_ARGUMENT, "knn: the device length scale is null");
    return knn_impl<float>(ref, n_ref, query, n_query, d, ls_dev, n_ls, m, has_cut, cut, out, flags, ws, ws_bytes,
                           stream, true);
}
nngp_status knn_f64_ls_device(const double *ref, int64_t n_ref, const double *query, int64_t n_query, int d,
                              const double *ls_dev, int n_ls, int m, int has_cut, int64_t cut, int32_t *out,
                              int32_t *flags, void *ws, size_t ws_bytes, cudaStream_t stream) {
    if (!ls_dev) return fail(NNGP_ERR_INVALID_ARGUMENT, "knn: the device length scale is null");
    return knn_impl<double>(ref, n_ref, query, n_query, d, ls_dev, n_ls, m, has_cut, cut, out, flags, ws, ws_bytes,
                            stream, true);
}
nngp_status knn_f64(const double *ref, int64_t n_ref, const double *query, int64_t n_query, int d, const double *ls,
                    int n_ls, int m, int has_cut, int64_t cut, int32_t *out, int32_t *flags, void *ws, size_t ws_bytes,
                    cudaStream_t stream) {
    return knn_impl<double>(ref, n_ref, query, n_query, d, ls, n_ls, m, has_cut, cut, out, flags, ws, ws_bytes, stream);
}

}  // namespace nngp
