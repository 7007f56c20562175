// Seed thresholds for the prefix neighbour search of the fit step.
//
// The search keeps, for every point i, the m nearest of the points j < i (calc_nn with
// ref_cut_index = 0, nngpr/cuda_kernel_accelerators.py:663-743, as called by
// nngpr/base_nngpr.py:530-535).  The tensor-core kernel streams the refs in index order and
// screens each against the row's current bound, the m-th best distance found so far; in random
// input order a row meets about m ln(i/m) list updates, and every one costs an exact rescoring
// and a heap insert.  That candidate work, not the screen, dominates the kernel at small d.
//
// Any m distinct refs j < i bound the row from above: the m-th smallest of their distances is
// >= the m-th smallest over all j < i.  This file finds such refs cheaply: two space-filling
// (Morton) orders of the scaled points, the second on a shifted grid, and for each point the
// refs within W positions of it in either order.  With the m-th smallest of those distances as
// the row's starting bound the screen passes about 40 refs per row instead of about 300 (d = 3,
// uniform data, W = 256).  The bound is computed with exactly the arithmetic of the search's
// exact rescoring, so it never excludes a true neighbour and the lists are bit-identical with or
// without seeds; only the number of candidates changes.
//
// Steps (all on the caller's stream): per-dimension bounds of the finite coordinates; 64-bit
// Morton keys (b = min(10, 64 / d) bits per dimension, interleaved) for both grids; a radix sort
// of each (CUB, key/index pairs); the inverse permutations; then one warp per point, points
// taken in curve order so that neighbouring warps read the same windows.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <string>

#include "common.cuh"
#include "knn_seed.cuh"

namespace nngp {
namespace seed {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kInfBits = 0x7F800000u;
constexpr uint32_t kTolBits = 1u << 12;  // stop the bisection within 2^12 ulp (5e-4 relative)

// monotone unsigned image of a float (for atomic min / max) and back
__device__ __forceinline__ uint32_t ord_of(float x) {
    const uint32_t u = __float_as_uint(x);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ord(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

__global__ void __launch_bounds__(kThreads) bounds_kernel(const float *__restrict__ xs, int64_t n, int d, int dp,
                                                          uint32_t *__restrict__ lo, uint32_t *__restrict__ hi) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int f = 0; f < d; ++f) {
        uint32_t mn = 0xFFFFFFFFu, mx = 0u;
        for (int64_t i = i0; i < n; i += stride) {
            const float v = xs[i * dp + f];
            if (isfinite(v)) {
                const uint32_t o = ord_of(v);
                mn = min(mn, o);
                mx = max(mx, o);
            }
        }
        mn = __reduce_min_sync(0xFFFFFFFFu, mn);
        mx = __reduce_max_sync(0xFFFFFFFFu, mx);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(lo + f, mn);
            atomicMax(hi + f, mx);
        }
    }
}

// Morton key of every point on grid `curve` (0: cells aligned with the bounds; 1: shifted by
// 1.23 % of the extent in every dimension); idx = 0..n-1.
__global__ void __launch_bounds__(kThreads) keys_kernel(const float *__restrict__ xs, int64_t n, int d, int dp,
                                                        const uint32_t *__restrict__ lo, const uint32_t *__restrict__ hi,
                                                        int bits, int curve, uint64_t *__restrict__ keys,
                                                        int32_t *__restrict__ idx) {
    float span = 0.f;
    for (int f = 0; f < d; ++f) {
        if (hi[f] >= lo[f]) span = fmaxf(span, from_ord(hi[f]) - from_ord(lo[f]));
    }
    const float cells = (float)(1u << bits);
    const float scale = span > 0.f && isfinite(span) ? 0.97f * cells / span : 0.f;
    const float shift = curve == 0 ? 0.f : 0.0123f * cells;
    const uint32_t qmax = (1u << bits) - 1u;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t key = 0;
        for (int f = 0; f < d; ++f) {
            const float base = hi[f] >= lo[f] ? from_ord(lo[f]) : 0.f;
            const float t = (xs[i * dp + f] - base) * scale + shift;
            const uint32_t q = t > 0.f ? (t < (float)qmax ? (uint32_t)t : qmax) : 0u;  // NaN -> 0
            for (int b = 0; b < bits; ++b) key |= (uint64_t)((q >> b) & 1u) << (b * d + f);
        }
        keys[i] = key;
        idx[i] = (int32_t)i;
    }
}

__global__ void __launch_bounds__(kThreads) inverse_kernel(const int32_t *__restrict__ order, int64_t n,
                                                           int32_t *__restrict__ pos) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        pos[order[k]] = (int32_t)k;
}

// Coordinates in a curve's order (row k = point order[k], dp floats) and, for curve 1, the
// curve-0 position of each of its points: the seed kernel's window reads become contiguous.
__global__ void __launch_bounds__(kThreads) gather_kernel(const float *__restrict__ xs, int64_t n, int dp,
                                                          const int32_t *__restrict__ order, float *__restrict__ xs_c) {
    const int64_t total = n * (dp / 4);
    const float4 *src = reinterpret_cast<const float4 *>(xs);
    float4 *dst = reinterpret_cast<float4 *>(xs_c);
    const int v4 = dp / 4;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / v4, v = e - k * v4;
        dst[e] = src[(int64_t)order[k] * v4 + v];
    }
}

__global__ void __launch_bounds__(kThreads) cross_pos_kernel(const int32_t *__restrict__ order1,
                                                             const int32_t *__restrict__ pos0, int64_t n,
                                                             int32_t *__restrict__ p0_of1) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        p0_of1[k] = pos0[order1[k]];
}

// Squared distance bits of the ref row r and the query coordinates qv in the search's exact
// arithmetic: ((r0 - q0)^2 + (r1 - q1)^2) + ..., every step rounded, over the D padded features.
template <int D>
__device__ __forceinline__ uint32_t dist_bits(const float *__restrict__ row, const float (&qv)[D]) {
    constexpr int V = (D + 3) / 4;
    const float4 *r4 = reinterpret_cast<const float4 *>(row);
    float r[4 * V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const float4 t = __ldg(r4 + v);
        r[4 * v] = t.x;
        r[4 * v + 1] = t.y;
        r[4 * v + 2] = t.z;
        r[4 * v + 3] = t.w;
    }
    const float t0 = sub_rn(r[0], qv[0]);
    float d2 = mul_rn(t0, t0);
#pragma unroll
    for (int f = 1; f < D; ++f) {
        const float t = sub_rn(r[f], qv[f]);
        d2 = add_rn(d2, mul_rn(t, t));
    }
    return __float_as_uint(d2);  // NaN bits lie above kInfBits and are never counted
}

// The m-th smallest of the warp's values (each lane holds N; 0xFFFFFFFF = none, NaN bits above
// kInfBits never count): bisection on the bit patterns, stopped within kTolBits above it, so
// at least m values are <= the result; kInfBits when fewer than m values are finite.
template <int N>
__device__ __forceinline__ uint32_t mth_smallest_bits(const uint32_t (&v)[N], int m) {
    constexpr unsigned FULL = 0xFFFFFFFFu;
    auto count_le = [&](uint32_t bound) -> int {
        int c = 0;
#pragma unroll
        for (int e = 0; e < N; ++e) c += v[e] <= bound ? 1 : 0;
        return (int)__reduce_add_sync(FULL, (unsigned)c);
    };
    if (count_le(kInfBits) < m) return kInfBits;
    uint32_t mn = 0xFFFFFFFFu, mx = 0u;
#pragma unroll
    for (int e = 0; e < N; ++e) {
        if (v[e] <= kInfBits) {
            mn = min(mn, v[e]);
            mx = max(mx, v[e]);
        }
    }
    uint32_t lo = __reduce_min_sync(FULL, mn), hi = __reduce_max_sync(FULL, mx);  // count_le(hi) >= m
    while (hi - lo > kTolBits) {  // invariant: count_le(hi) >= m; warp-uniform
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (count_le(mid) >= m) hi = mid;
        else lo = mid + 1;
    }
    return hi;
}

// One warp per point (taken in curve-0 order).  Lane values: squared-distance bits of the refs
// j < i in the window [p - W, p + W) of each curve (curve 1 skips refs inside curve 0's window,
// so every ref counts once); 0xFFFFFFFF for the other slots.  The row's seed is the m-th
// smallest value (bisection on the bit patterns, stopped within kTolBits above it), or +inf.
// xs0 / xs1: the coordinates in curve order; p0_of1[k] = curve-0 position of order1[k].
template <int D, int VPL>
__global__ void __launch_bounds__(kThreads) seed_kernel(const float *__restrict__ xs0, const float *__restrict__ xs1,
                                                        int64_t n, int dp, int m, const int32_t *__restrict__ order0,
                                                        const int32_t *__restrict__ order1,
                                                        const int32_t *__restrict__ p0_of1,
                                                        const int32_t *__restrict__ pos1, int combine,
                                                        int64_t row_lo, int64_t row_hi, float *__restrict__ seeds) {
    constexpr int W = VPL * 16;
    constexpr unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; k < n; k += nwarps) {
        const int64_t i = order0[k];
        if (i < row_lo || i >= row_hi) continue;  // another rank's rows (left unset)
        if (i < m) {  // fewer than m earlier points: no bound
            if (lane == 0 && !combine) seeds[i] = __uint_as_float(kInfBits);
            continue;
        }
        float qv[D];
#pragma unroll
        for (int f = 0; f < D; ++f) qv[f] = xs0[k * dp + f];
        uint32_t v[2 * VPL];
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int64_t pk = k - W + lane + 32 * t;
            uint32_t val = 0xFFFFFFFFu;
            if (pk >= 0 && pk < n) {
                const int64_t j = order0[pk];
                if (j < i) val = dist_bits<D>(xs0 + pk * dp, qv);
            }
            v[t] = val;
        }
        const int64_t p1 = pos1[i];
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int64_t pk = p1 - W + lane + 32 * t;
            uint32_t val = 0xFFFFFFFFu;
            if (pk >= 0 && pk < n) {
                const int64_t j = order1[pk];
                if (j < i) {
                    const int64_t pj = p0_of1[pk];
                    if (pj < k - W || pj >= k + W) val = dist_bits<D>(xs1 + pk * dp, qv);
                }
            }
            v[VPL + t] = val;
        }
        const uint32_t res = mth_smallest_bits<2 * VPL>(v, m);
        if (lane == 0) seeds[i] = combine ? fminf(seeds[i], __uint_as_float(res)) : __uint_as_float(res);
    }
}

// First position in keys[0, n) whose key is >= key (keys ascending).
__device__ __forceinline__ int64_t lower_bound_u64(const uint64_t *__restrict__ keys, int64_t n, uint64_t key) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Seeds of queries against refs (no prefix rule: every ref counts).  One warp per query, taken
// in curve-0 order (qorder) so that neighbouring warps read the same windows: the query's place
// in each curve of the refs (binary search of its key among the refs' sorted keys), the refs
// within W positions on either side (curve 1 skips refs inside curve 0's window), the m-th
// smallest squared distance in the search's exact arithmetic.
template <int D>
__global__ void __launch_bounds__(kThreads) qseed_kernel(const float *__restrict__ xs0, const float *__restrict__ xs1,
                                                         const uint64_t *__restrict__ keys0s,
                                                         const uint64_t *__restrict__ keys1s, int64_t n_ref,
                                                         const int32_t *__restrict__ p0_of1,
                                                         const float *__restrict__ xq, int64_t n_query,
                                                         const uint64_t *__restrict__ qkey0,
                                                         const uint64_t *__restrict__ qkey1,
                                                         const int32_t *__restrict__ qorder, int dp, int m,
                                                         float *__restrict__ seeds) {
    constexpr int VPL = 8, W = VPL * 16;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; k < n_query; k += nwarps) {
        const int64_t q = qorder[k];
        float qv[D];
#pragma unroll
        for (int f = 0; f < D; ++f) qv[f] = xq[q * dp + f];
        const int64_t c0 = lower_bound_u64(keys0s, n_ref, qkey0[q]);
        const int64_t c1 = lower_bound_u64(keys1s, n_ref, qkey1[q]);
        uint32_t v[2 * VPL];
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int64_t pk = c0 - W + lane + 32 * t;
            v[t] = (pk >= 0 && pk < n_ref) ? dist_bits<D>(xs0 + pk * dp, qv) : 0xFFFFFFFFu;
        }
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int64_t pk = c1 - W + lane + 32 * t;
            uint32_t val = 0xFFFFFFFFu;
            if (pk >= 0 && pk < n_ref) {
                const int64_t pj = p0_of1[pk];
                if (pj < c0 - W || pj >= c0 + W) val = dist_bits<D>(xs1 + pk * dp, qv);
            }
            v[VPL + t] = val;
        }
        const uint32_t res = mth_smallest_bits<2 * VPL>(v, m);
        if (lane == 0) seeds[q] = __uint_as_float(res);
    }
}

struct Layout {
    size_t keys_a, keys_b, keys0, keys1, idx0_a, idx0_b, idx1_a, idx1_b, pos0, pos1, p0of1, xs0, xs1, bounds, cub,
        cub_bytes, total;
};

Layout layout(int64_t n, int dp) {
    Layout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    L.keys_a = take((size_t)n * 8);
    L.keys_b = take((size_t)n * 8);
    L.keys0 = take((size_t)n * 8);
    L.keys1 = take((size_t)n * 8);
    L.idx0_a = take((size_t)n * 4);
    L.idx0_b = take((size_t)n * 4);
    L.idx1_a = take((size_t)n * 4);
    L.idx1_b = take((size_t)n * 4);
    L.pos0 = take((size_t)n * 4);
    L.pos1 = take((size_t)n * 4);
    L.p0of1 = take((size_t)n * 4);
    L.xs0 = take((size_t)n * dp * 4);
    L.xs1 = take((size_t)n * dp * 4);
    L.bounds = take(2 * 256 * 4);
    L.cub_bytes = align_up((size_t)(4u << 20) + (size_t)n / 2, 256);  // radix-sort scratch budget
    L.cub = take(L.cub_bytes);
    L.total = off + 256;
    return L;
}

struct SeedArgs {
    const float *xs0, *xs1;
    int64_t n;
    int dp, m;
    const int32_t *o0, *o1, *p0of1, *p1;
    int combine;
    int64_t row_lo, row_hi;
    float *seeds;
};

template <int D, int VPL>
void launch_seed(int grid, const SeedArgs &a, cudaStream_t stream) {
    seed_kernel<D, VPL><<<grid, kThreads, 0, stream>>>(a.xs0, a.xs1, a.n, a.dp, a.m, a.o0, a.o1, a.p0of1, a.p1,
                                                       a.combine, a.row_lo, a.row_hi, a.seeds);
}

template <int VPL>
bool dispatch_seed(int D, int grid, const SeedArgs &a, cudaStream_t stream) {
    switch (D) {
        case 1: launch_seed<1, VPL>(grid, a, stream); return true;
        case 2: launch_seed<2, VPL>(grid, a, stream); return true;
        case 3: launch_seed<3, VPL>(grid, a, stream); return true;
        case 4: launch_seed<4, VPL>(grid, a, stream); return true;
        case 5: launch_seed<5, VPL>(grid, a, stream); return true;
        case 6: launch_seed<6, VPL>(grid, a, stream); return true;
        case 7: launch_seed<7, VPL>(grid, a, stream); return true;
        case 8: launch_seed<8, VPL>(grid, a, stream); return true;
        case 12: launch_seed<12, VPL>(grid, a, stream); return true;
        case 16: launch_seed<16, VPL>(grid, a, stream); return true;
        case 20: launch_seed<20, VPL>(grid, a, stream); return true;
        case 24: launch_seed<24, VPL>(grid, a, stream); return true;
    }
    return false;
}

int grid_of(int64_t work) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((work + kThreads - 1) / kThreads, (int64_t)kNumSMsB200 * 8));
}


// One level: seeds of the points [0, n) from the windows of the curves of those points only
// (combine: keep the smaller of the old and the new bound).
// seeds == nullptr: only the curves (orders, inverse, sorted keys of both curves, coordinates in
// curve order), for the query seeds.
// Only the rows [row_lo, row_hi) get seeds (the others are left as they were).
nngp_status run_level(const float *xs, int64_t n, int d, int D, int dp, int m, int W, char *base, const Layout &L,
                      int combine, float *seeds, cudaStream_t stream, const int32_t **order0_out,
                      const int32_t **pos0_out, const uint64_t **keys0_out, int64_t row_lo = 0,
                      int64_t row_hi = INT64_MAX) {
    auto at = [&](size_t off) { return reinterpret_cast<void *>(base + off); };
    uint64_t *keys_a = static_cast<uint64_t *>(at(L.keys_a)), *keys_b = static_cast<uint64_t *>(at(L.keys_b));
    int32_t *idx[2][2] = {{static_cast<int32_t *>(at(L.idx0_a)), static_cast<int32_t *>(at(L.idx0_b))},
                          {static_cast<int32_t *>(at(L.idx1_a)), static_cast<int32_t *>(at(L.idx1_b))}};
    int32_t *pos[2] = {static_cast<int32_t *>(at(L.pos0)), static_cast<int32_t *>(at(L.pos1))};
    uint32_t *lo = static_cast<uint32_t *>(at(L.bounds)), *hi = lo + 256;
    const int bits = seed::bits(d);

    NNGP_CUDA_TRY(cudaMemsetAsync(lo, 0xFF, 256 * 4, stream));
    NNGP_CUDA_TRY(cudaMemsetAsync(hi, 0x00, 256 * 4, stream));
    bounds_kernel<<<grid_of(n), kThreads, 0, stream>>>(xs, n, d, dp, lo, hi);
    NNGP_CUDA_TRY(cudaGetLastError());
    const int32_t *order[2] = {nullptr, nullptr};
    for (int c = 0; c < 2; ++c) {
        keys_kernel<<<grid_of(n), kThreads, 0, stream>>>(xs, n, d, dp, lo, hi, bits, c, keys_a, idx[c][0]);
        NNGP_CUDA_TRY(cudaGetLastError());
        cub::DoubleBuffer<uint64_t> dk(keys_a, keys_b);
        cub::DoubleBuffer<int32_t> dv(idx[c][0], idx[c][1]);
        size_t need = 0;
        NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, dk, dv, (int)n, 0, bits * d, stream));
        if (need > L.cub_bytes)
            return fail(NNGP_ERR_WORKSPACE, "knn seeds: radix-sort scratch " + std::to_string(need) +
                                                " bytes exceeds the budget");
        size_t have = L.cub_bytes;
        NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(at(L.cub), have, dk, dv, (int)n, 0, bits * d, stream));
        order[c] = dv.Current();
        if ((c == 0 && keys0_out) || !seeds) {  // sorted keys, for cells along the curve or query positions
            NNGP_CUDA_TRY(cudaMemcpyAsync(at(c ? L.keys1 : L.keys0), dk.Current(), (size_t)n * 8,
                                          cudaMemcpyDeviceToDevice, stream));
        }
        inverse_kernel<<<grid_of(n), kThreads, 0, stream>>>(order[c], n, pos[c]);
        NNGP_CUDA_TRY(cudaGetLastError());
        gather_kernel<<<grid_of(n * (dp / 4)), kThreads, 0, stream>>>(xs, n, dp, order[c],
                                                                      static_cast<float *>(at(c ? L.xs1 : L.xs0)));
        NNGP_CUDA_TRY(cudaGetLastError());
    }
    int32_t *p0of1 = static_cast<int32_t *>(at(L.p0of1));
    cross_pos_kernel<<<grid_of(n), kThreads, 0, stream>>>(order[1], pos[0], n, p0of1);
    NNGP_CUDA_TRY(cudaGetLastError());
    if (order0_out) *order0_out = order[0];
    if (pos0_out) *pos0_out = pos[0];
    if (keys0_out) *keys0_out = static_cast<const uint64_t *>(at(L.keys0));
    if (!seeds) return NNGP_OK;
    const int grid = (int)std::min<int64_t>((n + kThreads / 32 - 1) / (kThreads / 32), (int64_t)kNumSMsB200 * 16);
    const SeedArgs sa{static_cast<const float *>(at(L.xs0)), static_cast<const float *>(at(L.xs1)), n, dp, m,
                      order[0], order[1], p0of1, pos[1], combine, row_lo, row_hi, seeds};
    const bool ok = W == 128 ? dispatch_seed<8>(D, grid, sa, stream) : dispatch_seed<16>(D, grid, sa, stream);
    if (!ok) return fail(NNGP_ERR_UNSUPPORTED, "knn seeds: no kernel for D = " + std::to_string(D));
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

// Query region of the query-seed workspace.
struct QLayout {
    size_t k0, k1, kb, kb2, ia, ib, cub, cub_bytes, total;
};
QLayout qlayout(int64_t nq) {
    QLayout Q{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    Q.k0 = take((size_t)nq * 8);
    Q.k1 = take((size_t)nq * 8);
    Q.kb = take((size_t)nq * 8);
    Q.kb2 = take((size_t)nq * 8);
    Q.ia = take((size_t)nq * 4);
    Q.ib = take((size_t)nq * 4);
    Q.cub_bytes = align_up((size_t)(4u << 20) + (size_t)nq / 2, 256);
    Q.cub = take(Q.cub_bytes);
    Q.total = off + 256;
    return Q;
}

template <int D>
void launch_qseed(int grid, const float *xs0, const float *xs1, const uint64_t *k0s, const uint64_t *k1s, int64_t n_ref,
                  const int32_t *p0of1, const float *xq, int64_t nq, const uint64_t *qk0, const uint64_t *qk1,
                  const int32_t *qorder, int dp, int m, float *seeds, cudaStream_t stream) {
    qseed_kernel<D><<<grid, kThreads, 0, stream>>>(xs0, xs1, k0s, k1s, n_ref, p0of1, xq, nq, qk0, qk1, qorder, dp, m,
                                                   seeds);
}

// Refinement levels: prefixes n / 8, n / 64, ... (while at least kMinPoints), run in a second
// workspace region sized for n / 8.
size_t sub_bytes(int64_t n, int dp) { return n / 8 >= kMinPoints ? layout(n / 8, dp).total : 0; }

}  // namespace

size_t workspace_query(int64_t n_ref, int64_t n_query, int dp) {
    if (n_ref < kMinPoints || n_query < 1) return 0;
    return align_up(layout(n_ref, dp).total, 256) + qlayout(n_query).total;
}

nngp_status query_seeds(const float *xs_ref, int64_t n_ref, const float *xq, int64_t n_query, int d, int D, int dp,
                        int m, void *ws, size_t ws_bytes, float *seeds, cudaStream_t stream, const int32_t **order0_out,
                        const int32_t **qorder_out) {
    if (n_ref < kMinPoints || n_query < 1 || m < 1 || d < 1 || d > 24 || D < d || dp % 4 != 0 || dp < D)
        return fail(NNGP_ERR_UNSUPPORTED, "knn query seeds: shape outside the seeded search");
    const Layout L = layout(n_ref, dp);
    if (!ws || ws_bytes < workspace_query(n_ref, n_query, dp))
        return fail(NNGP_ERR_WORKSPACE, "knn query seeds: workspace too small");
    char *base = reinterpret_cast<char *>(align_up(reinterpret_cast<uintptr_t>(ws), 256));
    const int32_t *order0 = nullptr;
    nngp_status st = run_level(xs_ref, n_ref, d, D, dp, m, 128, base, L, 0, nullptr, stream, &order0, nullptr, nullptr);
    if (st != NNGP_OK) return st;
    char *qb = base + align_up(L.total, 256);
    const QLayout Q = qlayout(n_query);
    auto qat = [&](size_t off) { return reinterpret_cast<void *>(qb + off); };
    auto at = [&](size_t off) { return reinterpret_cast<void *>(base + off); };
    const uint32_t *lo = static_cast<const uint32_t *>(at(L.bounds)), *hi = lo + 256;
    const int bits = seed::bits(d);
    uint64_t *qk0 = static_cast<uint64_t *>(qat(Q.k0)), *qk1 = static_cast<uint64_t *>(qat(Q.k1));
    int32_t *ia = static_cast<int32_t *>(qat(Q.ia));
    // the queries' keys on the refs' grids (their bounds: queries outside them clamp to the edge)
    keys_kernel<<<grid_of(n_query), kThreads, 0, stream>>>(xq, n_query, d, dp, lo, hi, bits, 1, qk1, ia);
    NNGP_CUDA_TRY(cudaGetLastError());
    keys_kernel<<<grid_of(n_query), kThreads, 0, stream>>>(xq, n_query, d, dp, lo, hi, bits, 0, qk0, ia);
    NNGP_CUDA_TRY(cudaGetLastError());
    // query order along curve 0 (sorts a copy of the keys; qk0 stays indexed by query)
    NNGP_CUDA_TRY(cudaMemcpyAsync(qat(Q.kb), qk0, (size_t)n_query * 8, cudaMemcpyDeviceToDevice, stream));
    cub::DoubleBuffer<uint64_t> dk(static_cast<uint64_t *>(qat(Q.kb)), static_cast<uint64_t *>(qat(Q.kb2)));
    cub::DoubleBuffer<int32_t> dv(ia, static_cast<int32_t *>(qat(Q.ib)));
    size_t need = 0;
    NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, dk, dv, (int)n_query, 0, bits * d, stream));
    if (need > Q.cub_bytes) return fail(NNGP_ERR_WORKSPACE, "knn query seeds: sort scratch exceeds the budget");
    size_t have = Q.cub_bytes;
    NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(qat(Q.cub), have, dk, dv, (int)n_query, 0, bits * d, stream));
    const int32_t *qorder = dv.Current();
    const int grid = (int)std::min<int64_t>((n_query + kThreads / 32 - 1) / (kThreads / 32), (int64_t)kNumSMsB200 * 16);
    const float *xs0 = static_cast<const float *>(at(L.xs0)), *xs1 = static_cast<const float *>(at(L.xs1));
    const uint64_t *k0s = static_cast<const uint64_t *>(at(L.keys0)), *k1s = static_cast<const uint64_t *>(at(L.keys1));
    const int32_t *p0of1 = static_cast<const int32_t *>(at(L.p0of1));
    switch (D) {
#define NNGP_QS(DD) \
    case DD: launch_qseed<DD>(grid, xs0, xs1, k0s, k1s, n_ref, p0of1, xq, n_query, qk0, qk1, qorder, dp, m, seeds, stream); break;
        NNGP_QS(1) NNGP_QS(2) NNGP_QS(3) NNGP_QS(4) NNGP_QS(5) NNGP_QS(6) NNGP_QS(7) NNGP_QS(8) NNGP_QS(12) NNGP_QS(16)
        NNGP_QS(20) NNGP_QS(24)
#undef NNGP_QS
        default: return fail(NNGP_ERR_UNSUPPORTED, "knn query seeds: no kernel for D = " + std::to_string(D));
    }
    NNGP_CUDA_TRY(cudaGetLastError());
    if (order0_out) *order0_out = order0;
    if (qorder_out) *qorder_out = qorder;
    return NNGP_OK;
}

size_t workspace(int64_t n, int dp) {
    return n < kMinPoints ? 0 : align_up(layout(n, dp).total, 256) + sub_bytes(n, dp);
}

int window() {
    const char *env = std::getenv("NNGP_KNN_SEED_W");
    if (!env) return 128;
    const int w = std::atoi(env);
    return (w == 0 || w == 128 || w == 256) ? w : 128;
}

nngp_status prefix_seeds(const float *xs, int64_t n, int d, int D, int dp, int m, void *ws, size_t ws_bytes,
                         float *seeds, cudaStream_t stream, const int32_t **order0_out, const int32_t **pos0_out,
                         const uint64_t **keys0_out, int64_t row_lo, int64_t row_hi) {
    const int W = window();
    if (row_hi < 0 || row_hi > n) row_hi = n;
    if (W == 0 || n < kMinPoints || m < 1 || d < 1 || d > 24 || D < d || dp % 4 != 0 || dp < D)
        return fail(NNGP_ERR_UNSUPPORTED, "knn seeds: shape outside the seeded search");
    const Layout L = layout(n, dp);
    if (!ws || ws_bytes < workspace(n, dp)) return fail(NNGP_ERR_WORKSPACE, "knn seeds: workspace too small");
    char *base = reinterpret_cast<char *>(align_up(reinterpret_cast<uintptr_t>(ws), 256));
    nngp_status st = run_level(xs, n, d, D, dp, m, W, base, L, 0, seeds, stream, order0_out, pos0_out, keys0_out,
                               row_lo, row_hi);
    if (st != NNGP_OK) return st;
    // rows i < n / 8 see few earlier points in the full windows: bound them again from the
    // curves of the prefix alone (any m earlier points bound a row; the smaller bound is kept)
    char *sub = base + align_up(L.total, 256);
    for (int64_t p = n / 8; p >= kMinPoints && p > row_lo; p /= 8) {
        st = run_level(xs, p, d, D, dp, m, W, sub, layout(p, dp), 1, seeds, stream, nullptr, nullptr, nullptr, row_lo,
                       row_hi);
        if (st != NNGP_OK) return st;
    }
    return NNGP_OK;
}

}  // namespace seed
}  // namespace nngp
