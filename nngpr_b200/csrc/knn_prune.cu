// Pruned prefix search: which rows go together and which ref tiles each group has to visit.
//
// The prefix search (every point i against the points j < i, calc_nn with ref_cut_index = 0,
// nngpr/cuda_kernel_accelerators.py:663-743) is brute force in the reference: n^2 / 2 pairs.
// With every row's seed (a proven upper bound of its m-th distance, knn_seed.cu) most pairs can
// be proven irrelevant in bulk: with points in space-filling-curve order, 128 consecutive points
// (a ref tile) and a group of rows are compact regions with small bounding boxes, and a ref tile
// whose box lies farther from the group's box than the largest seed of the group cannot hold a
// neighbour of any row.  The tensor-core search then streams, per group, only the listed tiles
// (d = 3, n = 434,874: about 125 tiles per group of 128 rows instead of about 1,700 on average)
// and checks j < i per candidate.
//
// Exactness: the FP32 squared distance the search compares, ((t0^2 + t1^2) + ...) with every
// step rounded and t_f = fl(x_jf - x_if), is at least (1 - u)^(D + 2) times the exact squared
// distance of the same FP32 coordinates (all terms are non-negative), minus at most
// (D + 2) 2^-150 from subnormal rounding; the box distance is at most the exact distance.  A tile
// is dropped only if box_distance^2 (1 - gamma) - 1e-37 > seed, gamma = (D + 3) 2^-23, so every
// ref in it has an FP32 distance above every row's bound and could never enter a list.  The
// left side is evaluated in FP32 with every operation rounded toward -inf (gaps, squares, sums,
// the shrink and the 1e-37), so it never exceeds its exact value and the rule stays safe.
//
// Rows: band = floor(log2(n / i)) groups rows whose prefixes differ by less than a factor of
// two, hence seeds of similar size.  A row whose seed exceeds 16 times its band's geometric mean
// (its windows held few nearby earlier points) would inflate its group's reach, so it goes to the
// index-order launch with the rows below n / 8, where it costs only its prefix.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <string>

#include "common.cuh"
#include "knn_prune.cuh"

namespace nngp {
namespace prune {
namespace {

constexpr int kThreads = 256;
constexpr int kEarlyShift = 3;       // rows below n / 8 take the index-order search
constexpr int kBands = kEarlyShift + 1;  // band b: rows [n / 2^(b + 1), n / 2^b) (the last only at rounding edges)
constexpr int kLooseLog2Q = 4 * 256;  // seed > 16 x band geometric mean (log2 in 1/256 units)
constexpr uint64_t kIndexOrderTag = 1ull << 36;  // above (band << 32 | curve position) for bands < 16
constexpr uint64_t kOutsideTag = 1ull << 37;     // rows outside the searched range: sorted last, not searched
// The pruned rows go back to index order when their tile lists hold more tiles than their
// index-order groups would stream.  Lists that exclude nothing hold about 4/3 of those tiles
// (a group in curve order needs the tiles up to its largest index, an index-order group up to
// about its mean); measured on B200 the pruned search wins up to a ratio of about 0.8 and loses
// from about 1.3 on.
constexpr double kFallbackFrac = 1.0;
constexpr int kStats = 3 * kBands + 3;  // per band: seed log sums, counts, pruned counts; index-order
                                        // count; sum of the pruned rows' indices; fallback flag

__device__ __forceinline__ int band_of(int64_t i, int64_t n) {
    int b = 0;
    while (b < kBands - 1 && (i << (b + 1)) < n) ++b;  // i < n / 2^(b + 1)
    return b;
}

// log2 of a finite non-negative seed in units of 1/256, clamped below (zero seeds: duplicates)
__device__ __forceinline__ long long log2q(float tau) {
    return llrint(fmax(log2((double)tau), -160.0) * 256.0);
}

// Box and smallest index of every ref tile (128 consecutive points of `order`); one warp per tile.
__global__ void __launch_bounds__(kThreads) tile_box_kernel(const float *__restrict__ xs, int64_t n, int d, int dp,
                                                            const int32_t *__restrict__ order, int64_t n_tiles,
                                                            float *__restrict__ tlo, float *__restrict__ thi,
                                                            int32_t *__restrict__ tmin) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; t < n_tiles; t += nw) {
        int32_t pt[kTileRefs / 32];
        int32_t mi = INT32_MAX;
#pragma unroll
        for (int q = 0; q < kTileRefs / 32; ++q) {
            const int64_t k = t * kTileRefs + q * 32 + lane;
            pt[q] = k < n ? order[k] : -1;
            if (pt[q] >= 0) mi = min(mi, pt[q]);
        }
        mi = __reduce_min_sync(0xFFFFFFFFu, mi);
        if (lane == 0) tmin[t] = mi;
        for (int f = 0; f < d; ++f) {
            float lo = pos_inf<float>(), hi = neg_inf<float>();  // NaN coordinates are skipped
#pragma unroll
            for (int q = 0; q < kTileRefs / 32; ++q) {
                if (pt[q] >= 0) {
                    const float v = xs[(int64_t)pt[q] * dp + f];
                    lo = fminf(lo, v);
                    hi = fmaxf(hi, v);
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                lo = fminf(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
                hi = fmaxf(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
            }
            if (lane == 0) {
                tlo[t * d + f] = lo;
                thi[t * d + f] = hi;
            }
        }
    }
}

// Ref order: points sorted by (index class, curve position), class = 3 - band: [0, n/8),
// [n/8, n/4), [n/4, n/2), [n/2, n).  A tile then holds refs of one class (up to the one tile at
// each class boundary), so a group of rows of band b skips whole tiles whose refs all come after
// its rows, and meets refs j > i only in its own class.
__global__ void __launch_bounds__(kThreads) ref_keys_kernel(int64_t n, const int32_t *__restrict__ pos0,
                                                            uint64_t *__restrict__ keys, int32_t *__restrict__ vals) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        keys[j] = (uint64_t)(kBands - 1 - band_of(j, n)) << 32 | (uint32_t)pos0[j];
        vals[j] = (int32_t)j;
    }
}

// Per band: sum of log2q(seed) over the finite seeds of the rows [early, row_hi) (early already
// raised to the shard's first row), and their count (integer sums: the result does not depend on
// the order of the atomics).
__global__ void __launch_bounds__(kThreads) band_stats_kernel(int64_t n, int64_t early, int64_t row_hi,
                                                              const float *__restrict__ seeds,
                                                              unsigned long long *__restrict__ sum,
                                                              unsigned long long *__restrict__ cnt) {
    long long s[kBands] = {};
    unsigned long long c[kBands] = {};
    for (int64_t i = early + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < row_hi;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float tau = seeds[i];
        if (!isinf(tau)) {
            const int b = band_of(i, n);
            s[b] += log2q(tau);
            c[b] += 1;
        }
    }
#pragma unroll
    for (int b = 0; b < kBands; ++b) {
        long long sv = s[b];
        unsigned long long cv = c[b];
        for (int o = 16; o > 0; o >>= 1) {
            sv += __shfl_xor_sync(0xFFFFFFFFu, sv, o);
            cv += __shfl_xor_sync(0xFFFFFFFFu, cv, o);
        }
        if ((threadIdx.x & 31) == 0 && cv > 0) {
            atomicAdd(sum + b, (unsigned long long)sv);  // two's complement: signed sums wrap correctly
            atomicAdd(cnt + b, cv);
        }
    }
}

// Sort keys of the rows [row_lo, row_hi): pruned rows (band << 32 | curve position), the others
// (2^36 | index); rows outside the range (2^37 | index).  Counts of pruned rows per band and of
// the index-order rows.
__global__ void __launch_bounds__(kThreads) classify_kernel(int64_t n, int64_t early, int64_t row_lo, int64_t row_hi,
                                                            const float *__restrict__ seeds,
                                                            const int32_t *__restrict__ pos0,
                                                            const unsigned long long *__restrict__ sum,
                                                            const unsigned long long *__restrict__ cnt,
                                                            uint64_t *__restrict__ keys, int32_t *__restrict__ vals,
                                                            unsigned long long *__restrict__ pruned_cnt,
                                                            unsigned long long *__restrict__ index_cnt,
                                                            unsigned long long *__restrict__ pruned_isum) {
    unsigned long long c[kBands] = {};
    unsigned long long ci = 0, si = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        vals[i] = (int32_t)i;
        if (i < row_lo || i >= row_hi) {
            keys[i] = kOutsideTag | (uint64_t)i;
            continue;
        }
        bool pruned = false;
        int b = 0;
        if (i >= early) {
            b = band_of(i, n);
            const float tau = seeds[i];
            if (!isinf(tau) && cnt[b] > 0) {
                const long long mean = (long long)sum[b] / (long long)cnt[b];
                pruned = log2q(tau) <= mean + kLooseLog2Q;
            }
        }
        keys[i] = pruned ? ((uint64_t)b << 32 | (uint32_t)pos0[i]) : (kIndexOrderTag | (uint64_t)i);
        if (pruned) {
            c[b] += 1;
            si += (unsigned long long)i;
        } else {
            ci += 1;
        }
    }
#pragma unroll
    for (int b = 0; b < kBands; ++b) {
        unsigned long long cv = c[b];
        for (int o = 16; o > 0; o >>= 1) cv += __shfl_xor_sync(0xFFFFFFFFu, cv, o);
        if ((threadIdx.x & 31) == 0 && cv > 0) atomicAdd(pruned_cnt + b, cv);
    }
    for (int o = 16; o > 0; o >>= 1) {
        ci += __shfl_xor_sync(0xFFFFFFFFu, ci, o);
        si += __shfl_xor_sync(0xFFFFFFFFu, si, o);
    }
    if ((threadIdx.x & 31) == 0 && ci > 0) atomicAdd(index_cnt, ci);
    if ((threadIdx.x & 31) == 0 && si > 0) atomicAdd(pruned_isum, si);
}

// Octree cell level of band b: cells of 2^(d L) per level hold about 256 of the band's pruned
// rows, so a band has at most cnt / 256 cells (at least one).
__device__ __forceinline__ int cell_level(unsigned long long cnt, int d, int bits) {
    int L = 0;
    while (L < bits && (cnt >> (d * (L + 1))) >= 256ull) ++L;
    return L;
}

// headpos[r] = r where a new (band, cell) segment starts among the pruned rows, else 0.
__global__ void __launch_bounds__(kThreads) segment_kernel(int64_t n, const uint64_t *__restrict__ skeys,
                                                           const int32_t *__restrict__ rows,
                                                           const int32_t *__restrict__ pos0,
                                                           const uint64_t *__restrict__ keys0,
                                                           const unsigned long long *__restrict__ pruned_cnt, int d,
                                                           int bits, int32_t *__restrict__ headpos) {
    unsigned long long total = 0;
    for (int b = 0; b < kBands; ++b) total += pruned_cnt[b];
    auto cell_of = [&](int64_t r, int b) -> uint64_t {
        const int L = cell_level(pruned_cnt[b], d, bits);
        const int shift = d * (bits - L);
        const uint64_t key = keys0[pos0[rows[r]]];
        return shift >= 64 ? 0ull : key >> shift;
    };
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        int32_t h = 0;
        if (r < (int64_t)total) {
            const int b = (int)(skeys[r] >> 32) & 15;
            bool head = r == 0;
            if (!head) {
                const int bp = (int)(skeys[r - 1] >> 32) & 15;
                head = bp != b || cell_of(r - 1, b) != cell_of(r, b);
            }
            h = head ? (int32_t)r : 0;
        }
        headpos[r] = h;
    }
}

// gh[r] = 1 where a group starts (every G rows of a segment), for the pruned rows.
__global__ void __launch_bounds__(kThreads) group_head_kernel(int64_t n, const int32_t *__restrict__ seg_start,
                                                              const unsigned long long *__restrict__ pruned_cnt, int G,
                                                              int32_t *__restrict__ gh) {
    unsigned long long total = 0;
    for (int b = 0; b < kBands; ++b) total += pruned_cnt[b];
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        gh[r] = (r < (int64_t)total && (r - seg_start[r]) % G == 0) ? 1 : 0;
}

__global__ void __launch_bounds__(kThreads) row_off_kernel(int64_t n, const int32_t *__restrict__ gh,
                                                           const int32_t *__restrict__ gid,
                                                           int32_t *__restrict__ row_off) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        if (gh[r]) row_off[gid[r]] = (int32_t)r;
}

__global__ void sizes_kernel(int64_t n, int G, const int32_t *__restrict__ gh, const int32_t *__restrict__ gid,
                             const unsigned long long *__restrict__ pruned_cnt,
                             const unsigned long long *__restrict__ index_cnt, int32_t *__restrict__ row_off,
                             DevSizes *__restrict__ pruned, DevSizes *__restrict__ index_order) {
    unsigned long long total = 0;
    for (int b = 0; b < kBands; ++b) total += pruned_cnt[b];
    const int64_t n_groups = (int64_t)gid[n - 1] + gh[n - 1];
    row_off[n_groups] = (int32_t)total;
    pruned->first_row = 0;
    pruned->n_rows = (int64_t)total;
    pruned->n_items = n_groups;
    pruned->n_groups = n_groups;
    index_order->first_row = (int64_t)total;
    index_order->n_rows = (int64_t)*index_cnt;
    index_order->n_groups = ((int64_t)*index_cnt + G - 1) / G;
    index_order->n_items = index_order->n_groups;
}

// Index-order fallback: when the listed tiles (offsets[max_groups]) exceed kFallbackFrac x the
// tiles the pruned rows' index-order groups would stream (sum of their indices / (tile x G)),
// every row of [row_lo, row_hi) takes the index-order launch and the pruned launch is empty.
__global__ void fallback_kernel(const int32_t *__restrict__ offsets, int64_t max_groups, int G, int64_t row_lo,
                                int64_t row_hi, const unsigned long long *__restrict__ pruned_isum,
                                DevSizes *__restrict__ pruned, DevSizes *__restrict__ index_order,
                                unsigned long long *__restrict__ flag) {
    const double listed = (double)offsets[max_groups];
    const double index_tiles = (double)*pruned_isum / ((double)kTileRefs * (double)G);
    const bool back = pruned->n_groups > 0 && listed > kFallbackFrac * index_tiles;
    *flag = back ? 1ull : 0ull;
    if (!back) return;
    const int64_t nr = row_hi - row_lo;
    *pruned = DevSizes{0, 0, 0, 0};
    *index_order = DevSizes{0, nr, (nr + G - 1) / G, (nr + G - 1) / G};
}

// Under the fallback the row order becomes the searched range ascending.
__global__ void __launch_bounds__(kThreads) fallback_rows_kernel(int64_t row_lo, int64_t row_hi,
                                                                 const unsigned long long *__restrict__ flag,
                                                                 int32_t *__restrict__ rows) {
    if (*flag == 0) return;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < row_hi - row_lo;
         k += (int64_t)gridDim.x * blockDim.x)
        rows[k] = (int32_t)(row_lo + k);
}

// Box, largest seed and largest index of every pruned group; one warp per group.
__global__ void __launch_bounds__(kThreads) group_box_kernel(const float *__restrict__ xs, int d, int dp,
                                                             const int32_t *__restrict__ rows,
                                                             const int32_t *__restrict__ row_off,
                                                             const DevSizes *__restrict__ pruned,
                                                             const float *__restrict__ seeds, int all_refs,
                                                             float *__restrict__ glo, float *__restrict__ ghi,
                                                             float *__restrict__ gtau, int32_t *__restrict__ glim) {
    const int lane = threadIdx.x & 31;
    const int64_t n_groups = pruned->n_groups;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; g < n_groups; g += nw) {
        const int64_t r0 = row_off[g], r1 = row_off[g + 1];
        float tau = 0.f;
        int32_t lim = -1;
        for (int64_t r = r0 + lane; r < r1; r += 32) {
            const int32_t i = rows[r];
            tau = fmaxf(tau, seeds[i]);
            lim = max(lim, i);
        }
        lim = __reduce_max_sync(0xFFFFFFFFu, lim);
        for (int o = 16; o > 0; o >>= 1) tau = fmaxf(tau, __shfl_xor_sync(0xFFFFFFFFu, tau, o));
        if (lane == 0) {
            gtau[g] = tau;
            glim[g] = all_refs ? INT32_MAX : lim;  // refs j < lim can serve some row of the group
        }
        for (int f = 0; f < d; ++f) {
            float lo = pos_inf<float>(), hi = neg_inf<float>();
            for (int64_t r = r0 + lane; r < r1; r += 32) {
                const float v = xs[(int64_t)rows[r] * dp + f];
                lo = fminf(lo, v);
                hi = fmaxf(hi, v);
            }
            for (int o = 16; o > 0; o >>= 1) {
                lo = fminf(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
                hi = fmaxf(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
            }
            if (lane == 0) {
                glo[g * d + f] = lo;
                ghi[g * d + f] = hi;
            }
        }
    }
}

struct Boxes {
    const float *tlo, *thi, *glo, *ghi, *gtau;
    const int32_t *tmin, *glim;
    int d;
    float shrink;  // 1 - gamma, gamma = (d + 3) 2^-23 (exact in FP32)
};

// 32-bit words of one group's tile masks
__host__ __device__ __forceinline__ int64_t mask_words(int64_t n_tiles) { return (n_tiles + 31) / 32; }

// The box of group g and its bound, held in registers by every lane of the warp that tests the
// group against all tiles.
struct GroupBox {
    float lo[kMaxDim], hi[kMaxDim];
    double tau;
    int32_t lim;
};

__device__ __forceinline__ GroupBox load_group(const Boxes &b, int64_t g) {
    GroupBox q;
#pragma unroll
    for (int f = 0; f < kMaxDim; ++f) {
        q.lo[f] = f < b.d ? b.glo[g * b.d + f] : 0.f;
        q.hi[f] = f < b.d ? b.ghi[g * b.d + f] : 0.f;
    }
    q.tau = (double)b.gtau[g];
    q.lim = b.glim[g];
    return q;
}

constexpr int kBoxChunk = 128;  // tiles whose boxes a CTA stages in shared memory at a time

// May ref tile tt of the staged chunk hold a neighbour of a row of the group (need), and does
// its box meet the group's (overlap)?  slo / shi: the chunk's boxes, feature-major.
__device__ __forceinline__ void tile_test(const Boxes &b, const GroupBox &q, const float (*slo)[kBoxChunk],
                                          const float (*shi)[kBoxChunk], int32_t tmin, int tt, bool &need,
                                          bool &overlap) {
    need = false;
    overlap = false;
    if (tmin >= q.lim) return;  // every ref of the tile comes after every row
    // lb <= the exact squared box distance: every FP32 operation rounded toward -inf
    float lb = 0.f;
    bool meet = true;
#pragma unroll
    for (int f = 0; f < kMaxDim; ++f) {
        if (f < b.d) {
            const float tl = slo[f][tt], th = shi[f][tt];
            meet = meet && !(tl > q.hi[f] || q.lo[f] > th);
            const float gap = fmaxf(0.f, fmaxf(__fsub_rd(tl, q.hi[f]), __fsub_rd(q.lo[f], th)));  // NaN -> 0
            lb = __fadd_rd(lb, __fmul_rd(gap, gap));
        }
    }
    need = isinf(q.tau) || !(__fsub_rd(__fmul_rd(lb, b.shrink), 1e-37f) > (float)q.tau);
    overlap = need && meet;
}

// One warp per group, the CTA's groups tested against chunks of kBoxChunk tiles whose boxes the
// CTA stages in shared memory (each box read once per CTA instead of once per group):
// counts[g] = tiles needed (0 for the slots past the groups), and the group's masks of needed
// tiles and of needed tiles whose box meets the group's (32 tiles per word:
// masks[(g * words + w) * 2 + {0, 1}]).
__global__ void __launch_bounds__(kThreads) count_kernel(Boxes b, const DevSizes *__restrict__ pruned,
                                                         int64_t max_groups, int64_t n_tiles,
                                                         int32_t *__restrict__ counts, uint32_t *__restrict__ masks) {
    __shared__ float slo[kMaxDim][kBoxChunk], shi[kMaxDim][kBoxChunk];
    __shared__ int32_t smin[kBoxChunk];
    constexpr int kWarps = kThreads / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t n_groups = pruned->n_groups;
    const int64_t words = mask_words(n_tiles);
    // the loop bounds are the same for every warp of the CTA (it synchronises inside)
    for (int64_t gb = (int64_t)blockIdx.x * kWarps; gb < max_groups; gb += (int64_t)gridDim.x * kWarps) {
        const int64_t g = gb + warp;
        const bool act = g < n_groups;
        GroupBox q{};
        if (act) q = load_group(b, g);
        int c = 0;
        for (int64_t t0 = 0; t0 < n_tiles; t0 += kBoxChunk) {
            const int nt = (int)min((int64_t)kBoxChunk, n_tiles - t0);
            __syncthreads();
            for (int i = threadIdx.x; i < nt * b.d; i += kThreads) {
                const int tt = i / b.d, f = i - tt * b.d;
                slo[f][tt] = b.tlo[(t0 + tt) * b.d + f];
                shi[f][tt] = b.thi[(t0 + tt) * b.d + f];
            }
            for (int i = threadIdx.x; i < nt; i += kThreads) smin[i] = b.tmin[t0 + i];
            __syncthreads();
            if (act) {
                for (int base = 0; base < nt; base += 32) {
                    const int tt = base + lane;
                    bool need = false, ov = false;
                    if (tt < nt) tile_test(b, q, slo, shi, smin[tt], tt, need, ov);
                    const unsigned nm = __ballot_sync(0xFFFFFFFFu, need), om = __ballot_sync(0xFFFFFFFFu, ov);
                    if (lane == 0) {
                        const int64_t w = (t0 + base) / 32;
                        masks[(g * words + w) * 2] = nm;
                        masks[(g * words + w) * 2 + 1] = om;
                    }
                    c += __popc(nm);
                }
            }
        }
        if (lane == 0 && g < max_groups) counts[g] = c;
    }
}

// One warp per group: the needed tiles at list[offsets[g] ..), first those whose box meets the
// group's box (they hold most of the rows' nearest refs, so the rows' bounds tighten early),
// then the others, each part in ascending order (from the masks of count_kernel).
__global__ void __launch_bounds__(kThreads) fill_kernel(const DevSizes *__restrict__ pruned, int64_t n_tiles,
                                                        const int32_t *__restrict__ offsets,
                                                        const uint32_t *__restrict__ masks,
                                                        int32_t *__restrict__ list) {
    const int lane = threadIdx.x & 31;
    const int64_t n_groups = pruned->n_groups;
    const int64_t words = mask_words(n_tiles);
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; g < n_groups; g += nw) {
        int64_t o = offsets[g];
        const uint32_t *mg = masks + g * words * 2;
        for (int pass = 0; pass < 2; ++pass) {
            for (int64_t wb = 0; wb < words; wb += 32) {
                const int64_t w = wb + lane;
                uint32_t bits = 0;
                if (w < words) bits = pass == 0 ? (mg[w * 2] & mg[w * 2 + 1]) : (mg[w * 2] & ~mg[w * 2 + 1]);
                const int cnt = __popc(bits);
                int pre = cnt;  // inclusive prefix over the lanes
#pragma unroll
                for (int k = 1; k < 32; k <<= 1) {
                    const int v = __shfl_up_sync(0xFFFFFFFFu, pre, k);
                    if (lane >= k) pre += v;
                }
                int64_t at = o + pre - cnt;
                while (bits) {
                    const int bpos = __ffs(bits) - 1;
                    bits &= bits - 1;
                    list[at++] = (int32_t)(w * 32 + bpos);
                }
                o += __shfl_sync(0xFFFFFFFFu, pre, 31);
            }
        }
    }
}

// ---- work items (split long tile ranges) ----
// Tiles of every group (0 past the groups): the list length (pruned) or the tiles below the
// limit of the group's last row (index order; rows ascend, the prefix search has cut 0).
__global__ void __launch_bounds__(kThreads) group_tiles_kernel(const DevSizes *__restrict__ sz, int64_t maxg,
                                                               const int32_t *__restrict__ offsets,
                                                               const int32_t *__restrict__ rows, int G, int64_t n,
                                                               int32_t *__restrict__ cnt) {
    const int64_t ng = sz->n_groups;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g <= maxg; g += (int64_t)gridDim.x * blockDim.x) {
        int64_t c = 0;
        if (g < ng) {
            if (offsets) {
                c = offsets[g + 1] - offsets[g];
            } else {
                const int64_t last = sz->first_row + min((g + 1) * (int64_t)G, sz->n_rows) - 1;
                const int64_t lim = min((int64_t)rows[last], n);
                c = (lim + kTileRefs - 1) / kTileRefs;
            }
        }
        cnt[g] = (int32_t)c;
    }
}

// Items per group: K = ceil(tiles / C) with C = max(kChunkTiles, ceil(2 total / kMaxSlots)), so
// the split groups need at most sum over them of (tiles / C + 1) < 2 total / C <= kMaxSlots
// partial slots.  S = K for split groups (their slots), else 0.
__global__ void __launch_bounds__(kThreads) split_kernel(const DevSizes *__restrict__ sz, int64_t maxg,
                                                         const int32_t *__restrict__ cnt,
                                                         const int32_t *__restrict__ cbase, int32_t *__restrict__ K,
                                                         int32_t *__restrict__ S) {
    const int64_t ng = sz->n_groups;
    const int64_t total = cbase[maxg];
    const int64_t C = max((int64_t)kChunkTiles, (2 * total + kMaxSlots - 1) / kMaxSlots);
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g <= maxg; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = g < ng ? max((int64_t)1, (cnt[g] + C - 1) / C) : 0;
        K[g] = (int32_t)k;
        S[g] = k > 1 ? (int32_t)k : 0;
    }
}

// Item descriptors (group, tile range, slot) and their sort keys (most tiles first; the slots
// past the items last).
__global__ void __launch_bounds__(kThreads) item_fill_kernel(const DevSizes *__restrict__ sz, int64_t maxg,
                                                             int64_t max_items, const int32_t *__restrict__ cnt,
                                                             const int32_t *__restrict__ K,
                                                             const int32_t *__restrict__ kbase,
                                                             const int32_t *__restrict__ sbase,
                                                             int32_t *__restrict__ group, int32_t *__restrict__ t0,
                                                             int32_t *__restrict__ t1, int32_t *__restrict__ slot,
                                                             uint32_t *__restrict__ okey, int32_t *__restrict__ oval) {
    const int64_t ng = sz->n_groups;
    const int64_t T = kbase[maxg];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += stride) {
        const int64_t k_n = K[g], c = cnt[g];
        for (int64_t k = 0; k < k_n; ++k) {
            const int64_t d = kbase[g] + k;
            const int64_t a = c * k / k_n, b = c * (k + 1) / k_n;
            group[d] = (int32_t)g;
            t0[d] = (int32_t)a;
            t1[d] = (int32_t)b;
            slot[d] = k_n > 1 ? sbase[g] + (int32_t)k : -1;
            okey[d] = 0xFFFFFFFFu - (uint32_t)(b - a);
            oval[d] = (int32_t)d;
        }
    }
    for (int64_t d = T + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < max_items; d += stride) {
        okey[d] = 0xFFFFFFFFu;
        oval[d] = (int32_t)d;
    }
}

__global__ void items_size_kernel(DevSizes *__restrict__ sz, int64_t maxg, const int32_t *__restrict__ kbase) {
    sz->n_items = kbase[maxg];
}

// One warp per (split group, row): the top m of the group's partial lists (each ascending).
__global__ void __launch_bounds__(kThreads) merge_kernel(const DevSizes *__restrict__ sz, int64_t maxg, int G,
                                                         const int32_t *__restrict__ K,
                                                         const int32_t *__restrict__ sbase,
                                                         const int32_t *__restrict__ row_off,
                                                         const int32_t *__restrict__ rows,
                                                         const unsigned long long *__restrict__ partial, int m,
                                                         int64_t out_base, int32_t *__restrict__ out) {
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int64_t ng = sz->n_groups;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < maxg * G; w += nw) {
        const int64_t g = w / G, r = w - g * G;
        if (g >= ng || K[g] <= 1) continue;
        int64_t r0, nr;
        if (row_off) {
            r0 = row_off[g];
            nr = row_off[g + 1] - r0;
        } else {
            r0 = sz->first_row + g * G;
            nr = min((int64_t)G, sz->first_row + sz->n_rows - r0);
        }
        if (r >= nr) continue;
        const int64_t s0 = sbase[g];
        unsigned long long cur = partial[(s0 * G + r) * 32 + lane];
        for (int64_t k = 1; k < K[g]; ++k) {
            const unsigned long long nx = partial[((s0 + k) * G + r) * 32 + (31 - lane)];
            cur = nx < cur ? nx : cur;  // the 32 smallest of both lists, a bitonic sequence
#pragma unroll
            for (int j = 16; j > 0; j >>= 1) {
                const unsigned long long o = __shfl_xor_sync(FULL, cur, j);
                cur = ((lane & j) == 0) ? (o < cur ? o : cur) : (o > cur ? o : cur);
            }
        }
        if (lane < m) out[((int64_t)rows[r0 + r] - out_base) * m + lane] = (int32_t)(uint32_t)cur;
    }
}

// Groups of G consecutive rows of a search of n_rows queries (all pruned, no index order).
__global__ void uniform_groups_kernel(int64_t n_rows, int G, int64_t n_groups, int32_t *__restrict__ row_off,
                                      DevSizes *__restrict__ pruned, DevSizes *__restrict__ index_order) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g <= n_groups; g += (int64_t)gridDim.x * blockDim.x)
        row_off[g] = (int32_t)min(g * (int64_t)G, n_rows);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *pruned = DevSizes{0, n_rows, n_groups, n_groups};
        *index_order = DevSizes{n_rows, 0, 0, 0};
    }
}

struct Layout {
    int64_t n_tiles, max_groups;
    size_t tlo, thi, tmin, stats, keys_a, keys_b, vals_a, vals_b, rvals_a, rvals_b, headpos, seg_start, gh, gid, row_off, sizes, glo,
        ghi, gtau, glim, counts, offsets, masks, list, cub, cub_bytes, total;
    int64_t maxg[2], max_items[2];
    size_t cnt[2], cbase[2], K[2], kbase[2], S[2], sbase[2], igroup[2], it0[2], it1[2], islot[2], okey_a[2], okey_b[2],
        oval_a[2], oval_b[2], partial[2];
};

// Groups: segments per band <= (pruned rows of the band) / 256 or 1, groups per segment
// <= rows / G + 1, so max_groups = n / G + n / 256 + 2 kBands bounds the count.
Layout layout(int64_t n, int d, int G) {
    Layout L{};
    L.n_tiles = (n + kTileRefs - 1) / kTileRefs;
    L.max_groups = n / G + n / 256 + 2 * kBands + 1;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    L.tlo = take((size_t)L.n_tiles * d * 4);
    L.thi = take((size_t)L.n_tiles * d * 4);
    L.tmin = take((size_t)L.n_tiles * 4);
    L.stats = take(kStats * 8);
    L.keys_a = take((size_t)n * 8);
    L.keys_b = take((size_t)n * 8);
    L.vals_a = take((size_t)n * 4);
    L.vals_b = take((size_t)n * 4);
    L.rvals_a = take((size_t)n * 4);
    L.rvals_b = take((size_t)n * 4);
    L.headpos = take((size_t)n * 4);
    L.seg_start = take((size_t)n * 4);
    L.gh = take((size_t)n * 4);
    L.gid = take((size_t)n * 4);
    L.row_off = take((size_t)(L.max_groups + 1) * 4);
    L.sizes = take(2 * sizeof(DevSizes));
    L.glo = take((size_t)L.max_groups * d * 4);
    L.ghi = take((size_t)L.max_groups * d * 4);
    L.gtau = take((size_t)L.max_groups * 4);
    L.glim = take((size_t)L.max_groups * 4);
    L.counts = take((size_t)(L.max_groups + 1) * 4);
    L.offsets = take((size_t)(L.max_groups + 1) * 4);
    L.masks = take((size_t)L.max_groups * mask_words(L.n_tiles) * 2 * 4);
    L.maxg[0] = L.max_groups;
    L.maxg[1] = (n + G - 1) / G;
    for (int p = 0; p < 2; ++p) {
        const int64_t g1 = L.maxg[p] + 1;
        L.max_items[p] = L.maxg[p] + kMaxSlots;
        L.cnt[p] = take((size_t)g1 * 4);
        L.cbase[p] = take((size_t)g1 * 4);
        L.K[p] = take((size_t)g1 * 4);
        L.kbase[p] = take((size_t)g1 * 4);
        L.S[p] = take((size_t)g1 * 4);
        L.sbase[p] = take((size_t)g1 * 4);
        for (size_t *f : {&L.igroup[p], &L.it0[p], &L.it1[p], &L.islot[p], &L.okey_a[p], &L.okey_b[p], &L.oval_a[p],
                          &L.oval_b[p]})
            *f = take((size_t)L.max_items[p] * 4);
        L.partial[p] = take((size_t)kMaxSlots * G * 32 * 8);
    }
    L.list = take((size_t)L.max_groups * L.n_tiles * 4);
    L.cub_bytes = align_up((size_t)(4u << 20) + (size_t)n / 2, 256);
    L.cub = take(L.cub_bytes);
    L.total = off + 256;
    return L;
}

int grid_of(int64_t threads) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((threads + kThreads - 1) / kThreads, (int64_t)kNumSMsB200 * 8));
}

// Work items of launch pl (0 pruned, 1 index order): per-group tile counts, the split, item
// descriptors sorted by tile count (most first); fills out's item fields for pl.
nngp_status plan_items(const Layout &L, char *base, int pl, DevSizes *sz, const int32_t *offsets, const int32_t *rows,
                       int G, int64_t n, Lists *out, cudaStream_t stream) {
    auto at = [&](size_t off) { return reinterpret_cast<void *>(base + off); };
    nngp_status st = NNGP_OK;
    const int64_t maxg = L.maxg[pl], g1 = maxg + 1, mi = L.max_items[pl];
    int32_t *cnt = static_cast<int32_t *>(at(L.cnt[pl])), *cbase = static_cast<int32_t *>(at(L.cbase[pl]));
    int32_t *K = static_cast<int32_t *>(at(L.K[pl])), *kbase = static_cast<int32_t *>(at(L.kbase[pl]));
    int32_t *S = static_cast<int32_t *>(at(L.S[pl])), *sbase = static_cast<int32_t *>(at(L.sbase[pl]));
    group_tiles_kernel<<<grid_of(g1), kThreads, 0, stream>>>(sz, maxg, offsets, rows, G, n, cnt);
    NNGP_CUDA_TRY(cudaGetLastError());
    auto scan = [&](int32_t *src, int32_t *dst) -> nngp_status {
        size_t nb = 0;
        NNGP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, nb, src, dst, (int)g1, stream));
        if (nb > L.cub_bytes) return fail(NNGP_ERR_WORKSPACE, "knn pruning: scan scratch exceeds the budget");
        nb = L.cub_bytes;
        NNGP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(at(L.cub), nb, src, dst, (int)g1, stream));
        return NNGP_OK;
    };
    if ((st = scan(cnt, cbase)) != NNGP_OK) return st;
    split_kernel<<<grid_of(g1), kThreads, 0, stream>>>(sz, maxg, cnt, cbase, K, S);
    NNGP_CUDA_TRY(cudaGetLastError());
    if ((st = scan(K, kbase)) != NNGP_OK) return st;
    if ((st = scan(S, sbase)) != NNGP_OK) return st;
    int32_t *ig = static_cast<int32_t *>(at(L.igroup[pl])), *i0 = static_cast<int32_t *>(at(L.it0[pl]));
    int32_t *i1 = static_cast<int32_t *>(at(L.it1[pl])), *is = static_cast<int32_t *>(at(L.islot[pl]));
    cub::DoubleBuffer<uint32_t> okb(static_cast<uint32_t *>(at(L.okey_a[pl])), static_cast<uint32_t *>(at(L.okey_b[pl])));
    cub::DoubleBuffer<int32_t> ovb(static_cast<int32_t *>(at(L.oval_a[pl])), static_cast<int32_t *>(at(L.oval_b[pl])));
    item_fill_kernel<<<grid_of(mi), kThreads, 0, stream>>>(sz, maxg, mi, cnt, K, kbase, sbase, ig, i0, i1, is,
                                                           okb.Current(), ovb.Current());
    NNGP_CUDA_TRY(cudaGetLastError());
    items_size_kernel<<<1, 1, 0, stream>>>(sz, maxg, kbase);
    NNGP_CUDA_TRY(cudaGetLastError());
    size_t need = 0;
    NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, okb, ovb, (int)mi, 0, 32, stream));
    if (need > L.cub_bytes) return fail(NNGP_ERR_WORKSPACE, "knn pruning: sort scratch exceeds the budget");
    size_t have = L.cub_bytes;
    NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(at(L.cub), have, okb, ovb, (int)mi, 0, 32, stream));
    tc::TcItems &ti = pl == 0 ? out->pruned_items : out->index_items;
    ti.group = ig;
    ti.t0 = i0;
    ti.t1 = i1;
    ti.slot = is;
    ti.order = ovb.Current();
    ti.partial = static_cast<unsigned long long *>(at(L.partial[pl]));
    out->split_k[pl] = K;
    out->slot_base[pl] = sbase;
    out->max_groups_of[pl] = maxg;
    out->max_items[pl] = mi;
    return NNGP_OK;
}

// Layout of a query search's plan: ref tiles of n_ref refs, uniform groups of the n_query rows,
// the pruned launch's items only.
Layout layout_query(int64_t n_ref, int64_t n_query, int d, int G) {
    Layout L{};
    L.n_tiles = (n_ref + kTileRefs - 1) / kTileRefs;
    L.max_groups = (n_query + G - 1) / G;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    L.tlo = take((size_t)L.n_tiles * d * 4);
    L.thi = take((size_t)L.n_tiles * d * 4);
    L.tmin = take((size_t)L.n_tiles * 4);
    L.row_off = take((size_t)(L.max_groups + 1) * 4);
    L.sizes = take(2 * sizeof(DevSizes));
    L.glo = take((size_t)L.max_groups * d * 4);
    L.ghi = take((size_t)L.max_groups * d * 4);
    L.gtau = take((size_t)L.max_groups * 4);
    L.glim = take((size_t)L.max_groups * 4);
    L.counts = take((size_t)(L.max_groups + 1) * 4);
    L.offsets = take((size_t)(L.max_groups + 1) * 4);
    L.masks = take((size_t)L.max_groups * mask_words(L.n_tiles) * 2 * 4);
    L.maxg[0] = L.max_groups;
    L.maxg[1] = 0;
    const int64_t g1 = L.maxg[0] + 1;
    L.max_items[0] = L.maxg[0] + kMaxSlots;
    L.cnt[0] = take((size_t)g1 * 4);
    L.cbase[0] = take((size_t)g1 * 4);
    L.K[0] = take((size_t)g1 * 4);
    L.kbase[0] = take((size_t)g1 * 4);
    L.S[0] = take((size_t)g1 * 4);
    L.sbase[0] = take((size_t)g1 * 4);
    for (size_t *f : {&L.igroup[0], &L.it0[0], &L.it1[0], &L.islot[0], &L.okey_a[0], &L.okey_b[0], &L.oval_a[0],
                      &L.oval_b[0]})
        *f = take((size_t)L.max_items[0] * 4);
    L.partial[0] = take((size_t)kMaxSlots * G * 32 * 8);
    L.list = take((size_t)L.max_groups * L.n_tiles * 4);
    L.cub_bytes = align_up((size_t)(4u << 20) + (size_t)(n_query + n_ref) / 2, 256);
    L.cub = take(L.cub_bytes);
    L.total = off + 256;
    return L;
}

}  // namespace

int64_t early_rows(int64_t n) { return n >> kEarlyShift; }

bool enabled() {
    const char *env = std::getenv("NNGP_KNN_PRUNE");
    return !(env && env[0] == '0');
}

size_t workspace(int64_t n, int d, int rows_per_group) {
    if (n < kMinPoints || n > kMaxPoints || d < 1 || d > kMaxDim || rows_per_group < 1) return 0;
    return layout(n, d, rows_per_group).total;
}

nngp_status build(const float *xs, int64_t n, int64_t row_lo, int64_t row_hi, int d, int dp, int G, int bits,
                  const float *seeds, const int32_t *order0, const int32_t *pos0, const uint64_t *keys0, void *ws,
                  size_t ws_bytes, Lists *out, cudaStream_t stream) {
    if (n < kMinPoints || n > kMaxPoints || d < 1 || d > kMaxDim || G < 1 || bits < 1 || d * bits > 64 || !xs ||
        !seeds || !order0 || !pos0 || !keys0 || !out)
        return fail(NNGP_ERR_UNSUPPORTED, "knn pruning: shape outside the pruned search");
    const Layout L = layout(n, d, G);
    if (!ws || ws_bytes < L.total) return fail(NNGP_ERR_WORKSPACE, "knn pruning: workspace too small");
    char *base = reinterpret_cast<char *>(align_up(reinterpret_cast<uintptr_t>(ws), 256));
    auto at = [&](size_t off) { return reinterpret_cast<void *>(base + off); };
    float *tlo = static_cast<float *>(at(L.tlo)), *thi = static_cast<float *>(at(L.thi));
    int32_t *tmin = static_cast<int32_t *>(at(L.tmin));
    unsigned long long *sum = static_cast<unsigned long long *>(at(L.stats)), *cnt = sum + kBands,
                       *pcnt = sum + 2 * kBands, *icnt = sum + 3 * kBands, *isum = sum + 3 * kBands + 1,
                       *fallback = sum + 3 * kBands + 2;
    if (row_lo < 0 || row_hi > n || row_lo > row_hi)
        return fail(NNGP_ERR_INVALID_ARGUMENT, "knn pruning: row range outside [0, n)");
    int32_t *headpos = static_cast<int32_t *>(at(L.headpos)), *seg_start = static_cast<int32_t *>(at(L.seg_start));
    int32_t *gh = static_cast<int32_t *>(at(L.gh)), *gid = static_cast<int32_t *>(at(L.gid));
    int32_t *row_off = static_cast<int32_t *>(at(L.row_off));
    DevSizes *sizes = static_cast<DevSizes *>(at(L.sizes));
    float *glo = static_cast<float *>(at(L.glo)), *ghi = static_cast<float *>(at(L.ghi));
    float *gtau = static_cast<float *>(at(L.gtau));
    int32_t *glim = static_cast<int32_t *>(at(L.glim));
    int32_t *counts = static_cast<int32_t *>(at(L.counts)), *offsets = static_cast<int32_t *>(at(L.offsets));
    int32_t *list = static_cast<int32_t *>(at(L.list));
    const int64_t early = early_rows(n);
    auto cub_check = [&](size_t need) -> nngp_status {
        return need <= L.cub_bytes ? NNGP_OK
                                   : fail(NNGP_ERR_WORKSPACE, "knn pruning: sort / scan scratch of " +
                                                                  std::to_string(need) + " bytes exceeds the budget");
    };

    // ref order (index class, curve position) and the boxes of its tiles
    ref_keys_kernel<<<grid_of(n), kThreads, 0, stream>>>(n, pos0, static_cast<uint64_t *>(at(L.keys_a)),
                                                         static_cast<int32_t *>(at(L.rvals_a)));
    NNGP_CUDA_TRY(cudaGetLastError());
    cub::DoubleBuffer<uint64_t> rk(static_cast<uint64_t *>(at(L.keys_a)), static_cast<uint64_t *>(at(L.keys_b)));
    cub::DoubleBuffer<int32_t> rv(static_cast<int32_t *>(at(L.rvals_a)), static_cast<int32_t *>(at(L.rvals_b)));
    size_t need0 = 0;
    NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need0, rk, rv, (int)n, 0, 36, stream));
    if (need0 > L.cub_bytes) return fail(NNGP_ERR_WORKSPACE, "knn pruning: sort scratch exceeds the budget");
    size_t have0 = L.cub_bytes;
    NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(at(L.cub), have0, rk, rv, (int)n, 0, 36, stream));
    const int32_t *ref_order = rv.Current();
    tile_box_kernel<<<grid_of(L.n_tiles * 32), kThreads, 0, stream>>>(xs, n, d, dp, ref_order, L.n_tiles, tlo, thi,
                                                                       tmin);
    NNGP_CUDA_TRY(cudaGetLastError());
    NNGP_CUDA_TRY(cudaMemsetAsync(sum, 0, kStats * 8, stream));
    band_stats_kernel<<<grid_of(n - early), kThreads, 0, stream>>>(n, std::max(early, row_lo), row_hi, seeds, sum,
                                                                   cnt);
    NNGP_CUDA_TRY(cudaGetLastError());
    classify_kernel<<<grid_of(n), kThreads, 0, stream>>>(n, early, row_lo, row_hi, seeds, pos0, sum, cnt,
                                                         static_cast<uint64_t *>(at(L.keys_a)),
                                                         static_cast<int32_t *>(at(L.vals_a)), pcnt, icnt, isum);
    NNGP_CUDA_TRY(cudaGetLastError());

    // rows: pruned (band, curve position) first, then the index-order rows ascending
    cub::DoubleBuffer<uint64_t> dk(static_cast<uint64_t *>(at(L.keys_a)), static_cast<uint64_t *>(at(L.keys_b)));
    cub::DoubleBuffer<int32_t> dv(static_cast<int32_t *>(at(L.vals_a)), static_cast<int32_t *>(at(L.vals_b)));
    size_t need = 0;
    NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, dk, dv, (int)n, 0, 38, stream));
    nngp_status st = cub_check(need);
    if (st != NNGP_OK) return st;
    size_t have = L.cub_bytes;
    NNGP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(at(L.cub), have, dk, dv, (int)n, 0, 38, stream));
    int32_t *rows = dv.Current();

    // groups: segments of one band and one octree cell, cut every G rows
    segment_kernel<<<grid_of(n), kThreads, 0, stream>>>(n, dk.Current(), rows, pos0, keys0, pcnt, d, bits, headpos);
    NNGP_CUDA_TRY(cudaGetLastError());
    need = 0;
    NNGP_CUDA_TRY(cub::DeviceScan::InclusiveScan(nullptr, need, headpos, seg_start, cub::Max(), (int)n, stream));
    if ((st = cub_check(need)) != NNGP_OK) return st;
    have = L.cub_bytes;
    NNGP_CUDA_TRY(cub::DeviceScan::InclusiveScan(at(L.cub), have, headpos, seg_start, cub::Max(), (int)n, stream));
    group_head_kernel<<<grid_of(n), kThreads, 0, stream>>>(n, seg_start, pcnt, G, gh);
    NNGP_CUDA_TRY(cudaGetLastError());
    need = 0;
    NNGP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, need, gh, gid, (int)n, stream));
    if ((st = cub_check(need)) != NNGP_OK) return st;
    have = L.cub_bytes;
    NNGP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(at(L.cub), have, gh, gid, (int)n, stream));
    row_off_kernel<<<grid_of(n), kThreads, 0, stream>>>(n, gh, gid, row_off);
    NNGP_CUDA_TRY(cudaGetLastError());
    sizes_kernel<<<1, 1, 0, stream>>>(n, G, gh, gid, pcnt, icnt, row_off, sizes, sizes + 1);
    NNGP_CUDA_TRY(cudaGetLastError());

    // tile lists, then the work order (longest list first)
    group_box_kernel<<<grid_of(L.max_groups * 32), kThreads, 0, stream>>>(xs, d, dp, rows, row_off, sizes, seeds, 0,
                                                                          glo, ghi, gtau, glim);
    NNGP_CUDA_TRY(cudaGetLastError());
    Boxes b{tlo, thi, glo, ghi, gtau, tmin, glim, d, 1.0f - (float)(d + 3) * 1.1920928955078125e-07f};
    NNGP_CUDA_TRY(cudaMemsetAsync(counts + L.max_groups, 0, sizeof(int32_t), stream));
    uint32_t *masks = static_cast<uint32_t *>(at(L.masks));
    count_kernel<<<grid_of(L.max_groups * 32), kThreads, 0, stream>>>(b, sizes, L.max_groups, L.n_tiles, counts,
                                                                       masks);
    NNGP_CUDA_TRY(cudaGetLastError());
    need = 0;
    NNGP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, need, counts, offsets, (int)(L.max_groups + 1), stream));
    if ((st = cub_check(need)) != NNGP_OK) return st;
    have = L.cub_bytes;
    NNGP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(at(L.cub), have, counts, offsets, (int)(L.max_groups + 1), stream));
    fallback_kernel<<<1, 1, 0, stream>>>(offsets, L.max_groups, G, row_lo, row_hi, isum, sizes, sizes + 1, fallback);
    NNGP_CUDA_TRY(cudaGetLastError());
    fallback_rows_kernel<<<grid_of(row_hi - row_lo), kThreads, 0, stream>>>(row_lo, row_hi, fallback, rows);
    NNGP_CUDA_TRY(cudaGetLastError());
    fill_kernel<<<grid_of(L.max_groups * 32), kThreads, 0, stream>>>(sizes, L.n_tiles, offsets, masks, list);
    NNGP_CUDA_TRY(cudaGetLastError());

    // work items of both launches: long tile ranges split, most tiles first
    for (int pl = 0; pl < 2; ++pl)
        if ((st = plan_items(L, base, pl, sizes + pl, pl == 0 ? offsets : nullptr, rows, G, n, out, stream)) != NNGP_OK)
            return st;

    out->rows = rows;
    out->ref_order = ref_order;
    out->pruned = sizes;
    out->index_order = sizes + 1;
    out->row_off = row_off;
    out->offsets = offsets;
    out->tiles = list;
    out->max_groups = L.max_groups;
    return NNGP_OK;
}

size_t workspace_query(int64_t n_ref, int64_t n_query, int d, int rows_per_group) {
    if (n_ref < kMinPoints || n_ref > kMaxPoints || n_query < 1 || d < 1 || d > kMaxDim || rows_per_group < 1) return 0;
    return layout_query(n_ref, n_query, d, rows_per_group).total;
}

nngp_status build_query(const float *xs_ref, int64_t n_ref, const float *xq, int64_t n_query, int d, int dp, int G,
                        const float *seeds, const int32_t *order0, const int32_t *qorder, void *ws, size_t ws_bytes,
                        Lists *out, cudaStream_t stream) {
    if (workspace_query(n_ref, n_query, d, G) == 0 || !xs_ref || !xq || !seeds || !order0 || !qorder || !out)
        return fail(NNGP_ERR_UNSUPPORTED, "knn pruning: shape outside the pruned query search");
    const Layout L = layout_query(n_ref, n_query, d, G);
    if (!ws || ws_bytes < L.total) return fail(NNGP_ERR_WORKSPACE, "knn pruning: workspace too small");
    char *base = reinterpret_cast<char *>(align_up(reinterpret_cast<uintptr_t>(ws), 256));
    auto at = [&](size_t off) { return reinterpret_cast<void *>(base + off); };
    float *tlo = static_cast<float *>(at(L.tlo)), *thi = static_cast<float *>(at(L.thi));
    int32_t *tmin = static_cast<int32_t *>(at(L.tmin));
    int32_t *row_off = static_cast<int32_t *>(at(L.row_off));
    DevSizes *sizes = static_cast<DevSizes *>(at(L.sizes));
    float *glo = static_cast<float *>(at(L.glo)), *ghi = static_cast<float *>(at(L.ghi));
    float *gtau = static_cast<float *>(at(L.gtau));
    int32_t *glim = static_cast<int32_t *>(at(L.glim));
    int32_t *counts = static_cast<int32_t *>(at(L.counts)), *offsets = static_cast<int32_t *>(at(L.offsets));
    int32_t *list = static_cast<int32_t *>(at(L.list));
    nngp_status st = NNGP_OK;

    tile_box_kernel<<<grid_of(L.n_tiles * 32), kThreads, 0, stream>>>(xs_ref, n_ref, d, dp, order0, L.n_tiles, tlo, thi,
                                                                       tmin);
    NNGP_CUDA_TRY(cudaGetLastError());
    uniform_groups_kernel<<<grid_of(L.max_groups + 1), kThreads, 0, stream>>>(n_query, G, L.max_groups, row_off, sizes,
                                                                              sizes + 1);
    NNGP_CUDA_TRY(cudaGetLastError());
    group_box_kernel<<<grid_of(L.max_groups * 32), kThreads, 0, stream>>>(xq, d, dp, qorder, row_off, sizes, seeds, 1,
                                                                          glo, ghi, gtau, glim);
    NNGP_CUDA_TRY(cudaGetLastError());
    Boxes b{tlo, thi, glo, ghi, gtau, tmin, glim, d, 1.0f - (float)(d + 3) * 1.1920928955078125e-07f};
    NNGP_CUDA_TRY(cudaMemsetAsync(counts + L.max_groups, 0, sizeof(int32_t), stream));
    uint32_t *masks = static_cast<uint32_t *>(at(L.masks));
    count_kernel<<<grid_of(L.max_groups * 32), kThreads, 0, stream>>>(b, sizes, L.max_groups, L.n_tiles, counts,
                                                                       masks);
    NNGP_CUDA_TRY(cudaGetLastError());
    size_t need = 0;
    NNGP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, need, counts, offsets, (int)(L.max_groups + 1), stream));
    if (need > L.cub_bytes) return fail(NNGP_ERR_WORKSPACE, "knn pruning: scan scratch exceeds the budget");
    size_t have = L.cub_bytes;
    NNGP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(at(L.cub), have, counts, offsets, (int)(L.max_groups + 1), stream));
    fill_kernel<<<grid_of(L.max_groups * 32), kThreads, 0, stream>>>(sizes, L.n_tiles, offsets, masks, list);
    NNGP_CUDA_TRY(cudaGetLastError());
    if ((st = plan_items(L, base, 0, sizes, offsets, qorder, G, n_ref, out, stream)) != NNGP_OK) return st;
    out->rows = qorder;
    out->ref_order = order0;
    out->pruned = sizes;
    out->index_order = sizes + 1;
    out->row_off = row_off;
    out->offsets = offsets;
    out->tiles = list;
    out->max_groups = L.max_groups;
    out->index_items = tc::TcItems{};
    out->split_k[1] = nullptr;
    out->max_items[1] = 0;
    return NNGP_OK;
}

nngp_status merge(const Lists &lists, int which, int G, int m, int64_t out_base, int32_t *out, cudaStream_t stream) {
    if (which < 0 || which > 1 || !lists.split_k[which]) return fail(NNGP_ERR_INVALID_ARGUMENT, "knn merge: no plan");
    const DevSizes *sz = which == 0 ? lists.pruned : lists.index_order;
    const tc::TcItems &ti = which == 0 ? lists.pruned_items : lists.index_items;
    const int64_t maxg = lists.max_groups_of[which];
    merge_kernel<<<grid_of(maxg * G * 32), kThreads, 0, stream>>>(sz, maxg, G, lists.split_k[which],
                                                                  lists.slot_base[which],
                                                                  which == 0 ? lists.row_off : nullptr, lists.rows,
                                                                  ti.partial, m, out_base, out);
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

}  // namespace prune
}  // namespace nngp
