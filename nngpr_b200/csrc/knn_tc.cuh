// Host-side handle of the tensor-core search kernels (knn_tc.cu), used by the dispatcher in knn.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nngp {
namespace tc {

constexpr int kTcRefTile = 128;    // refs per tile (UMMA N)
constexpr int kTcQueryTile = 128;  // queries per tile (UMMA M)

// Work items of one launch of the search.  All null: item k is group k (or, for the prefix
// search, heaviest first), over the group's whole tile range.  Otherwise item k is descriptor
// order[k]: group group[d], tiles [t0[d], t1[d]) of the group's range, and its rows' lists go to
// out (slot[d] < 0) or, sorted, as 32 keys (distance bits << 32 | index, ~0 when empty) per row to
// partial[(slot[d] * rows_per_item + row) * 32 ..] for a merge.
struct TcItems {
    const int32_t *group = nullptr, *t0 = nullptr, *t1 = nullptr, *slot = nullptr, *order = nullptr;
    unsigned long long *partial = nullptr;
};

using TcFn = void (*)(const unsigned char *, const float *, const double *, const unsigned int *, const float *,
                      const int32_t *, const int32_t *, const int64_t *, TcItems, const int32_t *, const int32_t *,
                      const int32_t *, int *, int64_t, int64_t, int, int64_t, int, int64_t, int32_t *, int32_t *, uint64_t);
// build(xs, n, n_pad, acc, perm, tiles, r2max): tile position i holds point perm[i] (i when perm is null)
using TcBuildFn = void (*)(const float *, int64_t, int64_t, const double *, const int32_t *, unsigned char *,
                           unsigned int *);

struct TcVariant {
    TcFn fn = nullptr;
    TcBuildFn build = nullptr;
    int smem = 0, stage_bytes = 0, dp = 0;
    int ctas_per_sm = 1;     // CTAs the shared memory of one SM holds (the kernel's launch bounds)
    int threads = 160;       // epilogue warps (4 per query tile) + the producer/MMA warp
    int rows_per_item = 128;  // queries per work item (128 per query tile)
};

}  // namespace tc

// Kernels for dimension D (exact for d <= 8, else round_up(d, 4): 12, 16, 20, 24); num_nn <= 32;
// fn == nullptr when the shape has no tensor-core variant.
tc::TcVariant tc_variant(int D, int M);

}  // namespace nngp
