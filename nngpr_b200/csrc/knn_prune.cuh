// Row groups and ref-tile lists of the pruned prefix search (knn_prune.cu), used by the
// dispatcher in knn.cu.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "knn_tc.cuh"
#include "nngp_b200.h"

namespace nngp {
namespace prune {

constexpr int64_t kMinPoints = 65536;  // below this the index-order search is short enough
constexpr int64_t kMaxPoints = 2000000;  // the tile lists' worst-case bound (groups x tiles) grows as n^2
constexpr int kMaxDim = 24;            // every shape of the tensor-core search (d <= 24)
constexpr int kTileRefs = 128;         // refs per tile (the tensor-core search's ref tile)

// Rows [0, early_rows(n)) = [0, n / 8) always take the index-order search: their prefixes are
// short, and the boxes of the sparse index classes they may use are large.
int64_t early_rows(int64_t n);

// NNGP_KNN_PRUNE=0 turns pruning off (seeded index-order search only).
bool enabled();

// Device-side sizes of one launch of the search (written by build, read by the kernel).
struct DevSizes {
    int64_t first_row;  // position of the launch's first row in Lists::rows
    int64_t n_rows;
    int64_t n_items;    // work items (a group's whole tile range or a chunk of it)
    int64_t n_groups;   // groups of rows
};

// A group whose tile range exceeds C = max(kChunkTiles, 2 x total tiles / kMaxSlots) tiles is
// split into items of about equal ranges, so that a launch with few groups still spreads over
// every SM; each item writes its rows' partial lists and merge() combines them (any global top-m
// ref is in the top-m of its item's range, so the merged lists are exact).
constexpr int kChunkTiles = 16;
constexpr int kMaxSlots = 1024;

struct Lists {
    const int32_t *rows = nullptr;        // n point indices: the pruned rows group after group, then
                                          // the index-order rows, ascending
    const int32_t *ref_order = nullptr;   // n point indices: tile position k holds point ref_order[k]
    const DevSizes *pruned = nullptr;     // the pruned launch
    const DevSizes *index_order = nullptr;  // the index-order launch (rows_per_group rows per item)
    const int32_t *row_off = nullptr;     // pruned group g: rows[row_off[g] .. row_off[g + 1])
    tc::TcItems pruned_items, index_items;  // work items of the two launches (most tiles first)
    const int32_t *split_k[2] = {nullptr, nullptr};     // items per group (pruned, index order)
    const int32_t *slot_base[2] = {nullptr, nullptr};   // first partial slot per split group
    int64_t max_groups_of[2] = {0, 0};
    const int32_t *offsets = nullptr;     // group g's tiles: tiles[offsets[g] .. offsets[g + 1])
    const int32_t *tiles = nullptr;       // ref tile ids (ref_order positions / 128)
    int64_t max_groups = 0;               // host-side bound of pruned->n_groups
    int64_t max_items[2] = {0, 0};        // host-side bounds of the launches' n_items
};

size_t workspace(int64_t n, int d, int rows_per_group);

// Plans the prefix search of n scaled points xs (row stride dp, d <= kMaxDim features) over
// itself, from the seeds and the curve order of knn_seed.cu (order0, pos0, keys0 with
// bits_per_dim bits per dimension).  Rows below early_rows(n) and rows whose seed is more than
// 16 times the geometric mean of their band's seeds go to the index-order launch; the others
// are sorted by (band = floor(log2(n / i)), curve position) and cut into groups of at most
// rows_per_group rows that never straddle a band or an octree cell of the curve (a cell level
// per band chosen so that cells hold about 256 of its rows).  Refs are ordered by (index class
// = 3 - band, curve position) and cut into tiles of 128 (ref_order; the caller builds the
// search's tiles in that order).  A ref tile is listed for a group unless (a) every point in it
// has an index >= every row of the group, or (b) the distance between the two bounding boxes,
// shrunk by the FP32 rounding bound, exceeds the largest seed of the group; tiles whose box meets
// the group's come first.  Neither rule excludes a neighbour of any row, so the search returns
// the same lists.  No host synchronisation: sizes stay on the device.
// Only the rows [row_lo, row_hi) are planned (a row shard of the multi-GPU fit step; [0, n) for
// the whole search); the refs are all n points.
nngp_status build(const float *xs, int64_t n, int64_t row_lo, int64_t row_hi, int d, int dp, int rows_per_group,
                  int bits_per_dim, const float *seeds, const int32_t *order0, const int32_t *pos0,
                  const uint64_t *keys0, void *ws, size_t ws_bytes, Lists *out, cudaStream_t stream);

// The same for a search of n_query queries against n_ref refs without a prefix rule (predict):
// the queries in curve-0 order (qorder, from knn_seed's query_seeds) cut into groups of
// rows_per_group, every ref tile (refs in their curve-0 order, order0) listed unless the box
// distance rule excludes it.  All rows take the pruned launch (index_order is empty).
size_t workspace_query(int64_t n_ref, int64_t n_query, int d, int rows_per_group);
nngp_status build_query(const float *xs_ref, int64_t n_ref, const float *xq, int64_t n_query, int d, int dp,
                        int rows_per_group, const float *seeds, const int32_t *order0, const int32_t *qorder, void *ws,
                        size_t ws_bytes, Lists *out, cudaStream_t stream);

// Combines the partial lists of the split groups of launch `which` (0 pruned, 1 index order)
// into out (num_nn m; row of point i at out[(i - out_base) * m]).  Runs after that launch on the
// same stream.
nngp_status merge(const Lists &lists, int which, int rows_per_group, int m, int64_t out_base, int32_t *out,
                  cudaStream_t stream);

}  // namespace prune
}  // namespace nngp
