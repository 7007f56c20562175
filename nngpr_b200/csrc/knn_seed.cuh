// Seed thresholds for the prefix neighbour search (knn_seed.cu), used by the dispatcher in knn.cu.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "nngp_b200.h"

namespace nngp {
namespace seed {

constexpr int64_t kMinPoints = 8192;  // below this the search is short and seeding does not pay

// Workspace bytes of prefix_seeds for n points of row stride dp (0 when n < kMinPoints).
size_t workspace(int64_t n, int dp);

// Window half-width in curve positions: NNGP_KNN_SEED_W = 128 or 256 (default 128: the faster
// fit step at d = 3, 8 and 16); 0 turns seeding off.
int window();

// seeds[i] >= the m-th smallest squared distance from point i to the points j < i, in the
// search's FP32 arithmetic (the squared distance of the scaled coordinates, ((t0^2 + t1^2) + ...),
// every step rounded), or +inf.  xs: n scaled points, row stride dp (zero padded), D the padded
// dimension the search kernel loops over.  Runs on `stream`; ws of workspace(n) bytes.
// order0 / pos0 / keys0 (optional): the curve-0 order of the points (a permutation of 0..n-1),
// its inverse and the curve-0 Morton keys in that order (key of point i = keys0[pos0[i]];
// bits() bits per dimension, interleaved), left in ws for the caller.
// row_lo / row_hi: only the rows [row_lo, row_hi) get seeds (a row shard; -1: up to n).
nngp_status prefix_seeds(const float *xs, int64_t n, int d, int D, int dp, int m, void *ws, size_t ws_bytes,
                         float *seeds, cudaStream_t stream, const int32_t **order0 = nullptr,
                         const int32_t **pos0 = nullptr, const uint64_t **keys0 = nullptr, int64_t row_lo = 0,
                         int64_t row_hi = -1);

// Seeds of a search of n_query queries against n_ref refs (no prefix rule): seeds[q] >= the m-th
// smallest squared distance from query q to the refs, in the search's FP32 arithmetic, from the
// refs' curve windows around the query's place in each curve.  xs_ref / xq: scaled points, row
// stride dp.  order0: the refs' curve-0 order (ref tiles of a pruned search use it); qorder: the
// queries in curve-0 order.  Runs on `stream`.
size_t workspace_query(int64_t n_ref, int64_t n_query, int dp);
// The query-search seeds are used (and budgeted) from this many queries on: below it the refs'
// sorts cost more than the seeds save.
constexpr int64_t kMinQueries = 16384;
inline size_t query_workspace_if(int64_t n_ref, int64_t n_query, int dp) {
    return n_query >= kMinQueries ? workspace_query(n_ref, n_query, dp) : 0;
}
nngp_status query_seeds(const float *xs_ref, int64_t n_ref, const float *xq, int64_t n_query, int d, int D, int dp,
                        int m, void *ws, size_t ws_bytes, float *seeds, cudaStream_t stream, const int32_t **order0,
                        const int32_t **qorder);

// Bits per dimension of the Morton keys for d features.
inline int bits(int d) { return d < 7 ? 10 : 64 / d; }

}  // namespace seed
}  // namespace nngp
