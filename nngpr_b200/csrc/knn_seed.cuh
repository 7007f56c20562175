// Seed thresholds for the prefix neighbour search (knn_seed.cu), used by the dispatcher in knn.cu.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "nngp_b200.h"

namespace nngp {
namespace seed {

constexpr int64_t kMinPoints = 8192;  // below this the search is short and seeding does not pay

// Workspace bytes of prefix_seeds for n points (0 when n < kMinPoints).
size_t workspace(int64_t n);

// Window half-width in curve positions: NNGP_KNN_SEED_W = 128 or 256 (default 256); 0 turns
// seeding off.
int window();

// seeds[i] >= the m-th smallest squared distance from point i to the points j < i, in the
// search's FP32 arithmetic (the squared distance of the scaled coordinates, ((t0^2 + t1^2) + ...),
// every step rounded), or +inf.  xs: n scaled points, row stride dp (zero padded), D the padded
// dimension the search kernel loops over.  Runs on `stream`; ws of workspace(n) bytes.
nngp_status prefix_seeds(const float *xs, int64_t n, int d, int D, int dp, int m, void *ws, size_t ws_bytes,
                         float *seeds, cudaStream_t stream);

}  // namespace seed
}  // namespace nngp
