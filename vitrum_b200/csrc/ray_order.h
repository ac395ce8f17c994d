// ray_order.h -- spatial trace order for incoherent ray batches.
//
// A counting sort of a ray batch by (Morton code of the point where the ray
// enters the scene box, direction octant): rays that enter the same small
// cell heading into the same octant land next to each other, so the 32 lanes
// of a traversal warp walk mostly the same nodes (fewer divergent node and
// triangle phases, more L1 hits).  The sort produces a permutation only; the
// traversal reads ray order[i] in slot i and writes each result at its own
// ray, so the results are those of the unsorted batch.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace vt {

struct RayOrderArgs {
  const float4* rays = nullptr;     // 2 float4 per ray (origin, tmin | direction, tmax)
  size_t n = 0;                     // ray count (capacity when n_dev is set)
  const uint32_t* n_dev = nullptr;  // when set, the ray count is read from this device word
  float lo[3] = {0, 0, 0};          // quantisation box (the scene's bounds)
  float hi[3] = {1, 1, 1};
  int cell_bits = 5;                // Morton bits per axis, 1..6: 2^(3*cell_bits + 3) buckets
  uint32_t* keys = nullptr;         // n words: each ray's bucket
  uint32_t* counts = nullptr;       // ray_order_count_words(cell_bits) words
  uint32_t* order = nullptr;        // n words: slot -> ray
};

constexpr int kRayOrderMaxCellBits = 6;
// Device words `counts` needs: one per bucket plus the scan's block sums.
size_t ray_order_count_words(int cell_bits);
// Enqueues the sort on `s` (memset of the buckets, key, scan, scatter: four launches).
void launch_ray_order(const RayOrderArgs& a, cudaStream_t s);

}  // namespace vt
