// nrc_cache.h -- owner of one neural radiance cache's device state: f32 master
// weights and hash table, Adam moments, gradients, fp16 copies the kernels
// read, and the step counter for the bias corrections.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "nrc.h"
#include "vt_common.h"

namespace vt {
namespace nrc {

class Cache {
 public:
  Cache(const Config& c, uint32_t seed);

  View view() const;
  size_t table_pairs() const { return (size_t)cfg_.levels << cfg_.log2_table; }

  // rgb[i] = network(records[i]) (stride in float4); or, with `radiance`,
  // radiance[path] += T * max(prediction, 0) for records carrying (path, T).
  void query(const float4* records, uint32_t stride, const uint32_t* n_dev, uint32_t n, float* rgb,
             float4* radiance, cudaStream_t s) const;
  // Gradients of the mean loss into the gradient buffers (cleared first).
  void gradients(const float4* samples, uint32_t n, cudaStream_t s);
  // gradients + Adam (clears the gradients).
  void train_step(const float4* samples, uint32_t n, cudaStream_t s);

  void get_params(float* weights, float* table) const;  // host arrays
  void set_params(const float* weights, const float* table);
  void set_aabb(const float* mn, const float* mx);
  // Screen-tile error statistics gathered by later training steps (nullptr: none).
  void set_error_tiles(float* stats, uint32_t width, uint32_t tile, uint32_t tiles_x) {
    tile_stats_ = stats;
    tile_width_ = width;
    tile_size_ = tile;
    tiles_x_ = tiles_x;
  }
  void clear_gradients(cudaStream_t s);
  // Query tiles in flight per inference CTA (1..4).
  void set_infer_tiles(int t) { cfg_.infer_tiles = t < 1 ? 1 : (t > 4 ? 4 : t); }
  // Clocks the kernels wait for their MMAs before giving up (0: kDefaultWaitCycles).
  void set_wait_cycles(long long c) { wait_cycles_ = c > 0 ? c : kDefaultWaitCycles; }

  const Config& config() const { return cfg_; }
  uint64_t steps() const { return step_; }
  float* d_loss() const { return loss_.ptr; }
  int* d_diag() const { return diag_.ptr; }
  const float* d_grad_w() const { return grad_w_.ptr; }
  const float2* d_grad_table() const { return grad_t_.ptr; }

 private:
  void adam(cudaStream_t s);
  Config cfg_;
  long long wait_cycles_ = kDefaultWaitCycles;
  float res_[kMaxLevels] = {};
  uint64_t step_ = 0;
  DeviceBuffer<float> w_, w_m_, w_v_, grad_w_;
  DeviceBuffer<__half> w16_;
  DeviceBuffer<float> t_, t_m_, t_v_;
  DeviceBuffer<float2> grad_t_;
  DeviceBuffer<__half2> t16_;
  DeviceBuffer<int> diag_;    // [0] wait expired, [1] non-finite optimiser events
  DeviceBuffer<float> loss_;
  float* tile_stats_ = nullptr;
  uint32_t tile_width_ = 0, tile_size_ = 16, tiles_x_ = 0;
};

}  // namespace nrc
}  // namespace vt
