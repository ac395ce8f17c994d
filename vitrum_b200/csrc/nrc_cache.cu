// nrc_cache.cu -- device state of a neural radiance cache and its C ABI
// (vt_nrc_*): construction, query, training step, gradients, snapshots.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/vitrum_pt.h"
#include "nrc_cache.h"

namespace vt {
namespace nrc {

namespace {

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uni(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

void validate(const Config& c) {
  if (c.levels < 1 || c.levels > kMaxLevels) fail(VT_ERR_INVALID_ARGUMENT, "levels must be in 1..16");
  if (c.log2_table < 4 || c.log2_table > 24) fail(VT_ERR_INVALID_ARGUMENT, "log2_table_size must be in 4..24");
  if (!(c.base_resolution >= 1.0f) || !std::isfinite(c.base_resolution))
    fail(VT_ERR_INVALID_ARGUMENT, "base_resolution must be finite and >= 1");
  if (!(c.growth >= 1.0f) || !std::isfinite(c.growth)) fail(VT_ERR_INVALID_ARGUMENT, "growth must be finite and >= 1");
  if (!(c.lr > 0.0f) || !(c.table_lr > 0.0f) || !std::isfinite(c.lr) || !std::isfinite(c.table_lr))
    fail(VT_ERR_INVALID_ARGUMENT, "learning rates must be finite and positive");
  const double top = std::floor((double)c.base_resolution * std::pow((double)c.growth, c.levels - 1));
  if (!(top < 1048576.0)) fail(VT_ERR_INVALID_ARGUMENT, "finest level resolution must stay below 2^20");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(c.aabb_min[k]) || !std::isfinite(c.aabb_max[k]) || !(c.aabb_max[k] >= c.aabb_min[k]))
      fail(VT_ERR_INVALID_ARGUMENT, "aabb must be finite with max >= min");
  if (c.infer_tiles < 1 || c.infer_tiles > 4) fail(VT_ERR_RANGE, "infer_tiles must be 0 or in 1..4");
}

}  // namespace

Cache::Cache(const Config& c, uint32_t seed) : cfg_(c) {
  validate(c);
  level_resolutions(cfg_, res_);
  // He-uniform hidden weights (variance 2 / fan_in), output rows 0..2 with
  // variance 1 / fan_in, rows 3..63 of the output layer zero; table U(-1e-4, 1e-4).
  std::vector<float> w(kWeights, 0.0f);
  uint64_t s = 0x5EEDull ^ ((uint64_t)seed << 17);
  for (int l = 0; l < kLayers; ++l) {
    const int rows = l + 1 < kLayers ? kWidth : kOut;
    const double a = l + 1 < kLayers ? std::sqrt(6.0 / kWidth) : std::sqrt(3.0 / kWidth);
    for (int r = 0; r < rows; ++r)
      for (int k = 0; k < kWidth; ++k) w[(size_t)l * kWidth * kWidth + r * kWidth + k] = (float)((2 * uni(s) - 1) * a);
  }
  std::vector<float> t(2 * table_pairs());
  for (auto& x : t) x = (float)((2 * uni(s) - 1) * 1e-4);
  w_.resize(kWeights);
  w_m_.resize(kWeights);
  w_v_.resize(kWeights);
  grad_w_.resize(kWeights);
  w16_.resize(kWeights);
  t_.resize(2 * table_pairs());
  t_m_.resize(2 * table_pairs());
  t_v_.resize(2 * table_pairs());
  grad_t_.resize(table_pairs());
  t16_.resize(table_pairs());
  diag_.resize(2);
  loss_.resize(1);
  VT_CUDA(cudaMemset(diag_.ptr, 0, diag_.bytes()));
  VT_CUDA(cudaMemset(loss_.ptr, 0, loss_.bytes()));
  set_params(w.data(), t.data());
}

View Cache::view() const {
  View v;
  v.w16 = w16_.ptr;
  v.table16 = t16_.ptr;
  v.grad_w = grad_w_.ptr;
  v.grad_table = grad_t_.ptr;
  v.levels = cfg_.levels;
  v.table_mask = (uint32_t)((1u << cfg_.log2_table) - 1u);
  for (int l = 0; l < kMaxLevels; ++l) v.res[l] = res_[l];
  for (int k = 0; k < 3; ++k) {
    const float ext = cfg_.aabb_max[k] - cfg_.aabb_min[k];
    v.aabb_min[k] = cfg_.aabb_min[k];
    v.aabb_inv[k] = ext > 1e-20f ? 1.0f / ext : 0.0f;
  }
  v.error = diag_.ptr;
  v.wait_cycles = wait_cycles_;
  v.loss = loss_.ptr;
  v.tile_stats = tile_stats_;
  v.tile_width = tile_width_;
  v.tile_size = tile_size_;
  v.tiles_x = tiles_x_;
  return v;
}

void Cache::set_aabb(const float* mn, const float* mx) {
  for (int k = 0; k < 3; ++k) {
    cfg_.aabb_min[k] = mn[k];
    cfg_.aabb_max[k] = mx[k];
  }
}

void Cache::query(const float4* records, uint32_t stride, const uint32_t* n_dev, uint32_t n, float* rgb,
                  float4* radiance, cudaStream_t s) const {
  launch_infer(view(), records, stride, n_dev, n, rgb, radiance, cfg_.infer_tiles, s);
}

void Cache::clear_gradients(cudaStream_t s) {
  VT_CUDA(cudaMemsetAsync(grad_w_.ptr, 0, grad_w_.bytes(), s));
  VT_CUDA(cudaMemsetAsync(grad_t_.ptr, 0, grad_t_.bytes(), s));
}

void Cache::gradients(const float4* samples, uint32_t n, cudaStream_t s) {
  clear_gradients(s);
  VT_CUDA(cudaMemsetAsync(loss_.ptr, 0, sizeof(float), s));
  launch_train(view(), samples, n, s);
}

void Cache::adam(cudaStream_t s) {
  ++step_;
  const float bc1 = (float)(1.0 - std::pow((double)cfg_.beta1, (double)step_));
  const float bc2 = (float)(1.0 - std::pow((double)cfg_.beta2, (double)step_));
  launch_adam(w_.ptr, w_m_.ptr, w_v_.ptr, grad_w_.ptr, w16_.ptr, kWeights, cfg_.lr, cfg_.beta1, cfg_.beta2,
              cfg_.eps, bc1, bc2, diag_.ptr + 1, s);
  launch_adam_table(t_.ptr, t_m_.ptr, t_v_.ptr, grad_t_.ptr, t16_.ptr, table_pairs(), cfg_.table_lr, cfg_.beta1,
                    cfg_.beta2, cfg_.eps, bc1, bc2, diag_.ptr + 1, s);
}

void Cache::train_step(const float4* samples, uint32_t n, cudaStream_t s) {
  VT_CUDA(cudaMemsetAsync(loss_.ptr, 0, sizeof(float), s));
  launch_train(view(), samples, n, s);  // gradients are zero here: Adam clears them
  adam(s);
}

void Cache::get_params(float* weights, float* table) const {
  if (weights) VT_CUDA(cudaMemcpy(weights, w_.ptr, w_.bytes(), cudaMemcpyDeviceToHost));
  if (table) VT_CUDA(cudaMemcpy(table, t_.ptr, t_.bytes(), cudaMemcpyDeviceToHost));
}

void Cache::set_params(const float* weights, const float* table) {
  if (weights) {
    std::vector<float> w(weights, weights + kWeights);
    for (int r = kOut; r < kWidth; ++r)
      for (int k = 0; k < kWidth; ++k) w[(size_t)(kLayers - 1) * kWidth * kWidth + r * kWidth + k] = 0.0f;
    std::vector<__half> h(kWeights);
    for (int i = 0; i < kWeights; ++i) {
      if (!std::isfinite(w[i]) || std::fabs(w[i]) > 65504.0f) fail(VT_ERR_RANGE, "weights must be finite fp16 values");
      h[i] = __float2half_rn(w[i]);
    }
    VT_CUDA(cudaMemcpy(w_.ptr, w.data(), w_.bytes(), cudaMemcpyHostToDevice));
    VT_CUDA(cudaMemcpy(w16_.ptr, h.data(), w16_.bytes(), cudaMemcpyHostToDevice));
    VT_CUDA(cudaMemset(w_m_.ptr, 0, w_m_.bytes()));
    VT_CUDA(cudaMemset(w_v_.ptr, 0, w_v_.bytes()));
    VT_CUDA(cudaMemset(grad_w_.ptr, 0, grad_w_.bytes()));
  }
  if (table) {
    const size_t n = 2 * table_pairs();
    std::vector<__half> h(n);
    for (size_t i = 0; i < n; ++i) {
      if (!std::isfinite(table[i]) || std::fabs(table[i]) > 65504.0f) fail(VT_ERR_RANGE, "table must be finite fp16 values");
      h[i] = __float2half_rn(table[i]);
    }
    VT_CUDA(cudaMemcpy(t_.ptr, table, t_.bytes(), cudaMemcpyHostToDevice));
    VT_CUDA(cudaMemcpy(t16_.ptr, h.data(), t16_.bytes(), cudaMemcpyHostToDevice));
    VT_CUDA(cudaMemset(t_m_.ptr, 0, t_m_.bytes()));
    VT_CUDA(cudaMemset(t_v_.ptr, 0, t_v_.bytes()));
    VT_CUDA(cudaMemset(grad_t_.ptr, 0, grad_t_.bytes()));
  }
  step_ = 0;
}

}  // namespace nrc
}  // namespace vt

// ---------------------------------------------------------------- C ABI
struct vt_nrc {
  int device = 0;
  cudaStream_t stream = nullptr;
  vt::nrc::Cache* cache = nullptr;
  vt::DeviceBuffer<float4> io;
  vt::DeviceBuffer<float> rgb;
};

namespace {

vt::nrc::Config to_config(const vt_nrc_config* c) {
  vt::nrc::Config k;
  k.levels = c->levels;
  k.log2_table = c->log2_table_size;
  k.base_resolution = c->base_resolution;
  k.growth = c->growth;
  k.lr = c->learning_rate;
  k.table_lr = c->table_learning_rate;
  for (int i = 0; i < 3; ++i) {
    k.aabb_min[i] = c->aabb_min[i];
    k.aabb_max[i] = c->aabb_max[i];
  }
  k.infer_tiles = c->infer_tiles > 0 ? c->infer_tiles : vt::nrc::kDefaultInferTiles;
  return k;
}

void check_diag(vt_nrc* h) {
  int d[2] = {0, 0};
  VT_CUDA(cudaMemcpy(d, h->cache->d_diag(), sizeof d, cudaMemcpyDeviceToHost));
  if (d[0]) {
    VT_CUDA(cudaMemset(h->cache->d_diag(), 0, sizeof(int)));
    vt::fail(VT_ERR_TIMEOUT, "tensor-core wait expired in an NRC kernel");
  }
}

void upload_samples(vt_nrc* h, const float* src, size_t n, size_t floats) {
  h->io.resize(std::max<size_t>(1, n * floats / 4));
  VT_CUDA(cudaMemcpyAsync(h->io.ptr, src, n * floats * sizeof(float), cudaMemcpyHostToDevice, h->stream));
}

}  // namespace

extern "C" {

vt_status vt_nrc_create(int32_t device, const vt_nrc_config* config, vt_nrc** out) {
  return vt::guard([&] {
    if (!config || !out) vt::fail(VT_ERR_INVALID_ARGUMENT, "config and out must be non-null");
    *out = nullptr;
    int count = 0;
    VT_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) vt::fail(VT_ERR_INVALID_ARGUMENT, "no such CUDA device");
    vt::DeviceScope ds(device);
    auto* h = new vt_nrc();
    try {
      h->device = device;
      VT_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
      h->cache = new vt::nrc::Cache(to_config(config), config->seed);
    } catch (...) {
      delete h->cache;
      if (h->stream) cudaStreamDestroy(h->stream);
      delete h;
      throw;
    }
    *out = h;
  });
}

vt_status vt_nrc_destroy(vt_nrc* h) {
  return vt::guard([&] {
    if (!h) return;
    vt::DeviceScope ds(h->device);
    cudaStreamSynchronize(h->stream);
    delete h->cache;
    h->io.release();
    h->rgb.release();
    cudaStreamDestroy(h->stream);
    delete h;
  });
}

vt_status vt_nrc_query(vt_nrc* h, const float* records, size_t n, float* rgb) {
  return vt::guard([&] {
    if (!h) vt::fail(VT_ERR_INVALID_ARGUMENT, "nrc is null");
    if (n && (!records || !rgb)) vt::fail(VT_ERR_INVALID_ARGUMENT, "records and rgb must be non-null");
    if (n > 0x7FFFFFFFull) vt::fail(VT_ERR_RANGE, "at most 2^31 - 1 queries per call");
    if (!n) return;
    vt::DeviceScope ds(h->device);
    upload_samples(h, records, n, VT_NRC_RECORD_FLOATS);
    h->rgb.resize(3 * n);
    h->cache->query(h->io.ptr, 4, nullptr, (uint32_t)n, h->rgb.ptr, nullptr, h->stream);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaMemcpyAsync(rgb, h->rgb.ptr, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    VT_CUDA(cudaStreamSynchronize(h->stream));
    check_diag(h);
  });
}

vt_status vt_nrc_train(vt_nrc* h, const float* samples, size_t n, float* loss) {
  return vt::guard([&] {
    if (!h) vt::fail(VT_ERR_INVALID_ARGUMENT, "nrc is null");
    if (!samples || !n) vt::fail(VT_ERR_INVALID_ARGUMENT, "samples must be non-empty");
    if (n > 0x7FFFFFFFull) vt::fail(VT_ERR_RANGE, "at most 2^31 - 1 samples per step");
    vt::DeviceScope ds(h->device);
    upload_samples(h, samples, n, VT_NRC_SAMPLE_FLOATS);
    h->cache->train_step(h->io.ptr, (uint32_t)n, h->stream);
    VT_CUDA(cudaGetLastError());
    float l = 0.0f;
    VT_CUDA(cudaMemcpyAsync(&l, h->cache->d_loss(), sizeof l, cudaMemcpyDeviceToHost, h->stream));
    VT_CUDA(cudaStreamSynchronize(h->stream));
    check_diag(h);
    if (loss) *loss = l;
  });
}

vt_status vt_nrc_gradients(vt_nrc* h, const float* samples, size_t n, float* grad_weights, float* grad_table,
                           float* loss) {
  return vt::guard([&] {
    if (!h) vt::fail(VT_ERR_INVALID_ARGUMENT, "nrc is null");
    if (!samples || !n || !grad_weights) vt::fail(VT_ERR_INVALID_ARGUMENT, "samples and grad_weights required");
    if (n > 0x7FFFFFFFull) vt::fail(VT_ERR_RANGE, "at most 2^31 - 1 samples");
    vt::DeviceScope ds(h->device);
    upload_samples(h, samples, n, VT_NRC_SAMPLE_FLOATS);
    h->cache->gradients(h->io.ptr, (uint32_t)n, h->stream);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaMemcpyAsync(grad_weights, h->cache->d_grad_w(), VT_NRC_WEIGHT_COUNT * sizeof(float),
                            cudaMemcpyDeviceToHost, h->stream));
    if (grad_table)
      VT_CUDA(cudaMemcpyAsync(grad_table, h->cache->d_grad_table(), h->cache->table_pairs() * sizeof(float2),
                              cudaMemcpyDeviceToHost, h->stream));
    float l = 0.0f;
    VT_CUDA(cudaMemcpyAsync(&l, h->cache->d_loss(), sizeof l, cudaMemcpyDeviceToHost, h->stream));
    h->cache->clear_gradients(h->stream);
    VT_CUDA(cudaStreamSynchronize(h->stream));
    check_diag(h);
    if (loss) *loss = l;
  });
}

vt_status vt_nrc_query_device(vt_nrc* h, const float* d_records, size_t n, float* d_rgb, void* cuda_stream) {
  return vt::guard([&] {
    if (!h) vt::fail(VT_ERR_INVALID_ARGUMENT, "nrc is null");
    if (n && (!d_records || !d_rgb)) vt::fail(VT_ERR_INVALID_ARGUMENT, "records and rgb must be non-null");
    if (n > 0x7FFFFFFFull) vt::fail(VT_ERR_RANGE, "at most 2^31 - 1 queries per call");
    if (reinterpret_cast<uintptr_t>(d_records) % 16) vt::fail(VT_ERR_INVALID_ARGUMENT, "records must be 16-byte aligned");
    vt::DeviceScope ds(h->device);
    h->cache->query(reinterpret_cast<const float4*>(d_records), 4, nullptr, (uint32_t)n, d_rgb, nullptr,
                    static_cast<cudaStream_t>(cuda_stream));
    VT_CUDA(cudaGetLastError());
  });
}

vt_status vt_nrc_train_device(vt_nrc* h, const float* d_samples, size_t n, void* cuda_stream) {
  return vt::guard([&] {
    if (!h) vt::fail(VT_ERR_INVALID_ARGUMENT, "nrc is null");
    if (!d_samples || !n) vt::fail(VT_ERR_INVALID_ARGUMENT, "samples must be non-empty");
    if (n > 0x7FFFFFFFull) vt::fail(VT_ERR_RANGE, "at most 2^31 - 1 samples per step");
    if (reinterpret_cast<uintptr_t>(d_samples) % 16) vt::fail(VT_ERR_INVALID_ARGUMENT, "samples must be 16-byte aligned");
    vt::DeviceScope ds(h->device);
    h->cache->train_step(reinterpret_cast<const float4*>(d_samples), (uint32_t)n, static_cast<cudaStream_t>(cuda_stream));
    VT_CUDA(cudaGetLastError());
  });
}

vt_status vt_nrc_get_params(vt_nrc* h, float* weights, float* table) {
  return vt::guard([&] {
    if (!h) vt::fail(VT_ERR_INVALID_ARGUMENT, "nrc is null");
    vt::DeviceScope ds(h->device);
    VT_CUDA(cudaStreamSynchronize(h->stream));
    h->cache->get_params(weights, table);
  });
}

vt_status vt_nrc_set_params(vt_nrc* h, const float* weights, const float* table) {
  return vt::guard([&] {
    if (!h) vt::fail(VT_ERR_INVALID_ARGUMENT, "nrc is null");
    vt::DeviceScope ds(h->device);
    VT_CUDA(cudaStreamSynchronize(h->stream));
    h->cache->set_params(weights, table);
  });
}

}  // extern "C"
