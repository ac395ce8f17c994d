// nrc.h -- neural radiance cache: multiresolution hash-grid encoding feeding a
// fully fused 64-wide MLP on the tcgen05 tensor cores, trained online with
// Adam (hand-written forward, backward and optimizer kernels).
//
// Model (Mueller et al. 2021 NRC with the Instant-NGP hash grid, as
// walkaround-hybrid/src/neural/nrc/ implements it):
//   input (64 fp16) = hash grid L x 2 features of the normalised position
//                     | real SH of degree 4 (16) of the outgoing direction
//                     | normal (3) | roughness (1) | diffuse albedo (3)
//                     | specular albedo (3) | 1 | 0 padding
//   5 hidden layers 64 -> 64 with ReLU, output layer 64 -> 3 (linear)
//   loss: relative L2 on the prediction's luminance (stop-gradient
//         denominator), fusedMlp.wgsl.ts:62-110
//   Adam (beta 0.9 / 0.999), f32 master weights and table, fp16 copies for the
//   kernels, non-finite guards and +-65504 clamp (fusedMlpTrainer.ts:30-80).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace vt {
namespace nrc {

constexpr int kWidth = 64;         // network width (input is padded to it)
constexpr int kLayers = 6;         // 5 hidden + output (output padded to 64 rows)
constexpr int kOut = 3;
constexpr int kMaxLevels = 16;
constexpr int kFeatures = 2;       // features per hash-table entry
constexpr int kEncWidth = kMaxLevels * kFeatures;  // 32 hash-grid inputs (unused levels are zero)
constexpr int kTile = 128;         // samples per MMA tile (M)
constexpr int kRecordFloats = 16;  // query / training features per sample
constexpr int kWeights = kLayers * kWidth * kWidth;

// Input column layout
enum : int { kColSh = 32, kColNormal = 48, kColRough = 51, kColDiffuse = 52, kColSpecular = 55, kColOne = 58 };

// Query tiles in flight per inference CTA when the configuration leaves it open:
// one CTA per SM keeps 4 T warps in flight; 1,048,576 queries of the 16 x 2^19
// grid took 0.75 / 0.46 / 0.40 / 0.39 ms with T = 1 / 2 / 3 / 4.
constexpr int kDefaultInferTiles = 4;

struct Config {
  int levels = 16;
  int log2_table = 19;
  float base_resolution = 16.0f;
  float growth = 1.5f;
  float lr = 1e-2f;          // MLP
  float table_lr = 1e-2f;    // hash grid
  float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  float aabb_min[3] = {0, 0, 0}, aabb_max[3] = {1, 1, 1};
  int infer_tiles = kDefaultInferTiles;  // query tiles of 128 in flight per inference CTA (1..4)
};

// Device-side view used by the kernels.
constexpr long long kDefaultWaitCycles = 2000000000ll;  // ~1 s at 2 GHz

struct View {
  const __half* w16 = nullptr;       // [6][64 out][64 in] fp16 weights
  const __half2* table16 = nullptr;  // [levels][T] fp16 feature pairs
  float* grad_w = nullptr;           // [6][64][64] f32 (training)
  float2* grad_table = nullptr;      // [levels][T] f32 pairs (training)
  int levels = 16;
  uint32_t table_mask = 0;           // T - 1
  float res[kMaxLevels] = {};        // per-level grid resolution floor(Nmin * b^l)
  float aabb_min[3] = {0, 0, 0};
  float aabb_inv[3] = {1, 1, 1};     // 1 / extent (0 for a flat axis)
  int* error = nullptr;              // non-zero: a bounded wait expired (kernel returned early)
  // clocks a kernel waits for its MMAs before it gives up (sets *error, drains
  // under the full limit, frees TMEM, returns); shortened only to test that path
  long long wait_cycles = kDefaultWaitCycles;
  float* loss = nullptr;             // sum of per-sample losses of a training step
  // error estimate per screen tile: samples whose target.w holds (pixel + 1) add
  // (prediction luminance, target luminance, 1) to tile_stats[3 * tile]
  float* tile_stats = nullptr;
  uint32_t tile_width = 0;           // image width in pixels
  uint32_t tile_size = 16;           // tile edge in pixels
  uint32_t tiles_x = 0;
};

// Features of one cache query / training sample: 4 float4
//   (P.xyz, wo.x) (wo.yz, n.xy) (n.z, roughness, diffuse.rg) (diffuse.b, specular.rgb)

// Inference over n records -> rgb[n] (or added into radiance[path] * throughput when
// `paths` is given: records are followed by (path id bits, T.rgb) float4 each).
// tiles_per_cta: query tiles of 128 in flight per CTA, one per warpgroup (1..4).
void launch_infer(const View& v, const float4* records, uint32_t rec_stride_f4, const uint32_t* n_dev, uint32_t n,
                  float* rgb_out, float4* radiance, int tiles_per_cta, cudaStream_t s);
// One training pass over n samples (records + float4 target per sample):
// accumulates mean-loss gradients into v.grad_w / v.grad_table (which must be zero).
void launch_train(const View& v, const float4* samples, uint32_t n, cudaStream_t s);
// Adam over `count` parameters: master -= lr * mhat / (sqrt(vhat) + eps); writes the
// fp16 copy and clears the gradient.  bc1/bc2 = 1 - beta^t.
void launch_adam(float* master, float* m, float* v, float* grad, __half* out16, size_t count, float lr,
                 float beta1, float beta2, float eps, float bc1, float bc2, int* diag, cudaStream_t s);
// The same for the table, whose f32 gradient pairs and fp16 copies are float2 / half2.
void launch_adam_table(float* master, float* m, float* v, float2* grad, __half2* out16, size_t pairs, float lr,
                       float beta1, float beta2, float eps, float bc1, float bc2, int* diag, cudaStream_t s);

// Host: level resolutions floor(base * growth^l) (nrcEncoding.ts levelResolution).
void level_resolutions(const Config& c, float* out);

}  // namespace nrc
}  // namespace vt
