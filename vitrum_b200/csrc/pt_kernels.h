// pt_kernels.h -- device views and launchers of the wavefront path tracer.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "pt_common.cuh"

namespace vt {
namespace pt {

// Scene as the shading kernels see it.  Geometry lives in the BVH's triangle
// records (vertices, source id in v0.w, material id in v1.w, reference
// normal + validity in the fourth float4).
// Positional delta lights (points, then spots), kPositionalF4 float4 each:
//   (position, 0), (intensity rgb, 0), (axis, cos outer), (cos inner, range, decay, 1 for a spot)
// Analytic area lights (rectangles, then discs), kAreaLightF4 float4 each:
//   (centre, 0 rectangle / 1 disc), (u half axis, area), (v half axis, 0), (radiance rgb, 0)
// a rectangle spans centre + [-1,1] u + [-1,1] v, a disc centre + u x + v y with
// x^2 + y^2 <= 1; the emitting side is u x v.
constexpr int kPositionalF4 = 4;
// Paths per wave when the options leave it open: 16 M (about 4.7 GB of wave
// state).  Larger waves shorten the tails of the late bounces' and the shadow
// rays' launches: the instanced 1080p frame took 45.0 / 37.9 / 33.9 ms and the
// box room 32.0 / 31.2 / 30.9 ms at 4 / 8 / 16 M paths.
constexpr int kDefaultWavePaths = 1 << 24;
constexpr int kAreaLightF4 = 4;

struct SceneView {
  const uint4* nodes = nullptr;
  const float4* tris = nullptr;
  int stack_depth = 16;
  const Material* materials = nullptr;
  uint32_t material_count = 0;
  // emissive triangles: 3 float4 each = (v0, emitter material bits), (v1, area), (v2, 0)
  const float4* emitters = nullptr;
  const float* emitter_cdf = nullptr;  // inclusive cumulative area / total, one per emitter
  uint32_t n_emitters = 0;
  float emit_area_total = 0.0f;
  const float4* points = nullptr;       // positional delta lights (layout above)
  uint32_t n_points = 0;
  const float4* area_lights = nullptr;  // analytic rectangle / disc lights (layout above)
  uint32_t n_area = 0;
  // directional lights: 2 float4 each = (direction towards the light, cos of the angular radius),
  // (rgb: irradiance of a delta light or radiance of a disc, 1 for delta)
  const float4* dirs = nullptr;
  uint32_t n_dirs = 0;
  // equirectangular environment (rgb as float4), with marginal/conditional CDFs
  const float4* env = nullptr;
  const float* env_marginal = nullptr;  // env_h + 1 entries
  const float* env_conditional = nullptr;  // env_h rows of env_w + 1 entries
  int env_w = 0, env_h = 0;
  float env_scale = 1.0f;
  float env_cos = 1.0f, env_sin = 0.0f;  // environment rotation about +y (rotationY)
  // light entries, chosen uniformly by NEE: the emissive-mesh group (if any),
  // positional lights, analytic area lights, directional lights, environment (if any)
  uint32_t n_light_entries = 0;
  // next-event selection: uniform over the entries, or (light_tree_mode) the
  // light tree over the positional entries (light_tree.h layout; nullptr when
  // there is one) with the distant entries (directionals, environment) outside it
  bool light_tree_mode = false;
  const float* light_tree = nullptr;
  // two-level scenes: instance records (4 float4: world-to-local rows, (blas root, id, material, 0))
  const float4* insts = nullptr;       // in top-level leaf order (traversal)
  const float4* inst_table = nullptr;  // by instance index (shading)
  uint32_t root = 0;                   // first node of the traversal
  float bias = 2e-5f;            // origin offset along the geometric normal, relative to max(1, |P|_inf)
};

// One scene of a batch (the batched persistent launch): its scene view,
// camera and sampling, and where its paths and pixels sit in the batch.
struct BatchScene {
  SceneView view;
  float inv_vp[16];
  uint32_t width = 0, height = 0, spp = 0, max_bounces = 0;
  uint32_t frame_seed = 0;
  uint32_t accum_offset = 0;            // first pixel of this scene in the batch accumulation
  unsigned long long path_begin = 0;    // first path of this scene in the batch's path space
};

// Auxiliary outputs (kernel.wgsl.ts:936-960): one float4 per pixel each.
// consts (device): view-projection (16 floats, row-major), the previous
// frame's view-projection (16), then as u32 bits the accumulated sample index
// whose first hit the normal / albedo / motion buffers record.
struct AuxView {
  float4* normal_depth = nullptr;  // (n * 0.5 + 0.5, distance) of the recorded sample's first hit
  float4* albedo = nullptr;        // (base colour, 1)
  float4* motion = nullptr;        // (pixels x, y, 0, 1)
  float4* moments = nullptr;       // (sum L, sum L^2, samples, 0), L = Rec. 709 luminance of a sample
  const float* consts = nullptr;
};
// then the camera block at kCamConsts: the inverse view-projection (16 floats,
// row-major) and the frame seed (u32 bits), written every frame so that a
// new camera or seed needs no new graph
constexpr int kCamConsts = 36;
constexpr int kAuxConsts = kCamConsts + 17;

struct FrameView {
  const float* cam = nullptr;  // device: inverse view-projection (16 floats, row-major), frame seed (u32 bits)
  uint32_t width = 0, height = 0;
  uint32_t spp_wave = 1;    // samples per pixel in one wave
  uint32_t max_bounces = 5;
  uint32_t paths = 0;       // width * height * spp_wave
  uint32_t sort_by_material = 1;
  // neural radiance cache
  uint32_t train = 0;                  // training wave: random pixels, one record per vertex, no accumulation
  uint32_t record_bounces = 0;         // record slots per training path
  uint32_t nrc_prefix = 0xFFFFFFFFu;   // render waves: hits of this bounce become cache queries
  const float* nrc_tile_error = nullptr;  // per screen tile: cache error estimate (render waves)
  float nrc_fallback = 0.0f;           // tiles above this error continue as plain path tracing
  uint32_t nrc_tile = 16, nrc_tiles_x = 0;
  float nrc_spread_c = 0.0f;           // > 0: spread termination (nrc_prefix unused): query at the first
                                       // vertex k >= 2 with a(x_k) > c * a0 (spreadTermination.ts:70-184)
  AuxView aux;              // null buffers: no auxiliary outputs (training waves, batches)
  // batch: paths of many scenes in one wave (scene id in bits 8-15 of the path flags)
  const BatchScene* batch = nullptr;
  uint32_t n_scenes = 0;
  unsigned long long batch_paths = 0;  // total paths of the batch
};

// Path queues (double-buffered), hit records, shadow queue and per-path radiance.
struct WaveBuffers {
  float4* rays[2] = {nullptr, nullptr};    // 2 float4 per path (vt_ray)
  uint4* state[2] = {nullptr, nullptr};    // (path id, rng, flags, prev pdf bits)
  float4* through[2] = {nullptr, nullptr}; // throughput rgb
  int4* hits = nullptr;
  uint32_t* order = nullptr;               // material-sorted permutation of the current queue
  uint32_t* keys = nullptr;
  float4* shadow_rays = nullptr;           // 2 float4 per shadow ray
  float4* shadow_contrib = nullptr;        // rgb, path id bits
  uint8_t* occluded = nullptr;
  float4* radiance = nullptr;              // per path id
  uint32_t* counters = nullptr;            // [queue0, queue1, shadow, hist[8], cursor[8], wave_sample]
  unsigned long long* trace_counter = nullptr;
  int* trace_status = nullptr;
  // neural radiance cache
  float4* nrc_records = nullptr;   // training: 6 float4 per (path, bounce) = features, (A rgb, valid), (T rgb, 0)
  float4* nrc_queries = nullptr;   // render: 5 float4 per query = features, (path bits, T rgb)
  uint32_t* nrc_seed = nullptr;    // training-wave counter (pixel choice and RNG key)
  // batch
  uint32_t* ray_root[2] = {nullptr, nullptr};  // traversal root node per queued ray
  uint32_t* shadow_root = nullptr;
  uint32_t* path_pixel = nullptr;              // batch accumulation pixel per path
  unsigned long long* batch_cursor = nullptr;  // first path of the next wave
};

enum : int {
  kCntShadow = 2, kCntHist = 3, kCntCursor = 11, kCntWaveSample = 19, kCntQuery = 20, kCntSamples = 21,
  kCntBatchPaths = 22,
  // the counting sorts' per-(CTA, key) counts and offsets (kSortGrid CTAs, up to 8 keys)
  kCntSortHist = 23, kCntSortOff = 23 + 148 * 8 * 8, kCntWords = 23 + 2 * 148 * 8 * 8
};
constexpr uint32_t kSortGrid = 148 * 8;  // CTAs of the counting sorts (one contiguous queue range each)

// Accumulation targets.
struct AccumView {
  float4* accum = nullptr;    // rgb sum, sample count (FP32, the displayed estimate)
  double* sum64 = nullptr;    // 3 per pixel, FP64 sum (oracle accumulation)
  double* sq64 = nullptr;     // 3 per pixel, FP64 sum of squares
  double* lum64 = nullptr;    // 4 per pixel, FP64 sums of L, L^2, L^3, L^4 (L: a sample's Rec. 709 luminance)
};

void launch_raygen(const FrameView& f, const WaveBuffers& w, cudaStream_t s);
void launch_sort_by_material(const SceneView& sc, const FrameView& f, const WaveBuffers& w, int cur,
                             uint32_t capacity, cudaStream_t s);
// w.order = the closest-hit queue `cur` partitioned by ray direction octant (trace order)
void launch_sort_rays(const WaveBuffers& w, int cur, uint32_t capacity, cudaStream_t s);
void launch_shade(const SceneView& sc, const FrameView& f, const WaveBuffers& w, int cur, uint32_t bounce,
                  uint32_t capacity, cudaStream_t s);
void launch_shadow_resolve(const WaveBuffers& w, uint32_t capacity, cudaStream_t s);
void launch_accumulate(const FrameView& f, const WaveBuffers& w, const AccumView& a, cudaStream_t s);
// Auxiliary outputs of the recorded sample, after the bounce-0 closest-hit trace
// (no-op without aux buffers or when this wave does not hold that sample).
void launch_aux_first_hit(const SceneView& sc, const FrameView& f, const WaveBuffers& w, cudaStream_t s);
// Batch: the next `capacity` paths of the batch's path space (device cursor),
// and their accumulation (atomic per pixel) followed by the cursor advance.
void launch_raygen_batch(const FrameView& f, const WaveBuffers& w, uint32_t capacity, cudaStream_t s);
void launch_accumulate_batch(const WaveBuffers& w, float4* accum, uint32_t capacity, cudaStream_t s);
// Present pass of an accumulation (sums with the sample count in .w): the mean
// through exposure and a tonemap (0 ACES filmic, 1 AgX, 2 Reinhard, 3 clamp,
// 4 none), then the sRGB OETF when `srgb` (present.wgsl.ts:59-80).
void launch_capture_mean(const float4* accum, size_t pixels, float4* out, cudaStream_t s);
void launch_present(const float4* accum, size_t pixels, int tonemap, float exposure, int srgb, float4* out,
                    cudaStream_t s);
// totals[0] += queue count traced this bounce, totals[1] += shadow rays traced
void launch_count_rays(const WaveBuffers& w, int cur, unsigned long long* totals, cudaStream_t s);

// Training samples from a finished training wave: target = (L_final - A) / T
// per recorded vertex (the radiance the path gathered after the vertex, per
// unit throughput), clamped to [0, 1024] (recordUnpack.ts NRC_MAX_TRAINING_TARGET);
// appended to `samples` (5 float4 each) up to `capacity`, then the remaining
// slots are filled cyclically from the collected ones.
void launch_nrc_targets(const WaveBuffers& w, uint32_t paths, uint32_t bounces, float4* samples, uint32_t capacity,
                        uint32_t query_bounce, cudaStream_t s);
// Error map update after a frame's training: err = EMA of |sum pred - sum target| / (sum target + 1e-3)
// over the tile's query-vertex samples; clears the sums.
void launch_nrc_tile_update(float* tile_stats, float* tile_error, uint32_t tiles, float alpha, cudaStream_t s);

}  // namespace pt
}  // namespace vt
