// pt_kernels.cu -- wavefront stages of the unidirectional path tracer.
//
// One wave = width*height*spp_wave paths.  Stages per bounce:
//   extend   closest hit of the live queue (k_trace, traverse.cu)
//   sort     counting sort of the queue by the hit's BSDF family (miss,
//            Lambert, conductor, dielectric) so shading warps run one family
//   shade    emission (MIS), next-event estimation on the area-light group,
//            point lights and the environment (one light entry chosen
//            uniformly, power-heuristic MIS against the BSDF pdf), BSDF
//            sampling, Russian roulette, warp-ballot compaction of survivors
//            and shadow rays into the next queues
//   shadow   any hit of the shadow queue (k_trace)
//   resolve  unoccluded shadow contributions added to the path's radiance
// and after the last bounce `accumulate` folds each pixel's samples into the
// FP32 accumulation (and, for the oracle, FP64 sums and sums of squares).
//
// Estimator (restated from pt-webgpu/src/wgsl/pathTrace/kernel.wgsl.ts:963-2030
// for the Lambert / GGX-conductor / smooth-dielectric subset):
//  - camera emission and emission after a delta event: weight 1;
//  - emission reached by a BSDF sample: power(pdf_bsdf, pdf_light);
//  - NEE: power(pdf_light, pdf_bsdf) for area / environment, 1 for points;
//    at the last vertex (no continuation is traced) NEE takes weight 1 so the
//    two strategies still sum to one for every path length;
//  - RR for bounce index > 2: survival clamp(max T, 0.1, 0.95), 2^-24 buckets.
#include <cuda_runtime.h>

#include <cstdint>

#include "light_tree.cuh"
#include "pt_common.cuh"
#include "pt_kernels.h"
#include "vt_common.h"

namespace vt {
namespace pt {

namespace {

constexpr uint32_t kFull = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t rand_bounded(uint32_t& s, uint32_t bound) {
  if (bound <= 1u) return 0u;
  const uint32_t threshold = (0u - bound) % bound;
  uint32_t v = pcg_next(s);
  for (int k = 0; k < 64 && v < threshold; ++k) v = pcg_next(s);  // P(retry) < bound / 2^32
  return v % bound;
}


// first index with cdf[i] > u (cdf inclusive, last entry 1)
__device__ __forceinline__ uint32_t cdf_search(const float* cdf, uint32_t n, float u) {
  uint32_t lo = 0, hi = n - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (cdf[mid] > u) hi = mid; else lo = mid + 1;
  }
  return lo;
}

// ---------------------------------------------------------------- environment
__device__ __forceinline__ void env_texel(const SceneView& sc, float3 dw, int& col, int& row, float& sin_t) {
  // world direction into the unrotated map: rotation about +y by -rotationY (rotateYNeg, connectCore.wgsl.ts:27-30)
  const float3 d = f3(sc.env_cos * dw.x - sc.env_sin * dw.z, dw.y, sc.env_sin * dw.x + sc.env_cos * dw.z);
  const float y = fminf(fmaxf(d.y, -1.0f), 1.0f);
  const float theta = acosf(y);
  // equirectangular convention u = phi / 2pi + 0.5 (wrapped), +x at the middle
  // column, row 0 at +y (environmentLookup, connect.wgsl.ts:139-142)
  float u = atan2f(d.z, d.x) * (0.5f / CUDART_PI_F) + 0.5f;
  if (u >= 1.0f) u -= 1.0f;
  col = min(sc.env_w - 1, (int)(u * sc.env_w));
  row = min(sc.env_h - 1, (int)(theta * (1.0f / CUDART_PI_F) * sc.env_h));
  sin_t = sinf(theta);
}

__device__ __forceinline__ float env_pdf_texel(const SceneView& sc, int col, int row, float sin_t) {
  if (!(sin_t > 0.0f)) return 0.0f;
  const float pm = sc.env_marginal[row + 1] - sc.env_marginal[row];
  const float* cc = sc.env_conditional + (size_t)row * (sc.env_w + 1);
  const float pc = cc[col + 1] - cc[col];
  return pm * pc * (float)sc.env_w * (float)sc.env_h / (2.0f * CUDART_PI_F * CUDART_PI_F * sin_t);
}

__device__ __forceinline__ float3 env_radiance(const SceneView& sc, int col, int row) {
  const float4 e = __ldg(sc.env + (size_t)row * sc.env_w + col);
  return f3(e.x, e.y, e.z) * sc.env_scale;
}

// ---------------------------------------------------------------- light sample
struct LightSample {
  float3 wi;
  float dist;       // distance to the light point (inf for the environment)
  float3 Le;        // emitted radiance (area/env) or intensity / dist^2 (point)
  float pdf;        // solid-angle pdf including the entry selection (delta: selection only)
  float pdf_light;  // the same without the selection: the density the MIS weights compare
  bool delta;
  bool valid;
};

// Distance falloff of point and spot lights: 1 / d^decay (none for decay <= 0.01;
// exactly 1 / d^2 for decay 2) times the range window clamp(1 - (d / range)^4, 0, 1)
// for range > 0 (pointSpotDistanceAttenuation, material.wgsl.ts:2176-2204).
__device__ __forceinline__ float positional_falloff(float dist, float d2, float range, float decay) {
  if (!(dist > 0.0f) || dist > 3.402823466e38f) return 0.0f;
  float a = 1.0f;
  if (decay > 0.01f) {
    const float den = decay == 2.0f ? d2 : powf(dist, decay);
    if (!(den > 0.0f)) a = 3.402823466e38f;
    else if (den > 3.402823466e38f) return 0.0f;
    else a = fminf(1.0f / den, 3.402823466e38f);
  }
  if (range > 0.0f) {
    const float q = dist / range, q2 = q * q;
    a *= clamp01(1.0f - q2 * q2);
  }
  return a;
}
// smoothstep(e0, e1, x) (kernel.wgsl.ts:1382, spot penumbra)
__device__ __forceinline__ float smoothstep_f(float e0, float e1, float x) {
  const float t = clamp01((x - e0) / (e1 - e0));
  return t * t * (3.0f - 2.0f * t);
}
// Shirley-Chiu concentric map of (a, b) in [-1,1]^2 to the unit disc
__device__ __forceinline__ float2 concentric_disc(float a, float b) {
  if (a == 0.0f && b == 0.0f) return make_float2(0.0f, 0.0f);
  float r, phi;
  if (fabsf(a) > fabsf(b)) {
    r = a;
    phi = (0.25f * CUDART_PI_F) * (b / a);
  } else {
    r = b;
    phi = 0.5f * CUDART_PI_F - (0.25f * CUDART_PI_F) * (a / b);
  }
  return make_float2(r * cosf(phi), r * sinf(phi));
}
// Nearest analytic area light that the ray (o, d) crosses from its emitting
// side before t_max: its radiance and the solid-angle density of reaching that
// point by sampling the light (connect.wgsl.ts:390-450; the lights are no occluders).
__device__ __forceinline__ bool area_light_hit(const SceneView& sc, float3 o, float3 d, float t_max, float3& Le,
                                               float& pdf_sa) {
  bool found = false;
  float best = t_max;
  for (uint32_t k = 0; k < sc.n_area; ++k) {
    const float4* q = sc.area_lights + kAreaLightF4 * (size_t)k;
    const float4 a0 = __ldg(q), a1 = __ldg(q + 1), a2 = __ldg(q + 2);
    const float3 U = f3(a1.x, a1.y, a1.z), V = f3(a2.x, a2.y, a2.z);
    const float3 nl = normalize(cross(U, V));
    const float den = dot(nl, d);
    if (!(den < 0.0f)) continue;  // behind or edge-on
    const float3 c = f3(a0.x, a0.y, a0.z);
    const float t = dot(nl, c - o) / den;
    if (!(t > 0.0f && t < best)) continue;
    const float3 rel = o + d * t - c;
    const float uu = dot(U, U), uv = dot(U, V), vv = dot(V, V), ru = dot(rel, U), rv = dot(rel, V);
    const float det = uu * vv - uv * uv;
    const float x = (ru * vv - rv * uv) / det, y = (rv * uu - ru * uv) / det;
    const bool inside = a0.w != 0.0f ? x * x + y * y <= 1.0f : (fabsf(x) <= 1.0f && fabsf(y) <= 1.0f);
    if (!inside) continue;
    best = t;
    found = true;
    const float4 a3 = __ldg(q + 3);
    Le = f3(a3.x, a3.y, a3.z);
    pdf_sa = t * t / (a1.w * -den);
  }
  return found;
}

// N: the unit normal on the incoming side for surfaces that only reflect,
// zero for transmissive ones (the light tree's receiver term)
__device__ LightSample sample_light(const SceneView& sc, float3 P, float3 N, uint32_t& rng) {
  LightSample ls;
  ls.valid = false;
  ls.delta = false;
  const uint32_t n = sc.n_light_entries;
  // entry selection: the light tree (one 24-bit draw, power x proximity x
  // orientation, lightTree.ts:1237-1319) or uniform; its probability is divided
  // out of the estimate but kept out of the MIS weights, as the reference does
  // (pt-webgpu mediumNee.wgsl.ts:14-37, connect.wgsl.ts:598)
  float psel;
  uint32_t e;
  if (sc.light_tree_mode) {
    const uint32_t n_dist = sc.n_dirs + (sc.env_marginal ? 1u : 0u);
    psel = lt::select(sc.light_tree, n - n_dist, n_dist, P.x, P.y, P.z, N.x, N.y, N.z, pcg_next(rng) >> 8, e);
    if (e >= n || !(psel > 0.0f)) return ls;
  } else {
    psel = 1.0f / (float)n;
    e = rand_bounded(rng, n);
  }
  const bool has_area = sc.n_emitters > 0;
  if (has_area) {
    if (e == 0) {
      const float u = rand01(rng);
      const uint32_t k = cdf_search(sc.emitter_cdf, sc.n_emitters, u);
      const float4 a = __ldg(sc.emitters + 3 * k), b = __ldg(sc.emitters + 3 * k + 1), c = __ldg(sc.emitters + 3 * k + 2);
      float u1 = rand01(rng), u2 = rand01(rng);
      const float su = sqrtf(u1);
      const float wa = 1.0f - su, wb = su * (1.0f - u2), wc = su * u2;
      const float3 A = f3(a.x, a.y, a.z), B = f3(b.x, b.y, b.z), C = f3(c.x, c.y, c.z);
      const float3 X = A * wa + B * wb + C * wc;
      const float3 nl = normalize(cross(B - A, C - A));
      const float3 d = X - P;
      const float d2 = dot(d, d);
      const float dist = sqrtf(d2);
      ls.wi = d * (1.0f / dist);
      const float cosl = -dot(ls.wi, nl);
      if (!(cosl > 0.0f) || !(dist > 0.0f)) return ls;
      const Material m = sc.materials[__float_as_uint(a.w)];
      ls.Le = m.emission;
      ls.dist = dist;
      ls.pdf_light = d2 / (sc.emit_area_total * cosl);
      ls.pdf = psel * ls.pdf_light;
      ls.valid = true;
      return ls;
    }
    e -= 1;
  }
  if (e < sc.n_points) {
    // point or spot light (kernel.wgsl.ts:1285-1397)
    const float4* q = sc.points + kPositionalF4 * (size_t)e;
    const float4 p = __ldg(q), I = __ldg(q + 1), ax = __ldg(q + 2), ex = __ldg(q + 3);
    const float3 d = f3(p.x, p.y, p.z) - P;
    const float d2 = dot(d, d);
    if (!(d2 > 0.0f)) return ls;
    const float dist = sqrtf(d2);
    if (ex.y > 0.0f && dist > ex.y) return ls;  // beyond the range
    ls.wi = d * (1.0f / dist);
    float cone = 1.0f;
    if (ex.w != 0.0f) {
      const float c = -dot(ls.wi, f3(ax.x, ax.y, ax.z));
      if (!(c >= ax.w)) return ls;
      cone = smoothstep_f(ax.w, fmaxf(ex.x, ax.w + 1e-6f), c);
    }
    ls.dist = dist;
    ls.Le = f3(I.x, I.y, I.z) * (cone * positional_falloff(dist, d2, ex.y, ex.z));
    ls.pdf = psel;
    ls.pdf_light = 1.0f;
    ls.delta = true;
    ls.valid = true;
    return ls;
  }
  e -= sc.n_points;
  if (e < sc.n_area) {
    // rectangle (uniform in [-1,1]^2) or disc (concentric map), one-sided
    // (kernel.wgsl.ts:1398-1493)
    const float4* q = sc.area_lights + kAreaLightF4 * (size_t)e;
    const float4 a0 = __ldg(q), a1 = __ldg(q + 1), a2 = __ldg(q + 2), a3 = __ldg(q + 3);
    const float xi1 = rand01(rng), xi2 = rand01(rng);
    float x = xi1 * 2.0f - 1.0f, y = xi2 * 2.0f - 1.0f;
    if (a0.w != 0.0f) {
      const float2 cd = concentric_disc(x, y);
      x = cd.x;
      y = cd.y;
    }
    const float3 U = f3(a1.x, a1.y, a1.z), V = f3(a2.x, a2.y, a2.z);
    const float3 X = f3(a0.x, a0.y, a0.z) + U * x + V * y;
    const float3 d = X - P;
    const float d2 = dot(d, d);
    const float dist = sqrtf(d2);
    if (!(dist > 0.0f)) return ls;
    ls.wi = d * (1.0f / dist);
    const float cosl = -dot(ls.wi, normalize(cross(U, V)));
    if (!(cosl > 0.0f)) return ls;
    ls.Le = f3(a3.x, a3.y, a3.z);
    ls.dist = dist;
    ls.pdf_light = d2 / (a1.w * cosl);
    ls.pdf = psel * ls.pdf_light;
    ls.valid = true;
    return ls;
  }
  e -= sc.n_area;
  if (e < sc.n_dirs) {
    const float4 dw = __ldg(sc.dirs + 2 * e), dl = __ldg(sc.dirs + 2 * e + 1);
    const float3 w = f3(dw.x, dw.y, dw.z);
    ls.dist = CUDART_INF_F;
    ls.Le = f3(dl.x, dl.y, dl.z);
    if (dl.w != 0.0f) {  // delta: irradiance along w
      ls.wi = w;
      ls.pdf = psel;
      ls.pdf_light = 1.0f;
      ls.delta = true;
    } else {  // disc of angular radius acos(dw.w): uniform in the cone
      const float u1 = rand01(rng), u2 = rand01(rng);
      const float ct = 1.0f - u1 * (1.0f - dw.w), st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
      const float ph = 2.0f * CUDART_PI_F * u2;
      float3 tu, tv;
      onb(w, tu, tv);
      ls.wi = tu * (st * cosf(ph)) + tv * (st * sinf(ph)) + w * ct;
      ls.pdf_light = 1.0f / (2.0f * CUDART_PI_F * (1.0f - dw.w));
      ls.pdf = psel * ls.pdf_light;
    }
    ls.valid = true;
    return ls;
  }
  // environment
  const float u1 = rand01(rng), u2 = rand01(rng);
  const uint32_t row = cdf_search(sc.env_marginal + 1, (uint32_t)sc.env_h, u1);
  const float* cc = sc.env_conditional + (size_t)row * (sc.env_w + 1);
  const uint32_t col = cdf_search(cc + 1, (uint32_t)sc.env_w, u2);
  const float m0 = sc.env_marginal[row], m1 = sc.env_marginal[row + 1];
  const float c0 = cc[col], c1 = cc[col + 1];
  const float fv = m1 > m0 ? (u1 - m0) / (m1 - m0) : 0.5f;
  const float fu = c1 > c0 ? (u2 - c0) / (c1 - c0) : 0.5f;
  const float v = ((float)row + fminf(fmaxf(fv, 0.0f), 0.999999f)) / (float)sc.env_h;
  const float u = ((float)col + fminf(fmaxf(fu, 0.0f), 0.999999f)) / (float)sc.env_w;
  const float theta = v * CUDART_PI_F, phi = (u - 0.5f) * 2.0f * CUDART_PI_F;
  const float st = sinf(theta);
  const float3 md = f3(st * cosf(phi), cosf(theta), st * sinf(phi));  // map space; to world by +rotationY
  ls.wi = f3(sc.env_cos * md.x + sc.env_sin * md.z, md.y, -sc.env_sin * md.x + sc.env_cos * md.z);
  ls.dist = CUDART_INF_F;
  ls.Le = env_radiance(sc, (int)col, (int)row);
  ls.pdf_light = env_pdf_texel(sc, (int)col, (int)row, st);
  ls.pdf = psel * ls.pdf_light;
  ls.valid = ls.pdf > 0.0f;
  return ls;
}

// solid-angle pdf of reaching an emissive triangle point by sampling the
// emissive-mesh entry (given that entry: the MIS density)
__device__ __forceinline__ float area_light_pdf(const SceneView& sc, float dist, float cosl) {
  if (!(cosl > 0.0f)) return 0.0f;
  return dist * dist / (sc.emit_area_total * cosl);
}

// ---------------------------------------------------------------- light-tree probe
__global__ void k_light_tree_select(const float* tree, uint32_t n_pos, uint32_t n_dist, const float* points,
                                    const float* normals, const uint32_t* buckets, size_t n, uint32_t* entry,
                                    float* pmf) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t e = 0xFFFFFFFFu;
  const float nx = normals ? normals[3 * i] : 0.0f, ny = normals ? normals[3 * i + 1] : 0.0f,
              nz = normals ? normals[3 * i + 2] : 0.0f;
  pmf[i] = lt::select(tree, n_pos, n_dist, points[3 * i], points[3 * i + 1], points[3 * i + 2], nx, ny, nz,
                      buckets[i] & (lt::kBuckets - 1u), e);
  entry[i] = e;
}

// ---------------------------------------------------------------- raygen
// Pixel of the j-th path of a sample plane (j < W * H): 4 x 8 pixel tiles in
// row-major tile order, so the 32 paths of a warp look through one compact
// tile (their rays, and the next bounce's origins, lie close together); the
// pixels outside the full tiles follow, the right strip then the bottom rows,
// each row-major.  A bijection of [0, W * H); the per-pixel sample streams are
// keyed by the pixel, so the image does not depend on it.  Measured per frame
// (box room / instanced cloud): rows of 32 pixels 28.39 / 30.45 ms, 16 x 2
// tiles 28.25 / 30.41, 8 x 4 28.22 / 29.75, 4 x 8 28.15 / 29.35, 2 x 16
// 28.15 / 29.58.
__device__ __forceinline__ uint32_t tile_pixel(uint32_t j, uint32_t W, uint32_t H) {
  constexpr uint32_t kTw = 4, kTh = 8;
  const uint32_t cols = W / kTw, rows = H / kTh;
  const uint32_t full = cols * rows * (kTw * kTh);
  if (j < full) {
    const uint32_t t = j / (kTw * kTh), r = j % (kTw * kTh);
    return ((t / cols) * kTh + r / kTw) * W + (t % cols) * kTw + r % kTw;
  }
  uint32_t k = j - full;
  const uint32_t rw = W - cols * kTw, strip = rw * rows * kTh;
  if (k < strip) return (k / rw) * W + cols * kTw + k % rw;
  k -= strip;
  return (rows * kTh + k / W) * W + k % W;
}

__global__ void k_raygen(FrameView f, WaveBuffers w) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) w.counters[0] = f.paths;
  if (i >= f.paths) return;
  const uint32_t wh = f.width * f.height;
  uint32_t pix = tile_pixel(i % wh, f.width, f.height), s = i / wh;
  const float* M = f.cam;
  const uint32_t frame_seed = __float_as_uint(__ldg(M + 16));
  uint32_t key;
  if (f.train) {
    // training paths: uniformly random pixels, a key stream of their own
    uint32_t h = pcg_init(i, *w.nrc_seed, 0x7A3D9E1Bu ^ frame_seed);
    pix = pcg_next(h) % wh;
    key = pcg_next(h) | 1u;
  } else {
    key = frame_seed ^ (w.counters[kCntWaveSample] + s);
  }
  const uint32_t x = pix % f.width, y = pix / f.width;
  uint32_t rng = pcg_init(x, y, key);
  const float jx = rand01(rng), jy = rand01(rng);
  const float u = ((float)x + jx) / (float)f.width, v = ((float)y + jy) / (float)f.height;
  const float nx = u * 2.0f - 1.0f, ny = 1.0f - v * 2.0f;
  float nf[4], fr[4];
  for (int r = 0; r < 4; ++r) {
    nf[r] = M[4 * r] * nx + M[4 * r + 1] * ny - M[4 * r + 2] + M[4 * r + 3];
    fr[r] = M[4 * r] * nx + M[4 * r + 1] * ny + M[4 * r + 2] + M[4 * r + 3];
  }
  const float3 o = f3(nf[0] / nf[3], nf[1] / nf[3], nf[2] / nf[3]);
  const float3 far = f3(fr[0] / fr[3], fr[1] / fr[3], fr[2] / fr[3]);
  const float3 d = normalize(far - o);
  w.rays[0][2 * i] = make_float4(o.x, o.y, o.z, 0.0f);
  w.rays[0][2 * i + 1] = make_float4(d.x, d.y, d.z, CUDART_INF_F);
  w.state[0][i] = make_uint4(i, rng, 1u /* previous event delta: camera */, 0u);
  if (f.train && w.path_pixel) w.path_pixel[i] = pix;
  w.through[0][i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
  w.radiance[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// ---------------------------------------------------------------- material sort
// the material id the closest-hit traversal wrote with the hit (instance
// material, or the triangle record's)
__device__ __forceinline__ uint32_t hit_material(const SceneView& sc, int4 h) { return (uint32_t)h.w; }

__device__ __forceinline__ uint32_t hit_key(const SceneView& sc, int4 h) {
  if (h.x < 0) return 0u;
  return 1u + sc.materials[hit_material(sc, h)].kind;
}

// Counting sorts of the queue (by BSDF family for shading, by ray direction
// octant for tracing) into w.order, stable and without global atomics: CTA b
// of the grid owns one contiguous, warp-aligned range of the queue; it writes
// each entry's key and its range's per-key counts, one small kernel turns the
// counts into per-(CTA, key) offsets, and the CTA then scatters its range in
// order (warp ballots, a per-chunk scan over its warps).
__device__ __forceinline__ void sort_range(uint32_t n, uint32_t& lo, uint32_t& hi) {
  const uint32_t per = (((n + gridDim.x - 1) / gridDim.x) + 31u) & ~31u;
  lo = min(n, blockIdx.x * per);
  hi = min(n, lo + per);
}

// MODE 0: key 0 for a miss, else 1 + the hit material's BSDF kind (K = 4);
// MODE 1: the ray's direction octant (K = 8)
template <int K, int MODE>
__global__ void __launch_bounds__(256) k_sort_keys(SceneView sc0, FrameView f, WaveBuffers w, int cur) {
  const uint32_t n = w.counters[cur];
  uint32_t lo, hi;
  sort_range(n, lo, hi);
  __shared__ uint32_t cnt[K];
  if (threadIdx.x < K) cnt[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t local[K];
#pragma unroll
  for (int k = 0; k < K; ++k) local[k] = 0;
  for (uint32_t base = lo; base < hi; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const bool valid = i < hi;
    uint32_t key = 0xFFu;
    if (valid) {
      if (MODE == 0) {
        const SceneView& sc = f.batch ? f.batch[(w.state[cur][i].z >> 8) & 0xFFu].view : sc0;
        key = hit_key(sc, w.hits[i]);
      } else {
        const float4 d = w.rays[cur][2 * (size_t)i + 1];
        key = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
      }
      w.keys[i] = key;
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint32_t m = __ballot_sync(kFull, valid && key == (uint32_t)k);
      if (lane == 0) local[k] += (uint32_t)__popc(m);
    }
  }
  if (lane == 0)
    for (int k = 0; k < K; ++k)
      if (local[k]) atomicAdd(&cnt[k], local[k]);
  __syncthreads();
  if (threadIdx.x < K) w.counters[kCntSortHist + blockIdx.x * K + threadIdx.x] = cnt[threadIdx.x];
}

// per-(CTA, key) start offsets: key-major, CTAs in order within a key
template <int K>
__global__ void __launch_bounds__(1024) k_sort_offsets(WaveBuffers w, uint32_t g) {
  __shared__ uint32_t h[kSortGrid * K];
  __shared__ uint32_t tot[K];
  for (uint32_t i = threadIdx.x; i < g * K; i += blockDim.x) h[i] = w.counters[kCntSortHist + i];
  __syncthreads();
  if (threadIdx.x < K) {
    uint32_t run = 0;
    for (uint32_t b = 0; b < g; ++b) {
      const uint32_t c = h[b * K + threadIdx.x];
      h[b * K + threadIdx.x] = run;
      run += c;
    }
    tot[threadIdx.x] = run;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < g * K; i += blockDim.x) {
    uint32_t pre = 0;
    for (uint32_t k = 0; k < i % K; ++k) pre += tot[k];
    w.counters[kCntSortOff + i] = h[i] + pre;
  }
}

template <int K>
__global__ void __launch_bounds__(256) k_sort_scatter(WaveBuffers w, int cur) {
  const uint32_t n = w.counters[cur];
  uint32_t lo, hi;
  sort_range(n, lo, hi);
  __shared__ uint32_t base_k[K];
  __shared__ uint32_t wcnt[8][K];
  if (threadIdx.x < K) base_k[threadIdx.x] = w.counters[kCntSortOff + blockIdx.x * K + threadIdx.x];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  for (uint32_t base = lo; base < hi; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const bool valid = i < hi;
    const uint32_t key = valid ? w.keys[i] : 0xFFu;
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint32_t m = __ballot_sync(kFull, valid && key == (uint32_t)k);
      if (lane == 0) wcnt[wid][k] = (uint32_t)__popc(m);
      if (key == (uint32_t)k) mine = m;
    }
    __syncthreads();
    if (valid) {
      uint32_t pos = base_k[key];
      for (uint32_t q = 0; q < wid; ++q) pos += wcnt[q][key];
      pos += (uint32_t)__popc(mine & ((1u << lane) - 1u));
      w.order[pos] = i;
    }
    __syncthreads();
    if (threadIdx.x < K) {
      uint32_t t = 0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += wcnt[q][threadIdx.x];
      base_k[threadIdx.x] += t;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- cache features
// (position, outgoing direction, normal facing it, roughness, diffuse albedo,
// specular albedo) as the radiance cache's 16-float record.
__device__ __forceinline__ void nrc_features(const Material& m, float3 P, float3 wo, float3 n, float4 (&q)[4]) {
  const bool diel = m.kind == kDielectric;
  const float3 dif = m.base_color * (diel ? 1.0f - m.transmission : 1.0f - m.metallic);
  const float3 spe = diel ? f3(1.0f, 1.0f, 1.0f) : opaque_f0(m);
  q[0] = make_float4(P.x, P.y, P.z, wo.x);
  q[1] = make_float4(wo.y, wo.z, n.x, n.y);
  q[2] = make_float4(n.z, m.roughness, dif.x, dif.y);
  q[3] = make_float4(dif.z, spe.x, spe.y, spe.z);
}

// ---------------------------------------------------------------- shade
// 8 resident blocks per SM (64 registers, some spilled to L1): the kernel is
// load-latency bound, and occupancy beats spill-free code here.
// ---------------------------------------------------------------- auxiliary outputs
// projectToNdc (kernelCore.wgsl.ts:28-42): clip = M (p, 1) scaled by its
// largest magnitude, (2, 2) when that is zero or not finite or w <= 0.
__device__ __forceinline__ float2 project_ndc(const float* M, float3 p) {
  float c[4];
  for (int r = 0; r < 4; ++r) c[r] = M[4 * r] * p.x + M[4 * r + 1] * p.y + M[4 * r + 2] * p.z + M[4 * r + 3];
  const float sc = fmaxf(fmaxf(fabsf(c[0]), fabsf(c[1])), fmaxf(fabsf(c[2]), fabsf(c[3])));
  if (!(sc > 0.0f) || sc > 3.402823e38f) return make_float2(2.0f, 2.0f);
  const float w = c[3] / sc;
  if (!(w > 0.0f)) return make_float2(2.0f, 2.0f);
  return make_float2((c[0] / sc) / w, (c[1] / sc) / w);
}

// First hit of the recorded sample (kernel.wgsl.ts:947-958), one thread per
// pixel after the wave's bounce-0 closest-hit trace: the normal facing the
// camera ray, the hit's distance from the ray origin, the base colour and the
// screen motion; misses write the reference's defaults.  Queue slot == path
// id at bounce 0, and the recorded sample's paths are one block of the wave
// (in tile_pixel order); waves that do not hold the sample return at once.
__global__ void k_aux_first_hit(SceneView sc, FrameView f, WaveBuffers w) {
  const uint32_t wh = f.width * f.height;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= wh) return;
  const uint32_t pix = tile_pixel(j, f.width, f.height);
  const uint32_t first = w.counters[kCntWaveSample], want = __float_as_uint(f.aux.consts[32]);
  if (want < first || want - first >= f.spp_wave) return;
  const uint32_t p = (want - first) * wh + j;
  const AuxView& a = f.aux;
  const int4 h = w.hits[p];
  if (h.x < 0) {
    a.normal_depth[pix] = make_float4(0.5f, 1.0f, 0.5f, 0.0f);
    a.albedo[pix] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    a.motion[pix] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    return;
  }
  const float4 r0 = w.rays[0][2 * p], r1 = w.rays[0][2 * p + 1];
  const float3 o = f3(r0.x, r0.y, r0.z), d = f3(r1.x, r1.y, r1.z);
  const float4 nr = __ldg(sc.tris + 4 * (size_t)(uint32_t)h.x + 3);
  float3 ng = f3(nr.x, nr.y, nr.z);
  if (h.z >= 0) {
    const float4* ir = sc.inst_table + 4 * (size_t)h.z;
    const float4 m0 = __ldg(ir), m1 = __ldg(ir + 1), m2 = __ldg(ir + 2);
    ng = normalize(f3(m0.x * ng.x + m1.x * ng.y + m2.x * ng.z, m0.y * ng.x + m1.y * ng.y + m2.y * ng.z,
                      m0.z * ng.x + m1.z * ng.y + m2.z * ng.z));
  }
  const float3 n = dot(d, ng) < 0.0f ? ng : -ng;
  const float3 P = o + d * __int_as_float(h.y);
  const float3 base = sc.materials[hit_material(sc, h)].base_color;
  a.normal_depth[pix] = make_float4(n.x * 0.5f + 0.5f, n.y * 0.5f + 0.5f, n.z * 0.5f + 0.5f, sqrtf(dot(P - o, P - o)));
  a.albedo[pix] = make_float4(base.x, base.y, base.z, 1.0f);
  const float2 c = project_ndc(a.consts, P), q = project_ndc(a.consts + 16, P);
  a.motion[pix] = make_float4((c.x - q.x) * 0.5f * (float)f.width, (c.y - q.y) * 0.5f * (float)f.height, 0.0f, 1.0f);
}

__global__ void __launch_bounds__(128, 8) k_shade(SceneView sc0, FrameView f, WaveBuffers w, int cur, uint32_t bounce) {
  const int nxt = cur ^ 1;
  const uint32_t n = w.counters[cur];
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n;
       base += gridDim.x * blockDim.x) {
    const uint32_t i = base + lane;
    const bool valid = i < n;
    bool alive = false, shadow = false, query = false;
    float4 next_o, next_d, sh_o, sh_d, sh_c;
    float4 qf[4];
    float4 qt;
    uint4 next_state;
    float3 T = f3(0.0f, 0.0f, 0.0f);
    uint32_t root_of_path = 0;
    float spread = 0.0f;  // running sum of spread terms (spread termination)
    if (valid) {
      const uint32_t p = f.sort_by_material ? w.order[i] : i;
      const float4 r0 = w.rays[cur][2 * p], r1 = w.rays[cur][2 * p + 1];
      const uint4 st = w.state[cur][p];
      const uint32_t sid = (st.z >> 8) & 0xFFu;
      const SceneView& sc = f.batch ? f.batch[sid].view : sc0;
      const bool last = bounce + 1 >= (f.batch ? f.batch[sid].max_bounces : f.max_bounces);
      root_of_path = sc.root;
      const float4 tp = w.through[cur][p];
      const int4 h = w.hits[p];
      T = f3(tp.x, tp.y, tp.z);
      const uint32_t path = st.x;
      uint32_t rng = st.y;
      const bool prev_delta = st.z & 1u;
      const float prev_pdf = __uint_as_float(st.w);
      const float3 o = f3(r0.x, r0.y, r0.z), d = f3(r1.x, r1.y, r1.z);
      float3 rad = f3(0.0f, 0.0f, 0.0f);
      if (sc.n_area) {
        // analytic area lights the incoming segment crossed (MIS against their sampling)
        float3 Le;
        float pa;
        if (area_light_hit(sc, o, d, h.x < 0 ? CUDART_INF_F : __int_as_float(h.y), Le, pa)) {
          const float wgt = prev_delta ? 1.0f : power_heuristic(prev_pdf, pa);
          rad = rad + T * Le * wgt;
        }
      }
      if (h.x < 0) {
        // escaped: discs of directional lights it points into (MIS against their cone sampling)
        for (uint32_t k = 0; k < sc.n_dirs; ++k) {
          const float4 dw = __ldg(sc.dirs + 2 * k), dl = __ldg(sc.dirs + 2 * k + 1);
          if (dl.w != 0.0f || dot(d, f3(dw.x, dw.y, dw.z)) < dw.w) continue;
          float wgt = 1.0f;
          if (!prev_delta)
            wgt = power_heuristic(prev_pdf, 1.0f / (2.0f * CUDART_PI_F * (1.0f - dw.w)));
          rad = rad + T * f3(dl.x, dl.y, dl.z) * wgt;
        }
        if (sc.env) {
          int col, row;
          float sin_t;
          env_texel(sc, d, col, row, sin_t);
          float wgt = 1.0f;
          if (!prev_delta && sc.env_marginal)
            wgt = power_heuristic(prev_pdf, env_pdf_texel(sc, col, row, sin_t));
          rad = rad + T * env_radiance(sc, col, row) * wgt;
        }
      } else {
        const float4* rec = sc.tris + 4 * (size_t)(uint32_t)h.x;
        const float4 nr = __ldg(rec + 3);
        const float t = __int_as_float(h.y);
        const Material m = sc.materials[hit_material(sc, h)];
        const float3 P = o + d * t;
        float3 ng = f3(nr.x, nr.y, nr.z);
        if (h.z >= 0) {
          // instance: world normal = (world-to-local)^T * local normal
          const float4* ir = sc.inst_table + 4 * (size_t)h.z;
          const float4 m0 = __ldg(ir), m1 = __ldg(ir + 1), m2 = __ldg(ir + 2);
          ng = normalize(f3(m0.x * ng.x + m1.x * ng.y + m2.x * ng.z, m0.y * ng.x + m1.y * ng.y + m2.y * ng.z,
                            m0.z * ng.x + m1.z * ng.y + m2.z * ng.z));
        }
        const float dn = dot(d, ng);
        const bool front = dn < 0.0f;
        if (m.emissive && front) {
          float wgt = 1.0f;
          if (!prev_delta) wgt = power_heuristic(prev_pdf, area_light_pdf(sc, t, -dn));
          rad = rad + T * m.emission * wgt;
        }
        const float3 n = front ? ng : -ng;  // facing the incoming ray
        const float off = sc.bias * fmaxf(1.0f, fmaxf(fabsf(P.x), fmaxf(fabsf(P.y), fabsf(P.z))));
        const float3 wo = -d;
        float3 tb, bb;
        onb(n, tb, bb);
        const float3 wol = to_local(wo, tb, bb, n);
        if (f.nrc_spread_c > 0.0f) {
          // a0 = t^2 / (4 pi |cos|) at the primary vertex (kept as sqrt in radiance.w); later
          // vertices add sqrt(t^2 / (p |cos|)) of the segment that reached them (delta segments add 0)
          const float ac = fabsf(dn) + 1e-7f;
          spread = tp.w;
          if (bounce == 0) {
            const float a0 = sqrtf(t * t / (4.0f * CUDART_PI_F * ac));
            float4 r = w.radiance[path];
            r.w = a0;
            w.radiance[path] = r;
          } else {
            if (!prev_delta) spread += prev_pdf > 0.0f ? sqrtf(t * t / (prev_pdf * ac)) : 3.0e19f;
            const float a0 = w.radiance[path].w;
            query = spread * spread > f.nrc_spread_c * a0 * a0;
          }
        } else {
          query = bounce == f.nrc_prefix;
        }
        if (query && f.nrc_tile_error) {
          // tiles whose cache error estimate is above the threshold keep path tracing
          const uint32_t pix = tile_pixel(path % (f.width * f.height), f.width, f.height);
          const uint32_t tile = (pix / f.width / f.nrc_tile) * f.nrc_tiles_x + (pix % f.width) / f.nrc_tile;
          if (f.nrc_tile_error[tile] > f.nrc_fallback) query = false;
        }
        if (f.train || query) nrc_features(m, P, wo, n, qf);
        if (f.train) {
          // training record: features, radiance gathered so far (incl. this
          // vertex's emission), throughput on arrival
          float4* rec = w.nrc_records + 6 * ((size_t)path * f.record_bounces + bounce);
          const float4 acc = w.radiance[path];
          rec[0] = qf[0];
          rec[1] = qf[1];
          rec[2] = qf[2];
          rec[3] = qf[3];
          rec[4] = make_float4(acc.x + rad.x, acc.y + rad.y, acc.z + rad.z, 1.0f);
          rec[5] = make_float4(T.x, T.y, T.z, 0.0f);
        }
        if (query) {
          // the path ends in the cache: its scattered radiance is predicted here
          qt = make_float4(__uint_as_float(path), T.x, T.y, T.z);
        } else {
          const float eta = front ? m.ior : 1.0f / m.ior;  // n_t / n_i for light arriving along wo
          const OpaqueSide os = surface_side(m, wol);
          // ---- next-event estimation (surfaces with a finite BSDF lobe)
          if (sc.n_light_entries > 0 && has_finite_support(m)) {
            const LightSample ls =
                sample_light(sc, P, (m.kind == kDielectric && m.transmission > 0.0f) ? f3(0.0f, 0.0f, 0.0f) : n, rng);
            if (ls.valid) {
              float3 fc;
              float pb;
              const float3 wil = to_local(ls.wi, tb, bb, n);
              bsdf_eval(m, os, eta, wol, wil, fc, pb);
              if (maxc(fc) > 0.0f) {
                const float wgt = (ls.delta || last) ? 1.0f : power_heuristic(ls.pdf_light, pb);
                const float3 c = T * fc * ls.Le * (wgt / ls.pdf);
                if (maxc(c) > 0.0f) {
                  const float3 so = P + n * (wil.z > 0.0f ? off : -off);
                  const float tmax = isinf(ls.dist) ? CUDART_INF_F : ls.dist * (1.0f - 1e-4f);
                  sh_o = make_float4(so.x, so.y, so.z, 0.0f);
                  sh_d = make_float4(ls.wi.x, ls.wi.y, ls.wi.z, tmax);
                  sh_c = make_float4(c.x, c.y, c.z, __uint_as_float(path));
                  shadow = true;
                }
              }
            }
          }
          // ---- BSDF sample
          if (!last) {
            const BsdfSample bs = sample_bsdf(m, os, eta, wol, rng);
            if (bs.valid) {
              const float3 wi = to_world(bs.wi, tb, bb, n);
              T = T * bs.weight;
              alive = true;
              const float3 no = P + n * (bs.wi.z > 0.0f ? off : -off);
              next_o = make_float4(no.x, no.y, no.z, 0.0f);
              next_d = make_float4(wi.x, wi.y, wi.z, CUDART_INF_F);
              next_state = make_uint4(path, 0u, bs.delta ? 1u : 0u, __float_as_uint(bs.pdf));
            }
          }
        }
        // ---- Russian roulette
        if (alive && bounce > 2) {
          const float q = represented_bernoulli(fminf(fmaxf(maxc(T), 0.1f), 0.95f));
          if (!(rand01(rng) < q)) alive = false;
          else T = T * (1.0f / q);
        }
      }
      next_state.y = rng;
      next_state.z |= sid << 8;
      if (maxc(rad) > 0.0f) {
        float4 acc = w.radiance[path];
        w.radiance[path] = make_float4(acc.x + rad.x, acc.y + rad.y, acc.z + rad.z, acc.w);
      }
    }
    // ---- warp-ballot compaction of survivors and shadow rays
    const uint32_t am = __ballot_sync(kFull, alive);
    if (am) {
      uint32_t b = 0;
      if (lane == (uint32_t)(__ffs(am) - 1)) b = atomicAdd(&w.counters[nxt], (uint32_t)__popc(am));
      b = __shfl_sync(kFull, b, __ffs(am) - 1);
      if (alive) {
        const uint32_t q = b + __popc(am & ((1u << lane) - 1u));
        w.rays[nxt][2 * q] = next_o;
        w.rays[nxt][2 * q + 1] = next_d;
        w.state[nxt][q] = next_state;
        w.through[nxt][q] = make_float4(T.x, T.y, T.z, spread);
        if (w.ray_root[nxt]) w.ray_root[nxt][q] = root_of_path;
      }
    }
    const uint32_t sm = __ballot_sync(kFull, shadow);
    if (sm) {
      uint32_t b = 0;
      if (lane == (uint32_t)(__ffs(sm) - 1)) b = atomicAdd(&w.counters[kCntShadow], (uint32_t)__popc(sm));
      b = __shfl_sync(kFull, b, __ffs(sm) - 1);
      if (shadow) {
        const uint32_t q = b + __popc(sm & ((1u << lane) - 1u));
        w.shadow_rays[2 * q] = sh_o;
        w.shadow_rays[2 * q + 1] = sh_d;
        w.shadow_contrib[q] = sh_c;
        if (w.shadow_root) w.shadow_root[q] = root_of_path;
      }
    }
    const uint32_t qm = __ballot_sync(kFull, query);
    if (qm) {
      uint32_t b = 0;
      if (lane == (uint32_t)(__ffs(qm) - 1)) b = atomicAdd(&w.counters[kCntQuery], (uint32_t)__popc(qm));
      b = __shfl_sync(kFull, b, __ffs(qm) - 1);
      if (query) {
        float4* o = w.nrc_queries + 5 * (size_t)(b + __popc(qm & ((1u << lane) - 1u)));
        o[0] = qf[0];
        o[1] = qf[1];
        o[2] = qf[2];
        o[3] = qf[3];
        o[4] = qt;
      }
    }
  }
}

__global__ void k_shadow_resolve(WaveBuffers w) {
  const uint32_t n = w.counters[kCntShadow];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (w.occluded[i]) continue;
    const float4 c = w.shadow_contrib[i];
    const uint32_t path = __float_as_uint(c.w);
    float4 acc = w.radiance[path];
    w.radiance[path] = make_float4(acc.x + c.x, acc.y + c.y, acc.z + c.z, acc.w);
  }
}

__global__ void k_accumulate(FrameView f, WaveBuffers w, AccumView a) {
  const uint32_t wh = f.width * f.height;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;  // path slot within a sample plane
  if (j >= wh) return;
  const uint32_t pix = tile_pixel(j, f.width, f.height);
  float3 s = f3(0.0f, 0.0f, 0.0f);
  float l1 = 0.0f, l2 = 0.0f;  // luminance moments (varianceMomentsBuffer, kernel.wgsl.ts:936-940)
  double s64[3] = {0, 0, 0}, q64[3] = {0, 0, 0}, m64[4] = {0, 0, 0, 0};
  for (uint32_t k = 0; k < f.spp_wave; ++k) {
    const float4 r = w.radiance[(size_t)k * wh + j];
    s = s + f3(r.x, r.y, r.z);
    const float lum = 0.2126f * r.x + 0.7152f * r.y + 0.0722f * r.z;
    l1 += lum;
    l2 += lum * lum;
    if (a.sum64) {
      const double v[3] = {r.x, r.y, r.z};
      for (int c = 0; c < 3; ++c) { s64[c] += v[c]; q64[c] += v[c] * v[c]; }
    }
    if (a.lum64) {
      const double L = 0.2126 * r.x + 0.7152 * r.y + 0.0722 * r.z, L2 = L * L;
      m64[0] += L;
      m64[1] += L2;
      m64[2] += L2 * L;
      m64[3] += L2 * L2;
    }
  }
  float4 acc = a.accum[pix];
  a.accum[pix] = make_float4(acc.x + s.x, acc.y + s.y, acc.z + s.z, acc.w + (float)f.spp_wave);
  if (f.aux.moments) {
    const float4 mo = f.aux.moments[pix];
    f.aux.moments[pix] = make_float4(mo.x + l1, mo.y + l2, mo.z + (float)f.spp_wave, 0.0f);
  }
  if (a.sum64) {
    for (int c = 0; c < 3; ++c) {
      a.sum64[3 * (size_t)pix + c] += s64[c];
      a.sq64[3 * (size_t)pix + c] += q64[c];
    }
  }
  if (a.lum64)
    for (int k = 0; k < 4; ++k) a.lum64[4 * (size_t)pix + k] += m64[k];
}

// next wave's samples start after this wave's (read by k_raygen)
__global__ void k_advance_wave(FrameView f, WaveBuffers w) { w.counters[kCntWaveSample] += f.spp_wave; }

__global__ void k_count_rays(WaveBuffers w, int cur, unsigned long long* totals) {
  totals[0] += w.counters[cur];
  totals[1] += w.counters[kCntShadow];
}

__global__ void k_nrc_targets(WaveBuffers w, uint32_t paths, uint32_t bounces, float4* samples, uint32_t capacity,
                              uint32_t query_bounce) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t total = paths * bounces;
  if (blockIdx.x == 0 && threadIdx.x == 0) *w.nrc_seed += 1u;  // next training wave draws new paths
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < total;
       base += gridDim.x * blockDim.x) {
    const uint32_t sl = base + lane;
    bool keep = false;
    float4 tg = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (sl < total) {
      const float4* rec = w.nrc_records + 6 * (size_t)sl;
      const float4 A = rec[4];
      if (A.w != 0.0f) {
        const float4 T = rec[5];
        const float4 L = w.radiance[sl / bounces];
        auto tgt = [](float l, float a, float t) {
          const float v = t > 0.0f ? (l - a) / t : 0.0f;
          return fminf(1024.0f, fmaxf(0.0f, v));
        };
        tg = make_float4(tgt(L.x, A.x, T.x), tgt(L.y, A.y, T.y), tgt(L.z, A.z, T.z), 0.0f);
        if (w.path_pixel && sl % bounces == query_bounce) tg.w = __uint_as_float(w.path_pixel[sl / bounces] + 1u);
        keep = isfinite(tg.x) && isfinite(tg.y) && isfinite(tg.z);
      }
    }
    const uint32_t km = __ballot_sync(kFull, keep);
    if (!km) continue;
    uint32_t b = 0;
    if (lane == (uint32_t)(__ffs(km) - 1)) b = atomicAdd(&w.counters[kCntSamples], (uint32_t)__popc(km));
    b = __shfl_sync(kFull, b, __ffs(km) - 1);
    if (keep) {
      const uint32_t q = b + __popc(km & ((1u << lane) - 1u));
      if (q < capacity) {
        const float4* rec = w.nrc_records + 6 * (size_t)sl;
        float4* o = samples + 5 * (size_t)q;
        o[0] = rec[0];
        o[1] = rec[1];
        o[2] = rec[2];
        o[3] = rec[3];
        o[4] = tg;
      }
    }
  }
}

__global__ void k_nrc_fill(WaveBuffers w, float4* samples, uint32_t capacity) {
  const uint32_t got = min(w.counters[kCntSamples], capacity);
  for (uint32_t i = got + blockIdx.x * blockDim.x + threadIdx.x; i < capacity; i += gridDim.x * blockDim.x) {
    float4* o = samples + 5 * (size_t)i;
    if (got == 0) {
      for (int k = 0; k < 5; ++k) o[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else {
      const float4* src = samples + 5 * (size_t)(i % got);
      for (int k = 0; k < 5; ++k) o[k] = src[k];
    }
  }
}

// ---------------------------------------------------------------- batch
// Paths of the whole batch form one index space: scene s owns
// [path_begin_s, path_begin_s + W_s H_s spp_s), pixel-major within a sample.
// Each wave takes the next `capacity` paths at the device cursor.
__global__ void k_raygen_batch(FrameView f, WaveBuffers w, uint32_t capacity) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long base = *w.batch_cursor;
  const unsigned long long left = base < f.batch_paths ? f.batch_paths - base : 0ull;
  const uint32_t cnt = left < capacity ? (uint32_t)left : capacity;
  if (i == 0) {
    w.counters[0] = cnt;
    w.counters[kCntBatchPaths] = cnt;
  }
  if (i >= cnt) return;
  const unsigned long long g = base + i;
  uint32_t lo = 0, hi = f.n_scenes - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (f.batch[mid].path_begin <= g) lo = mid; else hi = mid - 1;
  }
  const BatchScene& B = f.batch[lo];
  const unsigned long long local = g - B.path_begin;
  const uint32_t wh = B.width * B.height;
  const uint32_t pix = tile_pixel((uint32_t)(local % wh), B.width, B.height), sample = (uint32_t)(local / wh);
  const uint32_t x = pix % B.width, y = pix / B.width;
  uint32_t rng = pcg_init(x, y, B.frame_seed ^ sample);
  const float jx = rand01(rng), jy = rand01(rng);
  const float u = ((float)x + jx) / (float)B.width, v = ((float)y + jy) / (float)B.height;
  const float nx = u * 2.0f - 1.0f, ny = 1.0f - v * 2.0f;
  const float* M = B.inv_vp;
  float nf[4], fr[4];
  for (int r = 0; r < 4; ++r) {
    nf[r] = M[4 * r] * nx + M[4 * r + 1] * ny - M[4 * r + 2] + M[4 * r + 3];
    fr[r] = M[4 * r] * nx + M[4 * r + 1] * ny + M[4 * r + 2] + M[4 * r + 3];
  }
  const float3 o = f3(nf[0] / nf[3], nf[1] / nf[3], nf[2] / nf[3]);
  const float3 far = f3(fr[0] / fr[3], fr[1] / fr[3], fr[2] / fr[3]);
  const float3 d = normalize(far - o);
  w.rays[0][2 * i] = make_float4(o.x, o.y, o.z, 0.0f);
  w.rays[0][2 * i + 1] = make_float4(d.x, d.y, d.z, CUDART_INF_F);
  w.state[0][i] = make_uint4(i, rng, 1u | (lo << 8), 0u);
  w.through[0][i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
  w.radiance[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  w.ray_root[0][i] = B.view.root;
  w.path_pixel[i] = B.accum_offset + pix;
}

__global__ void k_accumulate_batch(WaveBuffers w, float4* accum) {
  const uint32_t cnt = w.counters[kCntBatchPaths];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const float4 r = w.radiance[i];
    float* a = reinterpret_cast<float*>(accum + w.path_pixel[i]);
    atomicAdd(a, r.x);
    atomicAdd(a + 1, r.y);
    atomicAdd(a + 2, r.z);
    atomicAdd(a + 3, 1.0f);
  }
}

__global__ void k_advance_batch(WaveBuffers w) { *w.batch_cursor += w.counters[kCntBatchPaths]; }

__global__ void k_nrc_tile_update(float* stats, float* err, uint32_t tiles, float alpha) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < tiles; t += gridDim.x * blockDim.x) {
    float* s = stats + 3 * (size_t)t;
    if (s[2] > 0.0f) {
      const float e = fabsf(s[0] - s[1]) / (s[1] + 1e-3f * s[2]);
      err[t] = isfinite(e) ? (1.0f - alpha) * err[t] + alpha * e : err[t];
    }
    s[0] = s[1] = s[2] = 0.0f;
  }
}

unsigned grid_for(uint32_t n, unsigned block) {
  unsigned g = (unsigned)((n + block - 1) / block);
  return g ? g : 1;
}

}  // namespace

// ---------------------------------------------------------------- present
// Tonemap operators of shared-samplers/src/wgsl/tonemap.wgsl.ts:8-60, restated:
// exposure scales each channel (NaN and non-positive exposure give 0, results
// stay finite); ACES filmic is Narkowicz's fit x(2.51x + 0.03) / (x(2.43x + 0.59)
// + 0.14) clamped to [0, 1]; AgX maps log2 exposure over [-12.47393, 4.026069]
// to [0, 1] and applies its sixth-order polynomial; Reinhard is x / (1 + x).
__device__ __forceinline__ float exposed(float c, float exposure) {
  if (c != c || !(exposure > 0.0f)) return 0.0f;
  const float m = fminf(fabsf(c) * fminf(exposure, 3.402823466e38f), 3.402823466e38f);
  return c < 0.0f ? -m : m;
}
__device__ __forceinline__ float tonemap_aces(float x) {
  const float v = fminf(fmaxf(x, 0.0f), 1e18f);  // the curve is 1 (clamped) long before v^2 overflows
  return clamp01(v * (2.51f * v + 0.03f) / (v * (2.43f * v + 0.59f) + 0.14f));
}
__device__ __forceinline__ float tonemap_agx(float c) {
  const float x = clamp01((log2f(fmaxf(c, 1e-6f)) + 12.47393f) / (12.47393f + 4.026069f));
  const float x2 = x * x, x4 = x2 * x2;
  return clamp01(15.5f * x4 * x2 - 40.14f * x4 * x + 31.96f * x4 - 6.868f * x2 * x + 0.4298f * x2 + 0.1191f * x -
                 0.00232f);
}
__device__ __forceinline__ float tonemap(float c, int mode, float exposure) {
  const float x = exposed(c, exposure);
  switch (mode) {
    case 1: return tonemap_agx(x);
    case 2: { const float v = fmaxf(x, 0.0f); return v / (1.0f + v); }
    case 3: return clamp01(x);
    case 4: return x;
    default: return tonemap_aces(x);
  }
}
// IEC 61966-2-1 sRGB encoding
__device__ __forceinline__ float srgb_oetf(float c) {
  const float v = fmaxf(c, 0.0f);
  return v <= 0.0031308f ? v * 12.92f : 1.055f * powf(v, 1.0f / 2.4f) - 0.055f;
}
__global__ void k_present(const float4* __restrict__ accum, size_t pixels, int mode, float exposure, int srgb,
                          float4* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pixels) return;
  const float4 a = accum[i];
  const float inv = a.w > 0.0f ? 1.0f / a.w : 0.0f;
  float r = tonemap(fmaxf(a.x * inv, 0.0f), mode, exposure);
  float g = tonemap(fmaxf(a.y * inv, 0.0f), mode, exposure);
  float b = tonemap(fmaxf(a.z * inv, 0.0f), mode, exposure);
  if (srgb) {
    r = srgb_oetf(r);
    g = srgb_oetf(g);
    b = srgb_oetf(b);
  }
  out[i] = make_float4(r, g, b, 1.0f);
}

// Mean radiance per pixel (captureFrame 'linear'): sum / count with the
// correctly rounded reciprocal and product, alpha 1 (0 where nothing landed).
__global__ void k_capture_mean(const float4* __restrict__ accum, size_t pixels, float4* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pixels) return;
  const float4 a = accum[i];
  const float inv = a.w > 0.0f ? __frcp_rn(a.w) : 0.0f;
  out[i] = make_float4(__fmul_rn(a.x, inv), __fmul_rn(a.y, inv), __fmul_rn(a.z, inv), 1.0f);
}

void launch_capture_mean(const float4* accum, size_t pixels, float4* out, cudaStream_t s) {
  if (pixels == 0) return;
  k_capture_mean<<<(unsigned)((pixels + 255) / 256), 256, 0, s>>>(accum, pixels, out);
}

void launch_present(const float4* accum, size_t pixels, int tonemap, float exposure, int srgb, float4* out,
                    cudaStream_t s) {
  if (pixels == 0) return;
  k_present<<<(unsigned)((pixels + 255) / 256), 256, 0, s>>>(accum, pixels, tonemap, exposure, srgb, out);
}

void launch_count_rays(const WaveBuffers& w, int cur, unsigned long long* totals, cudaStream_t s) {
  k_count_rays<<<1, 1, 0, s>>>(w, cur, totals);
}

void launch_raygen(const FrameView& f, const WaveBuffers& w, cudaStream_t s) {
  k_raygen<<<grid_for(f.paths, 256), 256, 0, s>>>(f, w);
}

void launch_sort_by_material(const SceneView& sc, const FrameView& f, const WaveBuffers& w, int cur,
                             uint32_t capacity, cudaStream_t s) {
  const unsigned g = grid_for(capacity, 256) < kSortGrid ? grid_for(capacity, 256) : kSortGrid;
  k_sort_keys<4, 0><<<g, 256, 0, s>>>(sc, f, w, cur);
  k_sort_offsets<4><<<1, 1024, 0, s>>>(w, g);
  k_sort_scatter<4><<<g, 256, 0, s>>>(w, cur);
}

void launch_sort_rays(const WaveBuffers& w, int cur, uint32_t capacity, cudaStream_t s) {
  const unsigned g = grid_for(capacity, 256) < kSortGrid ? grid_for(capacity, 256) : kSortGrid;
  k_sort_keys<8, 1><<<g, 256, 0, s>>>(SceneView{}, FrameView{}, w, cur);
  k_sort_offsets<8><<<1, 1024, 0, s>>>(w, g);
  k_sort_scatter<8><<<g, 256, 0, s>>>(w, cur);
}

void launch_shade(const SceneView& sc, const FrameView& f, const WaveBuffers& w, int cur, uint32_t bounce,
                  uint32_t capacity, cudaStream_t s) {
  cudaMemsetAsync(w.counters + (cur ^ 1), 0, sizeof(uint32_t), s);
  cudaMemsetAsync(w.counters + kCntShadow, 0, sizeof(uint32_t), s);
  const unsigned g = grid_for(capacity, 128) < 148 * 16 ? grid_for(capacity, 128) : 148 * 16;
  k_shade<<<g, 128, 0, s>>>(sc, f, w, cur, bounce);
}

void launch_shadow_resolve(const WaveBuffers& w, uint32_t capacity, cudaStream_t s) {
  const unsigned g = grid_for(capacity, 256) < 148 * 8 ? grid_for(capacity, 256) : 148 * 8;
  k_shadow_resolve<<<g, 256, 0, s>>>(w);
}

void launch_nrc_targets(const WaveBuffers& w, uint32_t paths, uint32_t bounces, float4* samples, uint32_t capacity,
                        uint32_t query_bounce, cudaStream_t s) {
  const uint32_t total = paths * bounces;
  const unsigned g = grid_for(total, 256) < 148 * 8 ? grid_for(total, 256) : 148 * 8;
  k_nrc_targets<<<g, 256, 0, s>>>(w, paths, bounces, samples, capacity, query_bounce);
  const unsigned gf = grid_for(capacity, 256) < 148 * 8 ? grid_for(capacity, 256) : 148 * 8;
  k_nrc_fill<<<gf, 256, 0, s>>>(w, samples, capacity);
}

void launch_raygen_batch(const FrameView& f, const WaveBuffers& w, uint32_t capacity, cudaStream_t s) {
  k_raygen_batch<<<grid_for(capacity, 256), 256, 0, s>>>(f, w, capacity);
}

void launch_accumulate_batch(const WaveBuffers& w, float4* accum, uint32_t capacity, cudaStream_t s) {
  const unsigned g = grid_for(capacity, 256) < 148 * 8 ? grid_for(capacity, 256) : 148 * 8;
  k_accumulate_batch<<<g, 256, 0, s>>>(w, accum);
  k_advance_batch<<<1, 1, 0, s>>>(w);
}

void launch_nrc_tile_update(float* tile_stats, float* tile_error, uint32_t tiles, float alpha, cudaStream_t s) {
  k_nrc_tile_update<<<grid_for(tiles, 256), 256, 0, s>>>(tile_stats, tile_error, tiles, alpha);
}

void launch_aux_first_hit(const SceneView& sc, const FrameView& f, const WaveBuffers& w, cudaStream_t s) {
  if (!f.aux.normal_depth) return;
  k_aux_first_hit<<<grid_for(f.width * f.height, 256), 256, 0, s>>>(sc, f, w);
}

void launch_accumulate(const FrameView& f, const WaveBuffers& w, const AccumView& a, cudaStream_t s) {
  k_accumulate<<<grid_for(f.width * f.height, 256), 256, 0, s>>>(f, w, a);
  k_advance_wave<<<1, 1, 0, s>>>(f, w);
}

}  // namespace pt
}  // namespace vt

extern "C" vt_status vt_light_tree_select_device(const float* d_tree, size_t node_count, uint32_t n_distant,
                                                 const float* d_points, const float* d_normals,
                                                 const uint32_t* d_buckets, size_t n, uint32_t* d_emitter,
                                                 float* d_pmf, void* cuda_stream) {
  return vt::guard([&] {
    if (n && (!d_points || !d_buckets || !d_emitter || !d_pmf)) vt::fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (node_count && !d_tree) vt::fail(VT_ERR_INVALID_ARGUMENT, "tree is null");
    if (node_count == 0 && n_distant == 0) vt::fail(VT_ERR_INVALID_ARGUMENT, "no entries");
    if (!n) return;
    // the positional entries are the tree's leaves ((node_count + 1) / 2); one without a tree
    const uint32_t n_pos = node_count ? (uint32_t)((node_count + 1) / 2) : 0u;
    vt::pt::k_light_tree_select<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)cuda_stream>>>(
        node_count > 1 ? d_tree : nullptr, n_pos, n_distant, d_points, d_normals, d_buckets, n, d_emitter, d_pmf);
    VT_CUDA(cudaGetLastError());
  });
}
