// pt_common.cuh -- device math, random numbers and BSDFs of the path tracer.
//
// Estimator pieces restated from the reference integrator
// (packages/pt-webgpu/src/wgsl/pathTrace/*, CPU mirror
// packages/pt-webgpu/src/__tests__/cpuTracer.ts):
//   PCG32 pcgInit / pcgNext / rand_f32    shared-samplers/src/wgsl/pcg.wgsl.ts:5-24
//   represented_bernoulli_probability     pcg.wgsl.ts (2^24-bucket rounding)
//   frame key frameSeed ^ frameIndex      pt-webgpu/src/wgsl/common.wgsl.ts:194-196
//   Russian roulette clamp(max T, .1, .95) kernelCore.wgsl.ts:54-67
//   cosine hemisphere + ONB                bsdf.wgsl.ts:1632-1663 (cpuTracer.ts:236-272)
//   GGX VNDF (Heitz 2018)                  bsdf.wgsl.ts:1710-1737 (cpuTracer.ts:280-306)
//   frDielectric                           material.wgsl.ts:2780 (cpuTracer.ts:313-324)
//   Schlick Fresnel                        material.wgsl.ts:2766
//   power heuristic (beta = 2)             material.wgsl.ts:2808-2822 (cpuTracer.ts:343-354)
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

namespace vt {
namespace pt {

// ------------------------------------------------------------------ float3 helpers
__host__ __device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float maxc(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
__device__ __forceinline__ float3 normalize(float3 a) {
  const float l2 = dot(a, a);
  return l2 > 1e-30f ? a * rsqrtf(l2) : f3(0.0f, 0.0f, 1.0f);
}

// ------------------------------------------------------------------ PCG32
__host__ __device__ __forceinline__ uint32_t pcg_init(uint32_t px, uint32_t py, uint32_t key) {
  uint32_t s = px * 1664525u + py * 1013904223u + key * 22695477u;
  s ^= s >> 17;
  s ^= s << 31;
  s ^= s >> 11;
  return s;
}
__host__ __device__ __forceinline__ uint32_t pcg_next(uint32_t& s) {
  s = s * 747796405u + 2891336453u;
  uint32_t w = ((s >> ((s >> 28) + 4u)) ^ s) * 277803737u;
  return (w >> 22) ^ w;
}
// 24-bit uniform in [0, 1)
__host__ __device__ __forceinline__ float rand01(uint32_t& s) { return (float)(pcg_next(s) >> 8) * (1.0f / 16777216.0f); }
// Probability realised by `rand01(s) < p` (rounded to a 2^-24 bucket, endpoints exact).
__host__ __device__ __forceinline__ float represented_bernoulli(float p) {
  if (!(p > 0.0f)) return 0.0f;
  if (p >= 1.0f) return 1.0f;
  float b = floorf(p * 16777216.0f + 0.5f);
  b = fminf(fmaxf(b, 1.0f), 16777215.0f);
  return b * (1.0f / 16777216.0f);
}

// ------------------------------------------------------------------ frames
__device__ __forceinline__ void onb(float3 n, float3& t, float3& b) {
  const float l2 = n.x * n.x + n.y * n.y;
  if (l2 > 1e-10f) {
    const float inv = rsqrtf(l2);
    t = f3(-n.y * inv, n.x * inv, 0.0f);
  } else {
    t = f3(1.0f, 0.0f, 0.0f);
  }
  b = cross(n, t);
}
__device__ __forceinline__ float3 to_world(float3 v, float3 t, float3 b, float3 n) { return t * v.x + b * v.y + n * v.z; }
__device__ __forceinline__ float3 to_local(float3 v, float3 t, float3 b, float3 n) {
  return f3(dot(v, t), dot(v, b), dot(v, n));
}

// ------------------------------------------------------------------ MIS
__device__ __forceinline__ float power_heuristic(float a, float b) {
  if (!(a >= 0.0f) || !(b >= 0.0f) || a > 3.402823466e38f || b > 3.402823466e38f) return 0.0f;
  const float m = fmaxf(a, b);
  if (!(m > 0.0f)) return 0.0f;
  const float x = a / m, y = b / m;
  return (x * x) / (x * x + y * y);
}

// ------------------------------------------------------------------ materials
enum MaterialKind : uint32_t { kLambert = 0, kConductor = 1, kDielectric = 2 };

struct Material {
  float3 base_color;
  float roughness;
  float3 emission;   // radiance emitted from the front face
  float ior;
  uint32_t kind;
  float alpha;       // GGX alpha = max(roughness^2, 1e-3)
  uint32_t emissive; // emission > 0
  uint32_t flags;    // VT_MATERIAL_* bits
};

__device__ __forceinline__ float3 schlick(float3 f0, float c) {
  const float m = fminf(fmaxf(1.0f - c, 0.0f), 1.0f);
  const float m2 = m * m, m5 = m2 * m2 * m;
  return f0 + (f3(1.0f, 1.0f, 1.0f) - f0) * m5;
}

__device__ __forceinline__ float fr_dielectric(float cos_i, float eta) {
  float ct = fminf(fmaxf(cos_i, -1.0f), 1.0f);
  float e = eta;
  if (ct < 0.0f) { e = 1.0f / e; ct = -ct; }
  const float sin2i = fmaxf(0.0f, 1.0f - ct * ct);
  const float sin2t = sin2i / (e * e);
  if (sin2t >= 1.0f) return 1.0f;
  const float cost = sqrtf(fmaxf(0.0f, 1.0f - sin2t));
  const float rpar = (e * ct - cost) / (e * ct + cost);
  const float rperp = (ct - e * cost) / (ct + e * cost);
  return 0.5f * (rpar * rpar + rperp * rperp);
}

// GGX distribution and Smith G1 in the local frame (n = +z)
__device__ __forceinline__ float ggx_d(float nh, float a) {
  const float a2 = a * a;
  const float d = nh * nh * (a2 - 1.0f) + 1.0f;
  return a2 / (CUDART_PI_F * d * d);
}
__device__ __forceinline__ float ggx_g1(float nv, float a) {
  const float a2 = a * a;
  return 2.0f * nv / (nv + sqrtf(a2 + (1.0f - a2) * nv * nv));
}
// Heitz 2018 visible-normal sample, wo and result in the local frame
__device__ __forceinline__ float3 ggx_vndf(float3 wo, float a, float u1, float u2) {
  const float3 vh = normalize(f3(a * wo.x, a * wo.y, wo.z));
  float3 t1, t2;
  onb(vh, t1, t2);
  const float r = sqrtf(u1);
  const float phi = 2.0f * CUDART_PI_F * u2;
  const float p1 = r * cosf(phi);
  float p2 = r * sinf(phi);
  const float s = 0.5f * (1.0f + vh.z);
  p2 = (1.0f - s) * sqrtf(fmaxf(0.0f, 1.0f - p1 * p1)) + s * p2;
  const float z = sqrtf(fmaxf(0.0f, 1.0f - p1 * p1 - p2 * p2));
  const float3 nh = t1 * p1 + t2 * p2 + vh * z;
  return normalize(f3(a * nh.x, a * nh.y, fmaxf(1e-6f, nh.z)));
}

// BSDF value * |cos(wi)| and solid-angle pdf for non-delta families.
// wo, wi in the local frame with the shading normal at +z (wo.z > 0).
__device__ __forceinline__ void bsdf_eval(const Material& m, float3 wo, float3 wi, float3& f_cos, float& pdf) {
  f_cos = f3(0.0f, 0.0f, 0.0f);
  pdf = 0.0f;
  if (wi.z <= 0.0f || wo.z <= 0.0f) return;
  if (m.kind == kLambert) {
    f_cos = m.base_color * (wi.z / CUDART_PI_F);
    pdf = wi.z / CUDART_PI_F;
  } else if (m.kind == kConductor) {
    const float3 h = normalize(wo + wi);
    const float d = ggx_d(h.z, m.alpha);
    const float g1o = ggx_g1(wo.z, m.alpha), g1i = ggx_g1(wi.z, m.alpha);
    const float3 F = schlick(m.base_color, fmaxf(0.0f, dot(wo, h)));
    f_cos = F * (d * g1o * g1i / (4.0f * wo.z));
    pdf = d * g1o / (4.0f * wo.z);
  }
}

}  // namespace pt
}  // namespace vt
