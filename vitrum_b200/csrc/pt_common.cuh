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
//   BSDF families                          see the materials section below
//   power heuristic (beta = 2)             material.wgsl.ts:2808-2822 (cpuTracer.ts:343-354)
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "ggx_albedo_lut.h"

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
// The reference's base BSDF restricted to the parameters the scene ABI carries
// (base colour, roughness, metallic, transmission, IOR, specular factor; no
// clearcoat / sheen / iridescence / anisotropy / thin film):
//   opaque    transmission 0 or metallic > 0: Lambert diffuse under a GGX
//             specular layer, F0 = mix(specular * ((ior-1)/(ior+1))^2, base,
//             metallic), Kulla-Conty multiple scattering
//             (evaluateBrdfFullWithClearcoatNormal, bsdf.wgsl.ts:809-916);
//             sampling picks GGX visible normals with probability
//             clamp(mix(.04, .96, max(lum F(N.V), metallic)), .04, .96), else
//             the cosine lobe, and weights by the full BSDF over the marginal
//             density (bsdf.wgsl.ts:2919-2998, 1863-1924, 1172-1211, 1555-1630)
//   dielectric transmission > 0 and metallic 0: a Schlick-Fresnel interface
//             (materialDielectricFresnel, bsdf.wgsl.ts:227-256, exact TIR)
//             that reflects, transmits (tinted by base * transmission) or, with
//             weight 1 - transmission, scatters diffusely; delta at roughness
//             0, else the Walter 2007 rough model on sampled visible normals
//             (bsdf.wgsl.ts:941-1033, 1099-1170, 1996-2160, 2618-2918)
// The kinds are sort buckets: opaque with metallic 0 / > 0, dielectric.
enum MaterialKind : uint32_t { kOpaque = 0, kMetal = 1, kDielectric = 2 };

struct Material {
  float3 base_color;
  float roughness;
  float3 emission;   // radiance emitted from the front face
  float ior;         // of the material side (the other side is 1)
  uint32_t kind;
  float alpha;       // GGX alpha = max(roughness^2, 1e-3)
  uint32_t emissive; // emission > 0
  uint32_t flags;    // VT_MATERIAL_* bits
  float metallic;
  float transmission;  // clamped to [0, 1]
  float specular;      // KHR_materials_specular factor: dielectric F0 scale and F90
  float f0_ior;        // specular * ((ior - 1) / (ior + 1))^2
};

__host__ __device__ __forceinline__ float clamp01(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
__host__ __device__ __forceinline__ float3 clamp01(float3 v) { return f3(clamp01(v.x), clamp01(v.y), clamp01(v.z)); }
// BT.709 luminance (shared-samplers/src/wgsl/luminance.wgsl.ts:28-30)
__host__ __device__ __forceinline__ float luminance(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
__device__ __forceinline__ float pow5(float x) {
  const float x2 = x * x;
  return x2 * x2 * x;
}

// global memory read through L1 (lanes index the tables divergently, which the
// constant cache would serialise)
static __device__ const float kGgxE[VT_GGX_ALBEDO_DIM * VT_GGX_ALBEDO_DIM] = {VT_GGX_E_VALUES};
static __device__ const float kGgxEavg[VT_GGX_ALBEDO_DIM] = {VT_GGX_EAVG_VALUES};

// Bilinear E_ss(mu, roughness), clamped to [0.02, 1] (ggxDirectionalAlbedo, material.wgsl.ts:2873-2891)
__device__ __forceinline__ float ggx_albedo(float mu, float r) {
  constexpr int kD = VT_GGX_ALBEDO_DIM;
  const float fr = clamp01(r) * (float)(kD - 1), fm = clamp01(mu) * (float)(kD - 1);
  const int r0 = (int)floorf(fr), m0 = (int)floorf(fm);
  const int r1 = min(r0 + 1, kD - 1), m1 = min(m0 + 1, kD - 1);
  const float tr = fr - (float)r0, tm = fm - (float)m0;
  const float e00 = __ldg(kGgxE + r0 * kD + m0), e01 = __ldg(kGgxE + r0 * kD + m1);
  const float e10 = __ldg(kGgxE + r1 * kD + m0), e11 = __ldg(kGgxE + r1 * kD + m1);
  const float e0 = e00 + (e01 - e00) * tm;
  const float e1 = e10 + (e11 - e10) * tm;
  return fminf(fmaxf(e0 + (e1 - e0) * tr, 0.02f), 1.0f);
}
// Linear E_avg(roughness), clamped to [0.3, 1] (ggxAverageAlbedo, material.wgsl.ts:2894-2901)
__device__ __forceinline__ float ggx_albedo_avg(float r) {
  constexpr int kD = VT_GGX_ALBEDO_DIM;
  const float fr = clamp01(r) * (float)(kD - 1);
  const int r0 = (int)floorf(fr), r1 = min(r0 + 1, kD - 1);
  const float tr = fr - (float)r0;
  const float a0 = __ldg(kGgxEavg + r0), a1 = __ldg(kGgxEavg + r1);
  return fminf(fmaxf(a0 + (a1 - a0) * tr, 0.3f), 1.0f);
}
// Kulla-Conty multiple-scattering BRDF (no cosine), f0 tinting the extra
// bounces through F_avg = f0 + (1 - f0) / 21 (material.wgsl.ts:2903-2931):
//   f_ms = F_avg^2 E_avg / (1 - F_avg (1 - E_avg)) * (1 - E(mu_o)) (1 - E(mu_i)) / (pi (1 - E_avg)).
// Everything but the (1 - E(mu_i)) factor depends on the outgoing side only.
__device__ __forceinline__ float3 ggx_multiscatter_o(float3 f0, float r, float nv) {
  const float eavg = ggx_albedo_avg(r);
  const float miss = 1.0f - eavg;
  if (miss < 1e-4f) return f3(0.0f, 0.0f, 0.0f);
  const float eo = ggx_albedo(nv, r);
  const float3 favg = f0 + (f3(1.0f, 1.0f, 1.0f) - f0) * (1.0f / 21.0f);
  const float3 den = f3(fmaxf(1.0f - favg.x * miss, 1e-4f), fmaxf(1.0f - favg.y * miss, 1e-4f),
                        fmaxf(1.0f - favg.z * miss, 1e-4f));
  const float3 fms = favg * favg * eavg;
  const float shape_o = (1.0f - eo) / fmaxf(CUDART_PI_F * miss, 1e-6f);
  return f3(fms.x / den.x, fms.y / den.y, fms.z / den.z) * shape_o;
}

// GGX distribution in the cancellation-free form (ggxD, material.wgsl.ts:2797-2804)
__device__ __forceinline__ float ggx_d(float nh, float a) {
  const float a2 = a * a;
  const float n2 = clamp01(nh * nh);
  const float d = (1.0f - n2) + n2 * a2;
  return a2 / (CUDART_PI_F * d * d);
}
// Smith G1 in the tangent form (roughDielectricSmithG1Wgsl, math/roughDielectric.ts:52-60)
__device__ __forceinline__ float smith_g1(float c, float a) {
  c = fmaxf(c, 0.0f);
  if (c <= 1e-6f) return 0.0f;
  const float c2 = c * c;
  const float t2 = fmaxf(0.0f, 1.0f - c2) / fmaxf(c2, 1e-10f);
  return 2.0f / (1.0f + sqrtf(1.0f + a * a * t2));
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
__device__ __forceinline__ float3 cosine_sample(float u1, float u2) {
  const float r = sqrtf(u1), phi = 2.0f * CUDART_PI_F * u2;
  return f3(r * cosf(phi), r * sinf(phi), sqrtf(fmaxf(0.0f, 1.0f - u1)));
}

// ---- opaque family
__device__ __forceinline__ float3 opaque_f0(const Material& m) {
  const float3 d = f3(m.f0_ior, m.f0_ior, m.f0_ior);
  return d + (m.base_color - d) * m.metallic;
}
__device__ __forceinline__ float3 opaque_fresnel(const Material& m, float3 f0, float c) {
  const float f90 = m.specular + (1.0f - m.specular) * m.metallic;
  return f0 + (f3(f90, f90, f90) - f0) * pow5(clamp01(1.0f - c));
}
// Per-vertex terms of the opaque BSDF that depend on the material and wo
// only, shared by the NEE evaluation and the BSDF sample of one vertex.
struct OpaqueSide {
  float3 f0;
  float nv;    // max(wo.z, 0)
  float sp;    // probability of the specular lobe (brdfFiniteBaseLobeWeights)
  float g1o;   // Smith G1 of wo
  float3 mso;  // multiple-scattering lobe without its (1 - E(mu_i)) factor
};
__device__ __forceinline__ OpaqueSide opaque_side(const Material& m, float3 wo) {
  OpaqueSide o;
  o.f0 = opaque_f0(m);
  o.nv = fmaxf(wo.z, 0.0f);
  const float fl = luminance(clamp01(opaque_fresnel(m, o.f0, o.nv)));
  o.sp = represented_bernoulli(fminf(fmaxf(0.04f + 0.92f * fmaxf(fl, m.metallic), 0.04f), 0.96f));
  o.g1o = smith_g1(o.nv, m.alpha);
  o.mso = ggx_multiscatter_o(clamp01(o.f0), m.roughness, o.nv);
  return o;
}
// BSDF * cos(wi) and the marginal sampling density; wo, wi in the local frame (n = +z)
__device__ __forceinline__ void opaque_eval(const Material& m, const OpaqueSide& o, float3 wo, float3 wi,
                                            float3& f_cos, float& pdf) {
  f_cos = f3(0.0f, 0.0f, 0.0f);
  pdf = 0.0f;
  const float nv = o.nv, nl = fmaxf(wi.z, 0.0f);
  if (nv <= 1e-5f || nl <= 1e-5f) return;
  const float3 h = normalize(wi + wo);
  const float nh = fmaxf(h.z, 0.0f), vh = fmaxf(dot(wo, h), 0.0f);
  const float3 F = clamp01(opaque_fresnel(m, o.f0, vh));
  const float3 kd = (f3(1.0f, 1.0f, 1.0f) - F) * (1.0f - m.metallic);
  const float d = ggx_d(nh, m.alpha);
  const float3 spec = F * (d * o.g1o * smith_g1(nl, m.alpha) / fmaxf(4.0f * nv * nl, 1e-6f));
  const float3 ms = o.mso * (1.0f - ggx_albedo(nl, m.roughness));
  f_cos = (kd * m.base_color * (1.0f / CUDART_PI_F) + spec + ms) * nl;
  pdf = (1.0f - o.sp) * nl * (1.0f / CUDART_PI_F) + o.sp * d * o.g1o / fmaxf(4.0f * nv, 1e-6f);
}

// ---- dielectric family
__device__ __forceinline__ float diel_fresnel(const Material& m, float c, float eta) {
  c = clamp01(fabsf(c));
  eta = fmaxf(fabsf(eta), 1e-8f);
  if (eta < 1.0f && 1.0f - c * c >= eta * eta) return 1.0f;  // total internal reflection
  return clamp01(m.f0_ior + (m.specular - m.f0_ior) * pow5(1.0f - c));
}
// (joint reflection, joint diffuse, joint transmission, P(reflection | not diffuse))
// as realised by rand01 thresholds (bsdfRepresentedDielectricEventProbabilities, bsdf.wgsl.ts:1036-1097)
__device__ __forceinline__ float4 diel_events(float d, float r, float t) {
  d = fmaxf(d, 0.0f);
  r = fmaxf(r, 0.0f);
  t = fmaxf(t, 0.0f);
  const float total = d + r + t;
  if (!(total > 0.0f)) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float dt = r + t;
  if (!(dt > 0.0f)) return make_float4(0.0f, 1.0f, 0.0f, 0.0f);
  if (!(d > 0.0f)) {
    const float rc = t > 0.0f ? represented_bernoulli(r / dt) : 1.0f;
    return make_float4(rc, 0.0f, 1.0f - rc, rc);
  }
  float pd, pdi;
  if (d <= dt) {
    pd = represented_bernoulli(d / total);
    pdi = 1.0f - pd;
  } else {
    pdi = represented_bernoulli(dt / total);
    pd = 1.0f - pdi;
  }
  float rc;
  if (!(r > 0.0f)) rc = 0.0f;
  else if (!(t > 0.0f)) rc = 1.0f;
  else if (r <= t) rc = represented_bernoulli(r / dt);
  else rc = 1.0f - represented_bernoulli(t / dt);
  const float pr = pdi * rc;
  return make_float4(pr, pd, pdi - pr, rc);
}
// event probabilities for the microfacet normal wm (bsdfDielectricFiniteEventProbabilities)
__device__ __forceinline__ float4 diel_event_probs(const Material& m, float eta, float cos_o, float wo_wm) {
  const float macro_t = 1.0f - diel_fresnel(m, cos_o, eta);
  const float fm = diel_fresnel(m, wo_wm, eta);
  return diel_events(clamp01(macro_t * (1.0f - m.transmission)), fm, m.transmission * clamp01(1.0f - fm));
}
// half vector of a transmission pair, on the side of n (bsdfRoughTransmissionHalfVector)
__device__ __forceinline__ float3 diel_half_t(float3 wo, float3 wi, float eta) {
  float3 wm = normalize(wo + wi * eta);
  if (wm.z < 0.0f) wm = -wm;
  return wm;
}
// visible-normal density of wm (bsdfGgxVisibleNormalPdf)
__device__ __forceinline__ float vndf_pdf(const Material& m, float3 wo, float3 wm) {
  const float no = fmaxf(wo.z, 1e-6f), om = dot(wo, wm);
  if (no <= 1e-5f || om <= 1e-6f || wm.z <= 0.0f) return 0.0f;
  return ggx_d(fmaxf(wm.z, 0.0f), m.alpha) * smith_g1(no, m.alpha) * om / no;
}
// BSDF * |cos(wi)| and marginal density; wo on the +z side, eta = n_t / n_i
// for light arriving from wo's side
__device__ __forceinline__ void diel_eval(const Material& m, float eta, float3 wo, float3 wi, float3& f_cos,
                                          float& pdf) {
  f_cos = f3(0.0f, 0.0f, 0.0f);
  pdf = 0.0f;
  const bool smooth = m.roughness <= 0.0f;
  const float co = wo.z, ci = wi.z;
  if (co <= 1e-5f) return;
  if (wi.z > 0.0f) {
    // same side: diffuse lobe plus rough reflection
    if (ci <= 1e-5f) return;
    const float3 wm = normalize(wo + wi);
    const float4 ev = diel_event_probs(m, eta, co, fabsf(dot(wo, wm)));
    const float macro_t = 1.0f - diel_fresnel(m, co, eta);
    float3 f = m.base_color * (macro_t * (1.0f - m.transmission) * (1.0f / CUDART_PI_F));
    float ps = 0.0f;
    if (!smooth) {
      const float d = ggx_d(fmaxf(wm.z, 0.0f), m.alpha);
      const float g1o = smith_g1(co, m.alpha);
      const float fm = diel_fresnel(m, fabsf(dot(wo, wm)), eta);
      const float r = d * g1o * smith_g1(ci, m.alpha) * fm / fmaxf(4.0f * co * ci, 1e-10f);
      f = f + f3(r, r, r);
      ps = d * g1o / fmaxf(4.0f * co, 1e-6f);
    }
    f_cos = f * ci;
    pdf = ev.y * ci * (1.0f / CUDART_PI_F) + ev.x * ps;
  } else {
    // opposite side: rough transmission only
    if (smooth || ci >= -1e-5f) return;
    const float3 wm = diel_half_t(wo, wi, eta);
    const float im = dot(wi, wm), om = dot(wo, wm);
    if (im * ci < 0.0f || om * co < 0.0f) return;
    const float den = im + om / eta;
    const float d = ggx_d(fmaxf(wm.z, 0.0f), m.alpha);
    const float g = smith_g1(co, m.alpha) * smith_g1(fabsf(ci), m.alpha);
    const float tr = 1.0f - diel_fresnel(m, fabsf(om), eta);
    const float ft = d * tr * g * fabsf(im * om / fmaxf(fabsf(den * den * ci * co), 1e-10f)) / (eta * eta);
    f_cos = m.base_color * (m.transmission * ft * fabsf(ci));
    const float4 ev = diel_event_probs(m, eta, co, fabsf(om));
    pdf = ev.z * vndf_pdf(m, wo, wm) * fabsf(im) / fmaxf(den * den, 1e-10f);
  }
}
// Finite-support BSDF of either family (0 for delta-only surfaces).
// `o` is opaque_side(m, wo) for the opaque family (unused for dielectrics).
__device__ __forceinline__ void bsdf_eval(const Material& m, const OpaqueSide& o, float eta, float3 wo, float3 wi,
                                          float3& f_cos, float& pdf) {
  if (m.kind == kDielectric) diel_eval(m, eta, wo, wi, f_cos, pdf);
  else opaque_eval(m, o, wo, wi, f_cos, pdf);
}
__device__ __forceinline__ OpaqueSide surface_side(const Material& m, float3 wo) {
  if (m.kind != kDielectric) return opaque_side(m, wo);
  OpaqueSide o;
  o.f0 = f3(0.0f, 0.0f, 0.0f);
  o.nv = fmaxf(wo.z, 0.0f);
  o.sp = 0.0f;
  o.g1o = 0.0f;
  o.mso = f3(0.0f, 0.0f, 0.0f);
  return o;
}
__device__ __forceinline__ bool has_finite_support(const Material& m) {
  return m.kind != kDielectric || m.roughness > 0.0f || m.transmission < 1.0f;
}

// One BSDF sample.  wo in the local frame (+z side), eta = n_t / n_i.
struct BsdfSample {
  float3 wi;       // local frame
  float3 weight;   // f * |cos| / pdf
  float pdf;       // event density (for delta events the discrete probability)
  bool delta;
  bool valid;
};
__device__ __forceinline__ BsdfSample sample_bsdf(const Material& m, const OpaqueSide& o, float eta, float3 wo,
                                                  uint32_t& rng) {
  BsdfSample s;
  s.wi = f3(0.0f, 0.0f, 1.0f);
  s.weight = f3(0.0f, 0.0f, 0.0f);
  s.pdf = 0.0f;
  s.delta = false;
  s.valid = false;
  if (m.kind != kDielectric) {
    const bool spec = rand01(rng) < o.sp;
    const float u1 = rand01(rng), u2 = rand01(rng);
    if (spec) {
      const float3 h = ggx_vndf(wo, m.alpha, u1, u2);
      s.wi = h * (2.0f * dot(wo, h)) - wo;
    } else {
      s.wi = cosine_sample(u1, u2);
    }
  } else {
    const bool smooth = m.roughness <= 0.0f;
    float3 wm = f3(0.0f, 0.0f, 1.0f);
    if (!smooth) {
      const float u1 = rand01(rng), u2 = rand01(rng);
      wm = ggx_vndf(wo, m.alpha, u1, u2);
    }
    // refraction about wm (transmitted direction of the incoming ray -wo)
    const float ci = dot(wo, wm);
    const float k = 1.0f - (1.0f - ci * ci) / (eta * eta);
    const bool can_refract = k >= 0.0f;
    const float fm = can_refract ? diel_fresnel(m, fabsf(ci), eta) : 1.0f;
    const float macro_t = 1.0f - diel_fresnel(m, wo.z, eta);
    const float4 ev = diel_events(clamp01(macro_t * (1.0f - m.transmission)), fm,
                                  m.transmission * clamp01(1.0f - fm));
    const bool diffuse = rand01(rng) < ev.y;
    bool refl = false;
    if (!diffuse) refl = rand01(rng) < ev.w;
    if (diffuse) {
      const float u1 = rand01(rng), u2 = rand01(rng);
      s.wi = cosine_sample(u1, u2);
    } else if (refl) {
      s.wi = wm * (2.0f * ci) - wo;
      if (smooth) {
        s.pdf = ev.x;
        s.weight = f3(fm, fm, fm) * (1.0f / fmaxf(ev.x, 1e-10f));
        s.delta = true;
        s.valid = ev.x > 0.0f;
        return s;
      }
      if (s.wi.z <= 1e-5f) return s;
    } else {
      if (!can_refract) return s;
      s.wi = normalize(wo * (-1.0f / eta) + wm * (ci / eta - sqrtf(k)));
      if (smooth) {
        s.pdf = ev.z;
        s.weight = m.base_color * (m.transmission * (1.0f - fm) / (eta * eta) / fmaxf(ev.z, 1e-10f));
        s.delta = true;
        s.valid = ev.z > 0.0f;
        return s;
      }
      if (s.wi.z >= -1e-5f) return s;
    }
  }
  // continuous events: the full BSDF over the marginal density
  float3 fc;
  float pdf;
  bsdf_eval(m, o, eta, wo, s.wi, fc, pdf);
  if (!(pdf > 0.0f) || fabsf(s.wi.z) <= 1e-8f) return s;
  s.pdf = pdf;
  s.weight = fc * (1.0f / pdf);
  s.valid = maxc(s.weight) > 0.0f;
  return s;
}

}  // namespace pt
}  // namespace vt
