/*
 * pt_oracle.c -- CPU restatement of the unidirectional path tracer.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the device path tracer).
 *
 * Follows the reference integrator's estimator for the plain-PT subset
 * (packages/pt-webgpu/src/wgsl/pathTrace/kernel.wgsl.ts:963-2030, CPU mirror
 * packages/pt-webgpu/src/__tests__/cpuTracer.ts:411-518 generalised to the
 * reference's base BSDF, listed at the BSDF section below):
 *   PCG32 and the frame key            shared-samplers/src/wgsl/pcg.wgsl.ts:5-24,
 *                                      pt-webgpu/src/wgsl/common.wgsl.ts:194-196
 *   primary ray from the inverse VP    kernelCore.wgsl.ts:22-26, common.wgsl.ts:431-470
 *   one light entry, uniform pick      kernel.wgsl.ts:1149-1675 (cpuTracer.ts:411-452)
 *   power-heuristic MIS                material.wgsl.ts:2808-2822
 *   GGX VNDF                           bsdf.wgsl.ts:1710-1737
 *   RR for bounce > 2                  kernelCore.wgsl.ts:54-67
 * with the same random-number consumption order as the device kernels, so
 * most samples follow the same path on both sides.  Visibility is the FP64
 * Moller-Trumbore test (compressedWideBvh.ts:551-614) over a binned-SAH BVH
 * built by orc_build_array_bvh.  Accumulates FP64 per-pixel sums and sums
 * of squares.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../vitrum_b200/csrc/ggx_albedo_lut.h"

long orc_build_array_bvh(const float* positions, long n_pos_words, int pos_stride, const uint32_t* indices,
                         long ntri, int idx_stride, int max_leaf, int nbins, int max_depth, uint32_t* out_nodes,
                         uint32_t* out_reordered_to_source);
int orc_tri_hit_d(const double o[3], const double d[3], const double a[3], const double b[3], const double c[3],
                  double tmin, double* t);
int orc_hw_threads(void);
long orc_lt_build(const double* power, const double* centroid, const double* aabb, const double* cone, long n,
                  float* out, long cap);
void orc_lt_merge_cones(const double* cones, long n, double* out6);
float orc_lt_select(const float* tree, long nodes, uint32_t n_pos, uint32_t n_dist, const float* p, const float* nrm,
                    float floor_d2, uint32_t bucket, int* emitter);

#define PI_F 3.14159265358979323846f

/* ---------------------------------------------------------------- RNG */
static uint32_t pcg_init(uint32_t px, uint32_t py, uint32_t key) {
  uint32_t s = px * 1664525u + py * 1013904223u + key * 22695477u;
  s ^= s >> 17;
  s ^= s << 31;
  s ^= s >> 11;
  return s;
}
static uint32_t pcg_next(uint32_t* s) {
  *s = *s * 747796405u + 2891336453u;
  uint32_t w = ((*s >> ((*s >> 28) + 4u)) ^ *s) * 277803737u;
  return (w >> 22) ^ w;
}
static float rand01(uint32_t* s) { return (float)(pcg_next(s) >> 8) * (1.0f / 16777216.0f); }
static float represented_bernoulli(float p) {
  if (!(p > 0.0f)) return 0.0f;
  if (p >= 1.0f) return 1.0f;
  float b = floorf(p * 16777216.0f + 0.5f);
  if (b < 1.0f) b = 1.0f;
  if (b > 16777215.0f) b = 16777215.0f;
  return b * (1.0f / 16777216.0f);
}
static uint32_t rand_bounded(uint32_t* s, uint32_t bound) {
  if (bound <= 1u) return 0u;
  uint32_t threshold = (0u - bound) % bound;
  uint32_t v = pcg_next(s);
  for (int k = 0; k < 64 && v < threshold; ++k) v = pcg_next(s);
  return v % bound;
}

/* ---------------------------------------------------------------- vectors */
typedef struct { float x, y, z; } v3;
static v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static v3 scl(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 cross3(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static float maxc(v3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
static v3 nrm(v3 a) {
  float l2 = dot3(a, a);
  return l2 > 1e-30f ? scl(a, 1.0f / sqrtf(l2)) : V(0, 0, 1);
}
static void onb(v3 n, v3* t, v3* b) {
  float l2 = n.x * n.x + n.y * n.y;
  if (l2 > 1e-10f) {
    float inv = 1.0f / sqrtf(l2);
    *t = V(-n.y * inv, n.x * inv, 0.0f);
  } else {
    *t = V(1, 0, 0);
  }
  *b = cross3(n, *t);
}

/* ---------------------------------------------------------------- scene */
typedef struct {
  float base[3], roughness, emission[3], ior;
  int kind; /* 0 opaque, 1 opaque metallic, 2 dielectric (transmission > 0, metallic 0) */
  float alpha;
  int emissive;
  unsigned flags; /* 1 single-sided (back faces ignored), 2 ignored by shadow rays */
  float metallic, transmission, specular, f0_ior;
} orc_mat_t;

typedef struct {
  const float* pos;       /* stride 4 */
  const uint32_t* idx;    /* stride 4 */
  const uint32_t* tmat;   /* per triangle */
  long ntri;
  uint32_t* nodes;        /* binary BVH */
  uint32_t* r2s;
  const orc_mat_t* mats;
  /* emitters */
  const uint32_t* em_tri; /* emissive triangle ids */
  const float* em_cdf;
  long n_em;
  float em_area;
  const float* points;    /* 16 floats each: position, 0, intensity, 0, axis, cos outer, cos inner, range, decay, spot */
  long n_points;
  const float* areas;     /* 16 floats each: centre, shape (0 rect / 1 disc), u, area, v, 0, radiance, 0 */
  long n_areas;
  const float* dirs; /* 8 floats: direction towards the light, cos(angular radius), rgb, delta */
  long n_dirs;
  const float* env;       /* W*H*3 */
  const float* env_marg;  /* H+1 */
  const float* env_cond;  /* H*(W+1) */
  int env_w, env_h, env_sampleable;
  float env_scale;
  float env_cos, env_sin; /* environment rotation about +y */
  int n_entries;
  int lt_mode;            /* 1: tree selection (light tree over the positional entries, distant ones outside) */
  float* lt;              /* the tree (16 floats per node), NULL below two positional entries */
  long lt_nodes;
  float bias;
  /* camera / frame */
  const float* inv_vp;    /* row-major */
  int width, height, max_bounces;
  uint32_t seed, sample_base;
  int spp;
  double* sum;
  double* sq;
  /* optional ray log: first `log_cap` rays of each kind (8 floats each) and totals */
  float* log_closest;
  float* log_shadow;
  long log_cap;
  long n_closest, n_shadow;  /* totals, updated atomically */
} orc_pt_t;

static void log_ray(orc_pt_t* S, int shadow, const double o[3], const double d[3], double tmax) {
  long k = __atomic_fetch_add(shadow ? &S->n_shadow : &S->n_closest, 1, __ATOMIC_RELAXED);
  float* buf = shadow ? S->log_shadow : S->log_closest;
  if (!buf || k >= S->log_cap) return;
  float* r = buf + 8 * k;
  r[0] = (float)o[0]; r[1] = (float)o[1]; r[2] = (float)o[2]; r[3] = 0.0f;
  r[4] = (float)d[0]; r[5] = (float)d[1]; r[6] = (float)d[2]; r[7] = (float)tmax;
}

static void tri_vertices(const orc_pt_t* S, long t, double a[3], double b[3], double c[3]) {
  const uint32_t* iv = S->idx + 4 * t;
  for (int k = 0; k < 3; ++k) {
    a[k] = S->pos[4 * iv[0] + k];
    b[k] = S->pos[4 * iv[1] + k];
    c[k] = S->pos[4 * iv[2] + k];
  }
}

static int box_hit(const float* mn, const float* mx, const double o[3], const double inv[3], double tmax, double* tn) {
  double t0 = 0.0, t1 = tmax;
  for (int k = 0; k < 3; ++k) {
    double a = (mn[k] - o[k]) * inv[k], b = (mx[k] - o[k]) * inv[k];
    if (a > b) { double x = a; a = b; b = x; }
    if (a > t0) t0 = a;
    if (b < t1) t1 = b;
    if (t1 < t0) return 0;
  }
  *tn = t0;
  return 1;
}

/* closest (any=0) or any (any=1) hit with t in (0, tmax); returns triangle id or -1 */
static long trace(const orc_pt_t* S, const double o[3], const double d[3], double tmax, int any, double* t_out) {
  double inv[3];
  for (int k = 0; k < 3; ++k) inv[k] = 1.0 / (fabs(d[k]) > 1e-30 ? d[k] : copysign(1e-30, d[k]));
  uint32_t stack[128];
  int sp = 0;
  stack[sp++] = 0;
  long best = -1;
  double closest = tmax;
  while (sp > 0) {
    uint32_t n = stack[--sp];
    const uint32_t* nd = S->nodes + 8 * (size_t)n;
    double tn;
    if (!box_hit((const float*)nd, (const float*)nd + 3, o, inv, closest, &tn)) continue;
    if ((nd[7] >> 16) == 0xFFFFu) {
      uint32_t cnt = nd[7] & 0xFFFFu;
      for (uint32_t i = 0; i < cnt; ++i) {
        long tri = S->r2s[nd[6] + i];
        double a[3], b[3], c[3], t;
        tri_vertices(S, tri, a, b, c);
        const unsigned fl = S->mats[S->tmat[tri]].flags;
        if (any && (fl & 2u)) continue; /* castShadow: false */
        if (orc_tri_hit_d(o, d, a, b, c, 0.0, &t) && t > 0.0 && t < closest) {
          if (fl & 1u) { /* single-sided: skip hits on the back face */
            const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
            const double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
            if (d[0] * n[0] + d[1] * n[1] + d[2] * n[2] > 0.0) continue;
          }
          closest = t;
          best = tri;
          if (any) { *t_out = t; return best; }
        }
      }
      continue;
    }
    uint32_t l = n + 1, r = n + nd[6];
    if (sp + 2 > 128) continue;
    /* near child on top */
    double tl = 0, tr = 0;
    const uint32_t* ln = S->nodes + 8 * (size_t)l;
    const uint32_t* rn = S->nodes + 8 * (size_t)r;
    int hl = box_hit((const float*)ln, (const float*)ln + 3, o, inv, closest, &tl);
    int hr = box_hit((const float*)rn, (const float*)rn + 3, o, inv, closest, &tr);
    if (hl && hr) {
      if (tl < tr) { stack[sp++] = r; stack[sp++] = l; } else { stack[sp++] = l; stack[sp++] = r; }
    } else if (hl) {
      stack[sp++] = l;
    } else if (hr) {
      stack[sp++] = r;
    }
  }
  *t_out = closest;
  return best;
}

/* ---------------------------------------------------------------- BSDF
 * The reference's base BSDF for the parameters the scene carries (base colour,
 * roughness, metallic, transmission, IOR, specular factor):
 *   opaque      evaluateBrdfFullWithClearcoatNormal  bsdf.wgsl.ts:809-916
 *               F0 / F90 (KHR specular)              bsdf.wgsl.ts:192-222
 *               lobe choice, marginal pdf            bsdf.wgsl.ts:1172-1211, 1555-1630
 *               sampling + finite finalizer          bsdf.wgsl.ts:2919-2998, 1863-1924
 *               Kulla-Conty lobe, E tables           material.wgsl.ts:2840-2931
 *   dielectric  Fresnel (Schlick, exact TIR)         bsdf.wgsl.ts:227-256
 *               events (represented Bernoulli)       bsdf.wgsl.ts:1036-1170
 *               rough reflection / transmission      bsdf.wgsl.ts:941-1033, 1996-2140
 *               sampling                             bsdf.wgsl.ts:2618-2812
 *   GGX D, Smith G1 (tangent form)                   material.wgsl.ts:2797-2804, math/roughDielectric.ts:52-60
 */
static const float ggx_e_tab[VT_GGX_ALBEDO_DIM * VT_GGX_ALBEDO_DIM] = {VT_GGX_E_VALUES};
static const float ggx_eavg_tab[VT_GGX_ALBEDO_DIM] = {VT_GGX_EAVG_VALUES};

static float clamp01f(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
static v3 clamp01v(v3 v) { return V(clamp01f(v.x), clamp01f(v.y), clamp01f(v.z)); }
static float lum(v3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
static float pow5f(float x) { float x2 = x * x; return x2 * x2 * x; }
static v3 mbase(const orc_mat_t* m) { return V(m->base[0], m->base[1], m->base[2]); }

static float ggx_albedo(float mu, float r) {
  const int D = VT_GGX_ALBEDO_DIM;
  float fr = clamp01f(r) * (float)(D - 1), fm = clamp01f(mu) * (float)(D - 1);
  int r0 = (int)floorf(fr), m0 = (int)floorf(fm);
  int r1 = r0 + 1 < D ? r0 + 1 : D - 1, m1 = m0 + 1 < D ? m0 + 1 : D - 1;
  float tr = fr - (float)r0, tm = fm - (float)m0;
  float e0 = ggx_e_tab[r0 * D + m0] + (ggx_e_tab[r0 * D + m1] - ggx_e_tab[r0 * D + m0]) * tm;
  float e1 = ggx_e_tab[r1 * D + m0] + (ggx_e_tab[r1 * D + m1] - ggx_e_tab[r1 * D + m0]) * tm;
  return fminf(fmaxf(e0 + (e1 - e0) * tr, 0.02f), 1.0f);
}
static float ggx_albedo_avg(float r) {
  const int D = VT_GGX_ALBEDO_DIM;
  float fr = clamp01f(r) * (float)(D - 1);
  int r0 = (int)floorf(fr), r1 = r0 + 1 < D ? r0 + 1 : D - 1;
  float tr = fr - (float)r0;
  return fminf(fmaxf(ggx_eavg_tab[r0] + (ggx_eavg_tab[r1] - ggx_eavg_tab[r0]) * tr, 0.3f), 1.0f);
}
/* F_avg^2 E_avg / (1 - F_avg (1 - E_avg)) * (1 - E(mu_o)) (1 - E(mu_i)) / (pi (1 - E_avg)) */
static v3 ggx_multiscatter(v3 f0, float r, float nv, float nl) {
  float eavg = ggx_albedo_avg(r), miss = 1.0f - eavg;
  if (miss < 1e-4f) return V(0, 0, 0);
  float eo = ggx_albedo(nv, r), ei = ggx_albedo(nl, r);
  v3 favg = add(f0, scl(sub(V(1, 1, 1), f0), 1.0f / 21.0f));
  v3 fms = scl(mul(favg, favg), eavg);
  float shape_o = (1.0f - eo) / fmaxf(PI_F * miss, 1e-6f);
  v3 mso = V(fms.x / fmaxf(1.0f - favg.x * miss, 1e-4f) * shape_o, fms.y / fmaxf(1.0f - favg.y * miss, 1e-4f) * shape_o,
             fms.z / fmaxf(1.0f - favg.z * miss, 1e-4f) * shape_o);
  return scl(mso, 1.0f - ei);
}
static float ggx_d(float nh, float a) {
  float a2 = a * a, n2 = clamp01f(nh * nh), d = (1.0f - n2) + n2 * a2;
  return a2 / (PI_F * d * d);
}
static float smith_g1(float c, float a) {
  c = fmaxf(c, 0.0f);
  if (c <= 1e-6f) return 0.0f;
  float c2 = c * c, t2 = fmaxf(0.0f, 1.0f - c2) / fmaxf(c2, 1e-10f);
  return 2.0f / (1.0f + sqrtf(1.0f + a * a * t2));
}
static v3 ggx_vndf(v3 wo, float a, float u1, float u2) {
  v3 vh = nrm(V(a * wo.x, a * wo.y, wo.z)), t1, t2;
  onb(vh, &t1, &t2);
  float r = sqrtf(u1), phi = 2.0f * PI_F * u2;
  float p1 = r * cosf(phi), p2 = r * sinf(phi), s = 0.5f * (1.0f + vh.z);
  p2 = (1.0f - s) * sqrtf(fmaxf(0.0f, 1.0f - p1 * p1)) + s * p2;
  float z = sqrtf(fmaxf(0.0f, 1.0f - p1 * p1 - p2 * p2));
  v3 nh = add(add(scl(t1, p1), scl(t2, p2)), scl(vh, z));
  return nrm(V(a * nh.x, a * nh.y, fmaxf(1e-6f, nh.z)));
}
static v3 cosine_sample(float u1, float u2) {
  float r = sqrtf(u1), phi = 2.0f * PI_F * u2;
  return V(r * cosf(phi), r * sinf(phi), sqrtf(fmaxf(0.0f, 1.0f - u1)));
}
static float power_h(float a, float b) {
  if (!(a >= 0.0f) || !(b >= 0.0f) || a > 3.402823466e38f || b > 3.402823466e38f) return 0.0f;
  float m = fmaxf(a, b);
  if (!(m > 0.0f)) return 0.0f;
  float x = a / m, y = b / m;
  return (x * x) / (x * x + y * y);
}

/* opaque family */
static v3 opaque_f0(const orc_mat_t* m) {
  v3 d = V(m->f0_ior, m->f0_ior, m->f0_ior);
  return add(d, scl(sub(mbase(m), d), m->metallic));
}
static v3 opaque_fresnel(const orc_mat_t* m, v3 f0, float c) {
  float f90 = m->specular + (1.0f - m->specular) * m->metallic;
  return add(f0, scl(sub(V(f90, f90, f90), f0), pow5f(clamp01f(1.0f - c))));
}
static float opaque_spec_prob(const orc_mat_t* m, v3 f0, float nv) {
  float fl = lum(clamp01v(opaque_fresnel(m, f0, nv)));
  return represented_bernoulli(fminf(fmaxf(0.04f + 0.92f * fmaxf(fl, m->metallic), 0.04f), 0.96f));
}
static void opaque_eval(const orc_mat_t* m, v3 wo, v3 wi, v3* fc, float* pdf) {
  *fc = V(0, 0, 0);
  *pdf = 0.0f;
  float nv = fmaxf(wo.z, 0.0f), nl = fmaxf(wi.z, 0.0f);
  if (nv <= 1e-5f || nl <= 1e-5f) return;
  v3 h = nrm(add(wi, wo));
  float nh = fmaxf(h.z, 0.0f), vh = fmaxf(dot3(wo, h), 0.0f);
  v3 f0 = opaque_f0(m);
  v3 F = clamp01v(opaque_fresnel(m, f0, vh));
  v3 kd = scl(sub(V(1, 1, 1), F), 1.0f - m->metallic);
  float d = ggx_d(nh, m->alpha), g1o = smith_g1(nv, m->alpha);
  v3 spec = scl(F, d * g1o * smith_g1(nl, m->alpha) / fmaxf(4.0f * nv * nl, 1e-6f));
  v3 ms = ggx_multiscatter(clamp01v(f0), m->roughness, nv, nl);
  *fc = scl(add(add(scl(mul(kd, mbase(m)), 1.0f / PI_F), spec), ms), nl);
  float sp = opaque_spec_prob(m, f0, nv);
  *pdf = (1.0f - sp) * nl * (1.0f / PI_F) + sp * d * g1o / fmaxf(4.0f * nv, 1e-6f);
}

/* dielectric family; eta = n_t / n_i for light arriving along wo, wo on +z */
static float diel_fresnel(const orc_mat_t* m, float c, float eta) {
  c = clamp01f(fabsf(c));
  eta = fmaxf(fabsf(eta), 1e-8f);
  if (eta < 1.0f && 1.0f - c * c >= eta * eta) return 1.0f;
  return clamp01f(m->f0_ior + (m->specular - m->f0_ior) * pow5f(1.0f - c));
}
/* (joint reflection, joint diffuse, joint transmission, P(reflection | not diffuse)) */
static void diel_events(float d, float r, float t, float out[4]) {
  d = fmaxf(d, 0.0f);
  r = fmaxf(r, 0.0f);
  t = fmaxf(t, 0.0f);
  float total = d + r + t, dt = r + t;
  out[0] = out[1] = out[2] = out[3] = 0.0f;
  if (!(total > 0.0f)) return;
  if (!(dt > 0.0f)) { out[1] = 1.0f; return; }
  if (!(d > 0.0f)) {
    float rc = t > 0.0f ? represented_bernoulli(r / dt) : 1.0f;
    out[0] = rc; out[2] = 1.0f - rc; out[3] = rc;
    return;
  }
  float pd, pdi, rc;
  if (d <= dt) { pd = represented_bernoulli(d / total); pdi = 1.0f - pd; }
  else { pdi = represented_bernoulli(dt / total); pd = 1.0f - pdi; }
  if (!(r > 0.0f)) rc = 0.0f;
  else if (!(t > 0.0f)) rc = 1.0f;
  else if (r <= t) rc = represented_bernoulli(r / dt);
  else rc = 1.0f - represented_bernoulli(t / dt);
  out[0] = pdi * rc; out[1] = pd; out[2] = pdi - pdi * rc; out[3] = rc;
}
static void diel_event_probs(const orc_mat_t* m, float eta, float cos_o, float wo_wm, float out[4]) {
  float macro_t = 1.0f - diel_fresnel(m, cos_o, eta), fm = diel_fresnel(m, wo_wm, eta);
  diel_events(clamp01f(macro_t * (1.0f - m->transmission)), fm, m->transmission * clamp01f(1.0f - fm), out);
}
static float vndf_pdf(const orc_mat_t* m, v3 wo, v3 wm) {
  float no = fmaxf(wo.z, 1e-6f), om = dot3(wo, wm);
  if (no <= 1e-5f || om <= 1e-6f || wm.z <= 0.0f) return 0.0f;
  return ggx_d(fmaxf(wm.z, 0.0f), m->alpha) * smith_g1(no, m->alpha) * om / no;
}
static void diel_eval(const orc_mat_t* m, float eta, v3 wo, v3 wi, v3* fc, float* pdf) {
  *fc = V(0, 0, 0);
  *pdf = 0.0f;
  int smooth = m->roughness <= 0.0f;
  float co = wo.z, ci = wi.z, ev[4];
  if (co <= 1e-5f) return;
  if (wi.z > 0.0f) {
    if (ci <= 1e-5f) return;
    v3 wm = nrm(add(wo, wi));
    diel_event_probs(m, eta, co, fabsf(dot3(wo, wm)), ev);
    float macro_t = 1.0f - diel_fresnel(m, co, eta);
    v3 f = scl(mbase(m), macro_t * (1.0f - m->transmission) * (1.0f / PI_F));
    float ps = 0.0f;
    if (!smooth) {
      float d = ggx_d(fmaxf(wm.z, 0.0f), m->alpha), g1o = smith_g1(co, m->alpha);
      float fm = diel_fresnel(m, fabsf(dot3(wo, wm)), eta);
      float r = d * g1o * smith_g1(ci, m->alpha) * fm / fmaxf(4.0f * co * ci, 1e-10f);
      f = add(f, V(r, r, r));
      ps = d * g1o / fmaxf(4.0f * co, 1e-6f);
    }
    *fc = scl(f, ci);
    *pdf = ev[1] * ci * (1.0f / PI_F) + ev[0] * ps;
  } else {
    if (smooth || ci >= -1e-5f) return;
    v3 wm = nrm(add(wo, scl(wi, eta)));
    if (wm.z < 0.0f) wm = scl(wm, -1.0f);
    float im = dot3(wi, wm), om = dot3(wo, wm);
    if (im * ci < 0.0f || om * co < 0.0f) return;
    float den = im + om / eta;
    float d = ggx_d(fmaxf(wm.z, 0.0f), m->alpha);
    float g = smith_g1(co, m->alpha) * smith_g1(fabsf(ci), m->alpha);
    float tr = 1.0f - diel_fresnel(m, fabsf(om), eta);
    float ft = d * tr * g * fabsf(im * om / fmaxf(fabsf(den * den * ci * co), 1e-10f)) / (eta * eta);
    *fc = scl(mbase(m), m->transmission * ft * fabsf(ci));
    diel_event_probs(m, eta, co, fabsf(om), ev);
    *pdf = ev[2] * vndf_pdf(m, wo, wm) * fabsf(im) / fmaxf(den * den, 1e-10f);
  }
}
static void bsdf_eval(const orc_mat_t* m, float eta, v3 wo, v3 wi, v3* fc, float* pdf) {
  if (m->kind == 2) diel_eval(m, eta, wo, wi, fc, pdf);
  else opaque_eval(m, wo, wi, fc, pdf);
}
static int has_finite_support(const orc_mat_t* m) {
  return m->kind != 2 || m->roughness > 0.0f || m->transmission < 1.0f;
}
typedef struct { v3 wi, weight; float pdf; int delta, valid; } bsample_t;
static bsample_t sample_bsdf(const orc_mat_t* m, float eta, v3 wo, uint32_t* rng) {
  bsample_t s;
  s.wi = V(0, 0, 1);
  s.weight = V(0, 0, 0);
  s.pdf = 0.0f;
  s.delta = 0;
  s.valid = 0;
  if (m->kind != 2) {
    float sp = opaque_spec_prob(m, opaque_f0(m), fmaxf(wo.z, 0.0f));
    int spec = rand01(rng) < sp;
    float u1 = rand01(rng), u2 = rand01(rng);
    if (spec) {
      v3 h = ggx_vndf(wo, m->alpha, u1, u2);
      s.wi = sub(scl(h, 2.0f * dot3(wo, h)), wo);
    } else {
      s.wi = cosine_sample(u1, u2);
    }
  } else {
    int smooth = m->roughness <= 0.0f;
    v3 wm = V(0, 0, 1);
    if (!smooth) {
      float u1 = rand01(rng), u2 = rand01(rng);
      wm = ggx_vndf(wo, m->alpha, u1, u2);
    }
    float ci = dot3(wo, wm), k = 1.0f - (1.0f - ci * ci) / (eta * eta);
    int can_refract = k >= 0.0f;
    float fm = can_refract ? diel_fresnel(m, fabsf(ci), eta) : 1.0f;
    float macro_t = 1.0f - diel_fresnel(m, wo.z, eta), ev[4];
    diel_events(clamp01f(macro_t * (1.0f - m->transmission)), fm, m->transmission * clamp01f(1.0f - fm), ev);
    int diffuse = rand01(rng) < ev[1], refl = 0;
    if (!diffuse) refl = rand01(rng) < ev[3];
    if (diffuse) {
      float u1 = rand01(rng), u2 = rand01(rng);
      s.wi = cosine_sample(u1, u2);
    } else if (refl) {
      s.wi = sub(scl(wm, 2.0f * ci), wo);
      if (smooth) {
        s.pdf = ev[0];
        s.weight = scl(V(fm, fm, fm), 1.0f / fmaxf(ev[0], 1e-10f));
        s.delta = 1;
        s.valid = ev[0] > 0.0f;
        return s;
      }
      if (s.wi.z <= 1e-5f) return s;
    } else {
      if (!can_refract) return s;
      s.wi = nrm(add(scl(wo, -1.0f / eta), scl(wm, ci / eta - sqrtf(k))));
      if (smooth) {
        s.pdf = ev[2];
        s.weight = scl(mbase(m), m->transmission * (1.0f - fm) / (eta * eta) / fmaxf(ev[2], 1e-10f));
        s.delta = 1;
        s.valid = ev[2] > 0.0f;
        return s;
      }
      if (s.wi.z >= -1e-5f) return s;
    }
  }
  v3 fc;
  float pdf;
  bsdf_eval(m, eta, wo, s.wi, &fc, &pdf);
  if (!(pdf > 0.0f) || fabsf(s.wi.z) <= 1e-8f) return s;
  s.pdf = pdf;
  s.weight = scl(fc, 1.0f / pdf);
  s.valid = maxc(s.weight) > 0.0f;
  return s;
}

/* ---------------------------------------------------------------- lights */
static int cdf_search(const float* cdf, int n, float u) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (cdf[mid] > u) hi = mid; else lo = mid + 1;
  }
  return lo;
}
static void env_texel(const orc_pt_t* S, v3 dw, int* col, int* row, float* st) {
  /* into the unrotated map (rotateYNeg, connectCore.wgsl.ts:27-30) */
  v3 d = V(S->env_cos * dw.x - S->env_sin * dw.z, dw.y, S->env_sin * dw.x + S->env_cos * dw.z);
  /* u = phi / 2pi + 0.5 (wrapped), row 0 at +y (environmentLookup, connect.wgsl.ts:139-142) */
  float y = fminf(fmaxf(d.y, -1.0f), 1.0f), theta = acosf(y);
  float u = atan2f(d.z, d.x) * (0.5f / PI_F) + 0.5f;
  if (u >= 1.0f) u -= 1.0f;
  *col = (int)(u * S->env_w);
  if (*col > S->env_w - 1) *col = S->env_w - 1;
  *row = (int)(theta * (1.0f / PI_F) * S->env_h);
  if (*row > S->env_h - 1) *row = S->env_h - 1;
  *st = sinf(theta);
}
static float env_pdf(const orc_pt_t* S, int col, int row, float st) {
  if (!(st > 0.0f)) return 0.0f;
  float pm = S->env_marg[row + 1] - S->env_marg[row];
  const float* cc = S->env_cond + (size_t)row * (S->env_w + 1);
  float pc = cc[col + 1] - cc[col];
  return pm * pc * (float)S->env_w * (float)S->env_h / (2.0f * PI_F * PI_F * st);
}
static v3 env_le(const orc_pt_t* S, int col, int row) {
  const float* e = S->env + 3 * ((size_t)row * S->env_w + col);
  return scl(V(e[0], e[1], e[2]), S->env_scale);
}

/* pdf includes the entry selection; pdf_light is the same without it (the MIS density) */
typedef struct { v3 wi, Le; float dist, pdf, pdf_light; int delta, valid; } lsample_t;

/* point / spot falloff: 1 / d^decay and the range window (material.wgsl.ts:2176-2204) */
static float positional_falloff(float dist, float d2, float range, float decay) {
  if (!(dist > 0.0f) || dist > 3.402823466e38f) return 0.0f;
  float a = 1.0f;
  if (decay > 0.01f) {
    float den = decay == 2.0f ? d2 : powf(dist, decay);
    if (!(den > 0.0f)) a = 3.402823466e38f;
    else if (den > 3.402823466e38f) return 0.0f;
    else a = fminf(1.0f / den, 3.402823466e38f);
  }
  if (range > 0.0f) {
    float q = dist / range, q2 = q * q;
    a *= clamp01f(1.0f - q2 * q2);
  }
  return a;
}
static float smoothstep_f(float e0, float e1, float x) {
  float t = clamp01f((x - e0) / (e1 - e0));
  return t * t * (3.0f - 2.0f * t);
}
/* Shirley-Chiu concentric map (kernel.wgsl.ts:1422-1426) */
static void concentric_disc(float a, float b, float* x, float* y) {
  if (a == 0.0f && b == 0.0f) { *x = 0.0f; *y = 0.0f; return; }
  float r, phi;
  if (fabsf(a) > fabsf(b)) { r = a; phi = (0.25f * PI_F) * (b / a); }
  else { r = b; phi = 0.5f * PI_F - (0.25f * PI_F) * (a / b); }
  *x = r * cosf(phi);
  *y = r * sinf(phi);
}
/* nearest analytic area light crossed by (o, d) from its emitting side before t_max
 * (connect.wgsl.ts:390-450) */
static int area_light_hit(const orc_pt_t* S, v3 o, v3 d, float t_max, v3* Le, float* pdf_sa) {
  int found = 0;
  float best = t_max;
  for (long k = 0; k < S->n_areas; ++k) {
    const float* q = S->areas + 16 * k;
    v3 U = V(q[4], q[5], q[6]), Vv = V(q[8], q[9], q[10]), nl = nrm(cross3(U, Vv));
    float den = dot3(nl, d);
    if (!(den < 0.0f)) continue;
    v3 c = V(q[0], q[1], q[2]);
    float t = dot3(nl, sub(c, o)) / den;
    if (!(t > 0.0f && t < best)) continue;
    v3 rel = sub(add(o, scl(d, t)), c);
    float uu = dot3(U, U), uv = dot3(U, Vv), vv = dot3(Vv, Vv), ru = dot3(rel, U), rv = dot3(rel, Vv);
    float det = uu * vv - uv * uv;
    float x = (ru * vv - rv * uv) / det, y = (rv * uu - ru * uv) / det;
    int inside = q[3] != 0.0f ? x * x + y * y <= 1.0f : (fabsf(x) <= 1.0f && fabsf(y) <= 1.0f);
    if (!inside) continue;
    best = t;
    found = 1;
    *Le = V(q[12], q[13], q[14]);
    *pdf_sa = t * t / (q[7] * -den);
  }
  return found;
}

/* N: the unit normal on the incoming side for surfaces that reflect only, else zero */
static lsample_t sample_light(const orc_pt_t* S, v3 P, v3 N, uint32_t* rng) {
  lsample_t ls;
  memset(&ls, 0, sizeof ls);
  /* entry selection: the light tree (one 24-bit draw) or uniform; the
   * selection probability is divided out of the estimate, not part of the MIS
   * weights (pt-webgpu mediumNee.wgsl.ts:14-37, connect.wgsl.ts:598) */
  float psel;
  uint32_t e;
  if (S->lt_mode) {
    float p3[3] = {P.x, P.y, P.z};
    int em = -1;
    uint32_t n_dist = (uint32_t)S->n_dirs + (S->env_sampleable ? 1u : 0u);
    float n3[3] = {N.x, N.y, N.z};
    psel = orc_lt_select(S->lt, S->lt_nodes, (uint32_t)S->n_entries - n_dist, n_dist, p3, n3, 1e-3f,
                         pcg_next(rng) >> 8, &em);
    if (em < 0 || em >= S->n_entries || !(psel > 0.0f)) return ls;
    e = (uint32_t)em;
  } else {
    psel = 1.0f / (float)S->n_entries;
    e = rand_bounded(rng, (uint32_t)S->n_entries);
  }
  if (S->n_em > 0) {
    if (e == 0) {
      float u = rand01(rng);
      int k = cdf_search(S->em_cdf, (int)S->n_em, u);
      double A[3], B[3], C[3];
      tri_vertices(S, S->em_tri[k], A, B, C);
      float u1 = rand01(rng), u2 = rand01(rng), su = sqrtf(u1);
      float wa = 1.0f - su, wb = su * (1.0f - u2), wc = su * u2;
      v3 a = V((float)A[0], (float)A[1], (float)A[2]), b = V((float)B[0], (float)B[1], (float)B[2]),
         c = V((float)C[0], (float)C[1], (float)C[2]);
      v3 X = add(add(scl(a, wa), scl(b, wb)), scl(c, wc));
      v3 nl = nrm(cross3(sub(b, a), sub(c, a)));
      v3 d = sub(X, P);
      float d2 = dot3(d, d), dist = sqrtf(d2);
      ls.wi = scl(d, 1.0f / dist);
      float cosl = -dot3(ls.wi, nl);
      if (!(cosl > 0.0f) || !(dist > 0.0f)) return ls;
      const orc_mat_t* m = &S->mats[S->tmat[S->em_tri[k]]];
      ls.Le = V(m->emission[0], m->emission[1], m->emission[2]);
      ls.dist = dist;
      ls.pdf_light = d2 / (S->em_area * cosl);
      ls.pdf = psel * ls.pdf_light;
      ls.valid = 1;
      return ls;
    }
    e -= 1;
  }
  if ((long)e < S->n_points) {
    /* point or spot light (kernel.wgsl.ts:1285-1397) */
    const float* p = S->points + 16 * e;
    v3 d = sub(V(p[0], p[1], p[2]), P);
    float d2 = dot3(d, d);
    if (!(d2 > 0.0f)) return ls;
    float dist = sqrtf(d2);
    if (p[13] > 0.0f && dist > p[13]) return ls;
    ls.wi = scl(d, 1.0f / dist);
    float cone = 1.0f;
    if (p[15] != 0.0f) {
      float c = -dot3(ls.wi, V(p[8], p[9], p[10]));
      if (!(c >= p[11])) return ls;
      cone = smoothstep_f(p[11], fmaxf(p[12], p[11] + 1e-6f), c);
    }
    ls.dist = dist;
    ls.Le = scl(V(p[4], p[5], p[6]), cone * positional_falloff(dist, d2, p[13], p[14]));
    ls.pdf = psel;
    ls.pdf_light = 1.0f;
    ls.delta = 1;
    ls.valid = 1;
    return ls;
  }
  e -= (uint32_t)S->n_points;
  if ((long)e < S->n_areas) {
    /* rectangle or disc, one-sided (kernel.wgsl.ts:1398-1493) */
    const float* q = S->areas + 16 * e;
    float xi1 = rand01(rng), xi2 = rand01(rng);
    float x = xi1 * 2.0f - 1.0f, y = xi2 * 2.0f - 1.0f;
    if (q[3] != 0.0f) concentric_disc(x, y, &x, &y);
    v3 U = V(q[4], q[5], q[6]), Vv = V(q[8], q[9], q[10]);
    v3 X = add(add(V(q[0], q[1], q[2]), scl(U, x)), scl(Vv, y));
    v3 d = sub(X, P);
    float d2 = dot3(d, d), dist = sqrtf(d2);
    if (!(dist > 0.0f)) return ls;
    ls.wi = scl(d, 1.0f / dist);
    float cosl = -dot3(ls.wi, nrm(cross3(U, Vv)));
    if (!(cosl > 0.0f)) return ls;
    ls.Le = V(q[12], q[13], q[14]);
    ls.dist = dist;
    ls.pdf_light = d2 / (q[7] * cosl);
    ls.pdf = psel * ls.pdf_light;
    ls.valid = 1;
    return ls;
  }
  e -= (uint32_t)S->n_areas;
  if ((long)e < S->n_dirs) {
    const float* q = S->dirs + 8 * e;
    v3 w = V(q[0], q[1], q[2]);
    ls.dist = INFINITY;
    ls.Le = V(q[4], q[5], q[6]);
    if (q[7] != 0.0f) {
      ls.wi = w;
      ls.pdf = psel;
      ls.pdf_light = 1.0f;
      ls.delta = 1;
    } else {
      float u1 = rand01(rng), u2 = rand01(rng);
      float ct = 1.0f - u1 * (1.0f - q[3]), st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct)), ph = 2.0f * PI_F * u2;
      v3 tu, tv;
      onb(w, &tu, &tv);
      ls.wi = add(add(scl(tu, st * cosf(ph)), scl(tv, st * sinf(ph))), scl(w, ct));
      ls.pdf_light = 1.0f / (2.0f * PI_F * (1.0f - q[3]));
      ls.pdf = psel * ls.pdf_light;
    }
    ls.valid = 1;
    return ls;
  }
  float u1 = rand01(rng), u2 = rand01(rng);
  int row = cdf_search(S->env_marg + 1, S->env_h, u1);
  const float* cc = S->env_cond + (size_t)row * (S->env_w + 1);
  int col = cdf_search(cc + 1, S->env_w, u2);
  float m0 = S->env_marg[row], m1 = S->env_marg[row + 1], c0 = cc[col], c1 = cc[col + 1];
  float fv = m1 > m0 ? (u1 - m0) / (m1 - m0) : 0.5f, fu = c1 > c0 ? (u2 - c0) / (c1 - c0) : 0.5f;
  float v = ((float)row + fminf(fmaxf(fv, 0.0f), 0.999999f)) / (float)S->env_h;
  float u = ((float)col + fminf(fmaxf(fu, 0.0f), 0.999999f)) / (float)S->env_w;
  float theta = v * PI_F, phi = (u - 0.5f) * 2.0f * PI_F, st = sinf(theta);
  v3 md = V(st * cosf(phi), cosf(theta), st * sinf(phi));
  ls.wi = V(S->env_cos * md.x + S->env_sin * md.z, md.y, -S->env_sin * md.x + S->env_cos * md.z);
  ls.dist = INFINITY;
  ls.Le = env_le(S, col, row);
  ls.pdf_light = env_pdf(S, col, row, st);
  ls.pdf = psel * ls.pdf_light;
  ls.valid = ls.pdf > 0.0f;
  return ls;
}

/* ---------------------------------------------------------------- integrator */
static v3 radiance_sample(orc_pt_t* S, int x, int y, uint32_t sample) {
  uint32_t rng = pcg_init((uint32_t)x, (uint32_t)y, S->seed ^ sample);
  float jx = rand01(&rng), jy = rand01(&rng);
  float u = ((float)x + jx) / (float)S->width, vv = ((float)y + jy) / (float)S->height;
  float nx = u * 2.0f - 1.0f, ny = 1.0f - vv * 2.0f;
  const float* M = S->inv_vp;
  float nf[4], fr[4];
  for (int r = 0; r < 4; ++r) {
    nf[r] = M[4 * r] * nx + M[4 * r + 1] * ny - M[4 * r + 2] + M[4 * r + 3];
    fr[r] = M[4 * r] * nx + M[4 * r + 1] * ny + M[4 * r + 2] + M[4 * r + 3];
  }
  v3 o = V(nf[0] / nf[3], nf[1] / nf[3], nf[2] / nf[3]);
  v3 d = nrm(sub(V(fr[0] / fr[3], fr[1] / fr[3], fr[2] / fr[3]), o));
  v3 T = V(1, 1, 1), L = V(0, 0, 0);
  int prev_delta = 1;
  float prev_pdf = 0.0f;
  for (int bounce = 0; bounce < S->max_bounces; ++bounce) {
    int last = bounce + 1 >= S->max_bounces;
    double od[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z}, t;
    log_ray(S, 0, od, dd, INFINITY);
    long tri = trace(S, od, dd, INFINITY, 0, &t);
    if (S->n_areas) {
      v3 le = V(0, 0, 0);
      float pa;
      if (area_light_hit(S, o, d, tri < 0 ? INFINITY : (float)t, &le, &pa)) {
        float w = prev_delta ? 1.0f : power_h(prev_pdf, pa);
        L = add(L, scl(mul(T, le), w));
      }
    }
    if (tri < 0) {
      for (long k = 0; k < S->n_dirs; ++k) {
        const float* q = S->dirs + 8 * k;
        if (q[7] != 0.0f || dot3(d, V(q[0], q[1], q[2])) < q[3]) continue;
        float w = 1.0f;
        if (!prev_delta) w = power_h(prev_pdf, 1.0f / (2.0f * PI_F * (1.0f - q[3])));
        L = add(L, scl(mul(T, V(q[4], q[5], q[6])), w));
      }
      if (S->env) {
        int col, row;
        float st;
        env_texel(S, d, &col, &row, &st);
        float w = 1.0f;
        if (!prev_delta && S->env_sampleable) w = power_h(prev_pdf, env_pdf(S, col, row, st));
        L = add(L, scl(mul(T, env_le(S, col, row)), w));
      }
      break;
    }
    double A[3], B[3], C[3];
    tri_vertices(S, tri, A, B, C);
    v3 a = V((float)A[0], (float)A[1], (float)A[2]), b = V((float)B[0], (float)B[1], (float)B[2]),
       c = V((float)C[0], (float)C[1], (float)C[2]);
    v3 ng = nrm(cross3(sub(b, a), sub(c, a)));
    const orc_mat_t* m = &S->mats[S->tmat[tri]];
    float tf = (float)t;
    v3 P = add(o, scl(d, tf));
    float dn = dot3(d, ng);
    int front = dn < 0.0f;
    if (m->emissive && front) {
      float w = 1.0f;
      if (!prev_delta) {
        float cosl = -dn;
        float pl = cosl > 0.0f ? tf * tf / (S->em_area * cosl) : 0.0f;
        w = power_h(prev_pdf, pl);
      }
      L = add(L, scl(mul(T, V(m->emission[0], m->emission[1], m->emission[2])), w));
    }
    v3 n = front ? ng : scl(ng, -1.0f);
    float off = S->bias * fmaxf(1.0f, fmaxf(fabsf(P.x), fmaxf(fabsf(P.y), fabsf(P.z))));
    v3 wo = scl(d, -1.0f), tb, bb;
    onb(n, &tb, &bb);
    v3 wol = V(dot3(wo, tb), dot3(wo, bb), dot3(wo, n));
    int alive = 0;
    float eta = front ? m->ior : 1.0f / m->ior;
    if (S->n_entries > 0 && has_finite_support(m)) {
      lsample_t ls = sample_light(S, P, m->kind == 2 && m->transmission > 0.0f ? V(0, 0, 0) : n, &rng);
      if (ls.valid) {
        v3 wil = V(dot3(ls.wi, tb), dot3(ls.wi, bb), dot3(ls.wi, n)), fc;
        float pb;
        bsdf_eval(m, eta, wol, wil, &fc, &pb);
        if (maxc(fc) > 0.0f) {
          float w = (ls.delta || last) ? 1.0f : power_h(ls.pdf_light, pb);
          v3 cc = scl(mul(mul(T, fc), ls.Le), w / ls.pdf);
          if (maxc(cc) > 0.0f) {
            v3 so = add(P, scl(n, wil.z > 0.0f ? off : -off));
            double sod[3] = {so.x, so.y, so.z}, sdd[3] = {ls.wi.x, ls.wi.y, ls.wi.z}, st2;
            double tmax = isinf(ls.dist) ? INFINITY : (double)(ls.dist * (1.0f - 1e-4f));
            log_ray(S, 1, sod, sdd, tmax);
            if (trace(S, sod, sdd, tmax, 1, &st2) < 0) L = add(L, cc);
          }
        }
      }
    }
    if (!last) {
      bsample_t bs = sample_bsdf(m, eta, wol, &rng);
      if (bs.valid) {
        v3 wi = add(add(scl(tb, bs.wi.x), scl(bb, bs.wi.y)), scl(n, bs.wi.z));
        T = mul(T, bs.weight);
        alive = 1;
        o = add(P, scl(n, bs.wi.z > 0.0f ? off : -off));
        d = wi;
        prev_delta = bs.delta;
        prev_pdf = bs.pdf;
      }
    }
    if (alive && bounce > 2) {
      float q = represented_bernoulli(fminf(fmaxf(maxc(T), 0.1f), 0.95f));
      if (!(rand01(&rng) < q)) alive = 0;
      else T = scl(T, 1.0f / q);
    }
    if (!alive) break;
  }
  return L;
}

typedef struct { orc_pt_t* S; long next; pthread_mutex_t mu; } pt_job_t;

static void* pt_worker(void* arg) {
  pt_job_t* j = (pt_job_t*)arg;
  orc_pt_t* S = j->S;
  long npx = (long)S->width * S->height;
  for (;;) {
    pthread_mutex_lock(&j->mu);
    long p = j->next++;
    pthread_mutex_unlock(&j->mu);
    if (p >= npx) break;
    int x = (int)(p % S->width), y = (int)(p / S->width);
    double s[3] = {0, 0, 0}, q[3] = {0, 0, 0};
    for (int k = 0; k < S->spp; ++k) {
      v3 L = radiance_sample(S, x, y, S->sample_base + (uint32_t)k);
      double v[3] = {L.x, L.y, L.z};
      for (int c = 0; c < 3; ++c) { s[c] += v[c]; q[c] += v[c] * v[c]; }
    }
    for (int c = 0; c < 3; ++c) { S->sum[3 * p + c] = s[c]; S->sq[3 * p + c] = q[c]; }
  }
  return NULL;
}

/* material record of 12 floats (layout at orc_pt_scene_create) */
static orc_mat_t make_mat(const float* m) {
  orc_mat_t r;
  memset(&r, 0, sizeof r);
  for (int k = 0; k < 3; ++k) { r.base[k] = m[k]; r.emission[k] = m[7 + k]; }
  r.roughness = m[3];
  r.ior = m[6] > 0 ? fmaxf(m[6], 1.0f) : 1.5f;
  r.metallic = m[4];
  r.transmission = clamp01f(m[5]);
  r.specular = m[11];
  float ratio = (r.ior - 1.0f) / (r.ior + 1.0f);
  r.f0_ior = ratio * ratio * r.specular;
  r.kind = (m[5] > 0 && m[4] == 0.0f) ? 2 : (m[4] > 0.0f ? 1 : 0);
  r.alpha = fmaxf(m[3] * m[3], 1e-3f);
  r.emissive = m[7] > 0 || m[8] > 0 || m[9] > 0;
  r.flags = (unsigned)m[10];
  return r;
}

/*
 * BSDF probes for the known-answer tests, in the shading frame (normal +z).
 * eta = n_t / n_i for light arriving along wo (dielectrics).
 */
float orc_smith_g1(float c, float alpha) { return smith_g1(c, alpha); }
float orc_ggx_d(float nh, float alpha) { return ggx_d(nh, alpha); }
void orc_ggx_vndf_batch(const float* wo, float alpha, const float* u, long n, float* wm) {
  v3 o = V(wo[0], wo[1], wo[2]);
  for (long i = 0; i < n; ++i) {
    v3 h = ggx_vndf(o, alpha, u[2 * i], u[2 * i + 1]);
    wm[3 * i] = h.x; wm[3 * i + 1] = h.y; wm[3 * i + 2] = h.z;
  }
}
void orc_vndf_pdf_batch(const float* mat12, const float* wo, const float* wm, long n, float* out) {
  orc_mat_t m = make_mat(mat12);
  v3 o = V(wo[0], wo[1], wo[2]);
  for (long i = 0; i < n; ++i) out[i] = vndf_pdf(&m, o, V(wm[3 * i], wm[3 * i + 1], wm[3 * i + 2]));
}
float orc_diel_fresnel(const float* mat12, float c, float eta) {
  orc_mat_t m = make_mat(mat12);
  return diel_fresnel(&m, c, eta);
}
void orc_diel_event_probs(const float* mat12, float eta, float cos_o, float wo_wm, float* out4) {
  orc_mat_t m = make_mat(mat12);
  diel_event_probs(&m, eta, cos_o, wo_wm, out4);
}
/* f * |cos wi| (rgb) and the sampling density of wi, for n directions wi */
void orc_bsdf_eval_batch(const float* mat12, float eta, const float* wo, const float* wi, long n, float* fc,
                         float* pdf) {
  orc_mat_t m = make_mat(mat12);
  v3 o = V(wo[0], wo[1], wo[2]);
  for (long i = 0; i < n; ++i) {
    v3 f;
    bsdf_eval(&m, eta, o, V(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), &f, &pdf[i]);
    fc[3 * i] = f.x; fc[3 * i + 1] = f.y; fc[3 * i + 2] = f.z;
  }
}
/* n samples of the BSDF from one PCG stream; flags bit 0 valid, bit 1 delta */
void orc_bsdf_sample_batch(const float* mat12, float eta, const float* wo, long n, uint32_t seed, float* wi,
                           float* weight, float* pdf, int* flags) {
  orc_mat_t m = make_mat(mat12);
  v3 o = V(wo[0], wo[1], wo[2]);
  uint32_t rng = pcg_init(seed, seed * 7u + 1u, 0x9E3779B9u);
  for (long i = 0; i < n; ++i) {
    bsample_t b = sample_bsdf(&m, eta, o, &rng);
    wi[3 * i] = b.wi.x; wi[3 * i + 1] = b.wi.y; wi[3 * i + 2] = b.wi.z;
    weight[3 * i] = b.weight.x; weight[3 * i + 1] = b.weight.y; weight[3 * i + 2] = b.weight.z;
    pdf[i] = b.pdf;
    flags[i] = (b.valid ? 1 : 0) | (b.delta ? 2 : 0);
  }
}

/*
 * The light tree over the positional light entries in sample_light's order:
 * the emissive-mesh group (one entry: power = sum of luminance x area, union
 * AABB, the triangles' one-sided cones merged), points, spots (cone along the
 * beam, half angle acos(cos outer)), rectangles and discs (one-sided cones)
 * (the reference's buildLightTreeInputForScene,
 * pt-webgpu/src/scene/emitterPacking.ts:1005-1232).  The distant entries
 * (directionals, the environment) are chosen outside the tree (orc_lt_select).
 */
static double lum_f(double r, double g, double b) { return (double)(float)(0.2126 * r + 0.7152 * g + 0.0722 * b); }
static void unit3(const double* v, double* o) {
  double l = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  for (int k = 0; k < 3; ++k) o[k] = l > 1e-12 ? v[k] / l : 0.0;
}
static void build_light_tree(orc_pt_t* S) {
  long n = (long)(S->n_em > 0 ? 1 : 0) + S->n_points + S->n_areas, k = 0;
  if (n < 2) return;
  double* pw = (double*)calloc((size_t)n, sizeof(double));
  double* cen = (double*)calloc((size_t)(3 * n), sizeof(double));
  double* box = (double*)calloc((size_t)(6 * n), sizeof(double));
  double* cone = (double*)calloc((size_t)(6 * n), sizeof(double));
  if (S->n_em > 0) {
    double* tc = (double*)calloc((size_t)(6 * S->n_em), sizeof(double));
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY}, p = 0.0;
    for (long t = 0; t < S->n_em; ++t) {
      double A[3], B[3], C[3];
      tri_vertices(S, S->em_tri[t], A, B, C);
      const orc_mat_t* m = &S->mats[S->tmat[S->em_tri[t]]];
      double e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]}, e2[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
      double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
      float area = (float)(0.5 * sqrt(cx * cx + cy * cy + cz * cz));
      p += (double)(float)(lum_f(m->emission[0], m->emission[1], m->emission[2]) * (double)area);
      for (int q = 0; q < 3; ++q) {
        mn[q] = fmin(mn[q], fmin(A[q], fmin(B[q], C[q])));
        mx[q] = fmax(mx[q], fmax(A[q], fmax(B[q], C[q])));
      }
      double nn[3] = {cx, cy, cz};
      unit3(nn, tc + 6 * t);
      tc[6 * t + 3] = 0.0;
      tc[6 * t + 4] = M_PI / 2;
      tc[6 * t + 5] = 1.0;
    }
    pw[k] = p;
    for (int q = 0; q < 3; ++q) {
      box[6 * k + q] = mn[q];
      box[6 * k + 3 + q] = mx[q];
      cen[3 * k + q] = 0.5 * mn[q] + 0.5 * mx[q];
    }
    orc_lt_merge_cones(tc, S->n_em, cone + 6 * k);
    free(tc);
    ++k;
  }
  for (long i = 0; i < S->n_points; ++i, ++k) {
    const float* q = S->points + 16 * i;
    pw[k] = lum_f(q[4], q[5], q[6]);
    for (int c = 0; c < 3; ++c) cen[3 * k + c] = box[6 * k + c] = box[6 * k + 3 + c] = q[c];
    if (q[15] != 0.0f) {
      double ax[3] = {q[8], q[9], q[10]};
      unit3(ax, cone + 6 * k);
      cone[6 * k + 3] = 0.0;
      cone[6 * k + 4] = acos(fmax(-1.0, fmin(1.0, (double)q[11])));
      cone[6 * k + 5] = 1.0;
    }
  }
  for (long i = 0; i < S->n_areas; ++i, ++k) {
    const float* q = S->areas + 16 * i;
    pw[k] = (double)(float)(lum_f(q[12], q[13], q[14]) * (double)q[7]);
    double U[3] = {q[4], q[5], q[6]}, W[3] = {q[8], q[9], q[10]};
    double r = sqrt(U[0] * U[0] + U[1] * U[1] + U[2] * U[2]);
    for (int c = 0; c < 3; ++c) {
      double h = q[3] != 0.0f ? r : fabs(U[c]) + fabs(W[c]);
      cen[3 * k + c] = q[c];
      box[6 * k + c] = (double)q[c] - h;
      box[6 * k + 3 + c] = (double)q[c] + h;
    }
    double nn[3] = {U[1] * W[2] - U[2] * W[1], U[2] * W[0] - U[0] * W[2], U[0] * W[1] - U[1] * W[0]};
    unit3(nn, cone + 6 * k);
    cone[6 * k + 3] = 0.0;
    cone[6 * k + 4] = M_PI / 2;
    cone[6 * k + 5] = 1.0;
  }
  S->lt = (float*)calloc((size_t)(16 * (2 * n)), sizeof(float));
  S->lt_nodes = orc_lt_build(pw, cen, box, cone, n, S->lt, 2 * n);
  if (S->lt_nodes <= 0) { free(S->lt); S->lt = NULL; S->lt_nodes = 0; }
  free(pw);
  free(cen);
  free(box);
  free(cone);
}

/*
 * Scene set-up, done once per scene: the binned-SAH BVH over all triangles
 * (orc_build_array_bvh), the material table, the emissive-triangle area CDF
 * and the environment's luminance CDFs.  materials: 12 floats each (base rgb
 * 0-2, roughness 3, metallic 4, transmission 5, ior 6, emission rgb 7-9,
 * flags 10, specular intensity 11); env: W*H*3 floats (NULL for none);
 * points: 16 floats each (points then spots); areas: 16 floats each
 * (rectangles then discs).  The caller keeps every input array alive until
 * orc_pt_scene_free.  Returns NULL on a build error.
 */
void* orc_pt_scene_create(const float* pos, long nvert, const uint32_t* idx, long ntri, const uint32_t* tri_mat,
                          const float* materials, int n_mat, const float* points, long n_points, const float* areas,
                          long n_areas, const float* dirs, long n_dirs, const float* env, int env_w, int env_h,
                          float env_scale, float env_rotation, float bias, int light_selection) {
  orc_pt_t* S = (orc_pt_t*)calloc(1, sizeof(orc_pt_t));
  if (!S) return NULL;
  S->env_cos = (float)cos((double)env_rotation);
  S->env_sin = (float)sin((double)env_rotation);
  S->pos = pos;
  S->idx = idx;
  S->tmat = tri_mat;
  S->ntri = ntri;
  S->nodes = (uint32_t*)malloc(sizeof(uint32_t) * 8 * (size_t)(2 * ntri + 1));
  S->r2s = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(ntri + 1));
  long nn = orc_build_array_bvh(pos, nvert * 4, 4, idx, ntri, 4, 4, 16, 58, S->nodes, S->r2s);
  if (nn < 0) { free(S->nodes); free(S->r2s); free(S); return NULL; }
  orc_mat_t* mats = (orc_mat_t*)calloc((size_t)(n_mat > 0 ? n_mat : 1), sizeof(orc_mat_t));
  for (int i = 0; i < n_mat; ++i) mats[i] = make_mat(materials + 12 * i);
  S->mats = mats;
  uint32_t* em = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(ntri + 1));
  float* cdf = (float*)malloc(sizeof(float) * (size_t)(ntri + 1));
  double total = 0.0;
  long ne = 0;
  for (long t = 0; t < ntri; ++t) {
    if (!mats[tri_mat[t]].emissive) continue;
    double a[3], b[3], c[3];
    tri_vertices(S, t, a, b, c);
    double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
    double area = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
    if (!(area > 0.0)) continue;
    em[ne] = (uint32_t)t;
    total += area;
    cdf[ne] = (float)total;
    ++ne;
  }
  for (long i = 0; i < ne; ++i) cdf[i] = (float)(cdf[i] / total);
  if (ne) cdf[ne - 1] = 1.0f;
  S->em_tri = em;
  S->em_cdf = cdf;
  S->n_em = ne;
  S->em_area = (float)total;
  S->points = points;
  S->n_points = n_points;
  S->areas = areas;
  S->n_areas = n_areas;
  S->dirs = dirs;
  S->n_dirs = n_dirs;
  if (env) {
    S->env = env;
    S->env_w = env_w;
    S->env_h = env_h;
    S->env_scale = env_scale > 0 ? env_scale : 1.0f;
    float* marg = (float*)malloc(sizeof(float) * (size_t)(env_h + 1));
    float* cond = (float*)malloc(sizeof(float) * (size_t)env_h * (env_w + 1));
    double tot = 0.0;
    double* rows = (double*)malloc(sizeof(double) * (size_t)env_h);
    double* cum = (double*)malloc(sizeof(double) * (size_t)env_w);
    for (int r = 0; r < env_h; ++r) {
      double st = sin(M_PI * (r + 0.5) / env_h), acc = 0.0;
      cond[(size_t)r * (env_w + 1)] = 0.0f;
      for (int c = 0; c < env_w; ++c) {
        const float* px = env + 3 * ((size_t)r * env_w + c);
        double lum = 0.2126 * px[0] + 0.7152 * px[1] + 0.0722 * px[2];
        acc += fmax(0.0, lum * S->env_scale) * st;
        cum[c] = acc;
      }
      for (int c = 0; c < env_w; ++c)
        cond[(size_t)r * (env_w + 1) + c + 1] = acc > 0 ? (float)(cum[c] / acc) : (float)(c + 1) / env_w;
      cond[(size_t)r * (env_w + 1) + env_w] = 1.0f;
      rows[r] = acc;
      tot += acc;
    }
    marg[0] = 0.0f;
    double run = 0.0;
    for (int r = 0; r < env_h; ++r) {
      run += rows[r];
      marg[r + 1] = tot > 0 ? (float)(run / tot) : (float)(r + 1) / env_h;
    }
    marg[env_h] = 1.0f;
    S->env_marg = marg;
    S->env_cond = cond;
    S->env_sampleable = tot > 0.0;
    free(rows);
    free(cum);
  }
  S->n_entries = (ne ? 1 : 0) + (int)n_points + (int)n_areas + (int)n_dirs + (S->env_sampleable ? 1 : 0);
  S->bias = bias;
  if (light_selection == 0 && S->n_entries >= 2) {
    S->lt_mode = 1;
    build_light_tree(S);
  }
  return S;
}

void orc_pt_scene_free(void* h) {
  orc_pt_t* S = (orc_pt_t*)h;
  if (!S) return;
  free(S->nodes);
  free(S->r2s);
  free((void*)S->mats);
  free((void*)S->em_tri);
  free((void*)S->em_cdf);
  free((void*)S->env_marg);
  free((void*)S->env_cond);
  free(S->lt);
  free(S);
}

/*
 * Render width x height pixels x spp samples of a scene made by
 * orc_pt_scene_create: FP64 sum and sum of squares (3 per pixel).  The
 * optional ray log keeps the first log_cap rays of each kind; ray_totals gets
 * the closest-hit and shadow rays traced by this call.  Returns 0.
 */
int orc_pt_scene_render(void* h, const float* inv_vp, int width, int height, int spp, int max_bounces, uint32_t seed,
                        uint32_t sample_base, int nthreads, double* sum, double* sq, float* log_closest,
                        float* log_shadow, long log_cap, long* ray_totals) {
  orc_pt_t* S = (orc_pt_t*)h;
  S->inv_vp = inv_vp;
  S->width = width;
  S->height = height;
  S->max_bounces = max_bounces;
  S->seed = seed;
  S->sample_base = sample_base;
  S->spp = spp;
  S->sum = sum;
  S->sq = sq;
  S->log_closest = log_closest;
  S->log_shadow = log_shadow;
  S->log_cap = log_cap;
  S->n_closest = 0;
  S->n_shadow = 0;
  pt_job_t job;
  job.S = S;
  job.next = 0;
  pthread_mutex_init(&job.mu, NULL);
  if (nthreads <= 0) nthreads = orc_hw_threads();
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], NULL, pt_worker, &job);
  for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
  pthread_mutex_destroy(&job.mu);
  if (ray_totals) { ray_totals[0] = S->n_closest; ray_totals[1] = S->n_shadow; }
  return 0;
}

/* One-shot form: scene set-up, render, free.  Returns 0, or -1 on a build error. */
int orc_pt_render(const float* pos, long nvert, const uint32_t* idx, long ntri, const uint32_t* tri_mat,
                  const float* materials, int n_mat, const float* points, long n_points, const float* areas,
                  long n_areas, const float* dirs,
                  long n_dirs, const float* env,
                  int env_w, int env_h, float env_scale, float env_rotation, const float* inv_vp, int width,
                  int height, int spp,
                  int max_bounces, uint32_t seed, uint32_t sample_base, float bias, int nthreads, double* sum,
                  double* sq, float* log_closest, float* log_shadow, long log_cap, long* ray_totals,
                  int light_selection) {
  void* h = orc_pt_scene_create(pos, nvert, idx, ntri, tri_mat, materials, n_mat, points, n_points, areas, n_areas,
                                dirs, n_dirs, env, env_w, env_h, env_scale, env_rotation, bias, light_selection);
  if (!h) return -1;
  orc_pt_scene_render(h, inv_vp, width, height, spp, max_bounces, seed, sample_base, nthreads, sum, sq, log_closest,
                      log_shadow, log_cap, ray_totals);
  orc_pt_scene_free(h);
  return 0;
}
