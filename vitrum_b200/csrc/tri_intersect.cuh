// tri_intersect.cuh -- device ray/triangle tests.
//
// wt_*  : the watertight f32 test of the reference
//         (packages/shared-bvh/src/opticalWatertightTriangle.ts:98-220,
//         WGSL twin shared-bvh/src/wgsl/opticalWatertightTriangle.wgsl.ts:129).
//         Every operation is an explicitly rounded binary32 intrinsic
//         (__fadd_rn & co. are never contracted into FMAs), so results are
//         bit-identical to the reference's Math.fround arithmetic.
// ff_*  : float-float (double-f32) Moller-Trumbore used once per ray to
//         report t and barycentrics of the chosen triangle to ~1e-12
//         relative, i.e. the FP64 values of the reference CPU query
//         (compressedWideBvh.ts:551-614) rounded to f32, while all
//         arithmetic stays in FP32 units.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

namespace vt {

// ---------------------------------------------------------------- ray setup
struct WtRay {
  float o[3];     // origin
  float d[3];     // direction as given
  float dn[3];    // d / ds (each component correctly rounded)
  float ds;       // max |d|
  float sx, sy, sz;
  int kx, ky, kz;
  bool ok;        // direction finite and non-zero
};

__device__ __forceinline__ float fsel3(const float v[3], int k) { return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]); }

__device__ __forceinline__ float max3n(float a, float b, float c) {
  // Math.max semantics on f32 values: NaN propagates.
  if (isnan(a) || isnan(b) || isnan(c)) return CUDART_NAN_F;
  return fmaxf(fmaxf(a, b), c);
}

__device__ __forceinline__ WtRay wt_setup(float ox, float oy, float oz, float dx, float dy, float dz) {
  WtRay r;
  r.o[0] = ox; r.o[1] = oy; r.o[2] = oz;
  r.d[0] = dx; r.d[1] = dy; r.d[2] = dz;
  r.ds = max3n(fabsf(dx), fabsf(dy), fabsf(dz));
  r.ok = (r.ds > 0.0f) && isfinite(r.ds);
  float* dn = r.dn;
  dn[0] = __fdiv_rn(dx, r.ds); dn[1] = __fdiv_rn(dy, r.ds); dn[2] = __fdiv_rn(dz, r.ds);
  int kz = fabsf(dn[1]) > fabsf(dn[0]) ? 1 : 0;
  if (fabsf(dn[2]) > fabsf(fsel3(dn, kz))) kz = 2;
  int kx = kz == 2 ? 0 : kz + 1;
  int ky = kx == 2 ? 0 : kx + 1;
  if (fsel3(dn, kz) < 0.0f) { int t = kx; kx = ky; ky = t; }
  float dkz = fsel3(dn, kz);
  r.sx = __fdiv_rn(fsel3(dn, kx), dkz);
  r.sy = __fdiv_rn(fsel3(dn, ky), dkz);
  r.sz = __frcp_rn(dkz);
  r.kx = kx; r.ky = ky; r.kz = kz;
  return r;
}

// edgeFunction, opticalWatertightTriangle.ts:19-26
__device__ __forceinline__ float wt_edge(float ax, float ay, float bx, float by) {
  if (ax == bx && ay == by) return 0.0f;
  bool ordered = ax < bx || (ax == bx && ay < by);
  float fx = ordered ? ax : bx, fy = ordered ? ay : by;
  float sx = ordered ? bx : ax, sy = ordered ? by : ay;
  float canon = __fsub_rn(__fmul_rn(fx, sy), __fmul_rn(fy, sx));
  return ordered ? canon : -canon;
}

// rayParameter, opticalWatertightTriangle.ts:28-51
__device__ __noinline__ float wt_ray_param(const float o[3], const float d[3], const float p[3]) {
  float del[3] = {__fsub_rn(p[0], o[0]), __fsub_rn(p[1], o[1]), __fsub_rn(p[2], o[2])};
  float dls = max3n(fabsf(del[0]), fabsf(del[1]), fabsf(del[2]));
  float drs = max3n(fabsf(d[0]), fabsf(d[1]), fabsf(d[2]));
  if (!(drs > 0.0f) || !isfinite(drs) || !isfinite(dls)) return -1.0f;
  if (!(dls > 0.0f)) return 0.0f;
  float dd[3] = {__fdiv_rn(d[0], drs), __fdiv_rn(d[1], drs), __fdiv_rn(d[2], drs)};
  float q[3] = {__fdiv_rn(del[0], dls), __fdiv_rn(del[1], dls), __fdiv_rn(del[2], dls)};
  float num = __fadd_rn(__fadd_rn(__fmul_rn(q[0], dd[0]), __fmul_rn(q[1], dd[1])), __fmul_rn(q[2], dd[2]));
  float den = __fadd_rn(__fadd_rn(__fmul_rn(dd[0], dd[0]), __fmul_rn(dd[1], dd[1])), __fmul_rn(dd[2], dd[2]));
  return __fmul_rn(__fdiv_rn(num, den), __fdiv_rn(dls, drs));
}

__device__ __forceinline__ bool lex_before(const float a[3], const float b[3]) {
  return a[0] < b[0] || (a[0] == b[0] && (a[1] < b[1] || (a[1] == b[1] && a[2] < b[2])));
}

// edgeRayParameter, opticalWatertightTriangle.ts:59-87
__device__ __noinline__ float wt_edge_ray_param(const float o[3], const float d[3], const float fi[3],
                                                const float si[3], float fpx, float fpy, float spx, float spy) {
  bool ordered = lex_before(fi, si);
  const float* f = ordered ? fi : si;
  const float* s = ordered ? si : fi;
  float ax = ordered ? fpx : spx, ay = ordered ? fpy : spy;
  float bx = ordered ? spx : fpx, by = ordered ? spy : fpy;
  float delx = __fsub_rn(bx, ax), dely = __fsub_rn(by, ay);
  float ip;
  if (fabsf(delx) >= fabsf(dely)) {
    if (delx == 0.0f) return -1.0f;
    ip = __fdiv_rn(-ax, delx);
  } else {
    if (dely == 0.0f) return -1.0f;
    ip = __fdiv_rn(-ay, dely);
  }
  float pt[3];
  for (int k = 0; k < 3; ++k) pt[k] = __fadd_rn(f[k], __fmul_rn(ip, __fsub_rn(s[k], f[k])));
  return wt_ray_param(o, d, pt);
}

struct WtHit {
  float t;
  float bary[3];
  int side;
  int mask;
};

// Tail of the test once the sign test passed: t, zero-edge cases, normal and
// side checks (opticalWatertightTriangle.ts:145-219).  Kept out of line and
// fed by value: it runs only for candidate hits.
__device__ __noinline__ bool wt_finish(const WtRay r, const float3 A, const float3 B, const float3 C, float e0,
                                       float e1, float e2, float det, float az, float bz, float cz, float apx,
                                       float apy, float bpx, float bpy, float cpx, float cpy, float exclusive_min_t,
                                       WtHit* out) {
  const float a[3] = {A.x, A.y, A.z}, b[3] = {B.x, B.y, B.z}, c[3] = {C.x, C.y, C.z};
  bool pos = det > 0.0f;
  float n0 = pos ? e0 : -e0, n1 = pos ? e1 : -e1, n2 = pos ? e2 : -e2;
  float st = __fadd_rn(__fadd_rn(__fmul_rn(e0, az), __fmul_rn(e1, bz)), __fmul_rn(e2, cz));
  float t = __fdiv_rn(__fdiv_rn(st, det), r.ds);
  int zc = (n0 == 0.0f) + (n1 == 0.0f) + (n2 == 0.0f);
  if (zc >= 2) {
    if (n0 != 0.0f) t = wt_ray_param(r.o, r.d, a);
    if (n1 != 0.0f) t = wt_ray_param(r.o, r.d, b);
    if (n2 != 0.0f) t = wt_ray_param(r.o, r.d, c);
  } else if (n0 == 0.0f) {
    t = wt_edge_ray_param(r.o, r.d, b, c, bpx, bpy, cpx, cpy);
  } else if (n1 == 0.0f) {
    t = wt_edge_ray_param(r.o, r.d, c, a, cpx, cpy, apx, apy);
  } else if (n2 == 0.0f) {
    t = wt_edge_ray_param(r.o, r.d, a, b, apx, apy, bpx, bpy);
  }
  float lo = exclusive_min_t > 0.0f ? exclusive_min_t : 0.0f;
  if (!(t > lo) || !isfinite(t)) return false;
  float e1r[3], e2r[3];
  for (int k = 0; k < 3; ++k) { e1r[k] = __fsub_rn(b[k], a[k]); e2r[k] = __fsub_rn(c[k], a[k]); }
  float es = 0.0f;
  for (int k = 0; k < 3; ++k) es = fmaxf(es, fabsf(e1r[k]));
  for (int k = 0; k < 3; ++k) es = fmaxf(es, fabsf(e2r[k]));
  if (!(es > 0.0f) || !isfinite(es)) return false;
  float s1[3], s2[3];
  for (int k = 0; k < 3; ++k) { s1[k] = __fdiv_rn(e1r[k], es); s2[k] = __fdiv_rn(e2r[k], es); }
  float nr[3] = {__fsub_rn(__fmul_rn(s1[1], s2[2]), __fmul_rn(s1[2], s2[1])),
                 __fsub_rn(__fmul_rn(s1[2], s2[0]), __fmul_rn(s1[0], s2[2])),
                 __fsub_rn(__fmul_rn(s1[0], s2[1]), __fmul_rn(s1[1], s2[0]))};
  float ns = max3n(fabsf(nr[0]), fabsf(nr[1]), fabsf(nr[2]));
  if (!(ns > 0.0f) || !isfinite(ns)) return false;
  float nd[3] = {__fdiv_rn(nr[0], ns), __fdiv_rn(nr[1], ns), __fdiv_rn(nr[2], ns)};
  float l2 = __fadd_rn(__fadd_rn(__fmul_rn(nd[0], nd[0]), __fmul_rn(nd[1], nd[1])), __fmul_rn(nd[2], nd[2]));
  float nl = __fsqrt_rn(l2);
  if (!(nl > 0.0f) || !isfinite(nl)) return false;
  float nn[3] = {__fdiv_rn(nd[0], nl), __fdiv_rn(nd[1], nl), __fdiv_rn(nd[2], nl)};
  float dn[3] = {__fdiv_rn(r.d[0], r.ds), __fdiv_rn(r.d[1], r.ds), __fdiv_rn(r.d[2], r.ds)};
  float sd = -__fadd_rn(__fadd_rn(__fmul_rn(dn[0], nn[0]), __fmul_rn(dn[1], nn[1])), __fmul_rn(dn[2], nn[2]));
  if (sd == 0.0f || !isfinite(sd)) return false;
  out->t = t;
  out->bary[0] = __fdiv_rn(e0, det);
  out->bary[1] = __fdiv_rn(e1, det);
  out->bary[2] = __fdiv_rn(e2, det);
  out->side = sd > 0.0f ? 1 : -1;
  out->mask = (n0 == 0.0f ? 1 : 0) | (n1 == 0.0f ? 2 : 0) | (n2 == 0.0f ? 4 : 0);
  return true;
}

// Projected (sheared) 2-D vertex from a float3 vertex.
__device__ __forceinline__ void wt_project3(const WtRay& r, float3 v, float& px, float& py, float& pz) {
  float vx = r.kx == 0 ? v.x : (r.kx == 1 ? v.y : v.z);
  float vy = r.ky == 0 ? v.x : (r.ky == 1 ? v.y : v.z);
  float vz = r.kz == 0 ? v.x : (r.kz == 1 ? v.y : v.z);
  float a = __fsub_rn(vx, fsel3(r.o, r.kx));
  float b = __fsub_rn(vy, fsel3(r.o, r.ky));
  pz = __fsub_rn(vz, fsel3(r.o, r.kz));
  px = __fsub_rn(a, __fmul_rn(r.sx, pz));
  py = __fsub_rn(b, __fmul_rn(r.sy, pz));
}

// Full watertight test.  Returns true on hit with t > max(exclusive_min_t, 0).
__device__ __forceinline__ bool wt_intersect(const WtRay& r, float3 a, float3 b, float3 c, float exclusive_min_t,
                                             WtHit* out) {
  if (!r.ok || isnan(exclusive_min_t)) return false;
  float apx, apy, az, bpx, bpy, bz, cpx, cpy, cz;
  wt_project3(r, a, apx, apy, az);
  wt_project3(r, b, bpx, bpy, bz);
  wt_project3(r, c, cpx, cpy, cz);
  float e0 = wt_edge(bpx, bpy, cpx, cpy);
  float e1 = wt_edge(cpx, cpy, apx, apy);
  float e2 = wt_edge(apx, apy, bpx, bpy);
  float det = __fadd_rn(__fadd_rn(e0, e1), e2);
  if (det == 0.0f || !isfinite(det)) return false;
  bool pos = det > 0.0f;
  if (pos ? (e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) : (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return false;
  return wt_finish(r, a, b, c, e0, e1, e2, det, __fmul_rn(az, r.sz), __fmul_rn(bz, r.sz), __fmul_rn(cz, r.sz),
                   apx, apy, bpx, bpy, cpx, cpy, exclusive_min_t, out);
}

// Rare tail of the traversal test: t for a hit whose projected point lies
// exactly on an edge or vertex (opticalWatertightTriangle.ts:151-162).
__device__ __noinline__ float wt_zero_edge_t(const WtRay r, const float3 A, const float3 B, const float3 C, float n0,
                                             float n1, float n2, float apx, float apy, float bpx, float bpy,
                                             float cpx, float cpy) {
  const float a[3] = {A.x, A.y, A.z}, b[3] = {B.x, B.y, B.z}, c[3] = {C.x, C.y, C.z};
  const int zc = (n0 == 0.0f) + (n1 == 0.0f) + (n2 == 0.0f);
  float t = -1.0f;
  if (zc >= 2) {
    if (n0 != 0.0f) t = wt_ray_param(r.o, r.d, a);
    if (n1 != 0.0f) t = wt_ray_param(r.o, r.d, b);
    if (n2 != 0.0f) t = wt_ray_param(r.o, r.d, c);
  } else if (n0 == 0.0f) {
    t = wt_edge_ray_param(r.o, r.d, b, c, bpx, bpy, cpx, cpy);
  } else if (n1 == 0.0f) {
    t = wt_edge_ray_param(r.o, r.d, c, a, cpx, cpy, apx, apy);
  } else {
    t = wt_edge_ray_param(r.o, r.d, a, b, apx, apy, bpx, bpy);
  }
  return t;
}

// Watertight test inside traversal.  Returns the exact f32 t when the
// triangle is hit with max(exclusive_min_t, 0) < t < closest, else -1.  The
// accept/reject decision is identical to wt_intersect followed by
// `t < closest`: the interval check only moves ahead of the normal/side
// checks (which can only reject), and the triangle-only part of those checks
// -- the reference's normal derivation -- comes precomputed in the record
// (`nrm` = (n.xyz, valid)), leaving the ray-dependent side determinant.
template <class NormalFetch>
__device__ __forceinline__ float wt_candidate(const WtRay& r, float3 a, float3 b, float3 c, float exclusive_min_t,
                                              float closest, NormalFetch nrm_fetch, bool cull_back = false) {
  float apx, apy, az, bpx, bpy, bz, cpx, cpy, cz;
  wt_project3(r, a, apx, apy, az);
  wt_project3(r, b, bpx, bpy, bz);
  wt_project3(r, c, cpx, cpy, cz);
  const float e0 = wt_edge(bpx, bpy, cpx, cpy);
  const float e1 = wt_edge(cpx, cpy, apx, apy);
  const float e2 = wt_edge(apx, apy, bpx, bpy);
  const float det = __fadd_rn(__fadd_rn(e0, e1), e2);
  if (det == 0.0f || !isfinite(det)) return -1.0f;
  const bool pos = det > 0.0f;
  if (pos ? (e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) : (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return -1.0f;
  const float lo = exclusive_min_t > 0.0f ? exclusive_min_t : 0.0f;
  const float st = __fadd_rn(__fadd_rn(__fmul_rn(e0, __fmul_rn(az, r.sz)), __fmul_rn(e1, __fmul_rn(bz, r.sz))),
                             __fmul_rn(e2, __fmul_rn(cz, r.sz)));
  float t;
  if (e0 != 0.0f && e1 != 0.0f && e2 != 0.0f) {
    // Cheap reject before the exact divisions: the fast quotient is within a
    // few ulp of the exact one while both operands stay below 2^126, so a
    // 1e-5 relative margin decides most far candidates without changing any result.
    if (fabsf(det) < 1e30f && r.ds < 1e30f) {
      const float ta = __fdividef(__fdividef(st, det), r.ds);
      if (ta > closest * 1.00001f + 1e-30f || ta < lo * 0.99999f - 1e-30f) return -1.0f;
    }
    t = __fdiv_rn(__fdiv_rn(st, det), r.ds);
  } else {
    t = wt_zero_edge_t(r, a, b, c, pos ? e0 : -e0, pos ? e1 : -e1, pos ? e2 : -e2, apx, apy, bpx, bpy, cpx, cpy);
  }
  if (!(t > lo) || !isfinite(t) || !(t < closest)) return -1.0f;
  const float4 nrm = nrm_fetch();
  if (!(nrm.w != 0.0f)) return -1.0f;
  const float sd = -__fadd_rn(__fadd_rn(__fmul_rn(r.dn[0], nrm.x), __fmul_rn(r.dn[1], nrm.y)),
                              __fmul_rn(r.dn[2], nrm.z));
  if (sd == 0.0f || !isfinite(sd)) return -1.0f;
  if (cull_back && sd < 0.0f) return -1.0f;  // single-sided surface seen from behind: traversal continues past it
  return t;
}

// ------------------------------------------------------------ float-float
struct ff {
  float hi, lo;
};
__device__ __forceinline__ ff ff_two_sum(float a, float b) {
  float s = __fadd_rn(a, b);
  float bb = __fsub_rn(s, a);
  float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return {s, e};
}
__device__ __forceinline__ ff ff_quick(float a, float b) {
  float s = __fadd_rn(a, b);
  return {s, __fsub_rn(b, __fsub_rn(s, a))};
}
__device__ __forceinline__ ff ff_add(ff a, ff b) {
  ff s = ff_two_sum(a.hi, b.hi);
  float e = __fadd_rn(s.lo, __fadd_rn(a.lo, b.lo));
  return ff_quick(s.hi, e);
}
__device__ __forceinline__ ff ff_neg(ff a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ ff ff_sub(ff a, ff b) { return ff_add(a, ff_neg(b)); }
__device__ __forceinline__ ff ff_mul(ff a, ff b) {
  float p = __fmul_rn(a.hi, b.hi);
  float e = __fmaf_rn(a.hi, b.hi, -p);
  e = __fmaf_rn(a.hi, b.lo, e);
  e = __fmaf_rn(a.lo, b.hi, e);
  return ff_quick(p, e);
}
__device__ __forceinline__ ff ff_div(ff a, ff b) {
  float q1 = __fdiv_rn(a.hi, b.hi);
  ff r = ff_sub(a, ff_mul(b, {q1, 0.0f}));
  float q2 = __fdiv_rn(r.hi, b.hi);
  ff r2 = ff_sub(r, ff_mul(b, {q2, 0.0f}));
  float q3 = __fdiv_rn(r2.hi, b.hi);
  ff q = ff_quick(q1, q2);
  return ff_add(q, {q3, 0.0f});
}
__device__ __forceinline__ ff ff_from(float a) { return {a, 0.0f}; }

// Moller-Trumbore in float-float arithmetic: edge/offset vectors and
// products with fma error terms.  Writes t, u (weight of b), v (weight of c)
// rounded to f32.  Returns false when det is zero.
__device__ __forceinline__ bool ff_refine_core(const ff e1[3], const ff e2[3], const ff ao[3], const ff dd[3],
                                               float* t_out, float* u_out, float* v_out) {
  ff n[3] = {ff_sub(ff_mul(e1[1], e2[2]), ff_mul(e1[2], e2[1])),
             ff_sub(ff_mul(e1[2], e2[0]), ff_mul(e1[0], e2[2])),
             ff_sub(ff_mul(e1[0], e2[1]), ff_mul(e1[1], e2[0]))};
  ff det = ff_neg(ff_add(ff_add(ff_mul(dd[0], n[0]), ff_mul(dd[1], n[1])), ff_mul(dd[2], n[2])));
  if (det.hi == 0.0f) return false;
  ff dao[3] = {ff_sub(ff_mul(ao[1], dd[2]), ff_mul(ao[2], dd[1])),
               ff_sub(ff_mul(ao[2], dd[0]), ff_mul(ao[0], dd[2])),
               ff_sub(ff_mul(ao[0], dd[1]), ff_mul(ao[1], dd[0]))};
  ff un = ff_add(ff_add(ff_mul(e2[0], dao[0]), ff_mul(e2[1], dao[1])), ff_mul(e2[2], dao[2]));
  ff vn = ff_neg(ff_add(ff_add(ff_mul(e1[0], dao[0]), ff_mul(e1[1], dao[1])), ff_mul(e1[2], dao[2])));
  ff tn = ff_add(ff_add(ff_mul(ao[0], n[0]), ff_mul(ao[1], n[1])), ff_mul(ao[2], n[2]));
  ff u = ff_div(un, det), v = ff_div(vn, det), t = ff_div(tn, det);
  *t_out = __fadd_rn(t.hi, t.lo);
  *u_out = __fadd_rn(u.hi, u.lo);
  *v_out = __fadd_rn(v.hi, v.lo);
  return true;
}

// f32 ray and vertices: the edge and offset vectors are exact (two_sum).
__device__ __noinline__ bool ff_refine(const float3 O, const float3 D, const float3 A, const float3 B,
                                       const float3 C, float* t_out, float* u_out, float* v_out) {
  const float o[3] = {O.x, O.y, O.z}, d[3] = {D.x, D.y, D.z};
  const float a[3] = {A.x, A.y, A.z}, b[3] = {B.x, B.y, B.z}, c[3] = {C.x, C.y, C.z};
  ff e1[3], e2[3], ao[3], dd[3];
  for (int k = 0; k < 3; ++k) {
    e1[k] = ff_two_sum(b[k], -a[k]);
    e2[k] = ff_two_sum(c[k], -a[k]);
    ao[k] = ff_two_sum(o[k], -a[k]);
    dd[k] = ff_from(d[k]);
  }
  return ff_refine_core(e1, e2, ao, dd, t_out, u_out, v_out);
}

// rows of an affine 3x4 map applied to an f32 point in float-float: exact
// products (fma error terms) summed with two_sum.
__device__ __forceinline__ ff ff_affine_row(float4 m, float x, float y, float z) {
  return ff_add(ff_add(ff_mul(ff_from(m.x), ff_from(x)), ff_mul(ff_from(m.y), ff_from(y))),
                ff_add(ff_mul(ff_from(m.z), ff_from(z)), ff_from(m.w)));
}

// World-space refinement of a hit on an instanced triangle: the local
// vertices are carried to world space through the instance's local-to-world
// rows in float-float, so t, u, v are those of the placed triangle against the
// f32 world ray, free of the rounding of the f32 world-to-local transform.
__device__ __noinline__ bool ff_refine_placed(const float3 O, const float3 D, const float4 l0, const float4 l1,
                                              const float4 l2, const float3 A, const float3 B, const float3 C,
                                              float* t_out, float* u_out, float* v_out) {
  const float3 v[3] = {A, B, C};
  ff w[3][3];
  for (int i = 0; i < 3; ++i) {
    w[i][0] = ff_affine_row(l0, v[i].x, v[i].y, v[i].z);
    w[i][1] = ff_affine_row(l1, v[i].x, v[i].y, v[i].z);
    w[i][2] = ff_affine_row(l2, v[i].x, v[i].y, v[i].z);
  }
  const float o[3] = {O.x, O.y, O.z}, d[3] = {D.x, D.y, D.z};
  ff e1[3], e2[3], ao[3], dd[3];
  for (int k = 0; k < 3; ++k) {
    e1[k] = ff_sub(w[1][k], w[0][k]);
    e2[k] = ff_sub(w[2][k], w[0][k]);
    ao[k] = ff_sub(ff_from(o[k]), w[0][k]);
    dd[k] = ff_from(d[k]);
  }
  return ff_refine_core(e1, e2, ao, dd, t_out, u_out, v_out);
}

}  // namespace vt
