// light_tree.cuh -- device selection of one light entry from the packed light
// tree (layout in light_tree.h), the reference's samplePackedLightTreeCPU /
// packedNodeImportanceUnchecked (packages/shared-samplers/src/lightTree.ts:938-1319)
// in f32 with every operation rounded on its own (no contraction), so the
// bucket split follows the same arithmetic as the CPU oracle.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "light_tree.h"

namespace vt {
namespace lt {

constexpr float kF32Max = 3.40282346638528859812e38f;
constexpr float kF32MinNormal = 1.17549435082228750797e-38f;

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float dot3r(float ax, float ay, float az, float bx, float by, float bz) {
  return fadd(fadd(fmul(ax, bx), fmul(ay, by)), fmul(az, bz));
}
__device__ __forceinline__ float max3abs(float a, float b, float c) {
  return fmaxf(fabsf(a), fmaxf(fabsf(b), fabsf(c)));
}

// squared distance from p to the box, scale-safe (packedDist2ToAabbCPU)
__device__ __forceinline__ float dist2_box(float px, float py, float pz, const float* b) {
  const float hx = fmaxf(fmaxf(fsub(fmul(0.5f, b[0]), fmul(0.5f, px)), 0.0f), fsub(fmul(0.5f, px), fmul(0.5f, b[3])));
  const float hy = fmaxf(fmaxf(fsub(fmul(0.5f, b[1]), fmul(0.5f, py)), 0.0f), fsub(fmul(0.5f, py), fmul(0.5f, b[4])));
  const float hz = fmaxf(fmaxf(fsub(fmul(0.5f, b[2]), fmul(0.5f, pz)), 0.0f), fsub(fmul(0.5f, pz), fmul(0.5f, b[5])));
  const float hs = max3abs(hx, hy, hz);
  if (!(hs >= kF32MinNormal)) return 0.0f;
  if (hs > fmul(0.5f, kF32Max)) return kF32Max;
  const float sx = fdiv(hx, hs), sy = fdiv(hy, hs), sz = fdiv(hz, hs);
  const float ss = dot3r(sx, sy, sz, sx, sy, sz);
  const float s = fmul(2.0f, hs);
  const float lim = __fsqrt_rn(fdiv(kF32Max, ss));
  if (s >= lim) return kF32Max;
  return fminf(kF32Max, fmul(fmul(s, s), ss));
}

// orientation-cone factor (packedConeFactorCPU): 1 inside the normal cone, a
// cosine-space taper to the emission bound, 0 beyond it
__device__ __forceinline__ float cone_factor(const float* n, float px, float py, float pz) {
  const float axs = max3abs(n[10], n[11], n[12]);
  if (!(axs > 0.0f) || axs > kF32Max) return 1.0f;
  const float ax = fdiv(n[10], axs), ay = fdiv(n[11], axs), az = fdiv(n[12], axs);
  const float al = __fsqrt_rn(dot3r(ax, ay, az, ax, ay, az));
  const float* mn = n + 4;
  const float* mx = n + 7;
  const float dvx = fsub(fsub(fmul(0.5f, px), fmul(0.25f, mn[0])), fmul(0.25f, mx[0]));
  const float dvy = fsub(fsub(fmul(0.5f, py), fmul(0.25f, mn[1])), fmul(0.25f, mx[1]));
  const float dvz = fsub(fsub(fmul(0.5f, pz), fmul(0.25f, mn[2])), fmul(0.25f, mx[2]));
  const float rx = fsub(fmul(0.25f, mx[0]), fmul(0.25f, mn[0]));
  const float ry = fsub(fmul(0.25f, mx[1]), fmul(0.25f, mn[1]));
  const float rz = fsub(fmul(0.25f, mx[2]), fmul(0.25f, mn[2]));
  const float ds = max3abs(dvx, dvy, dvz);
  if (!(ds >= kF32MinNormal) || ds > kF32Max) return 1.0f;
  const float sdx = fdiv(dvx, ds), sdy = fdiv(dvy, ds), sdz = fdiv(dvz, ds);
  const float sdl = __fsqrt_rn(dot3r(sdx, sdy, sdz, sdx, sdy, sdz));
  const float rs = max3abs(rx, ry, rz);
  float r_over_d = 0.0f;
  if (rs >= kF32MinNormal) {
    const float srx = fdiv(rx, rs), sry = fdiv(ry, rs), srz = fdiv(rz, rs);
    const float srl = __fsqrt_rn(dot3r(srx, sry, srz, srx, sry, srz));
    const float lr = fsub(fsub(fadd(log2f(rs), log2f(srl)), log2f(ds)), log2f(sdl));
    if (lr >= 0.0f) return 1.0f;
    r_over_d = exp2f(fmaxf(lr, -126.0f));
  }
  const float dx = fdiv(sdx, sdl), dy = fdiv(sdy, sdl), dz = fdiv(sdz, sdl);
  const float nx = fdiv(ax, al), ny = fdiv(ay, al), nz = fdiv(az, al);
  const float ct = fmaxf(-1.0f, fminf(1.0f, dot3r(nx, ny, nz, dx, dy, dz)));
  const float stu = fmaxf(0.0f, fminf(1.0f, r_over_d));
  const float ctu = __fsqrt_rn(fmaxf(0.0f, fsub(1.0f, fmul(stu, stu))));
  float ca = 1.0f;
  if (ct < ctu) {
    const float st = __fsqrt_rn(fmaxf(0.0f, fsub(1.0f, fmul(ct, ct))));
    ca = fmaxf(-1.0f, fminf(1.0f, fadd(fmul(ct, ctu), fmul(st, stu))));
  }
  if (ca < n[14]) return 0.0f;
  if (ca >= n[13]) return 1.0f;
  const float span = fsub(n[13], n[14]);
  if (!(span > 0.0f)) return 1.0f;
  return fmaxf(kF32MinNormal, fminf(1.0f, fdiv(fsub(ca, n[14]), span)));
}

// Receiver term (Conty Estevez & Kulla 2018's bound on the shading point's
// cosine): cos(max(0, theta_i - theta_u)) of the node seen from p above the
// plane of the unit normal (nx, ny, nz), theta_u the node's angular radius; 0
// when the node lies wholly below that plane, 1 for a zero normal
// (transmissive surfaces) or p inside the node's bounding sphere.
__device__ __forceinline__ float receiver_factor(const float* n, float px, float py, float pz, float nx, float ny,
                                                 float nz) {
  if (nx == 0.0f && ny == 0.0f && nz == 0.0f) return 1.0f;
  const float* mn = n + 4;
  const float* mx = n + 7;
  const float dvx = fsub(fadd(fmul(0.25f, mn[0]), fmul(0.25f, mx[0])), fmul(0.5f, px));
  const float dvy = fsub(fadd(fmul(0.25f, mn[1]), fmul(0.25f, mx[1])), fmul(0.5f, py));
  const float dvz = fsub(fadd(fmul(0.25f, mn[2]), fmul(0.25f, mx[2])), fmul(0.5f, pz));
  const float rx = fsub(fmul(0.25f, mx[0]), fmul(0.25f, mn[0]));
  const float ry = fsub(fmul(0.25f, mx[1]), fmul(0.25f, mn[1]));
  const float rz = fsub(fmul(0.25f, mx[2]), fmul(0.25f, mn[2]));
  const float ds = max3abs(dvx, dvy, dvz);
  if (!(ds >= kF32MinNormal) || ds > kF32Max) return 1.0f;
  const float sdx = fdiv(dvx, ds), sdy = fdiv(dvy, ds), sdz = fdiv(dvz, ds);
  const float sdl = __fsqrt_rn(dot3r(sdx, sdy, sdz, sdx, sdy, sdz));
  const float rs = max3abs(rx, ry, rz);
  float r_over_d = 0.0f;
  if (rs >= kF32MinNormal) {
    const float srx = fdiv(rx, rs), sry = fdiv(ry, rs), srz = fdiv(rz, rs);
    const float srl = __fsqrt_rn(dot3r(srx, sry, srz, srx, sry, srz));
    const float lr = fsub(fsub(fadd(log2f(rs), log2f(srl)), log2f(ds)), log2f(sdl));
    if (lr >= 0.0f) return 1.0f;
    r_over_d = exp2f(fmaxf(lr, -126.0f));
  }
  const float dx = fdiv(sdx, sdl), dy = fdiv(sdy, sdl), dz = fdiv(sdz, sdl);
  const float ct = fmaxf(-1.0f, fminf(1.0f, dot3r(nx, ny, nz, dx, dy, dz)));
  const float stu = fmaxf(0.0f, fminf(1.0f, r_over_d));
  const float ctu = __fsqrt_rn(fmaxf(0.0f, fsub(1.0f, fmul(stu, stu))));
  float ca = 1.0f;
  if (ct < ctu) {
    const float st = __fsqrt_rn(fmaxf(0.0f, fsub(1.0f, fmul(ct, ct))));
    ca = fmaxf(-1.0f, fminf(1.0f, fadd(fmul(ct, ctu), fmul(st, stu))));
  }
  return ca > 0.0f ? ca : 0.0f;
}

// importance of packed node `idx` for the point p (packedNodeImportanceUnchecked),
// times the receiver term for the normal n
__device__ __forceinline__ float importance(const float* tree, uint32_t idx, float px, float py, float pz, float nx,
                                            float ny, float nz) {
  const float* n = tree + (size_t)idx * kFloatsPerNode;
  const float power = n[1];
  if (!(power > 0.0f)) return 0.0f;
  const float d2 = fmaxf(fmaxf(dist2_box(px, py, pz, n + 4), kDist2Floor), kF32MinNormal);
  const float cone = cone_factor(n, px, py, pz);
  if (!(cone > 0.0f)) return 0.0f;
  const float recv = receiver_factor(n, px, py, pz, nx, ny, nz);
  if (!(recv > 0.0f)) return 0.0f;
  const float li = fadd(fsub(log2f(power), log2f(d2)), log2f(fmaxf(fmul(cone, recv), kF32MinNormal)));
  if (li >= 127.99999f) return kF32Max;
  if (li <= -126.0f) return kF32MinNormal;
  return fmaxf(kF32MinNormal, fminf(kF32Max, exp2f(li)));
}

// buckets of the current interval that go to the left child (allocateLeftBuckets)
__device__ __forceinline__ uint32_t left_buckets(uint32_t cur, uint32_t ll, uint32_t rl, float a, float b,
                                                 uint32_t reserve) {
  ll *= reserve;
  rl *= reserve;
  const uint32_t remaining = cur - (ll + rl);
  float p_left = 0.5f;
  if (!(a == 0.0f && b == 0.0f)) {
    const float s = fmaxf(a, b);
    const float l = fdiv(a, s), r = fdiv(b, s);
    p_left = fdiv(l, fadd(l, r));
  }
  const float ideal = fmul((float)remaining, p_left);
  const float extra = floorf(fadd(ideal, 0.5f));
  const uint32_t e = extra <= 0.0f ? 0u : (uint32_t)fminf(extra, (float)remaining);
  return ll + (e > remaining ? remaining : e);
}

// Buckets of the 2^24 draw given to the distant entries (directionals, the
// environment): n_dist / (n_dist + 1) of them, all when nothing is positional.
__device__ __forceinline__ uint32_t distant_buckets(uint32_t n_pos, uint32_t n_dist) {
  if (n_dist == 0) return 0u;
  if (n_pos == 0) return kBuckets;
  return (uint32_t)(((unsigned long long)kBuckets * n_dist) / (n_dist + 1u));
}

// One light entry for the point p with unit normal n (zero: no receiver term)
// from the 24-bit draw `bucket` (< 2^24): writes the entry and returns its
// selection probability (bucket count / 2^24).
// Entries 0 .. n_pos - 1 are positional and chosen by descending `tree` (the
// reference's bucket descent, started with the buckets the distant entries
// leave; nullptr: a single positional entry); entries n_pos .. are distant and
// share their buckets evenly.
__device__ __noinline__ float select(const float* tree, uint32_t n_pos, uint32_t n_dist, float px, float py, float pz,
                                     float nx, float ny, float nz, uint32_t bucket, uint32_t& entry) {
  const uint32_t D = distant_buckets(n_pos, n_dist);
  if (bucket < D) {
    const uint32_t j = (uint32_t)(((unsigned long long)bucket * n_dist) / D);
    // buckets b with floor(b n_dist / D) = j: [ceil(j D / n_dist), ceil((j + 1) D / n_dist))
    const unsigned long long lo = ((unsigned long long)j * D + n_dist - 1u) / n_dist;
    const unsigned long long hi = ((unsigned long long)(j + 1u) * D + n_dist - 1u) / n_dist;
    entry = n_pos + j;
    return (float)(hi - lo) * (1.0f / (float)kBuckets);
  }
  bucket -= D;
  uint32_t node = 0, cur = kBuckets - D;
  if (!tree) {
    entry = 0;
    return (float)cur * (1.0f / (float)kBuckets);
  }
  // defensive half: every leaf keeps (buckets / 2) / leaves of the tree's
  // buckets, the rest follows the importance (the reference keeps one bucket
  // per leaf, which lets a light the importance underrates near an occluded
  // bright neighbour be drawn with probability ~2^-24)
  uint32_t reserve = cur / (2u * (uint32_t)tree[15]);
  if (reserve < 1u) reserve = 1u;
  for (int guard = 0; guard < 64; ++guard) {
    const float* n = tree + (size_t)node * kFloatsPerNode;
    if (n[2] < 0.0f) {
      entry = (uint32_t)n[0];
      return (float)cur * (1.0f / (float)kBuckets);
    }
    const uint32_t l = (uint32_t)n[2], r = (uint32_t)n[3];
    const uint32_t lb = left_buckets(cur, (uint32_t)tree[(size_t)l * kFloatsPerNode + 15],
                                     (uint32_t)tree[(size_t)r * kFloatsPerNode + 15],
                                     importance(tree, l, px, py, pz, nx, ny, nz),
                                     importance(tree, r, px, py, pz, nx, ny, nz), reserve);
    if (bucket < lb) {
      cur = lb;
      node = l;
    } else {
      bucket -= lb;
      cur -= lb;
      node = r;
    }
  }
  entry = 0xFFFFFFFFu;  // deeper than any tree the host builds
  return 0.0f;
}

}  // namespace lt
}  // namespace vt
