// light_tree.cuh -- device selection of one light entry from the packed light
// tree (layout in light_tree.h): the reference's samplePackedLightTreeCPU bucket
// descent (packages/shared-samplers/src/lightTree.ts:938-1319) over an importance
// of the same quantity plus a receiver bound, in f32 with every operation
// rounded on its own (no contraction), so the bucket split follows the same
// arithmetic as the CPU oracle's restatement.
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

// cos(max(0, theta - theta_u)) for cos theta = c and the half-angle theta_u (cu, su)
__device__ __forceinline__ float bound_cos(float c, float cu, float su) {
  if (c >= cu) return 1.0f;
  const float s = __fsqrt_rn(fmaxf(0.0f, fsub(1.0f, fmul(c, c))));
  return fmaxf(-1.0f, fminf(1.0f, fadd(fmul(c, cu), fmul(s, su))));
}

// Importance of packed node `idx` for the point p with unit normal n (zero:
// none): the quantity of the reference's packedNodeImportanceUnchecked
// (lightTree.ts:1237-1319) -- power / max(dist^2 to the box, floor) times the
// orientation cone's taper at cos(max(0, theta - theta_u)) -- times the
// receiver bound cos(max(0, theta_i - theta_u)) on the shading cosine (Conty
// Estevez & Kulla 2018), theta_u the node's bounding-sphere half-angle.  It is
// evaluated directly, not in the reference's scale-safe log form: one
// reciprocal square root serves both bounds and the packed axis is unit (the
// build normalises it), about a fifth of the instructions.  Every operation
// is rounded on its own, as in the CPU oracle's restatement.
__device__ __forceinline__ float importance(const float* tree, uint32_t idx, float px, float py, float pz, float nx,
                                            float ny, float nz) {
  const float* n = tree + (size_t)idx * kFloatsPerNode;
  const float power = __ldg(n + 1);
  if (!(power > 0.0f)) return 0.0f;
  const float mnx = __ldg(n + 4), mny = __ldg(n + 5), mnz = __ldg(n + 6);
  const float mxx = __ldg(n + 7), mxy = __ldg(n + 8), mxz = __ldg(n + 9);
  const float ex = fmaxf(fmaxf(fsub(mnx, px), 0.0f), fsub(px, mxx));
  const float ey = fmaxf(fmaxf(fsub(mny, py), 0.0f), fsub(py, mxy));
  const float ez = fmaxf(fmaxf(fsub(mnz, pz), 0.0f), fsub(pz, mxz));
  const float d2 = fmaxf(dot3r(ex, ey, ez, ex, ey, ez), kDist2Floor);
  const float vx = fsub(px, fmul(0.5f, fadd(mnx, mxx)));
  const float vy = fsub(py, fmul(0.5f, fadd(mny, mxy)));
  const float vz = fsub(pz, fmul(0.5f, fadd(mnz, mxz)));
  const float hx = fmul(0.5f, fsub(mxx, mnx)), hy = fmul(0.5f, fsub(mxy, mny)), hz = fmul(0.5f, fsub(mxz, mnz));
  const float r2 = dot3r(hx, hy, hz, hx, hy, hz), l2 = dot3r(vx, vy, vz, vx, vy, vz);
  float w = 1.0f;
  if (l2 > r2 && l2 <= kF32Max) {  // p outside the bounding sphere
    const float inv = __frsqrt_rn(l2);
    const float su = fminf(1.0f, fmul(__fsqrt_rn(r2), inv));
    const float cu = __fsqrt_rn(fmaxf(0.0f, fsub(1.0f, fmul(su, su))));
    const float ax = __ldg(n + 10), ay = __ldg(n + 11), az = __ldg(n + 12);
    if (ax != 0.0f || ay != 0.0f || az != 0.0f) {
      const float ca = bound_cos(fmaxf(-1.0f, fminf(1.0f, fmul(dot3r(ax, ay, az, vx, vy, vz), inv))), cu, su);
      const float cos_o = __ldg(n + 13), cos_e = __ldg(n + 14);
      if (ca < cos_e) return 0.0f;
      if (ca < cos_o) {
        const float span = fsub(cos_o, cos_e);
        if (span > 0.0f) w = fmaxf(kF32MinNormal, fdiv(fsub(ca, cos_e), span));
      }
    }
    if (nx != 0.0f || ny != 0.0f || nz != 0.0f) {
      const float ci = bound_cos(fmaxf(-1.0f, fminf(1.0f, -fmul(dot3r(nx, ny, nz, vx, vy, vz), inv))), cu, su);
      if (!(ci > 0.0f)) return 0.0f;
      w = fmul(w, ci);
    }
  }
  const float imp = fdiv(fmul(power, w), d2);
  if (!(imp <= kF32Max)) return kF32Max;
  return fmaxf(kF32MinNormal, imp);
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
