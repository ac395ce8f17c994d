// light_tree.cuh -- device selection of one light entry from the packed light
// tree (layout in light_tree.h): the reference's samplePackedLightTreeCPU bucket
// descent (packages/shared-samplers/src/lightTree.ts:938-1319) over an importance
// of the same quantity plus a receiver bound.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "light_tree.h"

namespace vt {
namespace lt {

constexpr float kF32Max = 3.40282346638528859812e38f;
constexpr float kF32MinNormal = 1.17549435082228750797e-38f;


// sqrt(x) for x >= 0 through the hardware reciprocal square root (0 at 0)
__device__ __forceinline__ float fast_sqrt(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }

// cos(max(0, theta - theta_u)) for cos theta = c and the half-angle theta_u (cu, su)
__device__ __forceinline__ float bound_cos(float c, float cu, float su) {
  if (c >= cu) return 1.0f;
  const float s = fast_sqrt(fmaxf(0.0f, 1.0f - c * c));
  return fmaxf(-1.0f, fminf(1.0f, c * cu + s * su));
}

// Importance of packed node `idx` for the point p with unit normal n (zero:
// none): the quantity of the reference's packedNodeImportanceUnchecked
// (lightTree.ts:1237-1319) -- power / max(dist^2 to the box, floor) times the
// orientation cone's taper at cos(max(0, theta - theta_u)) -- times the
// receiver bound cos(max(0, theta_i - theta_u)) on the shading cosine (Conty
// Estevez & Kulla 2018), theta_u the node's bounding-sphere half-angle.  It is
// evaluated directly (one reciprocal square root serves both bounds, the
// packed axis is unit) with the hardware's approximate square roots and
// divisions: the selection and the probability it returns come from this one
// function, so the estimator is exact whatever the rounding; against the CPU
// oracle's correctly rounded restatement a split moves by a few of the 2^24
// buckets at most.
__device__ __forceinline__ float importance(const float* tree, uint32_t idx, float px, float py, float pz, float nx,
                                            float ny, float nz) {
  const float* n = tree + (size_t)idx * kFloatsPerNode;
  const float power = __ldg(n + 1);
  if (!(power > 0.0f)) return 0.0f;
  const float mnx = __ldg(n + 4), mny = __ldg(n + 5), mnz = __ldg(n + 6);
  const float mxx = __ldg(n + 7), mxy = __ldg(n + 8), mxz = __ldg(n + 9);
  const float ex = fmaxf(fmaxf(mnx - px, 0.0f), px - mxx);
  const float ey = fmaxf(fmaxf(mny - py, 0.0f), py - mxy);
  const float ez = fmaxf(fmaxf(mnz - pz, 0.0f), pz - mxz);
  const float d2 = fmaxf(ex * ex + ey * ey + ez * ez, kDist2Floor);
  const float vx = px - 0.5f * (mnx + mxx), vy = py - 0.5f * (mny + mxy), vz = pz - 0.5f * (mnz + mxz);
  const float hx = 0.5f * (mxx - mnx), hy = 0.5f * (mxy - mny), hz = 0.5f * (mxz - mnz);
  const float r2 = hx * hx + hy * hy + hz * hz, l2 = vx * vx + vy * vy + vz * vz;
  float w = 1.0f;
  if (l2 > r2 && l2 <= kF32Max) {  // p outside the bounding sphere
    const float inv = rsqrtf(l2);
    const float su = fminf(1.0f, fast_sqrt(r2) * inv);
    const float cu = fast_sqrt(fmaxf(0.0f, 1.0f - su * su));
    const float ax = __ldg(n + 10), ay = __ldg(n + 11), az = __ldg(n + 12);
    if (ax != 0.0f || ay != 0.0f || az != 0.0f) {
      const float ca = bound_cos(fmaxf(-1.0f, fminf(1.0f, (ax * vx + ay * vy + az * vz) * inv)), cu, su);
      const float cos_o = __ldg(n + 13), cos_e = __ldg(n + 14);
      if (ca < cos_e) return 0.0f;
      if (ca < cos_o) {
        const float span = cos_o - cos_e;
        if (span > 0.0f) w = fmaxf(kF32MinNormal, __fdividef(ca - cos_e, span));
      }
    }
    if (nx != 0.0f || ny != 0.0f || nz != 0.0f) {
      const float ci = bound_cos(fmaxf(-1.0f, fminf(1.0f, -(nx * vx + ny * vy + nz * vz) * inv)), cu, su);
      if (!(ci > 0.0f)) return 0.0f;
      w *= ci;
    }
  }
  // power * w / d2 (d2 >= the floor; __fdividef is exact enough below 2^126)
  const float imp = d2 < 1e37f ? __fdividef(power * w, d2) : (power * w) / d2;
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
    if (fmaxf(a, b) > 1e37f) {  // keep a + b and the approximate division in range
      a *= 0x1p-64f;
      b *= 0x1p-64f;
    }
    p_left = __fdividef(a, a + b);
  }
  const float ideal = (float)remaining * p_left;
  const float extra = floorf(ideal + 0.5f);
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
