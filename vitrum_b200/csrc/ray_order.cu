// ray_order.cu -- spatial trace order: counting sort of a ray batch by
// (Morton code of the ray's entry point into the scene box, direction octant).
//
// Four launches: clear the buckets; one pass computes each ray's bucket and
// counts it (warp-aggregated: lanes with the same bucket add once); a two-
// kernel exclusive scan turns counts into cursors; a second pass scatters each
// ray's index to its cursor.  No ordering within a bucket is promised: the
// traversal's results do not depend on the order rays are traced in.
#include "ray_order.h"

#include <algorithm>

namespace vt {

namespace {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint32_t kScanBlock = 4096;  // bucket words per scan CTA (1024 threads x 4)

struct Quant {
  float lo[3], hi[3], sc[3];
  uint32_t bits;
};

// 10-bit value -> its bits at positions 0, 3, 6, ... (Morton interleave)
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Bucket of ray i: the point where the ray's [tmin, tmax] segment enters the
// box (its origin when it starts inside), quantised to 2^bits cells per axis,
// Morton-interleaved, times 8 plus the direction octant.  Rays whose segment
// misses the box share the last cell.
__device__ __forceinline__ uint32_t ray_bucket(const float4* __restrict__ rays, size_t i, const Quant& q) {
  const float4 r0 = __ldg(rays + 2 * i), r1 = __ldg(rays + 2 * i + 1);
  const float o[3] = {r0.x, r0.y, r0.z}, d[3] = {r1.x, r1.y, r1.z};
  float tn = r0.w, tf = r1.w;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float dk = fabsf(d[k]) > 1e-30f ? d[k] : copysignf(1e-30f, d[k]);
    const float inv = 1.0f / dk;
    const float t0 = (q.lo[k] - o[k]) * inv, t1 = (q.hi[k] - o[k]) * inv;
    tn = fmaxf(tn, fminf(t0, t1));
    tf = fminf(tf, fmaxf(t0, t1));
  }
  const uint32_t oct = (d[0] < 0.0f ? 4u : 0u) | (d[1] < 0.0f ? 2u : 0u) | (d[2] < 0.0f ? 1u : 0u);
  const uint32_t cmax = (1u << q.bits) - 1u;
  uint32_t c[3] = {cmax, cmax, cmax};
  if (tn <= tf) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float p = fmaf(d[k], tn, o[k]);
      // NaN falls to cell 0 (fmaxf returns the number)
      const float x = fminf(fmaxf((p - q.lo[k]) * q.sc[k], 0.0f), (float)cmax);
      c[k] = min((uint32_t)x, cmax);
    }
  }
  const uint32_t m = (spread3(c[0]) << 2) | (spread3(c[1]) << 1) | spread3(c[2]);
  return (m << 3) | oct;
}

__device__ __forceinline__ uint32_t ray_count(const RayOrderArgs& a) {
  const size_t n = a.n_dev ? min((size_t)*a.n_dev, a.n) : a.n;
  return (uint32_t)n;
}

__global__ void __launch_bounds__(256) k_ro_keys(RayOrderArgs a, Quant q) {
  const uint32_t n = ray_count(a);
  const uint32_t lane = threadIdx.x & 31u;
  const size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t stride = ((size_t)gridDim.x * blockDim.x) & ~(size_t)31;
  for (size_t base = warp * 32; base < n; base += stride) {
    const size_t i = base + lane;
    const bool valid = i < n;
    const uint32_t active = __ballot_sync(kFull, valid);
    if (!valid) continue;
    const uint32_t key = ray_bucket(a.rays, i, q);
    a.keys[i] = key;
    const uint32_t peers = __match_any_sync(active, key);
    if (lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(a.counts + key, (uint32_t)__popc(peers));
  }
}

__global__ void __launch_bounds__(256) k_ro_scatter(RayOrderArgs a) {
  const uint32_t n = ray_count(a);
  const uint32_t lane = threadIdx.x & 31u;
  const size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t stride = ((size_t)gridDim.x * blockDim.x) & ~(size_t)31;
  for (size_t base = warp * 32; base < n; base += stride) {
    const size_t i = base + lane;
    const bool valid = i < n;
    const uint32_t active = __ballot_sync(kFull, valid);
    if (!valid) continue;
    const uint32_t key = a.keys[i];
    const uint32_t peers = __match_any_sync(active, key);
    const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
    uint32_t slot = 0;
    if (lane == leader) slot = atomicAdd(a.counts + key, (uint32_t)__popc(peers));
    slot = __shfl_sync(peers, slot, leader) + (uint32_t)__popc(peers & ((1u << lane) - 1u));
    a.order[slot] = (uint32_t)i;
  }
}

// Exclusive scan of one CTA's 4096 bucket words in place; the CTA's total to sums.
__global__ void __launch_bounds__(1024) k_ro_scan_local(uint32_t* __restrict__ c, uint32_t nb,
                                                        uint32_t* __restrict__ sums) {
  __shared__ uint32_t ws[32];
  const uint32_t base = blockIdx.x * kScanBlock + threadIdx.x * 4u;
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  uint32_t v[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) v[j] = base + j < nb ? c[base + j] : 0u;
  const uint32_t s = v[0] + v[1] + v[2] + v[3];
  uint32_t incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  if (lane == 31) ws[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    uint32_t x = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    ws[lane] = x;
  }
  __syncthreads();
  uint32_t run = incl - s + (wid ? ws[wid - 1] : 0u);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (base + j < nb) c[base + j] = run;
    run += v[j];
  }
  if (threadIdx.x == blockDim.x - 1) sums[blockIdx.x] = run;
}

// Adds the totals of the CTAs before it to each CTA's 4096 words.
__global__ void __launch_bounds__(1024) k_ro_scan_add(uint32_t* __restrict__ c, uint32_t nb,
                                                      const uint32_t* __restrict__ sums) {
  if (blockIdx.x == 0) return;
  __shared__ uint32_t ws[32];
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  uint32_t part = 0;
  for (uint32_t b = threadIdx.x; b < blockIdx.x; b += blockDim.x) part += sums[b];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
  if (lane == 0) ws[wid] = part;
  __syncthreads();
  uint32_t off = 0;
#pragma unroll 4
  for (int w = 0; w < 32; ++w) off += ws[w];
  const uint32_t base = blockIdx.x * kScanBlock + threadIdx.x * 4u;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (base + j < nb) c[base + j] += off;
}

uint32_t bucket_count(int cell_bits) { return 1u << (3 * cell_bits + 3); }

}  // namespace

size_t ray_order_count_words(int cell_bits) {
  const int cb = std::min(std::max(cell_bits, 1), kRayOrderMaxCellBits);
  const uint32_t nb = bucket_count(cb);
  return nb + (nb + kScanBlock - 1) / kScanBlock;
}

void launch_ray_order(const RayOrderArgs& a, cudaStream_t s) {
  if (a.n == 0) return;
  const int cb = std::min(std::max(a.cell_bits, 1), kRayOrderMaxCellBits);
  const uint32_t nb = bucket_count(cb);
  const uint32_t nblk = (nb + kScanBlock - 1) / kScanBlock;
  Quant q;
  q.bits = (uint32_t)cb;
  for (int k = 0; k < 3; ++k) {
    q.lo[k] = a.lo[k];
    q.hi[k] = a.hi[k];
    const float ext = a.hi[k] - a.lo[k];
    q.sc[k] = ext > 0.0f ? (float)(1u << cb) / ext : 0.0f;
  }
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t grid = std::min<size_t>((size_t)std::max(sms, 1) * 8, (a.n + 255) / 256);
  cudaMemsetAsync(a.counts, 0, (size_t)nb * sizeof(uint32_t), s);
  RayOrderArgs k = a;
  k.cell_bits = cb;
  k_ro_keys<<<(unsigned)grid, 256, 0, s>>>(k, q);
  k_ro_scan_local<<<nblk, 1024, 0, s>>>(a.counts, nb, a.counts + nb);
  if (nblk > 1) k_ro_scan_add<<<nblk, 1024, 0, s>>>(a.counts, nb, a.counts + nb);
  k_ro_scatter<<<(unsigned)grid, 256, 0, s>>>(k);
}

}  // namespace vt
