// nrc_kernels.cu -- neural radiance cache kernels for sm_100a.
//
// k_nrc_infer   persistent, three CTAs per SM; per tile of 128 queries: encode
//               (hash grid + SH4 + surface features) into a swizzled fp16 tile, then six
//               tcgen05.mma layers (M=128, N=64, K=64 as four K=16 steps) with
//               the fp32 accumulator in TMEM, ReLU + fp16 repack in the epilogue
//               between layers, prediction read from TMEM.
// k_nrc_train   persistent; per tile: encode, forward keeping every layer's
//               activations in shared memory, relative-L2 output gradient,
//               backward: per layer dW += G^T X (tensor core, accumulated across
//               the CTA's tiles in TMEM) and dX = G W (tensor core), ReLU mask
//               from the stored activations; the input gradient of the 32
//               hash-grid features is scattered into the table gradient with the
//               trilinear weights (nrcEncoding.ts hashGridBackward:214).
// k_nrc_adam    Adam with the reference's non-finite guards and +-65504 clamp.
//
// Every mbarrier wait is bounded (about one second of clocks); on expiry the
// kernel records v.error, waits (bounded) for its issued MMAs, frees its TMEM
// and returns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "nrc.h"
#include "tc_sm100.cuh"

namespace vt {
namespace nrc {

namespace {

constexpr long long kWaitCycles = kDefaultWaitCycles;  // drains after an expired wait
constexpr uint32_t kTileBytes = kTile * kWidth * 2;   // 16 KB activation tile
constexpr uint32_t kWBytes = kWidth * kWidth * 2;      // 8 KB weight tile
constexpr uint32_t kIdesc = tc::idesc_f16(128, 64, false, false);     // X * W^T
constexpr uint32_t kIdescBwd = tc::idesc_f16(128, 64, false, true);   // G * W
constexpr uint32_t kIdescWgrad = tc::idesc_f16(128, 64, true, true);  // G^T * X (rows 64.. unused)

__device__ __forceinline__ uint32_t grid_hash(uint32_t x, uint32_t y, uint32_t z) {
  // Instant-NGP spatial hash, nrcEncoding.ts spatialHash3D:107-115 (x prime 1)
  return x ^ (y * 2654435761u) ^ (z * 805459861u);
}

__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float2 unpack_h2(uint32_t u) {
  const __half2 h = *reinterpret_cast<const __half2*>(&u);
  return __half22float2(h);
}

__device__ __forceinline__ void store_row(uint8_t* tile, uint32_t r, const uint32_t (&p)[32]) {
#pragma unroll
  for (int j = 0; j < 8; ++j)
    *reinterpret_cast<uint4*>(tile + tc::sw128_offset(r, 8 * j)) = make_uint4(p[4 * j], p[4 * j + 1], p[4 * j + 2],
                                                                               p[4 * j + 3]);
}
__device__ __forceinline__ void load_row(const uint8_t* tile, uint32_t r, uint32_t (&p)[32]) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint4 q = *reinterpret_cast<const uint4*>(tile + tc::sw128_offset(r, 8 * j));
    p[4 * j] = q.x; p[4 * j + 1] = q.y; p[4 * j + 2] = q.z; p[4 * j + 3] = q.w;
  }
}

// normalised position in [0,1]^3 (normalizeToAabb, nrcEncoding.ts:166-178)
__device__ __forceinline__ float3 normalise(const View& v, float px, float py, float pz) {
  return make_float3(fminf(1.0f, fmaxf(0.0f, (px - v.aabb_min[0]) * v.aabb_inv[0])),
                     fminf(1.0f, fmaxf(0.0f, (py - v.aabb_min[1]) * v.aabb_inv[1])),
                     fminf(1.0f, fmaxf(0.0f, (pz - v.aabb_min[2]) * v.aabb_inv[2])));
}

// Real spherical harmonics of degree 4 (bands 0..3, 16 values) of unit d.
__device__ __forceinline__ void sh4(float x, float y, float z, float (&s)[16]) {
  const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  s[0] = 0.28209479177387814f;
  s[1] = -0.48860251190291987f * y;
  s[2] = 0.48860251190291987f * z;
  s[3] = -0.48860251190291987f * x;
  s[4] = 1.0925484305920792f * xy;
  s[5] = -1.0925484305920792f * yz;
  s[6] = 0.94617469575755997f * zz - 0.31539156525251999f;
  s[7] = -1.0925484305920792f * xz;
  s[8] = 0.54627421529603959f * (xx - yy);
  s[9] = 0.59004358992664352f * y * (3.0f * xx - yy) * -1.0f;
  s[10] = 2.8906114426405538f * xy * z;
  s[11] = 0.45704579946446572f * y * (1.0f - 5.0f * zz);
  s[12] = 0.3731763325901154f * z * (5.0f * zz - 3.0f);
  s[13] = 0.45704579946446572f * x * (1.0f - 5.0f * zz);
  s[14] = 1.4453057213202769f * z * (xx - yy);
  s[15] = 0.59004358992664352f * x * (3.0f * yy - xx);
}

// Encodes one record (4 float4) into 64 fp16 inputs packed as 32 half2 words.
__device__ __forceinline__ void encode(const View& v, float4 a, float4 b, float4 c, float4 d, uint32_t (&p)[32],
                                       float3& n01) {
  n01 = normalise(v, a.x, a.y, a.z);
  // all levels unrolled: the 8 x levels table gathers are independent and in flight together
#pragma unroll
  for (int l = 0; l < kMaxLevels; ++l) {
    float f0 = 0.0f, f1 = 0.0f;
    if (l < v.levels) {
      const float N = v.res[l];
      const float px = n01.x * N, py = n01.y * N, pz = n01.z * N;
      const float x0 = floorf(px), y0 = floorf(py), z0 = floorf(pz);
      const float fx = px - x0, fy = py - y0, fz = pz - z0;
      const uint32_t ix = (uint32_t)(int)x0, iy = (uint32_t)(int)y0, iz = (uint32_t)(int)z0;
      const __half2* tab = v.table16 + (size_t)l * (v.table_mask + 1u);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t cx = k & 1, cy = (k >> 1) & 1, cz = (k >> 2) & 1;
        const float w = (cx ? fx : 1.0f - fx) * (cy ? fy : 1.0f - fy) * (cz ? fz : 1.0f - fz);
        const uint32_t row = grid_hash(ix + cx, iy + cy, iz + cz) & v.table_mask;
        const float2 e = __half22float2(__ldg(tab + row));
        f0 = fmaf(w, e.x, f0);
        f1 = fmaf(w, e.y, f1);
      }
    }
    p[l] = pack_h2(f0, f1);
  }
  float s[16];
  sh4(a.w, b.x, b.y, s);
#pragma unroll
  for (int k = 0; k < 8; ++k) p[16 + k] = pack_h2(s[2 * k], s[2 * k + 1]);
  // normal (b.z, b.w, c.x), roughness c.y, diffuse (c.z, c.w, d.x), specular (d.y, d.z, d.w), 1
  p[24] = pack_h2(b.z, b.w);
  p[25] = pack_h2(c.x, c.y);
  p[26] = pack_h2(c.z, c.w);
  p[27] = pack_h2(d.x, d.y);
  p[28] = pack_h2(d.z, d.w);
  p[29] = pack_h2(1.0f, 0.0f);
  p[30] = 0u;
  p[31] = 0u;
}

// Scatter of the hash-feature input gradient g[0..31] (already scaled) into
// the f32 table gradient with the trilinear weights.
__device__ __forceinline__ void scatter_table(const View& v, float3 n01, const float (&g)[kEncWidth]) {
#pragma unroll
  for (int l = 0; l < kMaxLevels; ++l) {
    const float g0 = g[2 * l], g1 = g[2 * l + 1];
    if (l >= v.levels || (g0 == 0.0f && g1 == 0.0f)) continue;
    const float N = v.res[l];
    const float px = n01.x * N, py = n01.y * N, pz = n01.z * N;
    const float x0 = floorf(px), y0 = floorf(py), z0 = floorf(pz);
    const float fx = px - x0, fy = py - y0, fz = pz - z0;
    const uint32_t ix = (uint32_t)(int)x0, iy = (uint32_t)(int)y0, iz = (uint32_t)(int)z0;
    float2* gt = v.grad_table + (size_t)l * (v.table_mask + 1u);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t cx = k & 1, cy = (k >> 1) & 1, cz = (k >> 2) & 1;
      const float w = (cx ? fx : 1.0f - fx) * (cy ? fy : 1.0f - fy) * (cz ? fz : 1.0f - fz);
      const uint32_t row = grid_hash(ix + cx, iy + cy, iz + cz) & v.table_mask;
      atomicAdd(gt + row, make_float2(w * g0, w * g1));
    }
  }
}

// Shared-memory carve-up (dynamic, aligned to 1024 at run time).
struct Smem {
  uint8_t* w;        // 6 weight tiles
  uint8_t* act;      // activation tiles
  uint64_t* bar;
  uint32_t* tmem_slot;
};

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  const uint32_t s = tc::smem_u32(p);
  return p + (((s + 1023u) & ~1023u) - s);
}

// Loads the six fp16 weight tiles (row-major [out][in]) into swizzled tiles.
__device__ __forceinline__ void load_weights(const View& v, uint8_t* w) {
  for (uint32_t q = threadIdx.x; q < (uint32_t)(kLayers * kWidth * 8); q += blockDim.x) {
    const uint32_t l = q / (kWidth * 8), r = (q / 8) % kWidth, j = q % 8;
    const uint4 val = __ldg(reinterpret_cast<const uint4*>(v.w16 + (size_t)l * kWidth * kWidth + r * kWidth) + j);
    *reinterpret_cast<uint4*>(w + l * kWBytes + tc::sw128_offset(r, 8 * j)) = val;
  }
}

// Issue one 128x64x64 product (four K=16 steps) and commit to the barrier.
__device__ __forceinline__ void issue_fwd(uint32_t tmem_d, uint32_t a_tile, uint32_t w_tile) {
  tc::fence_after_sync();
#pragma unroll
  for (uint32_t kk = 0; kk < 4; ++kk) tc::mma_f16(tmem_d, tc::desc_k(a_tile, kk), tc::desc_k(w_tile, kk), kIdesc, kk);
}

// Thread-uniform bounded wait on the barrier's current phase.
// On failure `phase` keeps the parity of the phase still pending.
__device__ __forceinline__ bool wait_all(const View& v, uint64_t* bar, uint32_t& phase) {
  const bool ok = __syncthreads_and(tc::mbar_wait(bar, phase, v.wait_cycles)) != 0;
  if (ok) phase ^= 1u;
  return ok;
}

// 64 fp32 accumulator columns of this thread's row (its TMEM lane)
__device__ __forceinline__ void load_acc64(uint32_t taddr, uint32_t (&v)[64]) {
  uint32_t (&a)[16] = *reinterpret_cast<uint32_t(*)[16]>(&v[0]);
  uint32_t (&b)[16] = *reinterpret_cast<uint32_t(*)[16]>(&v[16]);
  uint32_t (&c)[16] = *reinterpret_cast<uint32_t(*)[16]>(&v[32]);
  uint32_t (&d)[16] = *reinterpret_cast<uint32_t(*)[16]>(&v[48]);
  tc::tmem_ld16(taddr, a);
  tc::tmem_ld16(taddr + 16, b);
  tc::tmem_ld16(taddr + 32, c);
  tc::tmem_ld16(taddr + 48, d);
  tc::tmem_wait_ld();
}

// On a timed-out wait: flag, give the issued MMAs a bounded chance to finish.
__device__ void fail_and_drain(const View& v, uint64_t* bar, uint32_t phase) {
  if (threadIdx.x == 0) {
    atomicExch(v.error, 1);
    tc::mbar_wait(bar, phase, kWaitCycles);
  }
  __syncthreads();
}

// ---------------------------------------------------------------- inference
// Named barrier of warpgroup g (ids 1..T; 0 is __syncthreads): the 128 threads
// of one tile synchronise without waiting for the CTA's other tiles.
__device__ __forceinline__ void group_sync(uint32_t id) {
  asm volatile("barrier.cta.sync %0, 128;" ::"r"(id) : "memory");
}
__device__ __forceinline__ bool group_and(uint32_t id, bool p) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred a, b;\n\tsetp.ne.u32 a, %1, 0;\n\tbarrier.cta.red.and.pred b, %2, 128, a;\n\t"
      "selp.u32 %0, 1, 0, b;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)p), "r"(id)
      : "memory");
  return r != 0;
}

// T tiles of 128 queries in flight per CTA, one per warpgroup (the MLP tile
// knob): the warpgroups share the CTA's weight tiles and TMEM allocation (64
// columns each) and run independently -- each encodes its tile (16 levels x 8
// table gathers per query), issues its own MMA chain from its first thread and
// waits on its own mbarrier -- so one tile's gathers overlap another's MMAs.
template <int T>
__global__ void __launch_bounds__(128 * T, T == 1 ? 3 : (T == 2 ? 2 : 1))
    k_nrc_infer(View v, const float4* __restrict__ recs, uint32_t stride, const uint32_t* __restrict__ n_dev,
                uint32_t n_host, float* __restrict__ rgb, float4* __restrict__ radiance) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = align1024(smem_raw);
  uint8_t* wt = base;
  const uint32_t tid = threadIdx.x & 127u, warp = tid >> 5, g = threadIdx.x >> 7, gid = g + 1;
  // this warpgroup's tile: each layer's MMA has finished reading it before the
  // epilogue writes the next layer's input over it
  uint8_t* act = base + kLayers * kWBytes + g * kTileBytes;
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + kLayers * kWBytes + T * kTileBytes) + g;
  uint32_t* slot = reinterpret_cast<uint32_t*>(reinterpret_cast<uint64_t*>(base + kLayers * kWBytes + T * kTileBytes) + T);
  constexpr uint32_t kCols = T == 1 ? 64u : (T == 2 ? 128u : 256u);  // a power of two >= 64 T
  const uint32_t n = n_dev ? *n_dev : n_host;
  if ((uint32_t)blockIdx.x * T * kTile >= n) return;  // uniform per CTA: no tile, no TMEM
  if (threadIdx.x < 32) {
    tc::tmem_alloc(slot, kCols);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::fence_mbar_init();
  }
  load_weights(v, wt);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot + 64u * g;
  const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
  const uint32_t w_s = tc::smem_u32(wt), a_s = tc::smem_u32(act);
  uint32_t phase = 0;
  bool failed = false;
  for (uint32_t tile = blockIdx.x * T + g; tile * kTile < n && !failed; tile += gridDim.x * T) {
    const uint32_t i = tile * kTile + tid;
    const bool valid = i < n;
    uint32_t p[32];
    float3 n01;
    const float4* r = recs + (size_t)(valid ? i : 0) * stride;
    encode(v, __ldg(r), __ldg(r + 1), __ldg(r + 2), __ldg(r + 3), p, n01);
    store_row(act, tid, p);
    tc::fence_async_smem();
    tc::fence_before_sync();
    group_sync(gid);
    for (int l = 0; l < kLayers; ++l) {
      if (tid == 0) {
        issue_fwd(tmem, a_s, w_s + l * kWBytes);
        tc::mma_commit(bar);
      }
      // thread-uniform bounded wait (per warpgroup); on failure `phase` keeps the pending parity
      if (!group_and(gid, tc::mbar_wait(bar, phase, v.wait_cycles))) { failed = true; break; }
      phase ^= 1u;
      tc::fence_after_sync();
      if (l + 1 < kLayers) {
        uint32_t acc[64];
        load_acc64(lane_addr, acc);
#pragma unroll
        for (int k = 0; k < 32; ++k)
          p[k] = pack_h2(fmaxf(__uint_as_float(acc[2 * k]), 0.0f), fmaxf(__uint_as_float(acc[2 * k + 1]), 0.0f));
        store_row(act, tid, p);
        tc::fence_async_smem();
        tc::fence_before_sync();
        group_sync(gid);
      } else {
        uint32_t o[16];
        tc::tmem_ld16(lane_addr, o);
        tc::tmem_wait_ld();
        tc::fence_before_sync();
        if (valid) {
          const float r0 = __uint_as_float(o[0]), r1 = __uint_as_float(o[1]), r2 = __uint_as_float(o[2]);
          if (radiance) {
            const float4 e = __ldg(recs + (size_t)i * stride + 4);  // (path bits, throughput rgb)
            const uint32_t path = __float_as_uint(e.x);
            float4 acc = radiance[path];
            acc.x += e.y * fmaxf(r0, 0.0f);
            acc.y += e.z * fmaxf(r1, 0.0f);
            acc.z += e.w * fmaxf(r2, 0.0f);
            radiance[path] = acc;
          } else {
            rgb[3 * (size_t)i] = r0;
            rgb[3 * (size_t)i + 1] = r1;
            rgb[3 * (size_t)i + 2] = r2;
          }
        }
      }
    }
  }
  if (failed) {
    // flag, give the issued MMAs a bounded chance to finish
    if (tid == 0) {
      atomicExch(v.error, 1);
      tc::mbar_wait(bar, phase, kWaitCycles);
    }
    group_sync(gid);
  }
  __syncthreads();
  if (threadIdx.x < 32) tc::tmem_dealloc(*slot, kCols);
}

// ---------------------------------------------------------------- training
// Relative L2 on luminance (fusedMlp.wgsl.ts:62-110): per-sample gradient
// 2/3 (p - t) / (lum(p)^2 + 1e-2) with the stop-gradient luminance
// lum = clamp(sum w_c p_c / max|p|, -1, 1) * max|p|; the 1/N of the mean is
// applied in fp32 when the accumulated gradients leave TMEM (loss scaling by
// N keeps the fp16 deltas in range); deltas clamp at +-65504, NaN -> 0.
__device__ __forceinline__ float rel_l2_lum(float p0, float p1, float p2) {
  const float s = fmaxf(fabsf(p0), fmaxf(fabsf(p1), fabsf(p2)));
  if (!(s > 0.0f)) return 0.0f;
  const float nl = 0.299f * (p0 / s) + 0.587f * (p1 / s) + 0.114f * (p2 / s);
  return fminf(1.0f, fmaxf(-1.0f, nl)) * s;
}

__global__ void __launch_bounds__(128, 1)
    k_nrc_train(View v, const float4* __restrict__ samples, uint32_t n) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = align1024(smem_raw);
  uint8_t* wt = base;                             // 6 x 8 KB
  uint8_t* G = base + kLayers * kWBytes;          // gradient tile
  uint8_t* X = G + kTileBytes;                    // X[0] = encoded input, X[l] = H_l (l = 1..5)
  uint64_t* bar = reinterpret_cast<uint64_t*>(X + kLayers * kTileBytes);
  uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  if ((uint32_t)blockIdx.x * kTile >= n) return;
  if (warp == 0) {
    tc::tmem_alloc(slot, 512);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::fence_mbar_init();
  }
  load_weights(v, wt);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;
  const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
  const uint32_t w_s = tc::smem_u32(wt), g_s = tc::smem_u32(G), x_s = tc::smem_u32(X);
  const float inv_n = 1.0f / (float)n;
  uint32_t phase = 0;
  bool failed = false;
  uint32_t tiles = 0;
  float loss = 0.0f;
  for (uint32_t tile = blockIdx.x; tile * kTile < n && !failed; tile += gridDim.x, ++tiles) {
    const uint32_t i = tile * kTile + tid;
    const bool valid = i < n;
    uint32_t p[32];
    float3 n01;
    const float4* r = samples + (size_t)(valid ? i : 0) * 5;
    encode(v, __ldg(r), __ldg(r + 1), __ldg(r + 2), __ldg(r + 3), p, n01);
    const float4 tgt = __ldg(r + 4);
    store_row(X, tid, p);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    // ---- forward, keeping H_1..H_5
    float pr[3] = {0.0f, 0.0f, 0.0f};
    for (int l = 0; l < kLayers && !failed; ++l) {
      if (tid == 0) {
        issue_fwd(tmem, x_s + l * kTileBytes, w_s + l * kWBytes);
        tc::mma_commit(bar);
      }
      if (!wait_all(v, bar, phase)) { failed = true; break; }
      tc::fence_after_sync();
      if (l + 1 < kLayers) {
        uint32_t acc[64];
        load_acc64(lane_addr, acc);
#pragma unroll
        for (int k = 0; k < 32; ++k)
          p[k] = pack_h2(fmaxf(__uint_as_float(acc[2 * k]), 0.0f), fmaxf(__uint_as_float(acc[2 * k + 1]), 0.0f));
        store_row(X + (l + 1) * kTileBytes, tid, p);
        tc::fence_async_smem();
      } else {
        uint32_t o[16];
        tc::tmem_ld16(lane_addr, o);
        tc::tmem_wait_ld();
        pr[0] = __uint_as_float(o[0]);
        pr[1] = __uint_as_float(o[1]);
        pr[2] = __uint_as_float(o[2]);
      }
      tc::fence_before_sync();
      __syncthreads();
    }
    if (failed) break;
    // ---- output gradient
    float g[3] = {0.0f, 0.0f, 0.0f};
    if (valid) {
      const float t3[3] = {tgt.x, tgt.y, tgt.z};
      bool fin = isfinite(pr[0]) && isfinite(pr[1]) && isfinite(pr[2]) && isfinite(t3[0]) && isfinite(t3[1]) &&
                 isfinite(t3[2]);
      if (fin) {
        const float lum = fminf(fabsf(rel_l2_lum(pr[0], pr[1], pr[2])), 1e19f);
        const float den = lum * lum + 1e-2f;
        const float sc = 2.0f / 3.0f / den;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float dlt = pr[c] - t3[c];
          float raw = dlt * sc;
          if (isnan(raw)) raw = 0.0f;
          g[c] = fminf(65504.0f, fmaxf(-65504.0f, raw));
          loss += dlt * dlt / den / 3.0f;
        }
      }
    }
    if (valid && v.tile_stats && __float_as_uint(tgt.w) != 0u && isfinite(pr[0]) && isfinite(pr[1]) &&
        isfinite(pr[2])) {
      // cache error estimate of the sample's screen tile (prediction vs target luminance)
      const uint32_t pix = __float_as_uint(tgt.w) - 1u;
      const uint32_t tile = (pix / v.tile_width / v.tile_size) * v.tiles_x + (pix % v.tile_width) / v.tile_size;
      float* ts = v.tile_stats + 3 * (size_t)tile;
      atomicAdd(ts, 0.2126f * fmaxf(pr[0], 0.0f) + 0.7152f * fmaxf(pr[1], 0.0f) + 0.0722f * fmaxf(pr[2], 0.0f));
      atomicAdd(ts + 1, 0.2126f * tgt.x + 0.7152f * tgt.y + 0.0722f * tgt.z);
      atomicAdd(ts + 2, 1.0f);
    }
#pragma unroll
    for (int k = 0; k < 32; ++k) p[k] = 0u;
    p[0] = pack_h2(g[0], g[1]);
    p[1] = pack_h2(g[2], 0.0f);
    store_row(G, tid, p);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    // ---- backward: layer 5 (output) down to 0
    for (int l = kLayers - 1; l >= 0 && !failed; --l) {
      if (tid == 0) {
        tc::fence_after_sync();
        const uint32_t x_in = x_s + l * kTileBytes;  // this layer's input
        const uint32_t dw = tmem + 64u + 64u * (uint32_t)l;
#pragma unroll
        for (uint32_t kk = 0; kk < 8; ++kk)  // K = 128 samples
          tc::mma_f16(dw, tc::desc_mn(g_s, kk, kTileBytes), tc::desc_mn(x_in, kk, kTileBytes), kIdescWgrad,
                      (tiles > 0 || kk > 0) ? 1u : 0u);
#pragma unroll
        for (uint32_t kk = 0; kk < 4; ++kk)  // K = 64 outputs of this layer
          tc::mma_f16(tmem, tc::desc_k(g_s, kk), tc::desc_mn(w_s + l * kWBytes, kk, kWBytes), kIdescBwd, kk);
        tc::mma_commit(bar);
      }
      if (!wait_all(v, bar, phase)) { failed = true; break; }
      tc::fence_after_sync();
      uint32_t acc[64];
      load_acc64(lane_addr, acc);  // dX_l
      tc::fence_before_sync();
      if (l > 0) {
        // G_{l-1} = dH_l * (H_l > 0)
        uint32_t h[32];
        load_row(X + l * kTileBytes, tid, h);
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          const float2 hv = unpack_h2(h[k]);
          const float a0 = hv.x > 0.0f ? __uint_as_float(acc[2 * k]) : 0.0f;
          const float a1 = hv.y > 0.0f ? __uint_as_float(acc[2 * k + 1]) : 0.0f;
          p[k] = pack_h2(fminf(65504.0f, fmaxf(-65504.0f, a0)), fminf(65504.0f, fmaxf(-65504.0f, a1)));
        }
        store_row(G, tid, p);
        tc::fence_async_smem();
      } else if (valid) {
        float ge[kEncWidth];
#pragma unroll
        for (int k = 0; k < kEncWidth; ++k) ge[k] = __uint_as_float(acc[k]) * inv_n;
        scatter_table(v, n01, ge);
      }
      __syncthreads();
    }
  }
  if (failed) {
    fail_and_drain(v, bar, phase);
  } else if (tiles > 0 && warp < 2) {
    // weight gradients: rows 0..63 of each dW accumulator (lanes of warps 0, 1)
    tc::fence_after_sync();
    for (int l = 0; l < kLayers; ++l) {
      uint32_t acc[64];
      load_acc64(lane_addr + 64u + 64u * (uint32_t)l, acc);
      float* gw = v.grad_w + (size_t)l * kWidth * kWidth + (size_t)tid * kWidth;
#pragma unroll
      for (int k = 0; k < 64; ++k) atomicAdd(gw + k, __uint_as_float(acc[k]) * inv_n);
    }
  }
  // loss: warp reduce then one atomic per warp
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
  if ((tid & 31u) == 0 && v.loss) atomicAdd(v.loss, loss * inv_n);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------- Adam
__device__ __forceinline__ bool fin(float x) { return x == x && fabsf(x) <= 3.402823e38f; }

// ibc1 / ibc2: 1 / (1 - beta^t), rounded once on the host (a product per value instead of two divisions)
__device__ __forceinline__ float adam_one(float cur, float& m, float& vv, float g, float lr, float b1, float b2,
                                          float eps, float ibc1, float ibc2, int* diag) {
  if (!fin(cur) || !fin(m) || !fin(vv) || vv < 0.0f) {
    m = 0.0f;
    vv = 0.0f;
    if (diag) atomicAdd(diag, 1);
    return fin(cur) ? cur : 0.0f;
  }
  if (!fin(g)) {
    if (diag) atomicAdd(diag, 1);
    return cur;
  }
  const float mi = b1 * m + (1.0f - b1) * g;
  const float vi = b2 * vv + (1.0f - b2) * g * g;
  const float mh = mi * ibc1, vh = vi * ibc2;
  const float up = cur - lr * mh / (sqrtf(vh) + eps);
  if (!fin(up) || !fin(mi) || !fin(vi)) {
    if (diag) atomicAdd(diag, 1);
    return cur;
  }
  m = mi;
  vv = vi;
  return fminf(65504.0f, fmaxf(-65504.0f, up));
}

__global__ void k_nrc_adam(float* __restrict__ master, float* __restrict__ m, float* __restrict__ v,
                           float* __restrict__ grad, __half* __restrict__ out16, size_t count, float lr, float b1,
                           float b2, float eps, float ibc1, float ibc2, int* diag) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    float mm = m[i], vv = v[i];
    const float up = adam_one(master[i], mm, vv, grad[i], lr, b1, b2, eps, ibc1, ibc2, diag);
    master[i] = up;
    m[i] = mm;
    v[i] = vv;
    grad[i] = 0.0f;
    out16[i] = __float2half_rn(up);
  }
}

__global__ void k_nrc_adam_table(float2* __restrict__ master, float2* __restrict__ m, float2* __restrict__ v,
                                 float2* __restrict__ grad, __half2* __restrict__ out16, size_t pairs, float lr,
                                 float b1, float b2, float eps, float ibc1, float ibc2, int* diag) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += (size_t)gridDim.x * blockDim.x) {
    float2 w = master[i], mm = m[i], vv = v[i];
    const float2 g = grad[i];
    w.x = adam_one(w.x, mm.x, vv.x, g.x, lr, b1, b2, eps, ibc1, ibc2, diag);
    w.y = adam_one(w.y, mm.y, vv.y, g.y, lr, b1, b2, eps, ibc1, ibc2, diag);
    master[i] = w;
    m[i] = mm;
    v[i] = vv;
    grad[i] = make_float2(0.0f, 0.0f);
    out16[i] = __floats2half2_rn(w.x, w.y);
  }
}

constexpr size_t infer_smem(int t) { return kLayers * kWBytes + (size_t)t * kTileBytes + 64 + 1024; }
constexpr size_t kTrainSmem = kLayers * kWBytes + (1 + kLayers) * kTileBytes + 64 + 1024;

int sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

}  // namespace

void level_resolutions(const Config& c, float* out) {
  for (int l = 0; l < kMaxLevels; ++l) out[l] = (float)std::floor((double)c.base_resolution * std::pow((double)c.growth, l));
}

template <int T>
void launch_infer_t(const View& v, const float4* records, uint32_t rec_stride_f4, const uint32_t* n_dev, uint32_t n,
                    float* rgb_out, float4* radiance, cudaStream_t s) {
  static int per_sm = 0;
  if (!per_sm) {
    cudaFuncSetAttribute(k_nrc_infer<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)infer_smem(T));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_nrc_infer<T>, 128 * T, infer_smem(T));
    // TMEM: 512 columns per SM, 64 T (rounded up to a power of two) per CTA
    const int cols = T == 1 ? 64 : (T == 2 ? 128 : 256);
    per_sm = per_sm < 512 / cols ? per_sm : 512 / cols;
    if (per_sm < 1) per_sm = 1;
  }
  const uint32_t tiles = (n + kTile - 1) / kTile;
  const uint32_t ctas = (tiles + T - 1) / T;
  const uint32_t cap = (uint32_t)(per_sm * sm_count());
  k_nrc_infer<T><<<ctas < cap ? ctas : cap, 128 * T, infer_smem(T), s>>>(v, records, rec_stride_f4, n_dev, n, rgb_out,
                                                                          radiance);
}

void launch_infer(const View& v, const float4* records, uint32_t rec_stride_f4, const uint32_t* n_dev, uint32_t n,
                  float* rgb_out, float4* radiance, int tiles_per_cta, cudaStream_t s) {
  if (n == 0) return;
  // tiles in flight per CTA: 1 to 4 (65 to 113 KB of shared memory).  Under the default
  // carve-out one CTA runs per SM, which keeps most of the unified L1 for the hash-table gathers:
  // asking for the largest shared-memory carve-out (three or two CTAs per SM) made two tiles per
  // CTA slower (0.47 -> 0.82 ms for 1,048,576 queries)
  if (tiles_per_cta >= 4) launch_infer_t<4>(v, records, rec_stride_f4, n_dev, n, rgb_out, radiance, s);
  else if (tiles_per_cta == 3) launch_infer_t<3>(v, records, rec_stride_f4, n_dev, n, rgb_out, radiance, s);
  else if (tiles_per_cta == 2) launch_infer_t<2>(v, records, rec_stride_f4, n_dev, n, rgb_out, radiance, s);
  else launch_infer_t<1>(v, records, rec_stride_f4, n_dev, n, rgb_out, radiance, s);
}

void launch_train(const View& v, const float4* samples, uint32_t n, cudaStream_t s) {
  if (n == 0) return;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_nrc_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem);
    attr = true;
  }
  const uint32_t tiles = (n + kTile - 1) / kTile;
  const uint32_t grid = tiles < (uint32_t)sm_count() ? tiles : (uint32_t)sm_count();
  k_nrc_train<<<grid, 128, kTrainSmem, s>>>(v, samples, n);
}

void launch_adam(float* master, float* m, float* v, float* grad, __half* out16, size_t count, float lr, float beta1,
                 float beta2, float eps, float bc1, float bc2, int* diag, cudaStream_t s) {
  if (!count) return;
  const size_t g = (count + 255) / 256;
  k_nrc_adam<<<(unsigned)(g < 148 * 16 ? g : 148 * 16), 256, 0, s>>>(master, m, v, grad, out16, count, lr, beta1,
                                                                      beta2, eps, 1.0f / bc1, 1.0f / bc2, diag);
}

void launch_adam_table(float* master, float* m, float* v, float2* grad, __half2* out16, size_t pairs, float lr,
                       float beta1, float beta2, float eps, float bc1, float bc2, int* diag, cudaStream_t s) {
  if (!pairs) return;
  const size_t g = (pairs + 255) / 256;
  k_nrc_adam_table<<<(unsigned)(g < 148 * 16 ? g : 148 * 16), 256, 0, s>>>(
      reinterpret_cast<float2*>(master), reinterpret_cast<float2*>(m), reinterpret_cast<float2*>(v), grad, out16,
      pairs, lr, beta1, beta2, eps, 1.0f / bc1, 1.0f / bc2, diag);
}

}  // namespace nrc
}  // namespace vt
