// traverse.cu -- closest-hit and any-hit traversal of the 8-wide compressed BVH.
//
// One thread per ray.  Per wide node: five 128-bit read-only loads, the
// eight quantised child slabs tested against [tmin, closest] in the ray's
// octant order, internal-child hits kept as an 8-bit group mask and leaf
// hits as a 32-bit triangle mask (Ylitie et al. 2017 node groups).  The
// group stack lives in shared memory, one column per thread.  Triangles use
// the reference's watertight f32 test (tri_intersect.cuh); the accepted hit
// is then re-evaluated once in float-float arithmetic for the reported t
// and barycentrics.
//
// Slab conservativeness: a child plane at p + q*2^e is evaluated as
// fma(q, 2^e*invd, (p - o)*invd); the rounding error of that expression is
// below 8u*|invd|*(|p| + 255*2^e + |o|) (u = 2^-24), so the near distance
// is lowered and the far distance raised by that amount.  Together with
// outward quantisation this never culls a box the exact ray touches.
#include <cuda_runtime.h>

#include <cstdint>

#include "bvh_types.h"
#include "traverse.h"
#include "tri_intersect.cuh"

namespace vt {

namespace {

constexpr int kBlock = 128;

__device__ __forceinline__ float u8f(uint32_t word, uint32_t sel) {
  // byte `sel` of `word` as a float, via the 2^23 mantissa trick
  return __uint_as_float(__byte_perm(word, 0x4B000000u, 0x7540u | sel)) - 8388608.0f;
}

struct Slab {
  float adj, on, of;  // q scale, near offset, far offset
};

__device__ __forceinline__ Slab make_slab(float p, float e_bits, float inv, float o) {
  float s = e_bits;                 // 2^e
  float adj = s * inv;
  float org = (p - o) * inv;
  float err = 4.76837158203125e-7f * fabsf(inv) * (fabsf(p) + 255.0f * s + fabsf(o));  // 8u
  Slab r;
  r.adj = adj;
  r.on = org - err;
  r.of = org + err;
  return r;
}

template <bool ANY, int STK>
__global__ void __launch_bounds__(kBlock) k_trace(const uint4* __restrict__ nodes, const float4* __restrict__ tris,
                                                  const float4* __restrict__ rays, size_t n,
                                                  int4* __restrict__ hits, uint8_t* __restrict__ occluded,
                                                  int* __restrict__ status) {
  extern __shared__ uint2 stack_mem[];  // [STK][kBlock], one column per thread
  uint2* const stack = stack_mem + threadIdx.x;
  const size_t ray = (size_t)blockIdx.x * kBlock + threadIdx.x;
  if (ray >= n) return;
  const float4 r0 = __ldg(rays + 2 * ray);
  const float4 r1 = __ldg(rays + 2 * ray + 1);
  const float tmin = r0.w;
  float closest = r1.w;
  const WtRay wr = wt_setup(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);

  auto safe = [](float d) { return fabsf(d) > 1e-30f ? d : copysignf(1e-30f, d); };
  const float ix = __frcp_rn(safe(r1.x)), iy = __frcp_rn(safe(r1.y)), iz = __frcp_rn(safe(r1.z));
  const bool nx = ix < 0.0f, ny = iy < 0.0f, nz = iz < 0.0f;
  const uint32_t oct = (nx ? 4u : 0u) | (ny ? 2u : 0u) | (nz ? 1u : 0u);

  int best = -1;
  float best_t = closest, best_u = 0.0f, best_v = 0.0f;
  bool done = false;

  // current internal-node group: base index, key-ordered hit bits (0..7), imask
  uint32_t gbase = 0, ghits = 0, gimask = 0;
  uint32_t tbase = 0, thits = 0;
  int sp = 0;
  uint32_t node = 0;

  while (true) {
    // ---- expand `node`
    {
      const uint4* np = nodes + (size_t)node * 5;
      const uint4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
      const uint32_t e = w0.w;
      const Slab sx = make_slab(__uint_as_float(w0.x), __uint_as_float((e & 0xFFu) << 23), ix, r0.x);
      const Slab sy = make_slab(__uint_as_float(w0.y), __uint_as_float(((e >> 8) & 0xFFu) << 23), iy, r0.y);
      const Slab sz = make_slab(__uint_as_float(w0.z), __uint_as_float(((e >> 16) & 0xFFu) << 23), iz, r0.z);
      const uint32_t imask = e >> 24;
      // q words: lo_x = w2.xy, lo_y = w2.zw, lo_z = w3.xy, hi_x = w3.zw, hi_y = w4.xy, hi_z = w4.zw
      const uint32_t nx0 = nx ? w3.z : w2.x, nx1 = nx ? w3.w : w2.y;
      const uint32_t fx0 = nx ? w2.x : w3.z, fx1 = nx ? w2.y : w3.w;
      const uint32_t ny0 = ny ? w4.x : w2.z, ny1 = ny ? w4.y : w2.w;
      const uint32_t fy0 = ny ? w2.z : w4.x, fy1 = ny ? w2.w : w4.y;
      const uint32_t nz0 = nz ? w4.z : w3.x, nz1 = nz ? w4.w : w3.y;
      const uint32_t fz0 = nz ? w3.x : w4.z, fz1 = nz ? w3.y : w4.w;
      uint32_t nh = 0, th = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t sel = (uint32_t)(j & 3);
        const float qnx = u8f(j < 4 ? nx0 : nx1, sel), qfx = u8f(j < 4 ? fx0 : fx1, sel);
        const float qny = u8f(j < 4 ? ny0 : ny1, sel), qfy = u8f(j < 4 ? fy0 : fy1, sel);
        const float qnz = u8f(j < 4 ? nz0 : nz1, sel), qfz = u8f(j < 4 ? fz0 : fz1, sel);
        const float tn = fmaxf(fmaxf(fmaf(qnx, sx.adj, sx.on), fmaf(qny, sy.adj, sy.on)),
                               fmaxf(fmaf(qnz, sz.adj, sz.on), tmin));
        const float tf = fminf(fminf(fmaf(qfx, sx.adj, sx.of), fmaf(qfy, sy.adj, sy.of)),
                               fminf(fmaf(qfz, sz.adj, sz.of), closest));
        if (tn <= tf) {
          if ((imask >> j) & 1u) {
            nh |= 1u << ((uint32_t)j ^ oct);
          } else {
            const uint32_t m = ((j < 4 ? w1.z : w1.w) >> (8 * (j & 3))) & 0xFFu;
            th |= ((1u << (m >> 5)) - 1u) << (m & 31u);
          }
        }
      }
      gbase = w1.x;
      ghits = nh;
      gimask = imask;
      tbase = w1.y;
      thits = th;
    }
    // ---- triangles of the expanded node
    while (thits) {
      const uint32_t k = (uint32_t)(__ffs(thits) - 1);
      thits &= thits - 1;
      const uint32_t tri = tbase + k;
      const float4 a = __ldg(tris + 3 * (size_t)tri), b = __ldg(tris + 3 * (size_t)tri + 1),
                   c = __ldg(tris + 3 * (size_t)tri + 2);
      WtHit h;
      if (wt_intersect(wr, make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z), make_float3(c.x, c.y, c.z),
                       tmin, &h) &&
          h.t < closest) {
        closest = h.t;
        best = (int)tri;
        best_t = h.t;
        best_u = h.bary[1];
        best_v = h.bary[2];
        if (ANY) { done = true; break; }
      }
    }
    if (ANY && done) break;
    // ---- next node: current group, else the stack
    while (ghits == 0) {
      if (sp == 0) break;
      --sp;
      const uint2 g = stack[sp * kBlock];
      gbase = g.x;
      ghits = g.y & 0xFFu;
      gimask = g.y >> 8;
    }
    if (ghits == 0) break;
    const uint32_t k = (uint32_t)(__ffs(ghits) - 1);
    ghits &= ghits - 1;
    const uint32_t slot = k ^ oct;
    node = gbase + __popc(gimask & ((1u << slot) - 1u));
    if (ghits) {
      if (sp < STK) {
        stack[sp * kBlock] = make_uint2(gbase, ghits | (gimask << 8));
        ++sp;
      } else {
        atomicOr(status, 1);  // stack capacity exceeded: result incomplete, reported to the host
      }
    }
  }

  if (ANY) {
    occluded[ray] = (uint8_t)(best >= 0 ? 1 : 0);
    return;
  }
  int4 out;
  if (best >= 0) {
    const float4 a = __ldg(tris + 3 * (size_t)best), b = __ldg(tris + 3 * (size_t)best + 1),
                 c = __ldg(tris + 3 * (size_t)best + 2);
    float t, u, v;
    if (ff_refine(make_float3(r0.x, r0.y, r0.z), make_float3(r1.x, r1.y, r1.z), make_float3(a.x, a.y, a.z),
                  make_float3(b.x, b.y, b.z), make_float3(c.x, c.y, c.z), &t, &u, &v)) {
      best_t = t;
      best_u = u;
      best_v = v;
    }
    out = make_int4((int)__float_as_uint(a.w), __float_as_int(best_t), __float_as_int(best_u), __float_as_int(best_v));
  } else {
    out = make_int4(-1, __float_as_int(r1.w), 0, 0);
  }
  hits[ray] = out;
}

__global__ void k_watertight_eval(const float* __restrict__ cases, size_t n, vt_watertight_result* out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* c = cases + 16 * i;
  WtRay r = wt_setup(c[0], c[1], c[2], c[3], c[4], c[5]);
  WtHit h;
  vt_watertight_result res;
  res.hit = wt_intersect(r, make_float3(c[6], c[7], c[8]), make_float3(c[9], c[10], c[11]),
                         make_float3(c[12], c[13], c[14]), c[15], &h)
                ? 1
                : 0;
  res.t = res.hit ? h.t : CUDART_INF_F;
  res.bary[0] = res.hit ? h.bary[0] : 0.0f;
  res.bary[1] = res.hit ? h.bary[1] : 0.0f;
  res.bary[2] = res.hit ? h.bary[2] : 0.0f;
  res.side = res.hit ? h.side : 0;
  res.zero_edge_mask = res.hit ? h.mask : 0;
  out[i] = res;
}

template <bool ANY, int STK>
void launch_stk(const TraceArgs& a, unsigned grid, cudaStream_t s) {
  const size_t smem = sizeof(uint2) * STK * kBlock;
  if (smem > 48 * 1024)  // opt-in above the default 48 KB dynamic limit
    cudaFuncSetAttribute(k_trace<ANY, STK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_trace<ANY, STK><<<grid, kBlock, smem, s>>>(a.nodes, a.tris, a.rays, a.n, a.hits, a.occluded, a.status);
}

template <bool ANY>
void launch_trace_t(const TraceArgs& a, cudaStream_t s) {
  const unsigned grid = (unsigned)((a.n + kBlock - 1) / kBlock);
  if (grid == 0) return;
  if (a.stack_depth <= 16) launch_stk<ANY, 16>(a, grid, s);
  else if (a.stack_depth <= 32) launch_stk<ANY, 32>(a, grid, s);
  else launch_stk<ANY, 64>(a, grid, s);
}

}  // namespace

void launch_trace_closest(const TraceArgs& a, cudaStream_t s) { launch_trace_t<false>(a, s); }
void launch_trace_any(const TraceArgs& a, cudaStream_t s) { launch_trace_t<true>(a, s); }

void launch_watertight_eval(const float* cases, size_t n, vt_watertight_result* out, cudaStream_t s) {
  if (n == 0) return;
  k_watertight_eval<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(cases, n, out);
}

}  // namespace vt
