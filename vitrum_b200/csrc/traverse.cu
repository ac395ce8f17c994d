// traverse.cu -- closest-hit and any-hit traversal of the 8-wide compressed BVH.
//
// One thread per ray.  Per wide node: five 128-bit read-only loads, the
// eight quantised child slabs tested against [tmin, closest] in the ray's
// octant order, internal-child hits kept as an 8-bit group mask and leaf
// hits as a 32-bit triangle mask (Ylitie et al. 2017 node groups).  The
// group stack is a per-thread local array (L1-cached where touched).  Triangles use
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

#include <algorithm>
#include <cstdint>

#include "bvh_types.h"
#include "traverse.h"
#include "tc_sm100.cuh"
#include "tri_intersect.cuh"

namespace vt {

namespace {

constexpr int kBlock = 128;
// Group-stack entries a ray can use: the launcher passes the tree's bound
// (two per wide level plus a few; 18 for an 8-level tree), capped here; a tree
// that needs more reports kTraceStackOverflow.  A shared-memory stack sized to
// that bound traced 1.9 % slower on the box room and 4 % slower on the
// instanced cloud than this local-memory one (shared memory taken from L1).
constexpr int kMaxStack = 64;
// Breadth-first prefix of the tree below `root` that every CTA copies into
// shared memory at start when staging is on: the root and its children and
// grandchildren of a full 8-wide tree (1 + 8 + 64), 5840 bytes.
constexpr uint32_t kHotNodes = 73;
constexpr long long kStagingWaitCycles = 2000000000LL;  // about a second

__device__ __forceinline__ uint64_t pack2(float a, float b) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
// three-input f32 max / min (sm_100)
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float lo32(uint64_t v) { return __uint_as_float((uint32_t)v); }
__device__ __forceinline__ float hi32(uint64_t v) { return __uint_as_float((uint32_t)(v >> 32)); }
// (near, far) t of one axis: bytes `sel` of the near / far words as floats (2^23
// mantissa trick, packed subtraction), then one packed FMA with (adj, adj) and (on, of)
__device__ __forceinline__ uint64_t slab2(uint32_t nw, uint32_t fw, uint32_t sel, uint64_t adj2, uint64_t off2) {
  const uint32_t a = __byte_perm(nw, 0x4B000000u, 0x7540u | sel), b = __byte_perm(fw, 0x4B000000u, 0x7540u | sel);
  uint64_t q, t;
  const uint64_t m = 0x4B0000004B000000ull;  // 2^23, 2^23
  asm("mov.b64 %0, {%1, %2};" : "=l"(q) : "r"(a), "r"(b));
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(q) : "l"(q), "l"(m));
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(t) : "l"(q), "l"(adj2), "l"(off2));
  return t;
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

// Per-lane ray state of the persistent kernel.
struct LaneRay {
  float tmin, closest;
  float ix, iy, iz;
  uint32_t oct;
  int best;  // triangle record index of the closest hit so far
};

// Per-ray traversal constants for origin o and direction d (world ray, or an
// instance's local ray: d is not renormalised, so t is the same in both).  The
// origin and direction are kept once, in the watertight test's state.
__device__ __forceinline__ void set_ray(LaneRay& R, WtRay& wr, float ox, float oy, float oz, float dx, float dy,
                                        float dz) {
  auto safe = [](float d) { return fabsf(d) > 1e-30f ? d : copysignf(1e-30f, d); };
  R.ix = __frcp_rn(safe(dx)); R.iy = __frcp_rn(safe(dy)); R.iz = __frcp_rn(safe(dz));
  R.oct = (R.ix < 0.0f ? 4u : 0u) | (R.iy < 0.0f ? 2u : 0u) | (R.iz < 0.0f ? 1u : 0u);
  wr = wt_setup(ox, oy, oz, dx, dy, dz);
}

// Reorders an 8-bit slot mask into key order: bit s moves to bit s ^ oct.
__device__ __forceinline__ uint32_t xor_permute8(uint32_t m, uint32_t oct) {
  if (oct & 1u) m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
  if (oct & 2u) m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
  if (oct & 4u) m = ((m & 0x0Fu) << 4) | ((m >> 4) & 0x0Fu);
  return m;
}

// Spreads bit s of an 8-bit mask to nibble s (0xF) of a 32-bit word.
__device__ __forceinline__ uint32_t nibble_spread8(uint32_t m) {
  m = (m | (m << 12)) & 0x000F000Fu;
  m = (m | (m << 6)) & 0x03030303u;
  m = (m | (m << 3)) & 0x11111111u;
  return m * 15u;
}

// Resident CTAs per SM the register budget is cut for: 8 (64 registers, some
// L1-cached spills) for single-level trees, 6 (80 registers) for two-level
// scenes, whose instance state spills several times more at 64 -- measured:
// box room 4 % faster at 8, instanced cloud 7 % slower at 8.
template <bool TWO>
constexpr int trace_min_blocks() { return TWO ? 6 : 8; }

// Watertight tests per loop iteration, at most.  Measured (B200, CUDA events):
// single-level trees one (box room 512^2 x 64 spp frame 30.7 -> 28.5 ms, its
// closest-hit traces 18.5 -> 16.4 ms; the 1,048,576-ray query 1.25 -> 1.19 ms;
// three: 31.1 ms and 1.41 ms), two-level scenes two (the instanced cloud's
// frame 30.6 ms against 30.7 with one and 32.0 with three).
template <bool TWO>
__host__ __device__ constexpr int tri_per_step() { return TWO ? 2 : 1; }

template <bool ANY, bool TWO, bool HOT>
__global__ void __launch_bounds__(kBlock, trace_min_blocks<TWO>())
    k_trace(const uint4* __restrict__ nodes, const float4* __restrict__ tris,
                                                  const float4* __restrict__ rays, size_t n,
                                                  int4* __restrict__ hits, uint8_t* __restrict__ occluded,
                                                  int* __restrict__ status,
                                                  unsigned long long* __restrict__ ray_counter,
                                                  const uint32_t* __restrict__ n_dev,
                                                  const float4* __restrict__ insts, uint32_t root,
                                                  const uint32_t* __restrict__ roots, uint32_t hot_count,
                                                  int stk, long long stage_wait,
                                                  const uint32_t* __restrict__ order,
                                                  const float4* __restrict__ inst_table) {
  // Persistent warps, one ray per lane.  Every iteration each live lane
  // (1) expands at most one wide node, (2) runs at most tri_per_step()
  // watertight triangle tests from a two-entry queue of triangle groups, and (3) picks
  // its next node without waiting for its queued triangles.  Node work and
  // triangle work therefore proceed in lock-step phases with most lanes
  // busy in each, and a lane whose ray finished takes the next unclaimed
  // ray from its warp's pool (one atomicAdd per 16 rays).
  // The group stack is a per-thread local array: the hardware interleaves it
  // across the warp, it is cached in L1 only where it is touched (rays rarely
  // go deep), and no shared memory is reserved for it, so the SM keeps its
  // largest L1 for nodes and triangle records.  `stk` <= kMaxStack entries are
  // used.  Dynamic shared memory holds only the hot_count staged nodes (80
  // bytes each) starting at nodes[root].
  extern __shared__ __align__(16) uint4 hot_mem[];
  __shared__ uint64_t hot_bar;
  uint2 stack[kMaxStack];
  const uint4* const hot = hot_mem;
  uint32_t hot_n = hot_count;  // staged nodes this CTA reads from shared memory
  if (HOT && hot_count) {
    // one bulk copy (TMA engine, no multicast) into shared memory, completed
    // on an mbarrier by transaction bytes
    if (threadIdx.x == 0) {
      const uint32_t bar = tc::smem_u32(&hot_bar), bytes = hot_count * 80u;
      tc::mbar_init(&hot_bar, 1);
      tc::fence_mbar_init();
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                   ::"r"(tc::smem_u32(hot)), "l"(nodes + (size_t)root * 5), "r"(bytes), "r"(bar)
                   : "memory");
    }
    __syncthreads();
    if (!tc::mbar_wait(&hot_bar, 0, stage_wait)) {
      // report, let a late copy land (full limit) so nothing writes this
      // CTA's shared memory after it, and traverse from global memory: the
      // results stay complete, the host reads the status bit
      atomicOr(status, kTraceStagingWait);
      tc::mbar_wait(&hot_bar, 0, kStagingWaitCycles);
      hot_n = 0;
    }
  }
  const uint32_t lane = threadIdx.x & 31u;
  constexpr uint32_t kFull = 0xFFFFFFFFu;
  // stack entry tags in x: bit 31 node group, bit 30 instance group, both: return
  // marker of an instance (two-level only); neither: triangle group
  constexpr uint32_t kNodeGroup = 0x80000000u;
  constexpr uint32_t kInstGroup = 0x40000000u;
  constexpr uint32_t kTagMask = 0xC0000000u;
  // rays per pool refill: small enough to spread short launches over all warps
  // (two-level: 16), 32 for single-level trees (box room 0.8 % faster than 16)
  constexpr uint32_t kChunk = TWO ? 16 : 32;

  bool live = false, exhausted = false;
  uint32_t ray = 0, pool_next = 0, pool_end = 0;
  const uint32_t n32 = n_dev ? *n_dev : (uint32_t)n;
  LaneRay R;
  WtRay wr;
  float wox = 0.f, woy = 0.f, woz = 0.f, wdx = 0.f, wdy = 0.f, wdz = 0.f;  // world ray (two-level)
  int cur_inst = -1, best_inst = -1;
  uint32_t cur_flags = 0;  // material flags of the instance being traversed (two-level)
  uint32_t gbase = 0, ghits = 0, gimask = 0, node = 0;
  uint32_t q0b = 0, q0m = 0, q1b = 0, q1m = 0;  // triangle-group queue (base, hit mask)
  bool expand = false;
  int sp = 0;

  while (true) {
    // ---- refill idle lanes from the warp's ray pool
    const uint32_t idle = __ballot_sync(kFull, !live);
    if (idle) {
      if (pool_next >= pool_end && !exhausted) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(ray_counter, (unsigned long long)kChunk);
        base = __shfl_sync(kFull, base, 0);
        pool_next = (uint32_t)(base < n32 ? base : n32);
        pool_end = base + kChunk < n32 ? (uint32_t)(base + kChunk) : n32;
        exhausted = base + kChunk >= n32;
      }
      const uint32_t avail = pool_end > pool_next ? pool_end - pool_next : 0u;
      const uint32_t rank = __popc(idle & ((1u << lane) - 1u));
      if (!live && rank < avail) {
        ray = pool_next + rank;
        if (order) ray = __ldg(order + ray);  // trace order differs from queue order
        const float4 r0 = __ldg(rays + 2 * (size_t)ray), r1 = __ldg(rays + 2 * (size_t)ray + 1);
        R.tmin = r0.w;
        R.closest = r1.w;
        set_ray(R, wr, r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
        if (TWO) { wox = r0.x; woy = r0.y; woz = r0.z; wdx = r1.x; wdy = r1.y; wdz = r1.z; }
        cur_inst = best_inst = -1;
        cur_flags = 0;
        R.best = -1;
        gbase = ghits = gimask = 0;
        q0m = q1m = 0;
        node = roots ? __ldg(roots + ray) : root;
        expand = true;
        sp = 0;
        live = true;
      }
      const uint32_t cnt = (uint32_t)__popc(idle);
      pool_next += avail < cnt ? avail : cnt;
      if (exhausted && pool_next >= pool_end && __ballot_sync(kFull, live) == 0) break;
    }
    if (!live) continue;

    // ---- (1) expand one node
    if (expand) {
      expand = false;
      const uint4* np = nodes + (size_t)node * 5;
      uint4 w0, w1, w2, w3, w4;
      if (HOT) {
        // staged prefix from shared memory, the rest from global (one generic load path)
        const uint32_t hrel = node - root;
        if (hrel < hot_n) np = hot + hrel * 5;
        w0 = np[0]; w1 = np[1]; w2 = np[2]; w3 = np[3]; w4 = np[4];
      } else {
        w0 = __ldg(np); w1 = __ldg(np + 1); w2 = __ldg(np + 2); w3 = __ldg(np + 3); w4 = __ldg(np + 4);
      }
      const uint32_t e = w0.w;
      const Slab sx = make_slab(__uint_as_float(w0.x), __uint_as_float((e & 0xFFu) << 23), R.ix, wr.o[0]);
      const Slab sy = make_slab(__uint_as_float(w0.y), __uint_as_float(((e >> 8) & 0xFFu) << 23), R.iy, wr.o[1]);
      const Slab sz = make_slab(__uint_as_float(w0.z), __uint_as_float(((e >> 16) & 0xFFu) << 23), R.iz, wr.o[2]);
      const uint32_t imask = e >> 24;
      const bool nx = R.oct & 4u, ny = R.oct & 2u, nz = R.oct & 1u;
      // q words: lo_x = w2.xy, lo_y = w2.zw, lo_z = w3.xy, hi_x = w3.zw, hi_y = w4.xy, hi_z = w4.zw
      const uint32_t nx0 = nx ? w3.z : w2.x, nx1 = nx ? w3.w : w2.y;
      const uint32_t fx0 = nx ? w2.x : w3.z, fx1 = nx ? w2.y : w3.w;
      const uint32_t ny0 = ny ? w4.x : w2.z, ny1 = ny ? w4.y : w2.w;
      const uint32_t fy0 = ny ? w2.z : w4.x, fy1 = ny ? w2.w : w4.y;
      const uint32_t nz0 = nz ? w4.z : w3.x, nz1 = nz ? w4.w : w3.y;
      const uint32_t fz0 = nz ? w3.x : w4.z, fz1 = nz ? w3.y : w4.w;
      const uint64_t ax2 = pack2(sx.adj, sx.adj), ay2 = pack2(sy.adj, sy.adj), az2 = pack2(sz.adj, sz.adj);
      const uint64_t ox2 = pack2(sx.on, sx.of), oy2 = pack2(sy.on, sy.of), oz2 = pack2(sz.on, sz.of);
      uint32_t hm = 0;  // slot-indexed hit mask
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t sel = (uint32_t)(j & 3);
        // near and far plane of one axis as one packed f32x2 conversion and FMA
        const uint64_t tx = slab2(j < 4 ? nx0 : nx1, j < 4 ? fx0 : fx1, sel, ax2, ox2);
        const uint64_t ty = slab2(j < 4 ? ny0 : ny1, j < 4 ? fy0 : fy1, sel, ay2, oy2);
        const uint64_t tz = slab2(j < 4 ? nz0 : nz1, j < 4 ? fz0 : fz1, sel, az2, oz2);
        const float tn = max3f(lo32(tx), lo32(ty), fmaxf(lo32(tz), R.tmin));
        const float tf = min3f(hi32(tx), hi32(ty), fminf(hi32(tz), R.closest));
        hm |= (tn <= tf) ? (1u << j) : 0u;
      }
      const uint32_t nh = xor_permute8(hm & imask, R.oct);
      uint32_t th = nibble_spread8(hm & ~imask) & w1.z;
      gbase = w1.x;
      ghits = nh;
      gimask = imask;
      if (TWO && cur_inst < 0 && th) {
        // top level: the leaf records are instances, entered through the stack
        // before this node's internal children (which wait below them)
        if (ghits) {
          if (sp < stk) {
            stack[sp] = make_uint2(gbase | kNodeGroup, ghits | (gimask << 8));
            ++sp;
          } else {
            atomicOr(status, kTraceStackOverflow);
          }
          ghits = 0;
        }
        if (sp < stk) {
          stack[sp] = make_uint2(w1.y | kInstGroup, th);
          ++sp;
        } else {
          atomicOr(status, kTraceStackOverflow);
        }
        th = 0;
      }
      if (th) {
        if (q0m == 0) { q0b = w1.y; q0m = th; }
        else if (q1m == 0) { q1b = w1.y; q1m = th; }
        else if (sp < stk) { stack[sp] = make_uint2(w1.y, th); ++sp; }
        else {
          // no room anywhere: test the group now (correct, only slower)
          while (th) {
            const uint32_t tri = w1.y + (uint32_t)(__ffs(th) - 1);
            th &= th - 1;
            const float4* rec = tris + 4 * (size_t)tri;
            const float4 a = __ldg(rec), b = __ldg(rec + 1), c = __ldg(rec + 2);
            const uint32_t fl = __float_as_uint(c.w) | cur_flags;
            if (ANY && (fl & VT_MATERIAL_NO_SHADOW)) continue;
            const float t = wt_candidate(wr, make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z),
                                         make_float3(c.x, c.y, c.z), R.tmin, R.closest,
                                         [rec] { return __ldg(rec + 3); }, (fl & VT_MATERIAL_SINGLE_SIDED) != 0);
            if (t >= 0.0f) { R.closest = t; R.best = (int)tri; best_inst = cur_inst; }
          }
        }
      }
    }

    // ---- (2) triangle tests from the queue head: one per iteration for
    // single-level trees, two for two-level scenes (see kTriPerStep)
    bool done = false;
#pragma unroll 1
    for (int rep = 0; rep < tri_per_step<TWO>(); ++rep) {
      if (q0m == 0) break;
      const uint32_t tri = q0b + (uint32_t)(__ffs(q0m) - 1);
      q0m &= q0m - 1;
      if (q0m == 0) { q0b = q1b; q0m = q1m; q1m = 0; }
      const float4* rec = tris + 4 * (size_t)tri;
      const float4 a = __ldg(rec), b = __ldg(rec + 1), c = __ldg(rec + 2);
      const uint32_t fl = __float_as_uint(c.w) | cur_flags;
      if (ANY && (fl & VT_MATERIAL_NO_SHADOW)) continue;
      const float t = wt_candidate(wr, make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z),
                                   make_float3(c.x, c.y, c.z), R.tmin, R.closest, [rec] { return __ldg(rec + 3); },
                                   (fl & VT_MATERIAL_SINGLE_SIDED) != 0);
      if (t >= 0.0f) {
        R.closest = t;
        R.best = (int)tri;
        best_inst = cur_inst;
        if (ANY) { done = true; break; }
      }
    }

    // ---- (3) next node: current group, else the stack (triangle groups join the queue)
    if (!done && !expand) {
      while (true) {
        if (ghits) {
          const uint32_t k = (uint32_t)(__ffs(ghits) - 1);
          ghits &= ghits - 1;
          const uint32_t slot = k ^ R.oct;
          node = gbase + __popc(gimask & ((1u << slot) - 1u));
          expand = true;
          if (ghits) {
            if (sp < stk) {
              stack[sp] = make_uint2(gbase | kNodeGroup, ghits | (gimask << 8));
              ++sp;
            } else {
              atomicOr(status, kTraceStackOverflow);  // stack capacity exceeded: result incomplete, reported to the host
            }
            ghits = 0;
          }
          break;
        }
        if (sp == 0) break;
        const uint2 g = stack[sp - 1];
        const uint32_t tag = g.x & kTagMask;
        if (TWO && tag == kTagMask) {
          // return marker: leave the instance once its queued triangles are tested
          if (q0m != 0) break;
          --sp;
          set_ray(R, wr, wox, woy, woz, wdx, wdy, wdz);
          cur_inst = -1;
          cur_flags = 0;
        } else if (TWO && tag == kInstGroup) {
          // enter the next instance of the group
          --sp;
          const uint32_t k = (uint32_t)(__ffs(g.y) - 1);
          const uint32_t rest = g.y & (g.y - 1);
          if (rest) { stack[sp] = make_uint2(g.x, rest); ++sp; }
          if (sp < stk) {
            stack[sp] = make_uint2(kTagMask, 0u);
            ++sp;
            const float4* ir = insts + 4 * (size_t)((g.x & ~kTagMask) + k);
            const float4 m0 = __ldg(ir), m1 = __ldg(ir + 1), m2 = __ldg(ir + 2);
            const uint4 meta = __ldg(reinterpret_cast<const uint4*>(ir + 3));
            const float lox = fmaf(m0.x, wox, fmaf(m0.y, woy, fmaf(m0.z, woz, m0.w)));
            const float loy = fmaf(m1.x, wox, fmaf(m1.y, woy, fmaf(m1.z, woz, m1.w)));
            const float loz = fmaf(m2.x, wox, fmaf(m2.y, woy, fmaf(m2.z, woz, m2.w)));
            const float ldx = fmaf(m0.x, wdx, fmaf(m0.y, wdy, m0.z * wdz));
            const float ldy = fmaf(m1.x, wdx, fmaf(m1.y, wdy, m1.z * wdz));
            const float ldz = fmaf(m2.x, wdx, fmaf(m2.y, wdy, m2.z * wdz));
            set_ray(R, wr, lox, loy, loz, ldx, ldy, ldz);
            cur_inst = (int)meta.y;
            cur_flags = meta.w;
            node = meta.x;
            expand = true;
            break;
          } else {
            atomicOr(status, kTraceStackOverflow);
          }
        } else if (tag == kNodeGroup) {
          --sp;
          gbase = g.x & ~kNodeGroup;
          ghits = g.y & 0xFFu;
          gimask = g.y >> 8;
        } else if (q1m == 0) {
          --sp;
          if (q0m == 0) { q0b = g.x; q0m = g.y; } else { q1b = g.x; q1m = g.y; }
        } else {
          break;  // queue full: test triangles first
        }
      }
      if (!expand && q0m == 0 && sp == 0) done = true;
    }
    if (!done) continue;

    // ---- ray finished: write its record, the lane is refilled next iteration
    live = false;
    if (ANY) {
      occluded[ray] = (uint8_t)(R.best >= 0 ? 1 : 0);
      continue;
    }
    // closest: (triangle record, watertight t, instance, material id); the
    // material lets shading skip the record -> material load.  k_refine_hits
    // turns the record into (source id, t, u, v) in a coalesced pass with every
    // lane busy
    int mat = -1;
    if (R.best >= 0)
      mat = (TWO && best_inst >= 0 && inst_table) ? __float_as_int(__ldg(inst_table + 4 * (size_t)best_inst + 3).z)
                                                  : __float_as_int(__ldg(tris + 4 * (size_t)R.best + 1).w);
    hits[ray] = make_int4(R.best, __float_as_int(R.closest), best_inst, mat);
  }
}

// Second pass of the closest-hit query: one thread per ray, float-float
// re-evaluation of the chosen triangle for t and barycentrics, record index
// replaced by the source triangle id (-1 and tmax for a miss).  Instance hits
// are re-evaluated in world space (the placed triangle against the world ray).
__global__ void __launch_bounds__(256) k_refine_hits(const float4* __restrict__ tris,
                                                      const float4* __restrict__ rays, size_t n,
                                                      int4* __restrict__ hits, const float4* __restrict__ inst_table,
                                                      const float4* __restrict__ inst_l2w,
                                                      int* __restrict__ inst_out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 h = hits[i];
  if (inst_out) inst_out[i] = h.x < 0 ? -1 : h.z;
  if (h.x < 0) {
    hits[i] = make_int4(-1, h.y, 0, 0);
    return;
  }
  float4 r0 = __ldg(rays + 2 * i), r1 = __ldg(rays + 2 * i + 1);
  const float4* rec = tris + 4 * (size_t)(uint32_t)h.x;
  const float4 a = __ldg(rec), b = __ldg(rec + 1), c = __ldg(rec + 2);
  const float3 A = make_float3(a.x, a.y, a.z), B = make_float3(b.x, b.y, b.z), C = make_float3(c.x, c.y, c.z);
  float t = __int_as_float(h.y), u = 0.0f, v = 0.0f;
  float tr, ur, vr;
  const bool placed = inst_table && h.z >= 0;
  bool ok;
  if (placed && inst_l2w) {
    const float4* lr = inst_l2w + 3 * (size_t)h.z;
    ok = ff_refine_placed(make_float3(r0.x, r0.y, r0.z), make_float3(r1.x, r1.y, r1.z), __ldg(lr), __ldg(lr + 1),
                          __ldg(lr + 2), A, B, C, &tr, &ur, &vr);
  } else {
    if (placed) {
      // the instance's local ray, computed as the traversal computed it
      const float4* ir = inst_table + 4 * (size_t)h.z;
      const float4 m0 = __ldg(ir), m1 = __ldg(ir + 1), m2 = __ldg(ir + 2);
      const float ox = r0.x, oy = r0.y, oz = r0.z, dx = r1.x, dy = r1.y, dz = r1.z;
      r0.x = fmaf(m0.x, ox, fmaf(m0.y, oy, fmaf(m0.z, oz, m0.w)));
      r0.y = fmaf(m1.x, ox, fmaf(m1.y, oy, fmaf(m1.z, oz, m1.w)));
      r0.z = fmaf(m2.x, ox, fmaf(m2.y, oy, fmaf(m2.z, oz, m2.w)));
      r1.x = fmaf(m0.x, dx, fmaf(m0.y, dy, m0.z * dz));
      r1.y = fmaf(m1.x, dx, fmaf(m1.y, dy, m1.z * dz));
      r1.z = fmaf(m2.x, dx, fmaf(m2.y, dy, m2.z * dz));
    }
    ok = ff_refine(make_float3(r0.x, r0.y, r0.z), make_float3(r1.x, r1.y, r1.z), A, B, C, &tr, &ur, &vr);
  }
  if (ok) {
    t = tr;
    u = ur;
    v = vr;
  } else if (!placed) {
    // degenerate in float-float too: report the watertight barycentrics
    WtRay wr = wt_setup(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
    WtHit wh;
    if (wt_intersect(wr, A, B, C, r0.w, &wh)) {
      u = wh.bary[1];
      v = wh.bary[2];
    }
  }
  hits[i] = make_int4((int)__float_as_uint(a.w), __float_as_int(t), __float_as_int(u), __float_as_int(v));
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

// Resident CTAs per SM of one instantiation with `smem` dynamic bytes (the
// opt-in above 48 KB is set first).
template <class K>
int resident_per_sm(K kern, size_t smem) {
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem);
  return per_sm;
}

template <bool ANY, bool TWO>
void launch_trace_k(const TraceArgs& a, cudaStream_t s) {
  auto plain = k_trace<ANY, TWO, false>;
  auto staged = k_trace<ANY, TWO, true>;
  const int stk = std::min(std::max(a.stack_depth, 4), kMaxStack);
  const size_t stack_bytes = 0;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = resident_per_sm(plain, stack_bytes);
  if (a.blocks_per_sm > 0) per_sm = std::min(per_sm, a.blocks_per_sm);
  // staged prefix: the nodes from nodes[root] on, for launches with one root,
  // a 16-aligned start (bulk copies), and no loss of resident CTAs
  uint32_t hot = 0;
  if (a.stage_nodes && !a.roots && a.node_count > a.root &&
      reinterpret_cast<uintptr_t>(a.nodes + (size_t)a.root * 5) % 16 == 0) {
    hot = (uint32_t)std::min<size_t>(kHotNodes, a.node_count - a.root);
    if (resident_per_sm(staged, stack_bytes + 80 * (size_t)hot) < per_sm) hot = 0;
  }
  // persistent grid: every resident slot once, never more blocks than rays need
  size_t grid = (size_t)std::max(1, sms) * (size_t)std::max(1, per_sm);
  grid = std::min(grid, (a.n + kBlock - 1) / kBlock);
  cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), s);
  (hot ? staged : plain)<<<(unsigned)grid, kBlock, stack_bytes + 80 * (size_t)hot, s>>>(
      a.nodes, a.tris, a.rays, a.n, a.hits, a.occluded, a.status, a.counter, a.n_dev, a.insts, a.root, a.roots, hot,
      stk, a.stage_wait_cycles > 0 ? a.stage_wait_cycles : kStagingWaitCycles, a.order, a.inst_table);
}

template <bool ANY>
void launch_trace_t(const TraceArgs& a, cudaStream_t s) {
  if (a.n == 0) return;
  if (a.insts) launch_trace_k<ANY, true>(a, s);
  else launch_trace_k<ANY, false>(a, s);
}

}  // namespace

void launch_trace_closest(const TraceArgs& a, cudaStream_t s) {
  launch_trace_t<false>(a, s);
  if (a.n)
    k_refine_hits<<<(unsigned)((a.n + 255) / 256), 256, 0, s>>>(a.tris, a.rays, a.n, a.hits, a.inst_table,
                                                                a.inst_l2w, a.inst_out);
}
void launch_trace_any(const TraceArgs& a, cudaStream_t s) { launch_trace_t<true>(a, s); }
void launch_trace_closest_records(const TraceArgs& a, cudaStream_t s) { launch_trace_t<false>(a, s); }

const char* trace_status_message(int status) {
  if (status & kTraceStackOverflow) return "traversal stack capacity exceeded";
  if (status & kTraceStagingWait) return "traversal node staging did not complete in time";
  return "traversal failed";
}

void launch_watertight_eval(const float* cases, size_t n, vt_watertight_result* out, cudaStream_t s) {
  if (n == 0) return;
  k_watertight_eval<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(cases, n, out);
}

}  // namespace vt
