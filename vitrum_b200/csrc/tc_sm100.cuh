// tc_sm100.cuh -- sm_100a tensor-core plumbing in inline PTX: tensor memory
// (TMEM) allocation, tcgen05.mma with shared-memory operand descriptors,
// completion through an mbarrier, TMEM -> register loads.
//
// Operand layout used throughout: 128-byte-swizzled tiles of 64 fp16 per row
// (one 128-byte row per matrix row), rows grouped by 8 into 1024-byte atoms
// (the canonical SWIZZLE_128B layout).  Within an atom, 16-byte chunk j of row
// r sits at chunk j ^ (r & 7).  Such a tile serves as
//   K-major operand  (rows = M or N, 64 K elements contiguous), and as
//   MN-major operand (rows = K, 64 M/N elements contiguous),
// so one stored weight tile W[n][k] is B for X·W^T (K-major) and for G·W
// (MN-major), and one stored activation tile X[m][k] is A for X·W^T (K-major)
// and B of the weight gradient G^T·X (MN-major).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace vt {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of (row r, element c) of a 64-column fp16 swizzled tile
__device__ __forceinline__ uint32_t sw128_offset(uint32_t r, uint32_t c) {
  const uint32_t lin = r * 128u + c * 2u;
  return lin ^ (((lin >> 7) & 7u) << 4);
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Non-blocking probe of phase `parity` (mbarrier.test_wait: returns at once).
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Limits below this many clocks poll with test_wait, whose return is immediate
// (try_wait may suspend the thread for a while before it gives up).
constexpr long long kShortWaitCycles = 1000000ll;
// Bounded wait for phase `parity`: false after ~`max_cycles` clocks.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long max_cycles) {
  const long long t0 = clock64();
  if (max_cycles < kShortWaitCycles) {
    while (!mbar_test_wait(bar, parity)) {
      if (clock64() - t0 > max_cycles) return false;
    }
    return true;
  }
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > max_cycles) return false;
  }
  return true;
}

// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---------------------------------------------------------------- TMEM
// Warp-collective: allocates `ncols` columns (power of two >= 32) and writes
// the TMEM base address to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp w of a
// warpgroup reads lanes 32w..32w+31; lane field in bits 16-31 of taddr)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---------------------------------------------------------------- MMA
// Shared-memory matrix descriptor, SWIZZLE_128B, version 1 (sm_100).
// lbo/sbo in bytes (multiples of 16).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}
// K-major operand: step kk of 16 fp16 K elements advances 32 bytes in the row
__device__ __forceinline__ uint64_t desc_k(uint32_t tile, uint32_t kk) { return sdesc(tile + kk * 32u, 16u, 1024u); }
// MN-major operand: step kk of 16 K rows advances two 8-row atoms; `lbo` is
// the byte distance to the next 64-element MN atom (M = 128 uses two)
__device__ __forceinline__ uint64_t desc_mn(uint32_t tile, uint32_t kk, uint32_t lbo) {
  return sdesc(tile + kk * 2048u, lbo, 1024u);
}

// Instruction descriptor, kind::f16: fp16 A/B, fp32 accumulate, shape M x N.
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t M, uint32_t N, bool a_mn, bool b_mn) {
  return (1u << 4) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// D[tmem] (+)= A * B, issued by one thread
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive on `bar` once every tcgen05 operation this thread issued has completed
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

}  // namespace tc
}  // namespace vt
