// bvh_encode_gpu.cu -- the 8-wide collapse and compressed-node encoding of
// bvh_encode.cpp on the GPU, producing the same node words and records.
//
//   1. parents of the binary nodes (children follow their parent: left at
//      i + 1, right at i + w6);
//   2. SAH-optimal collapse plan (Ylitie, Karras & Laine 2017, sec. 3.1),
//      bottom up: one thread per binary leaf climbs towards the root, the
//      second child to arrive at a node (an atomic counter per node) computes
//      its costs C(n), G(n, k) and splits from the children's, every value an
//      IEEE-double operation in the host's order, ties to the first minimum;
//   3. wide levels, top down, as the host's breadth-first queue: per level
//      one thread per wide node picks its children (the plan's frontier or the
//      reference's greedy rule) and slots; an exclusive scan over the level
//      gives each node its child base and record block, so numbering equals
//      the host's queue order; each node's 80 bytes and its leaf records are
//      then written, the internal children listed for the next level.
// Quantised child bounds are rounded outward exactly: each grid corner
// origin + q * 2^e is compared with the child bound through a nonoverlapping
// expansion of the sum (Shewchuk's grow-expansion of TwoSums), whose largest
// component carries the exact sign.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bvh_exact.h"
#include "bvh_host.h"
#include "vt_common.h"

namespace vt {

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kMerged = 0x80000000u;  // frontier entry: the leaf slot of a subtree (not its node)

struct DpNode {
  double c;        // C(n)
  double g[7];     // G(n, k), k = 2 .. 8
  uint32_t first, count;
  uint8_t split[7];
  uint8_t as_leaf;
};

__device__ __forceinline__ bool leaf_word(uint32_t w7) { return (w7 & kLeafFlag) != 0; }

__device__ __forceinline__ double half_area_d(const BinaryNode& n) {
  double dx = __dsub_rn((double)n.mx[0], (double)n.mn[0]);
  double dy = __dsub_rn((double)n.mx[1], (double)n.mn[1]);
  double dz = __dsub_rn((double)n.mx[2], (double)n.mn[2]);
  dx = dx > 0.0 ? dx : 0.0;  // std::max(0.0, x): x when x > 0, else 0
  dy = dy > 0.0 ? dy : 0.0;
  dz = dz > 0.0 ? dz : 0.0;
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dy), __dmul_rn(dy, dz)), __dmul_rn(dz, dx));
}

__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }  // std::min

__global__ void k_parents(const BinaryNode* __restrict__ nodes, uint32_t n, uint32_t* __restrict__ parent) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const BinaryNode b = nodes[i];
  if (leaf_word(b.w7)) return;
  parent[i + 1] = i;
  parent[i + b.w6] = i;
}

// loads a plan entry another thread wrote (L2, not a stale L1 line)
__device__ __forceinline__ void load_dp(const DpNode* p, DpNode& o) {
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(p);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&o);
#pragma unroll
  for (int k = 0; k < (int)(sizeof(DpNode) / 8); ++k) d[k] = __ldcg(s + k);
}

__global__ void k_plan(const BinaryNode* __restrict__ nodes, uint32_t n, const uint32_t* __restrict__ parent,
                       unsigned int* __restrict__ visits, DpNode* __restrict__ dp, double c_node, double c_tri,
                       int width) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const BinaryNode b = nodes[i];
  if (!leaf_word(b.w7)) return;
  DpNode d;
  d.first = b.w6;
  d.count = b.w7 & 0xFFFFu;
  d.c = __dmul_rn(__dmul_rn(c_tri, half_area_d(b)), (double)d.count);
  d.as_leaf = 1;
  for (int k = 0; k < 7; ++k) { d.g[k] = 0.0; d.split[k] = 0; }
  dp[i] = d;
  uint32_t x = parent[i];
  while (x != kNone) {
    __threadfence();
    if (atomicAdd(&visits[x], 1u) == 0u) return;  // the other child is not done yet
    __threadfence();
    const BinaryNode nb = nodes[x];
    const uint32_t l = x + 1, r = x + nb.w6;
    DpNode L, R;
    load_dp(dp + l, L);
    load_dp(dp + r, R);
    const bool lleaf = leaf_word(nodes[l].w7), rleaf = leaf_word(nodes[r].w7);
    DpNode o;
    o.first = L.first;
    o.count = L.count + R.count;
    const bool contiguous = R.first == L.first + L.count;
    for (int k = 2; k <= 8; ++k) {
      double best = INFINITY;
      int at = 1;
      for (int a = 1; a < k; ++a) {
        const double fl = (a < 2 || lleaf) ? L.c : dmin(L.c, L.g[a - 2]);
        const int bk = k - a;
        const double fr = (bk < 2 || rleaf) ? R.c : dmin(R.c, R.g[bk - 2]);
        const double v = __dadd_rn(fl, fr);
        if (v < best) { best = v; at = a; }
      }
      o.g[k - 2] = best;
      o.split[k - 2] = (uint8_t)at;
    }
    const double area = half_area_d(nb);
    o.c = __dadd_rn(__dmul_rn(c_node, area), o.g[width - 2]);
    o.as_leaf = 0;
    if (o.count <= 4 && contiguous) {
      const double leaf = __dmul_rn(__dmul_rn(c_tri, area), (double)o.count);
      if (leaf < o.c) {
        o.c = leaf;
        o.as_leaf = 1;
      }
    }
    dp[x] = o;
    x = parent[x];
  }
}

// The frontier of x over a slots (the host's SahCollapse::frontier), left first.
__device__ __forceinline__ void frontier(const BinaryNode* nodes, const DpNode* dp, uint32_t x, int a, uint32_t* out,
                                         int& m) {
  uint32_t sx[16];
  int sa[16], top = 0;
  sx[top] = x;
  sa[top++] = a;
  while (top > 0) {
    --top;
    const uint32_t y = sx[top];
    const int b = sa[top];
    const BinaryNode& ny = nodes[y];
    const DpNode& dy = dp[y];
    if (b >= 2 && !leaf_word(ny.w7) && dy.g[b - 2] < dy.c) {
      const int s = dy.split[b - 2];
      if (top + 2 > 16) { out[m++] = y; continue; }  // not reached: a frontier has at most 8 entries
      sx[top] = y + ny.w6;
      sa[top++] = b - s;
      sx[top] = y + 1;
      sa[top++] = s;
      continue;
    }
    if (m < 8) out[m++] = dy.as_leaf ? (y | kMerged) : y;
  }
}

// The reference's greedy rule (collectWideChildren, compressedWideBvh.ts:215-242).
__device__ __forceinline__ int greedy_children(const BinaryNode* nodes, uint32_t root, uint32_t out[8]) {
  const BinaryNode& r = nodes[root];
  if (leaf_word(r.w7)) { out[0] = root; return 1; }
  int n = 2;
  out[0] = root + 1;
  out[1] = root + r.w6;
  while (n < 8) {
    int at = -1;
    double best = -1;
    for (int i = 0; i < n; ++i) {
      const BinaryNode& c = nodes[out[i]];
      if (leaf_word(c.w7)) continue;
      const double a = half_area_d(c);
      if (a > best) { best = a; at = i; }
    }
    if (at < 0) break;
    const uint32_t x = out[at];
    for (int j = n; j > at + 1; --j) out[j] = out[j - 1];
    out[at] = x + 1;
    out[at + 1] = x + nodes[x].w6;
    ++n;
  }
  return n;
}

// Greedy slot assignment (the host's assign_slots), IEEE doubles in its order.
// Each (child, slot) cost is recomputed where it is compared (the same
// operations, so the same value) instead of being kept in an 8 x 8 array, and
// the slots come back packed in registers: slot of child i in bits 4i..4i+3.
__device__ __forceinline__ uint32_t assign_slots(const BinaryNode* nodes, const BinaryNode& parent, const uint32_t* ch,
                                                 int n) {
  const double pcx = __dmul_rn(0.5, __dadd_rn((double)parent.mn[0], (double)parent.mx[0]));
  const double pcy = __dmul_rn(0.5, __dadd_rn((double)parent.mn[1], (double)parent.mx[1]));
  const double pcz = __dmul_rn(0.5, __dadd_rn((double)parent.mn[2], (double)parent.mx[2]));
  double dx[8], dy[8], dz[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (i >= n) { dx[i] = dy[i] = dz[i] = 0.0; continue; }
    const BinaryNode c = nodes[ch[i] & ~kMerged];
    dx[i] = __dsub_rn(__dmul_rn(0.5, __dadd_rn((double)c.mn[0], (double)c.mx[0])), pcx);
    dy[i] = __dsub_rn(__dmul_rn(0.5, __dadd_rn((double)c.mn[1], (double)c.mx[1])), pcy);
    dz[i] = __dsub_rn(__dmul_rn(0.5, __dadd_rn((double)c.mn[2], (double)c.mx[2])), pcz);
  }
  uint32_t used_c = 0, used_s = 0, slots = 0xFFFFFFFFu;
  for (int round = 0; round < n; ++round) {
    int bi = -1, bs = -1;
    double bc = INFINITY;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (i >= n || ((used_c >> i) & 1u)) continue;
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        if ((used_s >> s) & 1u) continue;
        const double sx = (s & 4) ? -1.0 : 1.0, sy = (s & 2) ? -1.0 : 1.0, sz = (s & 1) ? -1.0 : 1.0;
        const double cost = __dadd_rn(__dadd_rn(__dmul_rn(dx[i], sx), __dmul_rn(dy[i], sy)), __dmul_rn(dz[i], sz));
        if (bi < 0 || cost < bc) { bc = cost; bi = i; bs = s; }
      }
    }
    used_c |= 1u << bi;
    used_s |= 1u << bs;
    slots = (slots & ~(0xFu << (4 * bi))) | ((uint32_t)bs << (4 * bi));
  }
  return slots;
}

struct LevelPlan {
  uint32_t ch[8];      // children (binary ids; kMerged: a subtree's leaf slot)
  int8_t slot_of[8];
  int32_t n;
};

// is child entry e a leaf slot?  (a merged subtree, or a binary leaf)
__device__ __forceinline__ bool entry_is_leaf(const BinaryNode* nodes, uint32_t e) {
  return (e & kMerged) || leaf_word(nodes[e].w7);
}

// sah: 0 the reference's greedy collapse, else the SAH-optimal collapse at that width (2..8)
__global__ void k_level_plan(const BinaryNode* __restrict__ nodes, const DpNode* __restrict__ dp, int sah,
                             const uint32_t* __restrict__ level, uint32_t n_level, LevelPlan* __restrict__ plan,
                             uint32_t* __restrict__ n_int, uint32_t* __restrict__ span) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_level) return;
  const uint32_t x = level[j];
  LevelPlan p;
  int n;
  if (sah) {
    n = 0;
    if (leaf_word(nodes[x].w7)) {
      p.ch[0] = x;
      n = 1;
    } else {
      const int s = dp[x].split[sah - 2];
      frontier(nodes, dp, x + 1, s, p.ch, n);
      frontier(nodes, dp, x + nodes[x].w6, sah - s, p.ch, n);
    }
  } else {
    n = greedy_children(nodes, x, p.ch);
  }
  const uint32_t slots = assign_slots(nodes, nodes[x], p.ch, n);
  uint32_t internal = 0;
  int first_leaf = 8, last_leaf = -1;
  for (int i = 0; i < n; ++i) {
    const int si = (int)((slots >> (4 * i)) & 0xFu);
    p.slot_of[i] = (int8_t)si;
    if (entry_is_leaf(nodes, p.ch[i])) {
      first_leaf = min(first_leaf, si);
      last_leaf = max(last_leaf, si);
    } else {
      ++internal;
    }
  }
  for (int i = n; i < 8; ++i) p.slot_of[i] = -1;
  p.n = n;
  plan[j] = p;
  n_int[j] = internal;
  span[j] = last_leaf >= 0 ? (uint32_t)(4 * (last_leaf - first_leaf) + 4) : 0u;
}

// Exclusive scans of two arrays in one CTA (levels are at most a few 100 k nodes).
__global__ void k_scan2(uint32_t* __restrict__ a, uint32_t* __restrict__ b, uint32_t n,
                        unsigned long long* __restrict__ totals) {
  __shared__ unsigned long long wa[32], wb[32];
  __shared__ unsigned long long carry_a, carry_b;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) { carry_a = 0; carry_b = 0; }
  __syncthreads();
  for (uint32_t base = 0; base < n; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const unsigned long long va = i < n ? a[i] : 0, vb = i < n ? b[i] : 0;
    unsigned long long sa = va, sb = vb;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long ta = __shfl_up_sync(0xFFFFFFFFu, sa, o), tb = __shfl_up_sync(0xFFFFFFFFu, sb, o);
      if (lane >= o) { sa += ta; sb += tb; }
    }
    if (lane == 31) { wa[w] = sa; wb[w] = sb; }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long ra = carry_a, rb = carry_b;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
        const unsigned long long xa = wa[q], xb = wb[q];
        wa[q] = ra;
        wb[q] = rb;
        ra += xa;
        rb += xb;
      }
      carry_a = ra;
      carry_b = rb;
    }
    __syncthreads();
    if (i < n) {
      a[i] = (uint32_t)(wa[w] + sa - va);
      b[i] = (uint32_t)(wb[w] + sb - vb);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    totals[0] = carry_a;
    totals[1] = carry_b;
  }
}

// smallest e with origin + 255 2^e >= hi (exactly), clamped to the normal range (the host's grid_exponent)
__device__ __forceinline__ int grid_exponent(float origin, float hi) {
  const double extent = __dsub_rn((double)hi, (double)origin);
  if (!(extent > 0)) return -126;
  int e;
  frexp(__ddiv_rn(extent, 255.0), &e);
  while (e > -126 && ldexp(255.0, e - 1) >= extent) --e;
  while (e < 127 && corner_sign(origin, 255, e, hi) < 0) ++e;
  return min(127, max(-126, e));
}

// Unit normal as the reference's watertight test derives it (the host's
// reference_normal): single precision, every operation rounded on its own.
__device__ __forceinline__ bool reference_normal(const float a[3], const float b[3], const float c[3], float nn[3]) {
  float e1r[3], e2r[3];
  for (int k = 0; k < 3; ++k) { e1r[k] = __fsub_rn(b[k], a[k]); e2r[k] = __fsub_rn(c[k], a[k]); }
  float es = 0.0f;
  for (int k = 0; k < 3; ++k) es = fmaxf(es, fabsf(e1r[k]));
  for (int k = 0; k < 3; ++k) es = fmaxf(es, fabsf(e2r[k]));
  if (!(es > 0.0f) || !isfinite(es)) return false;
  float s1[3], s2[3];
  for (int k = 0; k < 3; ++k) { s1[k] = __fdiv_rn(e1r[k], es); s2[k] = __fdiv_rn(e2r[k], es); }
  const float nr[3] = {__fsub_rn(__fmul_rn(s1[1], s2[2]), __fmul_rn(s1[2], s2[1])),
                       __fsub_rn(__fmul_rn(s1[2], s2[0]), __fmul_rn(s1[0], s2[2])),
                       __fsub_rn(__fmul_rn(s1[0], s2[1]), __fmul_rn(s1[1], s2[0]))};
  const float ns = fmaxf(fmaxf(fabsf(nr[0]), fabsf(nr[1])), fabsf(nr[2]));
  if (!(ns > 0.0f) || !isfinite(ns)) return false;
  const float nd[3] = {__fdiv_rn(nr[0], ns), __fdiv_rn(nr[1], ns), __fdiv_rn(nr[2], ns)};
  const float l2 = __fadd_rn(__fadd_rn(__fmul_rn(nd[0], nd[0]), __fmul_rn(nd[1], nd[1])), __fmul_rn(nd[2], nd[2]));
  const float nl = __fsqrt_rn(l2);
  if (!(nl > 0.0f) || !isfinite(nl)) return false;
  for (int k = 0; k < 3; ++k) nn[k] = __fdiv_rn(nd[k], nl);
  return true;
}

struct EmitArgs {
  const BinaryNode* nodes;
  const DpNode* dp;          // SAH plan (first / count of merged subtrees), null for the greedy rule
  const uint32_t* order;     // BVH-order triangle (or instance) permutation
  const float* pos;          // triangles: vertex positions (stride ps)
  int ps;
  const uint32_t* idx;       // triangles: indices (stride is)
  int is;
  const uint32_t* tri_mat;   // optional, one per source triangle
  const float* inst_recs;    // top level: 16 floats per instance (else null)
  uint32_t node_base, rec_base;
};

__global__ void k_level_emit(EmitArgs A, const uint32_t* __restrict__ level, uint32_t n_level,
                             const LevelPlan* __restrict__ plan, const uint32_t* __restrict__ int_off,
                             const uint32_t* __restrict__ rec_off, uint32_t level_start, uint32_t rec_start,
                             uint32_t* __restrict__ words, float* __restrict__ recs, uint32_t* __restrict__ next,
                             int* __restrict__ err) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_level) return;
  const BinaryNode parent = A.nodes[level[j]];
  const LevelPlan p = plan[j];
  int child_at_slot[8];
  for (int s = 0; s < 8; ++s) child_at_slot[s] = -1;
  for (int i = 0; i < p.n; ++i) child_at_slot[p.slot_of[i]] = i;
  uint32_t wl[20];
  for (int k = 0; k < 20; ++k) wl[k] = 0;
  uint8_t* bytes = reinterpret_cast<uint8_t*>(wl);
  const float pm[3] = {parent.mn[0], parent.mn[1], parent.mn[2]};
  memcpy(bytes, pm, 12);
  int ex[3];
  for (int k = 0; k < 3; ++k) {
    ex[k] = grid_exponent(parent.mn[k], parent.mx[k]);
    bytes[12 + k] = (uint8_t)(ex[k] + 127);
  }
  uint8_t imask = 0;
  const uint32_t child_base = A.node_base + level_start + n_level + int_off[j];
  int first_leaf = 8;
  for (int s = 0; s < 8; ++s) {
    const int ci = child_at_slot[s];
    if (ci >= 0 && entry_is_leaf(A.nodes, p.ch[ci])) { first_leaf = s; break; }
  }
  const uint32_t block = rec_start + rec_off[j];
  const uint32_t tri_base = A.rec_base + block - 4u * (uint32_t)(first_leaf < 8 ? first_leaf : 0);
  if ((unsigned long long)A.rec_base + block + 32 >= 0x40000000ull) atomicOr(err, 1);
  uint32_t tri_valid = 0;
  uint32_t q_int = 0;
  uint8_t* qlo = bytes + 32;
  uint8_t* qhi = bytes + 56;
  for (int s = 0; s < 8; ++s) {
    const int ci = child_at_slot[s];
    if (ci < 0) {
      for (int k = 0; k < 3; ++k) { qlo[k * 8 + s] = 255; qhi[k * 8 + s] = 0; }
      continue;
    }
    const uint32_t e = p.ch[ci];
    const uint32_t id = e & ~kMerged;
    const BinaryNode c = A.nodes[id];
    for (int k = 0; k < 3; ++k) {
      const double step = ldexp(1.0, ex[k]);
      const double lo = floor(__ddiv_rn(__dsub_rn((double)c.mn[k], (double)pm[k]), step));
      const double hi = ceil(__ddiv_rn(__dsub_rn((double)c.mx[k], (double)pm[k]), step));
      int ql = (int)fmin(255.0, fmax(0.0, lo));
      int qh = (int)fmin(255.0, fmax(0.0, hi));
      while (ql > 0 && corner_sign(pm[k], ql, ex[k], c.mn[k]) > 0) --ql;
      while (qh < 255 && corner_sign(pm[k], qh, ex[k], c.mx[k]) < 0) ++qh;
      qlo[k * 8 + s] = (uint8_t)ql;
      qhi[k * 8 + s] = (uint8_t)qh;
    }
    if (entry_is_leaf(A.nodes, e)) {
      uint32_t first, cnt;
      if (e & kMerged) {
        first = A.dp[id].first;
        cnt = A.dp[id].count;
      } else {
        first = c.w6;
        cnt = c.w7 & 0xFFFFu;
      }
      tri_valid |= ((1u << cnt) - 1u) << (4 * s);
      float* out = recs + 16 * ((size_t)block + 4 * (s - first_leaf));
      for (uint32_t t = 0; t < cnt; ++t) {
        const uint32_t src = A.order[first + t];
        float* rec = out + 16 * t;
        if (A.inst_recs) {
          for (int k = 0; k < 16; ++k) rec[k] = A.inst_recs[16 * (size_t)src + k];
          continue;
        }
        const uint32_t* iv = A.idx + (size_t)src * A.is;
        float v[3][3];
        for (int vi = 0; vi < 3; ++vi)
          for (int k = 0; k < 3; ++k) v[vi][k] = A.pos[(size_t)iv[vi] * A.ps + k];
        for (int vi = 0; vi < 3; ++vi)
          for (int k = 0; k < 3; ++k) rec[4 * vi + k] = v[vi][k];
        rec[3] = __uint_as_float(src);
        rec[7] = A.tri_mat ? __uint_as_float(A.tri_mat[src]) : 0.0f;
        rec[11] = 0.0f;
        float nn[3] = {0, 0, 0};
        const bool valid = reference_normal(v[0], v[1], v[2], nn);
        rec[12] = nn[0];
        rec[13] = nn[1];
        rec[14] = nn[2];
        rec[15] = valid ? 1.0f : 0.0f;
      }
    } else {
      imask |= (uint8_t)(1u << s);
      next[int_off[j] + q_int++] = id;
    }
  }
  memcpy(bytes + 24, &tri_valid, 4);
  bytes[15] = imask;
  memcpy(bytes + 16, &child_base, 4);
  memcpy(bytes + 20, &tri_base, 4);
  uint32_t* w = words + 20 * (size_t)(level_start + j);
  for (int k = 0; k < 20; ++k) w[k] = wl[k];
}

}  // namespace

WideBvhHost encode_wide_gpu(const BinaryBvhDevice& bin, const float* d_pos, int pos_stride, const uint32_t* d_idx,
                            int idx_stride, const uint32_t* d_tri_mat, uint32_t node_base, uint32_t rec_base,
                            const WideCollapse* sah, const float* d_inst_recs, cudaStream_t s, WideBvhDevice* keep) {
  WideBvhHost out;
  const uint32_t n = (uint32_t)bin.n_nodes;
  if (bin.ntri == 0 || n == 0) {
    // an empty tree: one node with all slots empty (inverted boxes), no records
    uint32_t w[20] = {};
    std::memset(reinterpret_cast<uint8_t*>(w) + 32, 0xFF, 24);
    out.nodes.assign(w, w + 20);
    out.depth = 1;
    if (keep) {
      keep->nodes.resize(20);
      VT_CUDA(cudaMemcpyAsync(keep->nodes.ptr, w, sizeof w, cudaMemcpyHostToDevice, s));
      keep->recs.resize(0);
      keep->n_nodes = 1;
      keep->n_recs = 0;
      VT_CUDA(cudaStreamSynchronize(s));
    }
    return out;
  }
  ScratchBuffer<DpNode> dp;
  const int width = sah ? std::min(std::max(sah->width, 2), 8) : 0;
  if (sah) {
    ScratchBuffer<uint32_t> parent(n, s);
    ScratchBuffer<unsigned int> visits(n, s);
    dp.resize(n, s);
    VT_CUDA(cudaMemsetAsync(parent.ptr, 0xFF, n * sizeof(uint32_t), s));
    VT_CUDA(cudaMemsetAsync(visits.ptr, 0, n * sizeof(unsigned int), s));
    k_parents<<<(n + 255) / 256, 256, 0, s>>>(bin.nodes.ptr, n, parent.ptr);
    VT_CUDA(cudaGetLastError());
    k_plan<<<(n + 255) / 256, 256, 0, s>>>(bin.nodes.ptr, n, parent.ptr, visits.ptr, dp.ptr, sah->c_node, sah->c_tri,
                                           width);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaStreamSynchronize(s));
  }
  // wide nodes: at most one per binary interior node (a lone leaf root: one)
  const uint32_t max_wide = n / 2 + 1;
  DeviceBuffer<uint32_t> words((size_t)20 * max_wide);
  size_t rec_cap = 28 + 4 * (size_t)bin.ntri + 64;
  DeviceBuffer<float> recs(16 * rec_cap);
  VT_CUDA(cudaMemsetAsync(recs.ptr, 0, recs.bytes(), s));
  ScratchBuffer<uint32_t> lvl_a(max_wide, s), lvl_b(max_wide, s), n_int(max_wide, s), span(max_wide, s);
  ScratchBuffer<LevelPlan> plan(max_wide, s);
  ScratchBuffer<unsigned long long> totals(2, s);
  ScratchBuffer<int> err(1, s);
  VT_CUDA(cudaMemsetAsync(err.ptr, 0, sizeof(int), s));
  const uint32_t root = 0;
  VT_CUDA(cudaMemcpyAsync(lvl_a.ptr, &root, sizeof root, cudaMemcpyHostToDevice, s));
  EmitArgs A{bin.nodes.ptr, sah ? dp.ptr : nullptr, bin.order.ptr, d_pos, pos_stride, d_idx, idx_stride, d_tri_mat,
             d_inst_recs, node_base, rec_base};
  uint32_t level_n = 1, level_start = 0, rec_used = 28;
  int depth = 0;
  ScratchBuffer<uint32_t>* cur = &lvl_a;
  ScratchBuffer<uint32_t>* nxt = &lvl_b;
  while (level_n) {
    ++depth;
    const unsigned blocks = (level_n + 127) / 128;
    k_level_plan<<<blocks, 128, 0, s>>>(bin.nodes.ptr, sah ? dp.ptr : nullptr, sah ? width : 0, cur->ptr, level_n,
                                        plan.ptr, n_int.ptr, span.ptr);
    VT_CUDA(cudaGetLastError());
    k_scan2<<<1, 1024, 0, s>>>(n_int.ptr, span.ptr, level_n, totals.ptr);
    VT_CUDA(cudaGetLastError());
    unsigned long long tot[2];
    VT_CUDA(cudaMemcpyAsync(tot, totals.ptr, sizeof tot, cudaMemcpyDeviceToHost, s));
    VT_CUDA(cudaStreamSynchronize(s));
    if (level_start + level_n + tot[0] > max_wide) fail(VT_ERR_BUILD, "wide encoding: more nodes than bounded");
    if (rec_used + tot[1] > rec_cap) {
      // grow the record array (more leaf slots than the first estimate)
      const size_t cap = std::max<size_t>(rec_used + tot[1] + 64, rec_cap * 3 / 2);
      DeviceBuffer<float> bigger(16 * cap);
      VT_CUDA(cudaMemsetAsync(bigger.ptr, 0, bigger.bytes(), s));
      VT_CUDA(cudaMemcpyAsync(bigger.ptr, recs.ptr, 16 * sizeof(float) * rec_used, cudaMemcpyDeviceToDevice, s));
      recs = std::move(bigger);
      rec_cap = cap;
    }
    k_level_emit<<<blocks, 128, 0, s>>>(A, cur->ptr, level_n, plan.ptr, n_int.ptr, span.ptr, level_start, rec_used,
                                        words.ptr, recs.ptr, nxt->ptr, err.ptr);
    VT_CUDA(cudaGetLastError());
    level_start += level_n;
    rec_used += (uint32_t)tot[1];
    level_n = (uint32_t)tot[0];
    std::swap(cur, nxt);
  }
  int bad = 0;
  VT_CUDA(cudaMemcpyAsync(&bad, err.ptr, sizeof bad, cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaStreamSynchronize(s));
  if (bad) fail(VT_ERR_BUILD, "leaf records exceed 2^30");
  out.depth = depth;
  out.nodes.resize((size_t)20 * level_start);
  out.tris.resize((size_t)16 * rec_used);
  VT_CUDA(cudaMemcpyAsync(out.nodes.data(), words.ptr, out.nodes.size() * 4, cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaMemcpyAsync(out.tris.data(), recs.ptr, out.tris.size() * 4, cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaStreamSynchronize(s));
  if (keep) {
    keep->nodes = std::move(words);
    keep->recs = std::move(recs);
    keep->n_nodes = level_start;
    keep->n_recs = rec_used;
  }
  return out;
}

}  // namespace vt
