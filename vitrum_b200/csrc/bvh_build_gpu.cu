// bvh_build_gpu.cu -- binned-SAH binary BVH built on the GPU, identical to
// the host build (and so to the reference's buildArrayBvh,
// packages/shared-bvh/src/buildArrayBvh.ts:342-780) word for word.
//
// Top down, one level of the tree per launch, one CTA per node of the level:
//   1. node bounds and centroid bounds (CTA reduction);
//   2. per axis with centroid span > 1e-9: up to 256 bins (count + bounds) in
//      shared memory, bounds kept as order-preserving 64-bit keys updated with
//      atomic min / max (exact and order-free), prefix / suffix sweeps with the
//      bounds rounded to f32 as the reference stores them, SAH cost;
//   3. stable partition of the node's index range by bin <= split (CTA scan,
//      chunk by chunk, through a scratch range), or the balanced fallback:
//      sort by (centroid on the widest axis, triangle index) -- bitonic in
//      shared memory up to 4096 triangles, two stable device radix passes
//      (index, then centroid) beyond -- and split at count / 2;
//   4. children appended to the next level's list.
// Bounds are minima / maxima (exact, order-free: -0 wins a min tie, +0 a max
// tie, as in JS Math.min / Math.max), every other operation is a single
// IEEE-double operation (__dadd_rn & co., no contraction), so the decisions
// equal the host's.  Afterwards subtree sizes give the preorder numbering
// (left child = i + 1, right = i + 1 + size(left)); a leaf's triangle offset
// is the start of its index range, which partitioning never moves again.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "bvh_host.h"
#include "vt_common.h"

namespace vt {

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxBins = 256;       // binCount in [2, 256], as the options allow
constexpr int kSortMax = 4096;      // fallback sorts up to this many in shared memory

struct GNode {
  uint32_t begin, count, depth;
  int32_t left, right;              // child node ids (-1: leaf)
  int32_t axis;                     // split axis, -1 leaf
  uint32_t size, pre;               // subtree node count, preorder index
  float mn[3], mx[3];
  int32_t big_sort;                 // 1: the fallback sort of this node runs as device radix passes
  int32_t pad;
};

__device__ __forceinline__ double jmin(double a, double b) {
  return a < b ? a : (b < a ? b : (signbit(a) ? a : b));
}
__device__ __forceinline__ double jmax(double a, double b) {
  return a > b ? a : (b > a ? b : (signbit(a) ? b : a));
}
__device__ __forceinline__ double half_sa(double mnx, double mny, double mnz, double mxx, double mxy, double mxz) {
  double dx = __dsub_rn(mxx, mnx), dy = __dsub_rn(mxy, mny), dz = __dsub_rn(mxz, mnz);
  dx = dx > 0 ? dx : 0;
  dy = dy > 0 ? dy : 0;
  dz = dz > 0 ? dz : 0;
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dy), __dmul_rn(dy, dz)), __dmul_rn(dz, dx));
}
__device__ __forceinline__ int bin_of(double c, double cmin, double span, int bins) {
  const double x = __ddiv_rn(__dsub_rn(c, cmin), span);
  const double f = floor(__dmul_rn(x, (double)bins));
  return f < (double)(bins - 1) ? (int)f : bins - 1;
}

// Order-preserving 64-bit key of a double: key(a) < key(b) iff a < b, and
// key(-0) < key(+0), so an integer min / max follows the JS tie rules (-0
// wins a min tie, +0 a max tie).
__device__ __forceinline__ unsigned long long okey(double d) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(d);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double okey_value(unsigned long long k) {
  return __longlong_as_double((long long)((k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k));
}

// Triangle bounds and centroids in double from the f32 vertices.
__global__ void k_prep(const float* __restrict__ pos, int ps, size_t nvert, const uint32_t* __restrict__ idx, int is,
                       uint32_t n, double* __restrict__ tb, double* __restrict__ cen, uint32_t* __restrict__ A,
                       int* __restrict__ bad) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  A[t] = t;
  const uint32_t* iv = idx + (size_t)t * is;
  if (iv[0] >= nvert || iv[1] >= nvert || iv[2] >= nvert) {
    atomicOr(bad, 1);  // out-of-range vertex: reported, nothing read
    return;
  }
  for (int k = 0; k < 3; ++k) {
    const double va = pos[(size_t)iv[0] * ps + k], vb = pos[(size_t)iv[1] * ps + k], vc = pos[(size_t)iv[2] * ps + k];
    const double lo = jmin(jmin(va, vb), vc), hi = jmax(jmax(va, vb), vc);
    tb[6 * (size_t)t + k] = lo;
    tb[6 * (size_t)t + 3 + k] = hi;
    cen[3 * (size_t)t + k] = __dmul_rn(0.5, __dadd_rn(lo, hi));
    if (!isfinite(lo) || !isfinite(hi)) atomicOr(bad, 2);
  }
}

// Per-bin arrays in dynamic shared memory (80 bytes per bin), laid out by bin_arrays().
struct Bins {
  unsigned long long (*mn)[3], (*mx)[3];  // bin bounds as okey()s
  float (*smn)[3], (*smx)[3];             // suffix bounds (f32, as stored)
  unsigned int* c;
  int* sc;
};
__host__ __device__ constexpr size_t bin_bytes(int bins) { return (size_t)bins * 80; }
__device__ __forceinline__ Bins bin_arrays(unsigned char* dyn, int bins) {
  Bins B;
  B.mn = reinterpret_cast<unsigned long long(*)[3]>(dyn);
  B.mx = reinterpret_cast<unsigned long long(*)[3]>(dyn + (size_t)bins * 24);
  B.smn = reinterpret_cast<float(*)[3]>(dyn + (size_t)bins * 48);
  B.smx = reinterpret_cast<float(*)[3]>(dyn + (size_t)bins * 60);
  B.c = reinterpret_cast<unsigned int*>(dyn + (size_t)bins * 72);
  B.sc = reinterpret_cast<int*>(dyn + (size_t)bins * 76);
  return B;
}

struct Shared {
  double red[kWarps][12];                        // CTA reduction of node / centroid bounds (up to 16 warps)
  double nb[12];                                 // node bounds (6) + centroid bounds (6)
  double best_cost;
  int best_axis, best_split, nl, decision;       // decision: 0 leaf, 1 SAH split, 2 fallback, 3 large fallback
  unsigned int scan[kWarps + 1];
};

__device__ void cta_bounds(const double* tb, const double* cen, const uint32_t* A, uint32_t b, uint32_t c, Shared& S) {
  double v[12];
  for (int k = 0; k < 3; ++k) {
    v[k] = INFINITY; v[3 + k] = -INFINITY; v[6 + k] = INFINITY; v[9 + k] = -INFINITY;
  }
  for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
    const uint32_t t = A[b + i];
    for (int k = 0; k < 3; ++k) {
      v[k] = jmin(v[k], tb[6 * (size_t)t + k]);
      v[3 + k] = jmax(v[3 + k], tb[6 * (size_t)t + 3 + k]);
      v[6 + k] = jmin(v[6 + k], cen[3 * (size_t)t + k]);
      v[9 + k] = jmax(v[9 + k], cen[3 * (size_t)t + k]);
    }
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; ++k) {
      v[k] = jmin(v[k], __shfl_xor_sync(0xFFFFFFFFu, v[k], o));
      v[3 + k] = jmax(v[3 + k], __shfl_xor_sync(0xFFFFFFFFu, v[3 + k], o));
      v[6 + k] = jmin(v[6 + k], __shfl_xor_sync(0xFFFFFFFFu, v[6 + k], o));
      v[9 + k] = jmax(v[9 + k], __shfl_xor_sync(0xFFFFFFFFu, v[9 + k], o));
    }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 12; ++k) S.red[w][k] = v[k];
  __syncthreads();
  if (threadIdx.x < 12) {
    const int k = threadIdx.x;
    const bool is_min = (k < 3) || (k >= 6 && k < 9);
    double r = S.red[0][k];
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) r = is_min ? jmin(r, S.red[q][k]) : jmax(r, S.red[q][k]);
    S.nb[k] = r;
  }
  __syncthreads();
}

// Bins of one axis into S.
__device__ void cta_bins(const double* tb, const double* cen, const uint32_t* A, uint32_t b, uint32_t c, int axis,
                         double cmin, double span, int bins, const Bins& B) {
  for (int j = threadIdx.x; j < bins; j += blockDim.x) {
    B.c[j] = 0;
    for (int k = 0; k < 3; ++k) { B.mn[j][k] = okey(INFINITY); B.mx[j][k] = okey(-INFINITY); }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
    const uint32_t t = A[b + i];
    const int j = bin_of(cen[3 * (size_t)t + axis], cmin, span, bins);
    atomicAdd(&B.c[j], 1u);
    for (int k = 0; k < 3; ++k) {
      atomicMin(&B.mn[j][k], okey(tb[6 * (size_t)t + k]));
      atomicMax(&B.mx[j][k], okey(tb[6 * (size_t)t + 3 + k]));
    }
  }
  __syncthreads();
}

// Sweeps and costs of one axis (thread 0), updating the best split: the
// suffix sweep into shared memory, then the prefix sweep beside the costs.
__device__ void choose(int axis, int bins, double parent_sa, const Bins& B, Shared& S) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  int c = 0;
  for (int i = bins - 1; i >= 0; --i) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = jmin(lo[k], okey_value(B.mn[i][k]));
      hi[k] = jmax(hi[k], okey_value(B.mx[i][k]));
      B.smn[i][k] = (float)lo[k];
      B.smx[i][k] = (float)hi[k];
    }
    c += (int)B.c[i];
    B.sc[i] = c;
  }
  for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
  c = 0;
  for (int s = 0; s < bins - 1; ++s) {
    float pmn[3], pmx[3];
    for (int k = 0; k < 3; ++k) {
      lo[k] = jmin(lo[k], okey_value(B.mn[s][k]));
      hi[k] = jmax(hi[k], okey_value(B.mx[s][k]));
      pmn[k] = (float)lo[k];
      pmx[k] = (float)hi[k];
    }
    c += (int)B.c[s];
    const int lc = c, rc = B.sc[s + 1];
    if (lc == 0 || rc == 0) continue;
    const double lsa = half_sa(pmn[0], pmn[1], pmn[2], pmx[0], pmx[1], pmx[2]);
    const double rsa = half_sa(B.smn[s + 1][0], B.smn[s + 1][1], B.smn[s + 1][2], B.smx[s + 1][0], B.smx[s + 1][1],
                               B.smx[s + 1][2]);
    const double num = __dadd_rn(__dmul_rn(lsa, (double)lc), __dmul_rn(rsa, (double)rc));
    const double cost = parent_sa > 0 ? __ddiv_rn(num, parent_sa) : num;
    if (cost < S.best_cost) {
      S.best_cost = cost;
      S.best_axis = axis;
      S.best_split = s;
      S.nl = lc;
    }
  }
}

// Stable partition of A[b, b+c) by bin <= split through tmp (same range).
__device__ void cta_partition(const double* cen, uint32_t* A, uint32_t* tmp, uint32_t b, uint32_t c, int axis,
                              double cmin, double span, int bins, int split, uint32_t nl, Shared& S) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t left_base = 0, right_base = 0;
  for (uint32_t base = 0; base < c; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const bool valid = i < c;
    uint32_t t = 0;
    bool go_left = false;
    if (valid) {
      t = A[b + i];
      go_left = bin_of(cen[3 * (size_t)t + axis], cmin, span, bins) <= split;
    }
    const unsigned int m = __ballot_sync(0xFFFFFFFFu, valid && go_left);
    const unsigned int before = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) S.scan[w] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned int run = 0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
        const unsigned int x = S.scan[q];
        S.scan[q] = run;
        run += x;
      }
      S.scan[kWarps] = run;
    }
    __syncthreads();
    const uint32_t lrank = S.scan[w] + before;
    const uint32_t nleft = S.scan[kWarps];
    if (valid) {
      if (go_left) tmp[b + left_base + lrank] = t;
      else tmp[b + nl + right_base + (i - base - lrank)] = t;
    }
    const uint32_t chunk = min((uint32_t)blockDim.x, c - base);
    left_base += nleft;
    right_base += chunk - nleft;
    __syncthreads();
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) A[b + i] = tmp[b + i];
  __syncthreads();
}

// Bitonic sort of A[b, b+c) by (cen[axis], index), c <= kSortMax, in dynamic shared memory.
__device__ void cta_sort(const double* cen, uint32_t* A, uint32_t b, uint32_t c, int axis, double* keys,
                         uint32_t* vals) {
  uint32_t m = 1;
  while (m < c) m <<= 1;
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    if (i < c) {
      const uint32_t t = A[b + i];
      keys[i] = cen[3 * (size_t)t + axis];
      vals[i] = t;
    } else {
      keys[i] = INFINITY;
      vals[i] = 0xFFFFFFFFu;
    }
  }
  __syncthreads();
  for (uint32_t k = 2; k <= m; k <<= 1)
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          const double ki = keys[i], kl = keys[l];
          const uint32_t vi = vals[i], vl = vals[l];
          const bool gt = ki > kl || (ki == kl && vi > vl);
          if (gt == up) {
            keys[i] = kl; keys[l] = ki;
            vals[i] = vl; vals[l] = vi;
          }
        }
      }
      __syncthreads();
    }
  for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) A[b + i] = vals[i];
  __syncthreads();
}

struct Params {
  int max_leaf, bins, max_depth;
  int sort_cap;  // the shared-memory fallback sort's capacity at this level (a power of two <= kSortMax)
};

__global__ void __launch_bounds__(kThreads) k_level(GNode* __restrict__ nodes, const int32_t* __restrict__ level,
                                                    int n_level, const double* __restrict__ tb,
                                                    const double* __restrict__ cen, uint32_t* __restrict__ A,
                                                    uint32_t* __restrict__ tmp, int32_t* __restrict__ next,
                                                    int* __restrict__ counters, Params p) {
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ Shared S;
  const Bins B = bin_arrays(dyn, p.bins);
  const int id = level[blockIdx.x];
  GNode& N = nodes[id];
  const uint32_t b = N.begin, c = N.count;
  cta_bounds(tb, cen, A, b, c, S);
  if (threadIdx.x == 0) {
    for (int k = 0; k < 3; ++k) {
      N.mn[k] = (float)S.nb[k];
      N.mx[k] = (float)S.nb[3 + k];
    }
    N.left = N.right = -1;
    N.axis = -1;
    N.big_sort = 0;
    S.best_cost = INFINITY;
    S.best_axis = 0;
    S.best_split = 0;
    S.nl = 0;
    S.decision = 0;
    if ((int)c > p.max_leaf && (int)N.depth >= p.max_depth) atomicOr(&counters[2], 1);  // depth cap: error
  }
  __syncthreads();
  if ((int)c <= p.max_leaf || (int)N.depth >= p.max_depth) return;
  const double parent_sa = half_sa(S.nb[0], S.nb[1], S.nb[2], S.nb[3], S.nb[4], S.nb[5]);
  for (int axis = 0; axis < 3; ++axis) {
    const double span = __dsub_rn(S.nb[9 + axis], S.nb[6 + axis]);
    if (span <= 1e-9) continue;
    cta_bins(tb, cen, A, b, c, axis, S.nb[6 + axis], span, p.bins, B);
    if (threadIdx.x == 0) choose(axis, p.bins, parent_sa, B, S);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (S.best_cost < (double)c && S.best_cost != INFINITY) {
      S.decision = 1;
    } else {
      int ax = 0;
      double widest = __dsub_rn(S.nb[9], S.nb[6]);
      for (int k = 1; k < 3; ++k) {
        const double wk = __dsub_rn(S.nb[9 + k], S.nb[6 + k]);
        if (wk > widest) { ax = k; widest = wk; }
      }
      S.best_axis = ax;
      S.nl = (int)(c / 2);
      S.decision = c <= (uint32_t)p.sort_cap ? 2 : 3;
    }
  }
  __syncthreads();
  const int ax = S.best_axis;
  if (S.decision == 1) {
    const double span = __dsub_rn(S.nb[9 + ax], S.nb[6 + ax]);
    cta_partition(cen, A, tmp, b, c, ax, S.nb[6 + ax], span, p.bins, S.best_split, (uint32_t)S.nl, S);
  } else if (S.decision == 2) {
    double* keys = reinterpret_cast<double*>(dyn + bin_bytes(p.bins));
    uint32_t* vals = reinterpret_cast<uint32_t*>(keys + p.sort_cap);
    cta_sort(cen, A, b, c, ax, keys, vals);
  }
  if (threadIdx.x == 0) {
    N.axis = ax;
    if (S.decision == 3) {
      N.big_sort = 1;
      atomicOr(&counters[3], 1);
    }
    const int l = atomicAdd(&counters[0], 2);
    N.left = l;
    N.right = l + 1;
    GNode& L = nodes[l];
    GNode& R = nodes[l + 1];
    L.begin = b;
    L.count = (uint32_t)S.nl;
    L.depth = N.depth + 1;
    R.begin = b + (uint32_t)S.nl;
    R.count = c - (uint32_t)S.nl;
    R.depth = N.depth + 1;
    atomicMax(&counters[4], max(S.nl, (int)(c - (uint32_t)S.nl)));  // the next level's largest node
    const int q = atomicAdd(&counters[1], 2);
    next[q] = l;
    next[q + 1] = l + 1;
  }
}

__global__ void k_sizes(GNode* nodes, const int32_t* level, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  GNode& N = nodes[level[i]];
  N.size = N.left < 0 ? 1u : 1u + nodes[N.left].size + nodes[N.right].size;
}

__global__ void k_preorder(GNode* nodes, const int32_t* level, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const GNode& N = nodes[level[i]];
  if (N.left < 0) return;
  nodes[N.left].pre = N.pre + 1;
  nodes[N.right].pre = N.pre + 1 + nodes[N.left].size;
}

// Keys of the large fallback sort: -0 canonicalised to +0 (the reference's
// comparator subtracts, so equal centroids tie and fall to the index), then
// mapped to order-preserving integers.
__global__ void k_sort_keys(const double* __restrict__ cen, const uint32_t* __restrict__ A, uint32_t c, int axis,
                            unsigned long long* __restrict__ keys) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c) return;
  double v = cen[3 * (size_t)A[i] + axis];
  if (v == 0.0) v = 0.0;
  keys[i] = okey(v);
}

__global__ void k_emit(const GNode* nodes, int n, BinaryNode* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const GNode& N = nodes[i];
  BinaryNode o;
  for (int k = 0; k < 3; ++k) { o.mn[k] = N.mn[k]; o.mx[k] = N.mx[k]; }
  if (N.left < 0) {
    o.w6 = N.begin;
    o.w7 = kLeafFlag | N.count;
  } else {
    o.w6 = nodes[N.right].pre - N.pre;
    o.w7 = (uint32_t)N.axis;
  }
  out[N.pre] = o;
}

}  // namespace

// Sorts A[0, c) by (cen[axis], index) with two stable device radix passes.
static void sort_segment_device(const double* cen, uint32_t* A, uint32_t c, int axis, cudaStream_t s) {
  ScratchBuffer<uint32_t> a2(c, s);
  ScratchBuffer<unsigned long long> k1(c, s), k2(c, s);
  size_t t1 = 0, t2 = 0;
  VT_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, t1, A, a2.ptr, (int)c, 0, 32, s));
  VT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t2, k1.ptr, k2.ptr, a2.ptr, A, (int)c, 0, 64, s));
  ScratchBuffer<unsigned char> tmp(std::max(t1, t2), s);
  size_t tb = tmp.count;
  VT_CUDA(cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, A, a2.ptr, (int)c, 0, 32, s));  // by index
  k_sort_keys<<<(c + 255) / 256, 256, 0, s>>>(cen, a2.ptr, c, axis, k1.ptr);
  VT_CUDA(cudaGetLastError());
  tb = tmp.count;
  VT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, tb, k1.ptr, k2.ptr, a2.ptr, A, (int)c, 0, 64, s));  // stable
  VT_CUDA(cudaStreamSynchronize(s));
}

BinaryBvhHost build_binary_gpu(const float* d_pos, size_t position_words, const uint32_t* d_idx, size_t index_words,
                               const BuildOptions& o, cudaStream_t s, BinaryBvhDevice* keep) {
  validate_options(o);
  if (position_words % o.position_stride) fail(VT_ERR_RANGE, "positions.length must be divisible by positionStride");
  if (index_words % o.index_stride) fail(VT_ERR_RANGE, "indices.length must be divisible by indexStride");
  const size_t ntri = index_words / o.index_stride;
  BinaryBvhHost out;
  if (ntri == 0) {
    BinaryNode n{};
    n.w7 = kLeafFlag;
    out.nodes.push_back(n);
    return out;
  }
  if (ntri >= (1u << 30)) fail(VT_ERR_RANGE, "too many triangles for one tree");
  ScratchBuffer<double> tb(6 * ntri, s), cen(3 * ntri, s);
  DeviceBuffer<uint32_t> A(ntri);
  ScratchBuffer<uint32_t> tmp(ntri, s);
  ScratchBuffer<GNode> nodes(2 * ntri, s);
  ScratchBuffer<int32_t> lvl_a(ntri + 2, s), lvl_b(ntri + 2, s), ids(ntri + 2, s);
  ScratchBuffer<int> counters(5, s);  // nodes, next-level size, depth error, large sorts, largest next node
  VT_CUDA(cudaMemsetAsync(counters.ptr, 0, 5 * sizeof(int), s));
  k_prep<<<(unsigned)((ntri + 255) / 256), 256, 0, s>>>(d_pos, o.position_stride, position_words / o.position_stride,
                                                        d_idx, o.index_stride, (uint32_t)ntri, tb.ptr, cen.ptr, A.ptr,
                                                        counters.ptr + 3);
  VT_CUDA(cudaGetLastError());
  {
    int bad = 0;
    VT_CUDA(cudaMemcpyAsync(&bad, counters.ptr + 3, sizeof bad, cudaMemcpyDeviceToHost, s));
    VT_CUDA(cudaStreamSynchronize(s));
    if (bad & 1) fail(VT_ERR_RANGE, "a triangle references an out-of-range vertex");
    if (bad & 2) fail(VT_ERR_RANGE, "positions must be finite");
  }
  GNode root{};
  root.begin = 0;
  root.count = (uint32_t)ntri;
  root.depth = 0;
  root.pre = 0;
  VT_CUDA(cudaMemcpyAsync(nodes.ptr, &root, sizeof root, cudaMemcpyHostToDevice, s));
  const int zero_one[5] = {1, 0, 0, 0, 0};
  VT_CUDA(cudaMemcpyAsync(counters.ptr, zero_one, sizeof zero_one, cudaMemcpyHostToDevice, s));
  int32_t root_id = 0;
  VT_CUDA(cudaMemcpyAsync(lvl_a.ptr, &root_id, sizeof root_id, cudaMemcpyHostToDevice, s));
  static bool attr = false;
  if (!attr) {
    const size_t most = bin_bytes(kMaxBins) + (size_t)kSortMax * (sizeof(double) + sizeof(uint32_t));
    VT_CUDA(cudaFuncSetAttribute(k_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most));
    attr = true;
  }
  Params p{o.max_leaf, o.bins, o.max_depth, kSortMax};
  uint32_t level_max = (uint32_t)ntri;  // the largest node of the current level
  // levels: node ids of each level kept for the size / preorder passes
  std::vector<std::vector<int32_t>> levels;
  std::vector<int32_t> cur = {0};
  ScratchBuffer<int32_t>* in = &lvl_a;
  ScratchBuffer<int32_t>* nx = &lvl_b;
  while (!cur.empty()) {
    levels.push_back(cur);
    VT_CUDA(cudaMemsetAsync(counters.ptr + 1, 0, sizeof(int), s));
    VT_CUDA(cudaMemsetAsync(counters.ptr + 4, 0, sizeof(int), s));
    // launch shape from the level's largest node: small nodes get small CTAs and
    // little shared memory, so that many of them run on each SM at once
    const int threads = level_max >= 2048 ? kThreads : level_max >= 256 ? 256 : level_max >= 64 ? 128 : 64;
    uint32_t cap = 1;
    while (cap < level_max && cap < (uint32_t)kSortMax) cap <<= 1;
    p.sort_cap = (int)cap;
    const size_t dyn = bin_bytes(o.bins) + (size_t)cap * (sizeof(double) + sizeof(uint32_t));
    k_level<<<(unsigned)cur.size(), threads, dyn, s>>>(nodes.ptr, in->ptr, (int)cur.size(), tb.ptr, cen.ptr, A.ptr,
                                                       tmp.ptr, nx->ptr, counters.ptr, p);
    VT_CUDA(cudaGetLastError());
    int cnt[5];
    VT_CUDA(cudaMemcpyAsync(cnt, counters.ptr, sizeof cnt, cudaMemcpyDeviceToHost, s));
    VT_CUDA(cudaStreamSynchronize(s));
    if (cnt[2]) {
      fail(VT_ERR_BUILD, "maxDepth=" + std::to_string(o.max_depth) + " prevents enforcing maxLeafTriangles=" +
                             std::to_string(o.max_leaf));
    }
    if (cnt[3]) {
      // fallback sorts of nodes too large for the shared-memory sort (rare): device radix passes
      for (int32_t idn : cur) {
        GNode N;
        VT_CUDA(cudaMemcpyAsync(&N, nodes.ptr + idn, sizeof N, cudaMemcpyDeviceToHost, s));
        VT_CUDA(cudaStreamSynchronize(s));
        if (N.big_sort) sort_segment_device(cen.ptr, A.ptr + N.begin, N.count, N.axis, s);
      }
      VT_CUDA(cudaMemsetAsync(counters.ptr + 3, 0, sizeof(int), s));
    }
    std::vector<int32_t> next(cnt[1]);
    if (cnt[1]) {
      VT_CUDA(cudaMemcpyAsync(next.data(), nx->ptr, cnt[1] * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      VT_CUDA(cudaStreamSynchronize(s));
    }
    std::swap(in, nx);
    cur = std::move(next);
    level_max = (uint32_t)cnt[4];
  }
  int total = 0;
  VT_CUDA(cudaMemcpyAsync(&total, counters.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaStreamSynchronize(s));
  // subtree sizes bottom-up, preorder indices top-down
  for (int L = (int)levels.size() - 1; L >= 0; --L) {
    // on the build's stream: a plain copy from pageable memory can return before
    // it lands, and a kernel on a non-blocking stream would not wait for it
    VT_CUDA(cudaMemcpyAsync(ids.ptr, levels[L].data(), levels[L].size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    k_sizes<<<(unsigned)((levels[L].size() + 255) / 256), 256, 0, s>>>(nodes.ptr, ids.ptr, (int)levels[L].size());
    VT_CUDA(cudaStreamSynchronize(s));
  }
  for (size_t L = 0; L < levels.size(); ++L) {
    // on the build's stream: a plain copy from pageable memory can return before
    // it lands, and a kernel on a non-blocking stream would not wait for it
    VT_CUDA(cudaMemcpyAsync(ids.ptr, levels[L].data(), levels[L].size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    k_preorder<<<(unsigned)((levels[L].size() + 255) / 256), 256, 0, s>>>(nodes.ptr, ids.ptr, (int)levels[L].size());
    VT_CUDA(cudaStreamSynchronize(s));
  }
  DeviceBuffer<BinaryNode> dout(total);
  k_emit<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(nodes.ptr, total, dout.ptr);
  VT_CUDA(cudaGetLastError());
  out.nodes.resize(total);
  out.reordered_to_source.resize(ntri);
  VT_CUDA(cudaMemcpyAsync(out.nodes.data(), dout.ptr, total * sizeof(BinaryNode), cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaMemcpyAsync(out.reordered_to_source.data(), A.ptr, ntri * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaStreamSynchronize(s));
  // deepest internal node: the last level holds only leaves
  out.depth = levels.size() >= 2 ? (int)levels.size() - 2 : 0;
  if (keep) {
    keep->nodes = std::move(dout);
    keep->order = std::move(A);
    keep->n_nodes = (size_t)total;
    keep->ntri = ntri;
  }
  return out;
}

}  // namespace vt
