// tlas_build_gpu.cu -- the top level over instance AABBs built on the GPU,
// identical to build_tlas_host (the reference's buildTlas,
// packages/shared-bvh/src/tlas.ts:859-989) word for word.
//
// Top down, one level of the tree per launch, one CTA per node of the level
// (as the triangle build): the CTA reduces bounds, centroid bounds and per-bin
// bounds in the host's sequence order (a minimum or maximum keeps the earlier
// of two equal values, as std::min / std::max over the instance list do, so
// signed zeros agree), one thread runs the cost sweeps in the host's
// arithmetic, the node's instance range is partitioned stably (CTA scan) or
// sorted by (centroid, instance) for the balanced fallback (bitonic in global
// memory), and its two children are appended to the next level.  Then
// subtree sizes bottom up, preorder numbers top down (the host's recursion
// order), interior bounds bottom up, and the nodes are written in preorder.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "bvh_host.h"
#include "vt_common.h"

namespace vt {

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxBins = 256;

struct TNode {
  uint32_t begin, count;
  int depth;
  int left, right;   // child node ids (creation order), -1: leaf
  int axis;
  uint32_t size, pre;
};

struct TShared {
  int error;
  double vred[kWarps];
  unsigned int pred[kWarps];
  double cb[6];  // centroid bounds
  unsigned int bc[kMaxBins];
  double bmn[kMaxBins][3], bmx[kMaxBins][3];
  double lsa[kMaxBins], rsa[kMaxBins];
  unsigned long long lc[kMaxBins], rc[kMaxBins];
  int have, baxis, bbin, fallback, axis;
  double bcost;
  unsigned int scan[kWarps + 1];
  unsigned int nl;
};

__device__ __forceinline__ double smin_(double acc, double x) { return x < acc ? x : acc; }  // std::min(acc, x)
__device__ __forceinline__ double smax_(double acc, double x) { return acc < x ? x : acc; }  // std::max(acc, x)

// (value, position) reduction of the CTA: the extreme value, the earliest
// position among equals (the value a sequential std::min / std::max keeps).
__device__ double cta_first_extreme(double v, unsigned int pos, bool is_min, TShared& S) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_down_sync(0xFFFFFFFFu, v, o);
    const unsigned int op = __shfl_down_sync(0xFFFFFFFFu, pos, o);
    const bool better = is_min ? (ov < v || (ov == v && op < pos)) : (ov > v || (ov == v && op < pos));
    if (better) { v = ov; pos = op; }
  }
  if (lane == 0) { S.vred[w] = v; S.pred[w] = pos; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bv = S.vred[0];
    unsigned int bp = S.pred[0];
    for (int q = 1; q < kWarps; ++q) {
      const double ov = S.vred[q];
      const unsigned int op = S.pred[q];
      const bool better = is_min ? (ov < bv || (ov == bv && op < bp)) : (ov > bv || (ov == bv && op < bp));
      if (better) { bv = ov; bp = op; }
    }
    S.vred[0] = bv;
  }
  __syncthreads();
  const double r = S.vred[0];
  __syncthreads();
  return r;
}

__device__ int tlas_bin(double c, double cmin, double ext, int bins) {
  const double t = floor(__dmul_rn(__ddiv_rn(__dsub_rn(c, cmin), ext), (double)bins));
  const double lo = 0.0 < t ? t : 0.0;                                  // std::max(0.0, t)
  const double hi = lo < (double)(bins - 1) ? lo : (double)(bins - 1);  // std::min<double>(bins - 1, .)
  return (int)hi;
}

__device__ double area2(const double* mn, const double* mx) {
  double d[3];
  for (int k = 0; k < 3; ++k) {
    const double x = __dsub_rn(mx[k], mn[k]);
    d[k] = 0.0 < x ? x : 0.0;
  }
  return __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[1]), __dmul_rn(d[1], d[2])), __dmul_rn(d[2], d[0])));
}

__device__ int min_balanced_depth(unsigned int count, int max_leaf) {
  const unsigned int leaves = (count + (unsigned int)max_leaf - 1u) / (unsigned int)max_leaf;
  return leaves <= 1 ? 0 : (int)ceil(log2((double)leaves));
}

// One node of the level per CTA.  counters: [0] nodes created, [1] next-level
// size, [2] error (1: depth).
__global__ void __launch_bounds__(kThreads) k_tlas_level(
    const double* __restrict__ mn, const double* __restrict__ mx, const double* __restrict__ cen,
    const int32_t* __restrict__ level, int max_leaf, int bins, int max_depth, uint32_t* __restrict__ W,
    uint32_t* __restrict__ tmp, double* __restrict__ skey, uint32_t* __restrict__ sval, TNode* __restrict__ nodes,
    double* __restrict__ nmn, double* __restrict__ nmx, int32_t* __restrict__ next, int* __restrict__ counters) {
  __shared__ TShared S;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ni = level[blockIdx.x];
  const TNode it = nodes[ni];
  const uint32_t b = it.begin, c = it.count;
  if ((int)c <= max_leaf) {
    // leaf: bounds over its instances, in list order
    for (int k = 0; k < 6; ++k) {
      const bool is_min = k < 3;
      double v = is_min ? INFINITY : -INFINITY;
      unsigned int pos = 0xFFFFFFFFu;
      for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
        const uint32_t r = W[b + i];
        const double x = is_min ? mn[3 * (size_t)r + k] : mx[3 * (size_t)r + (k - 3)];
        const bool better = is_min ? (x < v) : (x > v);
        if (pos == 0xFFFFFFFFu || better) { v = x; pos = i; }
      }
      const double red = cta_first_extreme(v, pos, is_min, S);
      if (threadIdx.x == 0) {
        if (is_min) nmn[3 * (size_t)ni + k] = smin_(INFINITY, red);
        else nmx[3 * (size_t)ni + (k - 3)] = smax_(-INFINITY, red);
      }
    }
    if (threadIdx.x == 0) {
      nodes[ni].left = nodes[ni].right = -1;
      nodes[ni].axis = -1;
    }
    return;
  }
  if (threadIdx.x == 0)
    S.error = (it.depth >= max_depth || min_balanced_depth(c, max_leaf) > max_depth - it.depth) ? 1 : 0;
  __syncthreads();
  if (S.error) {
    if (threadIdx.x == 0) atomicOr(&counters[2], 1);
    return;
  }
  // centroid bounds, in list order
  for (int k = 0; k < 6; ++k) {
    const bool is_min = k < 3;
    double v = is_min ? INFINITY : -INFINITY;
    unsigned int pos = 0xFFFFFFFFu;
    for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
      const double x = cen[3 * (size_t)W[b + i] + (k % 3)];
      const bool better = is_min ? (x < v) : (x > v);
      if (pos == 0xFFFFFFFFu || better) { v = x; pos = i; }
    }
    const double red = cta_first_extreme(v, pos, is_min, S);
    if (threadIdx.x == 0) S.cb[k] = is_min ? smin_(INFINITY, red) : smax_(-INFINITY, red);
  }
  __syncthreads();
  double ext[3];
  for (int k = 0; k < 3; ++k) ext[k] = __dsub_rn(S.cb[3 + k], S.cb[k]);
  if (threadIdx.x == 0) {
    S.have = 0;
    S.baxis = 0;
    S.bbin = 0;
    S.bcost = 0.0;
  }
  __syncthreads();
  if (!(ext[0] <= 0 && ext[1] <= 0 && ext[2] <= 0)) {
    for (int axis = 0; axis < 3; ++axis) {
      if (ext[axis] <= 0) continue;
      // per-bin count and bounds: warp q reduces bins q, q + 16, ... over the list in order
      for (int bin = w; bin < bins; bin += kWarps) {
        double v[6];
        unsigned int p[6];
        for (int k = 0; k < 6; ++k) { v[k] = k < 3 ? INFINITY : -INFINITY; p[k] = 0xFFFFFFFFu; }
        unsigned int cnt = 0;
        for (uint32_t i = lane; i < c; i += 32) {
          const uint32_t r = W[b + i];
          if (tlas_bin(cen[3 * (size_t)r + axis], S.cb[axis], ext[axis], bins) != bin) continue;
          ++cnt;
          for (int k = 0; k < 6; ++k) {
            const double x = k < 3 ? mn[3 * (size_t)r + k] : mx[3 * (size_t)r + (k - 3)];
            const bool better = k < 3 ? (x < v[k]) : (x > v[k]);
            if (p[k] == 0xFFFFFFFFu || better) { v[k] = x; p[k] = i; }
          }
        }
        for (int o = 16; o > 0; o >>= 1) {
          cnt += __shfl_down_sync(0xFFFFFFFFu, cnt, o);
          for (int k = 0; k < 6; ++k) {
            const double ov = __shfl_down_sync(0xFFFFFFFFu, v[k], o);
            const unsigned int op = __shfl_down_sync(0xFFFFFFFFu, p[k], o);
            const bool better = k < 3 ? (ov < v[k] || (ov == v[k] && op < p[k]))
                                      : (ov > v[k] || (ov == v[k] && op < p[k]));
            if (better) { v[k] = ov; p[k] = op; }
          }
        }
        if (lane == 0) {
          S.bc[bin] = cnt;
          for (int k = 0; k < 3; ++k) {
            S.bmn[bin][k] = smin_(INFINITY, v[k]);
            S.bmx[bin][k] = smax_(-INFINITY, v[3 + k]);
          }
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        unsigned long long cc = 0;
        for (int bb = 0; bb < bins; ++bb) {
          if (S.bc[bb]) {
            for (int k = 0; k < 3; ++k) { lo[k] = smin_(lo[k], S.bmn[bb][k]); hi[k] = smax_(hi[k], S.bmx[bb][k]); }
            cc += S.bc[bb];
          }
          S.lsa[bb] = area2(lo, hi);
          S.lc[bb] = cc;
        }
        for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
        cc = 0;
        for (int bb = bins - 1; bb >= 0; --bb) {
          if (S.bc[bb]) {
            for (int k = 0; k < 3; ++k) { lo[k] = smin_(lo[k], S.bmn[bb][k]); hi[k] = smax_(hi[k], S.bmx[bb][k]); }
            cc += S.bc[bb];
          }
          S.rsa[bb] = area2(lo, hi);
          S.rc[bb] = cc;
        }
        const double total = S.lsa[bins - 1];
        if (total > 0) {
          for (int bb = 0; bb < bins - 1; ++bb) {
            if (S.lc[bb] == 0 || S.rc[bb + 1] == 0) continue;
            const double sah = __ddiv_rn(__dadd_rn(__dmul_rn((double)S.lc[bb], S.lsa[bb]),
                                                   __dmul_rn((double)S.rc[bb + 1], S.rsa[bb + 1])), total);
            if (!S.have || sah < S.bcost) {
              S.have = 1;
              S.baxis = axis;
              S.bbin = bb;
              S.bcost = sah;
            }
          }
        }
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    S.axis = S.have ? S.baxis : 0;
    S.fallback = (!S.have || S.bcost >= (double)c) ? 1 : 0;
  }
  __syncthreads();
  if (!S.fallback) {
    // stable partition of the list into tmp by bin <= bbin: the left count first
    const int ax = S.baxis, split = S.bbin;
    unsigned int nleft_total = 0;
    for (uint32_t base = 0; base < c; base += blockDim.x) {
      const uint32_t i = base + threadIdx.x;
      const bool go = i < c && tlas_bin(cen[3 * (size_t)W[b + i] + ax], S.cb[ax], ext[ax], bins) <= split;
      const unsigned int m = __ballot_sync(0xFFFFFFFFu, go);
      if (lane == 0) S.scan[w] = __popc(m);
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned int t = 0;
        for (int q = 0; q < kWarps; ++q) t += S.scan[q];
        S.scan[kWarps] = t;
      }
      __syncthreads();
      nleft_total += S.scan[kWarps];
      __syncthreads();
    }
    uint32_t left_base = 0, right_base = 0;
    for (uint32_t base = 0; base < c; base += blockDim.x) {
      const uint32_t i = base + threadIdx.x;
      const bool valid = i < c;
      uint32_t r = 0;
      bool go = false;
      if (valid) {
        r = W[b + i];
        go = tlas_bin(cen[3 * (size_t)r + ax], S.cb[ax], ext[ax], bins) <= split;
      }
      const unsigned int m = __ballot_sync(0xFFFFFFFFu, valid && go);
      const unsigned int before = __popc(m & ((1u << lane) - 1u));
      if (lane == 0) S.scan[w] = __popc(m);
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned int run = 0;
        for (int q = 0; q < kWarps; ++q) {
          const unsigned int x = S.scan[q];
          S.scan[q] = run;
          run += x;
        }
        S.scan[kWarps] = run;
      }
      __syncthreads();
      const uint32_t lrank = S.scan[w] + before;
      if (valid) {
        if (go) tmp[b + left_base + lrank] = r;
        else tmp[b + nleft_total + right_base + (i - base - lrank)] = r;
      }
      const uint32_t chunk = min((uint32_t)blockDim.x, c - base);
      left_base += S.scan[kWarps];
      right_base += chunk - S.scan[kWarps];
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      const unsigned int nr = c - nleft_total;
      const bool bad = nleft_total == 0 || nr == 0 ||
                       min_balanced_depth(nleft_total, max_leaf) > max_depth - (it.depth + 1) ||
                       min_balanced_depth(nr, max_leaf) > max_depth - (it.depth + 1);
      S.fallback = bad ? 1 : 0;
      S.nl = nleft_total;
    }
    __syncthreads();
    if (!S.fallback)
      for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) W[b + i] = tmp[b + i];
    __syncthreads();
  }
  if (S.fallback) {
    if (threadIdx.x == 0) {
      int axis = 0;
      if (ext[1] > ext[axis]) axis = 1;
      if (ext[2] > ext[axis]) axis = 2;
      S.axis = axis;
      S.nl = c / 2;
    }
    __syncthreads();
    // bitonic sort of the list by (centroid on the axis, instance) in this node's
    // scratch range [2b, 2b + 2c) (disjoint from every other node of the level)
    const int ax = S.axis;
    uint32_t m2 = 1;
    while (m2 < c) m2 <<= 1;
    double* keys = skey + 2 * (size_t)b;
    uint32_t* vals = sval + 2 * (size_t)b;
    for (uint32_t i = threadIdx.x; i < m2; i += blockDim.x) {
      if (i < c) {
        const uint32_t r = W[b + i];
        keys[i] = cen[3 * (size_t)r + ax];
        vals[i] = r;
      } else {
        keys[i] = INFINITY;
        vals[i] = 0xFFFFFFFFu;
      }
    }
    __syncthreads();
    for (uint32_t k = 2; k <= m2; k <<= 1)
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t i = threadIdx.x; i < m2; i += blockDim.x) {
          const uint32_t l = i ^ j;
          if (l > i) {
            const bool up = (i & k) == 0;
            const double ki = keys[i], kl = keys[l];
            const uint32_t vi = vals[i], vl = vals[l];
            // the host's comparator: d = a - b; d != 0 ? d < 0 : instance order (padding last)
            const double d = __dsub_rn(ki, kl);
            const bool gt = (ki == INFINITY && kl == INFINITY) ? vi > vl : (d != 0 ? d > 0 : vi > vl);
            if (gt == up) {
              keys[i] = kl; keys[l] = ki;
              vals[i] = vl; vals[l] = vi;
            }
          }
        }
        __syncthreads();
      }
    for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) W[b + i] = vals[i];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int l = atomicAdd(&counters[0], 2);
    nodes[ni].left = l;
    nodes[ni].right = l + 1;
    nodes[ni].axis = S.axis;
    TNode L{}, R{};
    L.begin = b;
    L.count = S.nl;
    L.depth = it.depth + 1;
    R.begin = b + S.nl;
    R.count = c - S.nl;
    R.depth = it.depth + 1;
    nodes[l] = L;
    nodes[l + 1] = R;
    const int q = atomicAdd(&counters[1], 2);
    next[q] = l;
    next[q + 1] = l + 1;
  }
}

__global__ void k_tlas_sizes_bounds(TNode* nodes, const int32_t* level, int n, double* nmn, double* nmx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int id = level[i];
  TNode& N = nodes[id];
  if (N.left < 0) {
    N.size = 1;
    return;
  }
  N.size = 1u + nodes[N.left].size + nodes[N.right].size;
  for (int k = 0; k < 3; ++k) {
    nmn[3 * (size_t)id + k] = smin_(nmn[3 * (size_t)N.left + k], nmn[3 * (size_t)N.right + k]);
    nmx[3 * (size_t)id + k] = smax_(nmx[3 * (size_t)N.left + k], nmx[3 * (size_t)N.right + k]);
  }
}

__global__ void k_tlas_preorder(TNode* nodes, const int32_t* level, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TNode& N = nodes[level[i]];
  if (N.left < 0) return;
  nodes[N.left].pre = N.pre + 1;
  nodes[N.right].pre = N.pre + 1 + nodes[N.left].size;
}

__global__ void k_tlas_emit(const TNode* nodes, int n, const double* nmn, const double* nmx, BinaryNode* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TNode& N = nodes[i];
  BinaryNode o;
  for (int k = 0; k < 3; ++k) {
    o.mn[k] = (float)nmn[3 * (size_t)i + k];
    o.mx[k] = (float)nmx[3 * (size_t)i + k];
  }
  if (N.left < 0) {
    o.w6 = N.begin;
    o.w7 = kLeafFlag | N.count;
  } else {
    o.w6 = nodes[N.right].pre - N.pre;
    o.w7 = (uint32_t)N.axis;
  }
  out[N.pre] = o;
}

__global__ void k_tlas_prep(const double* __restrict__ aabbs, uint32_t n, double* __restrict__ mn,
                            double* __restrict__ mx, double* __restrict__ cen, uint32_t* __restrict__ W) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  W[i] = i;
  for (int k = 0; k < 3; ++k) {
    const double a = aabbs[6 * (size_t)i + k], b = aabbs[6 * (size_t)i + 3 + k];
    mn[3 * (size_t)i + k] = a;
    mx[3 * (size_t)i + k] = b;
    cen[3 * (size_t)i + k] = __dmul_rn(__dadd_rn(a, b), 0.5);
  }
}

}  // namespace

BinaryBvhHost build_tlas_gpu(const double* aabbs, size_t n, int max_leaf, int bins, int max_depth, cudaStream_t s,
                             BinaryBvhDevice* keep) {
  if (n == 0) fail(VT_ERR_INVALID_ARGUMENT, "buildTlas: instances list is empty");
  if (bins < 2 || bins > kMaxBins) fail(VT_ERR_RANGE, "binCount must be in [2, 256]");
  if (max_leaf < 1 || max_leaf > 4) fail(VT_ERR_RANGE, "maxLeaf must be in [1, 4]");
  if (n >= (1u << 30)) fail(VT_ERR_RANGE, "too many instances for one top level");
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      const double a = aabbs[6 * i + k], b = aabbs[6 * i + 3 + k];
      if (!std::isfinite(a) || !std::isfinite(b)) fail(VT_ERR_RANGE, "instance AABB is not finite");
      if (b < a) fail(VT_ERR_RANGE, "instance AABB is inverted");
    }
  {
    const size_t leaves = (n + max_leaf - 1) / max_leaf;
    const int need = leaves <= 1 ? 0 : (int)std::ceil(std::log2((double)leaves));
    if (need > max_depth) fail(VT_ERR_RANGE, "instances cannot fit the traversal-safe depth");
  }
  ScratchBuffer<double> d_aabbs(6 * n, s), mn(3 * n, s), mx(3 * n, s), cen(3 * n, s), skey(2 * n, s),
      nmn(3 * 2 * n, s), nmx(3 * 2 * n, s);
  DeviceBuffer<uint32_t> W(n);
  ScratchBuffer<uint32_t> tmp(n, s), sval(2 * n, s);
  ScratchBuffer<TNode> tn(2 * n, s);
  ScratchBuffer<int32_t> lvl_a(n + 2, s), lvl_b(n + 2, s), ids(n + 2, s);
  ScratchBuffer<int> counters(3, s);
  VT_CUDA(cudaMemcpyAsync(d_aabbs.ptr, aabbs, 6 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  k_tlas_prep<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_aabbs.ptr, (uint32_t)n, mn.ptr, mx.ptr, cen.ptr, W.ptr);
  VT_CUDA(cudaGetLastError());
  TNode root{};
  root.begin = 0;
  root.count = (uint32_t)n;
  root.left = root.right = -1;
  VT_CUDA(cudaMemcpyAsync(tn.ptr, &root, sizeof root, cudaMemcpyHostToDevice, s));
  const int init[3] = {1, 0, 0};
  VT_CUDA(cudaMemcpyAsync(counters.ptr, init, sizeof init, cudaMemcpyHostToDevice, s));
  const int32_t root_id = 0;
  VT_CUDA(cudaMemcpyAsync(lvl_a.ptr, &root_id, sizeof root_id, cudaMemcpyHostToDevice, s));
  std::vector<std::vector<int32_t>> levels;
  std::vector<int32_t> cur = {0};
  ScratchBuffer<int32_t>* in = &lvl_a;
  ScratchBuffer<int32_t>* nx = &lvl_b;
  while (!cur.empty()) {
    levels.push_back(cur);
    VT_CUDA(cudaMemsetAsync(counters.ptr + 1, 0, sizeof(int), s));
    k_tlas_level<<<(unsigned)cur.size(), kThreads, 0, s>>>(mn.ptr, mx.ptr, cen.ptr, in->ptr, max_leaf, bins, max_depth,
                                                           W.ptr, tmp.ptr, skey.ptr, sval.ptr, tn.ptr, nmn.ptr,
                                                           nmx.ptr, nx->ptr, counters.ptr);
    VT_CUDA(cudaGetLastError());
    int cnt[3];
    VT_CUDA(cudaMemcpyAsync(cnt, counters.ptr, sizeof cnt, cudaMemcpyDeviceToHost, s));
    VT_CUDA(cudaStreamSynchronize(s));
    if (cnt[2]) fail(VT_ERR_BUILD, "cannot encode the instances within the traversal-safe depth");
    std::vector<int32_t> next(cnt[1]);
    if (cnt[1]) {
      VT_CUDA(cudaMemcpyAsync(next.data(), nx->ptr, cnt[1] * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      VT_CUDA(cudaStreamSynchronize(s));
    }
    std::swap(in, nx);
    cur = std::move(next);
  }
  int total = 0;
  VT_CUDA(cudaMemcpyAsync(&total, counters.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaStreamSynchronize(s));
  // subtree sizes and interior bounds bottom up, preorder numbers top down
  for (int L = (int)levels.size() - 1; L >= 0; --L) {
    VT_CUDA(cudaMemcpyAsync(ids.ptr, levels[L].data(), levels[L].size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    k_tlas_sizes_bounds<<<(unsigned)((levels[L].size() + 255) / 256), 256, 0, s>>>(tn.ptr, ids.ptr,
                                                                                   (int)levels[L].size(), nmn.ptr,
                                                                                   nmx.ptr);
    VT_CUDA(cudaStreamSynchronize(s));
  }
  for (size_t L = 0; L < levels.size(); ++L) {
    VT_CUDA(cudaMemcpyAsync(ids.ptr, levels[L].data(), levels[L].size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    k_tlas_preorder<<<(unsigned)((levels[L].size() + 255) / 256), 256, 0, s>>>(tn.ptr, ids.ptr, (int)levels[L].size());
    VT_CUDA(cudaStreamSynchronize(s));
  }
  DeviceBuffer<BinaryNode> nodes(total);
  k_tlas_emit<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(tn.ptr, total, nmn.ptr, nmx.ptr, nodes.ptr);
  VT_CUDA(cudaGetLastError());
  BinaryBvhHost out;
  out.nodes.resize(total);
  out.reordered_to_source.resize(n);
  VT_CUDA(cudaMemcpyAsync(out.nodes.data(), nodes.ptr, total * sizeof(BinaryNode), cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaMemcpyAsync(out.reordered_to_source.data(), W.ptr, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaStreamSynchronize(s));
  if (keep) {
    keep->nodes = std::move(nodes);
    keep->order = std::move(W);
    keep->n_nodes = (size_t)total;
    keep->ntri = n;
  }
  return out;
}

}  // namespace vt
