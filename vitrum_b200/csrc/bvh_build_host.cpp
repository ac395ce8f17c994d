// bvh_build_host.cpp -- binned-SAH binary BVH, host reference build.
//
// Produces the same tree as the reference builder (buildArrayBvh,
// packages/shared-bvh/src/buildArrayBvh.ts:342-780): 16 bins per axis,
// axes skipped when the centroid span is <= 1e-9, cost
// (SA_L*N_L + SA_R*N_R)/SA_P with half-area SA (:223-231), leaf when the
// count is <= maxLeaf or the best cost is not below N, and the balanced
// median fallback on the widest centroid axis ordered by (centroid,
// triangle index) (:677-694).  All split arithmetic is IEEE double, as the
// reference's JS numbers are; node bounds are stored as f32 (:751-765).
// The subset order is kept stable through partitioning, so leaves list
// triangles in the reference's order and the packed output matches it word
// for word.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "bvh_host.h"
#include "vt_common.h"

namespace vt {

namespace {

inline double js_min(double a, double b) {
  if (a < b) return a;
  if (b < a) return b;
  return std::signbit(a) ? a : b;
}
inline double js_max(double a, double b) {
  if (a > b) return a;
  if (b > a) return b;
  return std::signbit(a) ? b : a;
}
inline double half_sa(double mnx, double mny, double mnz, double mxx, double mxy, double mxz) {
  double dx = mxx - mnx, dy = mxy - mny, dz = mxz - mnz;
  dx = dx > 0 ? dx : 0;
  dy = dy > 0 ? dy : 0;
  dz = dz > 0 ? dz : 0;
  return dx * dy + dy * dz + dz * dx;
}

struct Builder {
  const BuildOptions& o;
  std::vector<double> mn, mx, cen;  // 3 per triangle
  std::vector<BinaryNode> nodes;
  std::vector<uint32_t> ordered;
  std::vector<uint32_t> scratch;
  int max_depth_seen = 0;

  explicit Builder(const BuildOptions& opts) : o(opts) {}

  int bin_of(uint32_t t, int axis, double cmin, double span) const {
    double x = (cen[3 * t + axis] - cmin) / span;
    double f = std::floor(x * o.bins);
    return f < (double)(o.bins - 1) ? (int)f : o.bins - 1;
  }

  // Returns the node index; `a` is [begin, end) of the working index array.
  uint32_t build(uint32_t* a, size_t count, int depth) {
    uint32_t ni = (uint32_t)nodes.size();
    nodes.push_back(BinaryNode{});
    double nmn[3] = {INFINITY, INFINITY, INFINITY}, nmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    double cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = 0; i < count; ++i) {
      uint32_t t = a[i];
      for (int k = 0; k < 3; ++k) {
        nmn[k] = js_min(nmn[k], mn[3 * t + k]);
        nmx[k] = js_max(nmx[k], mx[3 * t + k]);
        cmn[k] = js_min(cmn[k], cen[3 * t + k]);
        cmx[k] = js_max(cmx[k], cen[3 * t + k]);
      }
    }
    for (int k = 0; k < 3; ++k) {
      nodes[ni].mn[k] = (float)nmn[k];
      nodes[ni].mx[k] = (float)nmx[k];
    }
    if ((int)count <= o.max_leaf) {
      nodes[ni].w6 = (uint32_t)ordered.size();
      nodes[ni].w7 = kLeafFlag | (uint32_t)count;
      ordered.insert(ordered.end(), a, a + count);
      return ni;
    }
    if (depth >= o.max_depth)
      fail(VT_ERR_BUILD, "maxDepth=" + std::to_string(o.max_depth) + " prevents enforcing maxLeafTriangles=" +
                             std::to_string(o.max_leaf) + ": depth " + std::to_string(depth) + " still contains " +
                             std::to_string(count) + " triangles");
    max_depth_seen = std::max(max_depth_seen, depth);
    const double parent_sa = half_sa(nmn[0], nmn[1], nmn[2], nmx[0], nmx[1], nmx[2]);
    const int K = o.bins;
    double best_cost = INFINITY;
    int best_axis = 0, best_split = 0;
    std::vector<double> bmn(3 * K), bmx(3 * K);
    std::vector<int> bc(K);
    std::vector<float> pmn(3 * K), pmx(3 * K), smn(3 * K), smx(3 * K);
    std::vector<int> pc(K), sc(K);
    for (int axis = 0; axis < 3; ++axis) {
      double span = cmx[axis] - cmn[axis];
      if (span <= 1e-9) continue;
      std::fill(bmn.begin(), bmn.end(), INFINITY);
      std::fill(bmx.begin(), bmx.end(), -INFINITY);
      std::fill(bc.begin(), bc.end(), 0);
      for (size_t i = 0; i < count; ++i) {
        uint32_t t = a[i];
        int b = bin_of(t, axis, cmn[axis], span);
        for (int k = 0; k < 3; ++k) {
          bmn[3 * b + k] = js_min(bmn[3 * b + k], mn[3 * t + k]);
          bmx[3 * b + k] = js_max(bmx[3 * b + k], mx[3 * t + k]);
        }
        bc[b] += 1;
      }
      double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      int c = 0;
      for (int i = 0; i < K; ++i) {
        for (int k = 0; k < 3; ++k) {
          lo[k] = js_min(lo[k], bmn[3 * i + k]);
          hi[k] = js_max(hi[k], bmx[3 * i + k]);
          pmn[3 * i + k] = (float)lo[k];
          pmx[3 * i + k] = (float)hi[k];
        }
        c += bc[i];
        pc[i] = c;
      }
      for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
      c = 0;
      for (int i = K - 1; i >= 0; --i) {
        for (int k = 0; k < 3; ++k) {
          lo[k] = js_min(lo[k], bmn[3 * i + k]);
          hi[k] = js_max(hi[k], bmx[3 * i + k]);
          smn[3 * i + k] = (float)lo[k];
          smx[3 * i + k] = (float)hi[k];
        }
        c += bc[i];
        sc[i] = c;
      }
      for (int s = 0; s < K - 1; ++s) {
        int lc = pc[s], rc = sc[s + 1];
        if (lc == 0 || rc == 0) continue;
        double lsa = half_sa(pmn[3 * s], pmn[3 * s + 1], pmn[3 * s + 2], pmx[3 * s], pmx[3 * s + 1], pmx[3 * s + 2]);
        double rsa = half_sa(smn[3 * s + 3], smn[3 * s + 4], smn[3 * s + 5], smx[3 * s + 3], smx[3 * s + 4],
                             smx[3 * s + 5]);
        double num = lsa * (double)lc + rsa * (double)rc;
        double cost = parent_sa > 0 ? num / parent_sa : num;
        if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = s; }
      }
    }
    int split_axis = best_axis;
    size_t nl = 0;
    bool done = false;
    if (best_cost < (double)count && best_cost != INFINITY) {
      double span = cmx[best_axis] - cmn[best_axis];
      if (scratch.size() < count) scratch.resize(count);
      size_t nr = 0;
      for (size_t i = 0; i < count; ++i) {
        if (bin_of(a[i], best_axis, cmn[best_axis], span) <= best_split) a[nl++] = a[i];
        else scratch[nr++] = a[i];
      }
      if (nl != 0 && nr != 0) {
        std::memcpy(a + nl, scratch.data(), nr * sizeof(uint32_t));
        done = true;
      } else if (nl == 0) {
        std::memcpy(a, scratch.data(), nr * sizeof(uint32_t));  // restore order (all went right)
      }
    }
    if (!done) {
      split_axis = 0;
      double widest = cmx[0] - cmn[0];
      for (int k = 1; k < 3; ++k)
        if (cmx[k] - cmn[k] > widest) { split_axis = k; widest = cmx[k] - cmn[k]; }
      const int ax = split_axis;
      std::sort(a, a + count, [&](uint32_t p, uint32_t q) {
        double d = cen[3 * p + ax] - cen[3 * q + ax];
        return d != 0 ? d < 0 : p < q;
      });
      nl = count / 2;
    }
    build(a, nl, depth + 1);
    uint32_t rc = build(a + nl, count - nl, depth + 1);
    nodes[ni].w6 = rc - ni;
    nodes[ni].w7 = (uint32_t)split_axis;
    return ni;
  }
};

}  // namespace

void validate_options(const BuildOptions& o) {
  if (o.position_stride != 3 && o.position_stride != 4) fail(VT_ERR_INVALID_ARGUMENT, "positionStride must be exactly 3 or 4");
  if (o.index_stride != 3 && o.index_stride != 4) fail(VT_ERR_INVALID_ARGUMENT, "indexStride must be exactly 3 or 4");
  if (o.max_leaf < 1 || o.max_leaf > 4)
    fail(VT_ERR_RANGE, "maxLeafTriangles must be in [1, 4] for 8-wide device nodes, got " + std::to_string(o.max_leaf));
  if (o.bins < 2 || o.bins > 256) fail(VT_ERR_RANGE, "binCount must be in [2, 256], got " + std::to_string(o.bins));
  if (o.traversal_tree < 1 || o.traversal_tree > 3) fail(VT_ERR_RANGE, "traversal_tree must be in [0, 3]");
  if (o.max_depth < 0 || o.max_depth > kMaxBinaryDepth)
    fail(VT_ERR_RANGE, "maxDepth must be in [0, 58], got " + std::to_string(o.max_depth));
}

BinaryBvhHost build_binary_host(const float* positions, size_t position_words, const uint32_t* indices,
                                size_t index_words, const BuildOptions& o) {
  validate_options(o);
  if (position_words % o.position_stride)
    fail(VT_ERR_RANGE, "positions.length must be divisible by positionStride");
  if (index_words % o.index_stride) fail(VT_ERR_RANGE, "indices.length must be divisible by indexStride");
  for (size_t i = 0; i < position_words; ++i)
    if (!std::isfinite(positions[i])) fail(VT_ERR_RANGE, "positions[" + std::to_string(i) + "] must be finite");
  const size_t ntri = index_words / o.index_stride;
  const size_t nvert = position_words / o.position_stride;
  BinaryBvhHost out;
  if (ntri == 0) {
    BinaryNode n{};
    n.w7 = kLeafFlag;
    out.nodes.push_back(n);
    return out;
  }
  Builder b(o);
  b.mn.resize(3 * ntri);
  b.mx.resize(3 * ntri);
  b.cen.resize(3 * ntri);
  for (size_t t = 0; t < ntri; ++t) {
    const uint32_t* iv = indices + t * o.index_stride;
    if (iv[0] >= nvert || iv[1] >= nvert || iv[2] >= nvert)
      fail(VT_ERR_RANGE, "triangle " + std::to_string(t) + " references an out-of-range vertex");
    for (int k = 0; k < 3; ++k) {
      double va = positions[(size_t)iv[0] * o.position_stride + k];
      double vb = positions[(size_t)iv[1] * o.position_stride + k];
      double vc = positions[(size_t)iv[2] * o.position_stride + k];
      double lo = js_min(js_min(va, vb), vc), hi = js_max(js_max(va, vb), vc);
      b.mn[3 * t + k] = lo;
      b.mx[3 * t + k] = hi;
      b.cen[3 * t + k] = 0.5 * (lo + hi);
    }
  }
  std::vector<uint32_t> work(ntri);
  std::iota(work.begin(), work.end(), 0u);
  b.nodes.reserve(2 * ntri);
  b.ordered.reserve(ntri);
  b.build(work.data(), ntri, 0);
  out.nodes = std::move(b.nodes);
  out.reordered_to_source = std::move(b.ordered);
  out.depth = b.max_depth_seen;
  return out;
}

// ---------------------------------------------------------------- TLAS
// The reference's buildTlas (shared-bvh/src/tlas.ts:330-579): per node the
// centroid AABB, 16 bins on every axis with a positive centroid extent,
// prefix/suffix unions of non-empty bins, cost (N_L*SA_L + N_R*SA_R)/SA_total
// with full surface area, leaf of <= max_leaf instances, and the balanced
// median split (widest centroid axis, ties by input index) when the SAH is
// degenerate, not improving, empty-sided or would exceed the depth budget.
// Interior bounds are the union of the two children (:562-575).
namespace {

struct TRec {
  uint32_t orig;
  double cen[3], mn[3], mx[3];
};

struct TlasBuilder {
  std::vector<TRec> recs;
  std::vector<BinaryNode> nodes;
  std::vector<double> nmn, nmx;  // exact (double) node bounds, 3 per node
  std::vector<uint32_t> perm;
  int max_leaf, bins, max_depth;

  static int min_balanced_depth(size_t count, int max_leaf) {
    const size_t leaves = (count + max_leaf - 1) / max_leaf;
    return leaves <= 1 ? 0 : (int)std::ceil(std::log2((double)leaves));
  }
  static double area(const double* mn, const double* mx) {
    double dx = std::max(0.0, mx[0] - mn[0]), dy = std::max(0.0, mx[1] - mn[1]), dz = std::max(0.0, mx[2] - mn[2]);
    return 2 * (dx * dy + dy * dz + dz * dx);
  }
  int bin_of(double c, double cmin, double ext) const {
    double t = std::floor((c - cmin) / ext * bins);
    return (int)std::min<double>(bins - 1, std::max(0.0, t));
  }

  uint32_t push() {
    nodes.push_back(BinaryNode{});
    nmn.resize(3 * nodes.size());
    nmx.resize(3 * nodes.size());
    return (uint32_t)nodes.size() - 1;
  }

  uint32_t build(std::vector<uint32_t>& sub, int depth) {
    const uint32_t me = (uint32_t)nodes.size();
    if ((int)sub.size() <= max_leaf) {
      const uint32_t ni = push();
      double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (uint32_t r : sub)
        for (int k = 0; k < 3; ++k) {
          mn[k] = std::min(mn[k], recs[r].mn[k]);
          mx[k] = std::max(mx[k], recs[r].mx[k]);
        }
      for (int k = 0; k < 3; ++k) { nmn[3 * ni + k] = mn[k]; nmx[3 * ni + k] = mx[k]; }
      nodes[ni].w6 = (uint32_t)perm.size();
      nodes[ni].w7 = kLeafFlag | (uint32_t)sub.size();
      for (uint32_t r : sub) perm.push_back(recs[r].orig);
      return me;
    }
    if (depth >= max_depth || min_balanced_depth(sub.size(), max_leaf) > max_depth - depth)
      fail(VT_ERR_BUILD, "cannot encode " + std::to_string(sub.size()) + " instances within the traversal-safe depth");
    double cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t r : sub)
      for (int k = 0; k < 3; ++k) {
        cmn[k] = std::min(cmn[k], recs[r].cen[k]);
        cmx[k] = std::max(cmx[k], recs[r].cen[k]);
      }
    const double ext[3] = {cmx[0] - cmn[0], cmx[1] - cmn[1], cmx[2] - cmn[2]};
    bool have = false;
    int baxis = 0, bbin = 0;
    double bcost = 0.0;
    if (!(ext[0] <= 0 && ext[1] <= 0 && ext[2] <= 0)) {
      std::vector<double> bmn(3 * bins), bmx(3 * bins), lsa(bins), rsa(bins);
      std::vector<size_t> bc(bins), lc(bins), rc(bins);
      for (int axis = 0; axis < 3; ++axis) {
        if (ext[axis] <= 0) continue;
        std::fill(bmn.begin(), bmn.end(), INFINITY);
        std::fill(bmx.begin(), bmx.end(), -INFINITY);
        std::fill(bc.begin(), bc.end(), 0);
        for (uint32_t r : sub) {
          const int b = bin_of(recs[r].cen[axis], cmn[axis], ext[axis]);
          for (int k = 0; k < 3; ++k) {
            bmn[3 * b + k] = std::min(bmn[3 * b + k], recs[r].mn[k]);
            bmx[3 * b + k] = std::max(bmx[3 * b + k], recs[r].mx[k]);
          }
          bc[b] += 1;
        }
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        size_t c = 0;
        for (int b = 0; b < bins; ++b) {
          if (bc[b]) {
            for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], bmn[3 * b + k]); hi[k] = std::max(hi[k], bmx[3 * b + k]); }
            c += bc[b];
          }
          lsa[b] = area(lo, hi);
          lc[b] = c;
        }
        for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
        c = 0;
        for (int b = bins - 1; b >= 0; --b) {
          if (bc[b]) {
            for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], bmn[3 * b + k]); hi[k] = std::max(hi[k], bmx[3 * b + k]); }
            c += bc[b];
          }
          rsa[b] = area(lo, hi);
          rc[b] = c;
        }
        const double total = lsa[bins - 1];
        if (total <= 0) continue;
        for (int b = 0; b < bins - 1; ++b) {
          if (lc[b] == 0 || rc[b + 1] == 0) continue;
          const double sah = ((double)lc[b] * lsa[b] + (double)rc[b + 1] * rsa[b + 1]) / total;
          if (!have || sah < bcost) { have = true; baxis = axis; bbin = b; bcost = sah; }
        }
      }
    }
    int axis = have ? baxis : 0;
    std::vector<uint32_t> left, right;
    bool fallback = !have || bcost >= (double)sub.size();
    if (!fallback) {
      for (uint32_t r : sub) (bin_of(recs[r].cen[baxis], cmn[baxis], ext[baxis]) <= bbin ? left : right).push_back(r);
      fallback = left.empty() || right.empty() ||
                 min_balanced_depth(left.size(), max_leaf) > max_depth - (depth + 1) ||
                 min_balanced_depth(right.size(), max_leaf) > max_depth - (depth + 1);
    }
    if (fallback) {
      axis = 0;
      if (ext[1] > ext[axis]) axis = 1;
      if (ext[2] > ext[axis]) axis = 2;
      std::vector<uint32_t> ord = sub;
      const int ax = axis;
      std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
        const double d = recs[a].cen[ax] - recs[b].cen[ax];
        return d != 0 ? d < 0 : recs[a].orig < recs[b].orig;
      });
      const size_t mid = ord.size() / 2;
      left.assign(ord.begin(), ord.begin() + mid);
      right.assign(ord.begin() + mid, ord.end());
    }
    const uint32_t ni = push();
    nodes[ni].w7 = (uint32_t)axis;
    sub.clear();
    sub.shrink_to_fit();
    build(left, depth + 1);
    const uint32_t ri = build(right, depth + 1);
    nodes[ni].w6 = ri - ni;
    for (int k = 0; k < 3; ++k) {
      nmn[3 * ni + k] = std::min(nmn[3 * (ni + 1) + k], nmn[3 * ri + k]);
      nmx[3 * ni + k] = std::max(nmx[3 * (ni + 1) + k], nmx[3 * ri + k]);
    }
    return me;
  }
};

}  // namespace

BinaryBvhHost build_tlas_host(const double* aabbs, size_t n, int max_leaf, int bins, int max_depth) {
  if (n == 0) fail(VT_ERR_INVALID_ARGUMENT, "buildTlas: instances list is empty");
  TlasBuilder b;
  b.max_leaf = max_leaf;
  b.bins = bins;
  b.max_depth = max_depth;
  b.recs.resize(n);
  for (size_t i = 0; i < n; ++i) {
    TRec& r = b.recs[i];
    r.orig = (uint32_t)i;
    for (int k = 0; k < 3; ++k) {
      r.mn[k] = aabbs[6 * i + k];
      r.mx[k] = aabbs[6 * i + 3 + k];
      if (!std::isfinite(r.mn[k]) || !std::isfinite(r.mx[k])) fail(VT_ERR_RANGE, "instance AABB is not finite");
      if (r.mx[k] < r.mn[k]) fail(VT_ERR_RANGE, "instance AABB is inverted");
      r.cen[k] = (r.mn[k] + r.mx[k]) * 0.5;
    }
  }
  if (TlasBuilder::min_balanced_depth(n, max_leaf) > max_depth)
    fail(VT_ERR_RANGE, "instances cannot fit the traversal-safe depth");
  std::vector<uint32_t> all(n);
  std::iota(all.begin(), all.end(), 0u);
  b.build(all, 0);
  BinaryBvhHost out;
  out.nodes = std::move(b.nodes);
  for (size_t i = 0; i < out.nodes.size(); ++i)
    for (int k = 0; k < 3; ++k) {
      out.nodes[i].mn[k] = (float)b.nmn[3 * i + k];
      out.nodes[i].mx[k] = (float)b.nmx[3 * i + k];
    }
  out.reordered_to_source = std::move(b.perm);
  return out;
}

}  // namespace vt
