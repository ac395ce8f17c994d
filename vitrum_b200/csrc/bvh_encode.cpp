// bvh_encode.cpp -- 8-wide collapse and compressed-node encoding.
//
// Collapse, two rules:
//  - the reference's greedy rule (collectWideChildren,
//    packages/shared-bvh/src/compressedWideBvh.ts:215-242): starting from the
//    two children of a binary interior node, repeatedly replace the interior
//    child of largest surface area by its two children until 8 slots are used
//    or only leaves remain.  The resulting wide topology is the reference's;
//    every reference-facing tree uses it.
//  - the SAH-optimal rule of Ylitie, Karras & Laine 2017 ("Efficient
//    incoherent ray traversal on GPUs through compressed wide BVHs", sec. 3.1)
//    for the renderer's own trees: a dynamic programme over the binary tree
//    picks, per wide node, the frontier of at most 8 descendants, and per
//    frontier subtree of at most 4 triangles whether it becomes one leaf slot,
//    minimising the surface-area cost sum(A(node)) * c_node +
//    sum(A(leaf) * triangles) * c_tri.  It only regroups the binary tree's
//    nodes, so the triangle set, the boxes and every hit are unchanged.
//
// Encoding (ours, for the GPU): breadth-first node numbering so the hottest
// nodes form a prefix, slot assignment for octant-ordered traversal, u8
// child bounds on a power-of-two grid anchored at the parent minimum, and
// each wide node's leaf triangles gathered as 64-byte records (vertices,
// source id, precomputed reference normal) in per-slot blocks of four.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <cstdint>
#include <vector>

#include "bvh_exact.h"
#include "bvh_host.h"

namespace vt {

static double half_area(const BinaryNode& n) {
  double dx = std::max(0.0, (double)n.mx[0] - n.mn[0]);
  double dy = std::max(0.0, (double)n.mx[1] - n.mn[1]);
  double dz = std::max(0.0, (double)n.mx[2] - n.mn[2]);
  return dx * dy + dy * dz + dz * dx;
}

int collect_wide_children(const BinaryNode* nodes, uint32_t root, uint32_t out[8]) {
  const BinaryNode& r = nodes[root];
  if (is_leaf_word(r.w7)) { out[0] = root; return 1; }
  int n = 2;
  out[0] = root + 1;
  out[1] = root + r.w6;
  while (n < 8) {
    int at = -1;
    double best = -1;
    for (int i = 0; i < n; ++i) {
      const BinaryNode& c = nodes[out[i]];
      if (is_leaf_word(c.w7)) continue;
      double a = half_area(c);
      if (a > best) { best = a; at = i; }
    }
    if (at < 0) break;
    uint32_t x = out[at];
    std::memmove(out + at + 2, out + at + 1, sizeof(uint32_t) * (n - at - 1));
    out[at] = x + 1;
    out[at + 1] = x + nodes[x].w6;
    ++n;
  }
  return n;
}

namespace {

// Ylitie et al. 2017, sec. 3.1, restated on this binary layout (left child
// at i + 1, right child at i + w6, so children follow their parent).
//   C(n)    cost of n as one slot of its parent:
//           min(leaf: c_tri * A(n) * count(n)   [count <= 4, contiguous],
//               node: c_node * A(n) + G(n, W))   W = width, 8 by default
//   G(n, k) cost of spreading n's subtree over k slots:
//           min over a in [1, k-1] of F(left, a) + F(right, k - a)
//   F(x, a) = C(x) for a = 1 or x a binary leaf, else min(C(x), G(x, a))
struct SahCollapse {
  const BinaryNode* nodes;
  size_t n;
  std::vector<double> c;        // C(n)
  std::vector<double> g;        // G(n, k) at 8 * n + k, k in [2, 8]
  std::vector<uint8_t> split;   // slots given to the left child at 8 * n + k
  std::vector<uint32_t> first, count;
  std::vector<uint8_t> as_leaf; // C(n) taken by the leaf branch
  std::vector<BinaryNode> ext;  // the binary nodes, then one leaf node per mergeable subtree
  std::vector<uint32_t> merged; // index in ext of n's merged leaf (n itself for binary leaves)

  double f(uint32_t x, int a) const {
    if (a < 2 || is_leaf_word(nodes[x].w7)) return c[x];
    return std::min(c[x], g[8 * (size_t)x + a]);
  }

  int width;

  SahCollapse(const BinaryBvhHost& bin, double c_node, double c_tri, int w)
      : nodes(bin.nodes.data()), n(bin.nodes.size()), c(n), g(8 * n, 0.0), split(8 * n, 0), first(n), count(n),
        as_leaf(n, 0), ext(bin.nodes), merged(n), width(w) {
    for (size_t i = n; i-- > 0;) {
      const BinaryNode& b = nodes[i];
      const double area = half_area(b);
      if (is_leaf_word(b.w7)) {
        first[i] = b.w6;
        count[i] = b.w7 & 0xFFFFu;
        c[i] = c_tri * area * count[i];
        as_leaf[i] = 1;
        merged[i] = (uint32_t)i;
        continue;
      }
      const uint32_t l = (uint32_t)i + 1, r = (uint32_t)i + b.w6;
      first[i] = first[l];
      count[i] = count[l] + count[r];
      const bool contiguous = first[r] == first[l] + count[l];
      for (int k = 2; k <= 8; ++k) {
        double best = INFINITY;
        int at = 1;
        for (int a = 1; a < k; ++a) {
          const double v = f(l, a) + f(r, k - a);
          if (v < best) { best = v; at = a; }
        }
        g[8 * i + k] = best;
        split[8 * i + k] = (uint8_t)at;
      }
      c[i] = c_node * area + g[8 * i + width];
      merged[i] = 0;
      if (count[i] <= 4 && contiguous) {
        const double leaf = c_tri * area * count[i];
        if (leaf < c[i]) {
          c[i] = leaf;
          as_leaf[i] = 1;
        }
        BinaryNode m = b;
        m.w6 = first[i];
        m.w7 = 0xFFFF0000u | count[i];
        merged[i] = (uint32_t)ext.size();
        ext.push_back(m);
      }
    }
  }

  // frontier of x over a slots, appended to out (indices into ext)
  void frontier(uint32_t x, int a, uint32_t* out, int& m) const {
    if (a >= 2 && !is_leaf_word(nodes[x].w7) && g[8 * (size_t)x + a] < c[x]) {
      const int s = split[8 * (size_t)x + a];
      frontier(x + 1, s, out, m);
      frontier(x + nodes[x].w6, a - s, out, m);
      return;
    }
    out[m++] = as_leaf[x] ? merged[x] : x;
  }

  // children of the wide node rooted at binary node x (never a merged leaf)
  int children(uint32_t x, uint32_t out[8]) const {
    if (is_leaf_word(ext[x].w7)) { out[0] = x; return 1; }
    const int s = split[8 * (size_t)x + width];
    int m = 0;
    frontier(x + 1, s, out, m);
    frontier(x + nodes[x].w6, width - s, out, m);
    return m;
  }
};

}  // namespace

// Greedy slot assignment: slot s is visited first by rays whose direction
// sign bits (x:4, y:2, z:1; bit set = negative) equal s, so it should hold
// the child lying furthest against that direction.
void assign_slots(const BinaryNode* nodes, const BinaryNode& parent, const uint32_t* ch, int n, int slot_of[8]) {
  double pc[3];
  for (int k = 0; k < 3; ++k) pc[k] = 0.5 * ((double)parent.mn[k] + parent.mx[k]);
  double cost[8][8];
  for (int i = 0; i < n; ++i) {
    const BinaryNode& c = nodes[ch[i]];
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = 0.5 * ((double)c.mn[k] + c.mx[k]) - pc[k];
    for (int s = 0; s < 8; ++s) {
      double sx = (s & 4) ? -1.0 : 1.0, sy = (s & 2) ? -1.0 : 1.0, sz = (s & 1) ? -1.0 : 1.0;
      cost[i][s] = d[0] * sx + d[1] * sy + d[2] * sz;
    }
  }
  bool used_c[8] = {}, used_s[8] = {};
  for (int i = 0; i < 8; ++i) slot_of[i] = -1;
  for (int round = 0; round < n; ++round) {
    int bi = -1, bs = -1;
    double bc = INFINITY;
    for (int i = 0; i < n; ++i) {
      if (used_c[i]) continue;
      for (int s = 0; s < 8; ++s) {
        if (used_s[s]) continue;
        if (bi < 0 || cost[i][s] < bc) { bc = cost[i][s]; bi = i; bs = s; }
      }
    }
    used_c[bi] = true;
    used_s[bs] = true;
    slot_of[bi] = bs;
  }
}

// Unit normal exactly as the reference's watertight test derives it from the
// triangle (opticalWatertightTriangle.ts:164-201): every operation single
// precision, individually rounded (this file is compiled without FMA
// contraction).  Returns false when that derivation rejects the triangle.
static bool reference_normal(const float a[3], const float b[3], const float c[3], float nn[3]) {
  float e1r[3], e2r[3];
  for (int k = 0; k < 3; ++k) { e1r[k] = b[k] - a[k]; e2r[k] = c[k] - a[k]; }
  float es = 0.0f;
  for (int k = 0; k < 3; ++k) es = std::max(es, std::fabs(e1r[k]));
  for (int k = 0; k < 3; ++k) es = std::max(es, std::fabs(e2r[k]));
  if (!(es > 0.0f) || !std::isfinite(es)) return false;
  float s1[3], s2[3];
  for (int k = 0; k < 3; ++k) { s1[k] = e1r[k] / es; s2[k] = e2r[k] / es; }
  float nr[3] = {s1[1] * s2[2] - s1[2] * s2[1], s1[2] * s2[0] - s1[0] * s2[2], s1[0] * s2[1] - s1[1] * s2[0]};
  float ns = std::max(std::max(std::fabs(nr[0]), std::fabs(nr[1])), std::fabs(nr[2]));
  if (!(ns > 0.0f) || !std::isfinite(ns)) return false;
  float nd[3] = {nr[0] / ns, nr[1] / ns, nr[2] / ns};
  float l2 = (nd[0] * nd[0] + nd[1] * nd[1]) + nd[2] * nd[2];
  float nl = std::sqrt(l2);
  if (!(nl > 0.0f) || !std::isfinite(nl)) return false;
  for (int k = 0; k < 3; ++k) nn[k] = nd[k] / nl;
  return true;
}

// Smallest e with origin + 255 * 2^e >= hi (exactly, corner_sign), clamped to the normal range.
static int grid_exponent(float origin, float hi) {
  const double extent = (double)hi - (double)origin;
  if (!(extent > 0)) return -126;
  int e;
  std::frexp(extent / 255.0, &e);  // extent/255 = m * 2^e, m in [0.5, 1)
  while (e > -126 && std::ldexp(255.0, e - 1) >= extent) --e;
  while (e < 127 && corner_sign(origin, 255, e, hi) < 0) ++e;
  return std::min(127, std::max(-126, e));
}

// Encodes the binary tree as 8-wide nodes.  Node indices are offset by
// node_base and record indices by rec_base (trees concatenated into shared
// arrays); emit(leaf, slot_records) writes a leaf's payload records (16
// floats each) for the leaf's binary node.
template <class Children, class EmitLeaf>
static WideBvhHost encode_core(const BinaryBvhHost& bin, const BinaryNode* nodes, uint32_t node_base,
                               uint32_t rec_base, Children children_of, EmitLeaf emit) {
  WideBvhHost out;
  const size_t nleaf_items = bin.reordered_to_source.size();
  std::vector<uint32_t> wide_bin;   // binary node behind each wide node (BFS order)
  std::vector<int> level;
  wide_bin.push_back(0);
  level.push_back(1);
  out.depth = 1;
  if (nleaf_items == 0) {
    uint32_t w[20] = {};
    // All-empty slots: inverted boxes (qlo 255, qhi 0), no children.
    std::memset(reinterpret_cast<uint8_t*>(w) + 32, 0xFF, 24);
    out.nodes.assign(w, w + 20);
    return out;
  }
  // 28 leading empty records: tri_base = block - 4 * first_leaf_slot then
  // never wraps, and stays below 2^30 (bits 30-31 tag stack entries).
  out.tris.reserve((nleaf_items + 28) * 24);
  out.tris.assign(16 * 28, 0.0f);
  for (size_t wi = 0; wi < wide_bin.size(); ++wi) {
    const BinaryNode& parent = nodes[wide_bin[wi]];
    uint32_t ch[8];
    int n = children_of(wide_bin[wi], ch);
    int slot_of[8];
    assign_slots(nodes, parent, ch, n, slot_of);
    int child_at_slot[8];
    for (int s = 0; s < 8; ++s) child_at_slot[s] = -1;
    for (int i = 0; i < n; ++i) child_at_slot[slot_of[i]] = i;

    uint8_t bytes[80];
    std::memset(bytes, 0, sizeof bytes);
    float p[3] = {parent.mn[0], parent.mn[1], parent.mn[2]};
    std::memcpy(bytes, p, 12);
    int ex[3];
    for (int k = 0; k < 3; ++k) {
      ex[k] = grid_exponent(parent.mn[k], parent.mx[k]);
      bytes[12 + k] = (uint8_t)(ex[k] + 127);
    }
    uint8_t imask = 0;
    const uint32_t child_base = node_base + (uint32_t)wide_bin.size();
    // leaf slot s uses records [block + 4*(s - first_leaf_slot), +count)
    int first_leaf = 8, last_leaf = -1;
    for (int s = 0; s < 8; ++s) {
      int ci = child_at_slot[s];
      if (ci >= 0 && is_leaf_word(nodes[ch[ci]].w7)) { first_leaf = std::min(first_leaf, s); last_leaf = s; }
    }
    const uint32_t block = (uint32_t)(out.tris.size() / 16);
    const uint32_t tri_base = rec_base + block - 4u * (uint32_t)(first_leaf < 8 ? first_leaf : 0);
    if ((uint64_t)rec_base + block + 32 >= 0x40000000ull) throw std::length_error("leaf records exceed 2^30");
    if (last_leaf >= 0) out.tris.resize(out.tris.size() + 16 * (size_t)(4 * (last_leaf - first_leaf) + 4), 0.0f);
    uint32_t tri_valid = 0;
    for (int s = 0; s < 8; ++s) {
      uint8_t* qlo = bytes + 32;  // qlo_x at +0, qlo_y at +8, qlo_z at +16
      uint8_t* qhi = bytes + 56;  // qhi_x at +0, qhi_y at +8, qhi_z at +16
      int ci = child_at_slot[s];
      if (ci < 0) {
        for (int k = 0; k < 3; ++k) { qlo[k * 8 + s] = 255; qhi[k * 8 + s] = 0; }
        continue;
      }
      const BinaryNode& c = nodes[ch[ci]];
      for (int k = 0; k < 3; ++k) {
        double step = std::ldexp(1.0, ex[k]);
        double lo = std::floor(((double)c.mn[k] - (double)p[k]) / step);
        double hi = std::ceil(((double)c.mx[k] - (double)p[k]) / step);
        int ql = (int)std::min(255.0, std::max(0.0, lo));
        int qh = (int)std::min(255.0, std::max(0.0, hi));
        // outward exactly: (c - p) / step rounds when c is tiny next to p
        while (ql > 0 && corner_sign(p[k], ql, ex[k], c.mn[k]) > 0) --ql;
        while (qh < 255 && corner_sign(p[k], qh, ex[k], c.mx[k]) < 0) ++qh;
        qlo[k * 8 + s] = (uint8_t)ql;
        qhi[k * 8 + s] = (uint8_t)qh;
      }
      if (is_leaf_word(c.w7)) {
        const uint32_t cnt = c.w7 & 0xFFFFu;
        tri_valid |= ((1u << cnt) - 1u) << (4 * s);
        emit(c, &out.tris[16 * ((size_t)block + 4 * (s - first_leaf))]);
      } else {
        imask |= (uint8_t)(1u << s);
        wide_bin.push_back(ch[ci]);
        level.push_back(level[wi] + 1);
        out.depth = std::max(out.depth, level[wi] + 1);
      }
    }
    std::memcpy(bytes + 24, &tri_valid, 4);
    bytes[15] = imask;
    std::memcpy(bytes + 16, &child_base, 4);
    std::memcpy(bytes + 20, &tri_base, 4);
    const uint32_t* w = reinterpret_cast<const uint32_t*>(bytes);
    out.nodes.insert(out.nodes.end(), w, w + 20);
  }
  return out;
}

WideBvhHost encode_wide(const BinaryBvhHost& bin, const float* positions, int pos_stride, const uint32_t* indices,
                        int idx_stride, const uint32_t* tri_materials, uint32_t node_base, uint32_t rec_base,
                        const WideCollapse* sah) {
  auto emit = [&](const BinaryNode& leaf, float* recs) {
    const uint32_t cnt = leaf.w7 & 0xFFFFu, first = leaf.w6;
    for (uint32_t t = 0; t < cnt; ++t) {
      const uint32_t src = bin.reordered_to_source[first + t];
      const uint32_t* iv = indices + (size_t)src * idx_stride;
      float* rec = recs + 16 * t;
      float v[3][3];
      for (int vi = 0; vi < 3; ++vi)
        for (int k = 0; k < 3; ++k) v[vi][k] = positions[(size_t)iv[vi] * pos_stride + k];
      for (int vi = 0; vi < 3; ++vi)
        for (int k = 0; k < 3; ++k) rec[4 * vi + k] = v[vi][k];
      std::memcpy(&rec[3], &src, 4);
      if (tri_materials) std::memcpy(&rec[7], &tri_materials[src], 4);
      float nn[3] = {0, 0, 0};
      const bool valid = reference_normal(v[0], v[1], v[2], nn);
      rec[12] = nn[0];
      rec[13] = nn[1];
      rec[14] = nn[2];
      rec[15] = valid ? 1.0f : 0.0f;
    }
  };
  if (sah && !bin.nodes.empty()) {
    const SahCollapse plan(bin, sah->c_node, sah->c_tri, std::min(std::max(sah->width, 2), 8));
    return encode_core(bin, plan.ext.data(), node_base, rec_base,
                       [&](uint32_t x, uint32_t* out) { return plan.children(x, out); }, emit);
  }
  const BinaryNode* nodes = bin.nodes.data();
  return encode_core(bin, nodes, node_base, rec_base,
                     [&](uint32_t x, uint32_t* out) { return collect_wide_children(nodes, x, out); }, emit);
}

WideBvhHost encode_wide_tlas(const BinaryBvhHost& tlas, const InstanceRecord* instances, uint32_t node_base) {
  const BinaryNode* nodes = tlas.nodes.data();
  return encode_core(tlas, nodes, node_base, 0,
                     [&](uint32_t x, uint32_t* out) { return collect_wide_children(nodes, x, out); },
                     [&](const BinaryNode& leaf, float* recs) {
    const uint32_t cnt = leaf.w7 & 0xFFFFu, first = leaf.w6;
    for (uint32_t i = 0; i < cnt; ++i) {
      const uint32_t inst = tlas.reordered_to_source[first + i];
      std::memcpy(recs + 16 * i, &instances[inst], sizeof(InstanceRecord));
    }
  });
}

}  // namespace vt
