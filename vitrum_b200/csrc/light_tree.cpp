// light_tree.cpp -- host build and packing of the light tree (light_tree.h).
//
// Follows buildLightTree / buildSubtree / mergeCones / packLightTreeForGPU
// (packages/shared-samplers/src/lightTree.ts:250-737): median split of the
// centroids along the widest centroid axis (ties by emitter index), a split by
// descending power when every centroid lies within 1e-4, union AABBs and
// power sums per node, Conty Estevez & Kulla orientation cones merged bottom
// up, pre-order node numbering.  The same steps are needed because the tree
// and its packed words define the selection probabilities the integrator's
// estimates divide by.
#include "light_tree.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>

#include "vt_common.h"

namespace vt {
namespace lt {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr float kMinNormal = 1.17549435082228750797e-38f;

struct Cone {
  double axis[3];
  double theta_o, theta_e;
};
const Cone kFullSphere{{0, 0, 0}, kPi, kPi};

struct Node {
  int emitter = -1;
  double power = 0.0;
  double mn[3], mx[3];
  int left = -1, right = -1;
  Cone cone = kFullSphere;
};

struct Item {
  int emitter;
  double power;
  double c[3], mn[3], mx[3];
  Cone cone;
};

double vlen(const double* v) {
  const double s = std::max(std::fabs(v[0]), std::max(std::fabs(v[1]), std::fabs(v[2])));
  if (s == 0.0) return 0.0;
  const double x = v[0] / s, y = v[1] / s, z = v[2] / s;
  return s * std::sqrt(x * x + y * y + z * z);
}

// mergeCones (lightTree.ts:250-307): a cone bounding both; full sphere when
// either is unoriented, the union reaches pi, or the axes are antiparallel.
Cone merge(const Cone& a, const Cone& b) {
  const double la = vlen(a.axis), lb = vlen(b.axis);
  if (la == 0.0 || lb == 0.0 || a.theta_o >= kPi || b.theta_o >= kPi)
    return Cone{{0, 0, 0}, kPi, std::min(kPi, std::max(a.theta_e, b.theta_e))};
  const Cone* A = &a;
  const Cone* B = &b;
  if (B->theta_o > A->theta_o) std::swap(A, B);
  const double lA = vlen(A->axis), lB = vlen(B->axis);
  const double ax[3] = {A->axis[0] / lA, A->axis[1] / lA, A->axis[2] / lA};
  const double bx[3] = {B->axis[0] / lB, B->axis[1] / lB, B->axis[2] / lB};
  const double cos_d = std::max(-1.0, std::min(1.0, ax[0] * bx[0] + ax[1] * bx[1] + ax[2] * bx[2]));
  const double d_theta = std::acos(cos_d);
  const double theta_e = std::min(kPi, std::max(A->theta_e, B->theta_e));
  if (std::min(d_theta + B->theta_o, kPi) <= A->theta_o) return Cone{{ax[0], ax[1], ax[2]}, A->theta_o, theta_e};
  const double theta_o = (A->theta_o + d_theta + B->theta_o) * 0.5;
  if (theta_o >= kPi) return Cone{{0, 0, 0}, kPi, theta_e};
  const double rot = theta_o - A->theta_o;
  double t[3] = {bx[0] - cos_d * ax[0], bx[1] - cos_d * ax[1], bx[2] - cos_d * ax[2]};
  const double tl = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  if (tl < 1e-8) return Cone{{0, 0, 0}, kPi, theta_e};
  for (double& x : t) x /= tl;
  const double cr = std::cos(rot), sr = std::sin(rot);
  return Cone{{ax[0] * cr + t[0] * sr, ax[1] * cr + t[1] * sr, ax[2] * cr + t[2] * sr}, theta_o, theta_e};
}

int build_subtree(std::vector<Item> items, std::vector<Node>& nodes) {
  const int idx = (int)nodes.size();
  if (items.size() == 1) {
    const Item& it = items[0];
    Node n;
    n.emitter = it.emitter;
    n.power = it.power;
    std::memcpy(n.mn, it.mn, sizeof n.mn);
    std::memcpy(n.mx, it.mx, sizeof n.mx);
    n.cone = it.cone;
    nodes.push_back(n);
    return idx;
  }
  double cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const Item& it : items)
    for (int k = 0; k < 3; ++k) {
      cmn[k] = std::min(cmn[k], it.c[k]);
      cmx[k] = std::max(cmx[k], it.c[k]);
    }
  const double sx = cmx[0] - cmn[0], sy = cmx[1] - cmn[1], sz = cmx[2] - cmn[2];
  std::vector<Item> sorted = items;
  if (std::max(sx, std::max(sy, sz)) < 1e-4) {
    std::sort(sorted.begin(), sorted.end(), [](const Item& a, const Item& b) {
      return a.power != b.power ? a.power > b.power : a.emitter < b.emitter;
    });
  } else {
    const int axis = (sx >= sy && sx >= sz) ? 0 : (sy >= sz ? 1 : 2);
    std::sort(sorted.begin(), sorted.end(), [axis](const Item& a, const Item& b) {
      return a.c[axis] != b.c[axis] ? a.c[axis] < b.c[axis] : a.emitter < b.emitter;
    });
  }
  const size_t mid = sorted.size() / 2;
  Node n;
  for (int k = 0; k < 3; ++k) { n.mn[k] = INFINITY; n.mx[k] = -INFINITY; }
  double total = 0.0;
  for (const Item& it : items) {  // union bounds and power in this call's item order
    for (int k = 0; k < 3; ++k) {
      n.mn[k] = std::min(n.mn[k], it.mn[k]);
      n.mx[k] = std::max(n.mx[k], it.mx[k]);
    }
    total += it.power;
    if (!std::isfinite(total)) fail(VT_ERR_RANGE, "light tree: total power overflowed");
  }
  n.power = total;
  nodes.push_back(n);
  const int l = build_subtree(std::vector<Item>(sorted.begin(), sorted.begin() + mid), nodes);
  const int r = build_subtree(std::vector<Item>(sorted.begin() + mid, sorted.end()), nodes);
  nodes[idx].left = l;
  nodes[idx].right = r;
  nodes[idx].cone = merge(nodes[l].cone, nodes[r].cone);
  return idx;
}

float next_down(float v) {
  if (std::isnan(v) || v == -INFINITY) return v;
  if (v == 0.0f) return -std::numeric_limits<float>::denorm_min();
  uint32_t b;
  std::memcpy(&b, &v, 4);
  b = v > 0.0f ? b - 1u : b + 1u;
  std::memcpy(&v, &b, 4);
  return v;
}

// conservativeConeCosineThreshold (lightTree.ts:193-204)
float cone_cos(double angle) {
  const float rounded = (float)std::cos(std::min(kPi, angle));
  float t = rounded;
  for (int s = 0; s < 64; ++s) t = next_down(t);
  const float abs_t = (float)((double)rounded - 3.814697265625e-06);  // 2^-18
  return std::max(-1.0f, std::min(t, abs_t));
}

// representedLightTreePower (lightTree.ts:214-224)
float represented_power(double p, double max_p) {
  if (!(p > 0.0) || !(max_p > 0.0)) return 0.0f;
  const double ratio = p / max_p;
  if (!(ratio > 0.0)) return kMinNormal;
  const float r = (float)ratio;
  return r > kMinNormal ? r : kMinNormal;
}

}  // namespace

void merge_into(Emitter& group, const std::vector<Emitter>& parts) {
  auto cone_of = [](const Emitter& e) {
    const double l = vlen(e.axis);
    if (!e.oriented || l == 0.0) return kFullSphere;
    return Cone{{e.axis[0] / l, e.axis[1] / l, e.axis[2] / l}, e.theta_o, std::min(kPi, e.theta_e)};
  };
  Cone c = parts.empty() ? kFullSphere : cone_of(parts[0]);
  for (size_t i = 1; i < parts.size(); ++i) c = merge(c, cone_of(parts[i]));
  group.oriented = vlen(c.axis) > 0.0 && c.theta_o < kPi;
  for (int k = 0; k < 3; ++k) group.axis[k] = group.oriented ? c.axis[k] : 0.0;
  group.theta_o = c.theta_o;
  group.theta_e = c.theta_e;
}

std::vector<float> build_packed(const std::vector<Emitter>& em) {
  if (em.empty()) fail(VT_ERR_INVALID_ARGUMENT, "light tree: at least one emitter required");
  if (em.size() > kBuckets) fail(VT_ERR_RANGE, "light tree: more emitters than the 24-bit selection domain");
  std::vector<Item> items(em.size());
  for (size_t i = 0; i < em.size(); ++i) {
    const Emitter& e = em[i];
    Item& it = items[i];
    it.emitter = (int)i;
    if (!(e.power >= 0.0) || !std::isfinite(e.power))
      fail(VT_ERR_RANGE, "light tree: emitter " + std::to_string(i) + " power must be finite and >= 0");
    it.power = e.power;
    for (int k = 0; k < 3; ++k) {
      if (!std::isfinite(e.centroid[k]) || !std::isfinite(e.mn[k]) || !std::isfinite(e.mx[k]) ||
          !std::isfinite((float)e.mn[k]) || !std::isfinite((float)e.mx[k]))
        fail(VT_ERR_RANGE, "light tree: emitter " + std::to_string(i) + " geometry is not finite in f32");
      if (e.mn[k] > e.mx[k]) fail(VT_ERR_RANGE, "light tree: emitter " + std::to_string(i) + " has min > max");
      it.c[k] = e.centroid[k];
      it.mn[k] = e.mn[k];
      it.mx[k] = e.mx[k];
    }
    const double l = vlen(e.axis);
    if (!e.oriented || l == 0.0) {
      it.cone = kFullSphere;
    } else {
      if (!(e.theta_o >= 0 && e.theta_o <= kPi && e.theta_e >= 0 && e.theta_e <= kPi))
        fail(VT_ERR_RANGE, "light tree: emitter " + std::to_string(i) + " cone angles must be in [0, pi]");
      it.cone = Cone{{e.axis[0] / l, e.axis[1] / l, e.axis[2] / l}, e.theta_o, std::min(kPi, e.theta_e)};
    }
  }
  std::vector<Node> nodes;
  nodes.reserve(2 * em.size());
  build_subtree(items, nodes);
  double max_p = 0.0;
  for (const Node& n : nodes) max_p = std::max(max_p, n.power);
  std::vector<float> out(nodes.size() * kFloatsPerNode, 0.0f);
  for (size_t i = 0; i < nodes.size(); ++i) {
    const Node& n = nodes[i];
    float* o = &out[i * kFloatsPerNode];
    o[0] = (float)n.emitter;
    o[1] = represented_power(n.power, max_p);
    o[2] = (float)n.left;
    o[3] = (float)n.right;
    for (int k = 0; k < 3; ++k) {
      o[4 + k] = (float)n.mn[k];
      o[7 + k] = (float)n.mx[k];
    }
    const double al = vlen(n.cone.axis);
    for (int k = 0; k < 3; ++k) o[10 + k] = al > 0.0 ? (float)(n.cone.axis[k] / al) : 0.0f;
    o[13] = cone_cos(n.cone.theta_o);
    o[14] = cone_cos(n.cone.theta_o + n.cone.theta_e);
  }
  // leaf counts, children after their parent in pre-order
  std::vector<uint32_t> leaves(nodes.size(), 0);
  for (size_t i = nodes.size(); i-- > 0;) {
    leaves[i] = nodes[i].left < 0 ? 1u : leaves[nodes[i].left] + leaves[nodes[i].right];
    out[i * kFloatsPerNode + 15] = (float)leaves[i];
  }
  return out;
}

}  // namespace lt
}  // namespace vt

using namespace vt;

extern "C" vt_status vt_light_tree_build(const vt_light_tree_emitter* emitters, size_t n, float* nodes,
                                         size_t float_capacity, size_t* node_count) {
  return guard([&] {
    if (n && !emitters) fail(VT_ERR_INVALID_ARGUMENT, "emitters is null");
    std::vector<lt::Emitter> em(n);
    for (size_t i = 0; i < n; ++i) {
      const vt_light_tree_emitter& s = emitters[i];
      lt::Emitter& e = em[i];
      e.power = s.power;
      for (int k = 0; k < 3; ++k) {
        e.centroid[k] = s.centroid[k];
        e.mn[k] = s.aabb_min[k];
        e.mx[k] = s.aabb_max[k];
        e.axis[k] = s.cone_axis[k];
      }
      e.oriented = s.oriented != 0;
      e.theta_o = s.cone_theta_o;
      e.theta_e = s.cone_theta_e;
    }
    const std::vector<float> packed = lt::build_packed(em);
    if (node_count) *node_count = packed.size() / lt::kFloatsPerNode;
    if (nodes) {
      if (float_capacity < packed.size()) fail(VT_ERR_RANGE, "node buffer too small");
      std::memcpy(nodes, packed.data(), packed.size() * sizeof(float));
    }
  });
}
