// light_tree.h -- the light tree the path tracer's next-event estimation
// selects emitters with (the reference's buildLightTree / packLightTreeForGPU,
// packages/shared-samplers/src/lightTree.ts:492-737).
//
// Host side: emitters in the engine's light-entry order go in; a pre-order
// binary tree comes out, packed as 16 floats per node:
//   [0] emitter index (-1 internal)   [1] power / max node power (f32, floored
//   to the smallest normal)           [2] left child  [3] right child (-1 leaf)
//   [4..6] AABB min  [7..9] AABB max  [10..12] unit cone axis (0: full sphere)
//   [13] cos(thetaO), [14] cos(min(pi, thetaO + thetaE)), both rounded
//   outward (64 f32 steps and 2^-18)  [15] leaves in the subtree.
// Device side (light_tree.cuh): one 24-bit draw descends the tree, splitting
// the current bucket interval between the children after reserving one bucket
// per leaf, in proportion to importance = power / max(dist^2 to the AABB,
// 1e-3) * orientation-cone factor; the selection probability is the final
// interval's bucket count / 2^24.
#pragma once

#include <cstdint>
#include <vector>

namespace vt {
namespace lt {

constexpr int kFloatsPerNode = 16;
constexpr uint32_t kBuckets = 1u << 24;  // LIGHT_TREE_BUCKET_COUNT, lightTree.ts:162
constexpr float kDist2Floor = 1e-3f;     // LT_DIST2_FLOOR, pt-webgpu material.wgsl.ts:2131

struct Emitter {
  double power = 0.0;            // luminance (x area for area emitters)
  double centroid[3] = {0, 0, 0};
  double mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
  bool oriented = false;         // false: full-sphere emitter (no orientation cone)
  double axis[3] = {0, 0, 0};
  double theta_o = 0.0, theta_e = 1.5707963267948966;
};

// The orientation cone of a group of emitters: the parts' cones merged in
// order (mergeCones, lightTree.ts:250); a full-sphere result clears `oriented`.
void merge_into(Emitter& group, const std::vector<Emitter>& parts);

// Builds and packs the tree (throws vt::Error on invalid input).
std::vector<float> build_packed(const std::vector<Emitter>& emitters);

}  // namespace lt
}  // namespace vt
