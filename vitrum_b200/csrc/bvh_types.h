// bvh_types.h -- memory layouts shared by the BVH builder and the traversal kernels.
//
// Binary node (32 bytes): the reference's packed layout
// (packages/shared-bvh/src/buildArrayBvh.ts:13-27): min xyz f32, max xyz f32,
// word6 = relative right-child offset (interior) or first triangle (leaf),
// word7 = split axis (interior) or 0xFFFF0000 | triangle count (leaf).
//
// Wide node (80 bytes = 5 x 16-byte words, read with five 128-bit loads):
//   q[0] = px, py, pz (f32 quantisation origin), exyz_imask
//          (bytes: biased exponents ex, ey, ez of the power-of-two grid step, imask)
//   q[1] = child_base, tri_base, tri_valid, 0
//   q[2] = qlo_x[8], qlo_y[8]      (u8 per slot)
//   q[3] = qlo_z[8], qhi_x[8]
//   q[4] = qhi_y[8], qhi_z[8]
// imask bit s = slot s holds an internal node; internal children are stored
// contiguously from child_base in slot order (index = child_base +
// popcount(imask & ((1<<s)-1))).  Leaf slot s owns triangle records
// tri_base + 4s .. tri_base + 4s + count - 1 and tri_valid has exactly those
// bits set, so a slot hit mask expands to a triangle mask with one nibble
// spread and an AND.  Empty slots: imask bit 0, no tri_valid bits, inverted
// quantised box.  Slots are assigned so that visiting key k = 0..7 at slot
// k ^ octant(ray) is near-to-far.
//
// Triangle record (64 bytes): four float4 = (v0.xyz, source id bits),
// (v1.xyz, 0), (v2.xyz, 0), (n.xyz, valid) where n is the unit normal the
// reference's watertight test derives from the triangle alone (exact f32
// operations of opticalWatertightTriangle.ts:164-201) and valid = 0 when that
// derivation rejects the triangle.  Traversal reads the first 48 bytes;
// the normal is read only for a hit that becomes the new closest.
#pragma once

#include <cstdint>

namespace vt {

constexpr uint32_t kLeafFlag = 0xFFFF0000u;
constexpr int kWideNodeWords = 5;       // uint4 per wide node
constexpr int kTriWords = 4;            // float4 per triangle record
constexpr int kMaxBinaryDepth = 58;     // BINARY_BVH_MAX_BUILD_DEPTH, strides.ts:119-125
constexpr int kTraversalStack = 64;     // wide-group stack entries per ray

struct BinaryNode {
  float mn[3];
  float mx[3];
  uint32_t w6;
  uint32_t w7;
};
static_assert(sizeof(BinaryNode) == 32, "binary node is 32 bytes");

inline bool is_leaf_word(uint32_t w7) { return (w7 >> 16) == 0xFFFFu; }

}  // namespace vt
