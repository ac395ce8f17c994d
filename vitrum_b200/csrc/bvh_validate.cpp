// bvh_validate.cpp -- structural proofs of the acceleration structures.
//
// validate_binary_encoding: the reference's publication proof of a packed
// binary BVH (validateBvhEncoding, packages/shared-bvh/src/validateBvhEncoding.ts:55):
// buffer extent, declared roots, reachability with exclusive ownership (no
// cycle, no shared child), split axes, finite ordered bounds that enclose both
// children, leaf triangle ranges that tile [0, triangleCount) exactly, and the
// worst-case live DFS stack (depth + 1) against the traversal's capacity.
//
// validate_wide: the same kind of proof for this library's 80-byte 8-wide
// nodes (layout in bvh_types.h), run on every tree the library builds before
// it is published to the device:
//   * every node is reached exactly once from the declared root, internal
//     children lie inside the node array;
//   * a leaf slot's tri_valid bits are contiguous from bit 4s, internal and
//     empty slots own none, empty slots carry the inverted box (255 / 0);
//   * the leaf records lie inside the record array and name every item
//     (triangle source id, or instance id for a top level) exactly once;
//   * conservative culling: every vertex of a leaf's triangles lies inside
//     the dequantised box (origin + q * 2^e, exact in 113-bit arithmetic) of its own slot
//     and of every ancestor slot a ray must pass to reach it (instance leaves
//     of a top level: skipped, their world boxes are not stored);
//   * the traversal's stack bound (two entries per level plus two) fits.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bvh_host.h"
#include "bvh_types.h"
#include "vt_common.h"

namespace vt {

namespace {

[[noreturn]] void bad(const std::string& what, const std::string& m) { fail(VT_ERR_BUILD, what + ": " + m); }

float f32_of(uint32_t w) {
  float f;
  std::memcpy(&f, &w, 4);
  return f;
}

}  // namespace

BinaryProof validate_binary_encoding(const uint32_t* words, size_t word_count, size_t total_nodes,
                                     const uint32_t* roots, size_t n_roots, int64_t tri_count, int stack_cap) {
  const std::string W = "validateBvhEncoding";
  if (word_count != total_nodes * 8)
    bad(W, "node buffer has " + std::to_string(word_count) + " words; expected exactly " +
               std::to_string(total_nodes * 8) + " for " + std::to_string(total_nodes) + " node(s)");
  if (stack_cap <= 0) bad(W, "traversalStackCapacity must be a positive integer");
  BinaryProof p;
  p.node_count = (int64_t)total_nodes;
  p.stack_capacity = stack_cap;
  p.triangle_count = tri_count;
  std::vector<uint32_t> rs;
  if (roots) rs.assign(roots, roots + n_roots);
  else if (total_nodes) rs.push_back(0);
  if (total_nodes == 0) {
    if (!rs.empty()) bad(W, "an empty node buffer cannot declare roots");
    if (tri_count > 0) bad(W, "empty node buffer cannot cover " + std::to_string(tri_count) + " triangle(s)");
    return p;
  }
  if (rs.empty()) bad(W, "non-empty node buffer must declare at least one root");
  std::vector<uint8_t> visited(total_nodes, 0), root_seen(total_nodes, 0);
  std::vector<std::pair<uint32_t, uint32_t>> ranges;
  struct Item { uint32_t node; int depth; };
  std::vector<Item> stack;
  for (uint32_t root : rs) {
    if (root >= total_nodes)
      bad(W, "root " + std::to_string(root) + " is outside [0, " + std::to_string(total_nodes - 1) + "]");
    if (root_seen[root]) bad(W, "root " + std::to_string(root) + " is declared more than once");
    root_seen[root] = 1;
    p.root_count += 1;
    stack.assign(1, Item{root, 0});
    while (!stack.empty()) {
      const Item it = stack.back();
      stack.pop_back();
      const uint32_t node = it.node;
      if (visited[node])
        bad(W, "node " + std::to_string(node) +
                   " is reachable more than once (cycle, shared child, or overlapping concatenated roots)");
      visited[node] = 1;
      p.max_depth = std::max<int64_t>(p.max_depth, it.depth);
      // ray-dependent child order: the deepest path plus one pending sibling per ancestor
      p.max_stack_entries = std::max<int64_t>(p.max_stack_entries, it.depth + 1);
      if (p.max_stack_entries > stack_cap)
        bad(W, "traversal requires " + std::to_string(p.max_stack_entries) +
                   " live stack entries, exceeding shader capacity " + std::to_string(stack_cap));
      const uint32_t* n = words + 8 * (size_t)node;
      float b[6];
      for (int k = 0; k < 6; ++k) b[k] = f32_of(n[k]);
      for (int k = 0; k < 6; ++k)
        if (!std::isfinite(b[k])) bad(W, "node " + std::to_string(node) + " has non-finite bounds");
      if (b[0] > b[3] || b[1] > b[4] || b[2] > b[5]) bad(W, "node " + std::to_string(node) + " has inverted bounds");
      if (is_leaf_word(n[7])) {
        p.leaf_node_count += 1;
        const uint32_t count = n[7] & 0xFFFFu, offset = n[6];
        if (tri_count >= 0) {
          if ((int64_t)offset > tri_count || (int64_t)count > tri_count - (int64_t)offset)
            bad(W, "leaf node " + std::to_string(node) + " triangle range [" + std::to_string(offset) + ", " +
                       std::to_string((uint64_t)offset + count) + ") exceeds triangle capacity " +
                       std::to_string(tri_count));
          ranges.emplace_back(offset, count);
        }
        continue;
      }
      p.interior_node_count += 1;
      if (n[7] > 2) bad(W, "interior node " + std::to_string(node) + " has invalid split axis " + std::to_string(n[7]));
      const uint64_t left = (uint64_t)node + 1, right = (uint64_t)node + n[6];
      if (n[6] <= 1 || left >= total_nodes || right >= total_nodes)
        bad(W, "interior node " + std::to_string(node) + " has invalid relative right-child offset " +
                   std::to_string(n[6]) + "; child indices would be " + std::to_string(left) + " and " +
                   std::to_string(right) + " for " + std::to_string(total_nodes) + " node(s)");
      for (uint64_t c : {left, right}) {
        const uint32_t* cn = words + 8 * c;
        // written as the reference does (a NaN child bound fails its own finiteness check instead)
        bool outside = false;
        for (int k = 0; k < 3; ++k) outside = outside || f32_of(cn[k]) < b[k] || f32_of(cn[3 + k]) > b[3 + k];
        if (outside) bad(W, "interior node " + std::to_string(node) + " bounds do not enclose child " + std::to_string(c));
      }
      stack.push_back(Item{(uint32_t)right, it.depth + 1});
      stack.push_back(Item{(uint32_t)left, it.depth + 1});
    }
  }
  size_t seen = 0;
  for (uint8_t v : visited) seen += v;
  if (seen != total_nodes)
    bad(W, std::to_string(total_nodes - seen) + " node(s) are unreachable from the " + std::to_string(rs.size()) +
               " declared root(s)");
  if (tri_count >= 0) {
    std::sort(ranges.begin(), ranges.end(),
              [](const std::pair<uint32_t, uint32_t>& a, const std::pair<uint32_t, uint32_t>& b) {
                return a.first < b.first;
              });
    uint64_t cursor = 0;
    for (const auto& r : ranges) {
      if (r.first != cursor)
        bad(W, "leaf triangle range [" + std::to_string(r.first) + ", " + std::to_string((uint64_t)r.first + r.second) +
                   ") " + (r.first < cursor ? "overlaps" : "leaves a gap after") + " triangle " +
                   std::to_string(cursor));
      cursor += r.second;
    }
    if ((int64_t)cursor != tri_count)
      bad(W, "leaf ranges cover " + std::to_string(cursor) + " triangle(s); expected " + std::to_string(tri_count));
  }
  return p;
}

WideProof validate_wide(const uint32_t* nodes_in, size_t n_local, const float* recs_in, size_t n_recs_local,
                        uint32_t root, size_t n_items, bool instance_records, int stack_cap, uint32_t node_base,
                        uint32_t rec_base) {
  const std::string W = "8-wide encoding proof";
  WideProof p;
  // absolute indexing: node i lives at nodes_in[20 * (i - node_base)]
  const uint32_t* nodes = nodes_in - 20 * (ptrdiff_t)node_base;
  const float* recs = recs_in - 16 * (ptrdiff_t)rec_base;
  const size_t n_nodes = node_base + n_local, n_recs = rec_base + n_recs_local;
  if (root < node_base || root >= n_nodes)
    bad(W, "root " + std::to_string(root) + " outside nodes [" + std::to_string(node_base) + ", " +
               std::to_string(n_nodes) + ")");
  std::vector<uint8_t> item_seen(n_items, 0);
  // breadth-first walk; each entry carries the intersection of its ancestors'
  // slot boxes -- what a ray must pass to reach it
  // boxes in 113-bit arithmetic: origin + q * 2^e is exact there (bvh_encode.cpp)
  using Q = __float128;
  struct Item { uint32_t node; int depth; Q cull[6]; };
  std::vector<Item> queue(1);
  queue[0].node = root;
  queue[0].depth = 1;
  for (int k = 0; k < 3; ++k) { queue[0].cull[k] = (Q)-INFINITY; queue[0].cull[3 + k] = (Q)INFINITY; }
  std::vector<uint8_t> visited(n_nodes - root, 0);  // this tree's nodes follow its root
  for (size_t qi = 0; qi < queue.size(); ++qi) {
    const Item it = queue[qi];
    const uint32_t node = it.node;
    if (node < root || node >= n_nodes) bad(W, "child index " + std::to_string(node) + " outside the tree's nodes");
    if (visited[node - root]) bad(W, "node " + std::to_string(node) + " is reachable more than once");
    visited[node - root] = 1;
    p.node_count += 1;
    p.depth = std::max<int64_t>(p.depth, it.depth);
    const uint32_t* w = nodes + 20 * (size_t)node;
    const uint8_t* bytes = reinterpret_cast<const uint8_t*>(w);
    const Q org[3] = {(Q)f32_of(w[0]), (Q)f32_of(w[1]), (Q)f32_of(w[2])};
    int ex[3];
    for (int k = 0; k < 3; ++k) ex[k] = (int)bytes[12 + k] - 127;
    const uint8_t imask = bytes[15];
    const uint32_t child_base = w[4], tri_base = w[5], tri_valid = w[6];
    const uint8_t* qlo = bytes + 32;
    const uint8_t* qhi = bytes + 56;
    int internal_seen = 0;
    for (int s = 0; s < 8; ++s) {
      const std::string at = "node " + std::to_string(node) + " slot " + std::to_string(s);
      const uint32_t nib = (tri_valid >> (4 * s)) & 0xFu;
      const bool internal = (imask >> s) & 1u;
      if (!internal && nib == 0) {
        for (int k = 0; k < 3; ++k)
          if (qlo[k * 8 + s] != 255 || qhi[k * 8 + s] != 0) bad(W, at + " is empty but its box is not inverted");
        continue;
      }
      Q box[6];
      for (int k = 0; k < 3; ++k) {
        if (qlo[k * 8 + s] > qhi[k * 8 + s]) bad(W, at + " has an inverted box");
        // the slot box, intersected with the ancestors' boxes
        const Q lo = org[k] + (Q)std::ldexp((double)qlo[k * 8 + s], ex[k]);
        const Q hi = org[k] + (Q)std::ldexp((double)qhi[k * 8 + s], ex[k]);
        box[k] = it.cull[k] > lo ? it.cull[k] : lo;
        box[3 + k] = it.cull[3 + k] < hi ? it.cull[3 + k] : hi;
      }
      if (internal) {
        if (nib) bad(W, at + " is internal and owns records");
        const uint64_t child = (uint64_t)child_base + internal_seen++;
        if (child >= n_nodes) bad(W, at + " child " + std::to_string(child) + " is outside the node array");
        Item c;
        c.node = (uint32_t)child;
        c.depth = it.depth + 1;
        std::memcpy(c.cull, box, sizeof box);
        queue.push_back(c);
        p.internal_slots += 1;
        continue;
      }
      if (nib != 0x1u && nib != 0x3u && nib != 0x7u && nib != 0xFu) bad(W, at + " record mask is not contiguous");
      p.leaf_slots += 1;
      const int cnt = nib == 0x1u ? 1 : nib == 0x3u ? 2 : nib == 0x7u ? 3 : 4;
      for (int i = 0; i < cnt; ++i) {
        const uint64_t r = (uint64_t)tri_base + 4u * (uint32_t)s + (uint32_t)i;
        if (r < rec_base || r >= n_recs)
          bad(W, at + " record " + std::to_string(r) + " is outside [" + std::to_string(rec_base) + ", " +
                     std::to_string(n_recs) + ")");
        const float* rec = recs + 16 * r;
        uint32_t id;
        std::memcpy(&id, rec + (instance_records ? 13 : 3), 4);
        if (id >= n_items) bad(W, "record " + std::to_string(r) + " names item " + std::to_string(id) + " of " +
                                      std::to_string(n_items));
        if (item_seen[id]) bad(W, "item " + std::to_string(id) + " is named by more than one leaf record");
        item_seen[id] = 1;
        p.items += 1;
        // a top level's leaves hold instances, whose world boxes are not stored;
        // a triangle the watertight normal derivation rejects (valid 0) is never hit
        if (instance_records || rec[15] == 0.0f) continue;
        for (int v = 0; v < 3; ++v)
          for (int k = 0; k < 3; ++k) {
            const Q x = (Q)rec[4 * v + k];
            if (!(x >= box[k] && x <= box[3 + k]))
              bad(W, at + ": a vertex of record " + std::to_string(r) + " lies outside the boxes that cull it");
          }
      }
    }
  }
  if (p.items != (int64_t)n_items)
    bad(W, "leaf records name " + std::to_string(p.items) + " of " + std::to_string(n_items) + " item(s)");
  p.stack_entries = 2 * p.depth + 2;
  if (p.stack_entries > stack_cap)
    bad(W, "traversal needs " + std::to_string(p.stack_entries) + " stack entries, capacity " + std::to_string(stack_cap));
  return p;
}

}  // namespace vt
