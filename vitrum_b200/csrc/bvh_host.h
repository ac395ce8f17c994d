// bvh_host.h -- host-side containers of the BVH build pipeline.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "bvh_types.h"

namespace vt {

struct BuildOptions {
  int position_stride = 4;
  int index_stride = 4;
  int max_leaf = 4;
  int bins = 16;
  int max_depth = kMaxBinaryDepth;
};

struct BinaryBvhHost {
  std::vector<BinaryNode> nodes;
  std::vector<uint32_t> reordered_to_source;
  int depth = 0;  // deepest interior level reached
};

struct WideBvhHost {
  std::vector<uint32_t> nodes;  // 20 words per wide node
  std::vector<float> tris;      // 16 floats per triangle record slot
  int depth = 0;
};

void validate_options(const BuildOptions& o);

// Binned-SAH binary build on host arrays (throws vt::Error).
BinaryBvhHost build_binary_host(const float* positions, size_t position_words, const uint32_t* indices,
                                size_t index_words, const BuildOptions& o);

// 8-wide collapse of one binary interior node (reference greedy rule).
int collect_wide_children(const BinaryNode* nodes, uint32_t root, uint32_t out[8]);

// tri_materials (optional, one per source triangle) is stored in each record's v1.w.
WideBvhHost encode_wide(const BinaryBvhHost& bin, const float* positions, int pos_stride, const uint32_t* indices,
                        int idx_stride, const uint32_t* tri_materials = nullptr);

}  // namespace vt
