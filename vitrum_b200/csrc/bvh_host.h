// bvh_host.h -- host-side containers of the BVH build pipeline.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "bvh_types.h"
#include "vt_common.h"

namespace vt {

struct BuildOptions {
  int position_stride = 4;
  int index_stride = 4;
  int max_leaf = 4;
  int bins = 16;
  int max_depth = kMaxBinaryDepth;
  // tree the queries traverse: 1 this tree, reference grouping; 2 this tree, SAH-optimal
  // grouping; 3 a second tree (<= 2 per leaf, 32 bins), SAH-optimal grouping
  int traversal_tree = 3;
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

// Structural proof of a packed binary BVH (the reference's validateBvhEncoding,
// shared-bvh/src/validateBvhEncoding.ts:55); throws vt::Error(VT_ERR_BUILD).
// roots == nullptr: root 0; tri_count < 0: leaf ranges are not checked.
struct BinaryProof {
  int64_t node_count = 0, root_count = 0, interior_node_count = 0, leaf_node_count = 0, max_depth = 0,
          max_stack_entries = 0, stack_capacity = 0, triangle_count = -1;
};
BinaryProof validate_binary_encoding(const uint32_t* words, size_t word_count, size_t total_nodes,
                                     const uint32_t* roots, size_t n_roots, int64_t tri_count, int stack_cap);
inline BinaryProof validate_binary(const BinaryBvhHost& b, int64_t tri_count, int stack_cap = 60) {
  return validate_binary_encoding(reinterpret_cast<const uint32_t*>(b.nodes.data()), b.nodes.size() * 8,
                                  b.nodes.size(), nullptr, 0, tri_count, stack_cap);
}

// Structural proof of one 8-wide tree (bvh_validate.cpp): node indices are
// absolute, the arrays start at node node_base / record rec_base; items are
// triangles (source id in v0.w) or, for a top level, instances (instance id).
struct WideProof {
  int64_t node_count = 0, internal_slots = 0, leaf_slots = 0, items = 0, depth = 0, stack_entries = 0;
};
WideProof validate_wide(const uint32_t* nodes, size_t n_nodes, const float* recs, size_t n_recs, uint32_t root,
                        size_t n_items, bool instance_records, int stack_cap, uint32_t node_base = 0,
                        uint32_t rec_base = 0);
// Device copies of a binary tree: nodes in preorder and the BVH-order
// triangle permutation (reordered_to_source).
struct BinaryBvhDevice {
  DeviceBuffer<BinaryNode> nodes;
  DeviceBuffer<uint32_t> order;
  size_t n_nodes = 0, ntri = 0;
};
// The same tree built on the GPU from device positions / indices; with keep,
// its device arrays are handed over for a device encoding.
BinaryBvhHost build_binary_gpu(const float* d_pos, size_t position_words, const uint32_t* d_idx, size_t index_words,
                               const BuildOptions& o, cudaStream_t s, BinaryBvhDevice* keep = nullptr);

// Binned-SAH binary build on host arrays (throws vt::Error).
BinaryBvhHost build_binary_host(const float* positions, size_t position_words, const uint32_t* indices,
                                size_t index_words, const BuildOptions& o);

// 8-wide collapse of one binary interior node (reference greedy rule).
int collect_wide_children(const BinaryNode* nodes, uint32_t root, uint32_t out[8]);

// Surface-area cost weights of the SAH-optimal collapse: c_node per wide node
// entered, c_tri per triangle tested, both per unit of box half-area; width:
// children per wide node at most (2..8; the node format holds 8).
struct WideCollapse {
  double c_node = 1.0;
  double c_tri = 0.5;
  int width = 8;
};

// Device copies of an encoded tree: 20 words per wide node, 16 floats per record.
struct WideBvhDevice {
  DeviceBuffer<uint32_t> nodes;
  DeviceBuffer<float> recs;
  size_t n_nodes = 0, n_recs = 0;
};
// encode_wide on the GPU from a device binary tree (bvh_encode_gpu.cu): the
// same node words and records.  Triangle records from d_pos / d_idx (and
// d_tri_mat), or, with d_inst_recs (16 floats per instance), a top level's
// instance records; sah == nullptr: the reference's greedy collapse.  The
// result is returned on the host; with keep also kept on the device.
WideBvhHost encode_wide_gpu(const BinaryBvhDevice& bin, const float* d_pos, int pos_stride, const uint32_t* d_idx,
                            int idx_stride, const uint32_t* d_tri_mat, uint32_t node_base, uint32_t rec_base,
                            const WideCollapse* sah, const float* d_inst_recs, cudaStream_t s,
                            WideBvhDevice* keep = nullptr);

// tri_materials (optional, one per source triangle) is stored in each record's v1.w.
// node_base / rec_base offset the encoded indices for trees concatenated into shared arrays.
// sah == nullptr: the reference's greedy collapse; else the SAH-optimal one with those weights.
WideBvhHost encode_wide(const BinaryBvhHost& bin, const float* positions, int pos_stride, const uint32_t* indices,
                        int idx_stride, const uint32_t* tri_materials = nullptr, uint32_t node_base = 0,
                        uint32_t rec_base = 0, const WideCollapse* sah = nullptr);

// Top-level instance record (64 bytes): world-to-local affine rows, then
// (BLAS root node, instance id, material, 0) as u32 bits.
struct InstanceRecord {
  float w2l[12];
  uint32_t blas_root;
  uint32_t instance_id;
  uint32_t material;
  uint32_t pad;
};
static_assert(sizeof(InstanceRecord) == 64, "instance record is 64 bytes");

// Binned-SAH TLAS over instance AABBs, the reference's buildTlas
// (shared-bvh/src/tlas.ts:859-989): aabbs = 6 doubles per instance.
BinaryBvhHost build_tlas_host(const double* aabbs, size_t n, int max_leaf = 1, int bins = 16,
                              int max_depth = kMaxBinaryDepth);

// The same top level built on the GPU (tlas_build_gpu.cu), word for word; with
// keep, its device arrays are handed over for a device encoding.
BinaryBvhHost build_tlas_gpu(const double* aabbs, size_t n, int max_leaf, int bins, int max_depth, cudaStream_t s,
                             BinaryBvhDevice* keep = nullptr);

// Wide encoding of a TLAS: leaf payload records are InstanceRecords.
WideBvhHost encode_wide_tlas(const BinaryBvhHost& tlas, const InstanceRecord* instances, uint32_t node_base);

}  // namespace vt
