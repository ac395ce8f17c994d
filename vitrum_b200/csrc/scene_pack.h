// scene_pack.h -- a vt_scene_desc packed into the device layouts (host arrays).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <vector>

#include "../../include/vitrum_pt.h"
#include "bvh_host.h"
#include "pt_common.cuh"
#include "vt_common.h"

namespace vt {

struct PackedScene {
  BinaryBvhHost binary;              // the tree (single level) or the top level over the instances
  bool two_level = false;
  std::vector<uint32_t> node_words;  // 20 words per wide node, indices offset by node_base
  std::vector<float> rec_floats;     // 16 floats per triangle record, offset by rec_base
  int depth = 1, stack_depth = 4;
  uint32_t root = 0;                 // first node of the traversal
  std::vector<float> inst_lanes, inst_tab, inst_rows;  // two-level: leaf-order records, by id, local-to-world rows
  size_t n_instances = 0;
  std::vector<pt::Material> mats;
  std::vector<float4> emitters;      // 3 float4 per emissive triangle (world space)
  std::vector<float> cdf;            // inclusive area CDF
  double emit_total = 0.0;
  std::vector<float4> points;        // kPositionalF4 float4 per point or spot light
  std::vector<float4> area_lights;   // kAreaLightF4 float4 per rectangle or disc light
  std::vector<float4> dirs;          // 2 float4 per directional light
  std::vector<float4> env;
  std::vector<float> marg, cond;
  bool has_env = false, env_sampleable = false;
  int env_w = 0, env_h = 0;
  float env_scale = 1.0f;
  float env_rotation = 0.0f;
  std::vector<float> light_tree;     // packed light tree over the light entries (two or more entries)
  size_t ntri = 0;
  // two-level: per mesh its bottom-level root node and local bounds; the deepest bottom level
  std::vector<uint32_t> blas_root;
  std::vector<std::array<double, 6>> local_box;
  std::vector<uint32_t> blas_rec_start;  // first triangle record of each mesh's block
  std::vector<int> blas_depths;          // wide depth of each bottom level
  int blas_depth = 0;
};

// Validates mesh m and appends its vertices (4 floats each), triangles (4 u32
// each, indices rebased) and triangle materials.
void append_mesh(const vt_mesh_desc& md, size_t m, size_t material_count, std::vector<float>& pos,
                 std::vector<uint32_t>& idx, std::vector<uint32_t>& tri_mat);
// One mesh's bottom-level tree (the engine's builder options and collapse),
// its node and record indices offset by node_base / rec_base.
struct BlasPack {
  WideBvhHost wide;
  std::array<double, 6> local_box;
};
// Where a scene's trees are built: on the GPU (device, stream) or on the host;
// validate runs the publication proofs on the result.
struct SceneBuild {
  bool gpu = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool validate = true;
  int bvh_width = 8;  // children per wide node at most of the triangle trees (2..8)
};
BlasPack pack_blas(const std::vector<float>& pos, const std::vector<uint32_t>& idx, uint32_t material,
                   uint32_t node_base, uint32_t rec_base, int max_leaf, const SceneBuild& sb = SceneBuild());

// Instances placed over bottom-level trees: records (world-to-local rows, BLAS
// root, id, material, material flags), world AABBs (6 doubles each) and
// local-to-world rows (12 floats each).
struct InstanceSet {
  std::vector<InstanceRecord> recs;
  std::vector<double> aabbs;
  std::vector<float> rows;
};
InstanceSet place_instances(const vt_instance_desc* insts, size_t n, const std::vector<pt::Material>& mats,
                            const std::vector<uint32_t>& blas_root,
                            const std::vector<std::array<double, 6>>& local_box);
// The top level over instance AABBs (6 doubles each) and its 8-wide encoding
// with instance records, on the GPU or on the host as sb says (the same words).
BinaryBvhHost build_top_level(const SceneBuild& sb, const double* aabbs, size_t n);
WideBvhHost encode_top_level(const SceneBuild& sb, const BinaryBvhHost& tl, const std::vector<InstanceRecord>& recs,
                             uint32_t root);
// New instance AABBs into an existing top level: same topology, bounds recomputed bottom-up.
void refit_tlas_host(BinaryBvhHost& tl, const double* aabbs, size_t n);

// Validates and packs; single-level trees are offset by node_base / rec_base
// (scenes concatenated into shared arrays); instanced scenes need both zero.
PackedScene pack_scene(const vt_scene_desc* sc, uint32_t node_base, uint32_t rec_base, int max_leaf = 4,
                       const SceneBuild& sb = SceneBuild());

// Triangles per leaf of the path tracer's own trees when the options leave it
// open: two per leaf traced the box room 4 % and the instanced cloud 7 % faster
// than the reference build's default of four (fewer watertight tests per ray
// for a few more node visits).
constexpr int kEngineLeafDefault = 2;
// SAH bins of the path tracer's trees: 32 instead of the reference's 16 traced
// the box room 1.4 % faster for a 0.05 s longer build.
constexpr int kEngineBins = 32;
// Wide collapse of the path tracer's triangle trees: the SAH-optimal rule with
// these weights traced the box room 4.9 % faster than the reference's greedy
// collapse (0.3 or 0.25 per triangle merged more leaves and was slower); the
// top level keeps the greedy collapse.
constexpr WideCollapse kEngineCollapse{1.0, 0.5};

// 4x4 inverse (Gauss-Jordan, partial pivoting); false when singular.
bool invert4(const double* m, double* inv);
// inverse(P * V) of column-major view / projection as a row-major float matrix.
void inverse_view_proj(const float* view, const float* proj, float* out_rm);
// P * V of column-major view / projection as a row-major float matrix.
void view_proj(const float* view, const float* proj, float* out_rm);

}  // namespace vt
