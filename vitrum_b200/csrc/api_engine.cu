// api_engine.cu -- the path-tracing engine behind the vitrum Engine contract.
//
// vt_create / vt_set_scene / vt_render_frame / vt_capture / vt_pick /
// vt_reset / vt_destroy mirror createPTEngine_WebGPU and the @vitrum/core
// Engine methods (packages/core/src/engine/index.ts:109-466,
// packages/pt-webgpu/src/index.ts:418-2363).  A frame is rendered as waves
// of width*height*spp_wave paths; each wave's launches (raygen, per bounce:
// extend, material sort, shade, shadow, resolve; accumulate) are captured
// once into a CUDA graph and replayed, the wave's sample offset living in
// device memory so replays need no parameter updates.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "bvh_host.h"
#include "nrc_cache.h"
#include "scene_pack.h"
#include "pt_kernels.h"
#include "ray_order.h"
#include "traverse.h"
#include "vt_common.h"

using vt::DeviceBuffer;
using vt::fail;

// Radiance-cache state of an engine.
struct NrcEngine {
  vt_nrc_render_options opts{};
  std::unique_ptr<vt::nrc::Cache> cache;
  vt::DeviceBuffer<float4> records, queries, samples;
  vt::DeviceBuffer<uint32_t> seed;
  vt::DeviceBuffer<float> tile_stats, tile_error;  // fallback: per screen tile (sums; error EMA)
  uint32_t tiles_x = 0, tiles_y = 0, tile_width = 0;
  uint32_t train_paths = 0;
  int frames = 0;  // frames rendered since the cache was created
};

// Morton bits per axis of the engine's spatial trace orders: closest-hit queues
// (sort_rays 2) by 2^6 cells per axis (2^21 buckets, about a hundred rays each at
// a 16 M-path wave on one room); shadow queues (sort_rays 3), whose rays from one
// cell head for the same few lights, by 2^4 (2^15 buckets: lanes of a warp share
// buckets, so the counting atomics aggregate).
constexpr int kEngineOrderCellBits = 6;
constexpr int kShadowOrderCellBits = 4;

struct vt_engine {
  int device = 0;
  vt_engine_options opts{};
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // shadow stream: bounce b's shadow trace and resolve run beside bounce b+1's
  // closest-hit trace (fork after shade b, join before shade b+1)
  cudaStream_t shadow_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // scene
  bool has_scene = false;
  vt::BinaryBvhHost binary;
  DeviceBuffer<uint4> nodes;
  DeviceBuffer<float4> tris;
  int wide_depth = 1;
  int stack_depth = 16;            // traversal stack entries the scene needs
  DeviceBuffer<float4> insts;      // instance records in top-level leaf order
  DeviceBuffer<float4> inst_table; // instance records by instance index
  DeviceBuffer<float4> inst_l2w;   // local-to-world rows by instance index (hit refinement)
  int64_t n_instances = 0;
  // two-level scenes, for instance updates: bottom-level roots / local bounds per
  // mesh, the deepest bottom level, the top level's first node, host materials
  std::vector<uint32_t> blas_root;
  std::vector<std::array<double, 6>> local_box;
  int blas_depth = 0;
  uint32_t tlas_root = 0;
  std::vector<vt::pt::Material> mats_host;
  // two-level scenes, for mesh updates: host copies of the bottom-level node
  // words (tlas_root wide nodes) and of the triangle records, each mesh's first
  // record and wide depth, and the current placements
  std::vector<uint32_t> blas_words;
  std::vector<float> rec_host;
  std::vector<uint32_t> blas_rec_start;
  std::vector<int> blas_depths;
  std::vector<size_t> mesh_tris;   // source triangles per mesh
  std::vector<vt_instance_desc> inst_descs;
  // vt_trace_rays staging
  DeviceBuffer<float4> q_rays;
  DeviceBuffer<int4> q_hits;
  DeviceBuffer<int> q_inst, q_status;
  DeviceBuffer<unsigned long long> q_counter;
  DeviceBuffer<vt::pt::Material> materials;
  DeviceBuffer<float4> emitters;
  DeviceBuffer<float> emitter_cdf;
  DeviceBuffer<float4> points, dirs, area_lights;
  DeviceBuffer<float4> env;
  DeviceBuffer<float> env_marginal, env_conditional;
  DeviceBuffer<float> light_tree;  // packed light tree (light_tree.h), empty below two light entries
  vt::pt::SceneView view;
  int64_t ntri = 0, n_emitters = 0;
  // accumulation
  int width = 0, height = 0;
  DeviceBuffer<float4> accum;
  DeviceBuffer<float4> present;     // present-pass output of vt_capture_output
  DeviceBuffer<double> sum64, sq64, lum64;
  // auxiliary outputs (first-hit normal / depth, albedo, motion; luminance
  // moments) and their per-frame constants (view-projections, recorded sample)
  DeviceBuffer<float4> aux_nd, aux_albedo, aux_motion, aux_moments;
  DeviceBuffer<float> aux_consts;
  float aux_host[vt::pt::kAuxConsts] = {};
  bool have_prev_camera = false;   // set by vt_set_previous_camera for the next frame only
  float prev_view[16] = {}, prev_proj[16] = {};
  int samples = 0;
  float inv_vp[16] = {};
  float view_m[16] = {}, proj_m[16] = {};
  bool have_camera = false;
  uint32_t frame_seed = 0;
  mutable uint32_t auto_wave_paths = 0;  // default wave size, fitted to free memory once (wave_paths_of)
  // wave buffers
  uint32_t capacity = 0;
  DeviceBuffer<float4> rays[2], through[2];
  DeviceBuffer<uint4> state[2];
  DeviceBuffer<int4> hits;
  DeviceBuffer<uint32_t> order, keys, counters;
  DeviceBuffer<float4> shadow_rays, shadow_contrib, radiance;
  DeviceBuffer<uint32_t> path_pixel;  // training paths: their pixel
  DeviceBuffer<uint8_t> occluded;
  DeviceBuffer<unsigned long long> trace_counter, shadow_counter, totals;
  DeviceBuffer<int> trace_status;
  std::unique_ptr<NrcEngine> nrc;
  int trace_blocks_per_sm = 0;      // traversal CTAs per SM (0: occupancy limit), from the autotuner
  bool trace_stage_nodes = false;   // traversal CTAs stage the top of the tree in shared memory
  int sort_rays = 0;               // trace order: 0 queue order; closest-hit queues of bounces >= 1 by
                                    // 1 direction octant or 2 origin cell (Morton) and octant; 3 shadow
                                    // queues by origin cell and octant
  DeviceBuffer<uint32_t> ray_order_counts;  // buckets of the spatial trace order (sort_rays 2)
  DeviceBuffer<uint32_t> shadow_keys, shadow_order, shadow_order_counts;  // the shadow queues' (sort_rays 3)
  long long debug_wait_cycles = 0;  // failure-detection hook: first-wait limit of bounded waits (0: default)
  // graph cache: one executable per wave shape and mode
  struct Graph {
    uint32_t spp_wave = 0, bounces = 0;
    int mode = 0;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<Graph> graphs;
  double last_ms = 0.0;
  // pick
  DeviceBuffer<float4> pick_ray;
  DeviceBuffer<int4> pick_hit;
  DeviceBuffer<int> pick_status;
  DeviceBuffer<unsigned long long> pick_counter;

  void drop_graphs() {
    for (auto& g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    graphs.clear();
  }
  ~vt_engine() {
    drop_graphs();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (shadow_stream) cudaStreamDestroy(shadow_stream);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

void nrc_rebuild(vt_engine* e);
void reset_accumulation(vt_engine* e);

template <class T>
void upload(DeviceBuffer<T>& dst, const std::vector<T>& src, cudaStream_t s) {
  dst.resize(std::max<size_t>(src.size(), 1));
  if (!src.empty()) VT_CUDA(cudaMemcpyAsync(dst.ptr, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

// ---------------------------------------------------------------- scene
static vt::SceneBuild scene_build_of(const vt_engine* e) {
  vt::SceneBuild sb;
  sb.gpu = e->opts.scene_build == 0;
  sb.device = e->device;
  sb.stream = e->stream;
  sb.validate = e->opts.debug != 0;
  sb.bvh_width = e->opts.bvh_width;
  return sb;
}

void set_scene(vt_engine* e, const vt_scene_desc* sc) {
  // Transactional replacement (the reference's staged upload with rollback,
  // pt-webgpu/src/scene/uploadSceneBuffers.ts, transactionalResourceReplacement.test.ts):
  // every device buffer of the new scene is allocated and filled first; only
  // when all of them succeeded do they replace the engine's, so a failure at
  // any stage leaves the previous scene and its image untouched.
  vt::PackedScene p = vt::pack_scene(sc, 0, 0, e->opts.bvh_max_leaf, scene_build_of(e));
  cudaStream_t s = e->stream;
  struct Staged {
    DeviceBuffer<uint4> nodes;
    DeviceBuffer<float4> tris, insts, inst_table, inst_l2w;
    DeviceBuffer<vt::pt::Material> materials;
    DeviceBuffer<float4> emitters, points, area_lights, dirs, env;
    DeviceBuffer<float> emitter_cdf, env_marginal, env_conditional, light_tree;
  } n;
  n.nodes.resize(p.node_words.size() / 4);
  VT_CUDA(cudaMemcpyAsync(n.nodes.ptr, p.node_words.data(), p.node_words.size() * 4, cudaMemcpyHostToDevice, s));
  n.tris.resize(std::max<size_t>(p.rec_floats.size() / 4, 1));
  if (!p.rec_floats.empty())
    VT_CUDA(cudaMemcpyAsync(n.tris.ptr, p.rec_floats.data(), p.rec_floats.size() * 4, cudaMemcpyHostToDevice, s));
  const bool two_level = p.two_level;
  std::vector<float4> il(p.inst_lanes.size() / 4), it(p.inst_tab.size() / 4), ir(p.inst_rows.size() / 4);
  if (!il.empty()) std::memcpy(il.data(), p.inst_lanes.data(), p.inst_lanes.size() * 4);
  if (!it.empty()) std::memcpy(it.data(), p.inst_tab.data(), p.inst_tab.size() * 4);
  if (!ir.empty()) std::memcpy(ir.data(), p.inst_rows.data(), p.inst_rows.size() * 4);
  upload(n.insts, il, s);
  upload(n.inst_table, it, s);
  upload(n.inst_l2w, ir, s);
  upload(n.materials, p.mats, s);
  upload(n.emitters, p.emitters, s);
  upload(n.emitter_cdf, p.cdf, s);
  upload(n.points, p.points, s);
  upload(n.area_lights, p.area_lights, s);
  upload(n.dirs, p.dirs, s);
  upload(n.env, p.env, s);
  upload(n.env_marginal, p.marg, s);
  upload(n.env_conditional, p.cond, s);
  upload(n.light_tree, p.light_tree, s);
  VT_CUDA(cudaStreamSynchronize(s));
  // commit
  e->drop_graphs();
  e->nodes = std::move(n.nodes);
  e->tris = std::move(n.tris);
  e->insts = std::move(n.insts);
  e->inst_table = std::move(n.inst_table);
  e->inst_l2w = std::move(n.inst_l2w);
  e->materials = std::move(n.materials);
  e->emitters = std::move(n.emitters);
  e->emitter_cdf = std::move(n.emitter_cdf);
  e->points = std::move(n.points);
  e->area_lights = std::move(n.area_lights);
  e->dirs = std::move(n.dirs);
  e->env = std::move(n.env);
  e->env_marginal = std::move(n.env_marginal);
  e->env_conditional = std::move(n.env_conditional);
  e->light_tree = std::move(n.light_tree);
  e->wide_depth = p.depth;
  e->stack_depth = p.stack_depth;
  e->n_instances = (int64_t)p.n_instances;
  vt::pt::SceneView v;
  v.nodes = e->nodes.ptr;
  v.tris = e->tris.ptr;
  v.stack_depth = e->stack_depth;
  v.insts = two_level ? e->insts.ptr : nullptr;
  v.inst_table = two_level ? e->inst_table.ptr : nullptr;
  v.root = p.root;
  v.materials = e->materials.ptr;
  v.material_count = (uint32_t)p.mats.size();
  v.emitters = e->emitters.ptr;
  v.emitter_cdf = e->emitter_cdf.ptr;
  v.n_emitters = (uint32_t)p.cdf.size();
  v.emit_area_total = (float)p.emit_total;
  v.points = e->points.ptr;
  v.n_points = (uint32_t)(p.points.size() / vt::pt::kPositionalF4);
  v.area_lights = e->area_lights.ptr;
  v.n_area = (uint32_t)(p.area_lights.size() / vt::pt::kAreaLightF4);
  v.dirs = e->dirs.ptr;
  v.n_dirs = (uint32_t)(p.dirs.size() / 2);
  v.env = p.has_env ? e->env.ptr : nullptr;
  v.env_marginal = p.env_sampleable ? e->env_marginal.ptr : nullptr;
  v.env_conditional = p.env_sampleable ? e->env_conditional.ptr : nullptr;
  v.env_w = p.env_w;
  v.env_h = p.env_h;
  v.env_scale = p.env_scale;
  v.env_cos = (float)std::cos((double)p.env_rotation);
  v.env_sin = (float)std::sin((double)p.env_rotation);
  v.n_light_entries = (v.n_emitters ? 1u : 0u) + v.n_points + v.n_area + v.n_dirs + (p.env_sampleable ? 1u : 0u);
  v.light_tree_mode = e->opts.light_selection == 0 && v.n_light_entries >= 2;
  v.light_tree = (v.light_tree_mode && !p.light_tree.empty()) ? e->light_tree.ptr : nullptr;
  e->view = v;
  e->binary = std::move(p.binary);
  e->blas_root = std::move(p.blas_root);
  e->local_box = std::move(p.local_box);
  e->blas_depth = p.blas_depth;
  e->tlas_root = p.root;
  e->mats_host = p.mats;
  e->blas_rec_start = std::move(p.blas_rec_start);
  e->blas_depths = std::move(p.blas_depths);
  if (two_level) {
    e->blas_words.assign(p.node_words.begin(), p.node_words.begin() + (size_t)p.root * 20);
    e->rec_host = std::move(p.rec_floats);
    e->inst_descs.assign(sc->instances, sc->instances + sc->instance_count);
    e->mesh_tris.resize(sc->mesh_count);
    for (size_t m = 0; m < sc->mesh_count; ++m) e->mesh_tris[m] = sc->meshes[m].triangle_count;
  } else {
    e->mesh_tris.clear();
    e->blas_words.clear();
    e->rec_host.clear();
    e->inst_descs.clear();
  }
  e->ntri = (int64_t)p.ntri;
  e->n_emitters = (int64_t)v.n_emitters;
  e->has_scene = true;
  if (e->nrc) nrc_rebuild(e);
  reset_accumulation(e);
  VT_CUDA(cudaStreamSynchronize(e->stream));
}

// New placements for the instances of a two-level scene (refitTlasTransforms /
// rebuildTlasReuseBlas, shared-bvh/src/scenePack.ts:1310, 1635): the bottom
// levels stay; the top level is refitted (same topology, new bounds) or rebuilt
// (binned SAH over the new instance bounds), re-encoded and uploaded.
void update_instances(vt_engine* e, const vt_instance_desc* insts, size_t n, bool rebuild) {
  if (!e->has_scene || e->n_instances == 0) fail(VT_ERR_STATE, "instance updates need a scene with instances");
  if (n != (size_t)e->n_instances)
    fail(VT_ERR_INVALID_ARGUMENT, "expected " + std::to_string(e->n_instances) + " instances, got " +
                                      std::to_string(n) + " (set a new scene to change the membership)");
  if (!insts) fail(VT_ERR_INVALID_ARGUMENT, "instances is null");
  vt::InstanceSet placed = vt::place_instances(insts, n, e->mats_host, e->blas_root, e->local_box);
  if (insts != e->inst_descs.data()) e->inst_descs.assign(insts, insts + n);
  vt::BinaryBvhHost tl;
  const vt::SceneBuild sb = scene_build_of(e);
  if (rebuild) {
    tl = vt::build_top_level(sb, placed.aabbs.data(), n);
  } else {
    tl = e->binary;
    vt::refit_tlas_host(tl, placed.aabbs.data(), n);
  }
  vt::WideBvhHost tw = vt::encode_top_level(sb, tl, placed.recs, e->tlas_root);
  cudaStream_t s = e->stream;
  VT_CUDA(cudaStreamSynchronize(s));
  e->drop_graphs();
  const size_t blas_u4 = (size_t)e->tlas_root * 5, tlas_u4 = tw.nodes.size() / 4;
  if (blas_u4 + tlas_u4 != e->nodes.count) {
    DeviceBuffer<uint4> grown(blas_u4 + tlas_u4);
    if (blas_u4)
      VT_CUDA(cudaMemcpyAsync(grown.ptr, e->nodes.ptr, blas_u4 * sizeof(uint4), cudaMemcpyDeviceToDevice, s));
    VT_CUDA(cudaStreamSynchronize(s));
    e->nodes = std::move(grown);
  }
  VT_CUDA(cudaMemcpyAsync(e->nodes.ptr + blas_u4, tw.nodes.data(), tw.nodes.size() * 4, cudaMemcpyHostToDevice, s));
  std::vector<float4> il(tw.tris.size() / 4), it(n * 4), ir(placed.rows.size() / 4);
  if (!il.empty()) std::memcpy(il.data(), tw.tris.data(), tw.tris.size() * 4);
  std::memcpy(it.data(), placed.recs.data(), n * sizeof(vt::InstanceRecord));
  if (!ir.empty()) std::memcpy(ir.data(), placed.rows.data(), placed.rows.size() * 4);
  upload(e->insts, il, s);
  upload(e->inst_table, it, s);
  upload(e->inst_l2w, ir, s);
  VT_CUDA(cudaStreamSynchronize(s));
  e->binary = std::move(tl);
  e->wide_depth = tw.depth + e->blas_depth;
  e->stack_depth = 2 * e->wide_depth + 6;
  e->view.nodes = e->nodes.ptr;
  e->view.stack_depth = e->stack_depth;
  e->view.insts = e->insts.ptr;
  e->view.inst_table = e->inst_table.ptr;
  reset_accumulation(e);
  VT_CUDA(cudaStreamSynchronize(e->stream));
}

// New geometry for one mesh of a two-level scene (rebuildPrimitiveBlas,
// shared-bvh/src/scenePack.ts:1763, and its in-place / resized splices
// :1006-1100): the mesh's bottom level is rebuilt and spliced into the
// concatenated node and record arrays; when its size changed, the later
// meshes' node and record indices and roots are rebased.  The top level is
// then refitted (or rebuilt) over the instances' new bounds.
void update_mesh(vt_engine* e, size_t m, const vt_mesh_desc* md, bool rebuild) {
  if (!e->has_scene || e->n_instances == 0)
    fail(VT_ERR_STATE, "mesh updates need a scene with instances (set the scene again to change a flat scene)");
  if (!md) fail(VT_ERR_INVALID_ARGUMENT, "mesh is null");
  const size_t nm = e->blas_root.size();
  if (m >= nm) fail(VT_ERR_RANGE, "mesh index " + std::to_string(m) + " out of range");
  std::vector<float> pos;
  std::vector<uint32_t> idx, tri_mat;
  vt::append_mesh(*md, m, e->mats_host.size(), pos, idx, tri_mat);
  const uint32_t node0 = e->blas_root[m], rec0 = e->blas_rec_start[m];
  const uint32_t node1 = m + 1 < nm ? e->blas_root[m + 1] : e->tlas_root;
  const uint32_t rec1 = m + 1 < nm ? e->blas_rec_start[m + 1] : (uint32_t)(e->rec_host.size() / 16);
  const uint32_t old_tlas_root = e->tlas_root;
  vt::BlasPack bp = vt::pack_blas(pos, idx, md->material, node0, rec0, e->opts.bvh_max_leaf, scene_build_of(e));
  const int64_t dn = (int64_t)(bp.wide.nodes.size() / 20) - (int64_t)(node1 - node0);
  const int64_t dr = (int64_t)(bp.wide.tris.size() / 16) - (int64_t)(rec1 - rec0);
  if ((int64_t)e->rec_host.size() / 16 + dr + 32 >= (int64_t)0x40000000)
    fail(VT_ERR_RANGE, "triangle records exceed 2^30");
  // splice, then rebase the later bottom levels (child base at word 4, triangle base at word 5)
  e->blas_words.erase(e->blas_words.begin() + (size_t)node0 * 20, e->blas_words.begin() + (size_t)node1 * 20);
  e->blas_words.insert(e->blas_words.begin() + (size_t)node0 * 20, bp.wide.nodes.begin(), bp.wide.nodes.end());
  e->rec_host.erase(e->rec_host.begin() + (size_t)rec0 * 16, e->rec_host.begin() + (size_t)rec1 * 16);
  e->rec_host.insert(e->rec_host.begin() + (size_t)rec0 * 16, bp.wide.tris.begin(), bp.wide.tris.end());
  const size_t later = (size_t)node0 + bp.wide.nodes.size() / 20;
  if (dn != 0 || dr != 0) {
    for (size_t w = later; w < e->blas_words.size() / 20; ++w) {
      e->blas_words[20 * w + 4] = (uint32_t)((int64_t)e->blas_words[20 * w + 4] + dn);
      e->blas_words[20 * w + 5] = (uint32_t)((int64_t)e->blas_words[20 * w + 5] + dr);
    }
    for (size_t k = m + 1; k < nm; ++k) {
      e->blas_root[k] = (uint32_t)((int64_t)e->blas_root[k] + dn);
      e->blas_rec_start[k] = (uint32_t)((int64_t)e->blas_rec_start[k] + dr);
    }
  }
  e->tlas_root = (uint32_t)((int64_t)e->tlas_root + dn);
  e->local_box[m] = bp.local_box;
  e->blas_depths[m] = bp.wide.depth;
  e->blas_depth = *std::max_element(e->blas_depths.begin(), e->blas_depths.end());
  e->ntri += (int64_t)md->triangle_count - (int64_t)e->mesh_tris[m];
  e->mesh_tris[m] = md->triangle_count;
  const size_t tlas_u4 = e->nodes.count - (size_t)old_tlas_root * 5;
  // upload the bottom levels and records; the top level follows in update_instances
  cudaStream_t s = e->stream;
  VT_CUDA(cudaStreamSynchronize(s));
  e->drop_graphs();
  const size_t blas_u4 = e->blas_words.size() / 4;
  e->nodes.resize(blas_u4 + tlas_u4);  // the top level's part is written by update_instances
  VT_CUDA(cudaMemcpyAsync(e->nodes.ptr, e->blas_words.data(), e->blas_words.size() * 4, cudaMemcpyHostToDevice, s));
  e->tris.resize(std::max<size_t>(e->rec_host.size() / 4, 1));
  VT_CUDA(cudaMemcpyAsync(e->tris.ptr, e->rec_host.data(), e->rec_host.size() * 4, cudaMemcpyHostToDevice, s));
  VT_CUDA(cudaStreamSynchronize(s));
  e->view.tris = e->tris.ptr;
  e->view.root = e->tlas_root;
  const std::vector<vt_instance_desc> insts = e->inst_descs;
  update_instances(e, insts.data(), insts.size(), rebuild);
}

// ---------------------------------------------------------------- waves
// Device bytes of wave state per path (ray queues, path state, hits, sort keys,
// shadow queue, radiance, pixel ids) -- about 300.
size_t wave_bytes_per_path(const vt_engine* e) {
  return 2 * (2 * sizeof(*e->rays[0].ptr) + sizeof(*e->through[0].ptr) + sizeof(*e->state[0].ptr)) +
         sizeof(*e->hits.ptr) + sizeof(*e->order.ptr) + sizeof(*e->keys.ptr) + 2 * sizeof(*e->shadow_rays.ptr) +
         sizeof(*e->shadow_contrib.ptr) + sizeof(*e->occluded.ptr) + sizeof(*e->radiance.ptr) +
         sizeof(*e->path_pixel.ptr);
}

// Paths per wave: the option, or kDefaultWavePaths halved (down to 1 M) until
// the wave state fits in half of the device memory that is free (counting the
// engine's own wave buffers as free), so that several engines on one GPU do
// not each claim ~4.7 GB.  Decided once per engine.
uint32_t wave_paths_of(const vt_engine* e) {
  if (e->opts.wave_paths > 0) return (uint32_t)e->opts.wave_paths;
  if (!e->auto_wave_paths) {
    size_t free_b = 0, total_b = 0;
    VT_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t per = wave_bytes_per_path(e);
    const size_t budget = (free_b + (size_t)e->capacity * per) / 2;
    uint32_t w = (uint32_t)vt::pt::kDefaultWavePaths;
    while (w > (1u << 20) && (size_t)w * per > budget) w >>= 1;
    e->auto_wave_paths = w;
  }
  return e->auto_wave_paths;
}

// Buffers of the shadow queues' spatial order, when sort_rays 3 asks for it.
void ensure_shadow_order(vt_engine* e) {
  if (e->sort_rays != 3 || e->shadow_order.count >= e->capacity) return;
  e->drop_graphs();
  e->shadow_keys.resize(e->capacity);
  e->shadow_order.resize(e->capacity);
  e->shadow_order_counts.resize(vt::ray_order_count_words(kShadowOrderCellBits));
}

void ensure_capacity(vt_engine* e, uint32_t cap) {
  if (e->capacity >= cap) {
    ensure_shadow_order(e);
    return;
  }
  e->drop_graphs();
  for (int q = 0; q < 2; ++q) {
    e->rays[q].resize(2 * (size_t)cap);
    e->through[q].resize(cap);
    e->state[q].resize(cap);
  }
  e->hits.resize(cap);
  e->order.resize(cap);
  e->keys.resize(cap);
  e->ray_order_counts.resize(vt::ray_order_count_words(kEngineOrderCellBits));
  e->shadow_rays.resize(2 * (size_t)cap);
  e->shadow_contrib.resize(cap);
  e->occluded.resize(cap);
  e->radiance.resize(cap);
  e->path_pixel.resize(cap);
  e->capacity = cap;
  ensure_shadow_order(e);
}

vt::pt::WaveBuffers wave_buffers(vt_engine* e) {
  vt::pt::WaveBuffers w;
  for (int q = 0; q < 2; ++q) {
    w.rays[q] = e->rays[q].ptr;
    w.state[q] = e->state[q].ptr;
    w.through[q] = e->through[q].ptr;
  }
  w.hits = e->hits.ptr;
  w.order = e->order.ptr;
  w.keys = e->keys.ptr;
  w.shadow_rays = e->shadow_rays.ptr;
  w.shadow_contrib = e->shadow_contrib.ptr;
  w.occluded = e->occluded.ptr;
  w.radiance = e->radiance.ptr;
  w.counters = e->counters.ptr;
  w.trace_counter = e->trace_counter.ptr;
  w.trace_status = e->trace_status.ptr;
  w.path_pixel = e->path_pixel.ptr;
  if (e->nrc) {
    w.nrc_records = e->nrc->records.ptr;
    w.nrc_queries = e->nrc->queries.ptr;
    w.nrc_seed = e->nrc->seed.ptr;
  }
  return w;
}

// Optional per-stage event pairs (profiling; never used while capturing a graph).
struct StageTimer {
  enum Stage { kRaygen, kTraceClosest, kSort, kShade, kTraceShadow, kResolve, kAccumulate, kNrcTrain, kNrcQuery,
               kStages };
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
  int open_stage = -1;
  cudaEvent_t open_ev = nullptr;
  int launches[kStages] = {};
  void begin(int st, cudaStream_t s) {
    cudaEventCreate(&open_ev);
    cudaEventRecord(open_ev, s);
    open_stage = st;
  }
  void end(cudaStream_t s) {
    cudaEvent_t e1;
    cudaEventCreate(&e1);
    cudaEventRecord(e1, s);
    marks.push_back({open_stage, {open_ev, e1}});
    launches[open_stage] += 1;
  }
  void collect(double* ms) {
    for (auto& m : marks) {
      float x = 0.0f;
      cudaEventElapsedTime(&x, m.second.first, m.second.second);
      ms[m.first] += x;
      cudaEventDestroy(m.second.first);
      cudaEventDestroy(m.second.second);
    }
    marks.clear();
  }
};

// (Re)creates the cache over the scene's bounds (training starts over).
void nrc_rebuild(vt_engine* e) {
  NrcEngine& n = *e->nrc;
  vt::nrc::Config c;
  const vt_nrc_config& k = n.opts.cache;
  c.levels = k.levels;
  c.log2_table = k.log2_table_size;
  c.base_resolution = k.base_resolution;
  c.growth = k.growth;
  c.lr = k.learning_rate;
  c.table_lr = k.table_learning_rate;
  c.infer_tiles = k.infer_tiles > 0 ? k.infer_tiles : vt::nrc::kDefaultInferTiles;
  float mn[3] = {0, 0, 0}, mx[3] = {1, 1, 1};
  if (e->has_scene && !e->binary.nodes.empty()) {
    const vt::BinaryNode& r = e->binary.nodes[0];
    for (int i = 0; i < 3; ++i) {
      const float pad = 1e-3f * std::max(1e-3f, r.mx[i] - r.mn[i]);
      if (r.mx[i] >= r.mn[i]) { mn[i] = r.mn[i] - pad; mx[i] = r.mx[i] + pad; }
    }
  }
  for (int i = 0; i < 3; ++i) { c.aabb_min[i] = mn[i]; c.aabb_max[i] = mx[i]; }
  n.cache = std::make_unique<vt::nrc::Cache>(c, k.seed);
  n.cache->set_wait_cycles(e->debug_wait_cycles);
  n.frames = 0;
  e->drop_graphs();
}

void ensure_nrc_buffers(vt_engine* e, uint32_t render_paths) {
  NrcEngine& n = *e->nrc;
  if (n.opts.fallback_error > 0.0f) {
    const uint32_t t = n.opts.fallback_tile > 0 ? (uint32_t)n.opts.fallback_tile : 16u;
    const uint32_t tx = ((uint32_t)e->width + t - 1) / t, ty = ((uint32_t)e->height + t - 1) / t;
    if (tx != n.tiles_x || ty != n.tiles_y || n.tile_width != (uint32_t)e->width) {
      e->drop_graphs();
      n.tiles_x = tx;
      n.tiles_y = ty;
      n.tile_width = (uint32_t)e->width;
      n.tile_stats.resize(3 * (size_t)tx * ty);
      n.tile_error.resize((size_t)tx * ty);
      VT_CUDA(cudaMemset(n.tile_stats.ptr, 0, n.tile_stats.bytes()));
      VT_CUDA(cudaMemset(n.tile_error.ptr, 0, n.tile_error.bytes()));  // no evidence yet: use the cache
    }
    n.cache->set_error_tiles(n.tile_stats.ptr, n.tile_width, t, tx);
  } else {
    n.cache->set_error_tiles(nullptr, 0, 16, 0);
  }
  const size_t rec = (size_t)n.train_paths * (size_t)e->opts.max_bounces * 6;
  const size_t smp = (size_t)n.opts.train_steps * (size_t)n.opts.train_batch * 5;
  const size_t qry = (size_t)std::max(render_paths, e->capacity) * 5;
  if (n.records.count < rec || n.samples.count < smp || n.queries.count < qry || !n.seed.ptr) {
    e->drop_graphs();
    if (n.records.count < rec) n.records.resize(rec);
    if (n.samples.count < smp) n.samples.resize(smp);
    if (n.queries.count < qry) n.queries.resize(qry);
    if (!n.seed.ptr) {
      n.seed.resize(1);
      VT_CUDA(cudaMemset(n.seed.ptr, 0, sizeof(uint32_t)));
    }
  }
}

// Wave modes: plain path tracing, render with cache queries, cache training.
enum WaveMode : int { kPlain = 0, kNrcRender = 1, kNrcTrain = 2 };

// Spatial trace order of one queue (vt::launch_ray_order) over the scene's bounds.
vt::RayOrderArgs spatial_order(const vt_engine* e, const float4* rays, uint32_t cap, const uint32_t* n_dev,
                               uint32_t* keys, uint32_t* counts, uint32_t* order, int cell_bits) {
  vt::RayOrderArgs o;
  o.rays = rays;
  o.n = cap;
  o.n_dev = n_dev;
  const vt::BinaryNode& r = e->binary.nodes[0];
  for (int i = 0; i < 3; ++i) {
    o.lo[i] = r.mn[i];
    o.hi[i] = r.mx[i];
  }
  o.cell_bits = cell_bits;
  o.keys = keys;
  o.counts = counts;
  o.order = order;
  return o;
}

void record_wave(vt_engine* e, uint32_t spp_wave, uint32_t bounces, cudaStream_t s, StageTimer* tm = nullptr,
                 int mode = kPlain) {
  auto B = [&](int st) { if (tm) tm->begin(st, s); };
  auto E = [&]() { if (tm) tm->end(s); };
  vt::pt::FrameView f;
  f.cam = e->aux_consts.ptr + vt::pt::kCamConsts;
  f.width = (uint32_t)e->width;
  f.height = (uint32_t)e->height;
  f.spp_wave = spp_wave;
  f.max_bounces = bounces;
  f.paths = f.width * f.height * spp_wave;
  f.sort_by_material = e->opts.sort_by_material > 0 ? 1u : 0u;
  if (mode == kNrcTrain) {
    f.train = 1;
    f.paths = e->nrc->train_paths;
    f.record_bounces = bounces;
    VT_CUDA(cudaMemsetAsync(e->nrc->records.ptr, 0, e->nrc->records.bytes(), s));
  } else if (mode == kNrcRender) {
    const NrcEngine& n = *e->nrc;
    if (n.opts.prefix_bounces == 0) {
      f.nrc_spread_c = n.opts.spread_c > 0.0f ? n.opts.spread_c : 0.01f;
    } else {
      f.nrc_prefix = (uint32_t)std::min<int>(n.opts.prefix_bounces, (int)bounces - 1);
    }
    if (n.opts.fallback_error > 0.0f && n.tile_error.ptr) {
      f.nrc_tile_error = n.tile_error.ptr;
      f.nrc_fallback = n.opts.fallback_error;
      f.nrc_tile = n.opts.fallback_tile > 0 ? (uint32_t)n.opts.fallback_tile : 16u;
      f.nrc_tiles_x = n.tiles_x;
    }
  }
  if (mode != kNrcTrain && e->aux_nd.ptr)
    f.aux = {e->aux_nd.ptr, e->aux_albedo.ptr, e->aux_motion.ptr, e->aux_moments.ptr, e->aux_consts.ptr};
  VT_CUDA(cudaMemsetAsync(e->counters.ptr + vt::pt::kCntQuery, 0, 2 * sizeof(uint32_t), s));
  const vt::pt::WaveBuffers w = wave_buffers(e);
  vt::pt::AccumView a;
  a.accum = e->accum.ptr;
  a.sum64 = e->sum64.ptr;
  a.sq64 = e->sq64.ptr;
  a.lum64 = e->lum64.ptr;
  const uint32_t cap = f.paths;
  B(StageTimer::kRaygen);
  vt::pt::launch_raygen(f, w, s);
  E();
  int cur = 0;
  // bounce b's shadow rays are traced on the shadow stream while bounce b+1's
  // closest hits are traced here; shade b+1 (which reuses the shadow buffers
  // and counters) waits for them.  Timed stage breakdowns run serially.
  const bool overlap = tm == nullptr;
  for (uint32_t b = 0; b < bounces; ++b) {
    vt::TraceArgs t;
    t.nodes = e->nodes.ptr;
    t.tris = e->tris.ptr;
    t.rays = w.rays[cur];
    t.n = cap;
    t.hits = w.hits;
    t.status = e->trace_status.ptr;
    t.counter = e->trace_counter.ptr;
    t.stack_depth = e->stack_depth;
    t.node_count = e->nodes.count / 5;
    t.stage_nodes = e->trace_stage_nodes;
    t.stage_wait_cycles = e->debug_wait_cycles;
    t.insts = e->view.insts;
    t.inst_table = e->view.inst_table;
    t.root = e->view.root;
    t.n_dev = w.counters + cur;
    t.blocks_per_sm = e->trace_blocks_per_sm;
    if (e->sort_rays == 1 && b > 0) {
      // scattered directions from bounce 1 on: trace the queue octant by octant
      B(StageTimer::kSort);
      vt::pt::launch_sort_rays(w, cur, cap, s);
      E();
      t.order = w.order;
    } else if (e->sort_rays == 2 && b > 0 && !e->binary.nodes.empty()) {
      // ... or grouped by the cell of the scene box the ray starts in and its octant
      B(StageTimer::kSort);
      vt::launch_ray_order(spatial_order(e, w.rays[cur], cap, w.counters + cur, w.keys, e->ray_order_counts.ptr,
                                         w.order, kEngineOrderCellBits),
                           s);
      E();
      t.order = w.order;
    }
    B(StageTimer::kTraceClosest);
    vt::launch_trace_closest_records(t, s);
    E();
    if (b == 0) vt::pt::launch_aux_first_hit(e->view, f, w, s);
    if (f.sort_by_material) {
      B(StageTimer::kSort);
      vt::pt::launch_sort_by_material(e->view, f, w, cur, cap, s);
      E();
    }
    if (overlap && b > 0) VT_CUDA(cudaStreamWaitEvent(s, e->ev_join, 0));
    B(StageTimer::kShade);
    vt::pt::launch_shade(e->view, f, w, cur, b, cap, s);
    E();
    vt::TraceArgs sh = t;
    sh.order = nullptr;
    sh.rays = w.shadow_rays;
    sh.hits = nullptr;
    sh.occluded = w.occluded;
    sh.n_dev = w.counters + vt::pt::kCntShadow;
    cudaStream_t ss = s;
    if (overlap) {
      VT_CUDA(cudaEventRecord(e->ev_fork, s));
      VT_CUDA(cudaStreamWaitEvent(e->shadow_stream, e->ev_fork, 0));
      ss = e->shadow_stream;
      sh.counter = e->shadow_counter.ptr;
    }
    if (e->sort_rays == 3 && !e->binary.nodes.empty() && e->shadow_order.ptr) {
      B(StageTimer::kSort);
      vt::launch_ray_order(spatial_order(e, w.shadow_rays, cap, w.counters + vt::pt::kCntShadow, e->shadow_keys.ptr,
                                         e->shadow_order_counts.ptr, e->shadow_order.ptr, kShadowOrderCellBits),
                           ss);
      E();
      sh.order = e->shadow_order.ptr;
    }
    B(StageTimer::kTraceShadow);
    vt::launch_trace_any(sh, ss);
    E();
    B(StageTimer::kResolve);
    vt::pt::launch_shadow_resolve(w, cap, ss);
    vt::pt::launch_count_rays(w, cur, e->totals.ptr, ss);
    E();
    if (overlap) VT_CUDA(cudaEventRecord(e->ev_join, ss));
    cur ^= 1;
  }
  if (overlap && bounces > 0) VT_CUDA(cudaStreamWaitEvent(s, e->ev_join, 0));
  if (mode == kNrcTrain) {
    B(StageTimer::kNrcTrain);
    const NrcEngine& n = *e->nrc;
    vt::pt::launch_nrc_targets(w, f.paths, bounces, n.samples.ptr,
                               (uint32_t)(n.opts.train_steps * n.opts.train_batch),
                               (uint32_t)std::max(1, n.opts.prefix_bounces), s);
    E();
    return;
  }
  if (mode == kNrcRender) {
    B(StageTimer::kNrcQuery);
    e->nrc->cache->query(w.nrc_queries, 5, w.counters + vt::pt::kCntQuery, cap, nullptr, w.radiance, s);
    E();
  }
  B(StageTimer::kAccumulate);
  vt::pt::launch_accumulate(f, w, a, s);
  E();
}

cudaGraphExec_t wave_graph(vt_engine* e, uint32_t spp_wave, uint32_t bounces, int mode = kPlain) {
  for (auto& g : e->graphs)
    if (g.spp_wave == spp_wave && g.bounces == bounces && g.mode == mode) return g.exec;
  cudaGraph_t graph = nullptr;
  VT_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  record_wave(e, spp_wave, bounces, e->stream, nullptr, mode);
  VT_CUDA(cudaStreamEndCapture(e->stream, &graph));
  cudaGraphExec_t exec = nullptr;
  cudaError_t err = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  VT_CUDA(err);
  e->graphs.push_back({spp_wave, bounces, mode, exec});
  return exec;
}

// Training part of a frame: one training wave (graph), then the optimiser
// steps (direct launches: the bias corrections change every step).
void nrc_train(vt_engine* e, uint32_t bounces, StageTimer* tm) {
  NrcEngine& n = *e->nrc;
  cudaStream_t s = e->stream;
  if (tm) {
    record_wave(e, 1, bounces, s, tm, kNrcTrain);
    tm->begin(StageTimer::kNrcTrain, s);
  } else {
    VT_CUDA(cudaGraphLaunch(wave_graph(e, 1, bounces, kNrcTrain), s));
  }
  const size_t stride = 5 * (size_t)n.opts.train_batch;
  for (int k = 0; k < n.opts.train_steps; ++k)
    n.cache->train_step(n.samples.ptr + stride * k, (uint32_t)n.opts.train_batch, s);
  if (n.opts.fallback_error > 0.0f && n.tile_error.ptr)
    vt::pt::launch_nrc_tile_update(n.tile_stats.ptr, n.tile_error.ptr, n.tiles_x * n.tiles_y, 0.25f, s);
  if (tm) tm->end(s);
}

void reset_accumulation(vt_engine* e) {
  e->samples = 0;
  if (e->accum.ptr) VT_CUDA(cudaMemsetAsync(e->accum.ptr, 0, e->accum.bytes(), e->stream));
  if (e->sum64.ptr) VT_CUDA(cudaMemsetAsync(e->sum64.ptr, 0, e->sum64.bytes(), e->stream));
  if (e->sq64.ptr) VT_CUDA(cudaMemsetAsync(e->sq64.ptr, 0, e->sq64.bytes(), e->stream));
  if (e->lum64.ptr) VT_CUDA(cudaMemsetAsync(e->lum64.ptr, 0, e->lum64.bytes(), e->stream));
  for (DeviceBuffer<float4>* b : {&e->aux_nd, &e->aux_albedo, &e->aux_motion, &e->aux_moments})
    if (b->ptr) VT_CUDA(cudaMemsetAsync(b->ptr, 0, b->bytes(), e->stream));
  VT_CUDA(cudaMemsetAsync(e->counters.ptr, 0, e->counters.bytes(), e->stream));
}

void render_frame(vt_engine* e, const vt_frame_input* in, vt_frame_output* out, double* stage_ms = nullptr,
                  int* stage_launches = nullptr) {
  if (!in || !out) fail(VT_ERR_INVALID_ARGUMENT, "input and output must be non-null");
  if (!e->has_scene) fail(VT_ERR_STATE, "renderFrame before setScene");
  if (in->width <= 0 || in->height <= 0 || in->width > 16384 || in->height > 16384)
    fail(VT_ERR_RANGE, "viewport must be 1..16384 pixels per side");
  if (in->samples < 0) fail(VT_ERR_RANGE, "samples must be >= 0");
  const int maxb = e->opts.max_bounces;
  const uint32_t bounces = (uint32_t)std::min(in->bounces > 0 ? in->bounces : maxb, maxb);
  float ivp[16];
  vt::inverse_view_proj(in->view, in->projection, ivp);
  const bool size_changed = in->width != e->width || in->height != e->height;
  const bool cam_changed = !e->have_camera || std::memcmp(ivp, e->inv_vp, sizeof ivp) != 0 ||
                           in->frame_seed != e->frame_seed;
  if (size_changed) {
    e->width = in->width;
    e->height = in->height;
    const size_t px = (size_t)in->width * in->height;
    e->accum.resize(px);
    for (DeviceBuffer<float4>* b : {&e->aux_nd, &e->aux_albedo, &e->aux_motion, &e->aux_moments}) b->resize(px);
    if (!e->aux_consts.ptr) e->aux_consts.resize(vt::pt::kAuxConsts);
    if (e->opts.oracle_accumulation) {
      e->sum64.resize(3 * px);
      e->sq64.resize(3 * px);
      e->lum64.resize(4 * px);
    }
  }
  if (size_changed || cam_changed) {
    std::memcpy(e->inv_vp, ivp, sizeof ivp);
    std::memcpy(e->view_m, in->view, sizeof e->view_m);
    std::memcpy(e->proj_m, in->projection, sizeof e->proj_m);
    e->frame_seed = in->frame_seed;
    e->have_camera = true;
    // the camera and the seed reach the kernels through the per-frame constants:
    // the captured graphs stay; a new size needs new ones
    if (size_changed) e->drop_graphs();
    reset_accumulation(e);
  }
  const bool prev_camera = e->have_prev_camera;
  e->have_prev_camera = false;  // the pair applies to this frame only
  const int room = e->opts.max_samples_per_pixel - e->samples;
  out->width = e->width;
  out->height = e->height;
  out->radiance_device = e->accum.ptr;
  if (room <= 0 || in->samples == 0) {
    out->kind = room <= 0 ? 1 : 0;
    out->samples_accumulated = e->samples;
    out->is_converged = room <= 0 ? 1 : 0;
    return;
  }
  const uint32_t spp = (uint32_t)std::min(in->samples, room);
  const uint32_t wh = (uint32_t)(e->width * e->height);
  const uint32_t wave_paths = wave_paths_of(e);
  uint32_t spp_wave = std::max<uint32_t>(1u, wave_paths / wh);
  spp_wave = std::min(spp_wave, spp);
  while (spp % spp_wave) --spp_wave;  // equal waves: one graph per frame shape
  ensure_capacity(e, wh * spp_wave);
  // auxiliary-output constants of this frame: view-projections and the last sample
  vt::view_proj(in->view, in->projection, e->aux_host);
  if (prev_camera) vt::view_proj(e->prev_view, e->prev_proj, e->aux_host + 16);
  else std::memcpy(e->aux_host + 16, e->aux_host, 16 * sizeof(float));
  const uint32_t last_sample = (uint32_t)e->samples + spp - 1u;
  std::memcpy(e->aux_host + 32, &last_sample, sizeof last_sample);
  std::memcpy(e->aux_host + vt::pt::kCamConsts, e->inv_vp, sizeof e->inv_vp);
  std::memcpy(e->aux_host + vt::pt::kCamConsts + 16, &e->frame_seed, sizeof e->frame_seed);
  VT_CUDA(cudaMemcpyAsync(e->aux_consts.ptr, e->aux_host, sizeof e->aux_host, cudaMemcpyHostToDevice, e->stream));
  // with the cache: train, then render waves that end in cache queries
  int mode = kPlain;
  uint32_t wave_bounces = bounces;
  if (e->nrc) {
    NrcEngine& n = *e->nrc;
    ensure_capacity(e, n.train_paths);
    ensure_nrc_buffers(e, wh * spp_wave);
    if (n.frames >= n.opts.warmup_frames) {
      mode = kNrcRender;
      // with the fallback, paths of high-error tiles continue past the query vertex
      wave_bounces = (n.opts.fallback_error > 0.0f || n.opts.prefix_bounces == 0)
                         ? bounces
                         : std::min<uint32_t>(bounces, (uint32_t)n.opts.prefix_bounces + 1u);
    }
  }
  if (stage_ms) {
    // profiling: the same launches, issued directly with events between stages
    StageTimer tm;
    VT_CUDA(cudaEventRecord(e->ev0, e->stream));
    if (e->nrc) nrc_train(e, bounces, &tm);
    for (uint32_t done = 0; done < spp; done += spp_wave)
      record_wave(e, spp_wave, wave_bounces, e->stream, &tm, mode);
    VT_CUDA(cudaEventRecord(e->ev1, e->stream));
    VT_CUDA(cudaEventSynchronize(e->ev1));
    VT_CUDA(cudaGetLastError());
    tm.collect(stage_ms);
    for (int k = 0; k < StageTimer::kStages; ++k) stage_launches[k] += tm.launches[k];
  } else {
    if (e->nrc) wave_graph(e, 1, bounces, kNrcTrain);  // capture outside the timed region
    cudaGraphExec_t g = wave_graph(e, spp_wave, wave_bounces, mode);
    VT_CUDA(cudaEventRecord(e->ev0, e->stream));
    if (e->nrc) nrc_train(e, bounces, nullptr);
    for (uint32_t done = 0; done < spp; done += spp_wave) VT_CUDA(cudaGraphLaunch(g, e->stream));
    VT_CUDA(cudaEventRecord(e->ev1, e->stream));
    VT_CUDA(cudaEventSynchronize(e->ev1));
  }
  if (e->nrc) {
    e->nrc->frames += 1;
    int d[2] = {0, 0};
    VT_CUDA(cudaMemcpy(d, e->nrc->cache->d_diag(), sizeof d, cudaMemcpyDeviceToHost));
    if (d[0]) {
      // the frame's cache queries may be missing: drop its samples with the
      // accumulation, so the next frame starts clean
      VT_CUDA(cudaMemset(e->nrc->cache->d_diag(), 0, sizeof(int)));
      reset_accumulation(e);
      fail(VT_ERR_TIMEOUT, "tensor-core wait expired in an NRC kernel");
    }
  }
  float ms = 0.0f;
  VT_CUDA(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
  e->last_ms = ms;
  int st = 0;
  VT_CUDA(cudaMemcpy(&st, e->trace_status.ptr, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) {
    // reported once; the frame's samples leave with the accumulation
    VT_CUDA(cudaMemset(e->trace_status.ptr, 0, sizeof(int)));
    reset_accumulation(e);
    fail(VT_ERR_BUILD, vt::trace_status_message(st));
  }
  e->samples += (int)spp;
  out->kind = 0;
  out->samples_accumulated = e->samples;
  out->is_converged = e->samples >= e->opts.max_samples_per_pixel ? 1 : 0;
}

void camera_ray(const vt_engine* e, float x, float y, float* ray8) {
  const float nx = (x / e->width) * 2.0f - 1.0f, ny = 1.0f - (y / e->height) * 2.0f;
  const float* M = e->inv_vp;
  double nf[4], fr[4];
  for (int r = 0; r < 4; ++r) {
    nf[r] = (double)M[4 * r] * nx + (double)M[4 * r + 1] * ny - M[4 * r + 2] + M[4 * r + 3];
    fr[r] = (double)M[4 * r] * nx + (double)M[4 * r + 1] * ny + M[4 * r + 2] + M[4 * r + 3];
  }
  double o[3], d[3], l = 0;
  for (int k = 0; k < 3; ++k) {
    o[k] = nf[k] / nf[3];
    d[k] = fr[k] / fr[3] - o[k];
    l += d[k] * d[k];
  }
  l = std::sqrt(l);
  for (int k = 0; k < 3; ++k) { ray8[k] = (float)o[k]; ray8[4 + k] = (float)(d[k] / l); }
  ray8[3] = 0.0f;
  ray8[7] = INFINITY;
}

}  // namespace

extern "C" {

vt_status vt_create(int32_t device, const vt_engine_options* options, vt_engine** out_engine) {
  return vt::guard([&] {
    if (!out_engine) fail(VT_ERR_INVALID_ARGUMENT, "out_engine is null");
    *out_engine = nullptr;
    auto e = std::make_unique<vt_engine>();
    e->device = device;
    if (options) e->opts = *options;
    if (e->opts.max_bounces == 0) e->opts.max_bounces = 8;
    if (e->opts.max_bounces < 1 || e->opts.max_bounces > 8) fail(VT_ERR_RANGE, "max_bounces must be in [1, 8]");
    if (e->opts.max_samples_per_pixel == 0) e->opts.max_samples_per_pixel = 4096;
    if (e->opts.max_samples_per_pixel < 1) fail(VT_ERR_RANGE, "max_samples_per_pixel must be >= 1");
    if (e->opts.wave_paths < 0) fail(VT_ERR_RANGE, "wave_paths must be >= 0");
    if (e->opts.bvh_max_leaf == 0) e->opts.bvh_max_leaf = vt::kEngineLeafDefault;
    if (e->opts.bvh_max_leaf < 1 || e->opts.bvh_max_leaf > 4) fail(VT_ERR_RANGE, "bvh_max_leaf must be in [0, 4]");
    if (e->opts.bvh_width == 0) e->opts.bvh_width = 8;
    if (e->opts.bvh_width < 2 || e->opts.bvh_width > 8) fail(VT_ERR_RANGE, "bvh_width must be 0 or in [2, 8]");
    if (e->opts.light_selection < 0 || e->opts.light_selection > 1) fail(VT_ERR_RANGE, "light_selection must be 0 or 1");
    if (e->opts.scene_build < 0 || e->opts.scene_build > 1) fail(VT_ERR_RANGE, "scene_build must be 0 or 1");
    vt::DeviceScope ds(device);
    VT_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    VT_CUDA(cudaEventCreate(&e->ev0));
    VT_CUDA(cudaEventCreate(&e->ev1));
    VT_CUDA(cudaStreamCreateWithFlags(&e->shadow_stream, cudaStreamNonBlocking));
    VT_CUDA(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
    VT_CUDA(cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
    e->shadow_counter.resize(1);
    e->counters.resize(vt::pt::kCntWords);
    VT_CUDA(cudaMemset(e->counters.ptr, 0, e->counters.bytes()));
    e->trace_counter.resize(1);
    e->trace_status.resize(1);
    VT_CUDA(cudaMemset(e->trace_status.ptr, 0, sizeof(int)));
    e->totals.resize(2);
    VT_CUDA(cudaMemset(e->totals.ptr, 0, e->totals.bytes()));
    *out_engine = e.release();
  });
}

vt_status vt_set_scene(vt_engine* e, const vt_scene_desc* scene) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "engine is null");
    vt::DeviceScope ds(e->device);
    set_scene(e, scene);
  });
}

vt_status vt_get_capabilities(const vt_engine* e, vt_capabilities* c) {
  return vt::guard([&] {
    if (!e || !c) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    c->max_bounces_limit = 8;
    c->max_samples_per_pixel = e->opts.max_samples_per_pixel;
    c->max_viewport = 16384;
    c->emitter_kinds = VT_EMITTER_POINT | VT_EMITTER_SPOT | VT_EMITTER_DIRECTIONAL | VT_EMITTER_RECT_AREA |
                       VT_EMITTER_DISC_AREA | VT_EMITTER_MESH_AREA | VT_EMITTER_ENVIRONMENT;
    c->material_features = VT_MATERIAL_FEATURE_BASE | VT_MATERIAL_FEATURE_TRANSMISSION |
                           VT_MATERIAL_FEATURE_SPECULAR | VT_MATERIAL_FEATURE_DOUBLE_SIDED |
                           VT_MATERIAL_FEATURE_CAST_SHADOW;
    c->features = VT_FEATURE_INSTANCES | VT_FEATURE_INSTANCE_UPDATES | VT_FEATURE_RADIANCE_CACHE | VT_FEATURE_BATCH |
                  VT_FEATURE_OUTPUT_CAPTURE | (e->opts.debug ? VT_FEATURE_PICK : 0u) |
                  (e->opts.oracle_accumulation ? VT_FEATURE_FP64_MOMENTS : 0u) | VT_FEATURE_AUX_OUTPUTS |
                  VT_FEATURE_MESH_UPDATES;
  });
}

vt_status vt_update_mesh(vt_engine* e, size_t mesh_index, const vt_mesh_desc* mesh, int32_t rebuild) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "engine is null");
    if (rebuild != 0 && rebuild != 1) fail(VT_ERR_RANGE, "rebuild must be 0 or 1");
    vt::DeviceScope ds(e->device);
    update_mesh(e, mesh_index, mesh, rebuild != 0);
  });
}

vt_status vt_update_instances(vt_engine* e, const vt_instance_desc* instances, size_t count, int32_t rebuild) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "engine is null");
    if (rebuild != 0 && rebuild != 1) fail(VT_ERR_RANGE, "rebuild must be 0 or 1");
    vt::DeviceScope ds(e->device);
    update_instances(e, instances, count, rebuild != 0);
  });
}

vt_status vt_render_frame(vt_engine* e, const vt_frame_input* input, vt_frame_output* output) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "engine is null");
    vt::DeviceScope ds(e->device);
    render_frame(e, input, output);
  });
}

vt_status vt_profile_frame(vt_engine* e, const vt_frame_input* input, vt_frame_output* output,
                           vt_stage_times* times) {
  return vt::guard([&] {
    if (!e || !times) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    vt::DeviceScope ds(e->device);
    double ms[StageTimer::kStages] = {};
    int launches[StageTimer::kStages] = {};
    render_frame(e, input, output, ms, launches);
    times->raygen_ms = ms[StageTimer::kRaygen];
    times->trace_closest_ms = ms[StageTimer::kTraceClosest];
    times->sort_ms = ms[StageTimer::kSort];
    times->shade_ms = ms[StageTimer::kShade];
    times->trace_shadow_ms = ms[StageTimer::kTraceShadow];
    times->resolve_ms = ms[StageTimer::kResolve];
    times->accumulate_ms = ms[StageTimer::kAccumulate];
    times->trace_closest_launches = launches[StageTimer::kTraceClosest];
    times->trace_shadow_launches = launches[StageTimer::kTraceShadow];
    times->nrc_train_ms = ms[StageTimer::kNrcTrain];
    times->nrc_query_ms = ms[StageTimer::kNrcQuery];
    times->frame_ms = e->last_ms;
  });
}

vt_status vt_capture_output(vt_engine* e, const vt_present_options* o, float* rgba, size_t cap) {
  return vt::guard([&] {
    if (!e || !o || !rgba) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (o->tonemap < 0 || o->tonemap > 4) fail(VT_ERR_RANGE, "tonemap must be in [0, 4]");
    if (!(o->exposure > 0.0f) || !std::isfinite(o->exposure)) fail(VT_ERR_RANGE, "exposure must be finite and > 0");
    if (o->srgb != 0 && o->srgb != 1) fail(VT_ERR_RANGE, "srgb must be 0 or 1");
    if (!e->accum.ptr) fail(VT_ERR_STATE, "captureFrame before renderFrame");
    const size_t px = (size_t)e->width * e->height;
    if (cap < 4 * px) fail(VT_ERR_RANGE, "capture buffer too small");
    vt::DeviceScope ds(e->device);
    e->present.resize(px);
    vt::pt::launch_present(e->accum.ptr, px, o->tonemap, o->exposure, o->srgb, e->present.ptr, e->stream);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaMemcpyAsync(rgba, e->present.ptr, px * sizeof(float4), cudaMemcpyDeviceToHost, e->stream));
    VT_CUDA(cudaStreamSynchronize(e->stream));
  });
}

vt_status vt_capture(vt_engine* e, float* rgba, size_t cap) {
  return vt::guard([&] {
    if (!e || !rgba) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (!e->accum.ptr) fail(VT_ERR_STATE, "captureFrame before renderFrame");
    const size_t px = (size_t)e->width * e->height;
    if (cap < 4 * px) fail(VT_ERR_RANGE, "capture buffer too small");
    vt::DeviceScope ds(e->device);
    // the mean on the device (the staging array of the present pass), then one
    // copy into the caller's memory (a direct DMA when it is page-locked)
    e->present.resize(px);
    vt::pt::launch_capture_mean(e->accum.ptr, px, e->present.ptr, e->stream);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaMemcpyAsync(rgba, e->present.ptr, px * sizeof(float4), cudaMemcpyDeviceToHost, e->stream));
    VT_CUDA(cudaStreamSynchronize(e->stream));
  });
}

vt_status vt_capture_moments(vt_engine* e, double* mean_rgb, double* var_rgb, size_t cap) {
  return vt::guard([&] {
    if (!e || !mean_rgb || !var_rgb) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (!e->opts.oracle_accumulation || !e->sum64.ptr) fail(VT_ERR_STATE, "engine has no FP64 accumulation");
    const size_t px = (size_t)e->width * e->height;
    if (cap < 3 * px) fail(VT_ERR_RANGE, "moment buffers too small");
    vt::DeviceScope ds(e->device);
    VT_CUDA(cudaStreamSynchronize(e->stream));
    VT_CUDA(cudaMemcpy(mean_rgb, e->sum64.ptr, 3 * px * sizeof(double), cudaMemcpyDeviceToHost));
    VT_CUDA(cudaMemcpy(var_rgb, e->sq64.ptr, 3 * px * sizeof(double), cudaMemcpyDeviceToHost));
    const double n = (double)e->samples;
    for (size_t i = 0; i < 3 * px; ++i) {
      const double m = n > 0 ? mean_rgb[i] / n : 0.0;
      const double q = n > 0 ? var_rgb[i] / n : 0.0;
      mean_rgb[i] = m;
      var_rgb[i] = n > 1 ? std::max(0.0, (q - m * m) * n / (n - 1)) : 0.0;
    }
  });
}

vt_status vt_capture_luminance_moments(vt_engine* e, double* out, size_t cap) {
  return vt::guard([&] {
    if (!e || !out) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (!e->opts.oracle_accumulation || !e->lum64.ptr) fail(VT_ERR_STATE, "engine has no FP64 accumulation");
    const size_t px = (size_t)e->width * e->height;
    if (cap < 4 * px) fail(VT_ERR_RANGE, "moment buffer too small");
    vt::DeviceScope ds(e->device);
    VT_CUDA(cudaStreamSynchronize(e->stream));
    VT_CUDA(cudaMemcpy(out, e->lum64.ptr, 4 * px * sizeof(double), cudaMemcpyDeviceToHost));
    const double n = (double)e->samples;
    for (size_t i = 0; i < px; ++i) {
      double* o = out + 4 * i;
      if (!(n > 1)) {
        o[0] = n > 0 ? o[0] / n : 0.0;
        o[1] = o[2] = o[3] = 0.0;
        continue;
      }
      // central moments from the raw ones
      const double m = o[0] / n, r2 = o[1] / n, r3 = o[2] / n, r4 = o[3] / n, mm = m * m;
      const double c2 = std::max(0.0, r2 - mm);
      const double c3 = r3 - 3.0 * m * r2 + 2.0 * mm * m;
      const double c4 = r4 - 4.0 * m * r3 + 6.0 * mm * r2 - 3.0 * mm * mm;
      o[0] = m;
      o[1] = c2 * n / (n - 1);
      o[2] = c2 > 0 ? c3 / (c2 * std::sqrt(c2)) : 0.0;
      o[3] = c2 > 0 ? std::max(-2.0, c4 / (c2 * c2) - 3.0) : 0.0;
    }
  });
}

vt_status vt_capture_aux(vt_engine* e, int32_t kind, float* rgba, size_t cap) {
  return vt::guard([&] {
    if (!e || !rgba) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (kind < VT_AUX_NORMAL_DEPTH || kind > VT_AUX_VARIANCE) fail(VT_ERR_RANGE, "unknown auxiliary output");
    if (!e->aux_nd.ptr) fail(VT_ERR_STATE, "captureFrame before renderFrame");
    const size_t px = (size_t)e->width * e->height;
    if (cap < 4 * px) fail(VT_ERR_RANGE, "capture buffer too small");
    vt::DeviceScope ds(e->device);
    VT_CUDA(cudaStreamSynchronize(e->stream));
    const DeviceBuffer<float4>& src = kind == VT_AUX_NORMAL_DEPTH ? e->aux_nd
                                      : kind == VT_AUX_ALBEDO     ? e->aux_albedo
                                      : kind == VT_AUX_MOTION     ? e->aux_motion
                                                                  : e->aux_moments;
    VT_CUDA(cudaMemcpy(rgba, src.ptr, px * sizeof(float4), cudaMemcpyDeviceToHost));
    if (kind == VT_AUX_VARIANCE) {
      // kernel.wgsl.ts:942-945: count = max(n, 1), varL = max(0, E[L^2] - E[L]^2)
      for (size_t i = 0; i < px; ++i) {
        float* m = rgba + 4 * i;
        const float n = std::max(m[2], 1.0f);
        const float mean = m[0] / n;
        m[0] = std::max(0.0f, m[1] / n - mean * mean);
        m[1] = m[2] = m[3] = 0.0f;
      }
    }
  });
}

vt_status vt_set_previous_camera(vt_engine* e, const float* prev_view, const float* prev_projection) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "null engine");
    if (!prev_view != !prev_projection) fail(VT_ERR_INVALID_ARGUMENT, "give both previous matrices or neither");
    if (!prev_view) {
      e->have_prev_camera = false;
      return;
    }
    for (int i = 0; i < 16; ++i)
      if (!std::isfinite(prev_view[i]) || !std::isfinite(prev_projection[i]))
        fail(VT_ERR_RANGE, "previous camera matrices must be finite");
    std::memcpy(e->prev_view, prev_view, sizeof e->prev_view);
    std::memcpy(e->prev_proj, prev_projection, sizeof e->prev_proj);
    e->have_prev_camera = true;
  });
}

vt_status vt_pick(vt_engine* e, float x, float y, int32_t* out_triangle) {
  return vt::guard([&] {
    if (!e || !out_triangle) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (!e->opts.debug) fail(VT_ERR_STATE, "pickPrimitive requires the debug option");
    if (!e->has_scene || !e->have_camera) fail(VT_ERR_STATE, "pickPrimitive before setScene/renderFrame");
    vt::DeviceScope ds(e->device);
    float ray[8];
    camera_ray(e, x, y, ray);
    e->pick_ray.resize(2);
    e->pick_hit.resize(1);
    e->pick_status.resize(1);
    e->pick_counter.resize(1);
    VT_CUDA(cudaMemcpyAsync(e->pick_ray.ptr, ray, sizeof ray, cudaMemcpyHostToDevice, e->stream));
    VT_CUDA(cudaMemsetAsync(e->pick_status.ptr, 0, sizeof(int), e->stream));
    vt::TraceArgs t;
    t.nodes = e->nodes.ptr;
    t.tris = e->tris.ptr;
    t.rays = e->pick_ray.ptr;
    t.n = 1;
    t.hits = e->pick_hit.ptr;
    t.status = e->pick_status.ptr;
    t.counter = e->pick_counter.ptr;
    t.stack_depth = e->stack_depth;
    t.node_count = e->nodes.count / 5;
    t.stage_nodes = e->trace_stage_nodes;
    t.stage_wait_cycles = e->debug_wait_cycles;
    t.insts = e->view.insts;
    t.root = e->view.root;
    t.inst_table = e->view.inst_table;
    vt::launch_trace_closest_records(t, e->stream);
    VT_CUDA(cudaGetLastError());
    int4 h;
    VT_CUDA(cudaMemcpyAsync(&h, e->pick_hit.ptr, sizeof h, cudaMemcpyDeviceToHost, e->stream));
    VT_CUDA(cudaStreamSynchronize(e->stream));
    if (h.x < 0) {
      *out_triangle = -1;
    } else if (h.z >= 0) {
      *out_triangle = h.z;
    } else {
      float4 v0;
      VT_CUDA(cudaMemcpy(&v0, e->tris.ptr + 4 * (size_t)h.x, sizeof v0, cudaMemcpyDeviceToHost));
      uint32_t id;
      std::memcpy(&id, &v0.w, 4);
      *out_triangle = (int32_t)id;
    }
  });
}

vt_status vt_engine_export_scene(const vt_engine* e, uint32_t* node_words, size_t word_capacity, float* records,
                                 size_t float_capacity, size_t* out_words, size_t* out_floats) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "engine is null");
    if (!e->has_scene) fail(VT_ERR_STATE, "export before setScene");
    vt::DeviceScope ds(e->device);
    const size_t nw = e->nodes.count * 4, nf = e->tris.count * 4;
    if (out_words) *out_words = nw;
    if (out_floats) *out_floats = nf;
    VT_CUDA(cudaStreamSynchronize(e->stream));
    if (node_words) {
      if (word_capacity < nw) fail(VT_ERR_RANGE, "node buffer too small");
      VT_CUDA(cudaMemcpy(node_words, e->nodes.ptr, nw * 4, cudaMemcpyDeviceToHost));
    }
    if (records) {
      if (float_capacity < nf) fail(VT_ERR_RANGE, "record buffer too small");
      VT_CUDA(cudaMemcpy(records, e->tris.ptr, nf * 4, cudaMemcpyDeviceToHost));
    }
  });
}

vt_status vt_engine_export_tlas(const vt_engine* e, uint32_t* nodes, size_t node_word_capacity,
                                uint32_t* instance_indices, size_t instance_capacity, size_t* node_count) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "engine is null");
    if (!e->has_scene || e->n_instances == 0) fail(VT_ERR_STATE, "the scene has no top level (no instances)");
    const vt::BinaryBvhHost& t = e->binary;
    if (node_count) *node_count = t.nodes.size();
    if (nodes) {
      if (node_word_capacity < t.nodes.size() * 8) fail(VT_ERR_RANGE, "node buffer too small");
      std::memcpy(nodes, t.nodes.data(), t.nodes.size() * 32);
    }
    if (instance_indices) {
      if (instance_capacity < t.reordered_to_source.size()) fail(VT_ERR_RANGE, "instance buffer too small");
      std::memcpy(instance_indices, t.reordered_to_source.data(), t.reordered_to_source.size() * 4);
    }
  });
}

vt_status vt_trace_rays(vt_engine* e, const vt_ray* rays, size_t n, vt_hit* hits, int32_t* instances) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "engine is null");
    if (n && (!rays || !hits)) fail(VT_ERR_INVALID_ARGUMENT, "rays and hits must be non-null");
    if (n > 0xFFFFFFFFull) fail(VT_ERR_RANGE, "at most 2^32 - 1 rays per call");
    if (!e->has_scene) fail(VT_ERR_STATE, "trace before setScene");
    if (!n) return;
    vt::DeviceScope ds(e->device);
    e->q_rays.resize(2 * n);
    e->q_hits.resize(n);
    e->q_inst.resize(n);
    e->q_status.resize(1);
    e->q_counter.resize(1);
    VT_CUDA(cudaMemcpyAsync(e->q_rays.ptr, rays, n * sizeof(vt_ray), cudaMemcpyHostToDevice, e->stream));
    VT_CUDA(cudaMemsetAsync(e->q_status.ptr, 0, sizeof(int), e->stream));
    vt::TraceArgs t;
    t.nodes = e->nodes.ptr;
    t.tris = e->tris.ptr;
    t.rays = e->q_rays.ptr;
    t.n = n;
    t.hits = e->q_hits.ptr;
    t.status = e->q_status.ptr;
    t.counter = e->q_counter.ptr;
    t.stack_depth = e->stack_depth;
    t.node_count = e->nodes.count / 5;
    t.stage_nodes = e->trace_stage_nodes;
    t.stage_wait_cycles = e->debug_wait_cycles;
    t.insts = e->view.insts;
    t.root = e->view.root;
    t.inst_table = e->view.inst_table;
    t.inst_l2w = e->view.inst_table ? e->inst_l2w.ptr : nullptr;
    t.inst_out = e->q_inst.ptr;
    vt::launch_trace_closest(t, e->stream);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaMemcpyAsync(hits, e->q_hits.ptr, n * sizeof(vt_hit), cudaMemcpyDeviceToHost, e->stream));
    if (instances)
      VT_CUDA(cudaMemcpyAsync(instances, e->q_inst.ptr, n * sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream));
    int st = 0;
    VT_CUDA(cudaMemcpyAsync(&st, e->q_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    VT_CUDA(cudaStreamSynchronize(e->stream));
    if (st) {
      VT_CUDA(cudaMemset(e->q_status.ptr, 0, sizeof(int)));
      fail(VT_ERR_BUILD, vt::trace_status_message(st));
    }
  });
}

vt_status vt_set_nrc(vt_engine* e, const vt_nrc_render_options* o) {
  return vt::guard([&] {
    if (!e || !o) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    vt::DeviceScope ds(e->device);
    VT_CUDA(cudaStreamSynchronize(e->stream));
    e->drop_graphs();
    if (!o->enabled) {
      e->nrc.reset();
      return;
    }
    if (o->prefix_bounces < 0 || o->prefix_bounces >= e->opts.max_bounces)
      fail(VT_ERR_RANGE, "prefix_bounces must be in [0, max_bounces - 1]");
    if (!(o->spread_c >= 0.0f)) fail(VT_ERR_RANGE, "spread_c must be >= 0");
    if (o->train_steps < 0 || o->train_steps > 64) fail(VT_ERR_RANGE, "train_steps must be in [0, 64]");
    if (o->train_batch < 128 || o->train_batch > (1 << 20) || o->train_batch % 128)
      fail(VT_ERR_RANGE, "train_batch must be a multiple of 128 in [128, 2^20]");
    if (o->train_paths < 0 || o->warmup_frames < 0) fail(VT_ERR_RANGE, "train_paths and warmup_frames must be >= 0");
    if (!(o->fallback_error >= 0.0f) || o->fallback_tile < 0 || o->fallback_tile > 4096)
      fail(VT_ERR_RANGE, "fallback_error must be >= 0 and fallback_tile in [0, 4096]");
    auto n = std::make_unique<NrcEngine>();
    n->opts = *o;
    n->train_paths = o->train_paths > 0 ? (uint32_t)o->train_paths
                                        : (uint32_t)std::max(1024, o->train_steps * o->train_batch / 2);
    e->nrc = std::move(n);
    try {
      nrc_rebuild(e);
    } catch (...) {
      e->nrc.reset();
      throw;
    }
  });
}

// The radiance cache's query tiles per inference CTA (0 without a cache), and
// a new value for it kept across cache rebuilds (0 leaves it).
static int nrc_tiles_of(const vt_engine* e) { return e->nrc && e->nrc->cache ? e->nrc->cache->config().infer_tiles : 0; }
static void set_nrc_tiles(vt_engine* e, int tiles) {
  if (!e->nrc || tiles <= 0) return;
  e->nrc->opts.cache.infer_tiles = tiles;
  if (e->nrc->cache) e->nrc->cache->set_infer_tiles(tiles);
}

vt_status vt_engine_autotune(vt_engine* e, const vt_frame_input* frame, vt_tuning_trial* report, size_t cap,
                             size_t* count) {
  return vt::guard([&] {
    if (!e || !frame) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (!e->has_scene) fail(VT_ERR_STATE, "autotune before setScene");
    if (frame->samples < 1) fail(VT_ERR_RANGE, "autotune needs a frame with samples >= 1");
    vt::DeviceScope ds(e->device);
    std::vector<vt_tuning_trial> trials;
    auto apply = [&](const vt_tuning& t) {
      e->opts.wave_paths = t.wave_paths;
      e->opts.sort_by_material = t.sort_by_material ? 1 : 0;
      e->trace_blocks_per_sm = t.trace_blocks_per_sm;
      e->trace_stage_nodes = t.stage_hot_nodes != 0;
      e->sort_rays = t.sort_rays;
      set_nrc_tiles(e, t.nrc_infer_tiles);
      e->drop_graphs();
    };
    auto time_it = [&](const vt_tuning& t) {
      apply(t);
      vt_frame_output out{};
      double best = 1e30;
      for (int rep = 0; rep < 3; ++rep) {  // first render captures the graph
        reset_accumulation(e);
        render_frame(e, frame, &out);
        if (rep) best = std::min(best, e->last_ms);
      }
      trials.push_back({t, best});
      return best;
    };
    vt_tuning best{(int32_t)wave_paths_of(e), e->opts.sort_by_material > 0 ? 1 : 0,
                   e->trace_blocks_per_sm, e->trace_stage_nodes ? 1 : 0, e->sort_rays, nrc_tiles_of(e)};
    double best_ms = time_it(best);
    // wave sizes up to the frame's paths (rounded up to a power of two) whose
    // wave state fits in half of the free device memory (the engine's own wave
    // buffers counted as free)
    size_t free_b = 0, total_b = 0;
    VT_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = (free_b + (size_t)e->capacity * wave_bytes_per_path(e)) / 2;
    const size_t frame_paths = (size_t)frame->width * frame->height * (size_t)frame->samples;
    for (int wp : {1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25, 1 << 26}) {
      if (wp == best.wave_paths) continue;
      if (wp > (1 << 24) && ((size_t)wp / 2 >= frame_paths || (size_t)wp * wave_bytes_per_path(e) > budget)) continue;
      vt_tuning t = best;
      t.wave_paths = wp;
      const double ms = time_it(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    {
      vt_tuning t = best;
      t.sort_by_material = best.sort_by_material ? 0 : 1;
      const double ms = time_it(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    for (int bp : {4, 6}) {
      if (bp == best.trace_blocks_per_sm) continue;
      vt_tuning t = best;
      t.trace_blocks_per_sm = bp;
      const double ms = time_it(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    {
      vt_tuning t = best;
      t.stage_hot_nodes = best.stage_hot_nodes ? 0 : 1;
      const double ms = time_it(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    const int sort_start = best.sort_rays;
    for (int sr : {0, 1, 2, 3}) {
      if (sr == sort_start) continue;
      vt_tuning t = best;
      t.sort_rays = sr;
      const double ms = time_it(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    if (e->nrc) {
      // the radiance cache's MLP tile: query tiles in flight per inference CTA
      const int tiles_start = best.nrc_infer_tiles;
      for (int nt : {1, 2, 3, 4}) {
        if (nt == tiles_start) continue;
        vt_tuning t = best;
        t.nrc_infer_tiles = nt;
        const double ms = time_it(t);
        if (ms < best_ms) { best_ms = ms; best = t; }
      }
    }
    apply(best);
    reset_accumulation(e);
    if (count) *count = trials.size();
    if (report)
      for (size_t i = 0; i < trials.size() && i < cap; ++i) report[i] = trials[i];
  });
}

vt_status vt_engine_autotune_bvh(vt_engine* e, const vt_scene_desc* sc, const vt_frame_input* frame,
                                 vt_bvh_shape_trial* report, size_t cap, size_t* count) {
  return vt::guard([&] {
    if (!e || !sc || !frame) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (frame->samples < 1) fail(VT_ERR_RANGE, "autotune needs a frame with samples >= 1");
    vt::DeviceScope ds(e->device);
    std::vector<vt_bvh_shape_trial> trials;
    const int width0 = e->opts.bvh_width, leaf0 = e->opts.bvh_max_leaf;
    int built_w = 0, built_l = 0;
    auto time_it = [&](int width, int leaf) {
      e->opts.bvh_width = width;
      e->opts.bvh_max_leaf = leaf;
      set_scene(e, sc);
      built_w = width;
      built_l = leaf;
      vt_frame_output out{};
      double best = 1e30;
      for (int rep = 0; rep < 3; ++rep) {  // first render captures the graph
        reset_accumulation(e);
        render_frame(e, frame, &out);
        if (rep) best = std::min(best, e->last_ms);
      }
      trials.push_back({width, leaf, best});
      return best;
    };
    // a candidate replaces the current shape only when it is 0.5 % faster: frame
    // times of equal shapes differ by ~0.1 % between runs
    constexpr double kMargin = 0.995;
    int bw = width0, bl = leaf0;
    double best_ms = time_it(bw, bl);
    for (int leaf = 1; leaf <= 4; ++leaf) {
      if (leaf == leaf0) continue;
      const double ms = time_it(width0, leaf);
      if (ms < best_ms * kMargin) { best_ms = ms; bl = leaf; }
    }
    for (int width : {8, 6, 4}) {
      if (width == width0) continue;
      const double ms = time_it(width, bl);
      if (ms < best_ms * kMargin) { best_ms = ms; bw = width; }
    }
    e->opts.bvh_width = bw;
    e->opts.bvh_max_leaf = bl;
    if (built_w != bw || built_l != bl) set_scene(e, sc);
    reset_accumulation(e);
    if (count) *count = trials.size();
    if (report)
      for (size_t i = 0; i < trials.size() && i < cap; ++i) report[i] = trials[i];
  });
}

vt_status vt_engine_get_tuning(const vt_engine* e, vt_tuning* t) {
  return vt::guard([&] {
    if (!e || !t) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    vt::DeviceScope ds(e->device);
    t->wave_paths = (int32_t)wave_paths_of(e);
    t->sort_by_material = e->opts.sort_by_material > 0 ? 1 : 0;
    t->trace_blocks_per_sm = e->trace_blocks_per_sm;
    t->stage_hot_nodes = e->trace_stage_nodes ? 1 : 0;
    t->sort_rays = e->sort_rays;
    t->nrc_infer_tiles = nrc_tiles_of(e);
  });
}

vt_status vt_engine_set_tuning(vt_engine* e, const vt_tuning* t) {
  return vt::guard([&] {
    if (!e || !t) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (t->wave_paths < 1024 || t->wave_paths > (1 << 26)) fail(VT_ERR_RANGE, "wave_paths must be in [1024, 2^26]");
    if (t->sort_by_material != 0 && t->sort_by_material != 1) fail(VT_ERR_RANGE, "sort_by_material must be 0 or 1");
    if (t->trace_blocks_per_sm < 0 || t->trace_blocks_per_sm > 16)
      fail(VT_ERR_RANGE, "trace_blocks_per_sm must be in [0, 16]");
    if (t->stage_hot_nodes != 0 && t->stage_hot_nodes != 1) fail(VT_ERR_RANGE, "stage_hot_nodes must be 0 or 1");
    if (t->sort_rays < 0 || t->sort_rays > 3) fail(VT_ERR_RANGE, "sort_rays must be in [0, 3]");
    if (t->nrc_infer_tiles < 0 || t->nrc_infer_tiles > 4) fail(VT_ERR_RANGE, "nrc_infer_tiles must be in [0, 4]");
    vt::DeviceScope ds(e->device);
    VT_CUDA(cudaStreamSynchronize(e->stream));
    e->opts.wave_paths = t->wave_paths;
    e->opts.sort_by_material = t->sort_by_material;
    e->trace_blocks_per_sm = t->trace_blocks_per_sm;
    e->trace_stage_nodes = t->stage_hot_nodes != 0;
    e->sort_rays = t->sort_rays;
    set_nrc_tiles(e, t->nrc_infer_tiles);
    e->drop_graphs();
  });
}

vt_status vt_engine_set_wait_limit(vt_engine* e, int64_t cycles) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "engine is null");
    if (!e->opts.debug) fail(VT_ERR_STATE, "the wait-limit hook requires the debug option");
    if (cycles < 0) fail(VT_ERR_RANGE, "cycles must be >= 0");
    vt::DeviceScope ds(e->device);
    VT_CUDA(cudaStreamSynchronize(e->stream));
    e->debug_wait_cycles = cycles;
    if (e->nrc) e->nrc->cache->set_wait_cycles(cycles);
    e->drop_graphs();  // captured launches hold the old limits
  });
}

vt_status vt_reset(vt_engine* e) {
  return vt::guard([&] {
    if (!e) fail(VT_ERR_INVALID_ARGUMENT, "engine is null");
    vt::DeviceScope ds(e->device);
    reset_accumulation(e);
    VT_CUDA(cudaStreamSynchronize(e->stream));
  });
}

vt_status vt_engine_get_stats(const vt_engine* e, vt_engine_stats* out) {
  return vt::guard([&] {
    if (!e || !out) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    vt::DeviceScope ds(e->device);
    unsigned long long t[2] = {0, 0};
    VT_CUDA(cudaStreamSynchronize(e->stream));
    VT_CUDA(cudaMemcpy(t, e->totals.ptr, sizeof t, cudaMemcpyDeviceToHost));
    out->closest_rays = t[0];
    out->shadow_rays = t[1];
    out->last_frame_ms = e->last_ms;
    out->triangle_count = e->ntri;
    out->emitter_count = e->n_emitters;
  });
}

vt_status vt_destroy(vt_engine* e) {
  return vt::guard([&] {
    if (!e) return;
    vt::DeviceScope ds(e->device);
    cudaStreamSynchronize(e->stream);
    delete e;
  });
}

}  // extern "C"
