// api_batch.cu -- many scenes rendered together (vt_batch_*): one device arena
// of concatenated BVHs and scene data, one path index space over all scenes'
// frames, waves drawn from it by a device cursor, every wave's stages captured
// into one CUDA graph per frame, and the autotuner over launch shapes.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/vitrum_pt.h"
#include "pt_kernels.h"
#include "scene_pack.h"
#include "traverse.h"
#include "vt_common.h"

using vt::DeviceBuffer;
using vt::fail;

struct vt_batch {
  int device = 0;
  vt_engine_options opts{};
  vt_tuning tuning{vt::pt::kDefaultWavePaths, 0, 0, 0, 0};
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // shadow stream: bounce b's shadow trace and resolve beside bounce b+1's closest-hit trace
  cudaStream_t shadow_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // scenes
  size_t count = 0;
  DeviceBuffer<uint4> nodes;
  DeviceBuffer<float4> tris;
  DeviceBuffer<vt::pt::Material> mats;
  DeviceBuffer<float4> emitters, points, dirs, env, areas;
  DeviceBuffer<float> cdf, marg, cond, ltree;
  DeviceBuffer<vt::pt::BatchScene> scenes;
  std::vector<vt::pt::BatchScene> host;
  unsigned long long total_paths = 0;
  uint32_t max_bounces = 1;
  int stack_depth = 4;
  size_t pixels = 0;
  DeviceBuffer<float4> accum;
  // waves
  uint32_t capacity = 0;
  DeviceBuffer<float4> rays[2], through[2];
  DeviceBuffer<uint4> state[2];
  DeviceBuffer<int4> hits;
  DeviceBuffer<uint32_t> order, keys, counters, ray_root[2], shadow_root, path_pixel;
  DeviceBuffer<float4> shadow_rays, shadow_contrib, radiance;
  DeviceBuffer<uint8_t> occluded;
  DeviceBuffer<unsigned long long> trace_counter, shadow_counter, totals, cursor;
  DeviceBuffer<int> trace_status;
  cudaGraphExec_t graph = nullptr;
  int graph_launches = 0;
  uint32_t waves = 0;

  void drop_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
  }
  ~vt_batch() {
    drop_graph();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (shadow_stream) cudaStreamDestroy(shadow_stream);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

template <class T>
void upload(DeviceBuffer<T>& dst, const std::vector<T>& src, cudaStream_t s) {
  dst.resize(std::max<size_t>(src.size(), 1));
  if (!src.empty()) VT_CUDA(cudaMemcpyAsync(dst.ptr, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

// Device bytes of wave state per path in flight.
size_t batch_bytes_per_path(const vt_batch* b) {
  return 2 * (2 * sizeof(*b->rays[0].ptr) + sizeof(*b->through[0].ptr) + sizeof(*b->state[0].ptr) +
              sizeof(*b->ray_root[0].ptr)) +
         sizeof(*b->hits.ptr) + sizeof(*b->order.ptr) + sizeof(*b->keys.ptr) + 2 * sizeof(*b->shadow_rays.ptr) +
         sizeof(*b->shadow_contrib.ptr) + sizeof(*b->shadow_root.ptr) + sizeof(*b->occluded.ptr) +
         sizeof(*b->radiance.ptr) + sizeof(*b->path_pixel.ptr);
}

void ensure_capacity(vt_batch* b, uint32_t cap) {
  if (b->capacity >= cap) return;
  b->drop_graph();
  for (int q = 0; q < 2; ++q) {
    b->rays[q].resize(2 * (size_t)cap);
    b->through[q].resize(cap);
    b->state[q].resize(cap);
    b->ray_root[q].resize(cap);
  }
  b->hits.resize(cap);
  b->order.resize(cap);
  b->keys.resize(cap);
  b->shadow_rays.resize(2 * (size_t)cap);
  b->shadow_contrib.resize(cap);
  b->shadow_root.resize(cap);
  b->occluded.resize(cap);
  b->radiance.resize(cap);
  b->path_pixel.resize(cap);
  b->capacity = cap;
}

vt::pt::WaveBuffers wave_buffers(vt_batch* b) {
  vt::pt::WaveBuffers w;
  for (int q = 0; q < 2; ++q) {
    w.rays[q] = b->rays[q].ptr;
    w.state[q] = b->state[q].ptr;
    w.through[q] = b->through[q].ptr;
    w.ray_root[q] = b->ray_root[q].ptr;
  }
  w.hits = b->hits.ptr;
  w.order = b->order.ptr;
  w.keys = b->keys.ptr;
  w.shadow_rays = b->shadow_rays.ptr;
  w.shadow_contrib = b->shadow_contrib.ptr;
  w.shadow_root = b->shadow_root.ptr;
  w.occluded = b->occluded.ptr;
  w.radiance = b->radiance.ptr;
  w.counters = b->counters.ptr;
  w.trace_counter = b->trace_counter.ptr;
  w.trace_status = b->trace_status.ptr;
  w.path_pixel = b->path_pixel.ptr;
  w.batch_cursor = b->cursor.ptr;
  return w;
}

// One wave: raygen from the cursor, max_bounces bounces (each scene's paths
// stop at their own bounce count), accumulation, cursor advance.  Returns the
// number of kernels it enqueues.
int record_wave(vt_batch* b, cudaStream_t s) {
  vt::pt::FrameView f;
  f.batch = b->scenes.ptr;
  f.n_scenes = (uint32_t)b->count;
  f.batch_paths = b->total_paths;
  f.max_bounces = b->max_bounces;
  f.sort_by_material = b->tuning.sort_by_material ? 1u : 0u;
  const vt::pt::WaveBuffers w = wave_buffers(b);
  const uint32_t cap = b->capacity;
  const vt::pt::SceneView unused;
  int k = 0;
  vt::pt::launch_raygen_batch(f, w, cap, s);
  k += 1;
  int cur = 0;
  for (uint32_t bo = 0; bo < b->max_bounces; ++bo) {
    vt::TraceArgs t;
    t.nodes = b->nodes.ptr;
    t.tris = b->tris.ptr;
    t.rays = w.rays[cur];
    t.n = cap;
    t.hits = w.hits;
    t.status = b->trace_status.ptr;
    t.counter = b->trace_counter.ptr;
    t.stack_depth = b->stack_depth;
    t.roots = w.ray_root[cur];
    t.n_dev = w.counters + cur;
    t.blocks_per_sm = b->tuning.trace_blocks_per_sm;
    if (b->tuning.sort_rays && bo > 0) {
      vt::pt::launch_sort_rays(w, cur, cap, s);
      t.order = w.order;
      k += 2;
    }
    vt::launch_trace_closest_records(t, s);
    k += 1;
    if (f.sort_by_material) {
      vt::pt::launch_sort_by_material(unused, f, w, cur, cap, s);
      k += 2;
    }
    // the previous bounce's shadow work (second stream) before this shade reuses its buffers
    if (bo > 0) VT_CUDA(cudaStreamWaitEvent(s, b->ev_join, 0));
    vt::pt::launch_shade(unused, f, w, cur, bo, cap, s);
    vt::TraceArgs sh = t;
    sh.order = nullptr;
    sh.rays = w.shadow_rays;
    sh.hits = nullptr;
    sh.occluded = w.occluded;
    sh.roots = w.shadow_root;
    sh.n_dev = w.counters + vt::pt::kCntShadow;
    sh.counter = b->shadow_counter.ptr;
    VT_CUDA(cudaEventRecord(b->ev_fork, s));
    VT_CUDA(cudaStreamWaitEvent(b->shadow_stream, b->ev_fork, 0));
    vt::launch_trace_any(sh, b->shadow_stream);
    vt::pt::launch_shadow_resolve(w, cap, b->shadow_stream);
    vt::pt::launch_count_rays(w, cur, b->totals.ptr, b->shadow_stream);
    VT_CUDA(cudaEventRecord(b->ev_join, b->shadow_stream));
    k += 4;
    cur ^= 1;
  }
  if (b->max_bounces > 0) VT_CUDA(cudaStreamWaitEvent(s, b->ev_join, 0));
  vt::pt::launch_accumulate_batch(w, b->accum.ptr, cap, s);
  return k + 2;
}

void build_graph(vt_batch* b) {
  b->drop_graph();
  b->waves = (uint32_t)((b->total_paths + b->capacity - 1) / b->capacity);
  cudaGraph_t g = nullptr;
  VT_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int k = 0;
  for (uint32_t i = 0; i < b->waves; ++i) k += record_wave(b, b->stream);
  VT_CUDA(cudaStreamEndCapture(b->stream, &g));
  cudaError_t err = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  VT_CUDA(err);
  b->graph_launches = k;
}

void render(vt_batch* b, vt_batch_stats* st) {
  if (!b->count) fail(VT_ERR_STATE, "render before set_scenes");
  const uint32_t want = (uint32_t)std::min<unsigned long long>((unsigned long long)b->tuning.wave_paths,
                                                              std::max<unsigned long long>(b->total_paths, 1ull));
  ensure_capacity(b, want);
  if (b->capacity != want) {  // a smaller wave than the buffers hold
    b->drop_graph();
    b->capacity = want;
  }
  if (!b->graph) build_graph(b);
  cudaStream_t s = b->stream;
  unsigned long long t0[2] = {0, 0}, t1[2] = {0, 0};
  VT_CUDA(cudaMemcpyAsync(t0, b->totals.ptr, sizeof t0, cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaMemsetAsync(b->accum.ptr, 0, b->accum.bytes(), s));
  VT_CUDA(cudaMemsetAsync(b->cursor.ptr, 0, sizeof(unsigned long long), s));
  VT_CUDA(cudaMemsetAsync(b->counters.ptr, 0, b->counters.bytes(), s));
  VT_CUDA(cudaEventRecord(b->ev0, s));
  VT_CUDA(cudaGraphLaunch(b->graph, s));
  VT_CUDA(cudaEventRecord(b->ev1, s));
  VT_CUDA(cudaMemcpyAsync(t1, b->totals.ptr, sizeof t1, cudaMemcpyDeviceToHost, s));
  VT_CUDA(cudaStreamSynchronize(s));
  int status = 0;
  VT_CUDA(cudaMemcpy(&status, b->trace_status.ptr, sizeof status, cudaMemcpyDeviceToHost));
  if (status) fail(VT_ERR_BUILD, vt::trace_status_message(status));
  float ms = 0.0f;
  VT_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  if (st) {
    st->frame_ms = ms;
    st->closest_rays = t1[0] - t0[0];
    st->shadow_rays = t1[1] - t0[1];
    st->waves = (int32_t)b->waves;
    st->kernel_launches = b->graph_launches;
  }
}

void validate_tuning(const vt_tuning& t) {
  if (t.wave_paths < 1024 || t.wave_paths > (1 << 26)) fail(VT_ERR_RANGE, "wave_paths must be in [1024, 2^26]");
  if (t.sort_by_material != 0 && t.sort_by_material != 1) fail(VT_ERR_RANGE, "sort_by_material must be 0 or 1");
  if (t.trace_blocks_per_sm < 0 || t.trace_blocks_per_sm > 16) fail(VT_ERR_RANGE, "trace_blocks_per_sm in [0, 16]");
  if (t.stage_hot_nodes != 0)
    fail(VT_ERR_RANGE, "stage_hot_nodes must be 0 for a batch (its launches carry one root node per ray)");
  if (t.sort_rays != 0 && t.sort_rays != 1) fail(VT_ERR_RANGE, "sort_rays must be 0 or 1");
}

}  // namespace

extern "C" {

vt_status vt_batch_create(int32_t device, const vt_engine_options* options, vt_batch** out) {
  return vt::guard([&] {
    if (!out) fail(VT_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    auto b = std::make_unique<vt_batch>();
    b->device = device;
    if (options) b->opts = *options;
    if (b->opts.max_bounces == 0) b->opts.max_bounces = 8;
    if (b->opts.max_bounces < 1 || b->opts.max_bounces > 8) fail(VT_ERR_RANGE, "max_bounces must be in [1, 8]");
    if (b->opts.bvh_max_leaf < 0 || b->opts.bvh_max_leaf > 4) fail(VT_ERR_RANGE, "bvh_max_leaf must be in [0, 4]");
    if (b->opts.bvh_width != 0 && (b->opts.bvh_width < 2 || b->opts.bvh_width > 8))
      fail(VT_ERR_RANGE, "bvh_width must be 0 or in [2, 8]");
    if (b->opts.wave_paths > 0) b->tuning.wave_paths = b->opts.wave_paths;
    if (b->opts.sort_by_material > 0) b->tuning.sort_by_material = 1;
    int n = 0;
    VT_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) fail(VT_ERR_INVALID_ARGUMENT, "no such CUDA device");
    vt::DeviceScope ds(device);
    VT_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    VT_CUDA(cudaEventCreate(&b->ev0));
    VT_CUDA(cudaEventCreate(&b->ev1));
    b->counters.resize(vt::pt::kCntWords);
    VT_CUDA(cudaMemset(b->counters.ptr, 0, b->counters.bytes()));
    b->trace_counter.resize(1);
    b->shadow_counter.resize(1);
    VT_CUDA(cudaStreamCreateWithFlags(&b->shadow_stream, cudaStreamNonBlocking));
    VT_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    VT_CUDA(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    b->trace_status.resize(1);
    VT_CUDA(cudaMemset(b->trace_status.ptr, 0, sizeof(int)));
    b->totals.resize(2);
    VT_CUDA(cudaMemset(b->totals.ptr, 0, b->totals.bytes()));
    b->cursor.resize(1);
    *out = b.release();
  });
}

vt_status vt_batch_set_scenes(vt_batch* b, const vt_scene_desc* scenes, const vt_frame_input* frames, size_t count) {
  return vt::guard([&] {
    if (!b) fail(VT_ERR_INVALID_ARGUMENT, "batch is null");
    if (!count || !scenes || !frames) fail(VT_ERR_INVALID_ARGUMENT, "scenes and frames must be non-empty");
    if (count > 256) fail(VT_ERR_RANGE, "at most 256 scenes per batch");
    for (size_t i = 0; i < count; ++i) {
      const vt_frame_input& f = frames[i];
      if (f.width <= 0 || f.height <= 0 || f.width > 16384 || f.height > 16384)
        fail(VT_ERR_RANGE, "scene " + std::to_string(i) + ": viewport must be 1..16384 pixels per side");
      if (f.samples < 1) fail(VT_ERR_RANGE, "scene " + std::to_string(i) + ": samples must be >= 1");
      if (f.bounces < 0 || f.bounces > b->opts.max_bounces)
        fail(VT_ERR_RANGE, "scene " + std::to_string(i) + ": bounces must be in [0, max_bounces]");
      if (scenes[i].instance_count) fail(VT_ERR_INVALID_ARGUMENT, "batch scenes must be single-level");
    }
    // pack the scenes in parallel (independent host builds), then place them
    std::vector<vt::PackedScene> packed(count);
    std::vector<std::string> errors(count);
    std::vector<vt_status> codes(count, VT_OK);
    std::atomic<size_t> next{0};
    const unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), (unsigned)count));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
      pool.emplace_back([&] {
        for (size_t i = next++; i < count; i = next++) {
          try {
            vt::SceneBuild sb;
            sb.bvh_width = b->opts.bvh_width > 0 ? b->opts.bvh_width : 8;
            packed[i] = vt::pack_scene(&scenes[i], 0, 0,
                                       b->opts.bvh_max_leaf > 0 ? b->opts.bvh_max_leaf : vt::kEngineLeafDefault, sb);
          } catch (const vt::Error& e) {
            codes[i] = e.status;
            errors[i] = e.what();
          } catch (const std::exception& e) {
            codes[i] = VT_ERR_INVALID_ARGUMENT;
            errors[i] = e.what();
          }
        }
      });
    for (auto& th : pool) th.join();
    for (size_t i = 0; i < count; ++i)
      if (codes[i] != VT_OK) fail(codes[i], "scene " + std::to_string(i) + ": " + errors[i]);
    // rebase: the scenes were packed at offset 0; shift node and record indices
    std::vector<uint32_t> nodes;
    std::vector<float> recs;
    std::vector<vt::pt::Material> mats;
    std::vector<float4> ems, pts, dls, env, arl;
    std::vector<float> cdf, marg, cond, ltree;
    struct Off { size_t mat, em, cdf, pt, dl, env, marg, cond, arl, lt; };
    std::vector<Off> off(count);
    b->host.assign(count, vt::pt::BatchScene{});
    unsigned long long path = 0;
    size_t pixels = 0;
    int depth = 1;
    uint32_t maxb = 1;
    for (size_t i = 0; i < count; ++i) {
      vt::PackedScene& p = packed[i];
      const uint32_t nb = (uint32_t)(nodes.size() / 20), rb = (uint32_t)(recs.size() / 16);
      // node words: child base (w1.x) of every node and triangle base (w1.y) of nodes with leaves
      for (size_t n = 0; n < p.node_words.size() / 20; ++n) {
        uint32_t* w = &p.node_words[20 * n];
        const uint32_t imask = w[3] >> 24;
        if (imask) w[4] += nb;
        if (w[6]) w[5] += rb;
      }
      off[i] = {mats.size(), ems.size(), cdf.size(), pts.size(), dls.size(), env.size(), marg.size(), cond.size(),
                arl.size(), ltree.size()};
      nodes.insert(nodes.end(), p.node_words.begin(), p.node_words.end());
      recs.insert(recs.end(), p.rec_floats.begin(), p.rec_floats.end());
      mats.insert(mats.end(), p.mats.begin(), p.mats.end());
      ems.insert(ems.end(), p.emitters.begin(), p.emitters.end());
      cdf.insert(cdf.end(), p.cdf.begin(), p.cdf.end());
      pts.insert(pts.end(), p.points.begin(), p.points.end());
      arl.insert(arl.end(), p.area_lights.begin(), p.area_lights.end());
      dls.insert(dls.end(), p.dirs.begin(), p.dirs.end());
      env.insert(env.end(), p.env.begin(), p.env.end());
      marg.insert(marg.end(), p.marg.begin(), p.marg.end());
      cond.insert(cond.end(), p.cond.begin(), p.cond.end());
      ltree.insert(ltree.end(), p.light_tree.begin(), p.light_tree.end());
      vt::pt::BatchScene& B = b->host[i];
      const vt_frame_input& f = frames[i];
      vt::inverse_view_proj(f.view, f.projection, B.inv_vp);
      B.width = (uint32_t)f.width;
      B.height = (uint32_t)f.height;
      B.spp = (uint32_t)f.samples;
      B.max_bounces = (uint32_t)(f.bounces > 0 ? f.bounces : b->opts.max_bounces);
      B.frame_seed = f.frame_seed;
      B.accum_offset = (uint32_t)pixels;
      B.path_begin = path;
      B.view.root = nb;
      path += (unsigned long long)f.width * f.height * f.samples;
      pixels += (size_t)f.width * f.height;
      depth = std::max(depth, p.depth);
      maxb = std::max(maxb, B.max_bounces);
      B.view.material_count = (uint32_t)p.mats.size();
      B.view.n_emitters = (uint32_t)p.cdf.size();
      B.view.emit_area_total = (float)p.emit_total;
      B.view.n_points = (uint32_t)(p.points.size() / vt::pt::kPositionalF4);
      B.view.n_area = (uint32_t)(p.area_lights.size() / vt::pt::kAreaLightF4);
      B.view.n_dirs = (uint32_t)(p.dirs.size() / 2);
      B.view.env_w = p.env_w;
      B.view.env_h = p.env_h;
      B.view.env_scale = p.env_scale;
      B.view.env_cos = (float)std::cos((double)p.env_rotation);
      B.view.env_sin = (float)std::sin((double)p.env_rotation);
      B.view.n_light_entries =
          (B.view.n_emitters ? 1u : 0u) + B.view.n_points + B.view.n_area + B.view.n_dirs + (p.env_sampleable ? 1u : 0u);
    }
    if (pixels > 0xFFFFFFFFull) fail(VT_ERR_RANGE, "batch holds more than 2^32 pixels");
    if (recs.size() / 16 >= (1u << 30) || nodes.size() / 20 >= (1u << 30))
      fail(VT_ERR_RANGE, "batch geometry exceeds 2^30 records or nodes");
    cudaStream_t s = b->stream;
    vt::DeviceScope ds(b->device);
    VT_CUDA(cudaStreamSynchronize(s));
    b->drop_graph();
    std::vector<uint4> n4(nodes.size() / 4);
    std::memcpy(n4.data(), nodes.data(), nodes.size() * 4);
    std::vector<float4> r4(recs.size() / 4);
    if (!recs.empty()) std::memcpy(r4.data(), recs.data(), recs.size() * 4);
    upload(b->nodes, n4, s);
    upload(b->tris, r4, s);
    upload(b->mats, mats, s);
    upload(b->emitters, ems, s);
    upload(b->cdf, cdf, s);
    upload(b->points, pts, s);
    upload(b->areas, arl, s);
    upload(b->dirs, dls, s);
    upload(b->env, env, s);
    upload(b->marg, marg, s);
    upload(b->cond, cond, s);
    upload(b->ltree, ltree, s);
    for (size_t i = 0; i < count; ++i) {
      vt::pt::SceneView& v = b->host[i].view;
      const vt::PackedScene& p = packed[i];
      v.nodes = b->nodes.ptr;
      v.tris = b->tris.ptr;
      v.stack_depth = 2 * depth + 2;
      v.materials = b->mats.ptr + off[i].mat;
      v.emitters = b->emitters.ptr + off[i].em;
      v.emitter_cdf = b->cdf.ptr + off[i].cdf;
      v.points = b->points.ptr + off[i].pt;
      v.area_lights = b->areas.ptr + off[i].arl;
      v.dirs = b->dirs.ptr + off[i].dl;
      v.env = p.has_env ? b->env.ptr + off[i].env : nullptr;
      v.env_marginal = p.env_sampleable ? b->marg.ptr + off[i].marg : nullptr;
      v.env_conditional = p.env_sampleable ? b->cond.ptr + off[i].cond : nullptr;
      v.light_tree_mode = v.n_light_entries >= 2;
      v.light_tree = p.light_tree.empty() ? nullptr : b->ltree.ptr + off[i].lt;
    }
    upload(b->scenes, b->host, s);
    b->accum.resize(std::max<size_t>(pixels, 1));
    VT_CUDA(cudaStreamSynchronize(s));
    b->count = count;
    b->total_paths = path;
    b->pixels = pixels;
    b->max_bounces = maxb;
    b->stack_depth = 2 * depth + 2;
  });
}

vt_status vt_batch_render(vt_batch* b, vt_batch_stats* st) {
  return vt::guard([&] {
    if (!b) fail(VT_ERR_INVALID_ARGUMENT, "batch is null");
    vt::DeviceScope ds(b->device);
    render(b, st);
  });
}

vt_status vt_batch_capture(vt_batch* b, size_t index, float* rgba, size_t cap) {
  return vt::guard([&] {
    if (!b || !rgba) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (index >= b->count) fail(VT_ERR_RANGE, "no such scene in the batch");
    const vt::pt::BatchScene& B = b->host[index];
    const size_t px = (size_t)B.width * B.height;
    if (cap < 4 * px) fail(VT_ERR_RANGE, "capture buffer too small");
    vt::DeviceScope ds(b->device);
    VT_CUDA(cudaStreamSynchronize(b->stream));
    VT_CUDA(cudaMemcpy(rgba, b->accum.ptr + B.accum_offset, px * sizeof(float4), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < px; ++i) {
      const float c = rgba[4 * i + 3];
      const float inv = c > 0.0f ? 1.0f / c : 0.0f;
      rgba[4 * i] *= inv;
      rgba[4 * i + 1] *= inv;
      rgba[4 * i + 2] *= inv;
      rgba[4 * i + 3] = 1.0f;
    }
  });
}

vt_status vt_batch_set_tuning(vt_batch* b, const vt_tuning* t) {
  return vt::guard([&] {
    if (!b || !t) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    validate_tuning(*t);
    b->tuning = *t;
    b->drop_graph();
  });
}

vt_status vt_batch_get_tuning(const vt_batch* b, vt_tuning* t) {
  return vt::guard([&] {
    if (!b || !t) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    *t = b->tuning;
  });
}

vt_status vt_batch_autotune(vt_batch* b, vt_tuning_trial* report, size_t cap, size_t* count) {
  return vt::guard([&] {
    if (!b) fail(VT_ERR_INVALID_ARGUMENT, "batch is null");
    if (!b->count) fail(VT_ERR_STATE, "autotune before set_scenes");
    vt::DeviceScope ds(b->device);
    // coordinate descent: wave size, then sorting, then traversal CTAs per SM;
    // each candidate is timed on one render of the batch after one warm-up
    const vt_tuning start = b->tuning;
    std::vector<vt_tuning_trial> trials;
    auto time_it = [&](const vt_tuning& t) {
      b->tuning = t;
      b->drop_graph();
      vt_batch_stats st{};
      render(b, &st);  // warm-up (and graph capture)
      render(b, &st);
      trials.push_back({t, st.frame_ms});
      return st.frame_ms;
    };
    vt_tuning best = start;
    double best_ms = time_it(best);
    // wave sizes up to the batch frame's paths whose wave state fits in half of
    // the free device memory (the batch's own wave buffers counted as free)
    size_t free_b = 0, total_b = 0;
    VT_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = (free_b + (size_t)b->capacity * batch_bytes_per_path(b)) / 2;
    for (int wp : {1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25, 1 << 26}) {
      if (wp == best.wave_paths) continue;
      if (wp > (1 << 24) &&
          ((unsigned long long)wp / 2 >= b->total_paths || (size_t)wp * batch_bytes_per_path(b) > budget))
        continue;
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
    for (int bp : {2, 4, 6}) {
      if (bp == best.trace_blocks_per_sm) continue;
      vt_tuning t = best;
      t.trace_blocks_per_sm = bp;
      const double ms = time_it(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    {
      vt_tuning t = best;
      t.sort_rays = best.sort_rays ? 0 : 1;
      const double ms = time_it(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
    b->tuning = best;
    b->drop_graph();
    if (count) *count = trials.size();
    if (report)
      for (size_t i = 0; i < trials.size() && i < cap; ++i) report[i] = trials[i];
  });
}

vt_status vt_batch_destroy(vt_batch* b) {
  return vt::guard([&] {
    if (!b) return;
    vt::DeviceScope ds(b->device);
    cudaStreamSynchronize(b->stream);
    delete b;
  });
}

}  // extern "C"
