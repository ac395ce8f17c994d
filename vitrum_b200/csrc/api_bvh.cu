// api_bvh.cu -- C-ABI entry points for the mesh acceleration structure.
//
// vt_bvh_build*        replaces buildArrayBvh + buildCompressedWideBvh
//                      (packages/shared-bvh/src/buildArrayBvh.ts:342,
//                      compressedWideBvh.ts:420)
// vt_bvh_trace_*       replaces intersectCompressedWideBvhFirstHit / AnyHit
//                      (compressedWideBvh.ts:754, :862)
// Errors follow the reference's conventions: invalid options or geometry
// raise (here: return a status and a message), nothing throws across the ABI.
#include <chrono>
#include <memory>
#include <cstring>
#include <string>
#include <vector>

#include "bvh_host.h"
#include "bvh_object.h"
#include "ray_order.h"
#include "traverse.h"
#include "vt_common.h"


namespace vt {

thread_local std::string t_last_error;
void set_last_error(const std::string& msg) { t_last_error = msg; }
void clear_last_error() { t_last_error.clear(); }

void configure_scratch_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  static bool done[64] = {};
  if (dev < 0 || dev >= 64 || done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    unsigned long long keep = 1ull << 30;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done[dev] = true;
}

thread_local long long t_alloc_fail_countdown = 0;  // 0: disarmed
void arm_allocation_failure(long long nth) { t_alloc_fail_countdown = nth > 0 ? nth : 0; }
bool injected_allocation_failure() {
  if (t_alloc_fail_countdown <= 0) return false;
  return --t_alloc_fail_countdown == 0;
}

static BuildOptions resolve(const vt_bvh_build_options* o) {
  BuildOptions r;
  if (!o) return r;
  if (o->position_stride) r.position_stride = o->position_stride;
  if (o->index_stride) r.index_stride = o->index_stride;
  if (o->max_leaf_triangles) r.max_leaf = o->max_leaf_triangles;
  if (o->bin_count) r.bins = o->bin_count;
  if (o->max_depth) r.max_depth = o->max_depth;
  if (o->traversal_tree) r.traversal_tree = o->traversal_tree;
  return r;
}

// The 8-wide grouping the traversal tree is encoded with (nullptr: the reference's rule).
static const WideCollapse* query_collapse(const BuildOptions& o) {
  static const WideCollapse kSah{1.0, 0.5, 8};
  return o.traversal_tree >= 2 ? &kSah : nullptr;
}
// Options of the separate traversal tree (traversal_tree 3): at most two
// triangles per leaf and 32 bins, as the engine's own trees.
static bool separate_tree(const BuildOptions& o) { return o.traversal_tree == 3; }
static BuildOptions traversal_options(const BuildOptions& o) {
  BuildOptions t = o;
  t.max_leaf = std::min(o.max_leaf, 2);
  t.bins = 32;
  return t;
}

// Proves and publishes an encoded tree: the device arrays come from the GPU
// encoder's output when there is one (dev), else from the host arrays.
static void publish(vt_bvh* b, const WideBvhHost& w, const WideBvhDevice* dev) {
  // publication proofs (the reference validates every tree it publishes)
  validate_binary(b->binary, b->ntri);
  validate_wide(w.nodes.data(), w.nodes.size() / 20, w.tris.data(), w.tris.size() / 16, 0, (size_t)b->ntri, false,
                kTraversalStack);
  DeviceScope ds(b->device);
  b->nodes.resize(w.nodes.size() / 4);
  b->tris.resize(std::max<size_t>(w.tris.size() / 4, 1));
  const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  VT_CUDA(cudaMemcpy(b->nodes.ptr, dev ? (const void*)dev->nodes.ptr : w.nodes.data(), w.nodes.size() * 4, kind));
  if (!w.tris.empty())
    VT_CUDA(cudaMemcpy(b->tris.ptr, dev ? (const void*)dev->recs.ptr : w.tris.data(), w.tris.size() * 4, kind));
  VT_CUDA(cudaDeviceSynchronize());  // the copies are complete before any stream of the caller's uses the tree
  b->wide_host_nodes = w.nodes;
  b->wide_host_recs = w.tris;
  b->status.resize(1);
  VT_CUDA(cudaMemset(b->status.ptr, 0, sizeof(int)));
  b->counter.resize(1);
  b->wide_count = (int64_t)(w.nodes.size() / 20);
  b->wide_depth = w.depth;
}

static vt_bvh* build_host(int device, const float* positions, size_t pw, const uint32_t* indices, size_t iw,
                          const vt_bvh_build_options* options) {
  auto t0 = std::chrono::steady_clock::now();
  auto b = std::make_unique<vt_bvh>();
  b->device = device;
  b->opts = resolve(options);
  b->binary = build_binary_host(positions, pw, indices, iw, b->opts);
  b->ntri = (int64_t)(iw / b->opts.index_stride);
  BinaryBvhHost trav;
  if (separate_tree(b->opts)) trav = build_binary_host(positions, pw, indices, iw, traversal_options(b->opts));
  const BinaryBvhHost& tb = separate_tree(b->opts) ? trav : b->binary;
  const WideBvhHost w = encode_wide(tb, positions, b->opts.position_stride, indices, b->opts.index_stride,
                                    nullptr, 0, 0, query_collapse(b->opts));
  publish(b.get(), w, nullptr);
  b->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return b.release();
}

static void check_trace_args(vt_bvh* b, const void* rays, size_t n, const void* out) {
  if (!b) fail(VT_ERR_INVALID_ARGUMENT, "bvh is null");
  if (n && (!rays || !out)) fail(VT_ERR_INVALID_ARGUMENT, "rays and output must be non-null");
  if (n > 0xFFFFFFFFull) fail(VT_ERR_RANGE, "at most 2^32 - 1 rays per call");
}

static TraceArgs trace_args(vt_bvh* b, const vt_ray* rays, size_t n) {
  TraceArgs a;
  a.nodes = b->nodes.ptr;
  a.tris = b->tris.ptr;
  a.rays = reinterpret_cast<const float4*>(rays);
  a.n = n;
  a.status = b->status.ptr;
  a.stack_depth = 2 * b->wide_depth + 2;  // one node group and one postponed triangle group per level
  a.counter = b->counter.ptr;
  a.node_count = b->nodes.count / 5;
  return a;
}

// Batches below this size trace in input order: the sort's four launches cost
// more than the coherence gains.
constexpr size_t kOrderMinRays = 1u << 16;

static bool ordered(const vt_bvh* b, size_t n) {
  return b->order_bits > 0 && n >= kOrderMinRays && !b->binary.nodes.empty();
}

// Scratch of the spatial trace order for batches of up to n rays (grown, never shrunk).
static void ensure_order_scratch(vt_bvh* b, size_t n) {
  if (!ordered(b, n)) return;
  if (b->order_keys.count < n) {
    b->order_keys.resize(n);
    b->order_idx.resize(n);
  }
  const size_t words = 2 * ray_order_count_words(b->order_bits);
  if (b->order_counts.count < words) b->order_counts.resize(words);
}

// Enqueues the spatial sort of a.rays[0, a.n) on s and points the launch at the
// permutation; `off` is the batch's first ray within the scratch, `k` picks the
// bucket array (0 / 1: the two chunk streams).
static void order_batch(vt_bvh* b, TraceArgs& a, size_t off, int k, cudaStream_t s) {
  if (!ordered(b, a.n)) return;
  RayOrderArgs o;
  o.rays = a.rays;
  o.n = a.n;
  const BinaryNode& r = b->binary.nodes[0];
  for (int i = 0; i < 3; ++i) {
    o.lo[i] = r.mn[i];
    o.hi[i] = r.mx[i];
  }
  o.cell_bits = b->order_bits;
  o.keys = b->order_keys.ptr + off;
  o.order = b->order_idx.ptr + off;
  o.counts = b->order_counts.ptr + (size_t)k * ray_order_count_words(b->order_bits);
  launch_ray_order(o, s);
  a.order = o.order;
}

static void check_status(vt_bvh* b) {
  int st = 0;
  VT_CUDA(cudaMemcpy(&st, b->status.ptr, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) {
    cudaMemset(b->status.ptr, 0, sizeof(int));
    fail(VT_ERR_BUILD, trace_status_message(st));
  }
}

}  // namespace vt

using namespace vt;

extern "C" {

const char* vt_last_error(void) { return t_last_error.c_str(); }
const char* vt_version(void) { return "vitrum_b200 0.1 (sm_100a)"; }

vt_status vt_debug_fail_device_allocation(int64_t nth) {
  return guard([&] {
    if (nth < 0) fail(VT_ERR_RANGE, "nth must be >= 0");
    arm_allocation_failure(nth);
  });
}

vt_status vt_bvh_build(int32_t device, const float* positions, size_t position_words, const uint32_t* indices,
                       size_t index_words, const vt_bvh_build_options* options, vt_bvh** out_bvh) {
  return guard([&] {
    if (!out_bvh) fail(VT_ERR_INVALID_ARGUMENT, "out_bvh is null");
    *out_bvh = nullptr;
    if (position_words && !positions) fail(VT_ERR_INVALID_ARGUMENT, "positions is null");
    if (index_words && !indices) fail(VT_ERR_INVALID_ARGUMENT, "indices is null");
    *out_bvh = build_host(device, positions, position_words, indices, index_words, options);
  });
}

vt_status vt_bvh_build_device(int32_t device, const float* d_positions, size_t position_words,
                              const uint32_t* d_indices, size_t index_words, const vt_bvh_build_options* options,
                              void* cuda_stream, vt_bvh** out_bvh) {
  return guard([&] {
    if (!out_bvh) fail(VT_ERR_INVALID_ARGUMENT, "out_bvh is null");
    *out_bvh = nullptr;
    DeviceScope ds(device);
    if (position_words && !d_positions) fail(VT_ERR_INVALID_ARGUMENT, "positions is null");
    if (index_words && !d_indices) fail(VT_ERR_INVALID_ARGUMENT, "indices is null");
    auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = (cudaStream_t)cuda_stream;
    auto b = std::make_unique<vt_bvh>();
    b->device = device;
    b->opts = resolve(options);
    // the binary tree and its 8-wide encoding are built on the GPU (every binCount
    // the options allow); the host receives copies for the publication proofs
    BinaryBvhDevice bd;
    b->binary = build_binary_gpu(d_positions, position_words, d_indices, index_words, b->opts, s, &bd);
    b->ntri = (int64_t)(index_words / b->opts.index_stride);
    BinaryBvhDevice td;
    if (separate_tree(b->opts))
      build_binary_gpu(d_positions, position_words, d_indices, index_words, traversal_options(b->opts), s, &td);
    WideBvhDevice wd;
    const WideBvhHost w = encode_wide_gpu(separate_tree(b->opts) ? td : bd, d_positions, b->opts.position_stride,
                                          d_indices, b->opts.index_stride, nullptr, 0, 0, query_collapse(b->opts),
                                          nullptr, s, &wd);
    publish(b.get(), w, &wd);
    b->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    *out_bvh = b.release();
  });
}

vt_status vt_bvh_export_wide(const vt_bvh* b, uint32_t* node_words, size_t word_capacity, float* records,
                             size_t float_capacity, size_t* out_words, size_t* out_floats) {
  return guard([&] {
    if (!b) fail(VT_ERR_INVALID_ARGUMENT, "bvh is null");
    if (out_words) *out_words = b->wide_host_nodes.size();
    if (out_floats) *out_floats = b->wide_host_recs.size();
    if (node_words) {
      if (word_capacity < b->wide_host_nodes.size()) fail(VT_ERR_RANGE, "node buffer too small");
      std::memcpy(node_words, b->wide_host_nodes.data(), b->wide_host_nodes.size() * 4);
    }
    if (records) {
      if (float_capacity < b->wide_host_recs.size()) fail(VT_ERR_RANGE, "record buffer too small");
      std::memcpy(records, b->wide_host_recs.data(), b->wide_host_recs.size() * 4);
    }
  });
}

vt_status vt_bvh_get_info(const vt_bvh* b, vt_bvh_info* info) {
  return guard([&] {
    if (!b || !info) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    info->triangle_count = b->ntri;
    info->binary_node_count = (int64_t)b->binary.nodes.size();
    info->wide_node_count = b->wide_count;
    info->wide_depth = b->wide_depth;
    info->binary_depth = b->binary.depth;
    info->build_ms = b->build_ms;
  });
}

vt_status vt_bvh_export_binary(const vt_bvh* b, uint32_t* nodes, size_t node_word_capacity,
                               uint32_t* reordered_to_source, size_t triangle_capacity) {
  return guard([&] {
    if (!b) fail(VT_ERR_INVALID_ARGUMENT, "bvh is null");
    if (nodes) {
      if (node_word_capacity < b->binary.nodes.size() * 8) fail(VT_ERR_RANGE, "node buffer too small");
      std::memcpy(nodes, b->binary.nodes.data(), b->binary.nodes.size() * 32);
    }
    if (reordered_to_source) {
      if (triangle_capacity < b->binary.reordered_to_source.size()) fail(VT_ERR_RANGE, "triangle buffer too small");
      std::memcpy(reordered_to_source, b->binary.reordered_to_source.data(),
                  b->binary.reordered_to_source.size() * 4);
    }
  });
}

vt_status vt_bvh_trace_closest_device(vt_bvh* b, const vt_ray* d_rays, size_t n, vt_hit* d_hits,
                                      void* cuda_stream) {
  return guard([&] {
    check_trace_args(b, d_rays, n, d_hits);
    DeviceScope ds(b->device);
    ensure_order_scratch(b, n);
    TraceArgs a = trace_args(b, d_rays, n);
    a.hits = reinterpret_cast<int4*>(d_hits);
    order_batch(b, a, 0, 0, (cudaStream_t)cuda_stream);
    launch_trace_closest(a, (cudaStream_t)cuda_stream);
    VT_CUDA(cudaGetLastError());
  });
}

vt_status vt_bvh_set_trace_order(vt_bvh* b, int32_t cell_bits) {
  return guard([&] {
    if (!b) fail(VT_ERR_INVALID_ARGUMENT, "bvh is null");
    if (cell_bits < 0 || cell_bits > kRayOrderMaxCellBits) fail(VT_ERR_RANGE, "cell_bits must be in [0, 6]");
    b->order_bits = cell_bits;
  });
}

vt_status vt_bvh_trace_any_device(vt_bvh* b, const vt_ray* d_rays, size_t n, uint8_t* d_occluded,
                                  void* cuda_stream) {
  return guard([&] {
    check_trace_args(b, d_rays, n, d_occluded);
    DeviceScope ds(b->device);
    ensure_order_scratch(b, n);
    TraceArgs a = trace_args(b, d_rays, n);
    a.occluded = d_occluded;
    order_batch(b, a, 0, 0, (cudaStream_t)cuda_stream);
    launch_trace_any(a, (cudaStream_t)cuda_stream);
    VT_CUDA(cudaGetLastError());
  });
}

// Host-buffer queries above this size run in chunks on two streams, so that the
// copies of one chunk overlap the traversal of the other (with page-locked host
// buffers the copies are asynchronous; with pageable ones they serialise, as
// any copy from pageable memory does).
constexpr size_t kQueryChunk = 1u << 19;

static void ensure_copy_streams(vt_bvh* b) {
  for (cudaStream_t& s : b->copy_streams)
    if (!s) VT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  b->chunk_counters.resize(2);
}

vt_status vt_bvh_trace_closest(vt_bvh* b, const vt_ray* rays, size_t n, vt_hit* hits) {
  return guard([&] {
    check_trace_args(b, rays, n, hits);
    if (!n) return;
    DeviceScope ds(b->device);
    b->rays_scratch.resize(2 * n);
    b->hits_scratch.resize(n);
    ensure_order_scratch(b, n);
    if (n <= kQueryChunk) {
      VT_CUDA(cudaMemcpy(b->rays_scratch.ptr, rays, n * sizeof(vt_ray), cudaMemcpyHostToDevice));
      TraceArgs a = trace_args(b, reinterpret_cast<const vt_ray*>(b->rays_scratch.ptr), n);
      a.hits = b->hits_scratch.ptr;
      order_batch(b, a, 0, 0, 0);
      launch_trace_closest(a, 0);
      VT_CUDA(cudaGetLastError());
      VT_CUDA(cudaMemcpy(hits, b->hits_scratch.ptr, n * sizeof(vt_hit), cudaMemcpyDeviceToHost));
    } else {
      ensure_copy_streams(b);
      VT_CUDA(cudaStreamSynchronize(0));  // earlier work on the legacy stream (builds, status resets) is done
      size_t k = 0;
      for (size_t c = 0; c < n; c += kQueryChunk, ++k) {
        cudaStream_t s = b->copy_streams[k & 1];
        const size_t m = std::min(kQueryChunk, n - c);
        VT_CUDA(cudaMemcpyAsync(b->rays_scratch.ptr + 2 * c, rays + c, m * sizeof(vt_ray), cudaMemcpyHostToDevice, s));
        TraceArgs a = trace_args(b, reinterpret_cast<const vt_ray*>(b->rays_scratch.ptr + 2 * c), m);
        a.hits = b->hits_scratch.ptr + c;
        a.counter = b->chunk_counters.ptr + (k & 1);
        order_batch(b, a, c, (int)(k & 1), s);
        launch_trace_closest(a, s);
        VT_CUDA(cudaGetLastError());
        VT_CUDA(cudaMemcpyAsync(hits + c, b->hits_scratch.ptr + c, m * sizeof(vt_hit), cudaMemcpyDeviceToHost, s));
      }
      for (cudaStream_t s : b->copy_streams) VT_CUDA(cudaStreamSynchronize(s));
    }
    check_status(b);
  });
}

vt_status vt_bvh_trace_any(vt_bvh* b, const vt_ray* rays, size_t n, uint8_t* occluded) {
  return guard([&] {
    check_trace_args(b, rays, n, occluded);
    if (!n) return;
    DeviceScope ds(b->device);
    b->rays_scratch.resize(2 * n);
    b->occ_scratch.resize(n);
    ensure_order_scratch(b, n);
    VT_CUDA(cudaMemcpy(b->rays_scratch.ptr, rays, n * sizeof(vt_ray), cudaMemcpyHostToDevice));
    TraceArgs a = trace_args(b, reinterpret_cast<const vt_ray*>(b->rays_scratch.ptr), n);
    a.occluded = b->occ_scratch.ptr;
    order_batch(b, a, 0, 0, 0);
    launch_trace_any(a, 0);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaMemcpy(occluded, b->occ_scratch.ptr, n, cudaMemcpyDeviceToHost));
    check_status(b);
  });
}

vt_status vt_validate_bvh_encoding(const uint32_t* node_words, size_t word_count, size_t total_nodes,
                                   const uint32_t* roots, size_t root_count, int64_t triangle_count,
                                   int32_t traversal_stack_capacity, vt_bvh_proof* out) {
  return guard([&] {
    if (word_count && !node_words) fail(VT_ERR_INVALID_ARGUMENT, "node_words is null");
    if (traversal_stack_capacity < 0) fail(VT_ERR_RANGE, "traversal_stack_capacity must be >= 0");
    BinaryProof p = validate_binary_encoding(node_words, word_count, total_nodes, roots, roots ? root_count : 0,
                                             triangle_count, traversal_stack_capacity ? traversal_stack_capacity : 60);
    if (out) {
      out->node_count = p.node_count;
      out->root_count = p.root_count;
      out->interior_node_count = p.interior_node_count;
      out->leaf_node_count = p.leaf_node_count;
      out->max_depth = p.max_depth;
      out->max_traversal_stack_entries = p.max_stack_entries;
      out->traversal_stack_capacity = p.stack_capacity;
      out->triangle_count = p.triangle_count;
    }
  });
}

vt_status vt_bvh_validate(const vt_bvh* b, vt_wide_proof* out) {
  return guard([&] {
    if (!b || !out) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    DeviceScope ds(b->device);
    std::vector<uint32_t> nodes(b->nodes.count * 4);
    std::vector<float> recs(b->tris.count * 4);
    VT_CUDA(cudaMemcpy(nodes.data(), b->nodes.ptr, nodes.size() * 4, cudaMemcpyDeviceToHost));
    VT_CUDA(cudaMemcpy(recs.data(), b->tris.ptr, recs.size() * 4, cudaMemcpyDeviceToHost));
    WideProof p = validate_wide(nodes.data(), nodes.size() / 20, recs.data(), recs.size() / 16, 0, (size_t)b->ntri,
                                false, kTraversalStack);
    out->node_count = p.node_count;
    out->internal_slots = p.internal_slots;
    out->leaf_slots = p.leaf_slots;
    out->triangle_count = p.items;
    out->depth = p.depth;
    out->stack_entries = p.stack_entries;
  });
}

vt_status vt_tlas_build(const double* aabbs, size_t n, int32_t max_leaf, int32_t bin_count, int32_t max_depth,
                        uint32_t* nodes, size_t node_word_capacity, uint32_t* instance_indices,
                        size_t instance_capacity, size_t* node_count) {
  return guard([&] {
    if (n && !aabbs) fail(VT_ERR_INVALID_ARGUMENT, "aabbs is null");
    if (max_leaf < 0 || bin_count < 0 || max_depth < 0) fail(VT_ERR_INVALID_ARGUMENT, "negative option");
    if (bin_count == 1) fail(VT_ERR_INVALID_ARGUMENT, "binCount must be at least 2");
    BinaryBvhHost t = build_tlas_host(aabbs, n, max_leaf ? max_leaf : 1, bin_count ? bin_count : 16,
                                      max_depth ? max_depth : kMaxBinaryDepth);
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

vt_status vt_bvh_destroy(vt_bvh* b) {
  return guard([&] {
    if (!b) return;
    DeviceScope ds(b->device);
    delete b;
  });
}

vt_status vt_watertight_eval_device(int32_t device, const float* d_cases, size_t n, vt_watertight_result* d_out,
                                    void* cuda_stream) {
  return guard([&] {
    if (n && (!d_cases || !d_out)) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    DeviceScope ds(device);
    launch_watertight_eval(d_cases, n, d_out, (cudaStream_t)cuda_stream);
    VT_CUDA(cudaGetLastError());
  });
}

}  // extern "C"
