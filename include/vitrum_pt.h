/*
 * vitrum_pt.h -- C ABI of the B200 ray-tracing backend (libvitrum_pt.so).
 *
 * Plain pointers and sizes only; every entry point returns vt_status
 * (VT_OK == 0) and never throws across the boundary.  The message of the
 * most recent failure on the calling thread is available from
 * vt_last_error().  Device pointers are CUDA global-memory addresses on the
 * device the object was created on; host pointers are ordinary memory.
 *
 * Each declaration names the reference interface it replaces (paths inside
 * the reference project jsquire4/vitrum).
 */
#ifndef VITRUM_PT_H
#define VITRUM_PT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t vt_status;
enum {
  VT_OK = 0,
  VT_ERR_INVALID_ARGUMENT = 1, /* TypeError / RangeError in the reference */
  VT_ERR_RANGE = 2,            /* a size or index outside its documented range */
  VT_ERR_CUDA = 3,             /* a CUDA runtime failure (latched, see vt_last_error) */
  VT_ERR_OUT_OF_MEMORY = 4,
  VT_ERR_STATE = 5,            /* call not valid in the object's state (disposed, no scene) */
  VT_ERR_BUILD = 6,            /* BVH build invariant violated (maxDepth, leaf cap) */
  VT_ERR_TIMEOUT = 7           /* a bounded device wait gave up */
};

/* Message of the last failed call on this thread ("" when none). */
const char* vt_last_error(void);
/* Library version string. */
const char* vt_version(void);

/* ------------------------------------------------------------------ */
/* Acceleration structure over one triangle mesh (shared-bvh)           */
/* ------------------------------------------------------------------ */

typedef struct vt_bvh vt_bvh;

/* Mirrors BuildArrayBvhOpts, packages/shared-bvh/src/buildArrayBvh.ts:277-318.
 * Zero fields select the reference defaults (stride 4/4, leaf 4, 16 bins,
 * maxDepth 58 = BINARY_BVH_MAX_BUILD_DEPTH, strides.ts:119-125). */
typedef struct vt_bvh_build_options {
  int32_t position_stride;    /* 3 or 4 floats per vertex */
  int32_t index_stride;       /* 3 or 4 u32 per triangle */
  int32_t max_leaf_triangles; /* 1..4 on the GPU path (8-wide nodes hold <= 4 triangles per child) */
  int32_t bin_count;          /* 2..256 */
  int32_t max_depth;          /* 0..58 */
} vt_bvh_build_options;

/* Build statistics filled by vt_bvh_build*(). */
typedef struct vt_bvh_info {
  int64_t triangle_count;
  int64_t binary_node_count;   /* nodes of the binned-SAH binary tree */
  int64_t wide_node_count;     /* 8-wide compressed nodes (80 bytes each) */
  int32_t wide_depth;          /* levels of the 8-wide tree */
  int32_t binary_depth;        /* deepest interior level of the binary tree */
  double build_ms;             /* wall time of the last build */
} vt_bvh_info;

/* One ray: 32 bytes, origin + tmin, direction + tmax (tmax may be +inf). */
typedef struct vt_ray {
  float ox, oy, oz, tmin;
  float dx, dy, dz, tmax;
} vt_ray;

/* One closest-hit record: 16 bytes.  prim = source triangle index or -1;
 * (u, v) are the weights of vertices 1 and 2 (w = 1 - u - v weights vertex 0). */
typedef struct vt_hit {
  int32_t prim;
  float t;
  float u;
  float v;
} vt_hit;

/*
 * Build the binned-SAH BVH (replaces buildArrayBvh, shared-bvh/src/buildArrayBvh.ts:342,
 * and its 8-wide collapse buildCompressedWideBvh, shared-bvh/src/compressedWideBvh.ts:420)
 * from HOST arrays.  The library copies the geometry to the device; the
 * caller keeps ownership of its arrays.  positions: position_words floats,
 * indices: index_words u32.
 */
vt_status vt_bvh_build(int32_t device, const float* positions, size_t position_words, const uint32_t* indices,
                       size_t index_words, const vt_bvh_build_options* options, vt_bvh** out_bvh);

/* Same build from DEVICE arrays (no host round trip for the geometry). */
vt_status vt_bvh_build_device(int32_t device, const float* d_positions, size_t position_words,
                              const uint32_t* d_indices, size_t index_words, const vt_bvh_build_options* options,
                              void* cuda_stream, vt_bvh** out_bvh);

vt_status vt_bvh_get_info(const vt_bvh* bvh, vt_bvh_info* out_info);

/*
 * Copy the binary tree back to the host in the reference's 32-byte node
 * layout (buildArrayBvh.ts:13-27): nodes = 8 u32 words per node,
 * reordered_to_source = one u32 per triangle (CpuBvhBuildResult.reorderedToSourceTriangle).
 * Capacities are in elements; pass NULL to skip an array.
 */
vt_status vt_bvh_export_binary(const vt_bvh* bvh, uint32_t* nodes, size_t node_word_capacity,
                               uint32_t* reordered_to_source, size_t triangle_capacity);

/*
 * Closest hit for n rays (replaces intersectCompressedWideBvhFirstHit,
 * shared-bvh/src/compressedWideBvh.ts:754).  DEVICE pointers: rays (n vt_ray),
 * hits (n vt_hit).  Enqueued on cuda_stream (NULL = default stream); returns
 * once the launch is enqueued.
 */
vt_status vt_bvh_trace_closest_device(vt_bvh* bvh, const vt_ray* d_rays, size_t n, vt_hit* d_hits,
                                      void* cuda_stream);

/*
 * Any hit for n rays (replaces intersectCompressedWideBvhAnyHit,
 * shared-bvh/src/compressedWideBvh.ts:862).  d_occluded: n bytes, 1 = hit.
 */
vt_status vt_bvh_trace_any_device(vt_bvh* bvh, const vt_ray* d_rays, size_t n, uint8_t* d_occluded,
                                  void* cuda_stream);

/* HOST-buffer variants: copy rays in, trace, copy hits out, synchronise. */
vt_status vt_bvh_trace_closest(vt_bvh* bvh, const vt_ray* rays, size_t n, vt_hit* hits);
vt_status vt_bvh_trace_any(vt_bvh* bvh, const vt_ray* rays, size_t n, uint8_t* occluded);

vt_status vt_bvh_destroy(vt_bvh* bvh);

/*
 * Closest hit for host rays without allocating any device memory.  No
 * counterpart in the reference: its query is a CPU function.  For callers
 * that cannot allocate -- hosts with a fixed, pre-reserved device memory
 * budget, or host-array callers (the Node addon) on a path where no
 * cudaMalloc may happen; vt_bvh_trace_closest grows per-object staging
 * instead.  Scratch is a library-wide device array of 3 MiB + 256 B, held by
 * every GPU that loads the library until exit; n is at most 65,536 rays per
 * call (VT_ERR_RANGE beyond).  The first call on a device looks up that
 * array's address and must precede any stream capture.  Calls that overlap
 * on the GPU race on the shared array.  Synchronous; same results as
 * vt_bvh_trace_closest.
 */
vt_status vt_bvh_trace_closest_noalloc(const vt_bvh* bvh, const vt_ray* rays, size_t n, vt_hit* hits);

/* ------------------------------------------------------------------ */
/* Triangle test (shared-bvh/src/opticalWatertightTriangle.ts:98)       */
/* ------------------------------------------------------------------ */

/* Result of the f32 watertight test for one ray/triangle pair. */
typedef struct vt_watertight_result {
  int32_t hit;
  float t;
  float bary[3];      /* weights of a, b, c */
  int32_t side;       /* +1 front, -1 back, 0 on miss */
  int32_t zero_edge_mask;
} vt_watertight_result;

/*
 * Evaluate intersectOpticalTriangleWatertightF32 on the GPU for n cases
 * (DEVICE pointers).  cases: 16 floats each = o.xyz, d.xyz, a.xyz, b.xyz,
 * c.xyz, exclusive_min_t.  Used to pin the device triangle test bit-exactly.
 */
vt_status vt_watertight_eval_device(int32_t device, const float* d_cases, size_t n, vt_watertight_result* d_out,
                                    void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* VITRUM_PT_H */
