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
  int32_t traversal_tree;     /* the tree the queries traverse (no reference option; the exported binary tree
                                 and every hit are the same whichever is chosen): 0 = default (3);
                                 1 = the exported tree grouped 8-wide by the reference's largest-area rule
                                 (compressedWideBvh.ts:215-242); 2 = the exported tree grouped by the
                                 SAH-optimal rule (Ylitie et al. 2017); 3 = a second binned-SAH tree built
                                 beside it with at most 2 triangles per leaf and 32 bins, grouped by the
                                 SAH-optimal rule (the engine's own trees; 12 % faster queries on the
                                 65,536-triangle benchmark for about twice the build time) */
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

/* Same build from DEVICE arrays, on the GPU: the binned-SAH binary tree (one
 * CTA per node per level, every binCount the options allow) and its 8-wide
 * encoding, word for word those of vt_bvh_build; the host receives copies for
 * the publication proofs and the exports. */
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

/* The published 8-wide nodes (20 words each) and triangle records (16 floats
 * each) of this backend's own encoding (no reference counterpart; the
 * reference's compressed nodes are a different layout).  Null buffers: only
 * the sizes are written to out_words / out_floats. */
vt_status vt_bvh_export_wide(const vt_bvh* bvh, uint32_t* node_words, size_t word_capacity, float* records,
                             size_t float_capacity, size_t* out_words, size_t* out_floats);

/*
 * Closest hit for n rays (replaces intersectCompressedWideBvhFirstHit,
 * shared-bvh/src/compressedWideBvh.ts:754).  DEVICE pointers: rays (n vt_ray),
 * hits (n vt_hit).  Enqueued on cuda_stream (NULL = default stream); returns
 * once the launch is enqueued.  With a spatial trace order set
 * (vt_bvh_set_trace_order), batches of 65,536 rays or more are sorted first;
 * the first such call at a new largest batch size allocates the sort's
 * scratch (8 bytes per ray plus the bucket arrays), so make it before any
 * stream capture.
 */
vt_status vt_bvh_trace_closest_device(vt_bvh* bvh, const vt_ray* d_rays, size_t n, vt_hit* d_hits,
                                      void* cuda_stream);

/*
 * Trace order of this BVH's query batches (no reference counterpart: the
 * reference traces one ray at a time).  cell_bits 1..6: batches of at least
 * 65,536 rays are traced grouped by the 2^cell_bits-per-axis cell of the scene
 * box where each ray enters it and by direction octant, so neighbouring lanes
 * walk the same nodes; 0: input order.  Results are the same either way (each
 * hit is written at its own ray).  Default 0: on rays spread uniformly over
 * the scene (the closest-hit benchmark's sphere of origins) the persistent
 * traversal, which refills each finished lane with the next ray, runs as fast
 * unsorted, and the sort's cost is not repaid.
 */
vt_status vt_bvh_set_trace_order(vt_bvh* bvh, int32_t cell_bits);

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

/* Structural proof of a packed binary BVH (validateBvhEncoding,
 * shared-bvh/src/validateBvhEncoding.ts:55, BvhEncodingProof). */
typedef struct vt_bvh_proof {
  int64_t node_count;
  int64_t root_count;
  int64_t interior_node_count;
  int64_t leaf_node_count;
  int64_t max_depth;
  int64_t max_traversal_stack_entries;   /* depth + 1: the deepest path plus one pending sibling per ancestor */
  int64_t traversal_stack_capacity;
  int64_t triangle_count;                /* -1 when not checked */
} vt_bvh_proof;

/*
 * Replaces validateBvhEncoding (validateBvhEncoding.ts:55): proves a packed
 * binary BVH (node_words = 8 u32 per node, buildArrayBvh.ts:13-27) safe for a
 * fixed-stack traversal -- buffer extent, declared roots, reachability with
 * exclusive ownership, split axes, finite ordered bounds enclosing both
 * children, leaf ranges tiling [0, triangle_count) exactly (triangle_count
 * < 0: not checked), and depth + 1 <= traversal_stack_capacity (0: 60).
 * roots == NULL: root 0.  A violation returns VT_ERR_BUILD with the
 * reference's message; host only.
 */
vt_status vt_validate_bvh_encoding(const uint32_t* node_words, size_t word_count, size_t total_nodes,
                                   const uint32_t* roots, size_t root_count, int64_t triangle_count,
                                   int32_t traversal_stack_capacity, vt_bvh_proof* out_proof);

/* Proof of this library's 8-wide tree as it lies on the device (read back):
 * every node reached once, record masks contiguous, every triangle named by
 * exactly one leaf record, every vertex inside its slot's and all ancestor
 * slots' dequantised boxes, stack bound within capacity.  The same proof runs
 * on every tree before it is published (vt_bvh_build*, vt_set_scene). */
typedef struct vt_wide_proof {
  int64_t node_count;
  int64_t internal_slots;
  int64_t leaf_slots;
  int64_t triangle_count;
  int64_t depth;
  int64_t stack_entries;
} vt_wide_proof;
vt_status vt_bvh_validate(const vt_bvh* bvh, vt_wide_proof* out_proof);

/* One emitter of a light tree (LightTreeBuildInput, shared-samplers/src/lightTree.ts:114-144). */
typedef struct vt_light_tree_emitter {
  double power;            /* luminance (x area for area emitters), >= 0 */
  double centroid[3];
  double aabb_min[3];
  double aabb_max[3];
  double cone_axis[3];     /* orientation cone (oriented = 1): emission axis, */
  double cone_theta_o;     /* spread of the axes and */
  double cone_theta_e;     /* emission half-angle beyond the axis (radians) */
  int32_t oriented;        /* 0: full-sphere emitter */
} vt_light_tree_emitter;

/*
 * Replaces buildLightTree + packLightTreeForGPU (lightTree.ts:492, 611): the
 * pre-order binary light tree over n emitters, packed as 16 floats per node
 * (emitter index, represented power, children, AABB, unit cone axis,
 * outward-rounded cosines of thetaO and thetaO + thetaE, subtree leaf count).
 * *node_count receives the node count (2n - 1); pass NULL to query it.  Host only.
 */
vt_status vt_light_tree_build(const vt_light_tree_emitter* emitters, size_t n, float* nodes, size_t float_capacity,
                              size_t* node_count);

/*
 * The device selection the path tracer's next-event estimation uses: for each
 * point (3 floats) and 24-bit draw, the selected entry and its probability
 * (bucket count / 2^24).  Entries 0 .. P-1 are the tree's leaves (P = (node_count
 * + 1) / 2, selected by samplePackedLightTreeCPU's descent, lightTree.ts:1237);
 * entries P .. P + n_distant - 1 are distant lights (directionals, an
 * environment), which take n_distant / (n_distant + 1) of the buckets (all of
 * them without a tree) shared evenly.  d_normals (3 floats per point, or null
 * for none) are unit receiver normals: the descent's importance is multiplied
 * by cos(max(0, theta_i - theta_u)) of each child seen from the point (Conty
 * Estevez & Kulla 2018), which the reference's importance leaves out; a zero
 * normal (transmissive surface) keeps the reference's importance.  Half of the
 * tree's buckets are split evenly over its leaves (the reference keeps one per
 * leaf).  DEVICE pointers; enqueued on cuda_stream.
 */
vt_status vt_light_tree_select_device(const float* d_tree, size_t node_count, uint32_t n_distant,
                                      const float* d_points, const float* d_normals, const uint32_t* d_buckets,
                                      size_t n, uint32_t* d_emitter, float* d_pmf, void* cuda_stream);

/*
 * Top-level build over instance world AABBs (replaces buildTlas,
 * shared-bvh/src/tlas.ts:859-989): binned SAH over the boxes' centroids, the
 * balanced median fallback for degenerate, non-improving or depth-unsafe
 * splits.  aabbs: n x 6 doubles (min xyz, max xyz) in instance order.  0 for
 * an option takes the reference's default (maxLeafSize 1, binCount 16,
 * maxDepth 58).  Writes the 32-byte reference node layout (8 u32 words per
 * node, buildArrayBvh.ts:13-27; leaves index the instance permutation) and the
 * instanceIndices permutation.  *node_count (optional) receives the node count;
 * pass NULL buffers to query it.  Host only: no device is touched.
 */
vt_status vt_tlas_build(const double* aabbs, size_t n, int32_t max_leaf, int32_t bin_count, int32_t max_depth,
                        uint32_t* nodes, size_t node_word_capacity, uint32_t* instance_indices,
                        size_t instance_capacity, size_t* node_count);

/*
 * Closest hit for host rays without allocating any device memory.  No
 * counterpart in the reference: its query is a CPU function.  For callers
 * that cannot allocate -- hosts with a fixed, pre-reserved device memory
 * budget, or host-array callers (the Node addon) on a path where no
 * cudaMalloc may happen; vt_bvh_trace_closest grows per-object staging
 * instead.  Scratch is a library-wide device array of 3 MiB + 256 B, held by
 * every GPU that loads the library until exit; n is at most 65,536 rays per
 * call (VT_ERR_RANGE beyond).  The first call on a device loads the module
 * that holds the array (lazy loading may allocate in the driver that once):
 * make it during set-up, before any stream capture -- a call with n == 0
 * does only that.  Calls that overlap on the GPU race on the shared array.
 * Runs on the legacy default stream and blocks until the hits are in host
 * memory; same results as vt_bvh_trace_closest.
 */
vt_status vt_bvh_trace_closest_noalloc(const vt_bvh* bvh, const vt_ray* rays, size_t n, vt_hit* hits);

/* ------------------------------------------------------------------ */
/* Path-tracing engine (@vitrum/core Engine, backend pt-webgpu)         */
/* ------------------------------------------------------------------ */

typedef struct vt_engine vt_engine;

/* Creation-time options (PTEngineWebGPUOptions, pt-webgpu/src/index.ts:219-345).
 * Zero selects the default. */
typedef struct vt_engine_options {
  int32_t max_bounces;            /* default 8 (PT_WEBGPU_MAX_BOUNCES, ptWebgpuValidation.ts:181), at most 8 */
  int32_t max_samples_per_pixel;  /* default 4096 (index.ts:370) */
  int32_t debug;                  /* 1 enables vt_pick (EngineOptions.debug, engine/factory.ts) */
  int32_t oracle_accumulation;    /* 1 keeps FP64 per-pixel sums and sums of squares */
  int32_t sort_by_material;       /* 1 = sort shading work by BSDF family; 0 (default) = queue order */
  int32_t wave_paths;             /* paths in flight per wave; 0 = 2^24 (~300 B of device state per path,
                                     about 4.7 GB), halved down to 2^20 until it fits half the free memory */
  int32_t bvh_max_leaf;           /* triangles per leaf of the engine's own trees, 1..4; 0 = 2 (the reference's
                                     builder with 2 instead of its default 4: the same hits, faster traversal) */
  int32_t light_selection;        /* next-event light selection: 0 = with two or more light entries, the light tree
                                     (shared-samplers/src/lightTree.ts: power x proximity x orientation) over the
                                     positional entries and the distant ones (directionals, environment) sharing
                                     n / (n + 1) of the selection evenly; 1 = uniform over the entries */
  int32_t scene_build;            /* where setScene builds the trees: 0 = on the GPU (binned-SAH binary tree, SAH-
                                     optimal 8-wide encoding and the instance top level); 1 = on the host (the same
                                     words, the reference pipeline the GPU build is checked against).  Debug
                                     engines also run the structural proofs on every tree they publish. */
  int32_t bvh_width;              /* children per wide node at most in the engine's own triangle trees, 2..8;
                                     0 = 8 (the node format's capacity; the SAH-optimal collapse fills it) */
} vt_engine_options;

/* Material (core MaterialSpec subset, core/src/scene/material.ts), the
 * reference's base BSDF: transmission > 0 with metallic 0 is a dielectric
 * interface (delta at roughness 0, rough GGX otherwise; 1 - transmission of the
 * refracted share scatters diffusely); anything else is opaque: Lambert
 * diffuse under a GGX specular layer with F0 = mix(specular_intensity *
 * ((ior-1)/(ior+1))^2, base_color, metallic) and Kulla-Conty multiple
 * scattering.  specular_intensity 0 with metallic 0 is a pure Lambertian.
 * emission is radiance leaving the front face (winding normal). */
typedef struct vt_material_desc {
  float base_color[3];
  float roughness;          /* [0, 1]; GGX alpha = max(roughness^2, 1e-3) */
  float metallic;           /* [0, 1] */
  float transmission;       /* [0, 1] */
  float ior;                /* 0: 1.5 */
  float emission[3];
  uint32_t flags;           /* VT_MATERIAL_* bits */
  float specular_intensity; /* KHR_materials_specular factor in [0, 1] (MaterialSpec.specularIntensity, default 1) */
} vt_material_desc;

/* Material flags (the hits traceClosest / traceAny skip and retrace past,
 * pt-webgpu/src/wgsl/pathTrace/intersection.wgsl.ts:462-528). */
#define VT_MATERIAL_SINGLE_SIDED 1u  /* back-face hits are ignored by every ray */
#define VT_MATERIAL_NO_SHADOW 2u     /* castShadow: false -- ignored by shadow (any-hit) rays */

/* One triangle mesh in world space. */
typedef struct vt_mesh_desc {
  const float* positions;   /* 3 floats per vertex */
  size_t vertex_count;
  const uint32_t* indices;  /* 3 per triangle */
  size_t triangle_count;
  uint32_t material;        /* index into vt_scene_desc.materials */
} vt_mesh_desc;

/* Point light (core PointEmitter, core/src/scene/emitters.ts:67-72) with the
 * reference's defaults: inverse-square falloff, no range cutoff.  A point light
 * with another falloff or a range is a vt_spot_light_desc with angle pi. */
typedef struct vt_point_light_desc {
  float position[3];
  float intensity[3];       /* radiant intensity; irradiance falls off as 1/d^2 */
} vt_point_light_desc;

/* Spot light (core SpotEmitter, core/src/scene/emitters.ts:74-85; NEE as
 * pt-webgpu/src/wgsl/pathTrace/kernel.wgsl.ts:1344-1397): a delta light at
 * `position` emitting `intensity` into the cone of half-angle `angle` around
 * `direction`, smoothly from the inner cone angle * (1 - penumbra) to the outer
 * edge, scaled by 1/d^decay (decay 0: none) and, with distance > 0, by
 * clamp(1 - (d / distance)^4, 0, 1) (pointSpotDistanceAttenuation,
 * material.wgsl.ts:2176-2204).  The reference's default decay is 2. */
typedef struct vt_spot_light_desc {
  float position[3];
  float direction[3];       /* beam axis (normalised on input) */
  float intensity[3];
  float angle;              /* outer half-angle, radians, in (0, pi] */
  float penumbra;           /* [0, 1] */
  float distance;           /* range cutoff; 0 = none */
  float decay;              /* falloff exponent >= 0 */
} vt_spot_light_desc;

/* Disc area light (core DiscAreaEmitter, emitters.ts:53-58): emits `radiance`
 * from the side `normal` faces; sampled by the concentric map, hit
 * analytically by BSDF rays (MIS), invisible to shadow rays and from behind,
 * and not an occluder (pt-webgpu/src/scene/emitterPacking.ts:78-93,
 * connect.wgsl.ts:390-450). */
typedef struct vt_disc_light_desc {
  float center[3];
  float normal[3];
  float radius;
  float radiance[3];
} vt_disc_light_desc;

/* Directional light (sun): light travelling along `direction`.  With
 * angular_radius 0 a delta light of irradiance `irradiance` at normal
 * incidence; otherwise a disc of that angular radius and that irradiance,
 * sampled by cone and reachable by BSDF rays that escape the scene (MIS). */
typedef struct vt_directional_light_desc {
  float direction[3];
  float irradiance[3];
  float angular_radius;     /* radians, < pi/2 */
} vt_directional_light_desc;

/* Rectangle light (core RectAreaEmitter, emitters.ts:60-65): corner + [0,1]
 * edge_u + [0,1] edge_v, emitting `radiance` from the side edge_u x edge_v
 * faces; an analytic emitter like vt_disc_light_desc (uniform area sampling,
 * analytic BSDF-ray hits, never an occluder). */
typedef struct vt_rect_light_desc {
  float corner[3];
  float edge_u[3];
  float edge_v[3];
  float radiance[3];
} vt_rect_light_desc;

/* One placement of a mesh (core instanced-mesh / transform; the TLAS instance
 * of shared-bvh/src/tlas.ts:859).  With instances present every mesh is a
 * bottom-level prototype in its local space and is drawn only through
 * instances; emissive materials are not allowed on instances. */
typedef struct vt_instance_desc {
  uint32_t mesh;              /* index into vt_scene_desc.meshes */
  uint32_t material;          /* material of this placement */
  float local_to_world[16];   /* column-major, invertible */
} vt_instance_desc;

/* Scene (core Scene, core/src/scene/index.ts:42-46): primitives, emitters,
 * environment.  The environment is an equirectangular RGB image: row 0 at +y
 * (theta = acos(y)), column u = atan2(z, x) / 2pi + 0.5, so +x is the middle
 * column (the reference's environmentLookup, pt-webgpu/src/wgsl/pathTrace/
 * connect.wgsl.ts:139-142). */
typedef struct vt_scene_desc {
  const vt_mesh_desc* meshes;
  size_t mesh_count;
  const vt_instance_desc* instances;  /* NULL / 0: the meshes are world-space geometry */
  size_t instance_count;
  const vt_material_desc* materials;
  size_t material_count;
  const vt_point_light_desc* point_lights;
  size_t point_light_count;
  const float* environment_rgb;  /* width * height * 3 floats, or NULL */
  int32_t environment_width;
  int32_t environment_height;
  float environment_intensity;
  const vt_directional_light_desc* directional_lights;
  size_t directional_light_count;
  const vt_rect_light_desc* rect_lights;
  size_t rect_light_count;
  const vt_spot_light_desc* spot_lights;
  size_t spot_light_count;
  const vt_disc_light_desc* disc_lights;
  size_t disc_light_count;
  float environment_rotation_y;  /* CCW rotation of the environment about +y, radians (HdriEnvironment.rotationY) */
} vt_scene_desc;

/* Procedural sky (core ProceduralSkyEnvironment, core/src/scene/environment.ts:59-71):
 * the Preetham 1999 daylight model baked into an equirectangular RGB map that
 * is then given as the scene's environment (the reference bakes 256 x 128:
 * pt-webgpu/src/scene/environmentPacking.ts:221-270).  Host only. */
typedef struct vt_sky_desc {
  float sun_direction[3];   /* towards the sun (zero: +y) */
  float turbidity;          /* clamped to [1.5, 30]; the reference's default 2 */
  float rayleigh;           /* >= 0, default 1 (scales the sky) */
  float mie_coefficient;    /* >= 0, default 0.005 (haze) */
  float mie_directional_g;  /* Henyey-Greenstein g of the haze, default 0.8 */
  float intensity;          /* >= 0, default 1 */
} vt_sky_desc;
vt_status vt_bake_preetham_sky(const vt_sky_desc* sky, int32_t width, int32_t height, float* rgb,
                               size_t float_capacity);

/* Per-frame input (core FrameInput, core/src/frame.ts:91): camera matrices
 * column-major, viewport, sampling. */
typedef struct vt_frame_input {
  float view[16];
  float projection[16];
  int32_t width;
  int32_t height;
  uint32_t frame_seed;
  int32_t samples;   /* samples per pixel to add in this call */
  int32_t bounces;   /* 0 = the engine's max_bounces */
} vt_frame_input;

/* FrameOutput (core/src/frame.ts:376-421).  radiance_device is the engine's
 * accumulation buffer (float4 per pixel: rgb sum, sample count), valid until
 * the next render or reset. */
typedef struct vt_frame_output {
  int32_t kind;                 /* 0 rendered, 1 skipped (converged) */
  int32_t samples_accumulated;
  int32_t is_converged;
  int32_t width;
  int32_t height;
  const void* radiance_device;
} vt_frame_output;

typedef struct vt_engine_stats {
  uint64_t closest_rays;   /* extension rays traced since vt_create */
  uint64_t shadow_rays;    /* shadow rays traced since vt_create */
  double last_frame_ms;    /* device time of the last vt_render_frame */
  int64_t triangle_count;
  int64_t emitter_count;
} vt_engine_stats;

/* Device time per wavefront stage of one profiled frame. */
typedef struct vt_stage_times {
  double raygen_ms;
  double trace_closest_ms;
  double sort_ms;
  double shade_ms;
  double trace_shadow_ms;
  double resolve_ms;
  double accumulate_ms;
  double frame_ms;
  int32_t trace_closest_launches;
  int32_t trace_shadow_launches;
  double nrc_train_ms;     /* training wave, targets and optimiser steps (0 without the cache) */
  double nrc_query_ms;     /* cache inference of the render waves */
} vt_stage_times;

/* createPTEngine_WebGPU (pt-webgpu/src/index.ts:2363) */
vt_status vt_create(int32_t device, const vt_engine_options* options, vt_engine** out_engine);
/* Engine.setScene (core/src/engine/index.ts:120; pt-webgpu index.ts:1120).  Copies the scene. */
vt_status vt_set_scene(vt_engine* engine, const vt_scene_desc* scene);
/* Engine.renderFrame (index.ts:251; pt-webgpu index.ts:1817): adds input->samples samples. */
vt_status vt_render_frame(vt_engine* engine, const vt_frame_input* input, vt_frame_output* output);
/* vt_render_frame issuing the wave stages directly (no graph replay) with
 * events between them; the frame timings FrameStats.passTimings would carry
 * (core/src/engine/telemetry.ts:15-40). */
vt_status vt_profile_frame(vt_engine* engine, const vt_frame_input* input, vt_frame_output* output,
                           vt_stage_times* out_times);
/* Engine.captureFrame (index.ts:466): mean radiance, RGBA float32, row-major, top-left. */
vt_status vt_capture(vt_engine* engine, float* rgba, size_t float_capacity);
/* FP64 per-pixel mean and per-sample variance (requires oracle_accumulation);
 * 3 doubles per pixel each. */
vt_status vt_capture_moments(vt_engine* engine, double* mean_rgb, double* variance_rgb, size_t double_capacity);
/* Per-pixel shape of the sample distribution of luminance L = 0.2126 R +
 * 0.7152 G + 0.0722 B (requires oracle_accumulation; FP64 sums of L .. L^4):
 * 4 doubles per pixel -- mean, per-sample variance (n - 1), skewness
 * m3 / m2^1.5 and excess kurtosis m4 / m2^2 - 3 (central moments; 0 for a
 * constant pixel).  No reference counterpart: the unbiasedness tests judge
 * +-4 sigma exceedances by these. */
vt_status vt_capture_luminance_moments(vt_engine* engine, double* out, size_t double_capacity);

/* Auxiliary frame outputs, the textures the reference's kernel writes beside
 * the radiance (pt-webgpu/src/wgsl/pathTrace/kernel.wgsl.ts:936-960), as RGBA
 * float32, row-major, top-left, one float4 per pixel:
 *   VT_AUX_NORMAL_DEPTH  first-hit normal (facing the camera ray) * 0.5 + 0.5,
 *                        distance from the camera ray's origin; a miss
 *                        (0.5, 1, 0.5, 0)
 *   VT_AUX_ALBEDO        first-hit base colour, 1; a miss 0
 *   VT_AUX_MOTION        screen motion of the first-hit point in pixels,
 *                        (ndc(viewProj) - ndc(prevViewProj)) * 0.5 * (width, height),
 *                        0, 1 (kernelCore.wgsl.ts:28-42 projection); a miss (0, 0, 0, 1)
 *   VT_AUX_VARIANCE      per-pixel variance of the sample luminance (Rec. 709
 *                        weights) over every sample accumulated since the last
 *                        reset, max(0, E[L^2] - E[L]^2), 0, 0, 0
 * The first three hold the first hit of the last sample of the latest
 * rendered frame (the reference stores them per sample, so the last one
 * stays); before any frame all four are zero. */
#define VT_AUX_NORMAL_DEPTH 0
#define VT_AUX_ALBEDO 1
#define VT_AUX_MOTION 2
#define VT_AUX_VARIANCE 3
vt_status vt_capture_aux(vt_engine* engine, int32_t kind, float* rgba, size_t float_capacity);
/* FrameInput.prevViewMatrix / prevProjMatrix (frameParamsPacker.ts:225-229):
 * the camera of the previous frame, column-major like vt_frame_input, for the
 * motion output of the NEXT vt_render_frame / vt_profile_frame only; that
 * frame uses its own matrices where none were set (zero motion).  NULL
 * clears a pending pair. */
vt_status vt_set_previous_camera(vt_engine* engine, const float* prev_view, const float* prev_projection);

/* What this engine renders (Engine.capabilities, core/src/engine/capabilities.ts;
 * pt-webgpu/src/capabilities.ts): limits and the supported scene features, for
 * the binding's capability / support-manifest object. */
#define VT_EMITTER_POINT 1u
#define VT_EMITTER_SPOT 2u
#define VT_EMITTER_DIRECTIONAL 4u
#define VT_EMITTER_RECT_AREA 8u
#define VT_EMITTER_DISC_AREA 16u
#define VT_EMITTER_MESH_AREA 32u        /* emissive materials on meshes (single-level scenes) */
#define VT_EMITTER_ENVIRONMENT 64u      /* equirectangular RGB image */
#define VT_MATERIAL_FEATURE_BASE 1u     /* base colour, roughness, metallic, emission */
#define VT_MATERIAL_FEATURE_TRANSMISSION 2u  /* transmission, ior (smooth and rough) */
#define VT_MATERIAL_FEATURE_SPECULAR 4u      /* KHR specular factor */
#define VT_MATERIAL_FEATURE_DOUBLE_SIDED 8u
#define VT_MATERIAL_FEATURE_CAST_SHADOW 16u
#define VT_FEATURE_INSTANCES 1u         /* two-level scenes */
#define VT_FEATURE_INSTANCE_UPDATES 2u  /* vt_update_instances */
#define VT_FEATURE_RADIANCE_CACHE 4u    /* vt_set_nrc */
#define VT_FEATURE_BATCH 8u             /* vt_batch_* */
#define VT_FEATURE_PICK 16u             /* vt_pick (engines created with debug) */
#define VT_FEATURE_OUTPUT_CAPTURE 32u   /* vt_capture_output */
#define VT_FEATURE_FP64_MOMENTS 64u     /* vt_capture_moments (oracle_accumulation) */
#define VT_FEATURE_AUX_OUTPUTS 128u     /* vt_capture_aux, vt_set_previous_camera */
#define VT_FEATURE_MESH_UPDATES 256u    /* vt_update_mesh */
typedef struct vt_capabilities {
  int32_t max_bounces_limit;        /* largest max_bounces */
  int32_t max_samples_per_pixel;    /* this engine's accumulation cap */
  int32_t max_viewport;             /* pixels per side */
  uint32_t emitter_kinds;           /* VT_EMITTER_* bits */
  uint32_t material_features;       /* VT_MATERIAL_FEATURE_* bits */
  uint32_t features;                /* VT_FEATURE_* bits available on this engine */
} vt_capabilities;
vt_status vt_get_capabilities(const vt_engine* engine, vt_capabilities* capabilities);

/* New placements for the instances of the current two-level scene (moving
 * instances, changing their mesh or material), without rebuilding any
 * bottom-level tree: refitTlasTransforms (shared-bvh/src/scenePack.ts:1310,
 * refitTlas tlas.ts:990-1012) with rebuild 0 -- the top level keeps its
 * topology and takes the new bounds -- or rebuildTlasReuseBlas
 * (scenePack.ts:1635) with rebuild 1 -- a new binned-SAH top level.  The
 * instance count must equal the scene's (VT_ERR_INVALID_ARGUMENT otherwise;
 * VT_ERR_STATE without an instanced scene).  Clears the accumulation. */
vt_status vt_update_instances(vt_engine* engine, const vt_instance_desc* instances, size_t count, int32_t rebuild);
/* rebuildPrimitiveBlas (shared-bvh/src/scenePack.ts:1763; splices :1006-1100):
 * new vertices / triangles / material for mesh `mesh_index` of a scene with
 * instances.  Its bottom-level tree is rebuilt and spliced in place (later
 * meshes rebased when its size changed), then the top level is refitted over
 * the instances' new bounds, or rebuilt when `rebuild` is 1.  The other meshes'
 * trees are untouched; accumulation restarts.  A scene without instances has
 * one flat tree: VT_ERR_STATE (set the scene again). */
vt_status vt_update_mesh(vt_engine* engine, size_t mesh_index, const vt_mesh_desc* mesh, int32_t rebuild);

/* captureFrame({colorSpace: 'output'}) (pt-webgpu/src/index.ts:2004-2033): the
 * present pass (pt-webgpu/src/wgsl/present.wgsl.ts; operators of
 * shared-samplers/src/wgsl/tonemap.wgsl.ts) applied to the accumulated mean:
 * exposure, tonemap, then the sRGB OETF.  The reference's defaults are ACES,
 * exposure 1, sRGB. */
typedef struct vt_present_options {
  int32_t tonemap;          /* 0 ACES filmic, 1 AgX, 2 Reinhard, 3 clamp to [0, 1], 4 none */
  float exposure;           /* linear multiplier, > 0 */
  int32_t srgb;             /* 1 apply the sRGB OETF (outputColorSpace 'srgb'), 0 keep linear */
} vt_present_options;
vt_status vt_capture_output(vt_engine* engine, const vt_present_options* options, float* rgba, size_t float_capacity);
/* Engine.debug.pickPrimitive (engine/debug.ts:33-35; pickPrimitiveCpu.ts:674):
 * under pixel (x, y) of the last frame's camera: the instance index in a
 * scene with instances, else the source triangle index; -1 on a miss. */
vt_status vt_pick(vt_engine* engine, float x, float y, int32_t* out_triangle);

/* The current scene's top-level tree (scenes with instances; VT_ERR_STATE
 * otherwise) in the reference layout of vt_tlas_build -- the tlasNodes and
 * tlasInstanceIndices buffers of packSceneFromCore (scenePack.ts:1104-1310). */
/* The engine's device node array (20 words per wide node: bottom levels, then
 * the top level) and triangle records (16 floats each) as they are on the GPU,
 * copied back (no reference counterpart; for comparing the GPU and host scene
 * builds).  Null buffers: only the sizes are written. */
vt_status vt_engine_export_scene(const vt_engine* engine, uint32_t* node_words, size_t word_capacity, float* records,
                                 size_t float_capacity, size_t* out_words, size_t* out_floats);

vt_status vt_engine_export_tlas(const vt_engine* engine, uint32_t* nodes, size_t node_word_capacity,
                                uint32_t* instance_indices, size_t instance_capacity, size_t* node_count);
/* Closest hit of host rays against the engine's scene (vt_bvh_trace_closest
 * on a whole scene, two-level when it has instances).  hits[i].prim is the
 * triangle index within its mesh in a scene with instances, else the index over
 * all meshes in order (-1 on a miss); t and (u, v) as vt_hit.  instances[i]
 * receives the instance index, or -1 on a miss or without instances (may be NULL).
 * No reference counterpart: the WebGPU engine exposes no ray query. */
vt_status vt_trace_rays(vt_engine* engine, const vt_ray* rays, size_t n, vt_hit* hits, int32_t* instances);
/* Engine.reset (pt-webgpu index.ts:2052): clears the accumulation. */
/*
 * Failure-detection hook (engines created with debug = 1; no reference
 * counterpart).  Bounds the first wait of each bounded device wait -- the
 * radiance-cache kernels' waits for their tensor-core products and the
 * traversal's wait for its shared-memory staging copy -- to `cycles` clocks;
 * 0 restores the default of about a second.  An expired wait makes the kernel
 * record it, wait for its own copies or products in flight under the full
 * limit, free its tensor memory and return, so vt_render_frame reports
 * VT_ERR_TIMEOUT (cache) or VT_ERR_BUILD (staging) and the engine stays usable.
 */
vt_status vt_engine_set_wait_limit(vt_engine* engine, int64_t cycles);

/*
 * Failure-injection hook (tests; the reference's FailureDevice of
 * pt-webgpu/src/__tests__/transactionalResourceReplacement.test.ts).  The nth
 * device allocation the library makes on the calling thread from now on fails
 * as an out-of-memory cudaMalloc would (VT_ERR_OUT_OF_MEMORY, "injected device
 * allocation failure"); 0 disarms.  vt_set_scene is transactional: a failure at
 * any stage leaves the engine's previous scene in place.
 */
vt_status vt_debug_fail_device_allocation(int64_t nth);

vt_status vt_reset(vt_engine* engine);
vt_status vt_engine_get_stats(const vt_engine* engine, vt_engine_stats* out_stats);
/* Engine.dispose */
vt_status vt_destroy(vt_engine* engine);

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

/* ------------------------------------------------------------------ */
/* Neural radiance cache (walkaround-hybrid/src/neural/nrc/)            */
/* ------------------------------------------------------------------ */

typedef struct vt_nrc vt_nrc;

/* NrcConfig (nrcSubsystem.ts:116-132) with the hash grid and optimiser
 * settings that matter here.  Fixed: 2 features per entry, 64-wide MLP with
 * 5 hidden ReLU layers and 3 linear outputs, fp16 weights and activations with
 * fp32 accumulation, Adam beta 0.9 / 0.999, eps 1e-8. */
typedef struct vt_nrc_config {
  int32_t levels;            /* hash-grid levels, 1..16 */
  int32_t log2_table_size;   /* entries per level = 2^log2_table_size, 4..24 */
  float base_resolution;     /* level l resolution = floor(base * growth^l) */
  float growth;
  float learning_rate;       /* MLP */
  float table_learning_rate; /* hash grid */
  float aabb_min[3];         /* positions are normalised into this box */
  float aabb_max[3];
  uint32_t seed;             /* weight / table initialisation */
  int32_t infer_tiles;       /* query tiles of 128 in flight per inference CTA, one per warpgroup (the MLP
                                tile: more tiles keep more table gathers in flight and overlap one tile's
                                gathers with another's tensor-core products), 1..4; 0 = the default (4) */
} vt_nrc_config;

/* Features of one cache query or training sample, 16 floats:
 * position xyz, outgoing direction xyz (unit), normal xyz, roughness,
 * diffuse albedo rgb, specular albedo rgb.  A training sample appends the
 * target radiance rgb and one unused float (20 floats). */
#define VT_NRC_RECORD_FLOATS 16
#define VT_NRC_SAMPLE_FLOATS 20
#define VT_NRC_WEIGHT_COUNT (6 * 64 * 64) /* [layer][out][in]; layer 5 uses rows 0..2 */

/* NrcSubsystem construction (nrcSubsystem.ts resolveNrcConfig + allocation). */
vt_status vt_nrc_create(int32_t device, const vt_nrc_config* config, vt_nrc** out);
vt_status vt_nrc_destroy(vt_nrc* nrc);
/* Cache query (nrcQuery.wgsl.ts): rgb[3 i..] = network(records[16 i..]), host arrays. */
vt_status vt_nrc_query(vt_nrc* nrc, const float* records, size_t n, float* rgb);
/* One optimiser step on n samples (fusedMlpTrainer.ts train step + the table
 * Adam of hashGridTableTrainer.ts); *loss receives the mean relative-L2 loss
 * before the step (may be NULL). */
vt_status vt_nrc_train(vt_nrc* nrc, const float* samples, size_t n, float* loss);
/* Gradients of the mean loss over n samples without an update (the
 * nrcEncodeBackwardHarness.ts / fusedMlpHarness.ts check path).  grad_table
 * receives levels * 2^log2 * 2 floats (may be NULL). */
vt_status vt_nrc_gradients(vt_nrc* nrc, const float* samples, size_t n, float* grad_weights, float* grad_table,
                           float* loss);
/* NrcStateSnapshot (nrcStateSnapshot.ts): f32 master weights and table. */
vt_status vt_nrc_get_params(vt_nrc* nrc, float* weights, float* table);
/* Replaces the parameters and clears the optimiser state. */
vt_status vt_nrc_set_params(vt_nrc* nrc, const float* weights, const float* table);
/* Device-pointer forms, enqueued on `cuda_stream` (NULL: the legacy default
 * stream); records / samples / rgb are device arrays with the layouts above.
 * No reference counterpart (the WebGPU subsystem binds its own buffers). */
vt_status vt_nrc_query_device(vt_nrc* nrc, const float* d_records, size_t n, float* d_rgb, void* cuda_stream);
vt_status vt_nrc_train_device(vt_nrc* nrc, const float* d_samples, size_t n, void* cuda_stream);

/* Path tracing with the cache (NrcSubsystem driven by the engine; Mueller et
 * al. 2021 as the reference runs it): every frame a training wave of plain
 * paths from random pixels records each vertex's features and the radiance
 * gathered after it (targets), `train_steps` Adam steps of `train_batch`
 * samples follow, then the render waves trace `prefix_bounces` bounces and end
 * each path in a cache query at the next vertex.  For the first
 * `warmup_frames` frames the render waves are plain path tracing. */
typedef struct vt_nrc_render_options {
  int32_t enabled;          /* 0: plain path tracing */
  int32_t prefix_bounces;   /* bounces before the query (1 queries the second vertex); 0: spread
                               termination (spreadTermination.ts): query at the first vertex k >= 2
                               whose accumulated spread a(x_k) exceeds spread_c * a0 */
  int32_t train_steps;      /* optimiser steps per frame (4) */
  int32_t train_batch;      /* samples per step (65536) */
  int32_t train_paths;      /* training paths per frame (0: train_steps * train_batch / 2) */
  int32_t warmup_frames;    /* plain frames while the cache warms up */
  vt_nrc_config cache;      /* aabb is replaced by the scene's bounds */
  float fallback_error;     /* > 0: screen tiles whose cache error estimate (EMA of the relative
                               luminance bias at the query vertex) exceeds this keep path tracing */
  int32_t fallback_tile;    /* tile edge in pixels (0: 16) */
  float spread_c;           /* spread termination constant (0: 0.01, the paper's c) */
} vt_nrc_render_options;

vt_status vt_set_nrc(vt_engine* engine, const vt_nrc_render_options* options);

/* ------------------------------------------------------------------ */
/* Batch: many scenes in one launch sequence                            */
/* ------------------------------------------------------------------ */
/* No reference counterpart (the WebGPU engine renders one scene per engine):
 * scenes of uneven size and resolution share every wave, so small frames do
 * not leave the GPU idle.  Paths of all scenes form one index space consumed
 * wave by wave through a device cursor; traversal takes a per-ray root; the
 * whole frame (all waves) is one CUDA graph.  Scenes must be single-level. */

typedef struct vt_batch vt_batch;

typedef struct vt_batch_stats {
  double frame_ms;            /* device time of the batch frame (all scenes) */
  uint64_t closest_rays;      /* extension rays traced by the frame */
  uint64_t shadow_rays;
  int32_t waves;
  int32_t kernel_launches;    /* kernels in the frame's graph */
} vt_batch_stats;

/* Launch-shape knobs, chosen by vt_batch_autotune or set directly. */
typedef struct vt_tuning {
  int32_t wave_paths;         /* paths per wave */
  int32_t sort_by_material;   /* 1 sort shading work by BSDF family, 0 not */
  int32_t trace_blocks_per_sm;/* persistent traversal CTAs per SM (0: occupancy limit) */
  int32_t stage_hot_nodes;    /* 1: each traversal CTA first copies the top of the tree (root,
                                 children, grandchildren) into shared memory with one bulk copy;
                                 0: every node read goes through L1/L2.  A batch takes 0 only
                                 (its launches carry one root per ray). */
  int32_t sort_rays;          /* trace order: 0 queue order; each closest-hit queue from bounce 1 on by
                                 1 direction octant (a counting sort by the signs of the direction) or
                                 2 the 2^6-per-axis cell of the scene box the ray starts in, then its
                                 octant (the spatial order of vt_bvh_set_trace_order); 3 each shadow
                                 queue by its 2^4-per-axis origin cell and octant (engines only;
                                 batches take 0 or 1) */
  int32_t nrc_infer_tiles;    /* engines rendering with the radiance cache: query tiles of 128 in flight per
                                 inference CTA (vt_nrc_config.infer_tiles, 1..4); 0 = unchanged */
} vt_tuning;

vt_status vt_batch_create(int32_t device, const vt_engine_options* options, vt_batch** out);
/* One frame per scene: frames[i].samples samples at frames[i].width x height with
 * frames[i].bounces (0: options.max_bounces) through the camera of frames[i]. */
vt_status vt_batch_set_scenes(vt_batch* batch, const vt_scene_desc* scenes, const vt_frame_input* frames,
                              size_t count);
/* Renders every scene's frame from a cleared accumulation. */
vt_status vt_batch_render(vt_batch* batch, vt_batch_stats* stats);
vt_status vt_batch_capture(vt_batch* batch, size_t index, float* rgba, size_t float_capacity);
vt_status vt_batch_set_tuning(vt_batch* batch, const vt_tuning* tuning);
vt_status vt_batch_get_tuning(const vt_batch* batch, vt_tuning* tuning);
/* The project's autotuner: times candidate launch shapes on this batch (each
 * candidate renders the batch once) and keeps the fastest; `report` receives
 * up to `report_capacity` (tuning, frame_ms) pairs tried. */
typedef struct vt_tuning_trial {
  vt_tuning tuning;
  double frame_ms;
} vt_tuning_trial;
vt_status vt_batch_autotune(vt_batch* batch, vt_tuning_trial* report, size_t report_capacity, size_t* report_count);
vt_status vt_batch_destroy(vt_batch* batch);

/* The autotuner for a single-scene engine: renders `frame` (from a cleared
 * accumulation) once per candidate launch shape after a warm-up and keeps the
 * fastest; later frames use it.  No reference counterpart. */
vt_status vt_engine_autotune(vt_engine* engine, const vt_frame_input* frame, vt_tuning_trial* report,
                             size_t report_capacity, size_t* report_count);
vt_status vt_engine_get_tuning(const vt_engine* engine, vt_tuning* tuning);
/* BVH-shape autotuner of a single-scene engine (no reference counterpart):
 * rebuilds `scene`'s trees for candidate shapes -- triangles per leaf (1..4)
 * at the current width, then collapse width (children per wide node, 8, 6, 4)
 * at the best leaf size -- renders `frame` with each after a warm-up and keeps
 * the fastest, a candidate replacing the current shape only when it is 0.5 %
 * faster (the engine ends with `scene` set in that shape and a cleared
 * accumulation).  The scene is read as vt_set_scene reads it. */
typedef struct vt_bvh_shape_trial {
  int32_t bvh_width;
  int32_t bvh_max_leaf;
  double frame_ms;
} vt_bvh_shape_trial;
vt_status vt_engine_autotune_bvh(vt_engine* engine, const vt_scene_desc* scene, const vt_frame_input* frame,
                                 vt_bvh_shape_trial* report, size_t report_capacity, size_t* report_count);
/* Sets the launch shape directly (e.g. one found by an earlier autotune). */
vt_status vt_engine_set_tuning(vt_engine* engine, const vt_tuning* tuning);

#ifdef __cplusplus
}
#endif

#endif /* VITRUM_PT_H */
