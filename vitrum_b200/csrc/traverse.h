// traverse.h -- launchers of the traversal kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/vitrum_pt.h"

namespace vt {

struct TraceArgs {
  const uint4* nodes = nullptr;   // 8-wide nodes, 5 uint4 each
  const float4* tris = nullptr;   // 3 float4 per triangle
  const float4* rays = nullptr;   // 2 float4 per ray (vt_ray)
  size_t n = 0;
  int4* hits = nullptr;           // vt_hit per ray (closest)
  uint8_t* occluded = nullptr;    // 1 byte per ray (any)
  int* status = nullptr;          // device word, bit 0 = stack capacity exceeded
  int stack_depth = 64;           // wide-tree depth bound
  unsigned long long* counter = nullptr;  // device word: next unclaimed ray (reset per launch)
  const uint32_t* n_dev = nullptr;  // when set, the ray count is read from this device word (n = capacity)
  const float4* insts = nullptr;    // two-level: instance records (4 float4 each); nodes[root] is the TLAS root
  uint32_t root = 0;                // first node to expand
  const float4* inst_table = nullptr;  // records by instance index: refinement of instance hits, and the
                                       // material id a closest hit of the path tracer carries
  const uint32_t* roots = nullptr;    // optional per-ray root node (rays of several scenes in one launch)
  const float4* inst_l2w = nullptr;   // refinement of instance hits: local-to-world rows (3 per instance)
  int* inst_out = nullptr;          // optional: instance index per ray (-1 miss / single level)
  int blocks_per_sm = 0;            // persistent CTAs per SM (0: the occupancy limit)
  size_t node_count = 0;            // nodes in `nodes` (0: unknown, no shared-memory staging)
  bool stage_nodes = false;         // each CTA copies the top of the tree below `root` into shared memory
  long long stage_wait_cycles = 0;  // clocks a CTA waits for that copy before it gives up (0: about a second)
  const uint32_t* order = nullptr;  // optional trace order: slot i traces ray order[i] (results stay at that ray)
};

// Bits of the device status word a traversal launch sets.
enum : int {
  kTraceStackOverflow = 1,  // a group did not fit the stack (the ray was finished without it)
  kTraceStagingWait = 2,    // the shared-memory node staging did not complete in time (global reads used)
};
const char* trace_status_message(int status);

void launch_trace_closest(const TraceArgs& a, cudaStream_t s);
// Closest hit without the refinement pass: hits hold (triangle record, watertight t bits, 0, 0).
void launch_trace_closest_records(const TraceArgs& a, cudaStream_t s);
void launch_trace_any(const TraceArgs& a, cudaStream_t s);
void launch_watertight_eval(const float* cases, size_t n, vt_watertight_result* out, cudaStream_t s);

}  // namespace vt
