// api_noalloc.cu -- closest-hit query for callers that cannot allocate device memory.
//
// Who needs it: hosts that hand this library a fixed memory budget and forbid
// any further driver allocation once they are running (an embedding renderer
// or plugin host with a pre-reserved arena), and host code that passes plain
// host arrays -- the Node addon's typed arrays -- on a path where a
// cudaMalloc may not happen.  The ordinary host-buffer call
// vt_bvh_trace_closest grows per-object staging with cudaMalloc whenever a
// batch is larger than any before it; this call never does.
//
// How: its scratch -- the ray counter and status word the persistent
// traversal kernel needs, plus device staging for the rays and hit records --
// is one file-scope __device__ array of kNoAllocScratchBytes (3 MiB + 256 B),
// which every GPU that loads the library holds until the process exits.
// Host code cannot use the array's name as a device address; every call looks
// the address up with cudaGetSymbolAddress while the BVH's device is current
// (a lookup, once the module is loaded), so nothing goes stale after a
// cudaDeviceReset.  The first call on each device is different: with lazy
// module loading (the CUDA 12 default) it loads this file's module, which may
// allocate in the driver once.  Make that first call during set-up -- a call
// with n == 0 does only this and traces nothing -- and before any CUDA stream
// capture begins.  All calls share the one array and it keeps the last
// call's contents: the status word is cleared here and the counter by the
// kernel launcher, and calls that overlap on the GPU (other threads, other
// streams) race on the array.  Each call runs on the legacy default stream
// and blocks until the hit records are in host memory.
#include <cuda_runtime.h>

#include <string>

#include "bvh_object.h"
#include "traverse.h"
#include "vt_common.h"

namespace {

constexpr size_t kNoAllocMaxRays = 65536;  // rays per call
constexpr size_t kHeaderBytes = 256;       // ray counter (8 B) + status word (4 B), padded
constexpr size_t kNoAllocScratchBytes = kHeaderBytes + kNoAllocMaxRays * (sizeof(vt_ray) + sizeof(vt_hit));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch on the current device.
unsigned char* scratch_address() {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr)
    vt::fail(VT_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
  return static_cast<unsigned char*>(p);
}

}  // namespace

extern "C" vt_status vt_bvh_trace_closest_noalloc(const vt_bvh* bvh, const vt_ray* rays, size_t n, vt_hit* hits) {
  return vt::guard([&] {
    if (!bvh) vt::fail(VT_ERR_INVALID_ARGUMENT, "bvh is null");
    if (n && (!rays || !hits)) vt::fail(VT_ERR_INVALID_ARGUMENT, "rays and hits must be non-null");
    if (n > kNoAllocMaxRays)
      vt::fail(VT_ERR_RANGE, "vt_bvh_trace_closest_noalloc takes at most " + std::to_string(kNoAllocMaxRays) +
                                 " rays per call, got " + std::to_string(n) + "; split the batch");
    vt::DeviceScope ds(bvh->device);
    unsigned char* base = scratch_address();
    if (n == 0) return;  // set-up call: the module is loaded and the address resolved
    auto* counter = reinterpret_cast<unsigned long long*>(base);
    auto* status = reinterpret_cast<int*>(base + 8);
    auto* d_rays = reinterpret_cast<float4*>(base + kHeaderBytes);
    auto* d_hits = reinterpret_cast<int4*>(base + kHeaderBytes + kNoAllocMaxRays * sizeof(vt_ray));
    VT_CUDA(cudaMemset(status, 0, sizeof(int)));
    VT_CUDA(cudaMemcpy(d_rays, rays, n * sizeof(vt_ray), cudaMemcpyHostToDevice));
    vt::TraceArgs a;
    a.nodes = bvh->nodes.ptr;
    a.tris = bvh->tris.ptr;
    a.rays = d_rays;
    a.n = n;
    a.hits = d_hits;
    a.status = status;
    a.counter = counter;
    a.stack_depth = 2 * bvh->wide_depth + 2;
    a.node_count = bvh->nodes.count / 5;
    vt::launch_trace_closest(a, 0);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaMemcpy(hits, d_hits, n * sizeof(vt_hit), cudaMemcpyDeviceToHost));
    int st = 0;
    VT_CUDA(cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) vt::fail(VT_ERR_BUILD, vt::trace_status_message(st));
  });
}
