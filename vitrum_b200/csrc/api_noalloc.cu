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
// Host code cannot use the array's name as a device address; the first call
// on each device looks the address up with cudaGetSymbolAddress while that
// device is current and caches it.  That first call must therefore come
// before any CUDA stream capture begins.  All calls share the one array and
// it keeps the last call's contents: the status word is cleared here and the
// counter by the kernel launcher, and calls that overlap on the GPU (other
// threads, other streams) race on the array.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "bvh_object.h"
#include "traverse.h"
#include "vt_common.h"

namespace {

constexpr size_t kNoAllocMaxRays = 65536;  // rays per call
constexpr size_t kHeaderBytes = 256;       // ray counter (8 B) + status word (4 B), padded
constexpr size_t kNoAllocScratchBytes = kHeaderBytes + kNoAllocMaxRays * (sizeof(vt_ray) + sizeof(vt_hit));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 128;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (which must be current).
unsigned char* scratch_for(int device) {
  if (device < 0 || device >= kMaxDevices) vt::fail(VT_ERR_RANGE, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      vt::fail(VT_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[device] = p;
  }
  return static_cast<unsigned char*>(g_scratch_addr[device]);
}

}  // namespace

extern "C" vt_status vt_bvh_trace_closest_noalloc(const vt_bvh* bvh, const vt_ray* rays, size_t n, vt_hit* hits) {
  return vt::guard([&] {
    if (!bvh) vt::fail(VT_ERR_INVALID_ARGUMENT, "bvh is null");
    if (n && (!rays || !hits)) vt::fail(VT_ERR_INVALID_ARGUMENT, "rays and hits must be non-null");
    if (n > kNoAllocMaxRays)
      vt::fail(VT_ERR_RANGE, "vt_bvh_trace_closest_noalloc takes at most " + std::to_string(kNoAllocMaxRays) +
                                 " rays per call, got " + std::to_string(n) + "; split the batch");
    if (n == 0) return;
    vt::DeviceScope ds(bvh->device);
    unsigned char* base = scratch_for(bvh->device);
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
