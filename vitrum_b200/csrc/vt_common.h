// vt_common.h -- shared host-side helpers of libvitrum_pt: error latching,
// CUDA checks and the device buffer RAII used by every C-ABI object.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/vitrum_pt.h"

namespace vt {

// Exception carrying a vt_status; caught at the C-ABI boundary.
struct Error : std::runtime_error {
  vt_status status;
  Error(vt_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string& msg);
void clear_last_error();

[[noreturn]] inline void fail(vt_status s, const std::string& m) { throw Error(s, m); }

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    vt_status s = (e == cudaErrorMemoryAllocation) ? VT_ERR_OUT_OF_MEMORY : VT_ERR_CUDA;
    fail(s, std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define VT_CUDA(call) ::vt::cuda_check((call), #call)

// Runs `fn` and converts exceptions into a vt_status plus thread-local message.
template <class F>
vt_status guard(F&& fn) {
  try {
    clear_last_error();
    fn();
    return VT_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return VT_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return VT_ERR_INVALID_ARGUMENT;
  } catch (...) {
    set_last_error("unknown error");
    return VT_ERR_INVALID_ARGUMENT;
  }
}

// Failure-injection hook for tests (vt_debug_fail_device_allocation): the
// nth DeviceBuffer allocation on this thread from the arming on fails as if
// cudaMalloc had run out of memory.  Returns true for the allocation that must fail.
void arm_allocation_failure(long long nth);
bool injected_allocation_failure();

// Owning device allocation (cudaMalloc / cudaFree), move-only.
template <class T>
struct DeviceBuffer {
  T* ptr = nullptr;
  size_t count = 0;
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t n) { resize(n); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), count(o.count) { o.ptr = nullptr; o.count = 0; }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) { release(); ptr = o.ptr; count = o.count; o.ptr = nullptr; o.count = 0; }
    return *this;
  }
  ~DeviceBuffer() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    count = 0;
  }
  void resize(size_t n) {
    if (n == count) return;
    release();
    if (n) {
      if (injected_allocation_failure()) fail(VT_ERR_OUT_OF_MEMORY, "injected device allocation failure");
      VT_CUDA(cudaMalloc(&ptr, n * sizeof(T)));
    }
    count = n;
  }
  size_t bytes() const { return count * sizeof(T); }
};

// Scratch device memory from the stream-ordered pool: allocation and release
// are enqueued on the stream (no device-wide synchronisation), and released
// blocks stay in the current device's pool (up to 1 GiB kept) for the next
// build's scratch.
void configure_scratch_pool();
template <class T>
struct ScratchBuffer {
  T* ptr = nullptr;
  size_t count = 0;
  cudaStream_t stream = nullptr;
  ScratchBuffer() = default;
  ScratchBuffer(size_t n, cudaStream_t s) { resize(n, s); }
  ScratchBuffer(const ScratchBuffer&) = delete;
  ScratchBuffer& operator=(const ScratchBuffer&) = delete;
  ScratchBuffer(ScratchBuffer&& o) noexcept : ptr(o.ptr), count(o.count), stream(o.stream) {
    o.ptr = nullptr;
    o.count = 0;
  }
  ScratchBuffer& operator=(ScratchBuffer&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      count = o.count;
      stream = o.stream;
      o.ptr = nullptr;
      o.count = 0;
    }
    return *this;
  }
  ~ScratchBuffer() { release(); }
  void release() {
    if (ptr) cudaFreeAsync(ptr, stream);
    ptr = nullptr;
    count = 0;
  }
  void resize(size_t n, cudaStream_t s) {
    release();
    stream = s;
    if (n) {
      if (injected_allocation_failure()) fail(VT_ERR_OUT_OF_MEMORY, "injected device allocation failure");
      configure_scratch_pool();
      VT_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ptr), n * sizeof(T), s));
    }
    count = n;
  }
  size_t bytes() const { return count * sizeof(T); }
};

// Sets the current device for the lifetime of the scope and restores it.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    VT_CUDA(cudaGetDevice(&prev));
    if (prev != dev) VT_CUDA(cudaSetDevice(dev));
  }
  ~DeviceScope() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace vt
