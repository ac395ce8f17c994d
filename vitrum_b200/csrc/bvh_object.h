// bvh_object.h -- the vt_bvh object behind the C ABI handle.
#pragma once

#include <vector>

#include <cuda_runtime.h>

#include <cstdint>

#include "bvh_host.h"
#include "vt_common.h"

struct vt_bvh {
  int device = 0;
  vt::BuildOptions opts;
  vt::BinaryBvhHost binary;              // binary tree in the reference layout (for export)
  vt::DeviceBuffer<uint4> nodes;         // 8-wide nodes
  vt::DeviceBuffer<float4> tris;         // triangle records
  vt::DeviceBuffer<int> status;          // traversal status word
  vt::DeviceBuffer<unsigned long long> counter;  // persistent-kernel ray counter (calls on one bvh are serialised)
  std::vector<uint32_t> wide_host_nodes;  // the published 8-wide nodes and records (host copies, for export)
  std::vector<float> wide_host_recs;
  int64_t ntri = 0;
  int64_t wide_count = 0;
  int wide_depth = 0;
  double build_ms = 0.0;
  // staging for the host-buffer entry points
  vt::DeviceBuffer<float4> rays_scratch;
  vt::DeviceBuffer<int4> hits_scratch;
  vt::DeviceBuffer<uint8_t> occ_scratch;
  // two streams and ray counters for the chunked host-buffer queries (created on first use)
  cudaStream_t copy_streams[2] = {nullptr, nullptr};
  vt::DeviceBuffer<unsigned long long> chunk_counters;
  // spatial trace order of query batches (vt_bvh_set_trace_order): Morton bits
  // per axis (0: input order), and its scratch, grown on demand: bucket keys and
  // the permutation (one word per ray each), two bucket arrays (one per stream)
  int order_bits = 0;
  vt::DeviceBuffer<uint32_t> order_keys, order_idx, order_counts;
  ~vt_bvh() {
    for (cudaStream_t& s : copy_streams)
      if (s) cudaStreamDestroy(s);
  }
};
