// Per-device library context (the object behind zk_ctx).
#pragma once
#include <cuda_runtime.h>

#include <mutex>

#include "msm.hpp"
#include "ntt.hpp"
#include "profile.hpp"
#include "runtime.hpp"

namespace zk {

// Buffers and streams of one in-flight proof (reused across proofs).
struct ProveWs {
  static constexpr int kStreams = 5;  // 0: witness/SpMV/H/MSM_H, 1: A, 2: B2, 3: C, 4: B1
  bool ready = false;
  int nstreams = kStreams;
  cudaStream_t st[kStreams] = {};
  cudaEvent_t ev_we = nullptr, ev_begin = nullptr;
  cudaEvent_t ev_done[kStreams] = {};
  DeviceBuffer we, aw, bw, cw, h;
  DeviceBuffer msm[kStreams];
  PinnedBuffer win[kStreams];
  void init();
  ~ProveWs();
};

}  // namespace zk

struct zk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  zk::NttTables ntt;
  zk::DeviceBuffer ntt_scratch;
  zk::DeviceBuffer msm_scratch;
  zk::MsmConfig msm_cfg[2];
  zk::ProveWs ws;
  zk::Stager stager;
  zk::Profiler prof;
  bool profiling = false;
  bool own_stream = true;  // false after zk_ctx_set_stream
  bool is_default = false;
};

namespace zk {

// Per-device default context (created on first use).
zk_ctx* default_ctx();
// Makes ctx's device current for the calling thread.
void use_device(zk_ctx* ctx);

}  // namespace zk
