// Per-device library context (the object behind zk_ctx).
#pragma once
#include <cuda_runtime.h>

#include <mutex>

#include "msm.hpp"
#include "ntt.hpp"
#include "runtime.hpp"

struct zk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  zk::NttTables ntt;
  zk::DeviceBuffer ntt_scratch;
  zk::DeviceBuffer msm_scratch;
  zk::MsmConfig msm_cfg[2];
  bool is_default = false;
};

namespace zk {

// Per-device default context (created on first use).
zk_ctx* default_ctx();
// Makes ctx's device current for the calling thread.
void use_device(zk_ctx* ctx);

}  // namespace zk
