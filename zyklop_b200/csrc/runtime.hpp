// Runtime plumbing shared by the CUDA library: status codes, error
// propagation, device buffers and per-context state.
//
// The reference exits the process on any CUDA error (G16_CUDA_CHECK,
// src/groth16.cu:105-112; NTT_CUDA_CHECK, include/ntt_bn254.cuh:38-45;
// G1_CUDA_CHECK, include/msm_g1.cuh:62-69).  Here every failure becomes a C++
// exception inside the library and a status code plus a thread-local message
// at the C ABI (include/zyklop_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/zyklop_b200.h"

namespace zk {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);

#define ZK_CUDA(call)                                                  \
  do {                                                                 \
    cudaError_t zk_e_ = (call);                                        \
    if (zk_e_ != cudaSuccess) ::zk::throw_cuda(zk_e_, #call, __FILE__, __LINE__); \
  } while (0)

#define ZK_CHECK_LAUNCH() ZK_CUDA(cudaGetLastError())

void count_launch(int n);
// after every kernel launch: counts it and surfaces launch errors
#define ZK_LAUNCHED()            \
  do {                           \
    ::zk::count_launch(1);       \
    ZK_CHECK_LAUNCH();           \
  } while (0)

#define ZK_REQUIRE(cond, code, msg)                         \
  do {                                                      \
    if (!(cond)) throw ::zk::Error((code), (msg));          \
  } while (0)

void set_last_error(int code, const char* msg);

// Free device memory on the current device, counting blocks the library's
// pool holds for reuse.
size_t device_free_bytes();
// Device / pinned-host allocations the library has made in this process.
void alloc_stats(uint64_t* dev_allocs, uint64_t* dev_bytes, uint64_t* host_allocs);
// Reserved and used bytes of the library's memory pool on `dev` (false if
// the device has no pool).
bool pool_usage(int dev, uint64_t* reserved, uint64_t* used);
// Returns the pool's unused blocks on the current device to the driver.
void release_cached_memory();

// Growable device allocation.  ensure() keeps the old allocation when it is
// large enough; growing frees the old one first (callers synchronize the
// streams that used it before growing).
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t cap = 0;
  int dev = 0;          // device the block lives on
  bool pooled = false;  // from the device's stream-ordered pool
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { release(); }
  void ensure(size_t bytes);
  void release();
  template <class T>
  T* as() const { return reinterpret_cast<T*>(ptr); }
};

// Growable page-locked host allocation (for asynchronous copies).
struct PinnedBuffer {
  void* ptr = nullptr;
  size_t cap = 0;
  PinnedBuffer() = default;
  PinnedBuffer(const PinnedBuffer&) = delete;
  PinnedBuffer& operator=(const PinnedBuffer&) = delete;
  ~PinnedBuffer() { release(); }
  void ensure(size_t bytes);
  void release();
  template <class T>
  T* as() const { return reinterpret_cast<T*>(ptr); }
};

// Host -> device copy of pageable memory (a mapped file, a caller buffer)
// through two pinned staging buffers: the CPU fills one chunk (with several
// threads) while the DMA engine drains the other.  Blocks until the source
// may be released; the device copy completes in stream order.
struct Stager {
  static constexpr size_t kChunk = size_t(32) << 20;
  PinnedBuffer buf[2];
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~Stager();
  void upload(void* dst, const void* src, size_t bytes, cudaStream_t st);
};

// Bump-pointer carve-out of a DeviceBuffer (256-byte aligned slices).
struct Carver {
  char* base;
  size_t off = 0;
  explicit Carver(void* b) : base(reinterpret_cast<char*>(b)) {}
  template <class T>
  T* take(size_t count) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
};

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int device_sm_count();

}  // namespace zk
