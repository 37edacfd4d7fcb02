// Runtime plumbing (see runtime.hpp).
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstring>
#include <string>

#include "runtime.hpp"

namespace zk {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(int code, const char* msg) {
  (void)code;
  g_last_error = msg ? msg : "";
}

const char* last_error() { return g_last_error.c_str(); }

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what,
           file, line);
  throw Error(e == cudaErrorMemoryAllocation ? ZK_ENOMEM : ZK_ECUDA, buf);
}

void DeviceBuffer::ensure(size_t bytes) {
  if (bytes <= cap && ptr) return;
  release();
  size_t want = align256(bytes ? bytes : 256);
  cudaError_t e = cudaMalloc(&ptr, want);
  if (e != cudaSuccess) {
    ptr = nullptr;
    cap = 0;
    (void)cudaGetLastError();
    char buf[160];
    snprintf(buf, sizeof(buf), "device allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
    throw Error(ZK_ENOMEM, buf);
  }
  cap = want;
}

void DeviceBuffer::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
}

int device_sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

}  // namespace zk
