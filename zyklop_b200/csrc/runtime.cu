// Runtime plumbing (see runtime.hpp).
#include <cuda_runtime.h>

#include <omp.h>

#include <atomic>
#include <cstdarg>
#include <cstring>
#include <string>

#include "runtime.hpp"

namespace zk {

namespace {
thread_local std::string g_last_error;
// allocations the library has made in this process (zk_memory_stats)
std::atomic<uint64_t> g_dev_allocs{0}, g_dev_alloc_bytes{0}, g_host_allocs{0};
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

namespace {
// One stream-ordered pool per device for every DeviceBuffer: freed blocks stay
// reserved (release threshold = all) and later allocations reuse them without
// the driver mapping or unmapping pages, which is most of what loading and
// freeing a circuit through cudaMalloc / cudaFree would cost.
constexpr int kMaxPoolDevices = 64;
struct DevPool {
  std::once_flag once;
  cudaMemPool_t pool = nullptr;
  cudaStream_t st = nullptr;  // allocation / free stream (synchronized on use)
  bool ok = false;
};
DevPool g_pools[kMaxPoolDevices];

DevPool* pool_of(int dev) {
  if (dev < 0 || dev >= kMaxPoolDevices) return nullptr;
  DevPool& p = g_pools[dev];
  std::call_once(p.once, [&] {
    int supported = 0;
    if (cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, dev) != cudaSuccess ||
        !supported) {
      (void)cudaGetLastError();
      return;
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (cudaMemPoolCreate(&p.pool, &props) != cudaSuccess) {
      (void)cudaGetLastError();
      return;
    }
    uint64_t keep = ~uint64_t(0);
    cudaMemPoolSetAttribute(p.pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (cudaStreamCreateWithFlags(&p.st, cudaStreamNonBlocking) != cudaSuccess) {
      (void)cudaGetLastError();
      return;
    }
    p.ok = true;
  });
  return p.ok ? &p : nullptr;
}
}  // namespace

void alloc_stats(uint64_t* dev_allocs, uint64_t* dev_bytes, uint64_t* host_allocs) {
  *dev_allocs = g_dev_allocs.load();
  *dev_bytes = g_dev_alloc_bytes.load();
  *host_allocs = g_host_allocs.load();
}

bool pool_usage(int dev, uint64_t* reserved, uint64_t* used) {
  *reserved = *used = 0;
  DevPool* p = pool_of(dev);
  if (!p) return false;
  cudaMemPoolGetAttribute(p->pool, cudaMemPoolAttrReservedMemCurrent, reserved);
  cudaMemPoolGetAttribute(p->pool, cudaMemPoolAttrUsedMemCurrent, used);
  return true;
}

size_t device_free_bytes() {
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  int dev = 0;
  cudaGetDevice(&dev);
  if (DevPool* p = pool_of(dev)) {
    uint64_t reserved = 0, used = 0;
    cudaMemPoolGetAttribute(p->pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(p->pool, cudaMemPoolAttrUsedMemCurrent, &used);
    if (reserved > used) fr += reserved - used;
  }
  return fr;
}

void release_cached_memory() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (DevPool* p = pool_of(dev)) {
    cudaStreamSynchronize(p->st);
    cudaMemPoolTrimTo(p->pool, 0);
  }
}

void DeviceBuffer::ensure(size_t bytes) {
  if (bytes <= cap && ptr) return;
  release();
  size_t want = align256(bytes ? bytes : 256);
  cudaGetDevice(&dev);
  cudaError_t e;
  if (DevPool* p = pool_of(dev)) {
    e = cudaMallocFromPoolAsync(&ptr, want, p->pool, p->st);
    // the block is usable from any stream once the allocation has executed
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->st);
    pooled = true;
  } else {
    e = cudaMalloc(&ptr, want);
    pooled = false;
  }
  if (e != cudaSuccess) {
    ptr = nullptr;
    cap = 0;
    (void)cudaGetLastError();
    char buf[160];
    snprintf(buf, sizeof(buf), "device allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
    throw Error(ZK_ENOMEM, buf);
  }
  cap = want;
  g_dev_allocs++;
  g_dev_alloc_bytes += want;
}

void DeviceBuffer::release() {
  if (ptr) {
    if (pooled) {
      int cur = 0;
      cudaGetDevice(&cur);
      if (cur != dev) cudaSetDevice(dev);
      // like cudaFree: no work still using the block may run after it is reused
      cudaDeviceSynchronize();
      if (DevPool* p = pool_of(dev)) cudaFreeAsync(ptr, p->st);
      if (cur != dev) cudaSetDevice(cur);
    } else {
      cudaFree(ptr);
    }
  }
  ptr = nullptr;
  cap = 0;
}

void PinnedBuffer::ensure(size_t bytes) {
  if (bytes <= cap && ptr) return;
  release();
  const size_t want = align256(bytes ? bytes : 256);
  cudaError_t e = cudaMallocHost(&ptr, want);
  if (e != cudaSuccess) {
    ptr = nullptr;
    (void)cudaGetLastError();
    throw Error(ZK_ENOMEM, std::string("pinned host allocation failed: ") + cudaGetErrorString(e));
  }
  cap = want;
  g_host_allocs++;
}

void PinnedBuffer::release() {
  if (ptr) cudaFreeHost(ptr);
  ptr = nullptr;
  cap = 0;
}

Stager::~Stager() {
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
}

namespace {
// host threads that copy into the pinned staging buffers: measured on the
// pool's 16-core hosts, 16 threads keep the copy at the PCIe rate (587 MB in
// 12 ms, the pinned-only DMA time) where 8 take 13-16 ms
int stage_threads() {
  static const int n = [] {
    const int p = omp_get_num_procs();
    return p < 1 ? 1 : (p > 16 ? 16 : p);
  }();
  return n;
}
}  // namespace

void Stager::upload(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (!bytes) return;
  for (int i = 0; i < 2; i++) {
    buf[i].ensure(kChunk);
    if (!ev[i]) ZK_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
  }
  const char* s = reinterpret_cast<const char*>(src);
  char* d = reinterpret_cast<char*>(dst);
  for (size_t off = 0, k = 0; off < bytes; off += kChunk, k++) {
    const size_t len = bytes - off < kChunk ? bytes - off : kChunk;
    const int b = (int)(k & 1);
    ZK_CUDA(cudaEventSynchronize(ev[b]));  // previous DMA from this buffer is done
    char* p = buf[b].as<char>();
    const long parts = (long)((len + (size_t(1) << 20) - 1) >> 20);
    const int nt = stage_threads();
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long q = 0; q < parts; q++) {
      const size_t o = (size_t)q << 20;
      const size_t l = len - o < (size_t(1) << 20) ? len - o : (size_t(1) << 20);
      memcpy(p + o, s + off + o, l);
    }
    ZK_CUDA(cudaMemcpyAsync(d + off, p, len, cudaMemcpyHostToDevice, st));
    ZK_CUDA(cudaEventRecord(ev[b], st));
  }
  ZK_CUDA(cudaEventSynchronize(ev[0]));
  ZK_CUDA(cudaEventSynchronize(ev[1]));
}

int device_sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

}  // namespace zk
