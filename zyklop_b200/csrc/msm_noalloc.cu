// zk_msm_g1_noalloc: the G1 MSM for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc: a plugin loaded into a host
// application that has already handed all of the device's memory to its own
// pool allocator, or a latency-critical loop where cudaMalloc's implicit
// device-wide synchronization is not acceptable.  This entry point runs the
// same MSM kernels as zk_msm_g1, but its scratch lives in a file-scope
// __device__ array of fixed size instead of a context arena, and it takes the
// caller's stream instead of a context, so it needs no allocation of its own.
//
// Limits and rules:
//   * at most kNoAllocMaxPoints = 2^16 points per call (the scratch array is
//     24 MiB and, once placed, is held by that GPU until the process exits);
//   * CUDA loads a library's device code lazily (by default since CUDA
//     12.2), so the array is placed in device memory when a device first
//     needs this module -- here, the first call's cudaGetSymbolAddress --
//     not when the library is loaded.  A caller whose host application
//     later hands all device memory to its own pool must make one warm-up
//     call on each device first; if the array cannot be placed, the call
//     returns ZK_ENOMEM with a message saying so;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current);
//   * the call copies the result to the host and synchronizes its stream,
//     so it cannot be made while that stream is being captured into a CUDA
//     graph: it checks and returns ZK_ENOTSUP;
//   * every call shares the one array: calls whose work overlaps on the GPU
//     (different streams, or different host threads) race and give wrong
//     results, so serialize them;
//   * the array keeps the previous call's contents; the kernels clear what
//     must start at zero (bucket counts and bucket sums) at the start of
//     every call.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "capi_util.hpp"
#include "msm.hpp"
#include "profile.hpp"
#include "runtime.hpp"

namespace {

constexpr size_t kNoAllocMaxPoints = size_t(1) << 16;
constexpr size_t kNoAllocScratchBytes = size_t(24) << 20;
constexpr int kMaxWindows = 256 / 4 + 1;  // windows of the smallest window size (4 bits)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// host-side: the array's device address on each device (null until set up)
void* g_noalloc_addr[kMaxDevices] = {};
std::mutex g_noalloc_mu;

int fail(int code, const char* msg) {
  zk::set_last_error(code, msg);
  return code;
}

}  // namespace

extern "C" int zk_msm_g1_noalloc(const uint64_t* d_px, const uint64_t* d_py,
                                 const uint64_t* d_scalars, size_t n, uint64_t* h_out,
                                 int* is_inf, void* stream) {
  if (!h_out) return fail(ZK_EINVAL, "zk_msm_g1_noalloc: NULL output");
  if (n && !(d_px && d_py && d_scalars)) return fail(ZK_EINVAL, "zk_msm_g1_noalloc: NULL input");
  if (n > kNoAllocMaxPoints) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "zk_msm_g1_noalloc: %zu points exceed the maximum of %zu (fixed scratch of %zu MiB); "
             "use zk_msm_g1 for larger MSMs",
             n, kNoAllocMaxPoints, kNoAllocScratchBytes >> 20);
    return fail(ZK_EINVAL, msg);
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ZK_ECUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(ZK_ENOTSUP, "zk_msm_g1_noalloc: device index too large");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) return fail(ZK_ECUDA, cudaGetErrorString(e));
  if (cap != cudaStreamCaptureStatusNone)
    return fail(ZK_ENOTSUP,
                "zk_msm_g1_noalloc: the stream is being captured; the call synchronizes its "
                "stream and cannot be captured");
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      // once per device, with that device current (it is: cudaGetDevice above)
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e == cudaErrorMemoryAllocation) {
        (void)cudaGetLastError();
        return fail(ZK_ENOMEM,
                    "zk_msm_g1_noalloc: no device memory left to place the fixed 24 MiB scratch "
                    "array (make a warm-up call before the application's pool takes the memory)");
      }
      if (e != cudaSuccess || !p) {
        (void)cudaGetLastError();
        return fail(ZK_ECUDA, "zk_msm_g1_noalloc: cudaGetSymbolAddress failed");
      }
      g_noalloc_addr[dev] = p;
    }
    scratch = g_noalloc_addr[dev];
  }
  // no event recording (it would create events); the calling thread's
  // profiler is put back on every return path
  struct ProfilerOff {
    zk::Profiler* saved = zk::current_profiler();
    ProfilerOff() { zk::set_current_profiler(nullptr); }
    ~ProfilerOff() { zk::set_current_profiler(saved); }
  } profiler_off;
  ZK_API_BEGIN
  // fixed settings: the 24 MiB bound above is checked against this layout
  zk::MsmConfig cfg;
  cfg.k0 = 64;
  cfg.chunk = 16;
  ZK_REQUIRE(zk::msm_scratch_bytes(n, false, cfg) <= kNoAllocScratchBytes, ZK_EINTERNAL,
             "zk_msm_g1_noalloc: scratch layout exceeds the fixed array");
  const zk::MsmResult r = zk::msm_g1_enqueue(zk::points_soa(d_px, d_py), d_scalars, n, scratch,
                                             kNoAllocScratchBytes, cfg, st);
  alignas(16) unsigned char h_windows[2 * kMaxWindows * 128];
  ZK_REQUIRE(r.bytes <= sizeof(h_windows), ZK_EINTERNAL, "zk_msm_g1_noalloc: too many windows");
  ZK_CUDA(cudaMemcpyAsync(h_windows, r.d_data, r.bytes, cudaMemcpyDeviceToHost, st));
  ZK_CUDA(cudaStreamSynchronize(st));
  const bool inf = zk::msm_g1_combine(h_windows, r, h_out);
  if (is_inf) *is_inf = inf ? 1 : 0;
  ZK_API_END
}
