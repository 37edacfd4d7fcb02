// Launch accounting and opt-in kernel timing.
//
// Every kernel launch of the library goes through count_launch(), so callers
// can read how many of the library's kernels ran (zk_launch_count).  When a
// context has profiling enabled, the hot kernels are bracketed with CUDA
// events recorded on the stream they are launched on; zk_ctx_profile sums
// them per kernel kind together with the work units (points, elements) each
// launch processed.  The reference's counterpart is its env-gated cudaEvent
// phase timers (ZK_G1_DEBUG, ZK_HPIPE_DEBUG: include/msm_g1.cuh:78-227,
// src/groth16.cu:951-1022).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <vector>

namespace zk {

void count_launch(int n);
uint64_t launch_count();

enum ProfKind { kProfAccumG1 = 0, kProfAccumG2, kProfNttPass, kProfSpmv, kProfKinds };

struct Profiler {
  struct Rec {
    int kind;
    cudaEvent_t a, b;
    double units;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  ~Profiler();
  cudaEvent_t get();
  // returns a record index; call end() after the launch
  size_t begin(int kind, double units, cudaStream_t st);
  void end(size_t rec, cudaStream_t st);
  // synchronizes, sums per kind, clears
  void collect(double* ms, double* launches, double* units);
};

// Profiler of the API call running on this thread (null when disabled).
Profiler* current_profiler();
void set_current_profiler(Profiler* p);

struct ProfScope {  // brackets one launch when profiling is on
  Profiler* p;
  size_t rec = 0;
  cudaStream_t st;
  ProfScope(int kind, double units, cudaStream_t s) : p(current_profiler()), st(s) {
    if (p) rec = p->begin(kind, units, st);
  }
  ~ProfScope() {
    if (p) p->end(rec, st);
  }
};

// Carry-chain IMAD throughput of the device (mad.lo.cc / madc.hi.cc pairs, as
// in the field multiplication), in 10^12 32-bit multiply-adds per second.
// Measured integer multiply-add throughput of the device in 10^12 ops/s at
// full occupancy: kind 0 = carry chains (mad.lo.cc / madc.hi.cc, the field
// products' mix), kind 1 = independent mad.lo / mad.hi streams (no carry).
double imad_probe(cudaStream_t st, int kind = 0);

}  // namespace zk
