// Per-device library context (the object behind zk_ctx).
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <vector>

#include "msm.hpp"
#include "ntt.hpp"
#include "profile.hpp"
#include "runtime.hpp"
#include "tune.hpp"

namespace zk {

// Largest MSM result copied to the host: 2 x 64 windows of G2 XYZZ points.
constexpr size_t kMaxWindowBytes = 2 * 64 * 256;

// Buffers and streams of one in-flight proof (reused across proofs).  A
// context has one for single proofs and a pool for batches (a proof server
// has its own); each can hold captured graphs of its device pipeline.
struct ProveWs {
  static constexpr int kStreams = 5;  // 0: witness/SpMV/H/MSM_H, 1: A, 2: B2, 3: C, 4: B1
  // ordered: stream priorities by chain (a proof that runs alone); workspaces
  // whose proofs run beside others' keep equal priorities
  explicit ProveWs(bool ordered = false) : ordered(ordered) {}
  bool ordered = false;
  bool ready = false;
  int nstreams = kStreams;      // streams the current proof spreads its MSMs over
  int env_nstreams = kStreams;  // ZYKLOP_PROVE_STREAMS, else kStreams
  cudaStream_t st[kStreams] = {};
  cudaEvent_t ev_we = nullptr, ev_begin = nullptr, ev_all = nullptr;
  cudaEvent_t ev_done[kStreams] = {};
  cudaEvent_t ev_merge = nullptr;  // C's buckets accumulated (H reduces them with its own)
  MsmMerge merge_c;
  DeviceBuffer we, aw, bw, cw, h;
  DeviceBuffer msm[kStreams];
  PinnedBuffer win[kStreams];
  PinnedBuffer flag;  // small host-visible status words (section-4 check)
  MsmResult res[kStreams];
  MsmConfig cfg[kStreams];  // settings of each MSM of the current proof
  // captured pipelines, one per (circuit, blinding); all are dropped when a
  // buffer they point into is reallocated
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    uint64_t circuit = 0;  // circuit id the graph was captured for
    bool blind = false;
    int ntt_lmax = 0;  // twiddle table the graph reads
    int ntt_bits = 0;  // NTT pass radix captured
    int nstreams = 0;  // MSM streams captured
    MsmConfig cfg[kStreams];  // settings of each MSM captured
    int tab_c[2] = {0, 0};  // fixed-base table windows captured (0: windowed)
    uint64_t kernels = 0;
    MsmResult res[kStreams];  // where and how the graph leaves each MSM's windows
  };
  static constexpr size_t kMaxGraphs = 8;
  std::vector<Graph> graphs;
  void init();
  void drop_graph();
  cudaEvent_t ev_begin_pool() { init(); return ev_begin; }
  ~ProveWs();
};

// Workspace of one fused batch group (see prove_batch_fused): streams, every
// job's witness and polynomial buffers, the two multi-instance MSM arenas and
// their pinned result copies.
struct FusedWs {
  static constexpr int kPolyStreams = 4;
  bool ready = false;
  // s1: staging, then the H chain; s2: the B2 chain; s3: the A / C / B1
  // chain; sp[]: SpMV and H polynomials of the jobs, round robin
  cudaStream_t s1 = nullptr, s2 = nullptr, s3 = nullptr, sp[kPolyStreams] = {};
  cudaEvent_t ev_staged = nullptr, ev_g2 = nullptr, ev_g1w = nullptr, ev_done = nullptr;
  cudaEvent_t ev_sp[kPolyStreams] = {};
  DeviceBuffer we, poly, g1w, gh, g2;
  PinnedBuffer win1w, winh, win2;
  DeviceBuffer hsync;  // work queue and step counters of the persistent H pipeline
  PinnedBuffer hflag;  // its timeout flag, copied back per group
  // captured device pipelines of groups (zk_ctx_set_graphs): one per group
  // signature (jobs, settings and buffer addresses), replayed when the same
  // group comes again; the MSM result metadata is kept with the graph
  struct Graph {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec = nullptr;
    MsmResult rw, rh, r2;
    uint64_t kernels = 0;
  };
  static constexpr size_t kMaxGraphs = 8;
  std::vector<Graph> graphs;
  void drop_graphs();
  ~FusedWs();
};

}  // namespace zk

struct zk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  zk::NttTables ntt;
  zk::DeviceBuffer ntt_scratch;
  zk::DeviceBuffer msm_scratch;
  zk::MsmConfig msm_cfg[2];       // explicit settings (c != 0) or defaults
  zk::TuneTable tune;             // autotuned settings
  int scalar_dist = 0;            // distribution hint for zk_msm_g1 / g2
  zk::ProveWs ws{true};  // single proofs (ordered streams)
  std::vector<std::unique_ptr<zk::ProveWs>> pool;  // in-flight batch workspaces
  zk::FusedWs fused[2];                            // fused batch groups (alternating)
  int batch_mode = 0;    // 0 auto, 1 in-flight pipelines, 2 fused groups
  int batch_group = 16;  // proofs per fused group
  bool use_graphs = false;  // replay captured per-circuit proof graphs
  int prove_streams = 0;    // MSM streams per proof (0: ZYKLOP_PROVE_STREAMS or 5)
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
