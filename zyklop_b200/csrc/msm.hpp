// Pippenger multi-scalar multiplication on G1 and G2 (host-side interface).
//
// Replaces the reference's msm_g1 (include/msm_g1.cuh:714-926) and
// msm_g2_device (include/msm_g2.cuh:669-854): same inputs (SoA affine
// Montgomery points with (0,0) = infinity, canonical scalars) and the same
// affine Montgomery result, computed by a different GPU design:
//
//   1. msm_hist     signed c-bit digits of every scalar, warp-aggregated
//                   per-(window, bucket) counts;
//   2. msm_scan     exclusive scan of the counts (bucket offsets);
//   3. msm_scatter  counting-sort of (point, sign) records by bucket;
//   4. msm_accum    load-balanced segmented reduction: each thread adds a
//                   fixed number K of consecutive sorted records with mixed
//                   XYZZ+affine additions, so a bucket's size never decides a
//                   thread's work (skewed scalars stay balanced); buckets that
//                   cross thread ranges leave partial sums that further levels
//                   of the same kernel combine;
//   5. msm_reduce_l1 / msm_reduce_blk
//                   sum_b (b+1) S_b per window: running sums over chunks of
//                   buckets, then block-parallel passes (suffix scan + tree
//                   sum over 128 partial pairs each) down to one (U, A) pair
//                   per window;
//   6. host         A + 2^log_span U, Horner over windows (latency-bound,
//                   done on one CPU core) and affine conversion.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "host_field.hpp"
#include "runtime.hpp"

namespace zk {

struct MsmConfig {
  int c = 0;          // window bits (0 = choose from n)
  int k0 = 0;         // sorted records per thread in the first accumulation level
                      // (0 = choose from n)
  int k1 = 16;        // partial records per thread in later levels
  int chunk = 0;      // buckets per thread in the bucket reduction (0 = choose from n)
  bool operator==(const MsmConfig& o) const {
    return c == o.c && k0 == o.k0 && k1 == o.k1 && chunk == o.chunk;
  }
};

// Affine input points: x of point i at x + i*stride coordinates, y likewise.
// stride 1 = separate x / y arrays (the reference's SoA msm_g1 arguments);
// stride 2 = interleaved (x, y) records as stored in zkey sections 5-9.
struct PointsView {
  const void* x;
  const void* y;
  uint32_t stride;
};
inline PointsView points_soa(const void* px, const void* py) { return {px, py, 1}; }
inline PointsView points_aos(const void* base, bool g2) {
  return {base, reinterpret_cast<const char*>(base) + (g2 ? 64 : 32), 2};
}

// Where an enqueued MSM leaves its result: per window w two XYZZ points U_w
// and A_w (all U first, then all A) with window sum A_w + 2^log_span U_w, and
// the total sum_w 2^(c w) window_w.  windows = 1 for fixed-base MSMs.
struct MsmResult {
  const void* d_data = nullptr;
  size_t bytes = 0;
  int windows = 0;
  int c = 0;
  int log_span = 0;
};

// Two MSMs whose results are added (a proof's C and H parts of pi_C) can
// share one bucket reduction.  The producer (`merge_out`) stops after its
// bucket accumulation and leaves its buckets, returning an empty result
// (zero windows: the point at infinity).  The consumer (`merge_in`, same
// kind, window bits and bucket count) adds those buckets into its own
// before its reduction, so its result is the sum of both MSMs.  `ready`
// (the caller's event) is recorded after the producer's accumulation; the
// producer's scratch must stay untouched until the consumer has run.
struct MsmMerge {
  const void* buckets = nullptr;
  size_t count = 0;
  int c = 0;
  bool fixed = false;
  bool g2 = false;
  cudaEvent_t ready = nullptr;
};

int msm_default_c(size_t n, bool g2);
// Window bits a windowed MSM of n points runs with under cfg.
int msm_effective_c(size_t n, bool g2, const MsmConfig& cfg);
int msm_default_k0(size_t n, bool fixed);
int msm_default_chunk(size_t n, bool fixed = false, int c = 0);

// Device scratch bytes one MSM of n points needs with this configuration.
size_t msm_scratch_bytes(size_t n, bool g2, const MsmConfig& cfg);

// Enqueue the GPU part of an MSM on `stream`; its result stays inside
// `scratch` (which must hold msm_scratch_bytes(n, ...) bytes) until copied.
// `merge_out` / `merge_in`: see MsmMerge.
MsmResult msm_g1_enqueue(const PointsView& pts, const uint64_t* scalars, size_t n, void* scratch,
                         size_t scratch_bytes, const MsmConfig& cfg, cudaStream_t stream,
                         MsmMerge* merge_out = nullptr, const MsmMerge* merge_in = nullptr);
MsmResult msm_g2_enqueue(const PointsView& pts, const uint64_t* scalars, size_t n, void* scratch,
                         size_t scratch_bytes, const MsmConfig& cfg, cudaStream_t stream);

// Fixed-base MSMs: precomputed window multiples of a resident base set.
// msm_precompute writes W = 254 / c + 1 records per point (table layout:
// record w * n + i = affine 2^(c w) P_i, (x, y) interleaved); the fixed-base
// enqueue then sorts all (point, window) digits into one shared bucket set and
// returns a single window sum (combine it with n_windows = 1).  Scalars are
// reduced mod r first, which requires points of order r (CRS points are).
size_t msm_table_bytes(size_t n, bool g2, int c);
size_t msm_scratch_bytes_fixed(size_t n, bool g2, int c, const MsmConfig& cfg, int inst = 1);
void msm_precompute(bool g2, const PointsView& pts, size_t n, int c, void* table,
                    cudaStream_t stream);
MsmResult msm_enqueue_fixed(bool g2, const void* table, const uint64_t* scalars, size_t n, int c,
                            void* scratch, size_t scratch_bytes, const MsmConfig& cfg,
                            cudaStream_t stream, MsmMerge* merge_out = nullptr,
                            const MsmMerge* merge_in = nullptr);
// Several fixed-base MSMs with the same window bits in one launch chain: one
// instance per (table, scalars, n); their records share the sort, the
// load-balanced accumulation and the bucket reduction (instance i's buckets
// take the place of window i).  Its level-0 accumulation is persistent: as
// many blocks as the device holds at once claim record tiles (instance,
// bucket range) from a device work queue.  Scratch:
// msm_scratch_bytes_fixed(sum of n, g2, c, cfg, inst).  The result holds one
// window sum per instance (msm_g*_combine_inst).
constexpr int kMsmMaxInstances = 64;
MsmResult msm_enqueue_fixed_multi(bool g2, int inst, const void* const* tables,
                                  const uint64_t* const* scalars, const size_t* n, int c,
                                  void* scratch, size_t scratch_bytes, const MsmConfig& cfg,
                                  cudaStream_t stream);

// Host combination of an MSM result (r.bytes copied from r.d_data) into an
// affine Montgomery point.  Returns true for the point at infinity.
// The same sums left in XYZZ coordinates (inst >= 0: that instance of a
// multi-instance result), for callers that batch the affine conversions.
host::Xyzz<host::Fp> msm_g1_combine_xyzz(const void* h_data, const MsmResult& r, int inst = -1);
host::Xyzz<host::Fp2> msm_g2_combine_xyzz(const void* h_data, const MsmResult& r, int inst = -1);
bool msm_g1_combine(const void* h_data, const MsmResult& r, uint64_t out[8]);
bool msm_g2_combine(const void* h_data, const MsmResult& r, uint64_t out[16]);
bool msm_g1_combine_inst(const void* h_data, const MsmResult& r, int inst, uint64_t out[8]);
bool msm_g2_combine_inst(const void* h_data, const MsmResult& r, int inst, uint64_t out[16]);

// Blocking convenience wrappers: enqueue, copy the window sums back, combine.
bool msm_g1_run(const PointsView& pts, const uint64_t* scalars, size_t n, DeviceBuffer& scratch,
                const MsmConfig& cfg, cudaStream_t stream, uint64_t out[8]);
bool msm_g2_run(const PointsView& pts, const uint64_t* scalars, size_t n, DeviceBuffer& scratch,
                const MsmConfig& cfg, cudaStream_t stream, uint64_t out[16]);

}  // namespace zk
