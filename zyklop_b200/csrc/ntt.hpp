// Fr number-theoretic transforms and the Groth16 H-polynomial pipeline.
//
// Convention (identical results to the reference, include/ntt_bn254.cuh:
// 190-464): natural-order DFT X[k] = sum_i x[i] w^(ik) with
// w = omega_N = 5^((r-1)/N); the inverse uses w^-1 and scales by 1/N.
// Elements are Montgomery Fr.
//
// Layout of the work: each transform runs as ceil(log N / 8) passes over HBM
// (8 = the default largest pass radix, tunable per size);
// a pass loads tiles of up to 256-point sub-transforms (times a few adjacent
// columns for coalescing) into shared memory, runs up to 8 radix-2 stages there
// and writes back.  Decimation-in-frequency passes take natural order to
// bit-reversed order, decimation-in-time passes the reverse, so the H
// pipeline (INTT -> coset shift -> NTT) never permutes: it keeps coefficients
// in bit-reversed order between the two transforms.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "runtime.hpp"

namespace zk {

constexpr int kMaxLogN = 27;  // Fr 2-adicity is 28; H needs omega_2n

// Twiddle tables tw[e] = w^e (forward) and w^-e (inverse), e < 2^(lmax-1),
// w a primitive 2^lmax-th root.  Smaller transforms read them with a stride.
// pass_bits[L]: largest radix (2^bits, 4..8) of one shared-memory pass for
// transforms of 2^L points (a tunable; kernels hold tiles of 1024 points).
constexpr int kMaxPassBits = 8;
struct NttTables {
  int lmax = -1;
  DeviceBuffer fwd, inv;
  int pass_bits[kMaxLogN + 1];
  NttTables() {
    for (int& b : pass_bits) b = kMaxPassBits;
  }
  void ensure(int log_n, cudaStream_t stream);
};

// In-place natural-order transform of 2^log_n elements (scratch: 32 << log_n
// bytes of device memory).
void ntt_inplace(NttTables& tw, uint64_t* a, int log_n, bool inverse, void* scratch,
                 cudaStream_t stream);

// H evaluations on the odd coset, following src/groth16.cu:1037-1090:
//   C = A*B; a,b,c = INTT(A,B,C); x_i *= omega_2n^i; A',B',C' = NTT(a,b,c);
//   h = A'B' - C' decoded to canonical.
// aw and bw (Montgomery, 2^log_n each) are overwritten; cw is scratch of the
// same size; h receives canonical Fr.
void hpoly(NttTables& tw, uint64_t* aw, uint64_t* bw, uint64_t* cw, int log_n, uint64_t* h,
           cudaStream_t stream);
// The same for `count` (1..kMaxHBatch) polynomials of one size in one
// launch per stage (grid.y runs over the polynomials' vectors).
constexpr int kMaxHBatch = 16;
void hpoly_batch(NttTables& tw, int count, uint64_t* const* aw, uint64_t* const* bw,
                 uint64_t* const* cw, int log_n, uint64_t* const* h, cudaStream_t stream);

// The H pipelines of up to kMaxHJobs jobs of any sizes in one persistent
// launch: resident blocks take (job, step, tile) work items in step order
// from a device work queue, and an item starts once every item of the same
// job's previous step is done (steps: A*B, the DIF passes, the coset scale,
// the DIT passes, h).  Each job's aw, bw are overwritten, cw is scratch and
// h receives the canonical result, as in hpoly.  `sync` is kHSyncWords u32
// of caller-owned device memory, cleared here on `stream`; a wait for a
// previous step gives up after about two seconds and sets sync[0] to 1 (the
// caller copies it back and fails the proof).
constexpr int kMaxHJobs = 32;
constexpr int kMaxHPasses = 7;                      // passes of >= 4 bits up to 2^28
constexpr int kMaxHSteps = 2 * kMaxHPasses + 3;
constexpr size_t kHSyncWords = 2 + (size_t)kMaxHJobs * kMaxHSteps;
struct HJob {
  uint64_t *aw, *bw, *cw, *h;
  int log_n;
};
void hpoly_multi(NttTables& tw, int count, const HJob* jobs, uint32_t* sync, cudaStream_t stream);

// Elementwise helpers over Montgomery / canonical Fr arrays.
void fr_encode(const uint64_t* in, uint64_t* out, size_t n, cudaStream_t stream);
void fr_decode(const uint64_t* in, uint64_t* out, size_t n, cudaStream_t stream);

}  // namespace zk
