// Harness that exposes the reference's own MSM and NTT entry points through a
// plain C ABI so that tests and the benchmark can run them (compiled for
// sm_100a from the reference headers by oracle/refbuild/Makefile).  Everything
// here is test infrastructure: it only moves buffers in and out of the
// reference functions named below and never changes what they compute.
//   msm_g1        include/msm_g1.cuh:918-926
//   msm_g2_device include/msm_g2.cuh:669
//   nttPrepare / ntt / nttDestroy include/ntt_bn254.cuh:190-281, 418-464
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>
#include "fp_bn254.cuh"
#include "fp2_bn254.cuh"
#include "fr_bn254.cuh"
#include "msm_g1.cuh"
#include "msm_g2.cuh"
#include "ntt_bn254.cuh"

extern "C" {

// G1 MSM over device-resident SoA inputs (px, py: n x 4 u64 Montgomery;
// sc: n x 4 u64 canonical).  out: x[4], y[4] Montgomery; returns 1 for the
// point at infinity, 0 otherwise.
int zkref_msm_g1_device(const uint64_t* d_px, const uint64_t* d_py,
                        const uint64_t* d_sc, int n, uint64_t* out) {
  FpPointAff r;
  msm_g1(d_px, d_py, d_sc, n, r);
  memcpy(out, r.X, 32);
  memcpy(out + 4, r.Y, 32);
  return r.infinity ? 1 : 0;
}

// G2 MSM over device-resident SoA inputs (px, py: n x 8 u64 [a0, a1]).
// out: x.a0, x.a1, y.a0, y.a1 (16 u64).
int zkref_msm_g2_device(const uint64_t* d_px, const uint64_t* d_py,
                        const uint64_t* d_sc, int n, uint64_t* out) {
  Fp2PointAff r;
  msm_g2_device(d_px, d_py, d_sc, n, r);
  memcpy(out, r.X, 64);
  memcpy(out + 8, r.Y, 64);
  return r.infinity ? 1 : 0;
}

// In-place natural-order NTT (inverse != 0: scaled inverse) of a device
// buffer of 2^log_n Montgomery Fr elements.
int zkref_ntt_device(uint64_t* d_a, int log_n, int inverse) {
  nttPrepare(log_n + 1);
  ntt(d_a, log_n, inverse != 0);
  cudaError_t e = cudaDeviceSynchronize();
  nttDestroy();
  return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"
