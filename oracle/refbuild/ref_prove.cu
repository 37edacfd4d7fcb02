// Harness that exposes the reference prover (src/groth16.cu:1143-1397,
// declared at include/groth16.cuh:119-123) through a C ABI so that tests and
// the benchmark's reference arm can call it in-process, compiled for sm_100a
// by oracle/refbuild/Makefile.  It converts nothing: the proof struct is
// copied out as the reference fills it (affine Montgomery coordinates).
#include <cstdint>
#include <cstring>
#include "groth16.cuh"

extern "C" {

// out: pi_A[8], pi_B[16], pi_C[8] u64 in the reference's layout.
int zkref_prove_files(const char* zkey_path, const char* wtns_path, uint64_t* out) {
  Groth16Proof p;
  groth16Prove(zkey_path, wtns_path, p);
  memcpy(out, p.pi_A, 64);
  memcpy(out + 8, p.pi_B, 128);
  memcpy(out + 24, p.pi_C, 64);
  return 0;
}

// snarkjs JSON text of a proof given in the reference layout.
int zkref_proof_json(const uint64_t* in, char* out, size_t out_size) {
  Groth16Proof p;
  memcpy(p.pi_A, in, 64);
  memcpy(p.pi_B, in + 8, 128);
  memcpy(p.pi_C, in + 24, 64);
  groth16ProofToSnarkjsJson(p, out, out_size);
  return 0;
}

// 256-byte EVM calldata of a proof given in the reference layout
// (groth16ProofToCalldata, src/groth16.cu:1514-1557).
int zkref_proof_calldata(const uint64_t* in, uint8_t* out, size_t out_size) {
  Groth16Proof p;
  memcpy(p.pi_A, in, 64);
  memcpy(p.pi_B, in + 8, 128);
  memcpy(p.pi_C, in + 24, 64);
  groth16ProofToCalldata(p, out, out_size);
  return 0;
}

}  // extern "C"
