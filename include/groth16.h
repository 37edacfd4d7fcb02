/*
 * C++ drop-in for the reference's public API header (include/groth16.cuh of
 * Julienbxl/Zyklop): the same structs and function signatures, implemented
 * over the zyklop_b200 C ABI (zyklop_b200.h).  Code written against the
 * reference links against libzyklop_b200.so instead.
 *
 * Differences a caller can observe: no nttPrepare / nttDestroy calls are
 * needed, and failures throw std::runtime_error (with zk_last_error()'s
 * message) where the reference calls exit(1).  groth16SparseMvm, declared but
 * never defined by the reference (include/groth16.cuh:197), is not provided.
 */
#pragma once
#include <cstddef>
#include <cstdint>

/* include/groth16.cuh:69-73 */
struct Groth16Proof {
  uint64_t pi_A[8];   /* G1 affine [x[4], y[4]], Montgomery Fp */
  uint64_t pi_B[16];  /* G2 affine [x.a0, x.a1, y.a0, y.a1], Montgomery Fp */
  uint64_t pi_C[8];   /* G1 affine, Montgomery Fp */
};

/* include/groth16.cuh:79-86 */
struct Groth16ZkeyHeader {
  uint32_t n_constraints;
  uint32_t n_vars;
  uint32_t n_public;
  uint32_t domain_size;
  int log_domain;
  uint64_t prime[4];
};

/* include/groth16.cuh:93-98: one section-4 coefficient as a caller holds it
 * in memory (matrix 0 = A, 1 = B, 2 = C).  Declared for source compatibility;
 * the prover reads section 4 straight from the zkey and takes no array of
 * these (groth16SparseMvm, the reference's only user, is not provided). */
struct Groth16CoefEntry {
  uint8_t matrix;
  uint32_t constraint;
  uint32_t signal;
  uint64_t value[4];
};

/* include/groth16.cuh:119-123 */
void groth16Prove(const char* zkey_path, const char* wtns_path, Groth16Proof& proof);
/* include/groth16.cuh:149-153 */
void groth16ProofToSnarkjsJson(const Groth16Proof& proof, char* out, size_t out_size);
/* include/groth16.cuh:163-167 */
void groth16ProofToCalldata(const Groth16Proof& proof, uint8_t* out, size_t out_size);
/* include/groth16.cuh:177-180 */
void groth16ReadZkeyHeader(const char* zkey_path, Groth16ZkeyHeader& hdr);
