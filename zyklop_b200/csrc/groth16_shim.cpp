// The reference's C++ API (include/groth16.h) over the C ABI.
#include "../../include/groth16.h"

#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/zyklop_b200.h"

static void zk_throw_if(int rc, const char* what) {
  if (rc != ZK_OK) throw std::runtime_error(std::string(what) + ": " + zk_last_error());
}

void groth16Prove(const char* zkey_path, const char* wtns_path, Groth16Proof& proof) {
  uint64_t p[32];
  zk_throw_if(zk_groth16_prove_files(nullptr, zkey_path, wtns_path, p), "groth16Prove");
  memcpy(proof.pi_A, p, 64);
  memcpy(proof.pi_B, p + 8, 128);
  memcpy(proof.pi_C, p + 24, 64);
}

static void pack(const Groth16Proof& proof, uint64_t* p) {
  memcpy(p, proof.pi_A, 64);
  memcpy(p + 8, proof.pi_B, 128);
  memcpy(p + 24, proof.pi_C, 64);
}

void groth16ProofToSnarkjsJson(const Groth16Proof& proof, char* out, size_t out_size) {
  uint64_t p[32];
  pack(proof, p);
  zk_throw_if(zk_proof_to_json(p, out, out_size), "groth16ProofToSnarkjsJson");
}

void groth16ProofToCalldata(const Groth16Proof& proof, uint8_t* out, size_t out_size) {
  uint64_t p[32];
  pack(proof, p);
  zk_throw_if(zk_proof_to_calldata(p, out, out_size), "groth16ProofToCalldata");
}

void groth16ReadZkeyHeader(const char* zkey_path, Groth16ZkeyHeader& hdr) {
  zk_zkey_header h;
  zk_throw_if(zk_read_zkey_header(zkey_path, &h), "groth16ReadZkeyHeader");
  hdr.n_constraints = h.n_constraints;
  hdr.n_vars = h.n_vars;
  hdr.n_public = h.n_public;
  hdr.domain_size = h.domain_size;
  hdr.log_domain = h.log_domain;
  memcpy(hdr.prime, h.prime, 32);
}
