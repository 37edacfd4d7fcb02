#pragma once
#include <cstdint>
#include <string>

namespace zk {

// canonical 256-bit integer (4 x u64 LE) -> decimal
std::string dec_string(const uint64_t v[4]);
// proof (pi_A[8], pi_B[16], pi_C[8], affine Montgomery) -> snarkjs JSON text
std::string proof_json(const uint64_t proof[32]);
// proof -> 256-byte EVM calldata (big-endian canonical)
void proof_calldata(const uint64_t proof[32], uint8_t out[256]);
// public signals (canonical, n x 4 u64) -> public.json text
std::string public_json(const uint64_t* values, uint32_t n_public);

}  // namespace zk
