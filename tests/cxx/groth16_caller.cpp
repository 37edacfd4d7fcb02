// A caller written against the reference's C++ API, the way its CLI uses it
// (src/main.cu:115-171): groth16ReadZkeyHeader, groth16Prove,
// groth16ProofToSnarkjsJson, groth16ProofToCalldata.  It includes only
// include/groth16.h and links libzyklop_b200.so, so it compiles and runs
// unchanged wherever reference code did.
//
//   groth16_caller <zkey> <wtns> <proof.json> <calldata.hex>
//
// Prints the header fields and the sizes of the API structs on stdout.
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "groth16.h"

int main(int argc, char** argv) {
  std::printf("sizeof Groth16Proof %zu Groth16ZkeyHeader %zu Groth16CoefEntry %zu\n",
              sizeof(Groth16Proof), sizeof(Groth16ZkeyHeader), sizeof(Groth16CoefEntry));
  if (argc < 5) {
    std::fprintf(stderr, "Usage: %s <zkey> <wtns> <proof.json> <calldata.hex>\n", argv[0]);
    return 1;
  }
  try {
    Groth16ZkeyHeader hdr;
    groth16ReadZkeyHeader(argv[1], hdr);
    std::printf("header %u %u %u %u %d\n", hdr.n_constraints, hdr.n_vars, hdr.n_public,
                hdr.domain_size, hdr.log_domain);
    Groth16Proof proof;
    groth16Prove(argv[1], argv[2], proof);
    char json[4096];
    groth16ProofToSnarkjsJson(proof, json, sizeof json);
    FILE* f = std::fopen(argv[3], "w");
    if (!f) return 2;
    std::fprintf(f, "%s\n", json);
    std::fclose(f);
    uint8_t cd[256];
    groth16ProofToCalldata(proof, cd, sizeof cd);
    f = std::fopen(argv[4], "w");
    if (!f) return 2;
    for (int i = 0; i < 256; i++) std::fprintf(f, "%02x", cd[i]);
    std::fprintf(f, "\n");
    std::fclose(f);
  } catch (const std::runtime_error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 3;
  }
  return 0;
}
