// `prover` command line: the reference's argv contract and outputs
// (src/main.cu:115-171):
//   prover <circuit.zkey> <witness.wtns> <proof.json> <public.json>
// prints the proof JSON on stdout, writes proof.json and public.json, exits 1
// with a usage message when arguments are missing.  Optional flags after the
// four paths: --blind <seed> adds Groth16 blinding r, s derived from the seed
// (the reference never blinds); --repeat <k> proves k times with the circuit
// resident and reports the per-proof time on stderr.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/groth16.h"
#include "../../include/zyklop_b200.h"

static int fail(const char* what) {
  fprintf(stderr, "[prover] %s: %s\n", what, zk_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 5) {
    fprintf(stderr, "Usage:   %s <circuit.zkey> <witness.wtns> <proof.json> <public.json>\n", argv[0]);
    fprintf(stderr, "Example: %s circuit_final.zkey witness.wtns proof.json public.json\n", argv[0]);
    return 1;
  }
  const char* zkey_path = argv[1];
  const char* wtns_path = argv[2];
  const char* proof_path = argv[3];
  const char* public_path = argv[4];
  long repeat = 1;
  bool blind = false;
  uint64_t blind_seed = 0;
  for (int i = 5; i < argc; i++) {
    if (!strcmp(argv[i], "--repeat") && i + 1 < argc) repeat = strtol(argv[++i], nullptr, 10);
    else if (!strcmp(argv[i], "--blind") && i + 1 < argc) {
      blind = true;
      blind_seed = strtoull(argv[++i], nullptr, 10);
    } else {
      fprintf(stderr, "[prover] unknown option %s\n", argv[i]);
      return 1;
    }
  }
  uint64_t proof[32];
  if (!blind && repeat <= 1) {
    if (zk_groth16_prove_files(nullptr, zkey_path, wtns_path, proof) != ZK_OK) return fail("prove");
  } else {
    zk_circuit* c = nullptr;
    if (zk_circuit_load_file(nullptr, zkey_path, &c) != ZK_OK) return fail("load zkey");
    // witness: wtns section 2 read through the library's public-json helper is
    // text; read the raw values here instead
    FILE* f = fopen(wtns_path, "rb");
    if (!f) {
      fprintf(stderr, "[prover] cannot open %s\n", wtns_path);
      return 1;
    }
    std::vector<uint8_t> wb;
    {
      fseek(f, 0, SEEK_END);
      long len = ftell(f);
      fseek(f, 0, SEEK_SET);
      wb.resize(len > 0 ? (size_t)len : 0);
      if (len > 0 && fread(wb.data(), 1, wb.size(), f) != wb.size()) {
        fclose(f);
        fprintf(stderr, "[prover] cannot read %s\n", wtns_path);
        return 1;
      }
      fclose(f);
    }
    // locate section 2 (values) of the wtns BinFile
    const uint8_t* values = nullptr;
    uint32_t n_vars = 0;
    if (wb.size() >= 12 && !memcmp(wb.data(), "wtns", 4)) {
      uint32_t ns;
      memcpy(&ns, &wb[8], 4);
      size_t pos = 12;
      for (uint32_t i = 0; i < ns && pos + 12 <= wb.size(); i++) {
        uint32_t t;
        uint64_t sz;
        memcpy(&t, &wb[pos], 4);
        memcpy(&sz, &wb[pos + 4], 8);
        pos += 12;
        if (sz > wb.size() - pos) break;
        if (t == 1 && sz >= 40) memcpy(&n_vars, &wb[pos + 36], 4);
        if (t == 2) values = &wb[pos];
        pos += sz;
      }
    }
    if (!values || !n_vars) {
      fprintf(stderr, "[prover] %s is not a valid wtns file\n", wtns_path);
      return 1;
    }
    uint64_t r[4] = {0, 0, 0, 0}, s[4] = {0, 0, 0, 0};
    if (blind) {  // small deterministic scalars from the seed (below 2^252)
      uint64_t x = blind_seed;
      for (int i = 0; i < 8; i++) {
        x = x * 6364136223846793005ULL + 1442695040888963407ULL;
        (i < 4 ? r : s)[i & 3] = x;
      }
      r[3] &= 0x0fffffffffffffffULL;
      s[3] &= 0x0fffffffffffffffULL;
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (long k = 0; k < repeat; k++)
      if (zk_prove(c, reinterpret_cast<const uint64_t*>(values), n_vars, blind ? r : nullptr,
                   blind ? s : nullptr, proof) != ZK_OK)
        return fail("prove");
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (repeat > 1) fprintf(stderr, "[prover] %ld proofs, %.3f ms per proof\n", repeat, ms / repeat);
    zk_circuit_free(c);
  }
  char json[4096];
  if (zk_proof_to_json(proof, json, sizeof(json)) != ZK_OK) return fail("serialize");
  printf("%s\n", json);
  FILE* pf = fopen(proof_path, "w");
  if (!pf) {
    fprintf(stderr, "[main] Cannot write to %s\n", proof_path);
    return 1;
  }
  fprintf(pf, "%s\n", json);
  fclose(pf);
  printf("[main] Proof written to %s\n", proof_path);
  Groth16ZkeyHeader hdr;
  try {
    groth16ReadZkeyHeader(zkey_path, hdr);
  } catch (const std::exception& e) {
    fprintf(stderr, "[prover] %s\n", e.what());
    return 1;
  }
  std::vector<char> pub(64 + 96 * (size_t)(hdr.n_public + 1));
  if (zk_public_json(wtns_path, hdr.n_public, pub.data(), pub.size()) != ZK_OK)
    return fail("public signals");
  FILE* qf = fopen(public_path, "w");
  if (!qf) {
    fprintf(stderr, "[main] Cannot write to %s\n", public_path);
    return 1;
  }
  fputs(pub.data(), qf);
  fclose(qf);
  printf("[main] Public signals written to %s\n", public_path);
  return 0;
}
