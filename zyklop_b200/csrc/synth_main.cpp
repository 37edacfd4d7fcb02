// `zk_synth`: writes the seeded synthetic inputs the benchmark and tests use,
// in a process of its own (so a process that times the reference build never
// loads this library).
//
//   zk_synth circuit <zkey> <wtns> <log_domain> <uniform|circom> <seed>
//       a Groth16 circuit + CRS (zk_synth_circuit): uniform = 2 nonzeros per
//       A/B row and uniform Fr inputs; circom = 1-4 nonzeros per row and the
//       circom-like witness mix (55% in {0,1}, 15% below 2^64, 30% uniform)
//   zk_synth points <group> <log_n> <seed> <px.bin> <py.bin>
//       2^log_n points k_i G of G1 (group 1) or G2 (group 2) as affine
//       Montgomery SoA arrays (n x 4 / n x 8 little-endian u64 per
//       coordinate, the reference's msm_g1 / msm_g2_device input layout);
//       k_i are 252-bit values from a splitmix64 stream seeded by <seed>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/zyklop_b200.h"

static int fail(const char* what) {
  fprintf(stderr, "[zk_synth] %s: %s\n", what, zk_last_error());
  return 1;
}

static uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

static bool write_file(const char* path, const void* data, size_t bytes) {
  FILE* f = fopen(path, "wb");
  if (!f) return false;
  const bool ok = fwrite(data, 1, bytes, f) == bytes;
  return fclose(f) == 0 && ok;
}

static int usage(const char* argv0) {
  fprintf(stderr,
          "Usage: %s circuit <zkey> <wtns> <log_domain> <uniform|circom> <seed>\n"
          "       %s points <group> <log_n> <seed> <px.bin> <py.bin>\n",
          argv0, argv0);
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 2) return usage(argv[0]);
  if (!strcmp(argv[1], "circuit") && argc == 7) {
    zk_synth_params p;
    p.log_domain = (uint32_t)strtoul(argv[4], nullptr, 10);
    p.n_public = 8;
    p.n_private_inputs = 8;
    const bool circom = !strcmp(argv[5], "circom");
    if (!circom && strcmp(argv[5], "uniform")) return usage(argv[0]);
    p.nnz_min = circom ? 1 : 2;
    p.nnz_max = circom ? 4 : 2;
    p.witness_kind = circom ? 1 : 0;
    p.seed = strtoull(argv[6], nullptr, 10);
    if (zk_synth_circuit(nullptr, &p, argv[2], argv[3]) != ZK_OK) return fail("synth circuit");
    return 0;
  }
  if (!strcmp(argv[1], "points") && argc == 7) {
    const int group = atoi(argv[2]);
    const int lg = atoi(argv[3]);
    if ((group != 1 && group != 2) || lg < 0 || lg > 28) return usage(argv[0]);
    uint64_t seed = strtoull(argv[4], nullptr, 10);
    const size_t n = size_t(1) << lg, w = group == 1 ? 4 : 8;
    std::vector<uint64_t> k(4 * n);
    for (size_t i = 0; i < n; i++) {
      for (int j = 0; j < 4; j++) k[4 * i + j] = splitmix64(seed);
      k[4 * i + 3] &= (uint64_t(1) << 60) - 1;
    }
    uint64_t *dk = nullptr, *dx = nullptr, *dy = nullptr;
    if (cudaMalloc(&dk, 32 * n) != cudaSuccess || cudaMalloc(&dx, 8 * w * n) != cudaSuccess ||
        cudaMalloc(&dy, 8 * w * n) != cudaSuccess) {
      fprintf(stderr, "[zk_synth] device allocation failed\n");
      return 1;
    }
    if (cudaMemcpy(dk, k.data(), 32 * n, cudaMemcpyHostToDevice) != cudaSuccess) {
      fprintf(stderr, "[zk_synth] copy failed\n");
      return 1;
    }
    if (zk_mul_generator(nullptr, group, dk, n, dx, dy) != ZK_OK) return fail("points");
    std::vector<uint64_t> h(w * n);
    for (int c = 0; c < 2; c++) {
      if (cudaMemcpy(h.data(), c ? dy : dx, 8 * w * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
        fprintf(stderr, "[zk_synth] copy failed\n");
        return 1;
      }
      if (!write_file(argv[5 + c], h.data(), 8 * w * n)) {
        fprintf(stderr, "[zk_synth] cannot write %s\n", argv[5 + c]);
        return 1;
      }
    }
    cudaFree(dk);
    cudaFree(dx);
    cudaFree(dy);
    return 0;
  }
  return usage(argv[0]);
}
