// Autotuned launch settings per (group, size, scalar distribution).
//
// Tunables, all of which leave results unchanged:
//   * windowed MSMs: window bits c, sorted records per accumulation thread k0
//     (the bucket-split threshold of the load-balanced accumulation: a bucket
//     with more records than k0 is split across threads), buckets per thread
//     in the bucket reduction (chunk);
//   * fixed-base MSMs: table window bits (under a memory cap), k0 and chunk;
//   * NTT: the largest radix of one shared-memory pass (2^bits).
// A context holds the table; settings given with zk_msm_set_config (c != 0)
// take precedence over it.  Sizes are keyed by round(log2 n), so a circuit
// of 2^k constraints (a few more witness variables than 2^k) and its H
// (2^k points) share the entries tuned at 2^k.
#pragma once
#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <tuple>

#include "msm.hpp"

struct zk_ctx;

namespace zk {

// Scalar distributions the tuner tells apart: uniform in Fr, and the skewed
// mix of circom-style witnesses (mostly bits and small integers).
enum ScalarDist { kDistUniform = 0, kDistSkewed = 1 };

struct TuneTable {
  // (group, log_n, dist, fixed-base window bits or 0) -> MSM settings
  std::map<std::tuple<int, int, int, int>, MsmConfig> msm;
  // (group, log_n, dist) -> fixed-base window bits
  std::map<std::tuple<int, int, int>, int> table_c;
};

int ceil_log2(size_t n);
int size_class(size_t n);  // round(log2 n)

// Settings for an MSM of n points: explicit context settings, else the tuned
// entry, else the defaults.
MsmConfig msm_config_for(const zk_ctx* ctx, bool g2, size_t n, int dist, int fixed_c);
// Fixed-base window bits for a point set of n points (tuned, else default).
int table_c_for(const zk_ctx* ctx, bool g2, size_t n, int dist);

// Classifies host scalars (canonical, 4 x u64 each) from an evenly spaced
// sample: skewed when at least 40% of them are below 2^64.
int detect_scalar_dist(const uint64_t* scalars, size_t n);

struct TuneResult {
  MsmConfig cfg;
  int table_c = 0;
  int pass_bits = 0;
  double ms = 0;
};

// Time candidate settings on seeded synthetic inputs (points k_i * G, scalars
// of the given distribution) on the context's stream and record the fastest.
TuneResult autotune_msm(zk_ctx* ctx, int group, int log_n, int dist, int fixed_c);
TuneResult autotune_table_c(zk_ctx* ctx, int group, int log_n, int dist, size_t max_table_bytes);
TuneResult autotune_ntt(zk_ctx* ctx, int log_n);

// One line per entry:  msm <group> <log_n> <dist> <fixed_c> <c> <k0> <k1> <chunk>
//                      table <group> <log_n> <dist> <c>
//                      ntt <log_n> <pass_bits>
std::string tune_export(const zk_ctx* ctx);
void tune_import(zk_ctx* ctx, const char* text);

}  // namespace zk
