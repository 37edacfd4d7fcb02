// Autotuner: times candidate MSM / fixed-base / NTT settings on seeded
// synthetic inputs and keeps the fastest per (group, size, scalar
// distribution) in the context (see tune.hpp).  No reference counterpart: the
// reference fixes C = 16 for G1 (include/msm_g1.cuh:714-926) and its bucket
// tiers at compile time.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <vector>

#include "capi_util.hpp"
#include "context.hpp"
#include "ntt.hpp"
#include "prover.hpp"
#include "tune.hpp"

namespace zk {

void mul_generator(int group, const uint64_t* scalars, size_t n, uint64_t* px, uint64_t* py,
                   cudaStream_t st);

int ceil_log2(size_t n) {
  int lg = 0;
  while ((size_t(1) << lg) < n) lg++;
  return lg;
}

int size_class(size_t n) { return n <= 1 ? 0 : (int)std::lround(std::log2((double)n)); }

MsmConfig msm_config_for(const zk_ctx* ctx, bool g2, size_t n, int dist, int fixed_c) {
  const MsmConfig& base = ctx->msm_cfg[g2 ? 1 : 0];
  if (base.c != 0) return base;  // explicit settings win
  const auto it = ctx->tune.msm.find(std::make_tuple(g2 ? 2 : 1, size_class(n), dist, fixed_c));
  if (it == ctx->tune.msm.end()) return base;
  MsmConfig r = it->second;
  r.k1 = base.k1;
  return r;
}

int table_c_for(const zk_ctx* ctx, bool g2, size_t n, int dist) {
  const auto it = ctx->tune.table_c.find(std::make_tuple(g2 ? 2 : 1, size_class(n), dist));
  return it != ctx->tune.table_c.end() ? it->second : msm_fixed_default_c(n, g2);
}

int detect_scalar_dist(const uint64_t* s, size_t n) {
  if (!n) return kDistUniform;
  const size_t samples = std::min<size_t>(n, 256);
  size_t small = 0;
  for (size_t k = 0; k < samples; k++) {
    const uint64_t* v = s + 4 * (k * n / samples);
    if (!(v[1] | v[2] | v[3])) small++;
  }
  return 10 * small >= 4 * samples ? kDistSkewed : kDistUniform;
}

namespace {

using Clock = std::chrono::steady_clock;

uint64_t splitmix(uint64_t& x) {
  uint64_t z = (x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// canonical scalars below 2^253 < r (uniform), or the circom-like mix:
// 55% in {0, 1}, 15% below 2^64, 30% uniform
void make_scalars(size_t n, int dist, uint64_t seed, std::vector<uint64_t>& out) {
  out.assign(4 * n, 0);
  uint64_t st = seed;
  for (size_t i = 0; i < n; i++) {
    uint64_t* v = &out[4 * i];
    const uint64_t u = splitmix(st) % 100;
    if (dist == kDistSkewed && u < 55) {
      v[0] = splitmix(st) & 1;
    } else if (dist == kDistSkewed && u < 70) {
      v[0] = splitmix(st);
    } else {
      for (int q = 0; q < 4; q++) v[q] = splitmix(st);
      v[3] &= (uint64_t(1) << 61) - 1;
    }
  }
}

struct Inputs {
  int group = 1;
  size_t n = 0;
  DeviceBuffer px, py, sc;
};

void make_inputs(zk_ctx* ctx, int group, size_t n, int dist, Inputs& in) {
  cudaStream_t st = ctx->stream;
  in.group = group;
  in.n = n;
  const size_t w = group == 1 ? 32 : 64;
  in.px.ensure(w * n);
  in.py.ensure(w * n);
  in.sc.ensure(32 * n);
  std::vector<uint64_t> h;
  make_scalars(n, kDistUniform, 0x5eed0001ull + n, h);  // point multipliers
  ZK_CUDA(cudaMemcpyAsync(in.sc.ptr, h.data(), 32 * n, cudaMemcpyHostToDevice, st));
  mul_generator(group, in.sc.as<uint64_t>(), n, in.px.as<uint64_t>(), in.py.as<uint64_t>(), st);
  ZK_CUDA(cudaStreamSynchronize(st));
  make_scalars(n, dist, 0x5eed0002ull + n + 7919 * dist, h);
  ZK_CUDA(cudaMemcpyAsync(in.sc.ptr, h.data(), 32 * n, cudaMemcpyHostToDevice, st));
  ZK_CUDA(cudaStreamSynchronize(st));
}

// Median wall time of one MSM with the given settings (enqueue, copy of the
// window sums, host combine), and its result for the cross-check.
double time_msm(zk_ctx* ctx, const Inputs& in, const MsmConfig& cfg, int fixed_c, const void* table,
                DeviceBuffer& scratch, int reps, std::vector<uint64_t>& result) {
  cudaStream_t st = ctx->stream;
  const bool g2 = in.group == 2;
  const size_t n = in.n;
  scratch.ensure(fixed_c ? msm_scratch_bytes_fixed(n, g2, fixed_c, cfg)
                         : msm_scratch_bytes(n, g2, cfg));
  PinnedBuffer win;
  win.ensure(kMaxWindowBytes);
  std::vector<double> t;
  uint64_t out[16] = {};
  for (int r = 0; r <= reps; r++) {
    const auto t0 = Clock::now();
    MsmResult res;
    if (fixed_c)
      res = msm_enqueue_fixed(g2, table, in.sc.as<uint64_t>(), n, fixed_c, scratch.ptr,
                              scratch.cap, cfg, st);
    else if (g2)
      res = msm_g2_enqueue(points_soa(in.px.ptr, in.py.ptr), in.sc.as<uint64_t>(), n, scratch.ptr,
                           scratch.cap, cfg, st);
    else
      res = msm_g1_enqueue(points_soa(in.px.ptr, in.py.ptr), in.sc.as<uint64_t>(), n, scratch.ptr,
                           scratch.cap, cfg, st);
    ZK_REQUIRE(res.bytes <= kMaxWindowBytes, ZK_EINTERNAL, "autotune: MSM result too large");
    ZK_CUDA(cudaMemcpyAsync(win.ptr, res.d_data, res.bytes, cudaMemcpyDeviceToHost, st));
    ZK_CUDA(cudaStreamSynchronize(st));
    if (g2)
      msm_g2_combine(win.ptr, res, out);
    else
      msm_g1_combine(win.ptr, res, out);
    if (r) t.push_back(std::chrono::duration<double, std::milli>(Clock::now() - t0).count());
  }
  result.assign(out, out + (g2 ? 16 : 8));
  std::sort(t.begin(), t.end());
  return t[t.size() / 2];
}

struct Search {
  zk_ctx* ctx;
  const Inputs& in;
  int fixed_c;
  const void* table;
  DeviceBuffer scratch;
  std::vector<uint64_t> expect;
  MsmConfig best;
  double best_ms = 1e30;
  int reps;
  Search(zk_ctx* x, const Inputs& i, int f, const void* t, int r)
      : ctx(x), in(i), fixed_c(f), table(t), reps(r) {}
  // `margin`: the fraction by which a candidate must beat the best so far
  void trial(const MsmConfig& cfg, double margin = 0) {
    std::vector<uint64_t> got;
    const double ms = time_msm(ctx, in, cfg, fixed_c, table, scratch, reps, got);
    if (expect.empty()) expect = got;
    ZK_REQUIRE(got == expect, ZK_EINTERNAL, "autotune: MSM settings disagree on the result");
    if (ms < best_ms * (1 - margin)) {
      best_ms = ms;
      best = cfg;
    }
  }
};

int reps_for(int log_n) { return log_n >= 20 ? 3 : 5; }

}  // namespace

TuneResult autotune_msm(zk_ctx* ctx, int group, int log_n, int dist, int fixed_c) {
  ZK_REQUIRE(group == 1 || group == 2, ZK_EINVAL, "autotune: group must be 1 or 2");
  ZK_REQUIRE(log_n >= 4 && log_n <= 24, ZK_EINVAL, "autotune: log_n must be in [4, 24]");
  ZK_REQUIRE(dist == kDistUniform || dist == kDistSkewed, ZK_EINVAL, "autotune: unknown distribution");
  ZK_REQUIRE(fixed_c == 0 || (fixed_c >= 4 && fixed_c <= 22), ZK_EINVAL,
             "autotune: fixed-base window bits must be 0 or 4..22");
  const bool g2 = group == 2;
  const size_t n = size_t(1) << log_n;
  Inputs in;
  make_inputs(ctx, group, n, dist, in);
  DeviceBuffer table;
  if (fixed_c) {
    table.ensure(msm_table_bytes(n, g2, fixed_c));
    msm_precompute(g2, points_soa(in.px.ptr, in.py.ptr), n, fixed_c, table.ptr, ctx->stream);
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  Search s(ctx, in, fixed_c, table.ptr, reps_for(log_n));
  MsmConfig cfg = ctx->msm_cfg[g2 ? 1 : 0];
  cfg.k0 = 64;
  cfg.chunk = 16;
  // Fixed-base MSMs start from the size defaults, which come from timing
  // whole proofs (overlapping MSMs), and leave them only for a clear win:
  // a lone MSM favours shorter dependency chains and its timing is noisy.
  double margin = 0;
  if (fixed_c) {
    cfg.k0 = msm_default_k0(n, true);
    cfg.chunk = msm_default_chunk(n, true, fixed_c);
    margin = 0.02;
  }
  if (!fixed_c) {
    // window bits first (the dominant choice), then the split threshold and
    // the reduction chunk at the best window
    for (int c = std::max(4, log_n - 6); c <= std::min(18, log_n - 1); c++) {
      MsmConfig k = cfg;
      k.c = c;
      s.trial(k);
    }
  } else {
    cfg.c = fixed_c;
    s.trial(cfg);
  }
  for (int k0 : {16, 32, 64, 128, 256}) {
    if (k0 == s.best.k0) continue;
    MsmConfig k = s.best;
    k.k0 = k0;
    s.trial(k, margin);
  }
  for (int chunk : {4, 8, 16, 32, 64}) {
    if (chunk == s.best.chunk) continue;
    MsmConfig k = s.best;
    k.chunk = chunk;
    s.trial(k, margin);
  }
  MsmConfig rec = s.best;
  if (fixed_c) rec.c = 0;  // fixed-base MSMs take c from their table
  ctx->tune.msm[std::make_tuple(group, log_n, dist, fixed_c)] = rec;
  TuneResult r;
  r.cfg = s.best;
  r.table_c = fixed_c;
  r.ms = s.best_ms;
  return r;
}

TuneResult autotune_table_c(zk_ctx* ctx, int group, int log_n, int dist, size_t max_table_bytes) {
  ZK_REQUIRE(group == 1 || group == 2, ZK_EINVAL, "autotune: group must be 1 or 2");
  ZK_REQUIRE(log_n >= 4 && log_n <= 24, ZK_EINVAL, "autotune: log_n must be in [4, 24]");
  ZK_REQUIRE(dist == kDistUniform || dist == kDistSkewed, ZK_EINVAL, "autotune: unknown distribution");
  const bool g2 = group == 2;
  const size_t n = size_t(1) << log_n;
  Inputs in;
  make_inputs(ctx, group, n, dist, in);
  DeviceBuffer table, scratch;
  std::vector<uint64_t> expect, got;
  TuneResult best;
  best.ms = 1e30;
  for (int c = std::max(6, log_n - 4); c <= std::min(22, log_n + 2); c++) {
    const size_t tb = msm_table_bytes(n, g2, c);
    if (max_table_bytes && tb > max_table_bytes) continue;
    table.ensure(tb);
    msm_precompute(g2, points_soa(in.px.ptr, in.py.ptr), n, c, table.ptr, ctx->stream);
    MsmConfig cfg = msm_config_for(ctx, g2, n, dist, c);
    cfg.c = c;
    const double ms = time_msm(ctx, in, cfg, c, table.ptr, scratch, reps_for(log_n), got);
    if (expect.empty()) expect = got;
    ZK_REQUIRE(got == expect, ZK_EINTERNAL, "autotune: table sizes disagree on the result");
    if (ms < best.ms) {
      best.ms = ms;
      best.table_c = c;
      best.cfg = cfg;
    }
  }
  ZK_REQUIRE(best.table_c, ZK_EINVAL, "autotune: no table fits the memory cap");
  ctx->tune.table_c[std::make_tuple(group, log_n, dist)] = best.table_c;
  return best;
}

TuneResult autotune_ntt(zk_ctx* ctx, int log_n) {
  ZK_REQUIRE(log_n >= 2 && log_n < kMaxLogN, ZK_EINVAL, "autotune: log_n out of range");
  cudaStream_t st = ctx->stream;
  const size_t n = size_t(1) << log_n;
  DeviceBuffer a, b, c, h;
  a.ensure(32 * n);
  b.ensure(32 * n);
  c.ensure(32 * n);
  h.ensure(32 * n);
  std::vector<uint64_t> v;
  make_scalars(n, kDistUniform, 0x5eed0003ull + n, v);
  ZK_CUDA(cudaMemcpyAsync(a.ptr, v.data(), 32 * n, cudaMemcpyHostToDevice, st));
  ZK_CUDA(cudaMemcpyAsync(b.ptr, v.data(), 32 * n, cudaMemcpyHostToDevice, st));
  ctx->ntt.ensure(log_n, st);
  cudaEvent_t e0, e1;
  ZK_CUDA(cudaEventCreate(&e0));
  ZK_CUDA(cudaEventCreate(&e1));
  TuneResult best;
  best.ms = 1e30;
  const int saved = ctx->ntt.pass_bits[log_n];
  int last_np = -1;
  for (int bits = kMaxPassBits; bits >= 4; bits--) {
    const int np = (log_n + bits - 1) / bits;
    if (np == last_np) continue;  // same split as a larger radix
    last_np = np;
    ctx->ntt.pass_bits[log_n] = bits;
    std::vector<float> t;
    for (int r = 0; r <= 5; r++) {
      ZK_CUDA(cudaEventRecord(e0, st));
      hpoly(ctx->ntt, a.as<uint64_t>(), b.as<uint64_t>(), c.as<uint64_t>(), log_n, h.as<uint64_t>(),
            st);
      ZK_CUDA(cudaEventRecord(e1, st));
      ZK_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      ZK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (r) t.push_back(ms);
    }
    std::sort(t.begin(), t.end());
    if (t[t.size() / 2] < best.ms) {
      best.ms = t[t.size() / 2];
      best.pass_bits = bits;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->ntt.pass_bits[log_n] = best.pass_bits ? best.pass_bits : saved;
  return best;
}

std::string tune_export(const zk_ctx* ctx) {
  std::ostringstream o;
  for (const auto& e : ctx->tune.msm) {
    const MsmConfig& m = e.second;
    o << "msm " << std::get<0>(e.first) << ' ' << std::get<1>(e.first) << ' '
      << std::get<2>(e.first) << ' ' << std::get<3>(e.first) << ' ' << m.c << ' ' << m.k0 << ' '
      << m.k1 << ' ' << m.chunk << '\n';
  }
  for (const auto& e : ctx->tune.table_c)
    o << "table " << std::get<0>(e.first) << ' ' << std::get<1>(e.first) << ' '
      << std::get<2>(e.first) << ' ' << e.second << '\n';
  for (int l = 0; l <= kMaxLogN; l++)
    if (ctx->ntt.pass_bits[l] != kMaxPassBits) o << "ntt " << l << ' ' << ctx->ntt.pass_bits[l] << '\n';
  return o.str();
}

void tune_import(zk_ctx* ctx, const char* text) {
  std::istringstream in(text ? text : "");
  std::string line;
  TuneTable t = ctx->tune;
  int bits[kMaxLogN + 1];
  memcpy(bits, ctx->ntt.pass_bits, sizeof(bits));
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string kind;
    if (!(ls >> kind) || kind[0] == '#') continue;
    if (kind == "msm") {
      int g, l, d, f;
      MsmConfig m;
      ZK_REQUIRE(bool(ls >> g >> l >> d >> f >> m.c >> m.k0 >> m.k1 >> m.chunk), ZK_EINVAL,
                 "tune import: malformed msm line");
      ZK_REQUIRE((g == 1 || g == 2) && l >= 0 && l <= 31 && (d == 0 || d == 1) && f >= 0 &&
                     f <= 22 && (m.c == 0 || (m.c >= 4 && m.c <= 21)) && m.k0 >= 1 &&
                     m.k0 <= 4096 && m.k1 >= 2 && m.k1 <= 4096 && m.chunk >= 2 &&
                     m.chunk <= 4096 && (m.chunk & (m.chunk - 1)) == 0,
                 ZK_EINVAL, "tune import: msm settings out of range");
      t.msm[std::make_tuple(g, l, d, f)] = m;
    } else if (kind == "table") {
      int g, l, d, c;
      ZK_REQUIRE(bool(ls >> g >> l >> d >> c), ZK_EINVAL, "tune import: malformed table line");
      ZK_REQUIRE((g == 1 || g == 2) && l >= 0 && l <= 31 && (d == 0 || d == 1) && c >= 4 && c <= 22,
                 ZK_EINVAL, "tune import: table settings out of range");
      t.table_c[std::make_tuple(g, l, d)] = c;
    } else if (kind == "ntt") {
      int l, b;
      ZK_REQUIRE(bool(ls >> l >> b), ZK_EINVAL, "tune import: malformed ntt line");
      ZK_REQUIRE(l >= 0 && l <= kMaxLogN && b >= 4 && b <= kMaxPassBits, ZK_EINVAL,
                 "tune import: ntt settings out of range");
      bits[l] = b;
    } else {
      throw Error(ZK_EINVAL, "tune import: unknown line kind '" + kind + "'");
    }
  }
  ctx->tune = t;
  memcpy(ctx->ntt.pass_bits, bits, sizeof(bits));
}

}  // namespace zk

// ---------------------------------------------------------------- C ABI
namespace {
void fill(zk_tune_result* out, const zk::TuneResult& r) {
  if (!out) return;
  out->c = r.cfg.c;
  out->k0 = r.cfg.k0;
  out->k1 = r.cfg.k1;
  out->chunk = r.cfg.chunk;
  out->table_c = r.table_c;
  out->pass_bits = r.pass_bits;
  out->ms = r.ms;
}
}  // namespace

extern "C" {

int zk_autotune_msm(zk_ctx* ctx, int group, int log_n, int dist, int fixed_c, zk_tune_result* out) {
  ZK_API_BEGIN
  ctx = zk::resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  fill(out, zk::autotune_msm(ctx, group, log_n, dist, fixed_c));
  ZK_API_END
}

int zk_autotune_table_c(zk_ctx* ctx, int group, int log_n, int dist, size_t max_table_bytes,
                        zk_tune_result* out) {
  ZK_API_BEGIN
  ctx = zk::resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  fill(out, zk::autotune_table_c(ctx, group, log_n, dist, max_table_bytes));
  ZK_API_END
}

int zk_autotune_ntt(zk_ctx* ctx, int log_n, zk_tune_result* out) {
  ZK_API_BEGIN
  ctx = zk::resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  fill(out, zk::autotune_ntt(ctx, log_n));
  ZK_API_END
}

int zk_tune_export(zk_ctx* ctx, char* buf, size_t cap, size_t* len) {
  ZK_API_BEGIN
  ctx = zk::resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  const std::string s = zk::tune_export(ctx);
  if (len) *len = s.size();
  ZK_REQUIRE(!buf || cap > s.size(), ZK_EINVAL, "zk_tune_export: buffer too small");
  if (buf) memcpy(buf, s.c_str(), s.size() + 1);
  ZK_API_END
}

int zk_tune_import(zk_ctx* ctx, const char* text) {
  ZK_API_BEGIN
  ctx = zk::resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  zk::tune_import(ctx, text);
  ZK_API_END
}

int zk_ctx_set_scalar_dist(zk_ctx* ctx, int dist) {
  ZK_API_BEGIN
  ctx = zk::resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ZK_REQUIRE(dist == 0 || dist == 1, ZK_EINVAL, "zk_ctx_set_scalar_dist: 0 (uniform) or 1 (skewed)");
  ctx->scalar_dist = dist;
  ZK_API_END
}

int zk_circuit_set_scalar_dist(zk_circuit* c, int dist) {
  ZK_API_BEGIN
  ZK_REQUIRE(c, ZK_EINVAL, "zk_circuit_set_scalar_dist: NULL circuit");
  ZK_REQUIRE(dist >= -1 && dist <= 1, ZK_EINVAL,
             "zk_circuit_set_scalar_dist: -1 (detect), 0 (uniform) or 1 (skewed)");
  zk::enter_ctx(c->ctx);
  std::lock_guard<std::mutex> g(c->ctx->mu);
  c->dist_auto = dist < 0;
  c->dist = dist < 0 ? 0 : dist;
  ZK_API_END
}

}  // extern "C"
