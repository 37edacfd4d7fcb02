// Groth16 prover on sm_100a (see prover.hpp).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <utility>
#include <vector>

#include "field.cuh"
#include "host_field.hpp"
#include "msm.hpp"
#include "profile.hpp"
#include "prover.hpp"
#include "scan.cuh"

namespace zk {
namespace {

// ------------------------------------------------- section-4 CSR (device)
// Entries are 11 u32 words: matrix, constraint, signal, value[8] (coef*R^2).
// Matrices other than A (0) and B (1) are skipped, as in the reference
// (src/groth16.cu:758-763); out-of-range rows / signals are counted as bad.
__global__ void k_coef_count(const uint32_t* __restrict__ raw, uint32_t nnz, uint32_t n,
                             uint32_t m1, uint32_t* __restrict__ cnt_a,
                             uint32_t* __restrict__ cnt_b, uint32_t* __restrict__ bad) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  const uint32_t* p = raw + 11 * e;
  const uint32_t mat = p[0], rowi = p[1], s = p[2];
  if (mat > 1) return;
  if (rowi >= n || s >= m1) {
    atomicAdd(bad, 1u);
    return;
  }
  atomicAdd(mat == 0 ? &cnt_a[rowi] : &cnt_b[rowi], 1u);
}

__global__ void k_coef_scatter(const uint32_t* __restrict__ raw, uint32_t nnz, uint32_t n,
                               uint32_t m1, uint32_t* __restrict__ cur_a,
                               uint32_t* __restrict__ cur_b, uint32_t* __restrict__ sig_a,
                               uint32_t* __restrict__ sig_b, uint32_t* __restrict__ val_a,
                               uint32_t* __restrict__ val_b) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  const uint32_t* p = raw + 11 * e;
  const uint32_t mat = p[0], rowi = p[1], s = p[2];
  if (mat > 1 || rowi >= n || s >= m1) return;
  const uint32_t pos = atomicAdd(mat == 0 ? &cur_a[rowi] : &cur_b[rowi], 1u);
  (mat == 0 ? sig_a : sig_b)[pos] = s;
  uint4* dst = reinterpret_cast<uint4*>((mat == 0 ? val_a : val_b) + 8 * (size_t)pos);
  dst[0] = make_uint4(p[3], p[4], p[5], p[6]);
  dst[1] = make_uint4(p[7], p[8], p[9], p[10]);
}

// Aw / Bw rows: sum_k (coef_k R^2) * w[sig_k] = coef . w in Montgomery form
// without an encode pass (src/groth16.cu:144-167).  w is canonical.
struct SpmvArgs {
  const uint32_t* row[2];
  const uint32_t* sig[2];
  const fr_t* val[2];
  fr_t* out[2];
};

__global__ void __launch_bounds__(256) k_spmv(SpmvArgs a, const fr_t* __restrict__ w, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int m = blockIdx.y;
  const uint32_t b = a.row[m][i], e = a.row[m][i + 1];
  fr_t acc = fe_zero<FrCfg>();
  for (uint32_t k = b; k < e; k++)
    acc = acc + fe_mul_inline(fe_ldg<FrCfg>(a.val[m], k), fe_ldg<FrCfg>(w, a.sig[m][k]));
  fe_store(a.out[m], i, acc);
}

unsigned blocks(size_t n, int th) { return (unsigned)((n + th - 1) / th); }

// ------------------------------------------------------ host group math
using G1 = host::Xyzz<host::Fp>;
using G2 = host::Xyzz<host::Fp2>;

host::Fp fp(const uint64_t* p) { return host::Fp::from_raw(p); }
host::Fp2 fp2(const uint64_t* p) { return host::Fp2{fp(p), fp(p + 4)}; }
G1 g1_aff(const uint64_t* p) { return G1::from_affine(fp(p), fp(p + 4)); }
G2 g2_aff(const uint64_t* p) { return G2::from_affine(fp2(p), fp2(p + 8)); }
void put_g1(const host::Fp& x, const host::Fp& y, uint64_t* out) {
  memcpy(out, x.v, 32);
  memcpy(out + 4, y.v, 32);
}
void put_g2(const host::Fp2& x, const host::Fp2& y, uint64_t* out) {
  memcpy(out, x.c0.v, 32);
  memcpy(out + 4, x.c1.v, 32);
  memcpy(out + 8, y.c0.v, 32);
  memcpy(out + 12, y.c1.v, 32);
}
int g1_out(const G1& g, uint64_t* out) {
  host::Fp x, y;
  const bool inf = g.to_affine(x, y);
  put_g1(x, y, out);
  return inf ? 1 : 0;
}
int g2_out(const G2& g, uint64_t* out) {
  host::Fp2 x, y;
  const bool inf = g.to_affine(x, y);
  put_g2(x, y, out);
  return inf ? 1 : 0;
}
template <class P>
P mul(const P& p, const uint64_t* k) {
  P acc = P::inf();
  for (int i = 255; i >= 0; i--) {
    acc = acc.dbl();
    if ((k[i >> 6] >> (i & 63)) & 1) acc = acc.add(p);
  }
  return acc;
}

}  // namespace

void ProveWs::init() {
  if (ready) return;
  ZK_CUDA(cudaEventCreateWithFlags(&ev_all, cudaEventDisableTiming));
  // ZYKLOP_PROVE_STREAMS=1 runs a proof's MSMs back to back on one stream
  // (a tuning knob: concurrent MSMs share L2 and the SMs)
  if (const char* e = getenv("ZYKLOP_PROVE_STREAMS")) {
    const int v = atoi(e);
    if (v >= 1 && v <= kStreams) env_nstreams = v;
  }
  // Stream priorities order block dispatch among a proof's MSM chains when
  // the proof runs alone: the B2 (G2) MSM, the longest chain, first; then
  // stream 0, whose H MSM starts only after the SpMV and the H pipeline; A,
  // C and B1 fill the SMs left over.  Measured on a 2^20 proof: 22.9 ms
  // against 23.4 ms with equal priorities (B2 alone first, or the H chain
  // alone or first, gave less).  Beside other proofs (in-flight batches, the
  // server) every proof's B2 would outrank the rest of the device's work:
  // batches ran ~10 % slower, so those workspaces keep equal priorities.
  int least = 0, greatest = 0;
  ZK_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  for (int i = 0; i < kStreams; i++) {
    const int prio = !ordered ? least : (i == 2 ? greatest : (i == 0 ? greatest / 2 : least));
    ZK_CUDA(cudaStreamCreateWithPriority(&st[i], cudaStreamNonBlocking, prio));
    ZK_CUDA(cudaEventCreateWithFlags(&ev_done[i], cudaEventDisableTiming));
  }
  ZK_CUDA(cudaEventCreateWithFlags(&ev_we, cudaEventDisableTiming));
  ZK_CUDA(cudaEventCreateWithFlags(&ev_begin, cudaEventDisableTiming));
  ZK_CUDA(cudaEventCreateWithFlags(&ev_merge, cudaEventDisableTiming));
  ready = true;
}

ProveWs::~ProveWs() {
  if (!ready) return;
  for (int i = 0; i < kStreams; i++) {
    cudaStreamSynchronize(st[i]);
    cudaStreamDestroy(st[i]);
    cudaEventDestroy(ev_done[i]);
  }
  cudaEventDestroy(ev_we);
  cudaEventDestroy(ev_merge);
  cudaEventDestroy(ev_begin);
  cudaEventDestroy(ev_all);
  drop_graph();
}

namespace {

// Sizes and verification-key points of a parsed zkey (no device work).
std::unique_ptr<zk_circuit> circuit_header(zk_ctx* ctx, const ZkeyView& z) {
  std::unique_ptr<zk_circuit> c(new zk_circuit());
  c->ctx = ctx;
  c->id = next_circuit_id();
  c->m1 = z.n_vars;
  c->l = z.n_public;
  c->n = z.domain;
  c->log_n = z.log_n;
  c->n_coefs = z.n_coefs;
  ZK_REQUIRE(c->log_n >= 1, ZK_EFORMAT, "zkey: domain must be at least 2");
  memcpy(c->alpha1, z.alpha1, 64);
  memcpy(c->beta1, z.beta1, 64);
  memcpy(c->beta2, z.beta2, 128);
  memcpy(c->gamma2, z.gamma2, 128);
  memcpy(c->delta1, z.delta1, 64);
  memcpy(c->delta2, z.delta2, 128);
  if (z.ic) c->ic.assign(z.ic, z.ic + 8 * ((size_t)c->l + 1));
  c->has_b1 = z.b1 != nullptr;
  return c;
}

enum PointSet { kSetA, kSetB1, kSetB2, kSetC, kSetH };

// Uploads one CRS point set on `st` (record 0 of A / B1 / B2 is alpha1 /
// beta1 / beta2, like the reference's extended buffers,
// src/groth16.cu:1199-1227).  Returns once the host source may be released;
// the copy completes in stream order.
void upload_points(zk_circuit* c, const ZkeyView& z, PointSet set, cudaStream_t st, Stager& sg) {
  const size_t m1 = c->m1, nc = m1 - c->l - 1;
  switch (set) {
    case kSetA:
      c->pts_a.ensure(64 * (m1 + 1));
      ZK_CUDA(cudaMemcpyAsync(c->pts_a.ptr, c->alpha1, 64, cudaMemcpyHostToDevice, st));
      sg.upload(c->pts_a.as<char>() + 64, z.a, 64 * m1, st);
      break;
    case kSetB1:
      if (!z.b1) return;
      c->pts_b1.ensure(64 * (m1 + 1));
      ZK_CUDA(cudaMemcpyAsync(c->pts_b1.ptr, c->beta1, 64, cudaMemcpyHostToDevice, st));
      sg.upload(c->pts_b1.as<char>() + 64, z.b1, 64 * m1, st);
      break;
    case kSetB2:
      c->pts_b2.ensure(128 * (m1 + 1));
      ZK_CUDA(cudaMemcpyAsync(c->pts_b2.ptr, c->beta2, 128, cudaMemcpyHostToDevice, st));
      sg.upload(c->pts_b2.as<char>() + 128, z.b2, 128 * m1, st);
      break;
    case kSetC:
      c->pts_c.ensure(64 * (nc ? nc : 1));
      sg.upload(c->pts_c.ptr, z.c, 64 * nc, st);
      break;
    case kSetH:
      c->pts_h.ensure(64 * (size_t)c->n);
      sg.upload(c->pts_h.ptr, z.h, 64 * (size_t)c->n, st);
      break;
  }
}

// Section 4 -> CSR on the device (the reference builds it on the host,
// src/groth16.cu:737-809).  Enqueued on `st`; *h_bad receives the count of
// entries outside the domain or witness once `st` reaches the copy.
struct CsrScratch {
  DeviceBuffer raw, tmp;
};
void build_csr(zk_circuit* c, const ZkeyView& z, cudaStream_t st, Stager& sg, CsrScratch& s,
               uint32_t* h_bad) {
  const size_t nnz = c->n_coefs, n = c->n;
  s.raw.ensure(44 * (nnz ? nnz : 1));
  sg.upload(s.raw.ptr, z.coefs, 44 * nnz, st);
  const size_t tiles = scan::tile_count(n + 1) + 1;
  auto carve_csr_tmp = [&](void* base, uint32_t** cnt, uint32_t** cur, uint32_t** tl,
                           uint32_t** bad) {
    Carver cv(base);
    for (int m = 0; m < 2; m++) cnt[m] = cv.take<uint32_t>(n + 1);
    for (int m = 0; m < 2; m++) cur[m] = cv.take<uint32_t>(n + 1);
    for (int m = 0; m < 2; m++) tl[m] = cv.take<uint32_t>(tiles);
    *bad = cv.take<uint32_t>(1);
    return cv.off;
  };
  uint32_t *cnt[2], *cur[2], *tl[2], *bad;
  s.tmp.ensure(carve_csr_tmp(nullptr, cnt, cur, tl, &bad));  // dry run: size with padding
  carve_csr_tmp(s.tmp.ptr, cnt, cur, tl, &bad);
  ZK_CUDA(cudaMemsetAsync(s.tmp.ptr, 0, s.tmp.cap, st));
  for (int m = 0; m < 2; m++) {
    c->row[m].ensure(4 * (n + 1));
    c->sig[m].ensure(4 * (nnz ? nnz : 1));
    c->val[m].ensure(32 * (nnz ? nnz : 1));
  }
  if (nnz) {
    k_coef_count<<<blocks(nnz, 256), 256, 0, st>>>(s.raw.as<uint32_t>(), (uint32_t)nnz, (uint32_t)n,
                                                  c->m1, cnt[0], cnt[1], bad);
    ZK_LAUNCHED();
  }
  for (int m = 0; m < 2; m++) scan::exclusive(cnt[m], cur[m], n + 1, tl[m], st);
  if (nnz) {
    k_coef_scatter<<<blocks(nnz, 256), 256, 0, st>>>(
        s.raw.as<uint32_t>(), (uint32_t)nnz, (uint32_t)n, c->m1, cur[0], cur[1],
        c->sig[0].as<uint32_t>(), c->sig[1].as<uint32_t>(), c->val[0].as<uint32_t>(),
        c->val[1].as<uint32_t>());
    ZK_LAUNCHED();
  }
  for (int m = 0; m < 2; m++)
    ZK_CUDA(cudaMemcpyAsync(c->row[m].ptr, cnt[m], 4 * (n + 1), cudaMemcpyDeviceToDevice, st));
  ZK_CUDA(cudaMemcpyAsync(h_bad, bad, 4, cudaMemcpyDeviceToHost, st));
}

}  // namespace

zk_circuit* circuit_load(zk_ctx* ctx, const BinFile& f) {
  const ZkeyView z = parse_zkey(f);
  std::unique_ptr<zk_circuit> c = circuit_header(ctx, z);
  cudaStream_t st = ctx->stream;
  Stager& sg = ctx->stager;
  for (PointSet set : {kSetA, kSetB2, kSetB1, kSetC, kSetH}) upload_points(c.get(), z, set, st, sg);
  CsrScratch scratch;
  uint32_t h_bad = 0;
  build_csr(c.get(), z, st, sg, scratch, &h_bad);
  ZK_CUDA(cudaStreamSynchronize(st));
  ZK_REQUIRE(h_bad == 0, ZK_EFORMAT, "zkey: section 4 has entries outside the domain or witness");
  ctx->ntt.ensure(c->log_n, st);
  return c.release();
}

int msm_fixed_default_c(size_t n, bool g2) {
  int lg = 0;
  while ((size_t(1) << lg) < n) lg++;
  int c = lg;
  (void)g2;
  if (c < 8) c = 8;
  if (c > 20) c = 20;
  return c;
}

void circuit_precompute(zk_circuit* c, int c_g1, int c_g2) {
  zk_ctx* ctx = c->ctx;
  cudaStream_t st = ctx->stream;
  const size_t m1 = c->m1, nc = (size_t)c->m1 - c->l - 1, n = c->n;
  const int g1c = c_g1 ? c_g1 : table_c_for(ctx, false, m1 + 1, c->dist);
  const int g2c = c_g2 ? c_g2 : table_c_for(ctx, true, m1 + 1, c->dist);
  ZK_REQUIRE(g1c >= 4 && g1c <= 22 && g2c >= 4 && g2c <= 22, ZK_EINVAL,
             "precompute: window bits must be in [4, 22]");
  auto build = [&](DeviceBuffer& tab, const DeviceBuffer& pts, size_t cnt, bool g2, int cb) {
    tab.ensure(msm_table_bytes(cnt ? cnt : 1, g2, cb));
    msm_precompute(g2, points_aos(pts.ptr, g2), cnt, cb, tab.ptr, st);
  };
  build(c->tab_a, c->pts_a, m1 + 1, false, g1c);
  build(c->tab_b2, c->pts_b2, m1 + 1, true, g2c);
  build(c->tab_c_pts, c->pts_c, nc, false, g1c);
  build(c->tab_h, c->pts_h, n, false, g1c);
  if (c->has_b1) build(c->tab_b1, c->pts_b1, m1 + 1, false, g1c);
  ZK_CUDA(cudaStreamSynchronize(st));
  c->tab_c[0] = g1c;
  c->tab_c[1] = g2c;
}

namespace {

std::atomic<uint64_t> g_circuit_ids{1};

// Settings of each of a proof's MSMs (indexed like ProveWs::msm): H's
// scalars are NTT outputs (uniform), the others are witness values.
void ws_msm_configs(zk_circuit* c, MsmConfig cfg[ProveWs::kStreams]) {
  const zk_ctx* ctx = c->ctx;
  const size_t m1 = c->m1, nc = m1 - c->l - 1;
  const int f1 = c->tab_c[0], f2 = c->tab_c[1];
  cfg[0] = msm_config_for(ctx, false, c->n, kDistUniform, f1);
  cfg[1] = msm_config_for(ctx, false, m1 + 1, c->dist, f1);
  cfg[2] = msm_config_for(ctx, true, m1 + 1, c->dist, f2);
  cfg[3] = msm_config_for(ctx, false, nc, c->dist, f1);
  cfg[4] = msm_config_for(ctx, false, m1 + 1, c->dist, f1);
}

// MSM scratch bytes of each of a proof's MSMs.
void ws_scratch_needs(zk_circuit* c, bool blind, const MsmConfig cfg[ProveWs::kStreams],
                      size_t need[ProveWs::kStreams]) {
  const size_t m1 = c->m1, n = c->n, nc = m1 - c->l - 1;
  const bool fixed = c->tab_c[0] != 0;
  auto scratch = [&](int i, size_t cnt, bool g2) {
    return fixed ? msm_scratch_bytes_fixed(cnt, g2, c->tab_c[g2 ? 1 : 0], cfg[i])
                 : msm_scratch_bytes(cnt, g2, cfg[i]);
  };
  need[0] = scratch(0, n, false);
  need[1] = scratch(1, m1 + 1, false);
  need[2] = scratch(2, m1 + 1, true);
  need[3] = scratch(3, nc, false);
  need[4] = blind ? scratch(4, m1 + 1, false) : 0;
}

// Sizes the workspace for this circuit (buffers, MSM scratch, result copies).
void ws_prepare(zk_circuit* c, ProveWs& ws, bool blind) {
  zk_ctx* ctx = c->ctx;
  ws.init();
  ws.nstreams = ctx->prove_streams ? ctx->prove_streams : ws.env_nstreams;
  const size_t m1 = c->m1, n = c->n;
  ws_msm_configs(c, ws.cfg);
  size_t need[ProveWs::kStreams];
  ws_scratch_needs(c, blind, ws.cfg, need);
  const bool grow = ws.we.cap < 32 * (m1 + 1) || ws.aw.cap < 32 * n ||
                    [&] {
                      for (int i = 0; i < ProveWs::kStreams; i++)
                        if (ws.msm[i].cap < need[i]) return true;
                      return false;
                    }();
  if (grow) {
    for (int i = 0; i < ProveWs::kStreams; i++) ZK_CUDA(cudaStreamSynchronize(ws.st[i]));
    ws.drop_graph();  // captured addresses change
  }
  ws.we.ensure(32 * (m1 + 1));
  ws.aw.ensure(32 * n);
  ws.bw.ensure(32 * n);
  ws.cw.ensure(32 * n);
  ws.h.ensure(32 * n);
  for (int i = 0; i < ProveWs::kStreams; i++) {
    if (need[i]) ws.msm[i].ensure(need[i]);
    ws.win[i].ensure(kMaxWindowBytes);
  }
  ctx->ntt.ensure(c->log_n, ws.st[0]);
}

// Witness into we = [1 || w_0 .. w_{m1-1}] on stream 0 (src/groth16.cu:1316-1326).
void ws_stage(zk_circuit* c, ProveWs& ws, const uint64_t* witness, bool on_device,
              Stager& stager) {
  cudaStream_t s0 = ws.st[0];
  uint64_t* we = ws.we.as<uint64_t>();
  ZK_CUDA(cudaMemsetAsync(we, 0, 32, s0));
  ZK_CUDA(cudaMemsetAsync(we, 1, 1, s0));
  if (on_device)
    ZK_CUDA(cudaMemcpyAsync(we + 4, witness, 32 * (size_t)c->m1, cudaMemcpyDeviceToDevice, s0));
  else
    stager.upload(we + 4, witness, 32 * (size_t)c->m1, s0);
}

// MSM i of a proof (indexed like ProveWs::msm) on stream i mod nstreams,
// after the staged witness; its window sums land in ws.win[i] and
// ev_done[i] marks them.  `mo` / `mi`: the C and H MSMs share one bucket
// reduction (msm.hpp, MsmMerge); C's own result is then empty.
void ws_msm(zk_circuit* c, ProveWs& ws, int i, bool g2, const DeviceBuffer& pts,
            const DeviceBuffer& tab, const uint64_t* sc, size_t cnt, MsmMerge* mo = nullptr,
            const MsmMerge* mi = nullptr) {
  const bool fixed = c->tab_c[0] != 0;
  const int si = i % ws.nstreams;
  cudaStream_t st = ws.st[si];
  if (si) ZK_CUDA(cudaStreamWaitEvent(st, ws.ev_we, 0));
  if (fixed)
    ws.res[i] = msm_enqueue_fixed(g2, tab.ptr, sc, cnt, c->tab_c[g2 ? 1 : 0], ws.msm[i].ptr,
                                  ws.msm[i].cap, ws.cfg[i], st, mo, mi);
  else if (g2)
    ws.res[i] = msm_g2_enqueue(points_aos(pts.ptr, true), sc, cnt, ws.msm[i].ptr, ws.msm[i].cap,
                               ws.cfg[i], st);
  else
    ws.res[i] = msm_g1_enqueue(points_aos(pts.ptr, false), sc, cnt, ws.msm[i].ptr, ws.msm[i].cap,
                               ws.cfg[i], st, mo, mi);
  ZK_REQUIRE(ws.res[i].bytes <= kMaxWindowBytes, ZK_EINTERNAL, "prove: MSM result too large");
  if (ws.res[i].bytes)
    ZK_CUDA(cudaMemcpyAsync(ws.win[i].ptr, ws.res[i].d_data, ws.res[i].bytes,
                            cudaMemcpyDeviceToHost, st));
  ZK_CUDA(cudaEventRecord(ws.ev_done[i], st));
}

// Whether the C MSM (index 3) and the H MSM (index 0) of a proof can share
// one bucket reduction: pi_C adds their results, so they can when both run
// with the same window bits (fixed-base: always, one G1 table size).
bool ws_merge_ch(const zk_circuit* c, const ProveWs& ws) {
  if (c->tab_c[0] != 0) return true;
  const size_t nc = c->m1 - c->l - 1;
  return msm_effective_c(nc, false, ws.cfg[3]) == msm_effective_c(c->n, false, ws.cfg[0]);
}

// The device part of a proof, from the staged witness to the MSM results in
// pinned host memory.  It begins and ends on stream 0 (other streams fork
// from and join back to it), issues no synchronizing call, and can therefore
// be captured into a CUDA graph.
void ws_pipeline(zk_circuit* c, ProveWs& ws, bool blind, ProveIntermediates* dbg) {
  zk_ctx* ctx = c->ctx;
  const size_t m1 = c->m1, n = c->n, l = c->l, nc = m1 - l - 1;
  cudaStream_t s0 = ws.st[0];
  uint64_t* we = ws.we.as<uint64_t>();
  ZK_CUDA(cudaEventRecord(ws.ev_we, s0));
  auto launch = [&](int i, bool g2, const DeviceBuffer& pts, const DeviceBuffer& tab,
                    const uint64_t* sc, size_t cnt) { ws_msm(c, ws, i, g2, pts, tab, sc, cnt); };
  // C leaves its buckets to H's reduction unless intermediates want each
  // MSM's own result
  const bool merge = !dbg && ws_merge_ch(c, ws);
  ws.merge_c = MsmMerge{};
  ws.merge_c.ready = ws.ev_merge;
  launch(1, false, c->pts_a, c->tab_a, we, m1 + 1);
  launch(2, true, c->pts_b2, c->tab_b2, we, m1 + 1);
  ws_msm(c, ws, 3, false, c->pts_c, c->tab_c_pts, we + 4 * (l + 2), nc,
         merge ? &ws.merge_c : nullptr);
  if (blind) launch(4, false, c->pts_b1, c->tab_b1, we, m1 + 1);

  spmv_enqueue(c, we, ws.aw.as<uint64_t>(), ws.bw.as<uint64_t>(), s0);
  if (dbg && (dbg->aw || dbg->bw)) {
    if (dbg->aw) ZK_CUDA(cudaMemcpyAsync(dbg->aw, ws.aw.ptr, 32 * n, cudaMemcpyDeviceToHost, s0));
    if (dbg->bw) ZK_CUDA(cudaMemcpyAsync(dbg->bw, ws.bw.ptr, 32 * n, cudaMemcpyDeviceToHost, s0));
  }
  hpoly(ctx->ntt, ws.aw.as<uint64_t>(), ws.bw.as<uint64_t>(), ws.cw.as<uint64_t>(), c->log_n,
        ws.h.as<uint64_t>(), s0);
  if (dbg) {
    // the H pipeline leaves the coset evaluations of A, B and C in aw, bw, cw
    const std::pair<uint64_t*, const DeviceBuffer*> outs[] = {
        {dbg->h, &ws.h}, {dbg->ea, &ws.aw}, {dbg->eb, &ws.bw}, {dbg->ec, &ws.cw}};
    for (const auto& o : outs)
      if (o.first) ZK_CUDA(cudaMemcpyAsync(o.first, o.second->ptr, 32 * n, cudaMemcpyDeviceToHost, s0));
  }
  ws_msm(c, ws, 0, false, c->pts_h, c->tab_h, ws.h.as<uint64_t>(), n, nullptr,
         merge ? &ws.merge_c : nullptr);
  for (int i = 1; i < (blind ? 5 : 4); i++) ZK_CUDA(cudaStreamWaitEvent(s0, ws.ev_done[i], 0));
}

// Runs the pipeline directly or as a replay of its captured graph.
void ws_launch(zk_circuit* c, ProveWs& ws, bool blind, bool use_graph, ProveIntermediates* dbg) {
  if (!use_graph || dbg) {
    ws_pipeline(c, ws, blind, dbg);
    return;
  }
  const zk_ctx* ctx = c->ctx;
  const int lmax = ctx->ntt.lmax, bits = ctx->ntt.pass_bits[c->log_n];
  auto same_cfg = [&](const ProveWs::Graph& x) {
    for (int i = 0; i < ProveWs::kStreams; i++)
      if (!(x.cfg[i] == ws.cfg[i])) return false;
    return true;
  };
  ProveWs::Graph* gr = nullptr;
  for (ProveWs::Graph& x : ws.graphs)
    if (x.circuit == c->id && x.blind == blind && x.ntt_lmax == lmax && x.ntt_bits == bits &&
        x.nstreams == ws.nstreams &&
        same_cfg(x) && x.tab_c[0] == c->tab_c[0] && x.tab_c[1] == c->tab_c[1])
      gr = &x;
  if (!gr) {
    if (ws.graphs.size() >= ProveWs::kMaxGraphs) {
      cudaGraphExecDestroy(ws.graphs.front().exec);
      ws.graphs.erase(ws.graphs.begin());
    }
    Profiler* saved = current_profiler();
    set_current_profiler(nullptr);  // no timing events inside a capture
    const uint64_t l0 = launch_count();
    cudaGraph_t g = nullptr;
    ZK_CUDA(cudaStreamBeginCapture(ws.st[0], cudaStreamCaptureModeThreadLocal));
    try {
      ws_pipeline(c, ws, blind, nullptr);
    } catch (...) {
      cudaStreamEndCapture(ws.st[0], &g);
      if (g) cudaGraphDestroy(g);
      set_current_profiler(saved);
      throw;
    }
    ZK_CUDA(cudaStreamEndCapture(ws.st[0], &g));
    set_current_profiler(saved);
    ProveWs::Graph x;
    const cudaError_t e = cudaGraphInstantiate(&x.exec, g, 0);
    cudaGraphDestroy(g);
    ZK_CUDA(e);
    x.kernels = launch_count() - l0;
    x.circuit = c->id;
    x.blind = blind;
    x.ntt_lmax = lmax;
    x.ntt_bits = bits;
    x.nstreams = ws.nstreams;
    for (int i = 0; i < ProveWs::kStreams; i++) x.cfg[i] = ws.cfg[i];
    x.tab_c[0] = c->tab_c[0];
    x.tab_c[1] = c->tab_c[1];
    for (int i = 0; i < ProveWs::kStreams; i++) x.res[i] = ws.res[i];
    ws.graphs.push_back(x);
    gr = &ws.graphs.back();
  }
  // the host combine reads these; another circuit's run may have replaced them
  for (int i = 0; i < ProveWs::kStreams; i++) ws.res[i] = gr->res[i];
  ZK_CUDA(cudaGraphLaunch(gr->exec, ws.st[0]));
  count_launch((int)gr->kernels);
}

// Waits for the device work, combines the MSM results, applies blinding.
void ws_finish(zk_circuit* c, ProveWs& ws, bool blind, const uint64_t* r, const uint64_t* s,
               uint64_t proof[32], ProveIntermediates* dbg = nullptr) {
  ZK_CUDA(cudaEventSynchronize(ws.ev_all));
  const G1 a = msm_g1_combine_xyzz(ws.win[1].ptr, ws.res[1]);
  const G2 b = msm_g2_combine_xyzz(ws.win[2].ptr, ws.res[2]);
  const G1 cc = msm_g1_combine_xyzz(ws.win[3].ptr, ws.res[3]);
  const G1 h = msm_g1_combine_xyzz(ws.win[0].ptr, ws.res[0]);
  G1 b1;
  if (blind) b1 = msm_g1_combine_xyzz(ws.win[4].ptr, ws.res[4]);
  if (dbg) {
    // each MSM's own affine result (the traced path only)
    dbg->inf[0] = g1_out(a, dbg->msm_a);
    dbg->inf[1] = g2_out(b, dbg->msm_b2);
    dbg->inf[2] = g1_out(cc, dbg->msm_c);
    dbg->inf[3] = g1_out(h, dbg->msm_h);
  }
  const ProofXyzz p = assemble_proof(c, a, b, cc.add(h), blind ? &b1 : nullptr, r, s);
  uint64_t* out = proof;
  proofs_to_affine(&p, 1, &out);
}

}  // namespace

void spmv_enqueue(zk_circuit* c, const uint64_t* we, uint64_t* aw, uint64_t* bw, cudaStream_t st) {
  SpmvArgs sa;
  for (int m = 0; m < 2; m++) {
    sa.row[m] = c->row[m].as<uint32_t>();
    sa.sig[m] = c->sig[m].as<uint32_t>();
    sa.val[m] = c->val[m].as<fr_t>();
  }
  sa.out[0] = reinterpret_cast<fr_t*>(aw);
  sa.out[1] = reinterpret_cast<fr_t*>(bw);
  ProfScope prof(kProfSpmv, (double)c->n_coefs, st);
  k_spmv<<<dim3(blocks(c->n, 256), 2), 256, 0, st>>>(sa, reinterpret_cast<const fr_t*>(we + 4),
                                                     (uint32_t)c->n);
  ZK_LAUNCHED();
}

ProofXyzz assemble_proof(const zk_circuit* c, const G1& a, const G2& b, const G1& c_plus_h,
                         const G1* b1, const uint64_t* r, const uint64_t* s) {
  ProofXyzz p{a, c_plus_h, b};
  if (b1) {
    const G1 d1 = g1_aff(c->delta1);
    p.a = p.a.add(mul(d1, r));
    p.b = p.b.add(mul(g2_aff(c->delta2), s));
    const G1 B1 = b1->add(mul(d1, s));
    host::Fr rs = host::Fr::from_raw(r).to_mont() * host::Fr::from_raw(s).to_mont();
    const host::Fr nrs = (-rs).from_mont();
    p.c = p.c.add(mul(p.a, s)).add(mul(B1, r)).add(mul(d1, nrs.v));
  }
  return p;
}

void proofs_to_affine(const ProofXyzz* p, size_t n, uint64_t* const* out) {
  std::vector<G1> g1(2 * n);
  std::vector<G2> g2(n);
  for (size_t i = 0; i < n; i++) {
    g1[2 * i] = p[i].a;
    g1[2 * i + 1] = p[i].c;
    g2[i] = p[i].b;
  }
  std::vector<host::Fp> x1(2 * n), y1(2 * n);
  std::vector<host::Fp2> x2(n), y2(n);
  std::unique_ptr<bool[]> inf1(new bool[2 * n]), inf2(new bool[n]);
  host::batch_to_affine(g1.data(), 2 * n, x1.data(), y1.data(), inf1.get(), g2.data(), n,
                        x2.data(), y2.data(), inf2.get());
  for (size_t i = 0; i < n; i++) {
    put_g1(x1[2 * i], y1[2 * i], out[i]);
    put_g2(x2[i], y2[i], out[i] + 8);
    put_g1(x1[2 * i + 1], y1[2 * i + 1], out[i] + 24);
  }
}

void check_job(zk_circuit* c, const uint64_t* witness, size_t n_witness, bool blind) {
  ZK_REQUIRE(c, ZK_EINVAL, "NULL circuit");
  ZK_REQUIRE(witness, ZK_EINVAL, "NULL witness");
  ZK_REQUIRE(n_witness >= c->m1, ZK_EWITNESS, "witness has fewer values than the circuit's nVars");
  ZK_REQUIRE(!blind || c->has_b1, ZK_EFORMAT, "blinding needs zkey section 6 (B1 points)");
}

// A host witness tells the circuit's scalar distribution (it keys the tuned
// MSM settings); device witnesses keep the last one seen.
void note_witness(zk_circuit* c, const uint64_t* witness, bool on_device) {
  if (c->dist_auto && !on_device) c->dist = detect_scalar_dist(witness, c->m1);
}


// Device bytes that preparing ws for this circuit would newly allocate (the
// proof server admits a request only when that much memory is free).
size_t ws_bytes_needed(zk_circuit* c, const ProveWs& ws, bool blind) {
  MsmConfig cfg[ProveWs::kStreams];
  ws_msm_configs(c, cfg);
  size_t need[ProveWs::kStreams];
  ws_scratch_needs(c, blind, cfg, need);
  const size_t m1 = c->m1, n = c->n;
  auto grow = [](const DeviceBuffer& b, size_t want) { return b.cap < want ? want : size_t(0); };
  size_t total = grow(ws.we, 32 * (m1 + 1)) + grow(ws.aw, 32 * n) + grow(ws.bw, 32 * n) +
                 grow(ws.cw, 32 * n) + grow(ws.h, 32 * n);
  for (int i = 0; i < ProveWs::kStreams; i++) total += grow(ws.msm[i], need[i]);
  if (c->ctx->ntt.lmax < c->log_n) total += 2 * 16 * n;  // twiddle tables of 2^(log_n-1)
  return total;
}

// Starts a proof from a host witness on ws's streams without waiting for it.
void ws_submit(zk_circuit* c, ProveWs& ws, const uint64_t* witness, bool blind, Stager& stager) {
  note_witness(c, witness, false);
  ws_prepare(c, ws, blind);
  ws_stage(c, ws, witness, false, stager);
  ws_launch(c, ws, blind, c->ctx->use_graphs, nullptr);
  ZK_CUDA(cudaEventRecord(ws.ev_all, ws.st[0]));
}

// True once the submitted proof's device work has ended (or failed).
bool ws_ready(ProveWs& ws) { return cudaEventQuery(ws.ev_all) != cudaErrorNotReady; }

// Combines a finished proof (raises the device error of a failed one).
void ws_collect(zk_circuit* c, ProveWs& ws, bool blind, const uint64_t* r, const uint64_t* s,
                uint64_t proof[32]) {
  ws_finish(c, ws, blind, r, s, proof);
}

uint64_t next_circuit_id() { return g_circuit_ids.fetch_add(1); }

void ProveWs::drop_graph() {
  for (Graph& g : graphs) cudaGraphExecDestroy(g.exec);
  graphs.clear();
}

void prove(zk_circuit* c, const uint64_t* witness, size_t n_witness, bool on_device,
           const uint64_t* r, const uint64_t* s, uint64_t proof[32], ProveIntermediates* dbg) {
  const bool blind = r && s;
  check_job(c, witness, n_witness, blind);
  zk_ctx* ctx = c->ctx;
  ProveWs& ws = ctx->ws;
  note_witness(c, witness, on_device);
  ws_prepare(c, ws, blind);
  // the proof starts after prior work on the context stream and ends before
  // later work on it, so callers can bracket it with events on that stream
  ZK_CUDA(cudaEventRecord(ws.ev_begin, ctx->stream));
  ZK_CUDA(cudaStreamWaitEvent(ws.st[0], ws.ev_begin, 0));
  ws_stage(c, ws, witness, on_device, ctx->stager);
  ws_launch(c, ws, blind, ctx->use_graphs, dbg);
  ZK_CUDA(cudaEventRecord(ws.ev_all, ws.st[0]));
  ZK_CUDA(cudaStreamWaitEvent(ctx->stream, ws.ev_all, 0));
  ws_finish(c, ws, blind, r, s, proof, dbg);
}

void prove_oneshot(zk_ctx* ctx, const BinFile& zkey, const uint64_t* witness, size_t n_witness,
                   uint64_t proof[32]) {
  const ZkeyView z = parse_zkey(zkey);
  std::unique_ptr<zk_circuit> cp = circuit_header(ctx, z);
  zk_circuit* c = cp.get();
  check_job(c, witness, n_witness, false);
  note_witness(c, witness, false);
  ProveWs& ws = ctx->ws;
  ws_prepare(c, ws, false);
  ws.flag.ensure(256);
  Stager& sg = ctx->stager;
  const size_t m1 = c->m1, n = c->n, l = c->l, nc = m1 - l - 1;
  cudaStream_t s0 = ws.st[0];
  ZK_CUDA(cudaEventRecord(ws.ev_begin, ctx->stream));
  for (int i = 0; i < ProveWs::kStreams; i++) ZK_CUDA(cudaStreamWaitEvent(ws.st[i], ws.ev_begin, 0));
  ws_stage(c, ws, witness, false, sg);
  ZK_CUDA(cudaEventRecord(ws.ev_we, s0));
  const uint64_t* we = ws.we.as<uint64_t>();
  const DeviceBuffer none;
  // each point set goes up on the stream of the MSM that reads it, and that
  // MSM starts at once; B2 (the longest MSM) first
  upload_points(c, z, kSetB2, ws.st[2 % ws.nstreams], sg);
  ws_msm(c, ws, 2, true, c->pts_b2, none, we, m1 + 1);
  upload_points(c, z, kSetA, ws.st[1 % ws.nstreams], sg);
  ws_msm(c, ws, 1, false, c->pts_a, none, we, m1 + 1);
  upload_points(c, z, kSetC, ws.st[3 % ws.nstreams], sg);
  const bool merge = ws_merge_ch(c, ws);
  ws.merge_c = MsmMerge{};
  ws.merge_c.ready = ws.ev_merge;
  ws_msm(c, ws, 3, false, c->pts_c, none, we + 4 * (l + 2), nc, merge ? &ws.merge_c : nullptr);
  // section 4 -> CSR -> A.w, B.w -> h on stream 0, the H points beside it
  CsrScratch csr;
  uint32_t* h_bad = ws.flag.as<uint32_t>();
  build_csr(c, z, s0, sg, csr, h_bad);
  spmv_enqueue(c, we, ws.aw.as<uint64_t>(), ws.bw.as<uint64_t>(), s0);
  hpoly(ctx->ntt, ws.aw.as<uint64_t>(), ws.bw.as<uint64_t>(), ws.cw.as<uint64_t>(), c->log_n,
        ws.h.as<uint64_t>(), s0);
  cudaStream_t sh = ws.st[4];
  upload_points(c, z, kSetH, sh, sg);
  ZK_CUDA(cudaEventRecord(ws.ev_done[4], sh));
  ZK_CUDA(cudaStreamWaitEvent(s0, ws.ev_done[4], 0));
  ws_msm(c, ws, 0, false, c->pts_h, none, ws.h.as<uint64_t>(), n, nullptr,
         merge ? &ws.merge_c : nullptr);
  for (int i = 1; i < 4; i++) ZK_CUDA(cudaStreamWaitEvent(s0, ws.ev_done[i], 0));
  ZK_CUDA(cudaEventRecord(ws.ev_all, s0));
  ZK_CUDA(cudaStreamWaitEvent(ctx->stream, ws.ev_all, 0));
  ws_finish(c, ws, false, nullptr, nullptr, proof);
  ZK_REQUIRE(*h_bad == 0, ZK_EFORMAT, "zkey: section 4 has entries outside the domain or witness");
}

void prove_batch(zk_ctx* ctx, size_t count, zk_circuit* const* cs, const uint64_t* const* wits,
                 const size_t* nwits, bool on_device, const uint64_t* rs, const uint64_t* ss,
                 uint64_t* proofs, int inflight) {
  ZK_REQUIRE(inflight >= 1 && inflight <= 16, ZK_EINVAL, "batch: in-flight proofs must be 1..16");
  ZK_REQUIRE(count == 0 || (cs && wits && nwits && proofs), ZK_EINVAL, "batch: NULL argument");
  const bool blind = rs && ss;
  for (size_t i = 0; i < count; i++) {
    ZK_REQUIRE(cs[i] && cs[i]->ctx == ctx, ZK_EINVAL, "batch: circuit from another context");
    check_job(cs[i], wits[i], nwits[i], blind);
  }
  while ((int)ctx->pool.size() < inflight) ctx->pool.emplace_back(new ProveWs());
  std::vector<long> job(inflight, -1);
  ZK_CUDA(cudaEventRecord(ctx->ws.ev_begin_pool(), ctx->stream));
  auto finish = [&](int k) {
    const long i = job[k];
    if (i < 0) return;
    ProveWs& ws = *ctx->pool[k];
    ws_finish(cs[i], ws, blind, blind ? rs + 4 * i : nullptr, blind ? ss + 4 * i : nullptr,
              proofs + 32 * i);
    job[k] = -1;
  };
  for (size_t i = 0; i < count; i++) {
    const int k = (int)(i % inflight);
    finish(k);  // the slot's previous proof: its host combine overlaps later proofs' GPU work
    ProveWs& ws = *ctx->pool[k];
    note_witness(cs[i], wits[i], on_device);
    ws_prepare(cs[i], ws, blind);
    ZK_CUDA(cudaStreamWaitEvent(ws.st[0], ctx->ws.ev_begin_pool(), 0));
    ws_stage(cs[i], ws, wits[i], on_device, ctx->stager);
    ws_launch(cs[i], ws, blind, ctx->use_graphs, nullptr);
    ZK_CUDA(cudaEventRecord(ws.ev_all, ws.st[0]));
    ZK_CUDA(cudaStreamWaitEvent(ctx->stream, ws.ev_all, 0));
    job[k] = (long)i;
  }
  for (int k = 0; k < inflight; k++) finish(k);
}

}  // namespace zk
