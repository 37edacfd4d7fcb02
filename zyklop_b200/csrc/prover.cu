// Groth16 prover on sm_100a (see prover.hpp).
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <memory>
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
void g1_out(const G1& g, uint64_t* out) {
  host::Fp x, y;
  g.to_affine(x, y);
  memcpy(out, x.v, 32);
  memcpy(out + 4, y.v, 32);
}
void g2_out(const G2& g, uint64_t* out) {
  host::Fp2 x, y;
  g.to_affine(x, y);
  memcpy(out, x.c0.v, 32);
  memcpy(out + 4, x.c1.v, 32);
  memcpy(out + 8, y.c0.v, 32);
  memcpy(out + 12, y.c1.v, 32);
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
  // ZYKLOP_PROVE_STREAMS=1 runs a proof's MSMs back to back on one stream
  // (a tuning knob: concurrent MSMs share L2 and the SMs)
  if (const char* e = getenv("ZYKLOP_PROVE_STREAMS")) {
    const int v = atoi(e);
    if (v >= 1 && v <= kStreams) nstreams = v;
  }
  for (int i = 0; i < kStreams; i++) {
    ZK_CUDA(cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking));
    ZK_CUDA(cudaEventCreateWithFlags(&ev_done[i], cudaEventDisableTiming));
  }
  ZK_CUDA(cudaEventCreateWithFlags(&ev_we, cudaEventDisableTiming));
  ZK_CUDA(cudaEventCreateWithFlags(&ev_begin, cudaEventDisableTiming));
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
  cudaEventDestroy(ev_begin);
}

zk_circuit* circuit_load(zk_ctx* ctx, const BinFile& f) {
  const ZkeyView z = parse_zkey(f);
  std::unique_ptr<zk_circuit> c(new zk_circuit());
  c->ctx = ctx;
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
  cudaStream_t st = ctx->stream;
  Stager& sg = ctx->stager;
  const size_t m1 = c->m1, nc = (size_t)c->m1 - c->l - 1;
  // CRS points: record 0 of A / B1 / B2 is alpha1 / beta1 / beta2
  c->pts_a.ensure(64 * (m1 + 1));
  ZK_CUDA(cudaMemcpyAsync(c->pts_a.ptr, c->alpha1, 64, cudaMemcpyHostToDevice, st));
  sg.upload(c->pts_a.as<char>() + 64, z.a, 64 * m1, st);
  c->pts_b2.ensure(128 * (m1 + 1));
  ZK_CUDA(cudaMemcpyAsync(c->pts_b2.ptr, c->beta2, 128, cudaMemcpyHostToDevice, st));
  sg.upload(c->pts_b2.as<char>() + 128, z.b2, 128 * m1, st);
  if (z.b1) {
    c->has_b1 = true;
    c->pts_b1.ensure(64 * (m1 + 1));
    ZK_CUDA(cudaMemcpyAsync(c->pts_b1.ptr, c->beta1, 64, cudaMemcpyHostToDevice, st));
    sg.upload(c->pts_b1.as<char>() + 64, z.b1, 64 * m1, st);
  }
  c->pts_c.ensure(64 * (nc ? nc : 1));
  sg.upload(c->pts_c.ptr, z.c, 64 * nc, st);
  c->pts_h.ensure(64 * (size_t)c->n);
  sg.upload(c->pts_h.ptr, z.h, 64 * (size_t)c->n, st);

  // section 4 -> CSR on the device
  const size_t nnz = c->n_coefs, n = c->n;
  DeviceBuffer raw, tmp;
  raw.ensure(44 * (nnz ? nnz : 1));
  sg.upload(raw.ptr, z.coefs, 44 * nnz, st);
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
  tmp.ensure(carve_csr_tmp(nullptr, cnt, cur, tl, &bad));  // dry run: size with padding
  carve_csr_tmp(tmp.ptr, cnt, cur, tl, &bad);
  ZK_CUDA(cudaMemsetAsync(tmp.ptr, 0, tmp.cap, st));
  for (int m = 0; m < 2; m++) {
    c->row[m].ensure(4 * (n + 1));
    c->sig[m].ensure(4 * (nnz ? nnz : 1));
    c->val[m].ensure(32 * (nnz ? nnz : 1));
  }
  if (nnz) {
    k_coef_count<<<blocks(nnz, 256), 256, 0, st>>>(raw.as<uint32_t>(), (uint32_t)nnz, (uint32_t)n,
                                                  c->m1, cnt[0], cnt[1], bad);
    ZK_LAUNCHED();
  }
  for (int m = 0; m < 2; m++) scan::exclusive(cnt[m], cur[m], n + 1, tl[m], st);
  if (nnz) {
    k_coef_scatter<<<blocks(nnz, 256), 256, 0, st>>>(
        raw.as<uint32_t>(), (uint32_t)nnz, (uint32_t)n, c->m1, cur[0], cur[1],
        c->sig[0].as<uint32_t>(), c->sig[1].as<uint32_t>(), c->val[0].as<uint32_t>(),
        c->val[1].as<uint32_t>());
    ZK_LAUNCHED();
  }
  for (int m = 0; m < 2; m++)
    ZK_CUDA(cudaMemcpyAsync(c->row[m].ptr, cnt[m], 4 * (n + 1), cudaMemcpyDeviceToDevice, st));
  uint32_t h_bad = 0;
  ZK_CUDA(cudaMemcpyAsync(&h_bad, bad, 4, cudaMemcpyDeviceToHost, st));
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
  const int g1c = c_g1 ? c_g1 : msm_fixed_default_c(m1 + 1, false);
  const int g2c = c_g2 ? c_g2 : msm_fixed_default_c(m1 + 1, true);
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

void prove(zk_circuit* c, const uint64_t* witness, size_t n_witness, bool on_device,
           const uint64_t* r, const uint64_t* s, uint64_t proof[32], ProveIntermediates* dbg) {
  zk_ctx* ctx = c->ctx;
  ZK_REQUIRE(n_witness >= c->m1, ZK_EWITNESS, "witness has fewer values than the circuit's nVars");
  ZK_REQUIRE(witness, ZK_EINVAL, "NULL witness");
  const bool blind = r && s;
  ZK_REQUIRE(!blind || c->has_b1, ZK_EFORMAT, "blinding needs zkey section 6 (B1 points)");
  ProveWs& ws = ctx->ws;
  ws.init();
  const size_t m1 = c->m1, n = c->n, l = c->l, nc = m1 - l - 1;
  ws.we.ensure(32 * (m1 + 1));
  ws.aw.ensure(32 * n);
  ws.bw.ensure(32 * n);
  ws.cw.ensure(32 * n);
  ws.h.ensure(32 * n);
  ctx->ntt.ensure(c->log_n, ws.st[0]);
  const MsmConfig& c1 = ctx->msm_cfg[0];
  const MsmConfig& c2 = ctx->msm_cfg[1];
  const bool fixed = c->tab_c[0] != 0;
  auto scratch = [&](size_t cnt, bool g2) {
    return fixed ? msm_scratch_bytes_fixed(cnt, g2, c->tab_c[g2 ? 1 : 0], g2 ? c2 : c1)
                 : msm_scratch_bytes(cnt, g2, g2 ? c2 : c1);
  };
  const size_t need[ProveWs::kStreams] = {scratch(n, false), scratch(m1 + 1, false),
                                          scratch(m1 + 1, true), scratch(nc, false),
                                          blind ? scratch(m1 + 1, false) : 0};
  for (int i = 0; i < ProveWs::kStreams; i++)
    if (need[i]) {
      if (ws.msm[i].cap < need[i]) ZK_CUDA(cudaStreamSynchronize(ws.st[i]));
      ws.msm[i].ensure(need[i]);
    }

  // the proof starts after prior work on the context stream and ends before
  // later work on it, so callers can bracket it with events on that stream
  ZK_CUDA(cudaEventRecord(ws.ev_begin, ctx->stream));
  for (int i = 0; i < ProveWs::kStreams; i++) ZK_CUDA(cudaStreamWaitEvent(ws.st[i], ws.ev_begin, 0));

  // 1. witness: we = [1 || w_0 .. w_{m1-1}] (src/groth16.cu:1316-1326)
  cudaStream_t s0 = ws.st[0];
  uint64_t* we = ws.we.as<uint64_t>();
  ZK_CUDA(cudaMemsetAsync(we, 0, 32, s0));
  ZK_CUDA(cudaMemsetAsync(we, 1, 1, s0));
  if (on_device)
    ZK_CUDA(cudaMemcpyAsync(we + 4, witness, 32 * m1, cudaMemcpyDeviceToDevice, s0));
  else
    ctx->stager.upload(we + 4, witness, 32 * m1, s0);
  ZK_CUDA(cudaEventRecord(ws.ev_we, s0));

  // 2. MSMs that only need the witness, on their own streams
  MsmResult res[ProveWs::kStreams];
  auto launch = [&](int i, bool g2, const DeviceBuffer& pts, const DeviceBuffer& tab,
                    const uint64_t* sc, size_t cnt) {
    const int si = i % ws.nstreams;
    cudaStream_t st = ws.st[si];
    if (si) ZK_CUDA(cudaStreamWaitEvent(st, ws.ev_we, 0));
    if (fixed)
      res[i] = msm_enqueue_fixed(g2, tab.ptr, sc, cnt, c->tab_c[g2 ? 1 : 0], ws.msm[i].ptr,
                                 ws.msm[i].cap, g2 ? c2 : c1, st);
    else if (g2)
      res[i] = msm_g2_enqueue(points_aos(pts.ptr, true), sc, cnt, ws.msm[i].ptr, ws.msm[i].cap, c2,
                              st);
    else
      res[i] = msm_g1_enqueue(points_aos(pts.ptr, false), sc, cnt, ws.msm[i].ptr, ws.msm[i].cap,
                              c1, st);
    ws.win[i].ensure(res[i].bytes);
    ZK_CUDA(cudaMemcpyAsync(ws.win[i].ptr, res[i].d_data, res[i].bytes, cudaMemcpyDeviceToHost, st));
    ZK_CUDA(cudaEventRecord(ws.ev_done[i], st));
  };
  launch(1, false, c->pts_a, c->tab_a, we, m1 + 1);
  launch(2, true, c->pts_b2, c->tab_b2, we, m1 + 1);
  launch(3, false, c->pts_c, c->tab_c_pts, we + 4 * (l + 2), nc);
  if (blind) launch(4, false, c->pts_b1, c->tab_b1, we, m1 + 1);

  // 3. SpMV -> H -> MSM_H on stream 0
  SpmvArgs sa;
  for (int m = 0; m < 2; m++) {
    sa.row[m] = c->row[m].as<uint32_t>();
    sa.sig[m] = c->sig[m].as<uint32_t>();
    sa.val[m] = c->val[m].as<fr_t>();
  }
  sa.out[0] = ws.aw.as<fr_t>();
  sa.out[1] = ws.bw.as<fr_t>();
  {
  ProfScope prof(kProfSpmv, (double)c->n_coefs, s0);
  k_spmv<<<dim3(blocks(n, 256), 2), 256, 0, s0>>>(sa, reinterpret_cast<const fr_t*>(we + 4),
                                                  (uint32_t)n);
  ZK_LAUNCHED();
  }
  ZK_CHECK_LAUNCH();
  if (dbg && (dbg->aw || dbg->bw)) {
    if (dbg->aw) ZK_CUDA(cudaMemcpyAsync(dbg->aw, ws.aw.ptr, 32 * n, cudaMemcpyDeviceToHost, s0));
    if (dbg->bw) ZK_CUDA(cudaMemcpyAsync(dbg->bw, ws.bw.ptr, 32 * n, cudaMemcpyDeviceToHost, s0));
    ZK_CUDA(cudaStreamSynchronize(s0));
  }
  hpoly(ctx->ntt, ws.aw.as<uint64_t>(), ws.bw.as<uint64_t>(), ws.cw.as<uint64_t>(), c->log_n,
        ws.h.as<uint64_t>(), s0);
  if (dbg && dbg->h) {
    ZK_CUDA(cudaMemcpyAsync(dbg->h, ws.h.ptr, 32 * n, cudaMemcpyDeviceToHost, s0));
    ZK_CUDA(cudaStreamSynchronize(s0));
  }
  launch(0, false, c->pts_h, c->tab_h, ws.h.as<uint64_t>(), n);

  // 4. host: combine the window sums, assemble the proof
  const int used = blind ? 5 : 4;
  for (int i = 0; i < used; i++) ZK_CUDA(cudaStreamWaitEvent(ctx->stream, ws.ev_done[i], 0));
  for (int i = 0; i < used; i++) ZK_CUDA(cudaEventSynchronize(ws.ev_done[i]));
  uint64_t pa[8], pb[16], pc[8], ph[8], pb1[8];
  msm_g1_combine(ws.win[1].ptr, res[1], pa);
  msm_g2_combine(ws.win[2].ptr, res[2], pb);
  msm_g1_combine(ws.win[3].ptr, res[3], pc);
  msm_g1_combine(ws.win[0].ptr, res[0], ph);
  G1 A = g1_aff(pa), Cc = g1_aff(pc).add(g1_aff(ph));
  G2 B = g2_aff(pb);
  if (blind) {
    msm_g1_combine(ws.win[4].ptr, res[4], pb1);
    const G1 d1 = g1_aff(c->delta1);
    A = A.add(mul(d1, r));
    B = B.add(mul(g2_aff(c->delta2), s));
    const G1 B1 = g1_aff(pb1).add(mul(d1, s));
    host::Fr rs = host::Fr::from_raw(r).to_mont() * host::Fr::from_raw(s).to_mont();
    const host::Fr nrs = (-rs).from_mont();
    Cc = Cc.add(mul(A, s)).add(mul(B1, r)).add(mul(d1, nrs.v));
  }
  g1_out(A, proof);
  g2_out(B, proof + 8);
  g1_out(Cc, proof + 24);
}

}  // namespace zk
