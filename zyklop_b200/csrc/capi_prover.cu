// C ABI of the Groth16 prover: circuits, proofs, files, serialization
// (declared in include/zyklop_b200.h).
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <string>

#include "capi_util.hpp"
#include "msm.hpp"
#include "prover.hpp"
#include "serialize.hpp"

using namespace zk;

extern "C" {

int zk_circuit_load_file(zk_ctx* ctx, const char* zkey_path, zk_circuit** out) {
  ZK_API_BEGIN
  ZK_REQUIRE(zkey_path && out, ZK_EINVAL, "zk_circuit_load_file: NULL argument");
  *out = nullptr;
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  auto f = BinFile::open(zkey_path, "zkey", 1);
  *out = circuit_load(ctx, *f);
  ZK_API_END
}

int zk_circuit_load_mem(zk_ctx* ctx, const uint8_t* zkey, size_t len, zk_circuit** out) {
  ZK_API_BEGIN
  ZK_REQUIRE(zkey && out, ZK_EINVAL, "zk_circuit_load_mem: NULL argument");
  *out = nullptr;
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  auto f = BinFile::wrap(zkey, len, "zkey", 1);
  *out = circuit_load(ctx, *f);
  ZK_API_END
}

int zk_circuit_free(zk_circuit* c) {
  ZK_API_BEGIN
  if (!c) return ZK_OK;
  zk_ctx* ctx = c->ctx;
  use_device(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  delete c;
  ZK_API_END
}

int zk_circuit_info(const zk_circuit* c, uint32_t* n_vars, uint32_t* n_public, uint32_t* domain) {
  ZK_API_BEGIN
  ZK_REQUIRE(c, ZK_EINVAL, "zk_circuit_info: NULL circuit");
  if (n_vars) *n_vars = c->m1;
  if (n_public) *n_public = c->l;
  if (domain) *domain = c->n;
  ZK_API_END
}

int zk_circuit_precompute(zk_circuit* c, int c_g1, int c_g2) {
  ZK_API_BEGIN
  ZK_REQUIRE(c, ZK_EINVAL, "zk_circuit_precompute: NULL circuit");
  enter_ctx(c->ctx);
  std::lock_guard<std::mutex> g(c->ctx->mu);
  circuit_precompute(c, c_g1, c_g2);
  ZK_API_END
}

int zk_msm_table_create(zk_ctx* ctx, int group, const uint64_t* d_px, const uint64_t* d_py,
                        size_t n, int c, zk_msm_table** out) {
  ZK_API_BEGIN
  ZK_REQUIRE(out, ZK_EINVAL, "zk_msm_table_create: NULL output");
  *out = nullptr;
  ZK_REQUIRE(group == 1 || group == 2, ZK_EINVAL, "zk_msm_table_create: group must be 1 or 2");
  ZK_REQUIRE(n == 0 || (d_px && d_py), ZK_EINVAL, "zk_msm_table_create: NULL points");
  ZK_REQUIRE(n < (size_t(1) << 27), ZK_EINVAL, "zk_msm_table_create: too many points");
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  std::unique_ptr<zk_msm_table> t(new zk_msm_table());
  t->ctx = ctx;
  t->group = group;
  t->n = n;
  t->c = c ? c : table_c_for(ctx, group == 2, n, ctx->scalar_dist);
  ZK_REQUIRE(t->c >= 4 && t->c <= 22, ZK_EINVAL, "zk_msm_table_create: c must be 0 or 4..22");
  t->table.ensure(msm_table_bytes(n ? n : 1, group == 2, t->c));
  msm_precompute(group == 2, points_soa(d_px, d_py), n, t->c, t->table.ptr, ctx->stream);
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  *out = t.release();
  ZK_API_END
}

int zk_msm_table_run(zk_msm_table* t, const uint64_t* d_scalars, size_t n, uint64_t* h_out,
                     int* is_inf) {
  ZK_API_BEGIN
  ZK_REQUIRE(t && h_out, ZK_EINVAL, "zk_msm_table_run: NULL argument");
  ZK_REQUIRE(n <= t->n, ZK_EINVAL, "zk_msm_table_run: more scalars than table points");
  ZK_REQUIRE(n == 0 || d_scalars, ZK_EINVAL, "zk_msm_table_run: NULL scalars");
  zk_ctx* ctx = enter_ctx(t->ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  const bool g2 = t->group == 2;
  const MsmConfig cfg = msm_config_for(ctx, g2, t->n, ctx->scalar_dist, t->c);
  // the table's records are laid out for t->n points: run over all of them
  // with zero scalars past n (a prefix of the table is not a table)
  const size_t cnt = t->n;
  DeviceBuffer sc;
  const uint64_t* scal = d_scalars;
  if (n < cnt) {
    sc.ensure(32 * cnt);
    ZK_CUDA(cudaMemsetAsync(sc.ptr, 0, 32 * cnt, ctx->stream));
    if (n) ZK_CUDA(cudaMemcpyAsync(sc.ptr, d_scalars, 32 * n, cudaMemcpyDeviceToDevice, ctx->stream));
    scal = sc.as<uint64_t>();
  }
  ctx->msm_scratch.ensure(msm_scratch_bytes_fixed(cnt, g2, t->c, cfg));
  const MsmResult r = msm_enqueue_fixed(g2, t->table.ptr, scal, cnt, t->c, ctx->msm_scratch.ptr,
                                        ctx->msm_scratch.cap, cfg, ctx->stream);
  alignas(16) uint8_t h[1024];
  ZK_REQUIRE(r.bytes <= sizeof(h), ZK_EINTERNAL, "zk_msm_table_run: result too large");
  ZK_CUDA(cudaMemcpyAsync(h, r.d_data, r.bytes, cudaMemcpyDeviceToHost, ctx->stream));
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  const bool inf = g2 ? msm_g2_combine(h, r, h_out) : msm_g1_combine(h, r, h_out);
  if (is_inf) *is_inf = inf ? 1 : 0;
  ZK_API_END
}

int zk_msm_table_free(zk_msm_table* t) {
  ZK_API_BEGIN
  if (!t) return ZK_OK;
  enter_ctx(t->ctx);
  std::lock_guard<std::mutex> g(t->ctx->mu);
  delete t;
  ZK_API_END
}

int zk_prove(zk_circuit* c, const uint64_t* h_witness, size_t n_witness, const uint64_t* r,
             const uint64_t* s, uint64_t* proof) {
  ZK_API_BEGIN
  ZK_REQUIRE(c && proof, ZK_EINVAL, "zk_prove: NULL argument");
  ZK_REQUIRE((r == nullptr) == (s == nullptr), ZK_EINVAL, "zk_prove: give both r and s or neither");
  enter_ctx(c->ctx);
  std::lock_guard<std::mutex> g(c->ctx->mu);
  prove(c, h_witness, n_witness, false, r, s, proof, nullptr);
  ZK_API_END
}

int zk_prove_device(zk_circuit* c, const uint64_t* d_witness, size_t n_witness, const uint64_t* r,
                    const uint64_t* s, uint64_t* proof) {
  ZK_API_BEGIN
  ZK_REQUIRE(c && proof, ZK_EINVAL, "zk_prove_device: NULL argument");
  ZK_REQUIRE((r == nullptr) == (s == nullptr), ZK_EINVAL,
             "zk_prove_device: give both r and s or neither");
  enter_ctx(c->ctx);
  std::lock_guard<std::mutex> g(c->ctx->mu);
  prove(c, d_witness, n_witness, true, r, s, proof, nullptr);
  ZK_API_END
}

int zk_prove_intermediates(zk_circuit* c, const uint64_t* h_witness, size_t n_witness,
                           uint64_t* aw, uint64_t* bw, uint64_t* h, uint64_t* proof) {
  ZK_API_BEGIN
  ZK_REQUIRE(c && proof, ZK_EINVAL, "zk_prove_intermediates: NULL argument");
  enter_ctx(c->ctx);
  std::lock_guard<std::mutex> g(c->ctx->mu);
  ProveIntermediates dbg;
  dbg.aw = aw;
  dbg.bw = bw;
  dbg.h = h;
  prove(c, h_witness, n_witness, false, nullptr, nullptr, proof, &dbg);
  ZK_API_END
}

int zk_prove_traced(zk_circuit* c, const uint64_t* h_witness, size_t n_witness,
                    zk_prove_trace* trace, uint64_t* proof) {
  ZK_API_BEGIN
  ZK_REQUIRE(c && trace && proof, ZK_EINVAL, "zk_prove_traced: NULL argument");
  enter_ctx(c->ctx);
  std::lock_guard<std::mutex> g(c->ctx->mu);
  ProveIntermediates dbg;
  dbg.aw = trace->aw;
  dbg.bw = trace->bw;
  dbg.ea = trace->ea;
  dbg.eb = trace->eb;
  dbg.ec = trace->ec;
  dbg.h = trace->h;
  prove(c, h_witness, n_witness, false, nullptr, nullptr, proof, &dbg);
  memcpy(trace->msm_a, dbg.msm_a, sizeof dbg.msm_a);
  memcpy(trace->msm_b2, dbg.msm_b2, sizeof dbg.msm_b2);
  memcpy(trace->msm_c, dbg.msm_c, sizeof dbg.msm_c);
  memcpy(trace->msm_h, dbg.msm_h, sizeof dbg.msm_h);
  for (int k = 0; k < 4; k++) trace->inf[k] = dbg.inf[k];
  ZK_API_END
}

int zk_prove_batch(zk_ctx* ctx, size_t count, zk_circuit* const* circuits,
                   const uint64_t* const* witnesses, const size_t* n_witness, int on_device,
                   const uint64_t* r, const uint64_t* s, uint64_t* proofs, int inflight) {
  ZK_API_BEGIN
  ZK_REQUIRE((r == nullptr) == (s == nullptr), ZK_EINVAL, "zk_prove_batch: give both r and s or neither");
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  bool fused = ctx->batch_mode == 2;
  if (ctx->batch_mode == 0) {  // auto: fused when every circuit has fixed-base tables
    fused = count > 0 && circuits;
    for (size_t i = 0; fused && i < count; i++) fused = circuits[i] && circuits[i]->tab_c[0] != 0;
  }
  if (fused)
    prove_batch_fused(ctx, count, circuits, witnesses, n_witness, on_device != 0, r, s, proofs,
                      ctx->batch_group);
  else
    prove_batch(ctx, count, circuits, witnesses, n_witness, on_device != 0, r, s, proofs, inflight);
  ZK_API_END
}

int zk_ctx_set_prove_streams(zk_ctx* ctx, int n) {
  ZK_API_BEGIN
  ZK_REQUIRE(n >= 0 && n <= zk::ProveWs::kStreams, ZK_EINVAL, "zk_ctx_set_prove_streams: 0..5");
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ctx->prove_streams = n;
  ZK_API_END
}

int zk_ctx_set_batch_mode(zk_ctx* ctx, int mode, int group) {
  ZK_API_BEGIN
  ZK_REQUIRE(mode >= 0 && mode <= 2, ZK_EINVAL, "zk_ctx_set_batch_mode: mode 0, 1 or 2");
  ZK_REQUIRE(group >= 1 && group <= 64, ZK_EINVAL, "zk_ctx_set_batch_mode: group 1..64");
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ctx->batch_mode = mode;
  ctx->batch_group = group;
  ZK_API_END
}

int zk_ctx_set_graphs(zk_ctx* ctx, int on) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ctx->use_graphs = on != 0;
  ZK_API_END
}

int zk_groth16_prove_mem(zk_ctx* ctx, const uint8_t* zkey, size_t zkey_len, const uint8_t* wtns,
                         size_t wtns_len, uint64_t* proof) {
  ZK_API_BEGIN
  ZK_REQUIRE(zkey && wtns && proof, ZK_EINVAL, "zk_groth16_prove_mem: NULL argument");
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  auto zf = BinFile::wrap(zkey, zkey_len, "zkey", 1);
  auto wf = BinFile::wrap(wtns, wtns_len, "wtns", 2);
  const WtnsView w = parse_wtns(*wf);
  prove_oneshot(ctx, *zf, w.values, w.n_vars, proof);
  ZK_API_END
}

int zk_groth16_prove_files(zk_ctx* ctx, const char* zkey_path, const char* wtns_path,
                           uint64_t* proof) {
  ZK_API_BEGIN
  ZK_REQUIRE(zkey_path && wtns_path && proof, ZK_EINVAL, "zk_groth16_prove_files: NULL argument");
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  auto zf = BinFile::open(zkey_path, "zkey", 1);
  auto wf = BinFile::open(wtns_path, "wtns", 2);
  const WtnsView w = parse_wtns(*wf);
  prove_oneshot(ctx, *zf, w.values, w.n_vars, proof);
  ZK_API_END
}

int zk_read_zkey_header(const char* zkey_path, zk_zkey_header* hdr) {
  ZK_API_BEGIN
  ZK_REQUIRE(zkey_path && hdr, ZK_EINVAL, "zk_read_zkey_header: NULL argument");
  auto zf = BinFile::open(zkey_path, "zkey", 1);
  const ZkeyView z = parse_zkey(*zf);
  hdr->n_constraints = z.domain_raw;
  hdr->n_vars = z.n_vars;
  hdr->n_public = z.n_public;
  hdr->domain_size = z.domain;
  hdr->log_domain = z.log_n;
  const uint64_t r[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL,
                         0x30644e72e131a029ULL};
  memcpy(hdr->prime, r, 32);
  ZK_API_END
}

int zk_proof_to_json(const uint64_t* proof, char* out, size_t out_size) {
  ZK_API_BEGIN
  ZK_REQUIRE(proof && out && out_size, ZK_EINVAL, "zk_proof_to_json: NULL argument");
  const std::string s = proof_json(proof);
  ZK_REQUIRE(s.size() + 1 <= out_size, ZK_EINVAL, "zk_proof_to_json: output buffer too small");
  memcpy(out, s.c_str(), s.size() + 1);
  ZK_API_END
}

int zk_proof_to_calldata(const uint64_t* proof, uint8_t* out, size_t out_size) {
  ZK_API_BEGIN
  ZK_REQUIRE(proof && out, ZK_EINVAL, "zk_proof_to_calldata: NULL argument");
  ZK_REQUIRE(out_size >= 256, ZK_EINVAL, "zk_proof_to_calldata: buffer smaller than 256 bytes");
  proof_calldata(proof, out);
  ZK_API_END
}

int zk_public_json(const char* wtns_path, uint32_t n_public, char* out, size_t out_size) {
  ZK_API_BEGIN
  ZK_REQUIRE(wtns_path && out && out_size, ZK_EINVAL, "zk_public_json: NULL argument");
  auto wf = BinFile::open(wtns_path, "wtns", 2);
  const WtnsView w = parse_wtns(*wf);
  ZK_REQUIRE(w.n_vars >= n_public + 1, ZK_EWITNESS, "witness has fewer than nPublic + 1 values");
  const std::string s = public_json(w.values + 4, n_public);
  ZK_REQUIRE(s.size() + 1 <= out_size, ZK_EINVAL, "zk_public_json: output buffer too small");
  memcpy(out, s.c_str(), s.size() + 1);
  ZK_API_END
}

}  // extern "C"
