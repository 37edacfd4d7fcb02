// Fused batched proving (see prover.hpp, prove_batch_fused).
//
// A group of proofs over circuits with fixed-base tables of the same window
// bits runs as:
//   s1: stage every job's witness we_j = [1 || w_j]            -> ev_staged
//   after ev_staged, concurrently:
//     s2: one multi-instance G2 MSM over every job's B2
//     s3: one multi-instance G1 MSM over every job's A, C (and B1)
//     sp[0..3]: SpMV per job, then (on sp[0]) every job's H pipeline in one
//               persistent launch (up to 32 jobs of any sizes per launch)
//   s1: (after sp[]) one multi-instance G1 MSM over every job's H, then
//       waits for s2 and s3
// With graphs on, everything after the staging is captured the first time a
// group of jobs comes and replayed when the same group comes again.
// so a group costs three MSM launch chains instead of four or five per
// proof, and each chain is as large as the group: the load-balanced
// accumulation (persistent blocks pulling (instance, bucket-range) record
// tiles from a device work queue) and the bucket reduction see every job's
// records at once.
// Each instance's window sum is exactly the single-MSM result, so proofs are
// unchanged.
// No reference counterpart (the reference proves one file pair per process).
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <utility>
#include <vector>

#include "context.hpp"
#include "msm.hpp"
#include "ntt.hpp"
#include "prover.hpp"
#include "tune.hpp"

namespace zk {
namespace {

constexpr size_t kGroupRecordCap = size_t(1) << 28;  // sorted records per MSM chain

struct Job {
  size_t idx;  // position in the caller's arrays
  zk_circuit* c;
};

struct Group {
  std::vector<Job> jobs;
  std::vector<size_t> we_off, poly_off;  // byte offsets into the workspace buffers
  MsmResult rw, rh, r2;  // A / C (/ B1) chain, H chain, B2 chain
  int per_job = 2;       // witness-side G1 instances per job: A, C (+ B1)
};

size_t records_of(const zk_circuit* c, bool blind) {
  const size_t m1 = c->m1, nc = m1 - c->l - 1;
  const size_t w1 = 254 / c->tab_c[0] + 1, w2 = 254 / c->tab_c[1] + 1;
  const size_t g1 = w1 * ((m1 + 1) * (blind ? 2 : 1) + nc);
  return std::max({g1, w1 * (size_t)c->n, w2 * (m1 + 1)});
}

void fused_init(FusedWs& f) {
  if (f.ready) return;
  for (cudaStream_t* s : {&f.s1, &f.s2, &f.s3})
    ZK_CUDA(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
  for (int q = 0; q < FusedWs::kPolyStreams; q++) {
    ZK_CUDA(cudaStreamCreateWithFlags(&f.sp[q], cudaStreamNonBlocking));
    ZK_CUDA(cudaEventCreateWithFlags(&f.ev_sp[q], cudaEventDisableTiming));
  }
  for (cudaEvent_t* e : {&f.ev_staged, &f.ev_g2, &f.ev_g1w, &f.ev_done})
    ZK_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  f.ready = true;
}

template <class WeOf, class PolyOf>
void fused_pipeline(zk_ctx* ctx, FusedWs& f, Group& g, bool blind, int c1, int c2,
                    const MsmConfig& cfgw, const MsmConfig& cfgh, const MsmConfig& cfg2,
                    WeOf we_of, PolyOf poly_of);

// Enqueues one group on f (whose previous group has been finished).  Returns
// once host witnesses are staged; the GPU work stays in flight.
void fused_launch(zk_ctx* ctx, FusedWs& f, Group& g, const uint64_t* const* wits, bool on_device,
                  bool blind, cudaEvent_t ev_begin) {
  fused_init(f);
  const int c1 = g.jobs[0].c->tab_c[0], c2 = g.jobs[0].c->tab_c[1];
  const size_t nj = g.jobs.size();
  g.per_job = blind ? 3 : 2;
  // layout
  size_t wbytes = 0, pbytes = 0, nw = 0, nh = 0, n2 = 0, nmaxw = 0, nmaxh = 0;
  int log_max = 1;
  g.we_off.clear();
  g.poly_off.clear();
  for (const Job& j : g.jobs) {
    const zk_circuit* c = j.c;
    const size_t m1 = c->m1, nc = m1 - c->l - 1;
    g.we_off.push_back(wbytes);
    wbytes += align256(32 * (m1 + 1));
    g.poly_off.push_back(pbytes);
    pbytes += 4 * align256(32 * (size_t)c->n);
    nw += (m1 + 1) * (blind ? 2 : 1) + nc;
    nh += c->n;
    n2 += m1 + 1;
    nmaxw = std::max(nmaxw, m1 + 1);
    nmaxh = std::max(nmaxh, (size_t)c->n);
    log_max = std::max(log_max, c->log_n);
  }
  const zk_circuit* c0 = g.jobs[0].c;
  const MsmConfig cfgw = msm_config_for(ctx, false, nmaxw, c0->dist, c1);
  const MsmConfig cfgh = msm_config_for(ctx, false, nmaxh, kDistUniform, c1);
  const MsmConfig cfg2 = msm_config_for(ctx, true, nmaxw, c0->dist, c2);
  const int instw = (int)nj * g.per_job, insth = (int)nj, inst2 = (int)nj;
  f.we.ensure(wbytes);
  f.poly.ensure(pbytes);
  f.g1w.ensure(msm_scratch_bytes_fixed(nw, false, c1, cfgw, instw));
  f.gh.ensure(msm_scratch_bytes_fixed(nh, false, c1, cfgh, insth));
  f.g2.ensure(msm_scratch_bytes_fixed(n2, true, c2, cfg2, inst2));
  f.win1w.ensure((size_t)instw * 2 * 128);
  f.winh.ensure((size_t)insth * 2 * 128);
  f.win2.ensure((size_t)inst2 * 2 * 256);
  ctx->ntt.ensure(log_max, f.s1);

  // stage the witnesses (after earlier work on the context stream)
  ZK_CUDA(cudaStreamWaitEvent(f.s1, ev_begin, 0));
  char* wb = f.we.as<char>();
  char* pb = f.poly.as<char>();
  auto we_of = [&](size_t k) { return reinterpret_cast<uint64_t*>(wb + g.we_off[k]); };
  auto poly_of = [&](size_t k, int part) {
    const size_t pn = align256(32 * (size_t)g.jobs[k].c->n);
    return reinterpret_cast<uint64_t*>(pb + g.poly_off[k] + part * pn);
  };
  for (size_t k = 0; k < nj; k++) {
    const zk_circuit* c = g.jobs[k].c;
    uint64_t* we = we_of(k);
    ZK_CUDA(cudaMemsetAsync(we, 0, 32, f.s1));
    ZK_CUDA(cudaMemsetAsync(we, 1, 1, f.s1));
    const uint64_t* w = wits[g.jobs[k].idx];
    if (on_device)
      ZK_CUDA(cudaMemcpyAsync(we + 4, w, 32 * (size_t)c->m1, cudaMemcpyDeviceToDevice, f.s1));
    else
      ctx->stager.upload(we + 4, w, 32 * (size_t)c->m1, f.s1);
  }
  // one status word per H launch (kMaxHJobs jobs each)
  const size_t nh_launch = (nj + kMaxHJobs - 1) / kMaxHJobs;
  f.hsync.ensure(kHSyncWords * sizeof(uint32_t));
  f.hflag.ensure(nh_launch * sizeof(uint32_t));
  for (size_t q = 0; q < nh_launch; q++) f.hflag.as<uint32_t>()[q] = 0;

  // the device pipeline from the staged witnesses on: replayed from a graph
  // when this group was captured before, else enqueued (and captured when
  // graphs are on)
  std::vector<uint64_t> key;
  if (ctx->use_graphs) {
    key = {(uint64_t)blind, (uint64_t)nj, (uint64_t)c1, (uint64_t)c2, (uint64_t)ctx->ntt.lmax};
    for (const Job& j : g.jobs) {
      key.push_back(j.c->id);
      key.push_back((uint64_t)ctx->ntt.pass_bits[j.c->log_n]);
    }
    for (const MsmConfig* m : {&cfgw, &cfgh, &cfg2})
      for (int v : {m->c, m->k0, m->k1, m->chunk}) key.push_back((uint64_t)(int64_t)v);
    for (const void* q : {f.we.ptr, f.poly.ptr, f.g1w.ptr, f.gh.ptr, f.g2.ptr, f.win1w.ptr,
                          f.winh.ptr, f.win2.ptr, f.hsync.ptr, f.hflag.ptr})
      key.push_back((uint64_t)(uintptr_t)q);
    for (FusedWs::Graph& x : f.graphs)
      if (x.key == key) {
        g.rw = x.rw;
        g.rh = x.rh;
        g.r2 = x.r2;
        ZK_CUDA(cudaGraphLaunch(x.exec, f.s1));
        count_launch((int)x.kernels);
        ZK_CUDA(cudaEventRecord(f.ev_done, f.s1));
        return;
      }
  }
  Profiler* saved = current_profiler();
  const uint64_t l0 = launch_count();
  if (ctx->use_graphs) {
    set_current_profiler(nullptr);  // no timing events inside a capture
    ZK_CUDA(cudaStreamBeginCapture(f.s1, cudaStreamCaptureModeThreadLocal));
  }
  try {
    fused_pipeline(ctx, f, g, blind, c1, c2, cfgw, cfgh, cfg2, we_of, poly_of);
  } catch (...) {
    if (ctx->use_graphs) {
      cudaGraph_t gr = nullptr;
      cudaStreamEndCapture(f.s1, &gr);
      if (gr) cudaGraphDestroy(gr);
      set_current_profiler(saved);
    }
    throw;
  }
  if (!ctx->use_graphs) {
    ZK_CUDA(cudaEventRecord(f.ev_done, f.s1));
    return;
  }
  cudaGraph_t gr = nullptr;
  ZK_CUDA(cudaStreamEndCapture(f.s1, &gr));
  set_current_profiler(saved);
  FusedWs::Graph x;
  const cudaError_t e = cudaGraphInstantiate(&x.exec, gr, 0);
  cudaGraphDestroy(gr);
  ZK_CUDA(e);
  x.key = std::move(key);
  x.rw = g.rw;
  x.rh = g.rh;
  x.r2 = g.r2;
  x.kernels = launch_count() - l0;
  if (f.graphs.size() >= FusedWs::kMaxGraphs) {
    cudaGraphExecDestroy(f.graphs.front().exec);
    f.graphs.erase(f.graphs.begin());
  }
  f.graphs.push_back(std::move(x));
  ZK_CUDA(cudaGraphLaunch(f.graphs.back().exec, f.s1));
  count_launch((int)f.graphs.back().kernels);
  // recorded outside the capture: an event recorded inside one is not
  // recorded when the graph replays
  ZK_CUDA(cudaEventRecord(f.ev_done, f.s1));
}

// The device part of a group after its witnesses are staged on s1: it
// begins and ends on s1 (the other streams fork from and join back to it)
// and issues no synchronizing call, so it can be captured into a graph.
template <class WeOf, class PolyOf>
void fused_pipeline(zk_ctx* ctx, FusedWs& f, Group& g, bool blind, int c1, int c2,
                    const MsmConfig& cfgw, const MsmConfig& cfgh, const MsmConfig& cfg2,
                    WeOf we_of, PolyOf poly_of) {
  const size_t nj = g.jobs.size();
  const int instw = (int)nj * g.per_job, insth = (int)nj, inst2 = (int)nj;
  ZK_CUDA(cudaEventRecord(f.ev_staged, f.s1));

  std::vector<const void*> tab(instw);
  std::vector<const uint64_t*> sc(instw);
  std::vector<size_t> cnt(instw);
  // B2 of every job on s2
  for (size_t k = 0; k < nj; k++) {
    tab[k] = g.jobs[k].c->tab_b2.ptr;
    sc[k] = we_of(k);
    cnt[k] = g.jobs[k].c->m1 + 1;
  }
  ZK_CUDA(cudaStreamWaitEvent(f.s2, f.ev_staged, 0));
  g.r2 = msm_enqueue_fixed_multi(true, inst2, tab.data(), sc.data(), cnt.data(), c2, f.g2.ptr,
                                 f.g2.cap, cfg2, f.s2);
  ZK_CUDA(cudaMemcpyAsync(f.win2.ptr, g.r2.d_data, g.r2.bytes, cudaMemcpyDeviceToHost, f.s2));
  ZK_CUDA(cudaEventRecord(f.ev_g2, f.s2));

  // A, C (and B1) of every job on s3
  for (size_t k = 0; k < nj; k++) {
    const zk_circuit* c = g.jobs[k].c;
    const size_t b = k * g.per_job;
    tab[b] = c->tab_a.ptr;
    sc[b] = we_of(k);
    cnt[b] = c->m1 + 1;
    tab[b + 1] = c->tab_c_pts.ptr;
    sc[b + 1] = we_of(k) + 4 * ((size_t)c->l + 2);
    cnt[b + 1] = c->m1 - c->l - 1;
    if (blind) {
      tab[b + 2] = c->tab_b1.ptr;
      sc[b + 2] = we_of(k);
      cnt[b + 2] = c->m1 + 1;
    }
  }
  ZK_CUDA(cudaStreamWaitEvent(f.s3, f.ev_staged, 0));
  g.rw = msm_enqueue_fixed_multi(false, instw, tab.data(), sc.data(), cnt.data(), c1, f.g1w.ptr,
                                 f.g1w.cap, cfgw, f.s3);
  ZK_CUDA(cudaMemcpyAsync(f.win1w.ptr, g.rw.d_data, g.rw.bytes, cudaMemcpyDeviceToHost, f.s3));
  ZK_CUDA(cudaEventRecord(f.ev_g1w, f.s3));

  // SpMV per job on the polynomial streams, then every job's H pipeline in
  // one persistent launch (work items of all sizes from one device queue)
  const int np = (int)std::min<size_t>(nj, FusedWs::kPolyStreams);
  for (int q = 0; q < np; q++) ZK_CUDA(cudaStreamWaitEvent(f.sp[q], f.ev_staged, 0));
  for (size_t k = 0; k < nj; k++)
    spmv_enqueue(g.jobs[k].c, we_of(k), poly_of(k, 0), poly_of(k, 1),
                 f.sp[k % FusedWs::kPolyStreams]);
  for (int q = 1; q < np; q++) {
    ZK_CUDA(cudaEventRecord(f.ev_sp[q], f.sp[q]));
    ZK_CUDA(cudaStreamWaitEvent(f.sp[0], f.ev_sp[q], 0));
  }
  for (size_t k0 = 0; k0 < nj; k0 += kMaxHJobs) {
    HJob hj[kMaxHJobs];
    const size_t cnt = std::min<size_t>(kMaxHJobs, nj - k0);
    for (size_t q = 0; q < cnt; q++) {
      const size_t k = k0 + q;
      hj[q] = HJob{poly_of(k, 0), poly_of(k, 1), poly_of(k, 2), poly_of(k, 3),
                   g.jobs[k].c->log_n};
    }
    hpoly_multi(ctx->ntt, (int)cnt, hj, f.hsync.as<uint32_t>(), f.sp[0]);
    // the launch's status word (the next launch clears the sync words)
    ZK_CUDA(cudaMemcpyAsync(f.hflag.as<uint32_t>() + k0 / kMaxHJobs, f.hsync.ptr,
                            sizeof(uint32_t), cudaMemcpyDeviceToHost, f.sp[0]));
  }
  ZK_CUDA(cudaEventRecord(f.ev_sp[0], f.sp[0]));
  ZK_CUDA(cudaStreamWaitEvent(f.s1, f.ev_sp[0], 0));

  // H of every job on s1
  for (size_t k = 0; k < nj; k++) {
    tab[k] = g.jobs[k].c->tab_h.ptr;
    sc[k] = poly_of(k, 3);
    cnt[k] = g.jobs[k].c->n;
  }
  g.rh = msm_enqueue_fixed_multi(false, insth, tab.data(), sc.data(), cnt.data(), c1, f.gh.ptr,
                                 f.gh.cap, cfgh, f.s1);
  ZK_CUDA(cudaMemcpyAsync(f.winh.ptr, g.rh.d_data, g.rh.bytes, cudaMemcpyDeviceToHost, f.s1));
  ZK_CUDA(cudaStreamWaitEvent(f.s1, f.ev_g2, 0));
  ZK_CUDA(cudaStreamWaitEvent(f.s1, f.ev_g1w, 0));
}

void fused_finish(FusedWs& f, const Group& g, bool blind, const uint64_t* rs, const uint64_t* ss,
                  uint64_t* proofs) {
  ZK_CUDA(cudaEventSynchronize(f.ev_done));
  const size_t nj = g.jobs.size();
  for (size_t q = 0; q < (nj + kMaxHJobs - 1) / kMaxHJobs; q++)
    ZK_REQUIRE(f.hflag.as<uint32_t>()[q] == 0, ZK_ETIMEOUT,
               "fused batch: a wait inside the H pipeline gave up");
  std::vector<ProofXyzz> px(nj);
  std::vector<uint64_t*> out(nj);
  for (size_t k = 0; k < nj; k++) {
    const size_t i = g.jobs[k].idx, b = k * g.per_job;
    const auto a = msm_g1_combine_xyzz(f.win1w.ptr, g.rw, (int)b);
    const auto c = msm_g1_combine_xyzz(f.win1w.ptr, g.rw, (int)b + 1);
    const auto h = msm_g1_combine_xyzz(f.winh.ptr, g.rh, (int)k);
    const auto b2 = msm_g2_combine_xyzz(f.win2.ptr, g.r2, (int)k);
    host::Xyzz<host::Fp> b1;
    if (blind) b1 = msm_g1_combine_xyzz(f.win1w.ptr, g.rw, (int)b + 2);
    px[k] = assemble_proof(g.jobs[k].c, a, b2, c.add(h), blind ? &b1 : nullptr,
                           blind ? rs + 4 * i : nullptr, blind ? ss + 4 * i : nullptr);
    out[k] = proofs + 32 * i;
  }
  // every proof of the group made affine with one shared inversion
  proofs_to_affine(px.data(), nj, out.data());
}

}  // namespace

void FusedWs::drop_graphs() {
  for (Graph& g : graphs) cudaGraphExecDestroy(g.exec);
  graphs.clear();
}

FusedWs::~FusedWs() {
  drop_graphs();
  if (!ready) return;
  for (cudaStream_t st : {s1, s2, s3}) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (int q = 0; q < kPolyStreams; q++) {
    cudaStreamSynchronize(sp[q]);
    cudaStreamDestroy(sp[q]);
    cudaEventDestroy(ev_sp[q]);
  }
  for (cudaEvent_t e : {ev_staged, ev_g2, ev_g1w, ev_done}) cudaEventDestroy(e);
}

void prove_batch_fused(zk_ctx* ctx, size_t count, zk_circuit* const* cs,
                       const uint64_t* const* wits, const size_t* nwits, bool on_device,
                       const uint64_t* rs, const uint64_t* ss, uint64_t* proofs, int group) {
  ZK_REQUIRE(group >= 1, ZK_EINVAL, "batch: group size must be >= 1");
  ZK_REQUIRE(count == 0 || (cs && wits && nwits && proofs), ZK_EINVAL, "batch: NULL argument");
  const bool blind = rs && ss;
  for (size_t i = 0; i < count; i++) {
    ZK_REQUIRE(cs[i] && cs[i]->ctx == ctx, ZK_EINVAL, "batch: circuit from another context");
    check_job(cs[i], wits[i], nwits[i], blind);
    ZK_REQUIRE(cs[i]->tab_c[0] != 0, ZK_EINVAL,
               "fused batch: every circuit needs fixed-base tables (zk_circuit_precompute)");
    note_witness(cs[i], wits[i], on_device);
  }
  // groups: same table window bits, bounded instances and records
  const int gmax = std::min(group, kMsmMaxInstances / (blind ? 3 : 2));
  std::map<std::pair<int, int>, std::vector<Job>> by_key;
  for (size_t i = 0; i < count; i++)
    by_key[{cs[i]->tab_c[0], cs[i]->tab_c[1]}].push_back(Job{i, cs[i]});
  std::vector<Group> groups;
  for (auto& kv : by_key) {
    Group cur;
    size_t recs = 0;
    for (const Job& j : kv.second) {
      const size_t r = records_of(j.c, blind);
      if (!cur.jobs.empty() && ((int)cur.jobs.size() >= gmax || recs + r > kGroupRecordCap)) {
        groups.push_back(std::move(cur));
        cur = Group();
        recs = 0;
      }
      cur.jobs.push_back(j);
      recs += r;
    }
    if (!cur.jobs.empty()) groups.push_back(std::move(cur));
  }
  ZK_CUDA(cudaEventRecord(ctx->ws.ev_begin_pool(), ctx->stream));
  const Group* pending[2] = {nullptr, nullptr};
  for (size_t gi = 0; gi < groups.size(); gi++) {
    FusedWs& f = ctx->fused[gi & 1];
    if (pending[gi & 1]) fused_finish(f, *pending[gi & 1], blind, rs, ss, proofs);
    fused_launch(ctx, f, groups[gi], wits, on_device, blind, ctx->ws.ev_begin);
    ZK_CUDA(cudaStreamWaitEvent(ctx->stream, f.ev_done, 0));
    pending[gi & 1] = &groups[gi];
  }
  for (size_t gi = groups.size() > 2 ? groups.size() - 2 : 0; gi < groups.size(); gi++)
    fused_finish(ctx->fused[gi & 1], groups[gi], blind, rs, ss, proofs);
}

}  // namespace zk
