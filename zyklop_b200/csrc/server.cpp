// Proof server: continuous batching over resident circuits.
//
// Requests (circuit, host witness, optional blinding) queue up; one worker
// thread keeps up to `max_inflight` proofs on the GPU, each in its own
// workspace slot with its own streams.  A request is admitted as soon as a
// slot is free and the device has room for that slot's buffers (admission by
// free memory); finished proofs are detected by polling their completion
// events, combined on the host and handed back, so requests that arrive while
// others run overlap with them on the device.  No reference counterpart: the
// reference proves one file pair per process.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "capi_util.hpp"
#include "prover.hpp"

namespace zk {
// prover.cu internals used by the server
size_t ws_bytes_needed(zk_circuit* c, const ProveWs& ws, bool blind);
void ws_submit(zk_circuit* c, ProveWs& ws, const uint64_t* witness, bool blind, Stager& stager);
bool ws_ready(ProveWs& ws);
void ws_collect(zk_circuit* c, ProveWs& ws, bool blind, const uint64_t* r, const uint64_t* s,
                uint64_t proof[32]);
}  // namespace zk

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  zk_circuit* circuit = nullptr;
  const uint64_t* witness = nullptr;
  size_t n_witness = 0;
  bool blind = false;
  bool waited = false;  // admission held it back at least once
  uint64_t r[4] = {0, 0, 0, 0}, s[4] = {0, 0, 0, 0};
  uint64_t proof[32] = {};
  int status = -1;  // -1 pending, else a ZK_* code
  std::string error;
  Clock::time_point submitted, done;
};

struct Slot {
  std::unique_ptr<zk::ProveWs> ws{new zk::ProveWs()};
  std::shared_ptr<Request> req;
};

}  // namespace

struct zk_server {
  zk_ctx* ctx = nullptr;
  int max_inflight = 4;
  size_t reserve = 0;  // device bytes admission keeps free
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> tickets;
  uint64_t next_ticket = 1;
  bool stopping = false;
  std::vector<Slot> slots;
  zk::Stager stager;
  std::thread worker;
  // statistics
  // admission order: 0 arrival order; 1 smallest circuit first among the
  // first kLookahead queued, except that a request older than max_wait goes
  // first (no starvation)
  static constexpr size_t kLookahead = 64;
  int policy = 1;
  std::chrono::milliseconds max_wait{500};
  uint64_t completed = 0, failed = 0;  // under mu
  std::atomic<uint64_t> peak_inflight{0}, admission_waits{0};  // written by the worker

  void run();
  size_t pick_locked() const {
    if (policy == 0 || Clock::now() - queue.front()->submitted > max_wait) return 0;
    size_t best = 0;
    const size_t look = std::min(queue.size(), kLookahead);
    for (size_t i = 1; i < look; i++)
      if (queue[i]->circuit->n < queue[best]->circuit->n) best = i;
    return best;
  }
  void deliver(const std::shared_ptr<Request>& r, int status, const std::string& err) {
    std::lock_guard<std::mutex> g(mu);
    r->status = status;
    r->error = err;
    r->done = Clock::now();
    if (status == ZK_OK) completed++;
    else failed++;
    cv_done.notify_all();
  }
};

void zk_server::run() {
  cudaSetDevice(ctx->device);
  for (;;) {
    // 1. collect finished proofs
    bool progressed = false;
    size_t busy = 0;
    for (Slot& sl : slots) {
      if (!sl.req) continue;
      busy++;
      if (!zk::ws_ready(*sl.ws)) continue;
      std::shared_ptr<Request> r = std::move(sl.req);
      try {
        zk::ws_collect(r->circuit, *sl.ws, r->blind, r->blind ? r->r : nullptr,
                       r->blind ? r->s : nullptr, r->proof);
        deliver(r, ZK_OK, "");
      } catch (const zk::Error& e) {
        deliver(r, e.code, e.what());
      } catch (const std::exception& e) {
        deliver(r, ZK_EINTERNAL, e.what());
      }
      progressed = true;
      busy--;
    }
    // 2. admit queued requests into free slots while memory allows
    for (;;) {
      std::shared_ptr<Request> r;
      {
        std::unique_lock<std::mutex> g(mu);
        if (queue.empty()) break;
        r = queue[pick_locked()];
      }
      Slot* free_slot = nullptr;
      for (Slot& sl : slots)
        if (!sl.req) {
          free_slot = &sl;
          break;
        }
      if (!free_slot && (int)slots.size() < max_inflight) {
        slots.emplace_back();
        free_slot = &slots.back();
      }
      if (!free_slot) break;
      size_t need = 0;
      try {
        need = zk::ws_bytes_needed(r->circuit, *free_slot->ws, r->blind);
      } catch (...) {
        need = 0;
      }
      if (need) {
        const size_t fr = zk::device_free_bytes();
        if (fr < need + reserve) {
          if (busy > 0) {  // wait for running proofs to release memory
            if (!r->waited) admission_waits++;
            r->waited = true;
            break;
          }
        }
      }
      {
        std::lock_guard<std::mutex> g(mu);
        const auto it = std::find(queue.begin(), queue.end(), r);
        if (it == queue.end()) continue;  // cancelled meanwhile
        queue.erase(it);
      }
      try {
        if (r->n_witness < r->circuit->m1)
          throw zk::Error(ZK_EWITNESS, "witness has fewer values than the circuit's nVars");
        std::lock_guard<std::mutex> g(ctx->mu);
        zk::set_current_profiler(nullptr);
        zk::ws_submit(r->circuit, *free_slot->ws, r->witness, r->blind, stager);
        free_slot->req = r;
        busy++;
        if (busy > peak_inflight.load()) peak_inflight.store(busy);
      } catch (const zk::Error& e) {
        deliver(r, e.code, e.what());
      } catch (const std::exception& e) {
        deliver(r, ZK_EINTERNAL, e.what());
      }
      progressed = true;
    }
    std::unique_lock<std::mutex> g(mu);
    if (stopping && queue.empty() && busy == 0) return;
    if (progressed) continue;
    if (busy == 0) {
      cv_work.wait(g, [&] { return stopping || !queue.empty(); });
    } else {
      g.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
}

extern "C" {

int zk_server_create(zk_ctx* ctx, int max_inflight, size_t reserve_bytes, zk_server** out) {
  ZK_API_BEGIN
  ZK_REQUIRE(out, ZK_EINVAL, "zk_server_create: NULL output");
  ZK_REQUIRE(max_inflight >= 1 && max_inflight <= 16, ZK_EINVAL, "zk_server_create: 1..16 in flight");
  *out = nullptr;
  ctx = zk::resolve_ctx(ctx);
  std::unique_ptr<zk_server> s(new zk_server());
  s->ctx = ctx;
  s->max_inflight = max_inflight;
  s->reserve = reserve_bytes;
  zk_server* raw = s.get();
  s->worker = std::thread([raw] { raw->run(); });
  *out = s.release();
  ZK_API_END
}

int zk_server_submit(zk_server* s, zk_circuit* c, const uint64_t* h_witness, size_t n_witness,
                     const uint64_t* r, const uint64_t* sb, uint64_t* ticket) {
  ZK_API_BEGIN
  ZK_REQUIRE(s && c && h_witness && ticket, ZK_EINVAL, "zk_server_submit: NULL argument");
  ZK_REQUIRE(c->ctx == s->ctx, ZK_EINVAL, "zk_server_submit: circuit from another context");
  ZK_REQUIRE((r == nullptr) == (sb == nullptr), ZK_EINVAL, "zk_server_submit: give both r and s or neither");
  ZK_REQUIRE(!r || c->has_b1, ZK_EFORMAT, "blinding needs zkey section 6 (B1 points)");
  auto q = std::make_shared<Request>();
  q->circuit = c;
  q->witness = h_witness;
  q->n_witness = n_witness;
  q->blind = r != nullptr;
  if (r) {
    memcpy(q->r, r, 32);
    memcpy(q->s, sb, 32);
  }
  q->submitted = Clock::now();
  {
    std::lock_guard<std::mutex> g(s->mu);
    ZK_REQUIRE(!s->stopping, ZK_EINVAL, "zk_server_submit: server is stopping");
    q->ticket = s->next_ticket++;
    s->tickets[q->ticket] = q;
    s->queue.push_back(q);
  }
  s->cv_work.notify_one();
  *ticket = q->ticket;
  ZK_API_END
}

int zk_server_wait(zk_server* s, uint64_t ticket, int timeout_ms, uint64_t* proof,
                   double* latency_ms) {
  ZK_API_BEGIN
  ZK_REQUIRE(s && proof, ZK_EINVAL, "zk_server_wait: NULL argument");
  std::unique_lock<std::mutex> g(s->mu);
  auto it = s->tickets.find(ticket);
  ZK_REQUIRE(it != s->tickets.end(), ZK_EINVAL, "zk_server_wait: unknown ticket");
  std::shared_ptr<Request> q = it->second;
  auto pred = [&] { return q->status >= 0; };
  if (timeout_ms < 0) s->cv_done.wait(g, pred);
  else if (!s->cv_done.wait_for(g, std::chrono::milliseconds(timeout_ms), pred))
    throw zk::Error(ZK_ETIMEOUT, "zk_server_wait: proof not ready before the timeout");
  s->tickets.erase(ticket);
  if (latency_ms)
    *latency_ms = std::chrono::duration<double, std::milli>(q->done - q->submitted).count();
  if (q->status != ZK_OK) throw zk::Error(q->status, q->error);
  memcpy(proof, q->proof, sizeof(q->proof));
  ZK_API_END
}

int zk_server_stats(zk_server* s, uint64_t* completed, uint64_t* failed, uint64_t* peak_inflight,
                    uint64_t* admission_waits) {
  ZK_API_BEGIN
  ZK_REQUIRE(s, ZK_EINVAL, "zk_server_stats: NULL server");
  std::lock_guard<std::mutex> g(s->mu);
  if (completed) *completed = s->completed;
  if (failed) *failed = s->failed;
  if (peak_inflight) *peak_inflight = s->peak_inflight.load();
  if (admission_waits) *admission_waits = s->admission_waits.load();
  ZK_API_END
}

int zk_server_set_policy(zk_server* s, int policy, int max_wait_ms) {
  ZK_API_BEGIN
  ZK_REQUIRE(s, ZK_EINVAL, "zk_server_set_policy: NULL server");
  ZK_REQUIRE(policy == 0 || policy == 1, ZK_EINVAL, "zk_server_set_policy: policy 0 or 1");
  ZK_REQUIRE(max_wait_ms >= 0, ZK_EINVAL, "zk_server_set_policy: negative wait");
  std::lock_guard<std::mutex> g(s->mu);
  s->policy = policy;
  s->max_wait = std::chrono::milliseconds(max_wait_ms);
  ZK_API_END
}

int zk_server_cancel_queued(zk_server* s, uint64_t* n_cancelled) {
  ZK_API_BEGIN
  ZK_REQUIRE(s, ZK_EINVAL, "zk_server_cancel_queued: NULL server");
  std::lock_guard<std::mutex> g(s->mu);
  const uint64_t n = s->queue.size();
  for (auto& q : s->queue) {
    q->status = ZK_ECANCELED;
    q->error = "request cancelled before it started";
    q->done = Clock::now();
  }
  s->queue.clear();
  s->cv_done.notify_all();
  if (n_cancelled) *n_cancelled = n;
  ZK_API_END
}

int zk_server_destroy(zk_server* s) {
  ZK_API_BEGIN
  if (!s) return ZK_OK;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  zk::use_device(s->ctx);
  delete s;
  ZK_API_END
}

}  // extern "C"
