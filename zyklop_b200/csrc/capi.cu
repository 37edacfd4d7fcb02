// C ABI entry points for contexts and primitives (include/zyklop_b200.h).
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <vector>

#include "capi_util.hpp"
#include "context.hpp"
#include "field.cuh"

namespace zk {
const char* last_error();
void mul_generator(int group, const uint64_t* scalars, size_t n, uint64_t* px, uint64_t* py,
                   cudaStream_t st);

namespace {

std::mutex g_default_mu;
std::vector<zk_ctx*> g_defaults;

template <class C>
__global__ void k_field_op(int op, fe<C>* __restrict__ out, const fe<C>* __restrict__ a,
                           const fe<C>* __restrict__ b, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const fe<C> x = fe_load<C>(a, i);
  fe<C> r;
  switch (op) {
    case ZK_OP_MUL: r = x * fe_load<C>(b, i); break;
    case ZK_OP_ADD: r = x + fe_load<C>(b, i); break;
    case ZK_OP_SUB: r = x - fe_load<C>(b, i); break;
    case ZK_OP_SQR: r = fe_sqr(x); break;
    case ZK_OP_NEG: r = fe_neg(x); break;
    case ZK_OP_INV: r = fe_inv(x); break;
    case ZK_OP_ENCODE: r = fe_to_mont(x); break;
    default: r = fe_from_mont(x); break;
  }
  fe_store(out, i, r);
}

}  // namespace

zk_ctx* default_ctx() {
  int dev = 0;
  ZK_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(g_default_mu);
  if ((int)g_defaults.size() <= dev) g_defaults.resize(dev + 1, nullptr);
  if (!g_defaults[dev]) {
    zk_ctx* c = new zk_ctx();
    c->device = dev;
    c->is_default = true;
    // a blocking stream: ordered after the caller's work on the legacy
    // default stream, which is where the reference runs everything
    ZK_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault));
    g_defaults[dev] = c;
  }
  return g_defaults[dev];
}

void use_device(zk_ctx* ctx) { ZK_CUDA(cudaSetDevice(ctx->device)); }

}  // namespace zk

using namespace zk;



extern "C" {

const char* zk_version(void) { return "zyklop_b200 0.1.0 (sm_100a)"; }

const char* zk_last_error(void) { return zk::last_error(); }

int zk_ctx_create(int device, zk_ctx** out) {
  ZK_API_BEGIN
  ZK_REQUIRE(out, ZK_EINVAL, "zk_ctx_create: out is NULL");
  *out = nullptr;
  int count = 0;
  ZK_CUDA(cudaGetDeviceCount(&count));
  ZK_REQUIRE(device >= 0 && device < count, ZK_EINVAL, "zk_ctx_create: no such device");
  ZK_CUDA(cudaSetDevice(device));
  zk_ctx* c = new zk_ctx();
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault);
  if (e != cudaSuccess) {
    delete c;
    throw_cuda(e, "cudaStreamCreateWithFlags", __FILE__, __LINE__);
  }
  *out = c;
  ZK_API_END
}

int zk_ctx_destroy(zk_ctx* ctx) {
  ZK_API_BEGIN
  if (!ctx || ctx->is_default) return ZK_OK;
  use_device(ctx);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  ZK_API_END
}

int zk_ctx_set_stream(zk_ctx* ctx, void* stream) {
  ZK_API_BEGIN
  ZK_REQUIRE(ctx && !ctx->is_default, ZK_EINVAL, "zk_ctx_set_stream: needs a context from zk_ctx_create");
  enter_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  if (ctx->own_stream) ZK_CUDA(cudaStreamDestroy(ctx->stream));
  ctx->stream = reinterpret_cast<cudaStream_t>(stream);
  ctx->own_stream = false;
  ZK_API_END
}

int zk_release_cached_memory(zk_ctx* ctx) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  release_cached_memory();
  ZK_API_END
}

int zk_memory_stats(int device, zk_memory_stats_t* out) {
  ZK_API_BEGIN
  ZK_REQUIRE(out, ZK_EINVAL, "zk_memory_stats: NULL output");
  alloc_stats(&out->device_allocations, &out->device_allocated_bytes, &out->pinned_allocations);
  pool_usage(device, &out->pool_reserved_bytes, &out->pool_used_bytes);
  ZK_API_END
}

int zk_launch_count(uint64_t* out) {
  ZK_API_BEGIN
  ZK_REQUIRE(out, ZK_EINVAL, "zk_launch_count: NULL output");
  *out = launch_count();
  ZK_API_END
}

int zk_ctx_set_profiling(zk_ctx* ctx, int on) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ctx->profiling = on != 0;
  ZK_API_END
}

int zk_ctx_profile(zk_ctx* ctx, zk_profile* out) {
  ZK_API_BEGIN
  ZK_REQUIRE(out, ZK_EINVAL, "zk_ctx_profile: NULL output");
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  static_assert(ZK_PROF_KINDS == kProfKinds, "profile kinds");
  ctx->prof.collect(out->ms, out->launches, out->units);
  ZK_API_END
}

int zk_imad_probe(zk_ctx* ctx, double* tiops) {
  ZK_API_BEGIN
  ZK_REQUIRE(tiops, ZK_EINVAL, "zk_imad_probe: NULL output");
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  *tiops = imad_probe(ctx->stream);
  ZK_API_END
}

int zk_int_probe(zk_ctx* ctx, int kind, double* tiops) {
  ZK_API_BEGIN
  ZK_REQUIRE(tiops && (kind == 0 || kind == 1), ZK_EINVAL, "zk_int_probe: kind must be 0 or 1");
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  *tiops = imad_probe(ctx->stream, kind);
  ZK_API_END
}

int zk_ctx_sync(zk_ctx* ctx) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  ZK_API_END
}

int zk_field_op(zk_ctx* ctx, int field, int op, uint64_t* d_out, const uint64_t* d_a,
                const uint64_t* d_b, size_t n) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ZK_REQUIRE(field == ZK_FIELD_FP || field == ZK_FIELD_FR, ZK_EINVAL, "zk_field_op: bad field");
  ZK_REQUIRE(op >= 0 && op <= ZK_OP_DECODE, ZK_EINVAL, "zk_field_op: bad op");
  ZK_REQUIRE(n == 0 || (d_out && d_a), ZK_EINVAL, "zk_field_op: NULL buffer");
  const bool binary = op == ZK_OP_MUL || op == ZK_OP_ADD || op == ZK_OP_SUB;
  ZK_REQUIRE(!binary || n == 0 || d_b, ZK_EINVAL, "zk_field_op: binary op needs b");
  if (n) {
    const unsigned g = (unsigned)((n + 255) / 256);
    if (field == ZK_FIELD_FP)
      k_field_op<FpCfg><<<g, 256, 0, ctx->stream>>>(op, reinterpret_cast<fp_t*>(d_out),
                                                    reinterpret_cast<const fp_t*>(d_a),
                                                    reinterpret_cast<const fp_t*>(d_b), n);
    else
      k_field_op<FrCfg><<<g, 256, 0, ctx->stream>>>(op, reinterpret_cast<fr_t*>(d_out),
                                                    reinterpret_cast<const fr_t*>(d_a),
                                                    reinterpret_cast<const fr_t*>(d_b), n);
    ZK_LAUNCHED();
  }
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  ZK_API_END
}

int zk_ntt(zk_ctx* ctx, uint64_t* d_a, uint32_t log_n, int inverse) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ZK_REQUIRE(d_a, ZK_EINVAL, "zk_ntt: NULL buffer");
  ZK_REQUIRE(log_n <= (uint32_t)kMaxLogN, ZK_EINVAL, "zk_ntt: log_n > 27");
  ctx->ntt_scratch.ensure((size_t)32 << log_n);
  ntt_inplace(ctx->ntt, d_a, (int)log_n, inverse != 0, ctx->ntt_scratch.ptr, ctx->stream);
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  ZK_API_END
}

int zk_hpoly(zk_ctx* ctx, uint64_t* d_aw, uint64_t* d_bw, uint32_t log_n, uint64_t* d_h) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ZK_REQUIRE(d_aw && d_bw && d_h, ZK_EINVAL, "zk_hpoly: NULL buffer");
  ZK_REQUIRE(log_n >= 1 && log_n < (uint32_t)kMaxLogN, ZK_EINVAL, "zk_hpoly: log_n out of range");
  ctx->ntt_scratch.ensure((size_t)32 << log_n);
  hpoly(ctx->ntt, d_aw, d_bw, ctx->ntt_scratch.as<uint64_t>(), (int)log_n, d_h, ctx->stream);
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  ZK_API_END
}

int zk_msm_g1(zk_ctx* ctx, const uint64_t* d_px, const uint64_t* d_py, const uint64_t* d_scalars,
              size_t n, uint64_t* h_out, int* is_inf) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ZK_REQUIRE(h_out, ZK_EINVAL, "zk_msm_g1: NULL output");
  ZK_REQUIRE(n == 0 || (d_px && d_py && d_scalars), ZK_EINVAL, "zk_msm_g1: NULL input");
  const bool inf = msm_g1_run(points_soa(d_px, d_py), d_scalars, n, ctx->msm_scratch,
                              msm_config_for(ctx, false, n, ctx->scalar_dist, 0), ctx->stream, h_out);
  if (is_inf) *is_inf = inf ? 1 : 0;
  ZK_API_END
}

int zk_msm_g2(zk_ctx* ctx, const uint64_t* d_px, const uint64_t* d_py, const uint64_t* d_scalars,
              size_t n, uint64_t* h_out, int* is_inf) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ZK_REQUIRE(h_out, ZK_EINVAL, "zk_msm_g2: NULL output");
  ZK_REQUIRE(n == 0 || (d_px && d_py && d_scalars), ZK_EINVAL, "zk_msm_g2: NULL input");
  const bool inf = msm_g2_run(points_soa(d_px, d_py), d_scalars, n, ctx->msm_scratch,
                              msm_config_for(ctx, true, n, ctx->scalar_dist, 0), ctx->stream, h_out);
  if (is_inf) *is_inf = inf ? 1 : 0;
  ZK_API_END
}

int zk_msm_set_config(zk_ctx* ctx, int group, int c, int k0, int k1, int chunk) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ZK_REQUIRE(group == 1 || group == 2, ZK_EINVAL, "zk_msm_set_config: group must be 1 or 2");
  ZK_REQUIRE(c == 0 || (c >= 4 && c <= 21), ZK_EINVAL, "zk_msm_set_config: c must be 0 or 4..21");
  ZK_REQUIRE(k0 >= 0 && k0 <= 4096 && k1 >= 2 && k1 <= 4096, ZK_EINVAL,
             "zk_msm_set_config: k0 in 0..4096 (0 = by size), k1 in 2..4096");
  ZK_REQUIRE(chunk == 0 || (chunk >= 2 && chunk <= 4096 && (chunk & (chunk - 1)) == 0), ZK_EINVAL,
             "zk_msm_set_config: chunk must be 0 (by size) or a power of two in 2..4096");
  MsmConfig& m = ctx->msm_cfg[group - 1];
  m.c = c;
  m.k0 = k0;
  m.k1 = k1;
  m.chunk = chunk;
  ZK_API_END
}

int zk_msm_scratch_bytes(zk_ctx* ctx, int group, size_t n, size_t* bytes) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  ZK_REQUIRE(bytes, ZK_EINVAL, "zk_msm_scratch_bytes: NULL output");
  ZK_REQUIRE(group == 1 || group == 2, ZK_EINVAL, "zk_msm_scratch_bytes: group must be 1 or 2");
  *bytes = msm_scratch_bytes(n, group == 2, msm_config_for(ctx, group == 2, n, ctx->scalar_dist, 0));
  ZK_API_END
}

int zk_mul_generator(zk_ctx* ctx, int group, const uint64_t* d_scalars, size_t n, uint64_t* d_px,
                     uint64_t* d_py) {
  ZK_API_BEGIN
  ctx = resolve_ctx(ctx);
  std::lock_guard<std::mutex> g(ctx->mu);
  ZK_REQUIRE(group == 1 || group == 2, ZK_EINVAL, "zk_mul_generator: group must be 1 or 2");
  ZK_REQUIRE(n == 0 || (d_scalars && d_px && d_py), ZK_EINVAL, "zk_mul_generator: NULL buffer");
  mul_generator(group, d_scalars, n, d_px, d_py, ctx->stream);
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  ZK_API_END
}

}  // extern "C"
