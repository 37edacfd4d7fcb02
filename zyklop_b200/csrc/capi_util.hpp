// Shared helpers of the C ABI translation units: every entry point runs its
// body inside ZK_API_BEGIN / ZK_API_END, which turns library exceptions into
// status codes and a thread-local message (zk_last_error).
#pragma once
#include <new>
#include <stdexcept>

#include "context.hpp"
#include "runtime.hpp"

#define ZK_API_BEGIN try {
#define ZK_API_END                                           \
  }                                                          \
  catch (const zk::Error& e) {                               \
    zk::set_last_error(e.code, e.what());                    \
    return e.code;                                           \
  }                                                          \
  catch (const std::bad_alloc&) {                            \
    zk::set_last_error(ZK_ENOMEM, "host allocation failed"); \
    return ZK_ENOMEM;                                        \
  }                                                          \
  catch (const std::exception& e) {                          \
    zk::set_last_error(ZK_EINTERNAL, e.what());              \
    return ZK_EINTERNAL;                                     \
  }                                                          \
  zk::set_last_error(ZK_OK, "");                             \
  return ZK_OK;

namespace zk {
const char* last_error();

// Makes ctx's device current and routes kernel timing to its profiler when
// profiling is on.
inline zk_ctx* enter_ctx(zk_ctx* ctx) {
  use_device(ctx);
  set_current_profiler(ctx->profiling ? &ctx->prof : nullptr);
  return ctx;
}

// ctx or the per-device default context, entered
inline zk_ctx* resolve_ctx(zk_ctx* ctx) { return enter_ctx(ctx ? ctx : default_ctx()); }
}  // namespace zk
