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

// ctx or the per-device default context, with its device made current
inline zk_ctx* resolve_ctx(zk_ctx* ctx) {
  if (!ctx) return default_ctx();
  use_device(ctx);
  return ctx;
}
}  // namespace zk
