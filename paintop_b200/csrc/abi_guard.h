// abi_guard.h -- no C++ exception crosses the C ABI.
//
// Every exported entry point that does host-side work runs its body through
// abi_guard. The library throws nothing itself, but the standard library it
// uses can (std::bad_alloc from containers and strings, std::system_error
// from std::thread and std::mutex). A host allocation failure becomes
// PT_OOM, anything else PT_INTERNAL, with the message on the context when
// there is one; RAII has released locks and device work is left as the
// failing call left it.
#pragma once

#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>

#include "../../include/paintop_cuda.h"
#include "ctx.h"

inline void abi_note(pt_ctx *ctx, const char *msg) noexcept {
  if (!ctx) return;
  try {
    ctx->last_error = msg;
  } catch (...) {
  }
}

template <class F>
inline pt_status abi_guard(pt_ctx *ctx, F &&body) noexcept {
  try {
    return body();
  } catch (const std::bad_alloc &) {
    abi_note(ctx, "host memory allocation failed");
    return PT_OOM;
  } catch (...) {
    abi_note(ctx, "unexpected host-side exception");
    return PT_INTERNAL;
  }
}

// Test hook: with PAINTOP_CUDA_FAULT set to "host-oom" or "host-exception",
// the entry points that call this throw std::bad_alloc or
// std::runtime_error after their argument checks and before any device
// work, so the guard's mapping is tested without a real failure.
inline void abi_test_fault() {
  const char *f = std::getenv("PAINTOP_CUDA_FAULT");
  if (!f) return;
  if (!std::strcmp(f, "host-oom")) throw std::bad_alloc();
  if (!std::strcmp(f, "host-exception")) throw std::runtime_error("injected host-side exception");
}
