// ctx.h -- the library context behind the opaque pt_ctx handle.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>
#include <string>

struct pt_ctx {
  int device = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;               // one call at a time per context
  void *arena = nullptr;       // device memory, grown to a high-water mark
  size_t arena_cap = 0;
  std::string last_error;
  double budget_s = 600.0;     // wall budget of one persistent solve
  int last_grid = 0;           // blocks of the last persistent launch
  int last_cfg = -1;           // tile configuration of the last solve
  int forced_cfg = -1;         // configuration override (-1: use the table)
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // call start, solve start/end, call end
  double last_solve_ms = 0.0;  // persistent kernel, CUDA events on `stream`
  double last_call_ms = 0.0;   // whole call from first upload to last download
  long long last_launches = 0; // kernels launched by the last call
  unsigned long long last_h2d = 0, last_d2h = 0;  // bytes the last solve moved each way
  bool graphs = true;          // capture device-pointer solves into a CUDA graph
  cudaGraphExec_t gexec = nullptr;
  std::string gkey;            // the plan the cached graph was captured for
  cudaGraphExec_t mgexec[2] = {nullptr, nullptr};  // multigrid-CG iteration: first / later
  std::string mgkey;           // the problem shape and arena the multigrid graphs were captured for
  long long mgnodes = 0;       // kernels in one of those iterations

  void drop_graphs() {
    if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }  // they point into the arena
    gkey.clear();
    for (auto &g : mgexec)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    mgkey.clear();
  }

  bool reserve(size_t bytes) {
    if (bytes <= arena_cap) return true;
    if (arena) {
      cudaStreamSynchronize(stream);
      drop_graphs();
      cudaFree(arena);
      arena = nullptr;
      arena_cap = 0;
    }
    size_t want = bytes + bytes / 4;
    if (cudaMalloc(&arena, want) != cudaSuccess) {
      cudaGetLastError();
      arena = nullptr;
      if (cudaMalloc(&arena, bytes) != cudaSuccess) {
        cudaGetLastError();
        arena = nullptr;
        return false;
      }
      want = bytes;
    }
    arena_cap = want;
    return true;
  }

  void release() {
    drop_graphs();
    for (auto &e : ev)
      if (e) { cudaEventDestroy(e); e = nullptr; }
    if (arena) cudaFree(arena);
    arena = nullptr;
    arena_cap = 0;
  }
};
