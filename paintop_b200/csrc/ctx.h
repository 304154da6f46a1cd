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
  bool graphs = true;          // capture device-pointer solves into a CUDA graph
  cudaGraphExec_t gexec = nullptr;
  std::string gkey;            // the plan the cached graph was captured for
  cudaGraphExec_t mgexec[2] = {nullptr, nullptr};  // multigrid-CG iteration: first / later
  std::string mgkey;           // the problem shape and arena the multigrid graphs were captured for
  long long mgnodes = 0;       // kernels in one of those iterations
  // host-buffer solves: row bands of an output that hold no interior tile are
  // copied back from the staged target on `stream2` while the solve runs
  cudaStream_t stream2 = nullptr;
  cudaEvent_t band_ev = nullptr;   // the band flags are on the host
  cudaEvent_t side_ev = nullptr;   // stream2's copies are done
  int *band_host = nullptr;        // pinned: one flag per band of every image
  size_t band_cap = 0;

  bool reserve_bands(size_t n) {
    if (!stream2 && cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking) != cudaSuccess) return false;
    if (!band_ev && cudaEventCreateWithFlags(&band_ev, cudaEventDisableTiming) != cudaSuccess) return false;
    if (!side_ev && cudaEventCreateWithFlags(&side_ev, cudaEventDisableTiming) != cudaSuccess) return false;
    if (n <= band_cap) return true;
    if (band_host) cudaFreeHost(band_host);
    band_host = nullptr;
    band_cap = 0;
    if (cudaHostAlloc(reinterpret_cast<void **>(&band_host), n * sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
      band_host = nullptr;
      return false;
    }
    band_cap = n;
    return true;
  }

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
    if (stream2) { cudaStreamSynchronize(stream2); cudaStreamDestroy(stream2); stream2 = nullptr; }
    if (band_ev) { cudaEventDestroy(band_ev); band_ev = nullptr; }
    if (side_ev) { cudaEventDestroy(side_ev); side_ev = nullptr; }
    if (band_host) { cudaFreeHost(band_host); band_host = nullptr; band_cap = 0; }
    if (arena) cudaFree(arena);
    arena = nullptr;
    arena_cap = 0;
  }
};
