// noalloc.cu -- pt_poisson_solve_noalloc: the solve for callers that must not
// allocate memory.
//
// Who needs it. Some hosts own all device memory themselves: a plugin running
// inside another framework's caching allocator must not call cudaMalloc or
// cudaFree behind that allocator's back, and a latency-critical thread cannot
// afford the device-wide synchronisation cudaMalloc/cudaFree may imply. Such a
// caller already holds device buffers for its images; it needs the solver to
// find its working memory somewhere that costs no allocation call.
//
// How. All scratch the solve needs (plane pools, tile list, per-system state,
// partial sums, history, barrier words) lives in one file-scope device array of
// fixed size, g_noalloc_scratch (PT_NOALLOC_SCRATCH_BYTES). Every GPU that loads
// the library holds that array until the process exits. The entry point computes
// its layout inside the array, rejects problems that do not fit, and launches
// the same kernels as pt_poisson_solve on the caller's stream. It makes no call
// to cudaMalloc, cudaFree, cudaStreamCreate or any other allocating routine and
// no host heap allocation: descriptors and results travel through stack arrays.
//
// Set-up. In host code the array's name is only a stand-in for the device
// symbol, not a device address. The first call on each device, with that
// device current, asks the runtime for the array's device address with
// cudaGetSymbolAddress and caches it; later calls on that device reuse it.
// Make that first call before any stream capture. Because the CUDA runtime
// loads modules lazily, that first call is also when the library's kernels and
// this array are placed on the device, which takes device memory once; the
// promise of no allocation holds from the second call on each device. The
// cached address belongs to the device's current context: after
// cudaDeviceReset it is stale, and calls after a reset are not supported.
// A stream that is capturing is refused with PT_INVALID_ARG.
//
// Sharing. Every call uses the same array and leaves its contents behind. A
// call clears what must start at zero (barrier and error words, history) and
// the assembly kernel initialises every cell a solve reads. Two calls whose
// work overlaps on the GPU would race on the array; this function prevents that
// within a process by holding a mutex for the whole call and waiting for its
// stream before it returns.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/paintop_cuda.h"
#include "rbsor_launch.h"
#include "abi_guard.h"

using namespace ptk;

namespace {

// The scratch array. 64 MiB is enough for one 1024x1024 single-channel image
// or one 512x512 RGBA image at 2000 sweeps of history.
static __device__ __align__(256) unsigned char g_noalloc_scratch[PT_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
constexpr uint32_t kMaxChannels = 8;

std::mutex g_mu;
void *g_scratch_dev[kMaxDevices] = {};  // device address of the array, per device

size_t aup(size_t v) { return (v + 255) / 256 * 256; }

__global__ void k_fill_tiles(Tile *tiles, int ntiles, int tiles_per_sys, int ntx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int r = t % tiles_per_sys;
  tiles[t] = Tile{t / tiles_per_sys, r % ntx, r / ntx, 0};
}

int default_config(const pt_problem &p) {
  const double total = (double)p.width * p.height * p.channels;
  return total < 4.0e6 ? 3 : 2;  // the built-in default of the tuned table
}

}  // namespace

extern "C" pt_status pt_poisson_solve_noalloc(const pt_problem *p, float *out_candidate,
                                              pt_report *reports, double *history,
                                              void *stream) {
  return abi_guard(nullptr, [&]() -> pt_status {
    if (!p || !reports) return PT_INVALID_ARG;
    if (!(p->flags & PT_FLAG_DEVICE_POINTERS)) return PT_INVALID_ARG;
    if (p->flags & (PT_FLAG_WARM_START | PT_FLAG_OMEGA_AUTO)) return PT_INVALID_ARG;
    if (p->channels > kMaxChannels) return PT_INVALID_ARG;
    if (p->channels > 0 && (p->width == 0 || p->height == 0 || !p->source_or_guidance ||
                            !p->target_or_anchor || !p->mask || !out_candidate))
      return PT_INVALID_ARG;
    // the limits pt_poisson_solve applies; they also keep W, H and the tile
    // counts below positive when cast to int
    const unsigned long long px = (unsigned long long)p->width * p->height;
    if (p->width > (1u << 30) || p->height > (1u << 30) || px > (1ull << 31) ||
        px * (p->channels ? p->channels : 1) > (1ull << 34))
      return PT_INVALID_ARG;
    if (!std::isfinite(p->lambda) || p->lambda < 0.0 || !std::isfinite(p->tolerance) ||
        p->tolerance <= 0.0 || !std::isfinite(p->omega) || p->omega <= 0.0 || p->omega >= 2.0 ||
        p->max_iterations > 1000000u)
      return PT_INVALID_ARG;
    const uint32_t C = p->channels;
    if (C == 0) {
      pt_report r{};
      r.converged = 1; r.stop_reason = PT_STOP_CONVERGED; r.tolerance = p->tolerance; r.channel = -1;
      reports[0] = r;
      return PT_OK;
    }
    abi_test_fault();

    // ---- layout inside the scratch array (no allocation)
    const int cfg = default_config(*p);
    const TileConfig tc = tile_config(cfg);
    const int W = (int)p->width, H = (int)p->height;
    const int pw = (int)(((size_t)(W + 1) / 2 + 3) / 4 * 4);
    const int ntx = (W + tc.tw - 1) / tc.tw, nty = (H + tc.th - 1) / tc.th;
    const long long tps = (long long)ntx * nty;
    const long long ntiles = tps * C;
    const long long plane = (long long)H * pw;
    const long long cells = 2 * plane * C;
    size_t o = 0, sys_o, st_o, claim_o, arrive_o, tiles_o, tc_o, tbox_o, act_o, e0_o, e1_o, g_o, cell_o, u_o, bp_o, part_o, fpart_o,
           hist_o, bar_o, err_o;
    auto take = [&](size_t bytes) { size_t r = o; o = aup(o + (bytes ? bytes : 1)); return r; };
    sys_o = take(C * sizeof(SysDesc));
    st_o = take(C * sizeof(SysState));
    claim_o = take(C * sizeof(unsigned long long));
    arrive_o = take(C * sizeof(unsigned));
    tiles_o = take(ntiles * sizeof(Tile));
    tc_o = take(ntiles * sizeof(int));
    tbox_o = take(ntiles * sizeof(int4));
    act_o = take(ntiles * sizeof(int));
    e0_o = take(cells * sizeof(float));
    e1_o = take(cells * sizeof(float));
    g_o = take(cells * sizeof(float));
    cell_o = take(cells);
    u_o = take(cells * sizeof(double));
    bp_o = take(cells * sizeof(double));
    part_o = take((size_t)tc.S * ntiles * sizeof(double));
    fpart_o = take(2 * ntiles * sizeof(double));
    hist_o = take((size_t)C * p->max_iterations * sizeof(double));
    bar_o = take(kBarWords * sizeof(unsigned));
    err_o = take(sizeof(int));
    if (o > (size_t)PT_NOALLOC_SCRATCH_BYTES) return PT_OOM;  // does not fit the fixed array

    std::lock_guard<std::mutex> lock(g_mu);
    cudaGetLastError();  // an earlier, unrelated runtime error must not fail this call's checks
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PT_NO_DEVICE;
    if (!g_scratch_dev[dev]) {
      // once per device, with that device current
      void *addr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
      if (e != cudaSuccess || !addr) {
        cudaGetLastError();
        return e == cudaErrorNoDevice ? PT_NO_DEVICE : PT_LAUNCH_FAILED;
      }
      g_scratch_dev[dev] = addr;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
      return PT_NO_DEVICE;
    char *base = static_cast<char *>(g_scratch_dev[dev]);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The call copies from host stack arrays and waits for its stream, neither of
    // which a capturing stream allows; refusing here leaves the caller's capture intact.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) { cudaGetLastError(); return PT_INVALID_ARG; }
    if (cap != cudaStreamCaptureStatusNone) return PT_INVALID_ARG;

    SysDesc descs[kMaxChannels];
    for (uint32_t c = 0; c < C; ++c) {
      SysDesc d{};
      d.inst = 0; d.chan = (int)c; d.W = W; d.H = H; d.C = (int)C; d.pw = pw;
      d.ntx = ntx; d.nty = nty; d.plane = plane; d.off = 2 * plane * c;
      d.tile0 = (int)(tps * c); d.ntiles = (int)tps;
      d.src = p->source_or_guidance; d.tgt = p->target_or_anchor; d.mask = p->mask;
      d.guess = nullptr; d.out = out_candidate;
      d.hist_off = (long long)c * p->max_iterations;
      d.omega = (float)p->omega;
      d.inv_denom = (float)(1.0 / (4.0 + p->lambda));
      d.lambda = p->lambda; d.tol = p->tolerance; d.max_it = (int)p->max_iterations; d.warm = 0;
      descs[c] = d;
    }

    KParams P{};
    P.sys = reinterpret_cast<const SysDesc *>(base + sys_o);
    P.st = reinterpret_cast<SysState *>(base + st_o);
    P.tiles = reinterpret_cast<const Tile *>(base + tiles_o);
    P.tcount = reinterpret_cast<int *>(base + tc_o);
    P.tbox = reinterpret_cast<int4 *>(base + tbox_o);
    P.act = reinterpret_cast<int *>(base + act_o);
    P.claim = reinterpret_cast<unsigned long long *>(base + claim_o);
    P.arrive = reinterpret_cast<unsigned *>(base + arrive_o);
    P.ntiles = (int)ntiles;
    P.nsys = (int)C;
    P.e0 = reinterpret_cast<float *>(base + e0_o);
    P.e1 = reinterpret_cast<float *>(base + e1_o);
    P.g = reinterpret_cast<float *>(base + g_o);
    P.cell = reinterpret_cast<uint8_t *>(base + cell_o);
    P.u = reinterpret_cast<double *>(base + u_o);
    P.bp = reinterpret_cast<double *>(base + bp_o);
    P.partial = reinterpret_cast<double *>(base + part_o);
    P.fpart = reinterpret_cast<double *>(base + fpart_o);
    P.hist = reinterpret_cast<double *>(base + hist_o);
    P.bar = reinterpret_cast<unsigned *>(base + bar_o);
    P.err = reinterpret_cast<int *>(base + err_o);
    P.budget_ns = 600ull * 1000000000ull;
    P.S = tc.S;

    // the array keeps the previous call's contents: zero what must start at zero
    cudaError_t e = cudaMemcpyAsync(base + sys_o, descs, C * sizeof(SysDesc), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + bar_o, 0, kBarWords * sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + err_o, 0, sizeof(int), st);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(base + hist_o, 0, (size_t)C * p->max_iterations * sizeof(double), st);
    if (e != cudaSuccess) { cudaGetLastError(); return PT_LAUNCH_FAILED; }
    k_fill_tiles<<<(unsigned)((ntiles + 255) / 256), 256, 0, st>>>(
        reinterpret_cast<Tile *>(base + tiles_o), (int)ntiles, (int)tps, ntx);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = launch_assembly(P, tc, st);
    int grid = 0;
    if (e == cudaSuccess) e = launch_solve(P, cfg, sms, st, &grid);
    if (e == cudaSuccess) e = launch_emit(P, 0, tc, (long long)W * H, st);
    SysState states[kMaxChannels];
    int kerr = 0;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(states, base + st_o, C * sizeof(SysState), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&kerr, base + err_o, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && history && p->max_iterations)
      e = cudaMemcpyAsync(history, base + hist_o, (size_t)C * p->max_iterations * sizeof(double),
                          cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { cudaGetLastError(); return PT_LAUNCH_FAILED; }
    if (kerr != 0) return PT_TIMEOUT;

    int worst = -1;
    for (uint32_t c = 0; c < C; ++c) {
      const SysState &s = states[c];
      pt_report r{};
      r.iterations = (uint32_t)s.iterations;
      r.stop_reason = s.status;
      r.converged = s.status == PT_STOP_CONVERGED;
      r.tolerance = p->tolerance;
      r.final_residual = s.last;
      r.history_len = r.iterations;
      r.omega_used = s.omega;
      r.refinements = (uint32_t)s.refinements;
      r.channel = (int)c;
      r.initial_residual = s.r0;
      reports[c] = r;
      if (worst < 0) {
        worst = (int)c;
      } else {
        const pt_report &a = reports[worst];
        if (r.iterations != a.iterations ? r.iterations > a.iterations
                                         : r.final_residual > a.final_residual)
          worst = (int)c;
      }
    }
    reports[C] = reports[worst];
    return PT_OK;
  });
}
