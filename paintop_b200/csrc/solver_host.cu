// solver_host.cu -- context, planning and the C-ABI solve entry points.
//
// pt_poisson_solve / pt_poisson_solve_batch replace the reference's per-channel
// chain blend_channels -> solve (crates/paintop-cpu/src/poisson_blend.rs:168-246,
// crates/paintop-cpu/src/poisson.rs:167-240) with one persistent launch over all
// channels of all images. Planning (tile grid, pool layout) needs only the
// problem extents, so a call issues no host synchronisation between its upload
// and its download.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/paintop_cuda.h"
#include "abi_guard.h"
#include "ctx.h"
#include "rbsor_launch.h"

using namespace ptk;

namespace {

constexpr size_t kAlign = 256;
size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

pt_status fail(pt_ctx *ctx, pt_status s, const std::string &msg) {
  if (ctx) ctx->last_error = msg;
  return s;
}

pt_status cuda_fail(pt_ctx *ctx, cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  if (ctx) ctx->last_error = m;
  if (e == cudaErrorMemoryAllocation) return PT_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return PT_NO_DEVICE;
  return PT_LAUNCH_FAILED;
}

// Host fault injection for tests of the error paths (no GPU fault involved):
// PAINTOP_CUDA_FAULT = "no-device" | "oom" | "launch".
int injected_fault() {
  const char *f = std::getenv("PAINTOP_CUDA_FAULT");
  if (!f) return 0;
  if (!std::strcmp(f, "no-device")) return 1;
  if (!std::strcmp(f, "oom")) return 2;
  if (!std::strcmp(f, "launch")) return 3;
  return 0;
}

bool finite(double v) { return std::isfinite(v); }

pt_status validate(pt_ctx *ctx, const pt_problem &p) {
  if (p.channels > 0 && (p.width == 0 || p.height == 0))
    return fail(ctx, PT_INVALID_ARG, "width and height must be >= 1");
  const unsigned long long px = (unsigned long long)p.width * p.height;
  if (p.width > (1u << 30) || p.height > (1u << 30) || px > (1ull << 31) ||
      px * (p.channels ? p.channels : 1) > (1ull << 34))
    return fail(ctx, PT_INVALID_ARG, "image too large");
  if (p.channels > 0 && (!p.source_or_guidance || !p.target_or_anchor || !p.mask))
    return fail(ctx, PT_INVALID_ARG, "source, target and mask must be non-null");
  if ((p.flags & PT_FLAG_WARM_START) && !p.initial_guess)
    return fail(ctx, PT_INVALID_ARG, "PT_FLAG_WARM_START needs initial_guess");
  if (!finite(p.lambda) || p.lambda < 0.0)
    return fail(ctx, PT_INVALID_ARG, "lambda must be a finite value >= 0");
  if (!finite(p.tolerance) || p.tolerance <= 0.0)
    return fail(ctx, PT_INVALID_ARG, "tolerance must be a finite value > 0");
  if (!(p.flags & (PT_FLAG_OMEGA_AUTO | PT_FLAG_MULTIGRID)) && (!finite(p.omega) || p.omega <= 0.0 || p.omega >= 2.0))
    return fail(ctx, PT_INVALID_ARG, "omega must be in (0, 2)");
  if (p.max_iterations > 1000000u)
    return fail(ctx, PT_INVALID_ARG, "max_iterations must be <= 1000000");
  return PT_OK;
}

struct Plan {
  int cfg;
  TileConfig tc;
  std::vector<SysDesc> sys;
  std::vector<Tile> tiles;
  long long cells = 0;     // elements per cell pool
  long long hist = 0;      // history entries
  long long in_floats = 0; // staged input floats (images + guesses)
  long long mask_floats = 0;
  long long out_floats = 0;
  std::vector<RegionDesc> regions;  // images labelled for the automatic omega
  long long rpix = 0;               // their pixels
};

// Arena layout (byte offsets) for one call.
struct Layout {
  size_t sys, st, claim, arrive, tiles, tcount, tbox, act, e0, e1, g, cell, u, bp, partial, fpart, hist, bar, err, in,
      mask, out, regions, label, rsize, rmax, bands, total;
};

// Row bands of every image (host-buffer solves: two ints each, the band's
// span of tile columns with interior cells).
size_t band_count(const Plan &pl) {
  size_t n = 0;
  for (const SysDesc &d : pl.sys)
    if (d.chan == 0) n += (size_t)d.nty;
  return n;
}

Layout layout(const Plan &pl, bool stage) {
  Layout L{};
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o = align_up(o + std::max<size_t>(bytes, 1), kAlign); return r; };
  const size_t nt = pl.tiles.size(), ns = pl.sys.size();
  L.sys = take(ns * sizeof(SysDesc));
  L.st = take(ns * sizeof(SysState));
  L.claim = take(ns * sizeof(unsigned long long));
  L.arrive = take(ns * sizeof(unsigned));
  L.tiles = take(nt * sizeof(Tile));
  L.tcount = take(nt * sizeof(int));
  L.tbox = take(nt * sizeof(int4));
  L.act = take(nt * sizeof(int));
  L.e0 = take(pl.cells * sizeof(float));
  L.e1 = take(pl.cells * sizeof(float));
  L.g = take(pl.cells * sizeof(float));
  L.cell = take(pl.cells);
  L.u = take(pl.cells * sizeof(double));
  L.bp = take(pl.cells * sizeof(double));
  L.partial = take((size_t)pl.tc.S * nt * sizeof(double));
  L.fpart = take(2 * nt * sizeof(double));
  L.hist = take(pl.hist * sizeof(double));
  L.bar = take(kBarWords * sizeof(unsigned));
  L.err = take(sizeof(int));
  L.in = stage ? take(pl.in_floats * sizeof(float)) : 0;
  L.mask = stage ? take(pl.mask_floats * sizeof(float)) : 0;
  L.out = stage ? take(pl.out_floats * sizeof(float)) : 0;
  L.regions = take(pl.regions.size() * sizeof(RegionDesc));
  L.label = take((size_t)pl.rpix * sizeof(int));
  L.rsize = take((size_t)pl.rpix * sizeof(int));
  L.rmax = take(pl.regions.size() * sizeof(int));
  L.bands = stage ? take(2 * band_count(pl) * sizeof(int)) : 0;
  L.total = o;
  return L;
}

}  // namespace

// ---------------------------------------------------------------------------
// tile-configuration choice (the autotuner's table; see autotune.cpp)
// ---------------------------------------------------------------------------
int ptk_choose_config(pt_ctx *ctx, const pt_problem *ps, uint32_t n);

pt_status ptk_solve_mg_batch(pt_ctx *ctx, const pt_problem *ps, uint32_t n, float *const *outs,
                             pt_report *const *reports, double *const *histories);

pt_status ptk_solve_batch(pt_ctx *ctx, const pt_problem *ps, uint32_t n, float *const *outs,
                          pt_report *const *reports, double *const *histories, int force_cfg) {
  if (!ctx) return PT_INVALID_ARG;
  if (n > 0 && (!ps || !outs || !reports)) return fail(ctx, PT_INVALID_ARG, "null batch arrays");
  for (uint32_t i = 0; i < n; ++i) {
    pt_status s = validate(ctx, ps[i]);
    if (s != PT_OK) return s;
    if (ps[i].channels > 0 && !outs[i]) return fail(ctx, PT_INVALID_ARG, "null output buffer");
    if (!reports[i]) return fail(ctx, PT_INVALID_ARG, "null report buffer");
  }
  const int fault = injected_fault();
  if (fault == 1) return fail(ctx, PT_NO_DEVICE, "injected: no device");
  if (fault == 2) return fail(ctx, PT_OOM, "injected: allocation failure");
  if (fault == 3) return fail(ctx, PT_LAUNCH_FAILED, "injected: launch failure");
  abi_test_fault();

  const bool mg = n > 0 && (ps[0].flags & PT_FLAG_MULTIGRID);
  for (uint32_t i = 0; i < n; ++i)
    if (((ps[i].flags & PT_FLAG_MULTIGRID) != 0) != mg)
      return fail(ctx, PT_INVALID_ARG, "PT_FLAG_MULTIGRID must agree across a batch");
  if (mg) return ptk_solve_mg_batch(ctx, ps, n, outs, reports, histories);  // every instance in each launch
  const bool devptr = n > 0 && (ps[0].flags & PT_FLAG_DEVICE_POINTERS);
  for (uint32_t i = 0; i < n; ++i)
    if (((ps[i].flags & PT_FLAG_DEVICE_POINTERS) != 0) != devptr)
      return fail(ctx, PT_INVALID_ARG, "PT_FLAG_DEVICE_POINTERS must agree across a batch");

  // ---- plan
  Plan pl;
  pl.cfg = force_cfg >= 0 ? force_cfg : ptk_choose_config(ctx, ps, n);
  pl.tc = tile_config(pl.cfg);
  std::vector<int> sys0(n, 0);
  for (uint32_t i = 0; i < n; ++i) {
    const pt_problem &p = ps[i];
    sys0[i] = (int)pl.sys.size();
    const int W = (int)p.width, H = (int)p.height, C = (int)p.channels;
    const int pw = (int)align_up((size_t)(W + 1) / 2, 4);
    const int ntx = (W + pl.tc.tw - 1) / pl.tc.tw, nty = (H + pl.tc.th - 1) / pl.tc.th;
    // automatic omega is chosen on the device from the region's extent
    const double omega = (p.flags & PT_FLAG_OMEGA_AUTO) ? -1.0 : p.omega;
    const long long img = (long long)W * H;
    int region1 = 0;
    if ((p.flags & PT_FLAG_OMEGA_AUTO) && C > 0 && img > 0) {
      pl.regions.push_back(RegionDesc{pl.rpix, W, H, (int)pl.sys.size(), 0});
      pl.rpix += img;
      region1 = (int)pl.regions.size();
    }
    for (int c = 0; c < C; ++c) {
      SysDesc d{};
      d.inst = (int)i; d.chan = c; d.W = W; d.H = H; d.C = C; d.pw = pw;
      d.ntx = ntx; d.nty = nty;
      d.plane = (long long)H * pw;
      d.off = pl.cells;
      pl.cells += 2 * d.plane;
      d.tile0 = (int)pl.tiles.size();
      d.ntiles = ntx * nty;
      for (int ty = 0; ty < nty; ++ty)
        for (int tx = 0; tx < ntx; ++tx) pl.tiles.push_back(Tile{(int)pl.sys.size(), tx, ty, 0});
      d.hist_off = pl.hist;
      pl.hist += p.max_iterations;
      d.omega = (float)omega;
      d.inv_denom = (float)(1.0 / (4.0 + p.lambda));
      d.lambda = p.lambda;
      d.tol = p.tolerance;
      d.max_it = (int)p.max_iterations;
      d.warm = (p.flags & PT_FLAG_WARM_START) ? 1 : 0;
      d.region1 = region1;
      pl.sys.push_back(d);
    }
    if (C > 0) {
      pl.in_floats += img * C * (1 + 1 + ((p.flags & PT_FLAG_WARM_START) ? 1 : 0));
      pl.mask_floats += img;
      pl.out_floats += img * C;
    }
  }
  const int nsys = (int)pl.sys.size();
  if (nsys == 0) {
    for (uint32_t i = 0; i < n; ++i) {
      pt_report r{};
      r.converged = 1; r.stop_reason = PT_STOP_CONVERGED; r.tolerance = ps[i].tolerance;
      r.channel = -1;
      reports[i][0] = r;
    }
    return PT_OK;
  }

  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaSetDevice");
  const Layout L = layout(pl, !devptr);
  if (!ctx->reserve(L.total)) return fail(ctx, PT_OOM, "device arena allocation failed");
  char *base = static_cast<char *>(ctx->arena);
  cudaStream_t st = ctx->stream;
  for (auto &e : ctx->ev)
    if (!e && cudaEventCreate(&e) != cudaSuccess) return fail(ctx, PT_LAUNCH_FAILED, "event create");
  cudaEventRecord(ctx->ev[0], st);

  // ---- stage inputs and bind the per-system image pointers
  unsigned long long h2d = 0, d2h = 0;  // bytes moved by this call
  {
    size_t in_off = 0, mask_off = 0, out_off = 0;
    for (uint32_t i = 0; i < n; ++i) {
      const pt_problem &p = ps[i];
      if (p.channels == 0) continue;
      const size_t img = (size_t)p.width * p.height, nf = img * p.channels;
      const float *src = p.source_or_guidance, *tgt = p.target_or_anchor, *mask = p.mask,
                  *guess = p.initial_guess;
      float *out = outs[i];
      if (!devptr) {
        // only the mask goes up now: which rows of the images the solve reads
        // is known once the tiles are counted (upload_active_rows below)
        float *in = reinterpret_cast<float *>(base + L.in) + in_off;
        float *dm = reinterpret_cast<float *>(base + L.mask) + mask_off;
        ce = cudaMemcpyAsync(dm, mask, img * sizeof(float), cudaMemcpyHostToDevice, st);
        if (ce != cudaSuccess) return cuda_fail(ctx, ce, "mask upload");
        h2d += img * sizeof(float);
        src = in; tgt = in + nf; mask = dm;
        guess = (p.flags & PT_FLAG_WARM_START) ? in + 2 * nf : nullptr;
        out = reinterpret_cast<float *>(base + L.out) + out_off;
        in_off += nf * ((p.flags & PT_FLAG_WARM_START) ? 3 : 2);
        mask_off += img;
        out_off += nf;
      }
      for (uint32_t c = 0; c < p.channels; ++c) {
        SysDesc &d = pl.sys[sys0[i] + c];
        d.src = src; d.tgt = tgt; d.mask = mask; d.out = out;
        d.guess = (p.flags & PT_FLAG_WARM_START) ? guess : nullptr;
      }
    }
  }
  h2d += pl.sys.size() * sizeof(SysDesc) + pl.tiles.size() * sizeof(Tile) + pl.regions.size() * sizeof(RegionDesc);
  ce = cudaMemcpyAsync(base + L.sys, pl.sys.data(), pl.sys.size() * sizeof(SysDesc),
                       cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(base + L.tiles, pl.tiles.data(), pl.tiles.size() * sizeof(Tile),
                         cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess && !pl.regions.empty())
    ce = cudaMemcpyAsync(base + L.regions, pl.regions.data(), pl.regions.size() * sizeof(RegionDesc),
                         cudaMemcpyHostToDevice, st);
  if (ce != cudaSuccess) return cuda_fail(ctx, ce, "plan upload");

  KParams P{};
  P.sys = reinterpret_cast<const SysDesc *>(base + L.sys);
  P.st = reinterpret_cast<SysState *>(base + L.st);
  P.tiles = reinterpret_cast<const Tile *>(base + L.tiles);
  P.tcount = reinterpret_cast<int *>(base + L.tcount);
  P.tbox = reinterpret_cast<int4 *>(base + L.tbox);
  P.act = reinterpret_cast<int *>(base + L.act);
  P.claim = reinterpret_cast<unsigned long long *>(base + L.claim);
  P.arrive = reinterpret_cast<unsigned *>(base + L.arrive);
  P.ntiles = (int)pl.tiles.size();
  P.nsys = nsys;
  P.e0 = reinterpret_cast<float *>(base + L.e0);
  P.e1 = reinterpret_cast<float *>(base + L.e1);
  P.g = reinterpret_cast<float *>(base + L.g);
  P.cell = reinterpret_cast<uint8_t *>(base + L.cell);
  P.u = reinterpret_cast<double *>(base + L.u);
  P.bp = reinterpret_cast<double *>(base + L.bp);
  P.partial = reinterpret_cast<double *>(base + L.partial);
  P.fpart = reinterpret_cast<double *>(base + L.fpart);
  P.hist = reinterpret_cast<double *>(base + L.hist);
  P.bar = reinterpret_cast<unsigned *>(base + L.bar);
  P.err = reinterpret_cast<int *>(base + L.err);
  P.budget_ns = (unsigned long long)(ctx->budget_s * 1e9);
  P.S = pl.tc.S;
  P.regions = reinterpret_cast<const RegionDesc *>(base + L.regions);
  P.nregions = (int)pl.regions.size();
  P.rpix = pl.rpix;
  P.label = reinterpret_cast<int *>(base + L.label);
  P.rsize = reinterpret_cast<int *>(base + L.rsize);
  P.rmax = reinterpret_cast<int *>(base + L.rmax);

  // ---- host buffers: upload only the part of the images the solve reads.
  // The tiles are counted from the masks, and for each image and row band of
  // tiles the first and last tile column holding interior cells come back to
  // the host (two ints per band). The solve reads source, target and guess
  // only at interior cells and their four neighbours, so each such band goes
  // up as one rectangle: its rows and one row either side, its span of tile
  // columns and one pixel either side. Only the band's span comes down; the
  // rest of the output is the target bit for bit and is filled on the host
  // while the GPU works.
  std::vector<int> spans;
  const size_t tw = (size_t)pl.tc.tw, th = (size_t)pl.tc.th;
  // the output that is the target: segments of rows, copied on the host by
  // worker threads while the device works (joined before the call returns,
  // on every path: the joiner is destroyed before the segments)
  struct HostRows { float *out; const float *tgt; size_t off, n; };
  std::vector<HostRows> host_rows;
  struct Joiner {
    std::vector<std::thread> pool;
    ~Joiner() {
      for (auto &t : pool) t.join();
    }
  } fill_job;
  if (!devptr) {
    int *bands = reinterpret_cast<int *>(base + L.bands);
    ce = launch_tile_count(P, pl.tc, st);
    size_t nb = 0;
    for (uint32_t i = 0; i < n && ce == cudaSuccess; ++i) {
      if (ps[i].channels == 0) continue;
      ce = launch_band_flags(P, sys0[i], bands + 2 * nb, st);
      nb += (size_t)pl.sys[sys0[i]].nty;
    }
    spans.assign(2 * nb, -1);
    if (ce == cudaSuccess && nb)
      ce = cudaMemcpyAsync(spans.data(), bands, 2 * nb * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "band spans");
    d2h += 2 * nb * sizeof(int);
    size_t boff = 0;
    for (uint32_t i = 0; i < n && ce == cudaSuccess; ++i) {
      const pt_problem &p = ps[i];
      if (p.channels == 0) continue;
      const SysDesc &d0 = pl.sys[sys0[i]];
      const size_t C = p.channels, W = p.width, H = p.height, pitch = W * C * sizeof(float);
      const int *f = spans.data() + 2 * boff;
      for (int ty = 0; ty < d0.nty && ce == cudaSuccess; ++ty) {
        if (f[2 * ty] < 0) continue;
        const size_t r0 = ty * th > 0 ? ty * th - 1 : 0, r1 = std::min(H, (ty + 1) * th + 1);
        const size_t x0 = f[2 * ty] * tw > 0 ? f[2 * ty] * tw - 1 : 0, x1 = std::min(W, (f[2 * ty + 1] + 1) * tw + 1);
        const size_t off = r0 * W * C + x0 * C, wb = (x1 - x0) * C * sizeof(float), rows = r1 - r0;
        ce = cudaMemcpy2DAsync(const_cast<float *>(d0.src) + off, pitch, p.source_or_guidance + off, pitch, wb, rows,
                               cudaMemcpyHostToDevice, st);
        if (ce == cudaSuccess)
          ce = cudaMemcpy2DAsync(const_cast<float *>(d0.tgt) + off, pitch, p.target_or_anchor + off, pitch, wb, rows,
                                 cudaMemcpyHostToDevice, st);
        if (ce == cudaSuccess && (p.flags & PT_FLAG_WARM_START))
          ce = cudaMemcpy2DAsync(const_cast<float *>(d0.guess) + off, pitch, p.initial_guess + off, pitch, wb, rows,
                                 cudaMemcpyHostToDevice, st);
        h2d += wb * rows * ((p.flags & PT_FLAG_WARM_START) ? 3 : 2);
      }
      boff += (size_t)d0.nty;
    }
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "input upload");

    // The output outside the bands' spans is the target bit for bit: whole
    // rows of bands without interior tiles, the row segments beside each
    // span. It does not depend on the solve, so it is copied now, beside the
    // device work, on worker threads: one host thread copies about 10 GB/s,
    // a fifth of PCIe, so a large fill is split over up to eight threads,
    // each taking one contiguous stretch of the concatenated segments; a fill
    // below 256 KB is done here.
    boff = 0;
    for (uint32_t i = 0; i < n; ++i) {
      if (ps[i].channels == 0) continue;
      const SysDesc &d0 = pl.sys[sys0[i]];
      const size_t C = ps[i].channels, W = ps[i].width, H = ps[i].height, row = W * C;
      const int *f = spans.data() + 2 * boff;
      for (int ty = 0; ty < d0.nty;) {
        const size_t r0 = ty * th;
        if (f[2 * ty] < 0) {  // a run of bands without interior tiles: whole rows
          int ty1 = ty + 1;
          while (ty1 < d0.nty && f[2 * ty1] < 0) ++ty1;
          const size_t r1 = std::min(H, ty1 * th);
          host_rows.push_back(HostRows{outs[i], ps[i].target_or_anchor, r0 * row, (r1 - r0) * row});
          ty = ty1;
          continue;
        }
        const size_t r1 = std::min(H, (ty + 1) * th);
        const size_t x0 = f[2 * ty] * tw, x1 = std::min(W, (f[2 * ty + 1] + 1) * tw);
        for (size_t y = r0; y < r1; ++y) {
          if (x0 > 0) host_rows.push_back(HostRows{outs[i], ps[i].target_or_anchor, y * row, x0 * C});
          if (x1 < W) host_rows.push_back(HostRows{outs[i], ps[i].target_or_anchor, y * row + x1 * C, (W - x1) * C});
        }
        ++ty;
      }
      boff += (size_t)d0.nty;
    }
    size_t total = 0;
    for (const HostRows &r : host_rows) total += r.n;
    const HostRows *segs = host_rows.data();
    const size_t nsegs = host_rows.size();
    auto fill = [segs, nsegs](size_t b0, size_t b1) {  // element range of the concatenation
      size_t at = 0;
      for (size_t k = 0; k < nsegs; ++k) {
        const HostRows &r = segs[k];
        const size_t lo = std::max(b0, at), hi = std::min(b1, at + r.n);
        if (lo < hi) std::memcpy(r.out + r.off + (lo - at), r.tgt + r.off + (lo - at), (hi - lo) * sizeof(float));
        at += r.n;
      }
    };
    const size_t bytes = total * sizeof(float);
    if (bytes < (256u << 10)) {
      fill(0, total);
    } else {
      const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
      const unsigned nt = (unsigned)std::min<size_t>(std::min(8u, hw), std::max<size_t>(1, bytes >> 22));
      // a stretch whose thread cannot be started is copied here instead
      for (unsigned k = 0; k < nt; ++k) {
        try {
          fill_job.pool.emplace_back(fill, total * k / nt, total * (k + 1) / nt);
        } catch (const std::system_error &) {
          fill(total * k / nt, total * (k + 1) / nt);
        }
      }
    }
  }

  int grid = 0;
  ce = prepare_solve(P, pl.cfg, ctx->sms, &grid);
  if (ce != cudaSuccess) return cuda_fail(ctx, ce, "solve prepare");
  ctx->last_grid = grid;
  ctx->last_cfg = pl.cfg;
  long long launches = 5;  // tile count, compaction, assembly, init, solve
  for (uint32_t i = 0; i < n; ++i) launches += ps[i].channels > 0 ? (devptr ? 1 : 2) : 0;  // emits, band flags
  if (!devptr) launches += 1;  // the first tile count

  // Everything from here to the results is stream work on the device: with
  // device pointers it is captured once into a CUDA graph and replayed while
  // the plan (descriptors, pointers, arena, configuration) stays the same.
  auto record = [&](cudaEvent_t ev, bool capturing) {
    // inside a capture an external record node still times the launch; the
    // flag is only valid while capturing
    return capturing ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal) : cudaEventRecord(ev, st);
  };
  bool any_warm = false;
  for (uint32_t i = 0; i < n; ++i) any_warm |= (ps[i].flags & PT_FLAG_WARM_START) != 0;
  auto enqueue = [&](bool capturing) -> cudaError_t {
    cudaError_t e = cudaMemsetAsync(base + L.bar, 0, kBarWords * sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + L.err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = launch_assembly(P, pl.tc, st, any_warm);
    if (e == cudaSuccess) e = record(ctx->ev[1], capturing);
    if (e == cudaSuccess) e = launch_prepared(P, pl.cfg, grid, st);
    if (e == cudaSuccess) e = record(ctx->ev[2], capturing);
    for (uint32_t i = 0; i < n && e == cudaSuccess; ++i)
      if (ps[i].channels > 0)
        e = launch_emit(P, sys0[i], pl.tc, (long long)ps[i].width * ps[i].height, st);
    if (devptr && histories)
      for (uint32_t i = 0; i < n && e == cudaSuccess; ++i) {
        if (!histories[i] || !ps[i].max_iterations) continue;
        for (uint32_t c = 0; c < ps[i].channels && e == cudaSuccess; ++c)
          e = cudaMemcpyAsync(histories[i] + (size_t)c * ps[i].max_iterations,
                              reinterpret_cast<double *>(base + L.hist) + pl.sys[sys0[i] + c].hist_off,
                              ps[i].max_iterations * sizeof(double), cudaMemcpyDeviceToDevice, st);
      }
    return e;
  };
  if (devptr && ctx->graphs) {
    std::string key(reinterpret_cast<const char *>(pl.sys.data()), pl.sys.size() * sizeof(SysDesc));
    const long long extra[6] = {pl.cfg, grid, (long long)(uintptr_t)base, (long long)L.total,
                                (long long)pl.tiles.size(), (long long)(histories != nullptr)};
    key.append(reinterpret_cast<const char *>(extra), sizeof(extra));
    if (histories)
      for (uint32_t i = 0; i < n; ++i) key.append(reinterpret_cast<const char *>(&histories[i]), sizeof(void *));
    if (!ctx->gexec || key != ctx->gkey) {
      if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
      cudaGraph_t g = nullptr;
      ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
      if (ce == cudaSuccess) {
        const cudaError_t e1 = enqueue(true);
        ce = cudaStreamEndCapture(st, &g);
        if (e1 != cudaSuccess) ce = e1;
      }
      if (ce == cudaSuccess) ce = cudaGraphInstantiate(&ctx->gexec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (ce != cudaSuccess) { ctx->gexec = nullptr; return cuda_fail(ctx, ce, "graph capture"); }
      ctx->gkey = key;
    }
    ce = cudaGraphLaunch(ctx->gexec, st);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "graph launch");
  } else {
    ce = enqueue(false);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "launch");
  }

  // ---- download
  std::vector<SysState> states(nsys);
  int kerr = 0;
  d2h += nsys * sizeof(SysState) + sizeof(int);
  ce = cudaMemcpyAsync(states.data(), base + L.st, nsys * sizeof(SysState), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(&kerr, base + L.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  // host buffers: each band's span of interior tiles comes down after the
  // emit (the rest of the output is being filled on the host)
  if (!devptr && ce == cudaSuccess) {
    size_t boff = 0;
    for (uint32_t i = 0; i < n && ce == cudaSuccess; ++i) {
      if (ps[i].channels == 0) continue;
      const SysDesc &d0 = pl.sys[sys0[i]];
      const size_t C = ps[i].channels, W = ps[i].width, H = ps[i].height, row = W * C;
      const int *f = spans.data() + 2 * boff;
      for (int ty = 0; ty < d0.nty && ce == cudaSuccess; ++ty) {
        if (f[2 * ty] < 0) continue;
        const size_t r0 = ty * th, r1 = std::min(H, (ty + 1) * th);
        const size_t x0 = f[2 * ty] * tw, x1 = std::min(W, (f[2 * ty + 1] + 1) * tw);
        const size_t off = r0 * row + x0 * C, wb = (x1 - x0) * C * sizeof(float);
        ce = cudaMemcpy2DAsync(outs[i] + off, row * sizeof(float), d0.out + off, row * sizeof(float), wb, r1 - r0,
                               cudaMemcpyDeviceToHost, st);
        d2h += wb * (r1 - r0);
      }
      boff += (size_t)d0.nty;
    }
  }
  if (histories && !devptr && ce == cudaSuccess) {
    for (uint32_t i = 0; i < n && ce == cudaSuccess; ++i) {
      if (!histories[i]) continue;
      for (uint32_t c = 0; c < ps[i].channels && ce == cudaSuccess; ++c) {
        const SysDesc &d = pl.sys[sys0[i] + c];
        const size_t cnt = ps[i].max_iterations;
        if (!cnt) continue;
        d2h += cnt * sizeof(double);
        ce = cudaMemcpyAsync(histories[i] + (size_t)c * cnt,
                             reinterpret_cast<double *>(base + L.hist) + d.hist_off, cnt * sizeof(double),
                             cudaMemcpyDeviceToHost, st);
      }
    }
  }
  if (ce != cudaSuccess) return cuda_fail(ctx, ce, "result download");
  cudaEventRecord(ctx->ev[3], st);
  ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) return cuda_fail(ctx, ce, "stream synchronize");
  {
    float a = 0.f, b = 0.f;
    if (cudaEventElapsedTime(&a, ctx->ev[1], ctx->ev[2]) != cudaSuccess) a = -1.f;
    if (cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[3]) != cudaSuccess) b = -1.f;
    cudaGetLastError();  // a failed timing query must not leak into later error checks
    ctx->last_solve_ms = a;
    ctx->last_call_ms = b;
    ctx->last_launches = launches;
    ctx->last_h2d = h2d;
    ctx->last_d2h = d2h;
  }
  if (kerr != KERR_NONE)
    return fail(ctx, PT_TIMEOUT, kerr == KERR_DEADLINE ? "solve exceeded its wall budget"
                                                       : "wait for work gave up (no progress)");

  // ---- reports
  for (uint32_t i = 0; i < n; ++i) {
    const pt_problem &p = ps[i];
    int worst = -1;
    for (uint32_t c = 0; c < p.channels; ++c) {
      const SysState &s = states[sys0[i] + c];
      pt_report r{};
      r.iterations = (uint32_t)s.iterations;
      r.stop_reason = s.status;
      r.converged = s.status == PT_STOP_CONVERGED;
      r.tolerance = p.tolerance;
      r.final_residual = s.last;
      r.history_len = r.iterations;
      r.omega_used = s.omega;
      r.refinements = (uint32_t)s.refinements;
      r.channel = (int)c;
      r.initial_residual = s.r0;
      r.warm_start = s.warm_used;
      reports[i][c] = r;
      // worse_of (poisson_blend.rs:240-246)
      if (worst < 0) worst = (int)c;
      else {
        const pt_report &a = reports[i][worst];
        const bool b_worse = (r.iterations != a.iterations) ? (r.iterations > a.iterations)
                                                             : (r.final_residual > a.final_residual);
        if (b_worse) worst = (int)c;
      }
    }
    if (worst >= 0) {
      reports[i][p.channels] = reports[i][worst];
    } else {
      pt_report r{};
      r.converged = 1; r.stop_reason = PT_STOP_CONVERGED; r.tolerance = p.tolerance; r.channel = -1;
      reports[i][0] = r;
    }
  }
  return PT_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

pt_status pt_ctx_create(int device, pt_ctx **out) {
  if (!out) return PT_INVALID_ARG;
  *out = nullptr;
  if (injected_fault() == 1) return PT_NO_DEVICE;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= 0) return PT_NO_DEVICE;
  if (device < 0 || device >= count) return PT_INVALID_ARG;
  cudaDeviceProp prop{};
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return PT_NO_DEVICE;
  if (prop.major != 10) return PT_NO_DEVICE;  // built for sm_100a only
  if (!prop.cooperativeLaunch) return PT_NO_DEVICE;
  pt_ctx *c = new (std::nothrow) pt_ctx();
  if (!c) return PT_OOM;
  c->device = device;
  c->sms = prop.multiProcessorCount;
  if (const char *g = std::getenv("PAINTOP_CUDA_GRAPHS")) c->graphs = std::strcmp(g, "0") != 0;
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return PT_LAUNCH_FAILED;
  }
  *out = c;
  return PT_OK;
}

pt_status pt_ctx_destroy(pt_ctx *ctx) {
  return abi_guard(ctx, [&]() -> pt_status {
    if (!ctx) return PT_OK;
    {
      std::lock_guard<std::mutex> lock(ctx->mu);
      cudaSetDevice(ctx->device);
      if (ctx->stream) cudaStreamSynchronize(ctx->stream);
      ctx->release();
      if (ctx->stream) cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return PT_OK;
  });
}

pt_status pt_poisson_solve(pt_ctx *ctx, const pt_problem *p, float *out_candidate, pt_report *reports,
                           double *history) {
  return abi_guard(ctx, [&]() -> pt_status {
    if (!ctx || !p || !reports) return PT_INVALID_ARG;
    float *outs[1] = {out_candidate};
    pt_report *reps[1] = {reports};
    double *hists[1] = {history};
    return ptk_solve_batch(ctx, p, 1, outs, reps, hists, -1);
  });
}

pt_status pt_poisson_solve_batch(pt_ctx *ctx, const pt_problem *ps, uint32_t n, float *const *outs,
                                 pt_report *const *reports, double *const *histories) {
  return abi_guard(ctx, [&]() -> pt_status {
    return ptk_solve_batch(ctx, ps, n, outs, reports, histories, -1);
  });
}

const char *pt_status_str(pt_status s) {
  switch (s) {
    case PT_OK: return "ok";
    case PT_NO_DEVICE: return "E_CUDA_UNAVAILABLE: no usable sm_100 CUDA device";
    case PT_INVALID_ARG: return "invalid argument";
    case PT_LAUNCH_FAILED: return "CUDA launch or copy failed";
    case PT_TIMEOUT: return "device watchdog expired";
    case PT_OOM: return "out of memory";
    case PT_INTERNAL: return "internal error";
  }
  return "unknown status";
}

const char *pt_ctx_last_error(const pt_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

void *pt_ctx_stream(const pt_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

pt_status pt_ctx_last_timing(const pt_ctx *ctx, double *solve_kernel_ms, double *call_ms,
                             int64_t *kernel_launches) {
  if (!ctx) return PT_INVALID_ARG;
  if (solve_kernel_ms) *solve_kernel_ms = ctx->last_solve_ms;
  if (call_ms) *call_ms = ctx->last_call_ms;
  if (kernel_launches) *kernel_launches = ctx->last_launches;
  return PT_OK;
}

pt_status pt_ctx_last_transfer(const pt_ctx *ctx, uint64_t *h2d_bytes, uint64_t *d2h_bytes) {
  if (!ctx) return PT_INVALID_ARG;
  if (h2d_bytes) *h2d_bytes = ctx->last_h2d;
  if (d2h_bytes) *d2h_bytes = ctx->last_d2h;
  return PT_OK;
}

pt_status pt_ctx_set_budget(pt_ctx *ctx, double seconds) {
  return abi_guard(ctx, [&]() -> pt_status {
    if (!ctx || !(seconds > 0.0) || !std::isfinite(seconds)) return PT_INVALID_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->budget_s = seconds;
    return PT_OK;
  });
}

}  // extern "C"
