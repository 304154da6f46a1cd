// mg_solver.cu -- multigrid-preconditioned conjugate gradients for the same
// discrete system the red-black SOR path solves, behind PT_FLAG_MULTIGRID.
//
// The system and its stopping bar are the reference's (crates/paintop-cpu/src/
// poisson.rs): interior cells are mask > 0.5 off the image border (:340-355),
// b is the guidance Laplacian fma(4, -c, L + R + U + D) (:364-373), non-interior
// cells hold the anchor, the residual is
//   r = fma(lambda + 4, -u, nsum) - fma(lambda, -anchor, b)        (:315-321)
// and a channel has converged when ||r|| <= tolerance * ||r(anchor)||, ||.||
// taken in FP64. What differs is the iteration: instead of thousands of
// sweeps, each outer step solves the correction equation A e = r
// (A = (4 + lambda) I - adjacency over interior cells) with conjugate
// gradients in FP32, preconditioned by one symmetric multigrid V-cycle, and
// adds e to the FP64 solution; the FP64 residual decides when to stop.
//
// Multigrid (cell-centred): level k halves level k-1 (ceil), a coarse cell is
// active when at least 3 of its 2 x 2 children are; the level-k operator is
// (4 e - sum of active neighbours) / 4^k + lambda e with zero outside the
// active cells; prolongation is bilinear (weights 3/4, 1/4 per axis) into
// active fine cells and restriction its transpose / 4; smoothing is red-black
// SOR (kSmoothOmega; plain Gauss-Seidel on the coarsest level), red then black
// before the coarse correction and black then red after it, so the V-cycle is
// a symmetric operator and a valid CG preconditioner. The channels of an image
// share its level masks. Every reduction is a fixed-order tree, so a rerun is
// byte-identical.
//
// Batches: every problem of a call (pt_poisson_solve_batch) keeps its own
// level hierarchy, its own CG scalars per channel and its own stopping, but
// all of them share each launch. A launch walks a table of blocks, each block
// one 32 x 8 tile of one instance's plane. The level-0 tiles, whose partial
// sums are reduced, are laid out per instance exactly as a call with that
// instance alone lays them out; every other kernel computes each cell from
// values no other block of the launch writes, so its result does not depend
// on the tiling. An instance's results are therefore bit for bit what it gets
// when solved alone. An (instance, channel) pair whose run has stopped skips
// the vector kernels and, in a call with several instances, the V-cycle.
//
// Report (pt_report): iterations = preconditioned CG iterations (each one
// V-cycle and one operator application); history[k] = relative residual after
// iteration k -- the CG recurrence's estimate scaled by the outer step's FP64
// residual, replaced by the exact FP64 value at the end of every outer step;
// refinements = outer steps after the first; omega_used = the smoother's
// relaxation factor. Stop reasons: converged at the FP64 bar; max-iterations
// when the CG iterations reach max_iterations; stalled when an outer step fails to
// lower the FP64 residual, or at once (0 iterations, interior set to NaN)
// when a NaN or infinity in the inputs makes the residual non-finite.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/paintop_cuda.h"
#include "ctx.h"

namespace {

constexpr int kThreads = 256;
constexpr double kInnerFloor = 2e-6;  // deepest relative reduction asked of one FP32 CG run

__device__ __forceinline__ double block_sum(double v, double *sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// Stencil and vector kernels run on tiles of (32, 8) threads over columns and
// rows; a tile strides over the rows of its instance's plane, grid.z is the
// channel. Kernels that reduce write one partial per tile and channel.
constexpr int kTx = 32, kTy = 8;

// One instance's plane as one launch tiles it. The blocks of a launch are the
// instances' tiles one after another; bmap[blockIdx.x] names the entry.
struct Geo {
  int W, H;           // the tiled plane (restriction: the coarse one)
  int gx, gy;         // tiles: gx across W (a half-sweep: across (W + 1) / 2), gy striding the rows
  int blk0;           // the instance's first block in the launch
  int C;              // its channels
  int unit0;          // its first (instance, channel) unit: CG scalars, scales, run flags, reductions
  int pad;
  long long part0;    // its first partial sum (level-0 reductions): C * gx * gy of them, channel-major
  long long o, oc;    // the plane's first cell in its level's one-channel (interior flags) and C-channel arrays
  long long o2, oc2;  // the same for the other plane of a two-level kernel
  int W2, H2;         // that plane (restriction: the fine level; prolongation: the coarse level)
  float s, d;         // the level's 4^-k and diagonal 4^(1-k) + lambda (restriction: the fine level's)
  double lambda;
};

// The block's entry, the entry's first unit and its channels: from the block
// table, or -- a launch over one instance, bmap null -- from the kernel's own
// parameter `one`, with no load before the block's first data.
__device__ __forceinline__ int4 entry_of(const int4 *__restrict__ bmap, const Geo &one) {
  return bmap ? bmap[blockIdx.x] : make_int4(0, one.unit0, one.C, 0);
}

// Which tile of its instance a block works on
__device__ __forceinline__ int tile_b(const Geo &g) { return (int)blockIdx.x - g.blk0; }

__device__ __forceinline__ double block_sum2(double v, double *sh) {
  const int t = threadIdx.y * kTx + threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int o = kTx * kTy / 2; o > 0; o >>= 1) {
    if (t < o) sh[t] += sh[t + o];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// Per-unit CG scalars: sc[unit] = {rho, rho_new, pq, rr, alpha, beta}
enum { S_RHO, S_RHO_NEW, S_PQ, S_RR, S_ALPHA, S_BETA, S_N };

// The caller-side buffers of one instance (device memory: the caller's, or
// the staged copies of host buffers)
struct Io {
  const float *guid, *anchor, *mask, *guess;
  float *out;
};

// ---- assembly ----------------------------------------------------------------
// interior flag, u = anchor (or the warm guess at interior cells), b' =
// fma(lambda, -anchor, laplacian(guidance)) at interior cells; level-0 tiles,
// grid.z 1 (each thread does all channels of its cells).
__global__ void __launch_bounds__(kTx * kTy) k_mg_assemble(const Geo *__restrict__ geo,
                                                           const int4 *__restrict__ bmap, const Geo one,
                                                           const Io *__restrict__ io, uint8_t *__restrict__ act,
                                                           double *__restrict__ u, double *__restrict__ bl,
                                                           double *__restrict__ uw) {
  const int4 bt = entry_of(bmap, one);
  const int gi = bt.x;
  const Geo g = bmap ? geo[gi] : one;
  const Io f = io[gi];
  const int C = g.C, W = g.W, H = g.H, b = tile_b(g), i = (b % g.gx) * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  uint8_t *a = act + g.o;
  double *u0 = u + g.oc, *b0 = bl + g.oc, *w0 = uw ? uw + g.oc : nullptr;
  for (int j = (b / g.gx) * kTy + threadIdx.y; j < H && i < W; j += g.gy * kTy) {
    const size_t q = (size_t)j * W + i;
    const bool in = W >= 3 && H >= 3 && i > 0 && j > 0 && i < W - 1 && j < H - 1 && f.mask[q] > 0.5f;
    a[q] = in ? 1 : 0;
    for (int c = 0; c < C; ++c) {  // a thread's channels are adjacent in the interleaved inputs
      const double av = (double)f.anchor[q * C + c];
      u0[c * N + q] = av;
      double bv = 0.0;
      if (in) {
        // poisson.rs:364-373: L, R, U, D, then fma(4, -centre, sum)
        const float *gd = f.guid;
        const double ctr = (double)gd[q * C + c];
        const double s = (double)gd[(q - 1) * C + c] + (double)gd[(q + 1) * C + c] + (double)gd[(q - W) * C + c] +
                         (double)gd[(q + W) * C + c];
        bv = fma(4.0, -ctr, s);
      }
      b0[c * N + q] = in ? fma(g.lambda, -av, bv) : 0.0;
      if (w0) w0[c * N + q] = (in && f.guess) ? (double)f.guess[q * C + c] : av;
    }
  }
}

// r = fma(lambda + 4, -u, nsum) - b' at interior cells (0 elsewhere) and
// per-tile partial sums of r^2.
__global__ void __launch_bounds__(kTx * kTy) k_mg_residual64(const Geo *__restrict__ geo,
                                                             const int4 *__restrict__ bmap, const Geo one,
                                                             const uint8_t *__restrict__ act,
                                                             const double *__restrict__ u,
                                                             const double *__restrict__ bl, double *__restrict__ r64,
                                                             double *__restrict__ part) {
  __shared__ double sh[kTx * kTy];
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z) return;
  const int W = g.W, H = g.H, gx = g.gx, gy = g.gy, b = tile_b(g), i = (b % gx) * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const uint8_t *a = act + g.o;
  const double *uc = u + g.oc + c * N, *bc = bl + g.oc + c * N;
  double *rc = r64 + g.oc + c * N;
  const double lambda = g.lambda;
  double acc = 0.0;
  for (int j = (b / gx) * kTy + threadIdx.y; j < H && i < W; j += gy * kTy) {
    const size_t q = (size_t)j * W + i;
    double r = 0.0;
    if (a[q]) {
      const double nsum = uc[q - 1] + uc[q + 1] + uc[q - W] + uc[q + W];  // L, R, U, D (poisson.rs:275-298)
      r = fma(lambda + 4.0, -uc[q], nsum) - bc[q];
    }
    rc[q] = r;
    acc += r * r;
  }
  const double t = block_sum2(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[g.part0 + (long long)c * gx * gy + b] = t;
}

// A unit's partial sums: part[start .. start + n - 1]
struct Red {
  long long start, n;
};

// out[unit * stride] = fixed-order sum of the unit's partials; grid (units)
__global__ void k_mg_reduce(const double *__restrict__ part, const Red *__restrict__ rtab, double *__restrict__ out,
                            int stride) {
  __shared__ double sh[kThreads];
  const Red rt = rtab[blockIdx.x];
  double acc = 0.0;
  for (long long k = threadIdx.x; k < rt.n; k += blockDim.x) acc += part[rt.start + k];
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) out[(long long)blockIdx.x * stride] = s;
}

// r32 = r64 / scale[unit] (0 where the unit is not being corrected)
__global__ void __launch_bounds__(kTx * kTy) k_mg_scale(const Geo *__restrict__ geo,
                                                        const int4 *__restrict__ bmap, const Geo one,
                                                        const double *__restrict__ r64,
                                                        const double *__restrict__ scale, float *__restrict__ r32) {
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z) return;
  const int W = g.W, H = g.H, b = tile_b(g), i = (b % g.gx) * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const double s = scale[g.unit0 + c];
  const double *rc = r64 + g.oc + c * N;
  float *oc = r32 + g.oc + c * N;
  for (int j = (b / g.gx) * kTy + threadIdx.y; j < H && i < W; j += g.gy * kTy) {
    const size_t q = (size_t)j * W + i;
    oc[q] = s > 0.0 ? (float)(rc[q] / s) : 0.0f;
  }
}

// u += scale[unit] * x at interior cells; a unit with scale 0 (not being
// corrected) is left as it is, bit for bit
__global__ void __launch_bounds__(kTx * kTy) k_mg_update(const Geo *__restrict__ geo,
                                                         const int4 *__restrict__ bmap, const Geo one,
                                                         const uint8_t *__restrict__ act, const float *__restrict__ x,
                                                         const double *__restrict__ scale, double *__restrict__ u) {
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z) return;
  const double s = scale[g.unit0 + c];
  if (s == 0.0) return;
  const int W = g.W, H = g.H, b = tile_b(g), i = (b % g.gx) * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const uint8_t *a = act + g.o;
  const float *xc = x + g.oc + c * N;
  double *uc = u + g.oc + c * N;
  for (int j = (b / g.gx) * kTy + threadIdx.y; j < H && i < W; j += g.gy * kTy) {
    const size_t q = (size_t)j * W + i;
    if (a[q]) uc[q] = fma(s, (double)xc[q], uc[q]);
  }
}

// ---- multigrid -----------------------------------------------------------------
// A coarse cell is active when at least kCoarseRule of its 2 x 2 children
// are. A cell made mostly of boundary would carry a correction the fine grid
// cannot use; on a CPU model of this preconditioner, requiring 3 children took
// the CG iterations to 1e-6 from 14 to 7 on eight polygons, 10 to 7 on an
// ellipse and 50 to 9 on a mask with 30% of its pixels missing at random.
constexpr int kCoarseRule = 3;

// Relaxation of the smoother's half-sweeps (symmetric SOR: the post-smoothing
// sweeps run the colours in reverse, so the V-cycle stays symmetric). The CPU
// model gave 6 CG iterations for 1.2-1.4 where plain Gauss-Seidel took 7 on
// the same four masks; the coarsest level keeps plain Gauss-Seidel.
constexpr float kSmoothOmega = 1.25f;

// Coarse interior flags from the fine ones; tiles of the coarse plane (the
// fine plane is the entry's second).
__global__ void __launch_bounds__(kTx * kTy) k_mg_coarsen(const Geo *__restrict__ geo,
                                                          const int4 *__restrict__ bmap, const Geo one,
                                                          const uint8_t *__restrict__ af, uint8_t *__restrict__ ac) {
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int Wc = g.W, Hc = g.H, Wf = g.W2, Hf = g.H2, b = tile_b(g), I = (b % g.gx) * kTx + threadIdx.x;
  const uint8_t *f = af + g.o2;
  uint8_t *cc = ac + g.o;
  for (int J = (b / g.gx) * kTy + threadIdx.y; J < Hc && I < Wc; J += g.gy * kTy) {
    int n = 0;
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        const int i = 2 * I + dx, j = 2 * J + dy;
        if (i < Wf && j < Hf) n += f[(size_t)j * Wf + i];
      }
    cc[(size_t)J * Wc + I] = n >= kCoarseRule ? 1 : 0;
  }
}

// V-cycle kernels return at once for a unit whose run flag is 0 (run null:
// no unit is skipped).
//
// One colour of red-black Gauss-Seidel on A_k e = rhs: e = (rhs + s * sum of
// neighbours) / d at active cells of that colour (inactive cells hold 0).
// x threads index the cells of one colour in a row (half-sweep tiles).
__global__ void __launch_bounds__(kTx * kTy) k_mg_smooth(const Geo *__restrict__ geo,
                                                         const int4 *__restrict__ bmap, const Geo one,
                                                         const uint8_t *__restrict__ act,
                                                         const float *__restrict__ rhs, float *__restrict__ e,
                                                         const double *__restrict__ run, int color) {
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z || (run && run[bt.y + c] == 0.0)) return;
  const int W = g.W, H = g.H, b = tile_b(g), m = (b % g.gx) * kTx + threadIdx.x;
  const float s = g.s, d = g.d;
  const size_t N = (size_t)W * H;
  const uint8_t *a = act + g.o;
  float *ec = e + g.oc + c * N;
  const float *rc = rhs + g.oc + c * N;
  // Two of the tile's rows per pass, both rows' loads before either update:
  // the neighbours read are of the other colour, which this half-sweep does
  // not write, so the two rows' accesses are independent and the loads of the
  // second row need not wait for the first row's store.
  const int step = g.gy * kTy;
  for (int j0 = (b / g.gx) * kTy + threadIdx.y; j0 < H; j0 += 2 * step) {
    const int j1 = j0 + step;
    const int i0 = 2 * m + ((j0 + color) & 1), i1 = 2 * m + ((j1 + color) & 1);
    const size_t q0 = (size_t)j0 * W + i0, q1 = (size_t)j1 * W + i1;
    const bool v0 = i0 < W && a[q0];
    const bool v1 = j1 < H && i1 < W && a[q1];
    float nb0 = 0.0f, e0 = 0.0f, r0 = 0.0f, nb1 = 0.0f, e1 = 0.0f, r1 = 0.0f;
    if (v0) {
      if (i0 > 0) nb0 += ec[q0 - 1];
      if (i0 < W - 1) nb0 += ec[q0 + 1];
      if (j0 > 0) nb0 += ec[q0 - W];
      if (j0 < H - 1) nb0 += ec[q0 + W];
      e0 = ec[q0];
      r0 = rc[q0];
    }
    if (v1) {
      if (i1 > 0) nb1 += ec[q1 - 1];
      if (i1 < W - 1) nb1 += ec[q1 + 1];
      if (j1 > 0) nb1 += ec[q1 - W];
      if (j1 < H - 1) nb1 += ec[q1 + W];
      e1 = ec[q1];
      r1 = rc[q1];
    }
    if (v0) {
      const float gs = (r0 + s * nb0) / d;
      ec[q0] = e0 + kSmoothOmega * (gs - e0);
    }
    if (v1) {
      const float gs = (r1 + s * nb1) / d;
      ec[q1] = e1 + kSmoothOmega * (gs - e1);
    }
  }
}

// The first half-sweep of a V-cycle level, from e = 0: e = rhs / d at active
// cells of colour 0 (red), 0 everywhere else, relaxed by kSmoothOmega -- what
// zeroing e and one red half-sweep produce, bit for bit, in one pass that
// writes every cell.
__global__ void __launch_bounds__(kTx * kTy) k_mg_smooth_first(const Geo *__restrict__ geo,
                                                               const int4 *__restrict__ bmap, const Geo one,
                                                               const uint8_t *__restrict__ act,
                                                               const float *__restrict__ rhs, float *__restrict__ e,
                                                               const double *__restrict__ run) {
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z || (run && run[bt.y + c] == 0.0)) return;
  const int W = g.W, H = g.H, b = tile_b(g), i = (b % g.gx) * kTx + threadIdx.x;
  const float s = g.s, d = g.d;
  const size_t N = (size_t)W * H;
  const uint8_t *a = act + g.o;
  float *ec = e + g.oc + c * N;
  const float *rc = rhs + g.oc + c * N;
  for (int j = (b / g.gx) * kTy + threadIdx.y; j < H && i < W; j += g.gy * kTy) {
    const size_t q = (size_t)j * W + i;
    const float gs = (rc[q] + s * 0.0f) / d;
    ec[q] = (a[q] && ((i + j) & 1) == 0) ? 0.0f + kSmoothOmega * (gs - 0.0f) : 0.0f;
  }
}

// The coarsest level (at most kCoarseMax cells): `sweeps` red-black sweeps,
// then as many in reverse colour order, from e = 0, in shared memory; one
// block per instance (blockIdx.x = its entry) and channel (blockIdx.z).
constexpr int kCoarseMax = 64;

__global__ void k_mg_coarse(const Geo *__restrict__ geo, const uint8_t *__restrict__ act,
                            const float *__restrict__ rhs, float *__restrict__ e, const double *__restrict__ run,
                            int sweeps) {
  __shared__ float se[kCoarseMax], sr[kCoarseMax];
  __shared__ uint8_t sa[kCoarseMax];
  const Geo &g = geo[blockIdx.x];
  const int c = blockIdx.z;
  if (c >= g.C || (run && run[g.unit0 + c] == 0.0)) return;
  const int W = g.W, H = g.H, n = W * H, t = threadIdx.x;
  const float s = g.s, d = g.d;
  const float *rc = rhs + g.oc + (long long)c * n;
  float *ecp = e + g.oc + (long long)c * n;
  if (t < n) {
    se[t] = 0.0f;
    sr[t] = rc[t];
    sa[t] = act[g.o + t];
  }
  __syncthreads();
  const int j = t / max(W, 1), i = t - j * W;
  for (int k = 0; k < 4 * sweeps; ++k) {
    // colour order R, B (first half) then B, R (second half)
    const int half = k / (2 * sweeps), step = k & 1;
    const int color = half == 0 ? step : 1 - step;
    float v = 0.0f;
    const bool mine = t < n && sa[t] && ((i + j) & 1) == color;
    if (mine) {
      float nb = 0.0f;
      if (i > 0) nb += se[t - 1];
      if (i < W - 1) nb += se[t + 1];
      if (j > 0) nb += se[t - W];
      if (j < H - 1) nb += se[t + W];
      v = (sr[t] + s * nb) / d;
    }
    __syncthreads();
    if (mine) se[t] = v;
    __syncthreads();
  }
  if (t < n) ecp[t] = se[t];
}

__device__ __forceinline__ float pw(int a) { return (a == 0 || a == 1) ? 0.75f : 0.25f; }  // a = fine - 2 * coarse

// The restriction of the level's residual, rhs_c(I, J) = sum over fine
// (2I + a, 2J + b), a, b in -1..2, of wx wy res_f / 4 with res_f = rhs - A e at
// active fine cells (0 elsewhere), evaluated on the fly so the residual is
// never stored. Tiles of the coarse plane; the fine plane is the second.
__global__ void __launch_bounds__(kTx * kTy) k_mg_resid_restrict(const Geo *__restrict__ geo,
                                                                 const int4 *__restrict__ bmap, const Geo one,
                                                                 const uint8_t *__restrict__ af,
                                                                 const float *__restrict__ rhsf,
                                                                 const float *__restrict__ ef,
                                                                 const uint8_t *__restrict__ ac,
                                                                 float *__restrict__ rhsc,
                                                                 const double *__restrict__ run) {
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z || (run && run[bt.y + c] == 0.0)) return;
  const int Wc = g.W, Hc = g.H, Wf = g.W2, Hf = g.H2, b = tile_b(g), I = (b % g.gx) * kTx + threadIdx.x;
  const float s = g.s, d = g.d;
  const size_t Nc = (size_t)Wc * Hc, Nf = (size_t)Wf * Hf;
  const float *e = ef + g.oc2 + c * Nf, *rh = rhsf + g.oc2 + c * Nf;
  const uint8_t *fa = af + g.o2, *ca = ac + g.o;
  float *out = rhsc + g.oc + c * Nc;
  for (int J = (b / g.gx) * kTy + threadIdx.y; J < Hc && I < Wc; J += g.gy * kTy) {
    const size_t q = (size_t)J * Wc + I;
    float v = 0.0f;
    if (ca[q]) {
      for (int bb = -1; bb <= 2; ++bb) {
        const int j = 2 * J + bb;
        if (j < 0 || j >= Hf) continue;
        float row = 0.0f;
        for (int aa = -1; aa <= 2; ++aa) {
          const int i = 2 * I + aa;
          if (i < 0 || i >= Wf) continue;
          const size_t f = (size_t)j * Wf + i;
          float r = 0.0f;
          if (fa[f]) {
            float nb = 0.0f;
            if (i > 0) nb += e[f - 1];
            if (i < Wf - 1) nb += e[f + 1];
            if (j > 0) nb += e[f - Wf];
            if (j < Hf - 1) nb += e[f + Wf];
            r = rh[f] - (d * e[f] - s * nb);
          }
          row += pw(aa) * r;
        }
        v += pw(bb) * row;
      }
      v *= 0.25f;
    }
    out[q] = v;
  }
}

// e_f += bilinear prolongation of e_c at active fine cells; tiles of the fine
// plane, the coarse plane is the second.
__global__ void __launch_bounds__(kTx * kTy) k_mg_prolong(const Geo *__restrict__ geo,
                                                          const int4 *__restrict__ bmap, const Geo one,
                                                          const uint8_t *__restrict__ af, float *__restrict__ ef,
                                                          const float *__restrict__ ec,
                                                          const double *__restrict__ run) {
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z || (run && run[bt.y + c] == 0.0)) return;
  const int Wf = g.W, Hf = g.H, Wc = g.W2, Hc = g.H2, b = tile_b(g), i = (b % g.gx) * kTx + threadIdx.x;
  const size_t Nc = (size_t)Wc * Hc, Nf = (size_t)Wf * Hf;
  const float *e = ec + g.oc2 + c * Nc;
  float *out = ef + g.oc + c * Nf;
  const uint8_t *fa = af + g.o;
  for (int j = (b / g.gx) * kTy + threadIdx.y; j < Hf && i < Wf; j += g.gy * kTy) {
    const size_t q = (size_t)j * Wf + i;
    if (!fa[q]) continue;
    const int I0 = i >> 1, J0 = j >> 1;
    const int I1 = (i & 1) ? I0 + 1 : I0 - 1, J1 = (j & 1) ? J0 + 1 : J0 - 1;
    auto at = [&](int I, int J) -> float {
      return (I >= 0 && I < Wc && J >= 0 && J < Hc) ? e[(size_t)J * Wc + I] : 0.0f;
    };
    const float v = 0.5625f * at(I0, J0) + 0.1875f * (at(I1, J0) + at(I0, J1)) + 0.0625f * at(I1, J1);
    out[q] += v;
  }
}

// ---- conjugate gradients (level-0 tiles) ---------------------------------------
__device__ __forceinline__ void zero_partial(const Geo &g, int c, double *part) {
  if (threadIdx.x == 0 && threadIdx.y == 0) part[g.part0 + (long long)c * g.gx * g.gy + tile_b(g)] = 0.0;
}

// q = A_0 p at active cells; partial sums of p.q
__global__ void __launch_bounds__(kTx * kTy) k_cg_apply(const Geo *__restrict__ geo,
                                                        const int4 *__restrict__ bmap, const Geo one,
                                                        const uint8_t *__restrict__ act, const float *__restrict__ p,
                                                        float *__restrict__ q, double *__restrict__ part,
                                                        const double *__restrict__ run) {
  __shared__ double sh[kTx * kTy];
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z) return;
  if (run[bt.y + c] == 0.0) {  // a stopped unit: its p.q is never read
    zero_partial(g, c, part);
    return;
  }
  const int W = g.W, H = g.H, gx = g.gx, gy = g.gy, b = tile_b(g), i = (b % gx) * kTx + threadIdx.x;
  const float d = g.d;
  const size_t N = (size_t)W * H;
  const uint8_t *a = act + g.o;
  const float *pc = p + g.oc + c * N;
  float *qc = q + g.oc + c * N;
  double acc = 0.0;
  // two of the tile's rows per pass, loads before stores (as in k_mg_smooth);
  // the partial sum still takes the rows in order
  const int step = gy * kTy;
  for (int j0 = (b / gx) * kTy + threadIdx.y; j0 < H && i < W; j0 += 2 * step) {
    const bool two = j0 + step < H;
    const size_t k0 = (size_t)j0 * W + i, k1 = k0 + (size_t)step * W;
    const bool a0 = a[k0] != 0, a1 = two && a[k1] != 0;
    // interior cells are never on the border: all four neighbours exist
    float c0 = 0.0f, s0 = 0.0f, c1 = 0.0f, s1 = 0.0f;
    if (a0) {
      c0 = pc[k0];
      s0 = pc[k0 - 1] + pc[k0 + 1] + pc[k0 - W] + pc[k0 + W];
    }
    if (a1) {
      c1 = pc[k1];
      s1 = pc[k1 - 1] + pc[k1 + 1] + pc[k1 - W] + pc[k1 + W];
    }
    float v0 = 0.0f, v1 = 0.0f;
    if (a0) {
      v0 = d * c0 - s0;
      acc += (double)c0 * (double)v0;
    }
    if (a1) {
      v1 = d * c1 - s1;
      acc += (double)c1 * (double)v1;
    }
    qc[k0] = v0;
    if (two) qc[k1] = v1;
  }
  const double t = block_sum2(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[g.part0 + (long long)c * gx * gy + b] = t;
}

// partial sums of a.b
__global__ void __launch_bounds__(kTx * kTy) k_cg_dot(const Geo *__restrict__ geo,
                                                      const int4 *__restrict__ bmap, const Geo one,
                                                      const float *__restrict__ x, const float *__restrict__ y,
                                                      double *__restrict__ part, const double *__restrict__ run) {
  __shared__ double sh[kTx * kTy];
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z) return;
  if (run[bt.y + c] == 0.0) {  // a stopped unit: its rho is never read
    zero_partial(g, c, part);
    return;
  }
  const int W = g.W, H = g.H, gx = g.gx, gy = g.gy, b = tile_b(g), i = (b % gx) * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const float *xc = x + g.oc + c * N, *yc = y + g.oc + c * N;
  double acc = 0.0;
  const int step = gy * kTy;
  for (int j0 = (b / gx) * kTy + threadIdx.y; j0 < H && i < W; j0 += 2 * step) {
    const bool two = j0 + step < H;
    const size_t o0 = (size_t)j0 * W + i, o1 = o0 + (size_t)step * W;
    const float x0 = xc[o0], y0 = yc[o0];
    const float x1 = two ? xc[o1] : 0.0f, y1 = two ? yc[o1] : 0.0f;
    acc += (double)x0 * (double)y0;
    if (two) acc += (double)x1 * (double)y1;
  }
  const double t = block_sum2(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[g.part0 + (long long)c * gx * gy + b] = t;
}

// p = z + beta p (beta = rho_new / rho; p = z on the first iteration)
__global__ void __launch_bounds__(kTx * kTy) k_cg_direction(const Geo *__restrict__ geo,
                                                            const int4 *__restrict__ bmap, const Geo one,
                                                            const float *__restrict__ z, float *__restrict__ p,
                                                            const double *__restrict__ sc,
                                                            const double *__restrict__ run, int first) {
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z || run[bt.y + c] == 0.0) return;
  const double *s = sc + (long long)(g.unit0 + c) * S_N;
  const float beta = first ? 0.0f : (float)(s[S_RHO] != 0.0 ? s[S_RHO_NEW] / s[S_RHO] : 0.0);
  const int W = g.W, H = g.H, b = tile_b(g), i = (b % g.gx) * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const float *zc = z + g.oc + c * N;
  float *pc = p + g.oc + c * N;
  // first: p is not read (it holds what the arena held); two rows per pass,
  // loads before stores
  const int step = g.gy * kTy;
  for (int j0 = (b / g.gx) * kTy + threadIdx.y; j0 < H && i < W; j0 += 2 * step) {
    const bool two = j0 + step < H;
    const size_t o0 = (size_t)j0 * W + i, o1 = o0 + (size_t)step * W;
    const float z0 = zc[o0], z1 = two ? zc[o1] : 0.0f;
    const float p0 = first ? 0.0f : pc[o0], p1 = (first || !two) ? 0.0f : pc[o1];
    pc[o0] = first ? z0 : z0 + beta * p0;
    if (two) pc[o1] = first ? z1 : z1 + beta * p1;
  }
}

__global__ void k_cg_scalars_after_dir(int U, double *__restrict__ sc) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < U; k += gridDim.x * blockDim.x)
    sc[(long long)k * S_N + S_RHO] = sc[(long long)k * S_N + S_RHO_NEW];
}

// x += alpha p, r -= alpha q (alpha = rho / p.q); partial sums of r.r
__global__ void __launch_bounds__(kTx * kTy) k_cg_step(const Geo *__restrict__ geo,
                                                       const int4 *__restrict__ bmap, const Geo one,
                                                       const float *__restrict__ p, const float *__restrict__ q,
                                                       float *__restrict__ x, float *__restrict__ r,
                                                       const double *__restrict__ sc, double *__restrict__ part,
                                                       const double *__restrict__ run) {
  __shared__ double sh[kTx * kTy];
  const int4 bt = entry_of(bmap, one);
  const Geo g = bmap ? geo[bt.x] : one;
  const int c = blockIdx.z;
  if (c >= bt.z) return;
  if (run[bt.y + c] == 0.0) {  // a stopped unit: x and r stay (p may never have been written)
    zero_partial(g, c, part);
    return;
  }
  const double *s = sc + (long long)(g.unit0 + c) * S_N;
  const float alpha = s[S_PQ] > 0.0 ? (float)(s[S_RHO] / s[S_PQ]) : 0.0f;
  const int W = g.W, H = g.H, gx = g.gx, gy = g.gy, b = tile_b(g), i = (b % gx) * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const float *pc = p + g.oc + c * N, *qc = q + g.oc + c * N;
  float *xc = x + g.oc + c * N, *rc = r + g.oc + c * N;
  double acc = 0.0;
  const int step = gy * kTy;  // two rows per pass, loads before stores
  for (int j0 = (b / gx) * kTy + threadIdx.y; j0 < H && i < W; j0 += 2 * step) {
    const bool two = j0 + step < H;
    const size_t o0 = (size_t)j0 * W + i, o1 = o0 + (size_t)step * W;
    const float p0 = pc[o0], q0 = qc[o0], x0 = xc[o0], r0 = rc[o0];
    float p1 = 0.0f, q1 = 0.0f, x1 = 0.0f, r1 = 0.0f;
    if (two) {
      p1 = pc[o1]; q1 = qc[o1]; x1 = xc[o1]; r1 = rc[o1];
    }
    xc[o0] = x0 + alpha * p0;
    const float rv0 = r0 - alpha * q0;
    rc[o0] = rv0;
    acc += (double)rv0 * (double)rv0;
    if (two) {
      xc[o1] = x1 + alpha * p1;
      const float rv1 = r1 - alpha * q1;
      rc[o1] = rv1;
      acc += (double)rv1 * (double)rv1;
    }
  }
  const double t = block_sum2(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[g.part0 + (long long)c * gx * gy + b] = t;
}

// out = interleave(u) at interior cells, the anchor elsewhere (bit for bit);
// level-0 tiles, grid.z 1
__global__ void __launch_bounds__(kTx * kTy) k_mg_emit(const Geo *__restrict__ geo,
                                                       const int4 *__restrict__ bmap, const Geo one,
                                                       const Io *__restrict__ io, const uint8_t *__restrict__ act,
                                                       const double *__restrict__ u) {
  const int4 bt = entry_of(bmap, one);
  const int gi = bt.x;
  const Geo g = bmap ? geo[gi] : one;
  const Io f = io[gi];
  const int C = g.C, W = g.W, H = g.H, b = tile_b(g), i = (b % g.gx) * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const uint8_t *a = act + g.o;
  const double *u0 = u + g.oc;
  for (int j = (b / g.gx) * kTy + threadIdx.y; j < H && i < W; j += g.gy * kTy) {
    const size_t q = (size_t)j * W + i;
    const bool in = a[q] != 0;
    for (int c = 0; c < C; ++c)  // a warp writes 32 whole pixels: C * 32 adjacent floats
      f.out[q * C + c] = in ? (float)u0[c * N + q] : f.anchor[q * C + c];
  }
}

// ---- host ----------------------------------------------------------------------
size_t aup(size_t b) { return (b + 255) & ~(size_t)255; }

// (32, 8)-thread tiles over w columns and h rows of one instance: at most
// about 8 tiles per SM per channel, at least min_bands bands of 8 rows per
// tile where the instance has them (a tile's first loads -- its table entry,
// geometry and run flag -- then serve several bands), at most 65535 rows of
// tiles.
//
// Level-0 launches, whose tiles write the partial sums, take kMinBands: a
// choice that depends on the instance alone, so its partial sums and their
// order are the same in any batch. A V-cycle launch reduces nothing and its
// result does not depend on the tiling; it takes kMinBands only when its
// instances have many tiles (more than kManyWaves waves of 8 per SM at one
// band each), and one band otherwise, so that the small launches of a single
// image's coarse levels keep their parallelism.
constexpr int kMinBands = 4;
constexpr long long kManyWaves = 4;
void tiles2(int w, int h, int sms, int min_bands, int &gx, int &gy) {
  gx = std::max(1, (w + kTx - 1) / kTx);
  const int bands = std::max(1, (h + kTy - 1) / kTy);
  gy = std::min(bands, std::max(1, sms * 8 / gx));
  gy = std::min(gy, (bands + min_bands - 1) / min_bands);
  gy = std::min(gy, 65535);
}
const dim3 kBlock2(kTx, kTy);

float level_s(int k) { return 1.0f / (float)(1u << (2 * std::min(k, 15))); }

// A call is cut into groups of at most this many level-0 tiles (and units);
// every launch of a group then has fewer blocks.
constexpr long long kGroupTiles = 1ll << 22;

// One instance (a problem with channels) of a group
struct Inst {
  int idx;                       // its index in the caller's arrays
  int W, H, C, L;                // extent, channels, levels
  double lambda;
  std::vector<int> w, h;         // level extents
  std::vector<long long> o, oc;  // level offsets in the one-channel and C-channel arrays
  int unit0 = 0;                 // first (instance, channel) unit
  long long part0 = 0;           // first level-0 partial sum
  int gx = 1, gy = 1;            // level-0 tiles
  bool dev = false, warm = false;
  size_t in = 0, mask = 0, guess = 0, out = 0;  // staged copies of host buffers
};

// One kind of launch at one level: its table entries and blocks
struct Launch {
  size_t geo = 0, bmap = 0;  // byte offsets of the tables in the table area
  int n = 0;                 // entries (instances)
  long long blocks = 0;
  Geo one{};                 // the entry of a launch over one instance (passed by value)
};

struct LevelArr {
  size_t act = 0, e = 0, rhs = 0;
};

// Tables built on the host and uploaded in one copy
struct Blob {
  std::vector<unsigned char> b;
  size_t put(const void *p, size_t n) {
    const size_t o = (b.size() + 15) & ~(size_t)15;
    b.resize(o + n);
    if (n) std::memcpy(b.data() + o, p, n);
    return o;
  }
};

Launch make_launch(Blob &blob, std::vector<Geo> &gs) {
  Launch l;
  l.n = (int)gs.size();
  if (gs.size() == 1) {  // one instance: its geometry goes by value, no block map
    gs[0].blk0 = 0;
    l.one = gs[0];
    l.blocks = (long long)gs[0].gx * gs[0].gy;
    l.geo = blob.put(gs.data(), sizeof(Geo));
    return l;
  }
  std::vector<int4> bm;
  long long blk = 0;
  for (size_t k = 0; k < gs.size(); ++k) {
    gs[k].blk0 = (int)blk;
    const long long nb = (long long)gs[k].gx * gs[k].gy;
    bm.insert(bm.end(), (size_t)nb, make_int4((int)k, gs[k].unit0, gs[k].C, 0));
    blk += nb;
  }
  l.blocks = blk;
  l.geo = blob.put(gs.data(), gs.size() * sizeof(Geo));
  l.bmap = blob.put(bm.data(), bm.size() * sizeof(int4));
  return l;
}

struct Mg {
  pt_ctx *ctx;
  cudaStream_t st;
  char *base = nullptr;
  unsigned Cmax = 1;
  int U = 0;
  std::vector<Inst> in;
  std::vector<LevelArr> lv;
  Launch all0;
  std::vector<Launch> full, half, restr, coarse;  // per level
  size_t tab = 0, rtab = 0, io = 0;
  size_t u = 0, bl = 0, uw = 0, r64 = 0, part = 0, red = 0, sc = 0, scale = 0, run = 0, x = 0, r = 0, z = 0, p = 0,
         q = 0;
  long long launches = 0;
  template <class T> T *at(size_t off) { return reinterpret_cast<T *>(base + off); }
  const Geo *geo(const Launch &l) { return at<Geo>(tab + l.geo); }
  const int4 *bmap(const Launch &l) { return l.n == 1 ? nullptr : at<int4>(tab + l.bmap); }
  dim3 grid(const Launch &l, unsigned z) { return dim3((unsigned)l.blocks, 1, z); }
};

void vcycle(Mg &m, float *rhs0, float *e0) {
  const int L = (int)m.lv.size();
  // Units whose run has stopped skip the V-cycle in a batch; a single image's
  // channels do the work regardless (their z is not read) and so spare every
  // block a load before its first data.
  const double *run = m.in.size() > 1 ? m.at<double>(m.run) : nullptr;
  const unsigned Cz = m.Cmax;
  for (int k = 0; k < L; ++k) {
    const LevelArr &v = m.lv[k];
    float *rhs = k == 0 ? rhs0 : m.at<float>(v.rhs), *e = k == 0 ? e0 : m.at<float>(v.e);
    const uint8_t *act = m.at<uint8_t>(v.act);
    const Launch &K = m.coarse[k];
    if (K.n) {  // instances whose coarsest level this is: symmetric sweeps in one block per channel
      k_mg_coarse<<<dim3((unsigned)K.n, 1, Cz), kCoarseMax, 0, m.st>>>(m.geo(K), act, rhs, e, run, 24);
      ++m.launches;
    }
    const Launch &F = m.full[k], &Hh = m.half[k], &R = m.restr[k];
    if (!F.n) continue;
    // red, black, red, black from e = 0 (the first red half-sweep writes all of e)
    k_mg_smooth_first<<<m.grid(F, Cz), kBlock2, 0, m.st>>>(m.geo(F), m.bmap(F), F.one, act, rhs, e, run);
    k_mg_smooth<<<m.grid(Hh, Cz), kBlock2, 0, m.st>>>(m.geo(Hh), m.bmap(Hh), Hh.one, act, rhs, e, run, 1);
    k_mg_smooth<<<m.grid(Hh, Cz), kBlock2, 0, m.st>>>(m.geo(Hh), m.bmap(Hh), Hh.one, act, rhs, e, run, 0);
    k_mg_smooth<<<m.grid(Hh, Cz), kBlock2, 0, m.st>>>(m.geo(Hh), m.bmap(Hh), Hh.one, act, rhs, e, run, 1);
    const LevelArr &cl = m.lv[k + 1];
    k_mg_resid_restrict<<<m.grid(R, Cz), kBlock2, 0, m.st>>>(m.geo(R), m.bmap(R), R.one, act, rhs, e,
                                                              m.at<uint8_t>(cl.act), m.at<float>(cl.rhs), run);
    m.launches += 5;
  }
  for (int k = L - 2; k >= 0; --k) {
    const Launch &F = m.full[k], &Hh = m.half[k];
    if (!F.n) continue;
    const LevelArr &v = m.lv[k], &cl = m.lv[k + 1];
    float *rhs = k == 0 ? rhs0 : m.at<float>(v.rhs), *e = k == 0 ? e0 : m.at<float>(v.e);
    const uint8_t *act = m.at<uint8_t>(v.act);
    k_mg_prolong<<<m.grid(F, Cz), kBlock2, 0, m.st>>>(m.geo(F), m.bmap(F), F.one, act, e, m.at<float>(cl.e), run);
    for (int t = 0; t < 2; ++t) {
      k_mg_smooth<<<m.grid(Hh, Cz), kBlock2, 0, m.st>>>(m.geo(Hh), m.bmap(Hh), Hh.one, act, rhs, e, run, 1);
      k_mg_smooth<<<m.grid(Hh, Cz), kBlock2, 0, m.st>>>(m.geo(Hh), m.bmap(Hh), Hh.one, act, rhs, e, run, 0);
    }
    m.launches += 5;
  }
}

pt_status mfail(pt_ctx *ctx, pt_status s, const std::string &msg) {
  ctx->last_error = msg;
  return s;
}

// One group of instances (ids: indices into ps, all with channels > 0)
pt_status solve_group(pt_ctx *ctx, const pt_problem *ps, const std::vector<int> &ids, float *const *outs,
                      pt_report *const *reports, double *const *histories, double &solve_ms, double &call_ms,
                      long long &launches) {
  const int sms = ctx->sms;
  Mg m;
  m.ctx = ctx;
  m.st = ctx->stream;
  // instances, their levels (halve, ceil, while a level has more than
  // kCoarseMax cells), units and level-0 partial sums
  int Lmax = 0;
  long long P = 0;
  bool any_warm = false;
  for (int id : ids) {
    const pt_problem &p = ps[id];
    Inst I;
    I.idx = id; I.W = (int)p.width; I.H = (int)p.height; I.C = (int)p.channels; I.lambda = p.lambda;
    I.dev = (p.flags & PT_FLAG_DEVICE_POINTERS) != 0;
    I.warm = (p.flags & PT_FLAG_WARM_START) != 0;
    int w = I.W, h = I.H, k = 0;
    for (;;) {
      I.w.push_back(w);
      I.h.push_back(h);
      if ((long long)w * h <= kCoarseMax || k >= 30) break;
      w = (w + 1) / 2; h = (h + 1) / 2; ++k;
    }
    I.L = (int)I.w.size();
    tiles2(I.W, I.H, sms, kMinBands, I.gx, I.gy);
    I.unit0 = m.U;
    m.U += I.C;
    I.part0 = P;
    P += (long long)I.C * I.gx * I.gy;
    Lmax = std::max(Lmax, I.L);
    m.Cmax = std::max(m.Cmax, (unsigned)I.C);
    any_warm |= I.warm;
    m.in.push_back(std::move(I));
  }
  const int U = m.U;
  std::vector<long long> cells(Lmax, 0), ccells(Lmax, 0);
  for (Inst &I : m.in)
    for (int k = 0; k < I.L; ++k) {
      I.o.push_back(cells[k]);
      I.oc.push_back(ccells[k]);
      cells[k] += (long long)I.w[k] * I.h[k];
      ccells[k] += (long long)I.C * I.w[k] * I.h[k];
    }

  // launch tables
  Blob blob;
  auto geo_at = [&](const Inst &I, int k, int tw, int th, int mb) {
    Geo g{};
    g.W = I.w[k]; g.H = I.h[k];
    tiles2(tw, th, sms, mb, g.gx, g.gy);
    g.C = I.C; g.unit0 = I.unit0; g.part0 = I.part0;
    g.o = I.o[k]; g.oc = I.oc[k];
    g.s = level_s(k);
    g.d = 4.0f * g.s + (float)I.lambda;
    g.lambda = I.lambda;
    return g;
  };
  auto second = [](Geo &g, const Inst &I, int k) {
    g.W2 = I.w[k]; g.H2 = I.h[k]; g.o2 = I.o[k]; g.oc2 = I.oc[k];
  };
  {
    std::vector<Geo> g0;
    for (const Inst &I : m.in) g0.push_back(geo_at(I, 0, I.W, I.H, kMinBands));
    m.all0 = make_launch(blob, g0);
  }
  m.full.resize(Lmax); m.half.resize(Lmax); m.restr.resize(Lmax); m.coarse.resize(Lmax);
  for (int k = 0; k < Lmax; ++k) {
    long long many = 0;  // the level's tiles at one band each, all channels
    for (const Inst &I : m.in)
      if (k < I.L - 1) {
        int gx, gy;
        tiles2(I.w[k], I.h[k], sms, 1, gx, gy);
        many += (long long)I.C * gx * gy;
      }
    const int mb = many > kManyWaves * 8 * sms ? kMinBands : 1;
    std::vector<Geo> gf, gh, gr, gk;
    for (const Inst &I : m.in) {
      if (k == I.L - 1) {
        gk.push_back(geo_at(I, k, 1, 1, 1));
      } else if (k < I.L - 1) {
        Geo f = geo_at(I, k, I.w[k], I.h[k], mb);
        second(f, I, k + 1);
        gf.push_back(f);
        gh.push_back(geo_at(I, k, (I.w[k] + 1) / 2, I.h[k], mb));
        Geo r = geo_at(I, k + 1, I.w[k + 1], I.h[k + 1], mb);  // coarse tiles, the fine level's operator
        r.s = level_s(k);
        r.d = 4.0f * r.s + (float)I.lambda;
        second(r, I, k);
        gr.push_back(r);
      }
    }
    m.full[k] = make_launch(blob, gf);
    m.half[k] = make_launch(blob, gh);
    m.restr[k] = make_launch(blob, gr);
    m.coarse[k] = make_launch(blob, gk);
  }
  {
    std::vector<Red> rt;
    for (const Inst &I : m.in)
      for (int c = 0; c < I.C; ++c)
        rt.push_back(Red{I.part0 + (long long)c * I.gx * I.gy, (long long)I.gx * I.gy});
    m.rtab = blob.put(rt.data(), rt.size() * sizeof(Red));
  }

  // arena: tables, levels, level-0 vectors, then the staged host buffers
  size_t o = 0;
  auto take = [&](size_t b) { size_t r = o; o = aup(o + std::max<size_t>(b, 1)); return r; };
  m.tab = take(blob.b.size());
  m.io = take(m.in.size() * sizeof(Io));
  m.lv.resize(Lmax);
  for (int k = 0; k < Lmax; ++k) {
    m.lv[k].act = take((size_t)cells[k]);
    if (k > 0) {
      m.lv[k].e = take((size_t)ccells[k] * sizeof(float));
      m.lv[k].rhs = take((size_t)ccells[k] * sizeof(float));
    }
  }
  const size_t NC = (size_t)ccells[0];
  m.u = take(NC * 8); m.bl = take(NC * 8); m.uw = any_warm ? take(NC * 8) : 0; m.r64 = take(NC * 8);
  m.part = take((size_t)P * 8); m.red = take((size_t)U * 8); m.sc = take((size_t)U * S_N * 8);
  m.scale = take((size_t)U * 8); m.run = take((size_t)U * 8);
  m.x = take(NC * 4); m.r = take(NC * 4); m.z = take(NC * 4); m.p = take(NC * 4); m.q = take(NC * 4);
  for (Inst &I : m.in) {
    if (I.dev) continue;
    const size_t n = (size_t)I.W * I.H, nc = n * I.C;
    I.in = take(nc * 2 * 4); I.mask = take(n * 4); I.guess = I.warm ? take(nc * 4) : 0; I.out = take(nc * 4);
  }
  if (!ctx->reserve(o)) return mfail(ctx, PT_OOM, "device arena allocation failed");
  m.base = static_cast<char *>(ctx->arena);
  cudaEventRecord(ctx->ev[0], m.st);

  // tables and inputs
  cudaError_t ce = cudaMemcpyAsync(m.base + m.tab, blob.b.data(), blob.b.size(), cudaMemcpyHostToDevice, m.st);
  std::vector<Io> io(m.in.size());
  for (size_t k = 0; k < m.in.size() && ce == cudaSuccess; ++k) {
    const Inst &I = m.in[k];
    const pt_problem &p = ps[I.idx];
    const size_t n = (size_t)I.W * I.H, nc = n * I.C;
    if (I.dev) {
      io[k] = Io{p.source_or_guidance, p.target_or_anchor, p.mask, I.warm ? p.initial_guess : nullptr, outs[I.idx]};
      continue;
    }
    float *in = m.at<float>(I.in);
    ce = cudaMemcpyAsync(in, p.source_or_guidance, nc * 4, cudaMemcpyHostToDevice, m.st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(in + nc, p.target_or_anchor, nc * 4, cudaMemcpyHostToDevice, m.st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(m.at<float>(I.mask), p.mask, n * 4, cudaMemcpyHostToDevice, m.st);
    if (ce == cudaSuccess && I.warm)
      ce = cudaMemcpyAsync(m.at<float>(I.guess), p.initial_guess, nc * 4, cudaMemcpyHostToDevice, m.st);
    io[k] = Io{in, in + nc, m.at<float>(I.mask), I.warm ? m.at<float>(I.guess) : nullptr, m.at<float>(I.out)};
  }
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(m.base + m.io, io.data(), io.size() * sizeof(Io), cudaMemcpyHostToDevice, m.st);
  if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("input upload: ") + cudaGetErrorString(ce));

  const Io *iod = m.at<Io>(m.io);
  const Launch &A = m.all0;
  const Geo *g0 = m.geo(A);
  const int4 *b0 = m.bmap(A);
  const dim3 ga = m.grid(A, m.Cmax);
  const Red *rtab = m.at<Red>(m.tab + m.rtab);
  uint8_t *act0 = m.at<uint8_t>(m.lv[0].act);
  double *u = m.at<double>(m.u), *bl = m.at<double>(m.bl), *r64 = m.at<double>(m.r64), *part = m.at<double>(m.part),
         *red = m.at<double>(m.red), *sc = m.at<double>(m.sc), *scale = m.at<double>(m.scale),
         *run = m.at<double>(m.run);
  float *x = m.at<float>(m.x), *r = m.at<float>(m.r), *z = m.at<float>(m.z), *pp = m.at<float>(m.p),
        *q = m.at<float>(m.q);
  k_mg_assemble<<<m.grid(A, 1), kBlock2, 0, m.st>>>(g0, b0, A.one, iod, act0, u, bl,
                                                     any_warm ? m.at<double>(m.uw) : nullptr);
  m.launches = 1;
  for (int k = 0; k + 1 < Lmax; ++k) {
    const Launch &R = m.restr[k];
    if (!R.n) continue;
    k_mg_coarsen<<<m.grid(R, 1), kBlock2, 0, m.st>>>(m.geo(R), m.bmap(R), R.one, m.at<uint8_t>(m.lv[k].act),
                                                     m.at<uint8_t>(m.lv[k + 1].act));
    ++m.launches;
  }
  cudaEventRecord(ctx->ev[1], m.st);

  // per-unit facts
  std::vector<int> uinst(U), maxit(U);
  std::vector<double> tol(U);
  for (size_t k = 0; k < m.in.size(); ++k)
    for (int c = 0; c < m.in[k].C; ++c) {
      const int un = m.in[k].unit0 + c;
      uinst[un] = (int)k;
      tol[un] = ps[m.in[k].idx].tolerance;
      maxit[un] = (int)ps[m.in[k].idx].max_iterations;
    }

  // FP64 residual norms per unit of the current u -> host
  std::vector<double> nrm(U);
  auto residual = [&](const double *uu) -> cudaError_t {
    k_mg_residual64<<<ga, kBlock2, 0, m.st>>>(g0, b0, A.one, act0, uu, bl, r64, part);
    k_mg_reduce<<<U, kThreads, 0, m.st>>>(part, rtab, red, 1);
    m.launches += 2;
    cudaError_t e = cudaMemcpyAsync(nrm.data(), red, (size_t)U * 8, cudaMemcpyDeviceToHost, m.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m.st);
    for (double &v : nrm) v = std::sqrt(v);
    return e;
  };
  ce = residual(u);
  if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("residual: ") + cudaGetErrorString(ce));
  const std::vector<double> r0 = nrm;  // ||r(anchor)|| per unit: the bar is tolerance * r0
  std::vector<int> warm_used(U, 0);
  if (any_warm) {
    double *uw = m.at<double>(m.uw);
    ce = residual(uw);
    if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("residual: ") + cudaGetErrorString(ce));
    // a guess is used per channel only if its residual is finite and below the anchor's
    for (int un = 0; un < U; ++un) {
      const Inst &I = m.in[uinst[un]];
      if (!I.warm || !(std::isfinite(nrm[un]) && nrm[un] < r0[un])) continue;
      warm_used[un] = 1;
      const size_t n = (size_t)I.W * I.H, off = (size_t)I.oc[0] + (size_t)(un - I.unit0) * n;
      cudaMemcpyAsync(u + off, uw + off, n * 8, cudaMemcpyDeviceToDevice, m.st);
    }
    ce = residual(u);
    if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("residual: ") + cudaGetErrorString(ce));
  }

  // per-unit state
  std::vector<int> its(U, 0), stop(U, -1), refines(U, 0);
  std::vector<double> cur = nrm;  // FP64 ||r|| of the current u
  std::vector<std::vector<double>> hist(U);
  std::vector<double> hscale(U, 0.0), hrun(U, 0.0), rr(U);
  bool poisoned = false;
  for (int un = 0; un < U; ++un) {
    if (r0[un] == 0.0) stop[un] = PT_STOP_CONVERGED;  // poisson.rs:178-185
    else if (!std::isfinite(cur[un])) {  // (before the bar: inf <= tol * inf would pass it)
      // a NaN or infinity reached the system: its residual can never improve,
      // which the reference ends by its stall rule with the region's cells
      // non-finite; here at once, with the interior set to NaN
      stop[un] = PT_STOP_STALLED;
      hscale[un] = std::nan("");
      poisoned = true;
    } else if (cur[un] <= tol[un] * r0[un]) stop[un] = PT_STOP_CONVERGED;
    else if (maxit[un] == 0) stop[un] = PT_STOP_MAX_ITERATIONS;
  }
  if (poisoned) {  // u = fma(NaN, 0, u) = NaN at interior cells of those units
    cudaMemcpyAsync(scale, hscale.data(), (size_t)U * 8, cudaMemcpyHostToDevice, m.st);
    cudaMemsetAsync(x, 0, NC * 4, m.st);
    k_mg_update<<<ga, kBlock2, 0, m.st>>>(g0, b0, A.one, act0, x, scale, u);
    ++m.launches;
    std::fill(hscale.begin(), hscale.end(), 0.0);
  }
  // One CG iteration: V-cycle z = M r, rho = r.z, p = z + beta p, q = A p,
  // alpha = rho / p.q, x += alpha p, r -= alpha q, ||r||^2 (to `red`). Its
  // launches depend only on the group's shapes and the arena, so they are
  // captured once into two CUDA graphs (first iteration, later ones) cached on
  // the context and replayed while shapes and arena stay the same.
  long long per_iteration = 0;
  const unsigned gsc = (unsigned)std::max(1, std::min((U + kThreads - 1) / kThreads, sms * 4));
  auto enqueue_iteration = [&](bool first) -> cudaError_t {
    const long long l0 = m.launches;
    vcycle(m, r, z);
    k_cg_dot<<<ga, kBlock2, 0, m.st>>>(g0, b0, A.one, r, z, part, run);
    k_mg_reduce<<<U, kThreads, 0, m.st>>>(part, rtab, sc + S_RHO_NEW, S_N);
    k_cg_direction<<<ga, kBlock2, 0, m.st>>>(g0, b0, A.one, z, pp, sc, run, first ? 1 : 0);
    k_cg_scalars_after_dir<<<gsc, kThreads, 0, m.st>>>(U, sc);
    k_cg_apply<<<ga, kBlock2, 0, m.st>>>(g0, b0, A.one, act0, pp, q, part, run);
    k_mg_reduce<<<U, kThreads, 0, m.st>>>(part, rtab, sc + S_PQ, S_N);
    k_cg_step<<<ga, kBlock2, 0, m.st>>>(g0, b0, A.one, pp, q, x, r, sc, part, run);
    k_mg_reduce<<<U, kThreads, 0, m.st>>>(part, rtab, red, 1);
    m.launches += 8;
    per_iteration = m.launches - l0;
    return cudaGetLastError();
  };
  if (ctx->graphs) {
    // the graphs' arguments are arena offsets and the tables' contents
    std::string key(reinterpret_cast<const char *>(&m.base), sizeof(m.base));
    std::vector<size_t> offs = {o, m.tab, m.rtab, m.part, m.red, m.sc, m.run, m.x, m.r, m.z, m.p, m.q,
                                (size_t)m.Cmax, (size_t)U};
    for (const LevelArr &v : m.lv) offs.insert(offs.end(), {v.act, v.e, v.rhs});
    key.append(reinterpret_cast<const char *>(offs.data()), offs.size() * sizeof(size_t));
    key.append(reinterpret_cast<const char *>(blob.b.data()), blob.b.size());
    if (key != ctx->mgkey || !ctx->mgexec[0] || !ctx->mgexec[1]) {
      for (auto &ge : ctx->mgexec)
        if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
      ctx->mgkey.clear();
      const long long saved = m.launches;
      for (int g = 0; g < 2 && ce == cudaSuccess; ++g) {
        cudaGraph_t graph = nullptr;
        ce = cudaStreamBeginCapture(m.st, cudaStreamCaptureModeThreadLocal);
        if (ce == cudaSuccess) {
          const cudaError_t e1 = enqueue_iteration(g == 0);
          ce = cudaStreamEndCapture(m.st, &graph);
          if (e1 != cudaSuccess) ce = e1;
        }
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&ctx->mgexec[g], graph, 0);
        if (graph) cudaGraphDestroy(graph);
      }
      m.launches = saved;
      ctx->mgnodes = per_iteration;
      if (ce != cudaSuccess) {
        for (auto &ge : ctx->mgexec)
          if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
        return mfail(ctx, PT_LAUNCH_FAILED, std::string("graph capture: ") + cudaGetErrorString(ce));
      }
      ctx->mgkey = std::move(key);
    }
  }
  int outer = 0;
  while (std::any_of(stop.begin(), stop.end(), [](int s) { return s < 0; })) {
    // scale this outer step's residual to unit norm; units that stopped get 0
    for (int un = 0; un < U; ++un) {
      hscale[un] = stop[un] < 0 ? cur[un] : 0.0;
      hrun[un] = stop[un] < 0 ? 1.0 : 0.0;
    }
    cudaMemcpyAsync(scale, hscale.data(), (size_t)U * 8, cudaMemcpyHostToDevice, m.st);
    cudaMemcpyAsync(run, hrun.data(), (size_t)U * 8, cudaMemcpyHostToDevice, m.st);
    cudaMemsetAsync(sc, 0, (size_t)U * S_N * 8, m.st);
    k_mg_scale<<<ga, kBlock2, 0, m.st>>>(g0, b0, A.one, r64, scale, r);
    cudaMemsetAsync(x, 0, NC * 4, m.st);
    m.launches += 1;
    // inner target: a quarter of the remaining bar, at most as deep as FP32
    // goes from a unit residual; a run whose residual stops falling (less than
    // 30% over 4 iterations: the FP32 floor) hands over to the next outer step
    std::vector<double> target(U), rel(U, 1.0);
    std::vector<std::vector<double>> seen(U);
    std::vector<int> going(U);
    for (int un = 0; un < U; ++un) {
      going[un] = stop[un] < 0;
      target[un] = going[un] ? std::max(0.25 * tol[un] * r0[un] / cur[un], kInnerFloor) : 1.0;
    }
    for (int it = 0;; ++it) {
      const int g = it == 0 ? 0 : 1;
      if (ctx->mgexec[g]) {
        ce = cudaGraphLaunch(ctx->mgexec[g], m.st);
        m.launches += ctx->mgnodes;
      } else {
        ce = enqueue_iteration(it == 0);
      }
      if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("cg: ") + cudaGetErrorString(ce));
      ce = cudaMemcpyAsync(rr.data(), red, (size_t)U * 8, cudaMemcpyDeviceToHost, m.st);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(m.st);
      if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("cg: ") + cudaGetErrorString(ce));
      bool any = false, changed = false;
      for (int un = 0; un < U; ++un) {
        if (!going[un]) continue;
        its[un] += 1;
        rel[un] = std::sqrt(rr[un]);  // relative to this outer step's unit residual
        hist[un].push_back(rel[un] * cur[un] / r0[un]);
        seen[un].push_back(rel[un]);
        const size_t n = seen[un].size();
        const bool stuck = n > 4 && seen[un][n - 1] > 0.7 * seen[un][n - 5];
        if (rel[un] <= target[un] || stuck || its[un] >= maxit[un] || !std::isfinite(rel[un])) {
          going[un] = 0;
          hrun[un] = 0.0;
          changed = true;
        }
        any |= going[un] != 0;
      }
      if (!any) break;
      if (changed) cudaMemcpyAsync(run, hrun.data(), (size_t)U * 8, cudaMemcpyHostToDevice, m.st);
    }
    // u += scale * x, then the FP64 residual decides
    k_mg_update<<<ga, kBlock2, 0, m.st>>>(g0, b0, A.one, act0, x, scale, u);
    ++m.launches;
    const std::vector<double> prev = cur;
    ce = residual(u);
    if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("residual: ") + cudaGetErrorString(ce));
    for (int un = 0; un < U; ++un) {
      if (stop[un] >= 0) continue;
      cur[un] = nrm[un];
      if (!hist[un].empty()) hist[un].back() = cur[un] / r0[un];
      if (outer > 0) refines[un] += 1;
      if (cur[un] <= tol[un] * r0[un]) stop[un] = PT_STOP_CONVERGED;
      else if (its[un] >= maxit[un]) stop[un] = PT_STOP_MAX_ITERATIONS;
      else if (!(cur[un] < prev[un] * (1.0 - 1e-12))) stop[un] = PT_STOP_STALLED;
    }
    ++outer;
  }
  cudaEventRecord(ctx->ev[2], m.st);
  k_mg_emit<<<m.grid(A, 1), kBlock2, 0, m.st>>>(g0, b0, A.one, iod, act0, u);
  ++m.launches;
  ce = cudaSuccess;
  for (size_t k = 0; k < m.in.size() && ce == cudaSuccess; ++k) {
    const Inst &I = m.in[k];
    if (!I.dev)
      ce = cudaMemcpyAsync(outs[I.idx], m.at<float>(I.out), (size_t)I.W * I.H * I.C * 4, cudaMemcpyDeviceToHost,
                           m.st);
    double *hp = histories ? histories[I.idx] : nullptr;
    if (!hp) continue;
    const uint32_t cap = ps[I.idx].max_iterations;
    for (int c = 0; c < I.C && ce == cudaSuccess; ++c) {
      const std::vector<double> &h = hist[I.unit0 + c];
      const size_t n = std::min<size_t>(h.size(), cap);
      if (!n) continue;
      ce = cudaMemcpyAsync(hp + (size_t)c * cap, h.data(), n * 8,
                           I.dev ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost, m.st);
    }
  }
  if (ce == cudaSuccess) ce = cudaEventRecord(ctx->ev[3], m.st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(m.st);
  if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("result download: ") + cudaGetErrorString(ce));
  {
    float a = 0.f, b = 0.f;
    if (cudaEventElapsedTime(&a, ctx->ev[1], ctx->ev[2]) != cudaSuccess) a = -1.f;
    if (cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[3]) != cudaSuccess) b = -1.f;
    cudaGetLastError();
    solve_ms += a;
    call_ms += b;
    launches += m.launches;
  }
  for (const Inst &I : m.in) {
    pt_report *reps = reports[I.idx];
    const pt_problem &p = ps[I.idx];
    int worst = -1;
    for (int c = 0; c < I.C; ++c) {
      const int un = I.unit0 + c;
      pt_report rep{};
      rep.iterations = (uint32_t)its[un];
      rep.stop_reason = stop[un];
      rep.converged = stop[un] == PT_STOP_CONVERGED;
      rep.tolerance = p.tolerance;
      rep.final_residual = r0[un] == 0.0 ? cur[un] : cur[un] / r0[un];
      rep.history_len = (uint32_t)std::min<size_t>(hist[un].size(), p.max_iterations);
      rep.omega_used = kSmoothOmega;
      rep.refinements = (uint32_t)refines[un];
      rep.channel = c;
      rep.initial_residual = r0[un];
      rep.warm_start = warm_used[un];
      reps[c] = rep;
      // worse_of (poisson_blend.rs:240-246)
      if (worst < 0) worst = c;
      else {
        const pt_report &a = reps[worst];
        const bool b_worse = (rep.iterations != a.iterations) ? (rep.iterations > a.iterations)
                                                              : (rep.final_residual > a.final_residual);
        if (b_worse) worst = c;
      }
    }
    reps[I.C] = reps[worst];
  }
  return PT_OK;
}

}  // namespace

// Problems with PT_FLAG_MULTIGRID (pt_poisson_solve, pt_poisson_solve_batch):
// all of a call's instances share each launch, in groups of at most
// kGroupTiles level-0 tiles.
pt_status ptk_solve_mg_batch(pt_ctx *ctx, const pt_problem *ps, uint32_t n, float *const *outs,
                             pt_report *const *reports, double *const *histories) {
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return mfail(ctx, PT_NO_DEVICE, cudaGetErrorString(ce));
  for (auto &e : ctx->ev)
    if (!e && cudaEventCreate(&e) != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, "event create");
  double solve_ms = 0.0, call_ms = 0.0;
  long long launches = 0, tiles = 0, units = 0;
  bool ran = false;
  std::vector<int> ids;
  auto flush = [&]() -> pt_status {
    if (ids.empty()) return PT_OK;
    const pt_status s = solve_group(ctx, ps, ids, outs, reports, histories, solve_ms, call_ms, launches);
    ids.clear();
    tiles = units = 0;
    ran = true;
    return s;
  };
  for (uint32_t i = 0; i < n; ++i) {
    const pt_problem &p = ps[i];
    if (p.channels == 0) {
      pt_report r{};
      r.converged = 1; r.stop_reason = PT_STOP_CONVERGED; r.tolerance = p.tolerance; r.channel = -1;
      reports[i][0] = r;
      continue;
    }
    int gx, gy;
    tiles2((int)p.width, (int)p.height, ctx->sms, kMinBands, gx, gy);
    const long long t = (long long)gx * gy;
    if (!ids.empty() && (tiles + t > kGroupTiles || units + p.channels > kGroupTiles)) {
      const pt_status s = flush();
      if (s != PT_OK) return s;
    }
    ids.push_back((int)i);
    tiles += t;
    units += p.channels;
  }
  const pt_status s = flush();
  if (s != PT_OK) return s;
  if (ran) {
    ctx->last_solve_ms = solve_ms;
    ctx->last_call_ms = call_ms;
    ctx->last_launches = launches;
    ctx->last_h2d = ctx->last_d2h = 0;  // not counted on this path
  }
  return PT_OK;
}
