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
// Gauss-Seidel, red then black before the coarse correction and black then
// red after it, so the V-cycle is a symmetric operator and a valid CG
// preconditioner. All channels of an image share the level masks and are
// processed by the same launches. Every reduction is a fixed-order tree, so a
// rerun is byte-identical.
//
// Report (pt_report): iterations = preconditioned CG iterations (each one
// V-cycle and one operator application); history[k] = relative residual after
// iteration k -- the CG recurrence's estimate scaled by the outer step's FP64
// residual, replaced by the exact FP64 value at the end of every outer step;
// refinements = outer steps after the first; omega_used = the smoother's
// relaxation factor. Stop reasons: converged at the FP64 bar; max-iterations when the
// CG iterations reach max_iterations; stalled when an outer step fails to
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

// ---- assembly ----------------------------------------------------------------
// interior flag, u = anchor (or the warm guess at interior cells), b' =
// fma(lambda, -anchor, laplacian(guidance)) at interior cells, all channels.
__global__ void k_mg_assemble(int W, int H, int C, const float *__restrict__ guid, const float *__restrict__ anchor,
                              const float *__restrict__ mask, const float *__restrict__ guess, double lambda,
                              uint8_t *__restrict__ act, double *__restrict__ u, double *__restrict__ bl,
                              double *__restrict__ uw) {
  const long long N = (long long)W * H;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N * C;
       p += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(p / N);
    const long long q = p - (long long)c * N;
    const int j = (int)(q / W), i = (int)(q - (long long)j * W);
    const bool in = W >= 3 && H >= 3 && i > 0 && j > 0 && i < W - 1 && j < H - 1 && mask[q] > 0.5f;
    if (c == 0) act[q] = in ? 1 : 0;
    const double a = (double)anchor[q * C + c];
    u[p] = a;
    double b = 0.0;
    if (in) {
      // poisson.rs:364-373: L, R, U, D, then fma(4, -centre, sum)
      const double ctr = (double)guid[q * C + c];
      const double s = (double)guid[(q - 1) * C + c] + (double)guid[(q + 1) * C + c] + (double)guid[(q - W) * C + c] +
                       (double)guid[(q + W) * C + c];
      b = fma(4.0, -ctr, s);
    }
    bl[p] = in ? fma(lambda, -a, b) : 0.0;
    if (uw) uw[p] = (in && guess) ? (double)guess[q * C + c] : a;
  }
}

// Stencil and vector kernels run on 2-D grids: threads (32, 8) over columns
// and rows, grid.y strides over rows, grid.z is the channel; all index math is
// 32-bit (a level has at most 2^31 cells). Kernels that reduce write one
// partial per block, (blockIdx.y * gridDim.x + blockIdx.x), per channel.
constexpr int kTx = 32, kTy = 8;

__device__ __forceinline__ int block_index() { return blockIdx.y * gridDim.x + blockIdx.x; }
__device__ __forceinline__ int blocks_per_channel() { return gridDim.x * gridDim.y; }

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

// r = fma(lambda + 4, -u, nsum) - b' at interior cells (0 elsewhere) and
// per-block partial sums of r^2.
__global__ void __launch_bounds__(kTx * kTy) k_mg_residual64(int W, int H, const uint8_t *__restrict__ act,
                                                             const double *__restrict__ u,
                                                             const double *__restrict__ bl, double lambda,
                                                             double *__restrict__ r64, double *__restrict__ part) {
  __shared__ double sh[kTx * kTy];
  const int c = blockIdx.z;
  const size_t N = (size_t)W * H;
  const double *uc = u + c * N;
  const int i = blockIdx.x * kTx + threadIdx.x;
  double acc = 0.0;
  for (int j = blockIdx.y * kTy + threadIdx.y; j < H && i < W; j += gridDim.y * kTy) {
    const size_t q = (size_t)j * W + i;
    double r = 0.0;
    if (act[q]) {
      const double nsum = uc[q - 1] + uc[q + 1] + uc[q - W] + uc[q + W];  // L, R, U, D (poisson.rs:275-298)
      r = fma(lambda + 4.0, -uc[q], nsum) - bl[c * N + q];
    }
    r64[c * N + q] = r;
    acc += r * r;
  }
  const double t = block_sum2(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[(size_t)c * blocks_per_channel() + block_index()] = t;
}

// out[c * stride] = fixed-order sum of part[c][0 .. n-1]; grid (C)
__global__ void k_mg_reduce(const double *__restrict__ part, int n, double *__restrict__ out, int stride) {
  __shared__ double sh[kThreads];
  double acc = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) acc += part[(long long)blockIdx.x * n + k];
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) out[(long long)blockIdx.x * stride] = s;
}

// r32 = r64 / scale[c] (0 where the channel is not being corrected)
__global__ void __launch_bounds__(kTx * kTy) k_mg_scale(int W, int H, const double *__restrict__ r64,
                                                        const double *__restrict__ scale, float *__restrict__ r32) {
  const int c = blockIdx.z, i = blockIdx.x * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const double s = scale[c];
  for (int j = blockIdx.y * kTy + threadIdx.y; j < H && i < W; j += gridDim.y * kTy) {
    const size_t o = c * N + (size_t)j * W + i;
    r32[o] = s > 0.0 ? (float)(r64[o] / s) : 0.0f;
  }
}

// u += scale[c] * x at interior cells
__global__ void __launch_bounds__(kTx * kTy) k_mg_update(int W, int H, const uint8_t *__restrict__ act,
                                                         const float *__restrict__ x, const double *__restrict__ scale,
                                                         double *__restrict__ u) {
  const int c = blockIdx.z, i = blockIdx.x * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const double s = scale[c];
  for (int j = blockIdx.y * kTy + threadIdx.y; j < H && i < W; j += gridDim.y * kTy) {
    const size_t q = (size_t)j * W + i;
    if (act[q]) u[c * N + q] = fma(s, (double)x[c * N + q], u[c * N + q]);
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

__global__ void k_mg_coarsen(int Wf, int Hf, const uint8_t *__restrict__ af, int Wc, int Hc, uint8_t *__restrict__ ac) {
  const long long N = (long long)Wc * Hc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < N; q += (long long)gridDim.x * blockDim.x) {
    const int J = (int)(q / Wc), I = (int)(q - (long long)J * Wc);
    int n = 0;
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        const int i = 2 * I + dx, j = 2 * J + dy;
        if (i < Wf && j < Hf) n += af[(long long)j * Wf + i];
      }
    ac[q] = n >= kCoarseRule ? 1 : 0;
  }
}

// One colour of red-black Gauss-Seidel on A_k e = rhs: e = (rhs + s * sum of
// neighbours) / d at active cells of that colour (inactive cells hold 0).
// x threads index the cells of one colour in a row.
__global__ void __launch_bounds__(kTx * kTy) k_mg_smooth(int W, int H, const uint8_t *__restrict__ act,
                                                         const float *__restrict__ rhs, float *__restrict__ e, float s,
                                                         float d, int color) {
  const int c = blockIdx.z, m = blockIdx.x * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  float *ec = e + c * N;
  const float *rc = rhs + c * N;
  for (int j = blockIdx.y * kTy + threadIdx.y; j < H; j += gridDim.y * kTy) {
    const int i = 2 * m + ((j + color) & 1);
    if (i >= W) continue;
    const size_t q = (size_t)j * W + i;
    if (!act[q]) continue;
    float nb = 0.0f;
    if (i > 0) nb += ec[q - 1];
    if (i < W - 1) nb += ec[q + 1];
    if (j > 0) nb += ec[q - W];
    if (j < H - 1) nb += ec[q + W];
    const float gs = (rc[q] + s * nb) / d;
    ec[q] = ec[q] + kSmoothOmega * (gs - ec[q]);
  }
}

// The first half-sweep of a V-cycle level, from e = 0: e = rhs / d at active
// cells of colour 0 (red), 0 everywhere else, relaxed by kSmoothOmega -- what
// zeroing e and one red half-sweep produce, bit for bit, in one pass that
// writes every cell.
__global__ void __launch_bounds__(kTx * kTy) k_mg_smooth_first(int W, int H, const uint8_t *__restrict__ act,
                                                               const float *__restrict__ rhs, float *__restrict__ e,
                                                               float s, float d) {
  const int c = blockIdx.z, i = blockIdx.x * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  for (int j = blockIdx.y * kTy + threadIdx.y; j < H && i < W; j += gridDim.y * kTy) {
    const size_t q = (size_t)j * W + i;
    const float gs = (rhs[c * N + q] + s * 0.0f) / d;
    e[c * N + q] = (act[q] && ((i + j) & 1) == 0) ? 0.0f + kSmoothOmega * (gs - 0.0f) : 0.0f;
  }
}

// The coarsest level (at most kCoarseMax cells): `sweeps` red-black sweeps,
// then as many in reverse colour order, from e = 0, in shared memory; one
// block per channel.
constexpr int kCoarseMax = 64;

__global__ void k_mg_coarse(int W, int H, const uint8_t *__restrict__ act, const float *__restrict__ rhs,
                            float *__restrict__ e, float s, float d, int sweeps) {
  __shared__ float se[kCoarseMax], sr[kCoarseMax];
  __shared__ uint8_t sa[kCoarseMax];
  const int n = W * H, c = blockIdx.x, t = threadIdx.x;
  if (t < n) {
    se[t] = 0.0f;
    sr[t] = rhs[(long long)c * n + t];
    sa[t] = act[t];
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
  if (t < n) e[(long long)c * n + t] = se[t];
}

__device__ __forceinline__ float pw(int a) { return (a == 0 || a == 1) ? 0.75f : 0.25f; }  // a = fine - 2 * coarse

// The restriction of the level's residual, rhs_c(I, J) = sum over fine
// (2I + a, 2J + b), a, b in -1..2, of wx wy res_f / 4 with res_f = rhs - A e at
// active fine cells (0 elsewhere), evaluated on the fly so the residual is
// never stored.
__global__ void __launch_bounds__(kTx * kTy) k_mg_resid_restrict(int Wf, int Hf, const uint8_t *__restrict__ af,
                                                                 const float *__restrict__ rhsf,
                                                                 const float *__restrict__ ef, float s, float d, int Wc,
                                                                 int Hc, const uint8_t *__restrict__ ac,
                                                                 float *__restrict__ rhsc) {
  const int c = blockIdx.z, I = blockIdx.x * kTx + threadIdx.x;
  const size_t Nc = (size_t)Wc * Hc, Nf = (size_t)Wf * Hf;
  const float *e = ef + c * Nf, *rh = rhsf + c * Nf;
  for (int J = blockIdx.y * kTy + threadIdx.y; J < Hc && I < Wc; J += gridDim.y * kTy) {
    const size_t q = (size_t)J * Wc + I;
    float v = 0.0f;
    if (ac[q]) {
      for (int b = -1; b <= 2; ++b) {
        const int j = 2 * J + b;
        if (j < 0 || j >= Hf) continue;
        float row = 0.0f;
        for (int a = -1; a <= 2; ++a) {
          const int i = 2 * I + a;
          if (i < 0 || i >= Wf) continue;
          const size_t f = (size_t)j * Wf + i;
          float r = 0.0f;
          if (af[f]) {
            float nb = 0.0f;
            if (i > 0) nb += e[f - 1];
            if (i < Wf - 1) nb += e[f + 1];
            if (j > 0) nb += e[f - Wf];
            if (j < Hf - 1) nb += e[f + Wf];
            r = rh[f] - (d * e[f] - s * nb);
          }
          row += pw(a) * r;
        }
        v += pw(b) * row;
      }
      v *= 0.25f;
    }
    rhsc[c * Nc + q] = v;
  }
}

// e_f += bilinear prolongation of e_c at active fine cells
__global__ void __launch_bounds__(kTx * kTy) k_mg_prolong(int Wf, int Hf, const uint8_t *__restrict__ af,
                                                          float *__restrict__ ef, int Wc, int Hc,
                                                          const float *__restrict__ ec) {
  const int c = blockIdx.z, i = blockIdx.x * kTx + threadIdx.x;
  const size_t Nc = (size_t)Wc * Hc, Nf = (size_t)Wf * Hf;
  const float *e = ec + c * Nc;
  for (int j = blockIdx.y * kTy + threadIdx.y; j < Hf && i < Wf; j += gridDim.y * kTy) {
    const size_t q = (size_t)j * Wf + i;
    if (!af[q]) continue;
    const int I0 = i >> 1, J0 = j >> 1;
    const int I1 = (i & 1) ? I0 + 1 : I0 - 1, J1 = (j & 1) ? J0 + 1 : J0 - 1;
    auto at = [&](int I, int J) -> float {
      return (I >= 0 && I < Wc && J >= 0 && J < Hc) ? e[(size_t)J * Wc + I] : 0.0f;
    };
    const float v = 0.5625f * at(I0, J0) + 0.1875f * (at(I1, J0) + at(I0, J1)) + 0.0625f * at(I1, J1);
    ef[c * Nf + q] += v;
  }
}

// ---- conjugate gradients -------------------------------------------------------
// q = A_0 p at active cells; partial sums of p.q
__global__ void __launch_bounds__(kTx * kTy) k_cg_apply(int W, int H, const uint8_t *__restrict__ act,
                                                        const float *__restrict__ p, float d, float *__restrict__ q,
                                                        double *__restrict__ part) {
  __shared__ double sh[kTx * kTy];
  const int c = blockIdx.z, i = blockIdx.x * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const float *pc = p + c * N;
  double acc = 0.0;
  for (int j = blockIdx.y * kTy + threadIdx.y; j < H && i < W; j += gridDim.y * kTy) {
    const size_t k = (size_t)j * W + i;
    float v = 0.0f;
    if (act[k]) {
      // interior cells are never on the border: all four neighbours exist
      v = d * pc[k] - (pc[k - 1] + pc[k + 1] + pc[k - W] + pc[k + W]);
      acc += (double)pc[k] * (double)v;
    }
    q[c * N + k] = v;
  }
  const double t = block_sum2(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[(size_t)c * blocks_per_channel() + block_index()] = t;
}

// partial sums of a.b
__global__ void __launch_bounds__(kTx * kTy) k_cg_dot(int W, int H, const float *__restrict__ a,
                                                      const float *__restrict__ b, double *__restrict__ part) {
  __shared__ double sh[kTx * kTy];
  const int c = blockIdx.z, i = blockIdx.x * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  double acc = 0.0;
  for (int j = blockIdx.y * kTy + threadIdx.y; j < H && i < W; j += gridDim.y * kTy) {
    const size_t o = c * N + (size_t)j * W + i;
    acc += (double)a[o] * (double)b[o];
  }
  const double t = block_sum2(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[(size_t)c * blocks_per_channel() + block_index()] = t;
}

// Per-channel scalars: sc[c] = {rho, rho_new, pq, rr, alpha, beta, run}
enum { S_RHO, S_RHO_NEW, S_PQ, S_RR, S_ALPHA, S_BETA, S_RUN, S_N };

// p = z + beta p (beta = rho_new / rho; p = z on the first iteration)
__global__ void __launch_bounds__(kTx * kTy) k_cg_direction(int W, int H, const float *__restrict__ z,
                                                            float *__restrict__ p, const double *__restrict__ sc,
                                                            int first) {
  const int c = blockIdx.z, i = blockIdx.x * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const double *s = sc + c * S_N;
  if (s[S_RUN] == 0.0) return;
  const float beta = first ? 0.0f : (float)(s[S_RHO] != 0.0 ? s[S_RHO_NEW] / s[S_RHO] : 0.0);
  for (int j = blockIdx.y * kTy + threadIdx.y; j < H && i < W; j += gridDim.y * kTy) {
    const size_t o = c * N + (size_t)j * W + i;
    p[o] = first ? z[o] : z[o] + beta * p[o];  // first: p is not read (it holds what the arena held)
  }
}

__global__ void k_cg_scalars_after_dir(int C, double *__restrict__ sc) {
  for (int c = threadIdx.x; c < C; c += blockDim.x) sc[c * S_N + S_RHO] = sc[c * S_N + S_RHO_NEW];
}

// x += alpha p, r -= alpha q (alpha = rho / p.q); partial sums of r.r
__global__ void __launch_bounds__(kTx * kTy) k_cg_step(int W, int H, const float *__restrict__ p,
                                                       const float *__restrict__ q, float *__restrict__ x,
                                                       float *__restrict__ r, const double *__restrict__ sc,
                                                       double *__restrict__ part) {
  __shared__ double sh[kTx * kTy];
  const int c = blockIdx.z, i = blockIdx.x * kTx + threadIdx.x;
  const size_t N = (size_t)W * H;
  const double *s = sc + c * S_N;
  if (s[S_RUN] == 0.0) {  // a stopped channel: x and r stay (p may never have been written)
    if (threadIdx.x == 0 && threadIdx.y == 0) part[(size_t)c * blocks_per_channel() + block_index()] = 0.0;
    return;
  }
  const float alpha = s[S_PQ] > 0.0 ? (float)(s[S_RHO] / s[S_PQ]) : 0.0f;
  double acc = 0.0;
  for (int j = blockIdx.y * kTy + threadIdx.y; j < H && i < W; j += gridDim.y * kTy) {
    const size_t o = c * N + (size_t)j * W + i;
    x[o] += alpha * p[o];
    const float rv = r[o] - alpha * q[o];
    r[o] = rv;
    acc += (double)rv * (double)rv;
  }
  const double t = block_sum2(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[(size_t)c * blocks_per_channel() + block_index()] = t;
}

// out = interleave(u) at interior cells, the anchor elsewhere (bit for bit)
__global__ void k_mg_emit(int W, int H, int C, const uint8_t *__restrict__ act, const double *__restrict__ u,
                          const float *__restrict__ anchor, float *__restrict__ out) {
  const long long N = (long long)W * H;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < N * C;
       k += (long long)gridDim.x * blockDim.x) {
    const long long q = k / C;
    const int c = (int)(k - q * C);
    out[k] = act[q] ? (float)u[(long long)c * N + q] : anchor[k];
  }
}

// ---- host ----------------------------------------------------------------------
struct Level {
  int W, H;
  size_t act, e, rhs;  // arena offsets
  float s, d;
};

size_t aup(size_t b) { return (b + 255) & ~(size_t)255; }

struct Mg {
  pt_ctx *ctx;
  cudaStream_t st;
  char *base = nullptr;
  int W, H, C;
  long long N;
  std::vector<Level> lv;
  size_t u, bl, uw, r64, part, red, sc, scale, x, r, z, p, q;
  size_t in, mask, guess, out;  // staged inputs (host buffers)
  int nb;                        // blocks per channel of the reductions
  long long launches = 0;
  template <class T> T *at(size_t off) { return reinterpret_cast<T *>(base + off); }
};

// (32, 8) threads over w columns and h rows, channels in z; at most about 8
// blocks per SM per channel (rows are strided), at most 65535 in y.
dim3 grid2(int w, int h, int C, int sms) {
  const int gx = std::max(1, (w + kTx - 1) / kTx);
  int gy = std::max(1, (h + kTy - 1) / kTy);
  gy = std::min(gy, std::max(1, sms * 8 / gx));
  gy = std::min(gy, 65535);
  return dim3(gx, gy, C);
}
const dim3 kBlock2(kTx, kTy);

unsigned blocks(long long n, int sms) {
  return (unsigned)std::max<long long>(1, std::min<long long>((n + kThreads - 1) / kThreads, (long long)sms * 8));
}

void vcycle(Mg &m, size_t rhs0, size_t e0) {
  const int L = (int)m.lv.size();
  const int sms = m.ctx->sms;
  for (int k = 0; k < L; ++k) {
    Level &v = m.lv[k];
    const size_t rhs = k == 0 ? rhs0 : v.rhs, e = k == 0 ? e0 : v.e;
    const dim3 gh = grid2((v.W + 1) / 2, v.H, m.C, sms), g = grid2(v.W, v.H, m.C, sms);
    if (k == L - 1) {  // the coarsest level: symmetric sweeps in one block per channel
      k_mg_coarse<<<m.C, kCoarseMax, 0, m.st>>>(v.W, v.H, m.at<uint8_t>(v.act), m.at<float>(rhs), m.at<float>(e),
                                                 v.s, v.d, 24);
      ++m.launches;
      break;
    }
    // red, black, red, black from e = 0 (the first red half-sweep writes all of e)
    k_mg_smooth_first<<<g, kBlock2, 0, m.st>>>(v.W, v.H, m.at<uint8_t>(v.act), m.at<float>(rhs), m.at<float>(e), v.s,
                                               v.d);
    k_mg_smooth<<<gh, kBlock2, 0, m.st>>>(v.W, v.H, m.at<uint8_t>(v.act), m.at<float>(rhs), m.at<float>(e), v.s, v.d,
                                          1);
    k_mg_smooth<<<gh, kBlock2, 0, m.st>>>(v.W, v.H, m.at<uint8_t>(v.act), m.at<float>(rhs), m.at<float>(e), v.s, v.d,
                                          0);
    k_mg_smooth<<<gh, kBlock2, 0, m.st>>>(v.W, v.H, m.at<uint8_t>(v.act), m.at<float>(rhs), m.at<float>(e), v.s, v.d,
                                          1);
    m.launches += 4;
    Level &cl = m.lv[k + 1];
    const dim3 gc = grid2(cl.W, cl.H, m.C, sms);
    k_mg_resid_restrict<<<gc, kBlock2, 0, m.st>>>(v.W, v.H, m.at<uint8_t>(v.act), m.at<float>(rhs), m.at<float>(e),
                                                  v.s, v.d, cl.W, cl.H, m.at<uint8_t>(cl.act), m.at<float>(cl.rhs));
    ++m.launches;
  }
  for (int k = L - 2; k >= 0; --k) {
    Level &v = m.lv[k], &cl = m.lv[k + 1];
    const size_t rhs = k == 0 ? rhs0 : v.rhs, e = k == 0 ? e0 : v.e;
    const dim3 gh = grid2((v.W + 1) / 2, v.H, m.C, sms), g = grid2(v.W, v.H, m.C, sms);
    k_mg_prolong<<<g, kBlock2, 0, m.st>>>(v.W, v.H, m.at<uint8_t>(v.act), m.at<float>(e), cl.W, cl.H,
                                           m.at<float>(cl.e));
    for (int t = 0; t < 2; ++t) {
      k_mg_smooth<<<gh, kBlock2, 0, m.st>>>(v.W, v.H, m.at<uint8_t>(v.act), m.at<float>(rhs), m.at<float>(e), v.s,
                                             v.d, 1);
      k_mg_smooth<<<gh, kBlock2, 0, m.st>>>(v.W, v.H, m.at<uint8_t>(v.act), m.at<float>(rhs), m.at<float>(e), v.s,
                                             v.d, 0);
    }
    m.launches += 5;
  }
}

pt_status mfail(pt_ctx *ctx, pt_status s, const std::string &msg) {
  ctx->last_error = msg;
  return s;
}

}  // namespace

// One problem through multigrid-preconditioned CG (called by pt_poisson_solve
// and pt_poisson_solve_batch for problems with PT_FLAG_MULTIGRID).
pt_status ptk_solve_mg(pt_ctx *ctx, const pt_problem &p, float *out_candidate, pt_report *reports, double *history) {
  const int W = (int)p.width, H = (int)p.height, C = (int)p.channels;
  const bool dev = (p.flags & PT_FLAG_DEVICE_POINTERS) != 0, warm = (p.flags & PT_FLAG_WARM_START) != 0;
  if (C == 0) {
    pt_report r{};
    r.converged = 1; r.stop_reason = PT_STOP_CONVERGED; r.tolerance = p.tolerance; r.channel = -1;
    reports[0] = r;
    return PT_OK;
  }
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return mfail(ctx, PT_NO_DEVICE, cudaGetErrorString(ce));
  for (auto &e : ctx->ev)
    if (!e && cudaEventCreate(&e) != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, "event create");
  Mg m;
  m.ctx = ctx; m.st = ctx->stream; m.W = W; m.H = H; m.C = C; m.N = (long long)W * H;
  const long long N = m.N, NC = N * C;
  const dim3 g0 = grid2(W, H, C, ctx->sms);  // level-0 grid of every reducing kernel
  m.nb = (int)(g0.x * g0.y);
  // levels: halve (ceil) while the level has more than 64 cells
  {
    int w = W, h = H, k = 0;
    for (;;) {
      const float s = 1.0f / (float)(1u << (2 * std::min(k, 15)));
      m.lv.push_back(Level{w, h, 0, 0, 0, s, 4.0f * s + (float)p.lambda});
      if ((long long)w * h <= kCoarseMax || k >= 30) break;
      w = (w + 1) / 2; h = (h + 1) / 2; ++k;
    }
  }
  size_t o = 0;
  auto take = [&](size_t b) { size_t r = o; o = aup(o + std::max<size_t>(b, 1)); return r; };
  for (size_t k = 0; k < m.lv.size(); ++k) {
    Level &v = m.lv[k];
    const size_t n = (size_t)v.W * v.H;
    v.act = take(n);
    if (k > 0) { v.e = take(n * C * sizeof(float)); v.rhs = take(n * C * sizeof(float)); }
  }
  m.u = take(NC * 8); m.bl = take(NC * 8); m.uw = warm ? take(NC * 8) : 0; m.r64 = take(NC * 8);
  m.part = take((size_t)m.nb * C * 8); m.red = take((size_t)C * 8); m.sc = take((size_t)C * S_N * 8);
  m.scale = take((size_t)C * 8);
  m.x = take(NC * 4); m.r = take(NC * 4); m.z = take(NC * 4); m.p = take(NC * 4); m.q = take(NC * 4);
  if (!dev) {
    m.in = take(NC * 2 * 4); m.mask = take(N * 4); m.guess = warm ? take(NC * 4) : 0; m.out = take(NC * 4);
  }
  if (!ctx->reserve(o)) return mfail(ctx, PT_OOM, "device arena allocation failed");
  m.base = static_cast<char *>(ctx->arena);
  cudaEventRecord(ctx->ev[0], m.st);

  const float *guid = p.source_or_guidance, *anc = p.target_or_anchor, *msk = p.mask, *gs = p.initial_guess;
  float *out = out_candidate;
  if (!dev) {
    float *in = m.at<float>(m.in);
    ce = cudaMemcpyAsync(in, guid, NC * 4, cudaMemcpyHostToDevice, m.st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(in + NC, anc, NC * 4, cudaMemcpyHostToDevice, m.st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(m.at<float>(m.mask), msk, N * 4, cudaMemcpyHostToDevice, m.st);
    if (ce == cudaSuccess && warm) ce = cudaMemcpyAsync(m.at<float>(m.guess), gs, NC * 4, cudaMemcpyHostToDevice, m.st);
    if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("input upload: ") + cudaGetErrorString(ce));
    guid = in; anc = in + NC; msk = m.at<float>(m.mask); gs = warm ? m.at<float>(m.guess) : nullptr;
    out = m.at<float>(m.out);
  }
  const int sms = ctx->sms;
  const unsigned gall = blocks(NC, sms);
  uint8_t *act0 = m.at<uint8_t>(m.lv[0].act);
  double *u = m.at<double>(m.u), *bl = m.at<double>(m.bl), *r64 = m.at<double>(m.r64), *part = m.at<double>(m.part),
         *red = m.at<double>(m.red), *sc = m.at<double>(m.sc), *scale = m.at<double>(m.scale);
  float *x = m.at<float>(m.x), *r = m.at<float>(m.r), *z = m.at<float>(m.z), *pp = m.at<float>(m.p),
        *q = m.at<float>(m.q);
  k_mg_assemble<<<gall, kThreads, 0, m.st>>>(W, H, C, guid, anc, msk, gs, p.lambda, act0, u, bl,
                                             warm ? m.at<double>(m.uw) : nullptr);
  m.launches = 1;
  for (size_t k = 1; k < m.lv.size(); ++k) {
    const Level &f = m.lv[k - 1], &v = m.lv[k];
    k_mg_coarsen<<<blocks((long long)v.W * v.H, sms), kThreads, 0, m.st>>>(f.W, f.H, m.at<uint8_t>(f.act), v.W, v.H,
                                                                           m.at<uint8_t>(v.act));
    ++m.launches;
  }
  cudaEventRecord(ctx->ev[1], m.st);

  // FP64 residual norms per channel of the current u -> host
  std::vector<double> nrm(C);
  auto residual = [&](const double *uu) -> cudaError_t {
    k_mg_residual64<<<g0, kBlock2, 0, m.st>>>(W, H, act0, uu, bl, p.lambda, r64, part);
    k_mg_reduce<<<C, kThreads, 0, m.st>>>(part, m.nb, red, 1);
    m.launches += 2;
    cudaError_t e = cudaMemcpyAsync(nrm.data(), red, C * 8, cudaMemcpyDeviceToHost, m.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m.st);
    for (double &v : nrm) v = std::sqrt(v);
    return e;
  };
  ce = residual(u);
  if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("residual: ") + cudaGetErrorString(ce));
  const std::vector<double> r0 = nrm;  // ||r(anchor)|| per channel: the bar is tolerance * r0
  std::vector<int> warm_used(C, 0);
  if (warm) {
    double *uw = m.at<double>(m.uw);
    ce = residual(uw);
    if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("residual: ") + cudaGetErrorString(ce));
    // a guess is used per channel only if its residual is finite and below the anchor's
    for (int c = 0; c < C; ++c)
      if (std::isfinite(nrm[c]) && nrm[c] < r0[c]) {
        warm_used[c] = 1;
        cudaMemcpyAsync(u + (long long)c * N, uw + (long long)c * N, N * 8, cudaMemcpyDeviceToDevice, m.st);
      }
    ce = residual(u);
    if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("residual: ") + cudaGetErrorString(ce));
  }

  // per-channel state
  std::vector<int> its(C, 0), stop(C, -1), refines(C, 0);
  std::vector<double> cur = nrm;  // FP64 ||r|| of the current u
  std::vector<std::vector<double>> hist(C);
  std::vector<double> hsc(C * S_N, 0.0), hscale(C, 0.0), rr(C);
  bool poisoned = false;
  for (int c = 0; c < C; ++c) {
    if (r0[c] == 0.0) stop[c] = PT_STOP_CONVERGED;  // poisson.rs:178-185
    else if (!std::isfinite(cur[c])) {  // (before the bar: inf <= tol * inf would pass it)
      // a NaN or infinity reached the system: its residual can never improve,
      // which the reference ends by its stall rule with the region's cells
      // non-finite; here at once, with the interior set to NaN
      stop[c] = PT_STOP_STALLED;
      hscale[c] = std::nan("");
      poisoned = true;
    } else if (cur[c] <= p.tolerance * r0[c]) stop[c] = PT_STOP_CONVERGED;
    else if (p.max_iterations == 0) stop[c] = PT_STOP_MAX_ITERATIONS;
  }
  if (poisoned) {  // u = fma(NaN, 0, u) = NaN at interior cells of those channels
    cudaMemcpyAsync(scale, hscale.data(), C * 8, cudaMemcpyHostToDevice, m.st);
    cudaMemsetAsync(x, 0, NC * 4, m.st);
    k_mg_update<<<g0, kBlock2, 0, m.st>>>(W, H, act0, x, scale, u);
    ++m.launches;
    std::fill(hscale.begin(), hscale.end(), 0.0);
  }
  const float d0 = m.lv[0].d;
  // One CG iteration: V-cycle z = M r, rho = r.z, p = z + beta p, q = A p,
  // alpha = rho / p.q, x += alpha p, r -= alpha q, ||r||^2 (to `red`). Its
  // launches depend only on the problem's shape and the arena, so they are
  // captured once into two CUDA graphs (first iteration, later ones) cached on
  // the context and replayed while shape and arena stay the same.
  long long per_iteration = 0;
  auto enqueue_iteration = [&](bool first) -> cudaError_t {
    const long long l0 = m.launches;
    vcycle(m, m.r, m.z);
    k_cg_dot<<<g0, kBlock2, 0, m.st>>>(W, H, r, z, part);
    k_mg_reduce<<<C, kThreads, 0, m.st>>>(part, m.nb, sc + S_RHO_NEW, S_N);
    k_cg_direction<<<g0, kBlock2, 0, m.st>>>(W, H, z, pp, sc, first ? 1 : 0);
    k_cg_scalars_after_dir<<<1, 32, 0, m.st>>>(C, sc);
    k_cg_apply<<<g0, kBlock2, 0, m.st>>>(W, H, act0, pp, d0, q, part);
    k_mg_reduce<<<C, kThreads, 0, m.st>>>(part, m.nb, sc + S_PQ, S_N);
    k_cg_step<<<g0, kBlock2, 0, m.st>>>(W, H, pp, q, x, r, sc, part);
    k_mg_reduce<<<C, kThreads, 0, m.st>>>(part, m.nb, red, 1);
    m.launches += 8;
    per_iteration = m.launches - l0;
    return cudaGetLastError();
  };
  if (ctx->graphs) {
    std::string key(reinterpret_cast<const char *>(&m.base), sizeof(m.base));
    const double shape[6] = {(double)W, (double)H, (double)C, p.lambda, (double)m.nb, (double)o};
    key.append(reinterpret_cast<const char *>(shape), sizeof(shape));
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
      ctx->mgkey = key;
    }
  }
  int outer = 0;
  while (std::any_of(stop.begin(), stop.end(), [](int s) { return s < 0; })) {
    // scale this outer step's residual to unit norm; channels that stopped get 0
    for (int c = 0; c < C; ++c) {
      hscale[c] = stop[c] < 0 ? cur[c] : 0.0;
      hsc[c * S_N + S_RUN] = stop[c] < 0 ? 1.0 : 0.0;
    }
    cudaMemcpyAsync(scale, hscale.data(), C * 8, cudaMemcpyHostToDevice, m.st);
    cudaMemcpyAsync(sc, hsc.data(), C * S_N * 8, cudaMemcpyHostToDevice, m.st);
    k_mg_scale<<<g0, kBlock2, 0, m.st>>>(W, H, r64, scale, r);
    cudaMemsetAsync(x, 0, NC * 4, m.st);
    m.launches += 1;
    // inner target: a quarter of the remaining bar, at most as deep as FP32
    // goes from a unit residual; a run whose residual stops falling (less than
    // 30% over 4 iterations: the FP32 floor) hands over to the next outer step
    std::vector<double> target(C), rel(C, 1.0);
    std::vector<std::vector<double>> seen(C);
    std::vector<int> run(C);
    for (int c = 0; c < C; ++c) {
      run[c] = stop[c] < 0;
      target[c] = run[c] ? std::max(0.25 * p.tolerance * r0[c] / cur[c], kInnerFloor) : 1.0;
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
      ce = cudaMemcpyAsync(rr.data(), red, C * 8, cudaMemcpyDeviceToHost, m.st);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(m.st);
      if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("cg: ") + cudaGetErrorString(ce));
      bool any = false;
      for (int c = 0; c < C; ++c) {
        if (!run[c]) continue;
        its[c] += 1;
        rel[c] = std::sqrt(rr[c]);  // relative to this outer step's unit residual
        hist[c].push_back(rel[c] * cur[c] / r0[c]);
        seen[c].push_back(rel[c]);
        const size_t n = seen[c].size();
        const bool stuck = n > 4 && seen[c][n - 1] > 0.7 * seen[c][n - 5];
        if (rel[c] <= target[c] || stuck || its[c] >= (int)p.max_iterations || !std::isfinite(rel[c])) {
          run[c] = 0;
          hsc[c * S_N + S_RUN] = 0.0;
          cudaMemcpyAsync(sc + c * S_N + S_RUN, &hsc[c * S_N + S_RUN], 8, cudaMemcpyHostToDevice, m.st);
        }
        any |= run[c] != 0;
      }
      if (!any) break;
    }
    // u += scale * x, then the FP64 residual decides
    k_mg_update<<<g0, kBlock2, 0, m.st>>>(W, H, act0, x, scale, u);
    ++m.launches;
    const std::vector<double> prev = cur;
    ce = residual(u);
    if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("residual: ") + cudaGetErrorString(ce));
    for (int c = 0; c < C; ++c) {
      if (stop[c] >= 0) continue;
      cur[c] = nrm[c];
      if (!hist[c].empty()) hist[c].back() = cur[c] / r0[c];
      if (outer > 0) refines[c] += 1;
      if (cur[c] <= p.tolerance * r0[c]) stop[c] = PT_STOP_CONVERGED;
      else if (its[c] >= (int)p.max_iterations) stop[c] = PT_STOP_MAX_ITERATIONS;
      else if (!(cur[c] < prev[c] * (1.0 - 1e-12))) stop[c] = PT_STOP_STALLED;
    }
    ++outer;
  }
  cudaEventRecord(ctx->ev[2], m.st);
  k_mg_emit<<<gall, kThreads, 0, m.st>>>(W, H, C, act0, u, anc, out);
  ++m.launches;
  if (!dev) ce = cudaMemcpyAsync(out_candidate, out, NC * 4, cudaMemcpyDeviceToHost, m.st);
  if (ce == cudaSuccess && history)
    for (int c = 0; c < C; ++c) {
      const size_t n = std::min<size_t>(hist[c].size(), p.max_iterations);
      if (!n) continue;
      ce = cudaMemcpyAsync(history + (size_t)c * p.max_iterations, hist[c].data(), n * 8,
                           dev ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost, m.st);
      if (ce != cudaSuccess) break;
    }
  if (ce == cudaSuccess) ce = cudaEventRecord(ctx->ev[3], m.st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(m.st);
  if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("result download: ") + cudaGetErrorString(ce));
  {
    float a = 0.f, b = 0.f;
    if (cudaEventElapsedTime(&a, ctx->ev[1], ctx->ev[2]) != cudaSuccess) a = -1.f;
    if (cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[3]) != cudaSuccess) b = -1.f;
    cudaGetLastError();
    ctx->last_solve_ms = a;
    ctx->last_call_ms = b;
    ctx->last_launches = m.launches;
  }
  int worst = -1;
  for (int c = 0; c < C; ++c) {
    pt_report rep{};
    rep.iterations = (uint32_t)its[c];
    rep.stop_reason = stop[c];
    rep.converged = stop[c] == PT_STOP_CONVERGED;
    rep.tolerance = p.tolerance;
    rep.final_residual = r0[c] == 0.0 ? cur[c] : cur[c] / r0[c];
    rep.history_len = (uint32_t)std::min<size_t>(hist[c].size(), p.max_iterations);
    rep.omega_used = kSmoothOmega;
    rep.refinements = (uint32_t)refines[c];
    rep.channel = c;
    rep.initial_residual = r0[c];
    rep.warm_start = warm_used[c];
    reports[c] = rep;
    // worse_of (poisson_blend.rs:240-246)
    if (worst < 0) worst = c;
    else {
      const pt_report &a = reports[worst];
      const bool b_worse = (rep.iterations != a.iterations) ? (rep.iterations > a.iterations)
                                                            : (rep.final_residual > a.final_residual);
      if (b_worse) worst = c;
    }
  }
  reports[C] = reports[worst];
  return PT_OK;
}
