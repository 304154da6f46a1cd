/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of paintop's CPU Poisson / screened-Poisson solver
 * (the `cpu.reference@1` implementation of `repair.poisson_blend@1` and
 * `repair.screened_poisson@1`). Only the tests, the smoke check and the CPU
 * baseline leg of the benchmark may load this code, and only as the checker or
 * the timed CPU baseline; the product path (the CUDA library) never calls it.
 *
 * Provenance (reference paths are relative to the paintop source tree):
 *   crates/paintop-cpu/src/poisson.rs:73-85    constants (centre weight 4, stall
 *                                              window 16, stall improvement 1e-12)
 *   crates/paintop-cpu/src/poisson.rs:167-240  solve()
 *   crates/paintop-cpu/src/poisson.rs:244-265  sweep_once()  (row-major SOR)
 *   crates/paintop-cpu/src/poisson.rs:275-298  neighbour_sum() (L+R+U+D, clamp)
 *   crates/paintop-cpu/src/poisson.rs:305-325  residual_l2()
 *   crates/paintop-cpu/src/poisson.rs:329-355  MASK_THRESHOLD, classify_cells()
 *   crates/paintop-cpu/src/poisson.rs:364-373  guidance_laplacian()
 *   crates/paintop-cpu/src/poisson_blend.rs:153-246  channel_f64, blend_channels,
 *                                              worse_of (worst-channel report)
 *
 * Every Rust `a.mul_add(b, c)` is written as `fma(a, b, c)`; the file is built
 * with -ffp-contract=off and without fast-math so that no other contraction or
 * reassociation happens. Loop order, operand order and the f64 -> f32 output
 * cast (round to nearest even) follow the Rust source, so the restatement is
 * bit-faithful on IEEE-754 hardware. The Rust op itself cannot be built here
 * (no Rust toolchain), so bit-identity to it is pinned by (1) an independent
 * pure-Python restatement with exactly-rounded fma that this code must match
 * bit for bit, and (2) every analytic known-answer test of the reference's own
 * suites, ported to pytest.
 */
#include "poisson_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#if defined(__FAST_MATH__)
#error "the oracle must be built without fast-math"
#endif

#define CENTRE_WEIGHT 4.0
#define STALL_WINDOW 16u
#define STALL_IMPROVEMENT 1e-12

/* poisson.rs:275-298 -- out-of-grid neighbours are replaced by the centre. */
static inline double neighbour_sum(const double *field, size_t col, size_t row,
                                   size_t width, size_t height) {
  const double centre = field[row * width + col];
  const double left = (col == 0) ? centre : field[row * width + col - 1];
  const double right = (col + 1 == width) ? centre : field[row * width + col + 1];
  const double up = (row == 0) ? centre : field[(row - 1) * width + col];
  const double down = (row + 1 == height) ? centre : field[(row + 1) * width + col];
  return left + right + up + down;
}

/* poisson.rs:340-355 */
void pr_classify_cells(const float *mask, size_t width, size_t height, uint8_t *cells) {
  memset(cells, PR_BOUNDARY, width * height);
  if (width < 3 || height < 3) return;
  for (size_t row = 1; row < height - 1; ++row)
    for (size_t col = 1; col < width - 1; ++col) {
      const size_t idx = row * width + col;
      if (mask[idx] > PR_MASK_THRESHOLD) cells[idx] = PR_INTERIOR;
    }
}

/* poisson.rs:364-373 */
double pr_guidance_laplacian(const double *field, size_t col, size_t row, size_t width,
                             size_t height) {
  const double centre = field[row * width + col];
  return fma(CENTRE_WEIGHT, -centre, neighbour_sum(field, col, row, width, height));
}

/* poisson.rs:244-265 */
static void sweep_once(const pr_system *s, double *field, double denom, double omega) {
  for (size_t row = 0; row < s->height; ++row)
    for (size_t col = 0; col < s->width; ++col) {
      const size_t idx = row * s->width + col;
      if (s->cells[idx] != PR_INTERIOR) continue;
      const double nsum = neighbour_sum(field, col, row, s->width, s->height);
      const double target = fma(s->lambda, s->anchor[idx], nsum - s->rhs[idx]) / denom;
      field[idx] = fma(omega, target - field[idx], field[idx]);
    }
}

/* poisson.rs:305-325 */
static double residual_l2(const pr_system *s, const double *field) {
  double sum_sq = 0.0;
  for (size_t row = 0; row < s->height; ++row)
    for (size_t col = 0; col < s->width; ++col) {
      const size_t idx = row * s->width + col;
      if (s->cells[idx] != PR_INTERIOR) continue;
      const double nsum = neighbour_sum(field, col, row, s->width, s->height);
      const double lhs = fma(s->lambda + CENTRE_WEIGHT, -field[idx], nsum);
      const double rhs = fma(s->lambda, -s->anchor[idx], s->rhs[idx]);
      const double r = lhs - rhs;
      sum_sq = fma(r, r, sum_sq);
    }
  return sqrt(sum_sq);
}

double pr_residual_l2(const pr_system *s, const double *field) { return residual_l2(s, field); }

/* poisson.rs:167-240 */
void pr_solve(const pr_system *s, pr_controls c, double *field, double *history,
              pr_report *rep) {
  const size_t count = s->width * s->height;
  memcpy(field, s->anchor, count * sizeof(double));
  const double initial_residual = residual_l2(s, field);
  rep->tolerance = c.tolerance;
  if (initial_residual == 0.0) {
    rep->iterations = 0;
    rep->converged = 1;
    rep->stop_reason = PR_CONVERGED;
    rep->final_residual = 0.0;
    return;
  }
  const double denom = CENTRE_WEIGHT + s->lambda;
  int converged = 0;
  int stop_reason = PR_MAX_ITERATIONS;
  double last_relative = 1.0;
  uint32_t iterations = 0;
  double best_relative = INFINITY;
  uint32_t since = 0;
  for (uint32_t sweep = 0; sweep < c.max_iterations; ++sweep) {
    sweep_once(s, field, denom, c.omega);
    iterations = sweep + 1;
    const double relative = residual_l2(s, field) / initial_residual;
    if (history) history[sweep] = relative;
    last_relative = relative;
    if (relative <= c.tolerance) {
      converged = 1;
      stop_reason = PR_CONVERGED;
      break;
    }
    if (relative < best_relative * (1.0 - STALL_IMPROVEMENT)) {
      best_relative = relative;
      since = 0;
    } else {
      since += 1;
      if (since >= STALL_WINDOW) {
        stop_reason = PR_STALLED;
        break;
      }
    }
  }
  rep->iterations = iterations;
  rep->converged = converged;
  rep->stop_reason = stop_reason;
  rep->final_residual = last_relative;
}

/* poisson_blend.rs:240-246: (b.iterations, b.final_residual) > (a.iterations,
 * a.final_residual), lexicographic with IEEE `>` on the f64 (false on NaN). */
int pr_worse(const pr_report *a, const pr_report *b) {
  if (b->iterations != a->iterations) return b->iterations > a->iterations;
  return b->final_residual > a->final_residual;
}

/* poisson_blend.rs:168-236 */
int pr_blend_channels(const float *source, const float *target, const float *mask,
                      size_t channels, size_t width, size_t height, pr_controls c,
                      double lambda, float *out, pr_report *per_channel,
                      double *histories, int *worst_channel) {
  const size_t count = width * height;
  uint8_t *cells = (uint8_t *)malloc(count ? count : 1);
  double *src = (double *)malloc((count ? count : 1) * sizeof(double));
  double *anchor = (double *)malloc((count ? count : 1) * sizeof(double));
  double *rhs = (double *)malloc((count ? count : 1) * sizeof(double));
  double *field = (double *)malloc((count ? count : 1) * sizeof(double));
  if (!cells || !src || !anchor || !rhs || !field) {
    free(cells); free(src); free(anchor); free(rhs); free(field);
    return -1;
  }
  pr_classify_cells(mask, width, height, cells);
  int worst = -1;
  for (size_t ch = 0; ch < channels; ++ch) {
    for (size_t p = 0; p < count; ++p) {
      src[p] = (double)source[p * channels + ch];
      anchor[p] = (double)target[p * channels + ch];
      rhs[p] = 0.0;
    }
    for (size_t row = 0; row < height; ++row)
      for (size_t col = 0; col < width; ++col) {
        const size_t idx = row * width + col;
        if (cells[idx] == PR_INTERIOR)
          rhs[idx] = pr_guidance_laplacian(src, col, row, width, height);
      }
    const pr_system sys = {width, height, cells, rhs, anchor, lambda};
    pr_report rep;
    pr_solve(&sys, c, field, histories ? histories + ch * (size_t)c.max_iterations : NULL,
             &rep);
    for (size_t p = 0; p < count; ++p) out[p * channels + ch] = (float)field[p];
    per_channel[ch] = rep;
    if (worst < 0 || pr_worse(&per_channel[worst], &rep)) worst = (int)ch;
  }
  *worst_channel = worst;
  free(cells); free(src); free(anchor); free(rhs); free(field);
  return 0;
}
