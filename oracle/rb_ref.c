/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 red-black SOR: the GPU backend's method restated on the CPU in FP64,
 * so the GPU's iteration counts and residual histories (FP32 sweeps with FP64
 * residuals and FP64 residual correction) can be checked against the same
 * ordering computed entirely in FP64. The per-cell update, the residual, the
 * relative-residual normalisation, the tolerance test and the stall rule are
 * the reference's (crates/paintop-cpu/src/poisson.rs:167-325); only the visiting
 * order differs from poisson.rs:244-265: all cells with (x + y) even ("red")
 * first, then all cells with (x + y) odd. Within a colour no cell reads another
 * cell of its colour, so the order inside a colour does not matter.
 */
#include "poisson_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CENTRE_WEIGHT 4.0
#define STALL_WINDOW 16u
#define STALL_IMPROVEMENT 1e-12

static inline double nsum_at(const double *f, size_t col, size_t row, size_t w, size_t h) {
  const double c = f[row * w + col];
  const double l = (col == 0) ? c : f[row * w + col - 1];
  const double r = (col + 1 == w) ? c : f[row * w + col + 1];
  const double u = (row == 0) ? c : f[(row - 1) * w + col];
  const double d = (row + 1 == h) ? c : f[(row + 1) * w + col];
  return l + r + u + d;
}

static void half_sweep(const pr_system *s, double *field, double denom, double omega, int colour) {
  for (size_t row = 0; row < s->height; ++row) {
    size_t col0 = ((size_t)colour + row) & 1u;
    for (size_t col = col0; col < s->width; col += 2) {
      const size_t idx = row * s->width + col;
      if (s->cells[idx] != PR_INTERIOR) continue;
      const double ns = nsum_at(field, col, row, s->width, s->height);
      const double target = fma(s->lambda, s->anchor[idx], ns - s->rhs[idx]) / denom;
      field[idx] = fma(omega, target - field[idx], field[idx]);
    }
  }
}

void pr_rb_solve(const pr_system *s, pr_controls c, double *field, double *history,
                 pr_report *rep) {
  const size_t count = s->width * s->height;
  memcpy(field, s->anchor, count * sizeof(double));
  const double r0 = pr_residual_l2(s, field);
  rep->tolerance = c.tolerance;
  if (r0 == 0.0) {
    rep->iterations = 0;
    rep->converged = 1;
    rep->stop_reason = PR_CONVERGED;
    rep->final_residual = 0.0;
    return;
  }
  const double denom = CENTRE_WEIGHT + s->lambda;
  int converged = 0, stop_reason = PR_MAX_ITERATIONS;
  double last = 1.0, best = INFINITY;
  uint32_t iterations = 0, since = 0;
  for (uint32_t sweep = 0; sweep < c.max_iterations; ++sweep) {
    half_sweep(s, field, denom, c.omega, 0);
    half_sweep(s, field, denom, c.omega, 1);
    iterations = sweep + 1;
    const double rel = pr_residual_l2(s, field) / r0;
    if (history) history[sweep] = rel;
    last = rel;
    if (rel <= c.tolerance) {
      converged = 1;
      stop_reason = PR_CONVERGED;
      break;
    }
    if (rel < best * (1.0 - STALL_IMPROVEMENT)) {
      best = rel;
      since = 0;
    } else if (++since >= STALL_WINDOW) {
      stop_reason = PR_STALLED;
      break;
    }
  }
  rep->iterations = iterations;
  rep->converged = converged;
  rep->stop_reason = stop_reason;
  rep->final_residual = last;
}

int pr_rb_blend_channels(const float *source, const float *target, const float *mask,
                         size_t channels, size_t width, size_t height, pr_controls c,
                         double lambda, double *out_f64, pr_report *per_channel,
                         double *histories) {
  const size_t count = width * height;
  const size_t n = count ? count : 1;
  uint8_t *cells = (uint8_t *)malloc(n);
  double *src = (double *)malloc(n * sizeof(double));
  double *anchor = (double *)malloc(n * sizeof(double));
  double *rhs = (double *)malloc(n * sizeof(double));
  double *field = (double *)malloc(n * sizeof(double));
  if (!cells || !src || !anchor || !rhs || !field) {
    free(cells); free(src); free(anchor); free(rhs); free(field);
    return -1;
  }
  pr_classify_cells(mask, width, height, cells);
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
    pr_rb_solve(&sys, c, field, histories ? histories + ch * (size_t)c.max_iterations : NULL,
                &per_channel[ch]);
    for (size_t p = 0; p < count; ++p) out_f64[p * channels + ch] = field[p];
  }
  free(cells); free(src); free(anchor); free(rhs); free(field);
  return 0;
}
