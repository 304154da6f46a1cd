/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 "tight" oracle: a different method (conjugate gradients) on the same
 * discrete system the reference solver relaxes, driven to a relative residual
 * far below anything the op is asked for (1e-12 by default). It is the yardstick
 * for the error of the red-black GPU solution and of the lexicographic CPU
 * solution against the exact discrete fixed point.
 *
 * The system (crates/paintop-cpu/src/poisson.rs:305-325, residual_l2): at every
 * interior cell
 *     nsum(u) - (4 + lambda) u - (b - lambda * anchor) = 0,
 * boundary cells pinned to the anchor. Moving the boundary neighbours to the
 * right-hand side gives the SPD system A u = f with
 *     A = (4 + lambda) I - N_interior,  f = lambda*anchor - b + sum_bnd anchor,
 * whose residual f - A u equals the reference residual r(u). Jacobi
 * preconditioning of A is a constant scaling (its diagonal is 4 + lambda), so
 * the preconditioned iteration is plain CG. The relative residual is
 * normalised, as in the reference (poisson.rs:170-172,206), by the residual of
 * the anchor image.
 *
 * Parallel with OpenMP over fixed row chunks; every dot product is summed per
 * chunk and then in chunk order, so the result does not depend on the thread
 * count.
 */
#include "poisson_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NCHUNK 64

typedef struct {
  size_t w, h;
  const uint8_t *cells;
  double lambda;
} cg_grid;

static void chunk_rows(size_t h, int k, size_t *r0, size_t *r1) {
  *r0 = (h * (size_t)k) / NCHUNK;
  *r1 = (h * (size_t)(k + 1)) / NCHUNK;
}

/* q = A p over interior cells (p is zero on boundary cells). */
static void apply_a(const cg_grid *g, const double *p, double *q) {
  const double d = 4.0 + g->lambda;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk_rows(g->h, k, &r0, &r1);
    for (size_t row = r0; row < r1; ++row)
      for (size_t col = 0; col < g->w; ++col) {
        const size_t i = row * g->w + col;
        if (g->cells[i] != PR_INTERIOR) { q[i] = 0.0; continue; }
        /* interior cells are never on the border: all four neighbours exist */
        const double nsum = p[i - 1] + p[i + 1] + p[i - g->w] + p[i + g->w];
        q[i] = d * p[i] - nsum;
      }
  }
}

/* r = reference residual of the full field u (boundary cells hold the anchor). */
static void true_residual(const cg_grid *g, const double *u, const double *rhs,
                          const double *anchor, double *r) {
  const double d = 4.0 + g->lambda;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk_rows(g->h, k, &r0, &r1);
    for (size_t row = r0; row < r1; ++row)
      for (size_t col = 0; col < g->w; ++col) {
        const size_t i = row * g->w + col;
        if (g->cells[i] != PR_INTERIOR) { r[i] = 0.0; continue; }
        const double nsum = u[i - 1] + u[i + 1] + u[i - g->w] + u[i + g->w];
        r[i] = nsum - d * u[i] - (rhs[i] - g->lambda * anchor[i]);
      }
  }
}

static double dot(const cg_grid *g, const double *a, const double *b) {
  double part[NCHUNK];
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk_rows(g->h, k, &r0, &r1);
    double s = 0.0;
    for (size_t i = r0 * g->w; i < r1 * g->w; ++i) s += a[i] * b[i];
    part[k] = s;
  }
  double s = 0.0;
  for (int k = 0; k < NCHUNK; ++k) s += part[k];
  return s;
}

int pr_cg_solve(const pr_system *s, double rel_tol, uint32_t max_iterations, double *field,
                double *achieved) {
  const size_t n = s->width * s->height;
  const cg_grid g = {s->width, s->height, s->cells, s->lambda};
  memcpy(field, s->anchor, n * sizeof(double));
  if (s->width < 3 || s->height < 3) { if (achieved) *achieved = 0.0; return 0; }
  double *r = (double *)calloc(n, sizeof(double));
  double *p = (double *)calloc(n, sizeof(double));
  double *q = (double *)calloc(n, sizeof(double));
  if (!r || !p || !q) { free(r); free(p); free(q); return -1; }
  true_residual(&g, field, s->rhs, s->anchor, r);
  double rr = dot(&g, r, r);
  const double r0 = sqrt(rr);
  if (r0 == 0.0) { if (achieved) *achieved = 0.0; free(r); free(p); free(q); return 0; }
  memcpy(p, r, n * sizeof(double));
  uint32_t it = 0;
  int done = 0;
  while (!done && it < max_iterations) {
    apply_a(&g, p, q);
    const double pq = dot(&g, p, q);
    if (!(pq > 0.0)) break;
    const double alpha = rr / pq;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) {
      field[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    ++it;
    if (it % 64 == 0) true_residual(&g, field, s->rhs, s->anchor, r);
    const double rr_new = dot(&g, r, r);
    if (sqrt(rr_new) <= rel_tol * r0) {
      /* confirm on the true residual before stopping */
      true_residual(&g, field, s->rhs, s->anchor, r);
      const double rt = dot(&g, r, r);
      if (sqrt(rt) <= rel_tol * r0) { rr = rt; done = 1; break; }
      memcpy(p, r, n * sizeof(double)); /* restart from the true residual */
      rr = rt;
      continue;
    }
    const double beta = rr_new / rr;
    rr = rr_new;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) p[i] = r[i] + beta * p[i];
  }
  true_residual(&g, field, s->rhs, s->anchor, r);
  if (achieved) *achieved = sqrt(dot(&g, r, r)) / r0;
  free(r); free(p); free(q);
  return (int)it;
}

int pr_cg_blend_channels(const float *source, const float *target, const float *mask,
                         size_t channels, size_t width, size_t height, double lambda,
                         double rel_tol, uint32_t max_iterations, double *out_f64,
                         double *achieved) {
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
  int iters = 0;
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
    double ach = 0.0;
    const int it = pr_cg_solve(&sys, rel_tol, max_iterations, field, &ach);
    if (it < 0) { iters = -1; break; }
    iters += it;
    if (achieved) achieved[ch] = ach;
    for (size_t p = 0; p < count; ++p) out_f64[p * channels + ch] = field[p];
  }
  free(cells); free(src); free(anchor); free(rhs); free(field);
  return iters;
}
