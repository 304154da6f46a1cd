/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 tight oracle for large systems: conjugate gradients preconditioned by an
 * algebraic multigrid V-cycle, on the same discrete system the reference solver
 * relaxes (crates/paintop-cpu/src/poisson.rs:305-325, residual_l2):
 *     nsum(u) - (4 + lambda) u - (b - lambda * anchor) = 0   at interior cells,
 * boundary cells pinned to the anchor (classification poisson.rs:340-355). As in
 * cg_ref.c the boundary neighbours move to the right-hand side, giving the SPD
 * system A u = f with A = (4 + lambda) I - N_interior, whose residual f - A u is
 * the reference residual r(u). The stop test is the reference's relative
 * residual ||r(u)|| / ||r(anchor)|| (poisson.rs:170-172,206), evaluated on the
 * true FP64 residual of the iterate.
 *
 * Plain CG needs O(diameter) iterations per decade of residual: about 10^4 to
 * reach 1e-12 on a 1300-pixel region. This oracle reaches the same tolerance
 * in a few dozen iterations, which makes FP64 reference solutions of the
 * 2048x2048 and 4096x4096 workloads affordable on the host cores. The method
 * does not matter for the oracle's use; the certified FP64 residual does.
 *
 * Preconditioner (a symmetric positive definite V-cycle):
 *  - coarsening: 2x2 aggregation. Coarse cell (X, Y) gathers fine cells
 *    (2X..2X+1, 2Y..2Y+1); the prolongation P is piecewise constant and the
 *    coarse operator is the Galerkin product P^T A P. For a 5-point operator it
 *    is again 5-point: the diagonal sums the block's diagonals plus twice its
 *    internal couplings, and the coupling to the east (south) neighbour sums
 *    the two fine couplings that cross the block edge. Every level is therefore
 *    exact algebra on the level below: SPD, with no geometric assumptions about
 *    the mask.
 *  - smoothing: red-black Gauss-Seidel, NU sweeps red-then-black before the
 *    coarse correction and NU sweeps black-then-red after it, so the
 *    post-smoother is the adjoint of the pre-smoother.
 *  - the coarse correction is scaled by ALPHA (over-correction compensates the
 *    low energy of a piecewise-constant interpolant); for 0 < ALPHA < 2 the
 *    two-grid operator stays an A-norm contraction, so the V-cycle stays SPD.
 *  - the coarsest level (at most COARSE_CELLS cells per side) gets
 *    COARSE_SWEEPS symmetric sweeps.
 *
 * Every pass is parallel over fixed row chunks (OpenMP); red-black updates do
 * not depend on the order of cells within a colour and every dot product is
 * summed per chunk and then in chunk order, so results do not depend on the
 * thread count.
 */
#include "poisson_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NCHUNK 256
#define MAX_LEVELS 24
#define NU 2
#define ALPHA 1.8
#define COARSE_CELLS 8
#define COARSE_SWEEPS 64

typedef struct {
  size_t w, h, n;
  double *d, *e, *s; /* diagonal; coupling to (x+1, y); coupling to (x, y+1) */
  double *x, *b, *r; /* level solution, right-hand side, residual */
} level_t;

typedef struct {
  int nlev;
  level_t L[MAX_LEVELS];
} hier_t;

static void chunk(size_t h, int k, size_t *r0, size_t *r1) {
  *r0 = (h * (size_t)k) / NCHUNK;
  *r1 = (h * (size_t)(k + 1)) / NCHUNK;
}

static void free_hier(hier_t *H) {
  for (int l = 0; l < H->nlev; ++l) {
    level_t *L = &H->L[l];
    free(L->d); free(L->e); free(L->s); free(L->x); free(L->b); free(L->r);
  }
  H->nlev = 0;
}

static int alloc_level(level_t *L, size_t w, size_t h) {
  L->w = w; L->h = h; L->n = w * h;
  const size_t n = L->n ? L->n : 1;
  L->d = (double *)calloc(n, sizeof(double));
  L->e = (double *)calloc(n, sizeof(double));
  L->s = (double *)calloc(n, sizeof(double));
  L->x = (double *)calloc(n, sizeof(double));
  L->b = (double *)calloc(n, sizeof(double));
  L->r = (double *)calloc(n, sizeof(double));
  return (L->d && L->e && L->s && L->x && L->b && L->r) ? 0 : -1;
}

/* Level 0: A = (4 + lambda) I - N over interior cells. */
static void fine_operator(level_t *L, const uint8_t *cells, double lambda) {
  const size_t w = L->w, h = L->h;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk(h, k, &r0, &r1);
    for (size_t y = r0; y < r1; ++y)
      for (size_t x = 0; x < w; ++x) {
        const size_t i = y * w + x;
        const int in = cells[i] == PR_INTERIOR;
        L->d[i] = in ? 4.0 + lambda : 0.0;
        L->e[i] = (in && x + 1 < w && cells[i + 1] == PR_INTERIOR) ? -1.0 : 0.0;
        L->s[i] = (in && y + 1 < h && cells[i + w] == PR_INTERIOR) ? -1.0 : 0.0;
      }
  }
}

/* Galerkin P^T A P for 2x2 piecewise-constant aggregation. */
static void coarse_operator(const level_t *F, level_t *Cc) {
  const size_t fw = F->w, fh = F->h, cw = Cc->w, ch = Cc->h;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk(ch, k, &r0, &r1);
    for (size_t Y = r0; Y < r1; ++Y)
      for (size_t X = 0; X < cw; ++X) {
        double D = 0.0, E = 0.0, S = 0.0;
        for (size_t dy = 0; dy < 2; ++dy)
          for (size_t dx = 0; dx < 2; ++dx) {
            const size_t x = 2 * X + dx, y = 2 * Y + dy;
            if (x >= fw || y >= fh) continue;
            const size_t i = y * fw + x;
            D += F->d[i];
            /* horizontal coupling from (x, y) to (x+1, y) */
            if (dx == 0) D += 2.0 * F->e[i];
            else E += F->e[i];
            /* vertical coupling from (x, y) to (x, y+1) */
            if (dy == 0) D += 2.0 * F->s[i];
            else S += F->s[i];
          }
        const size_t I = Y * cw + X;
        Cc->d[I] = D;
        Cc->e[I] = (X + 1 < cw) ? E : 0.0;
        Cc->s[I] = (Y + 1 < ch) ? S : 0.0;
      }
  }
}

static int build_hier(hier_t *H, size_t w, size_t h, const uint8_t *cells, double lambda) {
  memset(H, 0, sizeof(*H));
  if (alloc_level(&H->L[0], w, h)) return -1;
  H->nlev = 1;
  fine_operator(&H->L[0], cells, lambda);
  while (H->nlev < MAX_LEVELS) {
    const level_t *F = &H->L[H->nlev - 1];
    if (F->w <= COARSE_CELLS && F->h <= COARSE_CELLS) break;
    level_t *Cc = &H->L[H->nlev];
    if (alloc_level(Cc, (F->w + 1) / 2, (F->h + 1) / 2)) return -1;
    H->nlev++;
    coarse_operator(F, Cc);
  }
  return 0;
}

/* One red-black half-sweep of colour c: x_i = (b_i - sum_j a_ij x_j) / a_ii. */
static void gs_colour(level_t *L, int c) {
  const size_t w = L->w, h = L->h;
  const double *d = L->d, *e = L->e, *s = L->s, *b = L->b;
  double *x = L->x;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk(h, k, &r0, &r1);
    for (size_t y = r0; y < r1; ++y)
      for (size_t xx = (y + (size_t)c) & 1; xx < w; xx += 2) {
        const size_t i = y * w + xx;
        if (!(d[i] > 0.0)) continue;
        double off = 0.0;
        if (xx > 0) off += e[i - 1] * x[i - 1];
        if (xx + 1 < w) off += e[i] * x[i + 1];
        if (y > 0) off += s[i - w] * x[i - w];
        if (y + 1 < h) off += s[i] * x[i + w];
        x[i] = (b[i] - off) / d[i];
      }
  }
}

/* r = b - A x on one level. */
static void level_residual(level_t *L) {
  const size_t w = L->w, h = L->h;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk(h, k, &r0, &r1);
    for (size_t y = r0; y < r1; ++y)
      for (size_t xx = 0; xx < w; ++xx) {
        const size_t i = y * w + xx;
        if (!(L->d[i] > 0.0)) { L->r[i] = 0.0; continue; }
        double ax = L->d[i] * L->x[i];
        if (xx > 0) ax += L->e[i - 1] * L->x[i - 1];
        if (xx + 1 < w) ax += L->e[i] * L->x[i + 1];
        if (y > 0) ax += L->s[i - w] * L->x[i - w];
        if (y + 1 < h) ax += L->s[i] * L->x[i + w];
        L->r[i] = L->b[i] - ax;
      }
  }
}

/* b_coarse = P^T r_fine (sum over the 2x2 block). */
static void restrict_res(const level_t *F, level_t *Cc) {
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk(Cc->h, k, &r0, &r1);
    for (size_t Y = r0; Y < r1; ++Y)
      for (size_t X = 0; X < Cc->w; ++X) {
        double v = 0.0;
        for (size_t dy = 0; dy < 2; ++dy)
          for (size_t dx = 0; dx < 2; ++dx) {
            const size_t x = 2 * X + dx, y = 2 * Y + dy;
            if (x < F->w && y < F->h) v += F->r[y * F->w + x];
          }
        const size_t I = Y * Cc->w + X;
        Cc->b[I] = Cc->d[I] > 0.0 ? v : 0.0;
      }
  }
}

/* x_fine += ALPHA * P x_coarse on active fine cells. */
static void prolong_add(level_t *F, const level_t *Cc) {
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk(F->h, k, &r0, &r1);
    for (size_t y = r0; y < r1; ++y)
      for (size_t x = 0; x < F->w; ++x) {
        const size_t i = y * F->w + x;
        if (F->d[i] > 0.0) F->x[i] += ALPHA * Cc->x[(y / 2) * Cc->w + x / 2];
      }
  }
}

static void vcycle(hier_t *H, int l) {
  level_t *L = &H->L[l];
  memset(L->x, 0, L->n * sizeof(double));
  if (l == H->nlev - 1) {
    for (int k = 0; k < COARSE_SWEEPS; ++k) { gs_colour(L, 0); gs_colour(L, 1); }
    for (int k = 0; k < COARSE_SWEEPS; ++k) { gs_colour(L, 1); gs_colour(L, 0); }
    return;
  }
  for (int k = 0; k < NU; ++k) { gs_colour(L, 0); gs_colour(L, 1); }
  level_residual(L);
  restrict_res(L, &H->L[l + 1]);
  vcycle(H, l + 1);
  prolong_add(L, &H->L[l + 1]);
  for (int k = 0; k < NU; ++k) { gs_colour(L, 1); gs_colour(L, 0); }
}

/* reference residual of the full field u (boundary cells hold the anchor) */
static void true_residual(const pr_system *s, const double *u, double *r) {
  const size_t w = s->width, h = s->height;
  const double dg = 4.0 + s->lambda;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk(h, k, &r0, &r1);
    for (size_t y = r0; y < r1; ++y)
      for (size_t x = 0; x < w; ++x) {
        const size_t i = y * w + x;
        if (s->cells[i] != PR_INTERIOR) { r[i] = 0.0; continue; }
        const double nsum = u[i - 1] + u[i + 1] + u[i - w] + u[i + w];
        r[i] = nsum - dg * u[i] - (s->rhs[i] - s->lambda * s->anchor[i]);
      }
  }
}

static double dotv(size_t w, size_t h, const double *a, const double *b) {
  double part[NCHUNK];
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk(h, k, &r0, &r1);
    double acc = 0.0;
    for (size_t i = r0 * w; i < r1 * w; ++i) acc += a[i] * b[i];
    part[k] = acc;
  }
  double acc = 0.0;
  for (int k = 0; k < NCHUNK; ++k) acc += part[k];
  return acc;
}

/* q = A p at interior cells (p is zero elsewhere) */
static void apply_fine(const level_t *L, const double *p, double *q) {
  const size_t w = L->w, h = L->h;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < NCHUNK; ++k) {
    size_t r0, r1;
    chunk(h, k, &r0, &r1);
    for (size_t y = r0; y < r1; ++y)
      for (size_t x = 0; x < w; ++x) {
        const size_t i = y * w + x;
        if (!(L->d[i] > 0.0)) { q[i] = 0.0; continue; }
        q[i] = L->d[i] * p[i] + L->e[i - 1] * p[i - 1] + L->e[i] * p[i + 1] +
               L->s[i - w] * p[i - w] + L->s[i] * p[i + w];
      }
  }
}

int pr_mgcg_solve(const pr_system *s, double rel_tol, uint32_t max_iterations,
                  const double *initial, double *field, double *achieved) {
  const size_t w = s->width, h = s->height, n = w * h;
  memcpy(field, s->anchor, n * sizeof(double));
  if (initial)
    for (size_t i = 0; i < n; ++i)
      if (s->cells[i] == PR_INTERIOR) field[i] = initial[i];
  if (achieved) *achieved = 0.0;
  if (w < 3 || h < 3) return 0;
  double *r = (double *)calloc(n, sizeof(double));
  double *p = (double *)calloc(n, sizeof(double));
  double *q = (double *)calloc(n, sizeof(double));
  double *r_anchor = (double *)calloc(n, sizeof(double));
  hier_t H;
  if (!r || !p || !q || !r_anchor || build_hier(&H, w, h, s->cells, s->lambda)) {
    free(r); free(p); free(q); free(r_anchor);
    free_hier(&H);
    return -1;
  }
  level_t *L0 = &H.L[0];
  true_residual(s, s->anchor, r_anchor);
  const double r0 = sqrt(dotv(w, h, r_anchor, r_anchor));
  free(r_anchor);
  int it = 0;
  if (r0 == 0.0 || !isfinite(r0)) goto done;
  true_residual(s, field, r);
  if (sqrt(dotv(w, h, r, r)) <= rel_tol * r0) goto done;
  for (;;) { /* restart loop: each pass starts from the true residual */
    memcpy(L0->b, r, n * sizeof(double));
    vcycle(&H, 0);
    memcpy(p, L0->x, n * sizeof(double));
    double rz = dotv(w, h, r, L0->x);
    int restart = 0;
    while ((uint32_t)it < max_iterations) {
      apply_fine(L0, p, q);
      const double pq = dotv(w, h, p, q);
      if (!(pq > 0.0)) { restart = 0; break; }
      const double a = rz / pq;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < (long)n; ++i) {
        field[i] += a * p[i];
        r[i] -= a * q[i];
      }
      ++it;
      if (sqrt(dotv(w, h, r, r)) <= rel_tol * r0) {
        true_residual(s, field, r);
        restart = !(sqrt(dotv(w, h, r, r)) <= rel_tol * r0);
        break;
      }
      memcpy(L0->b, r, n * sizeof(double));
      vcycle(&H, 0);
      const double rz_new = dotv(w, h, r, L0->x);
      const double beta = rz_new / rz;
      rz = rz_new;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < (long)n; ++i) p[i] = L0->x[i] + beta * p[i];
    }
    if (!restart || (uint32_t)it >= max_iterations) break;
  }
done:
  true_residual(s, field, r);
  if (achieved) *achieved = r0 > 0.0 ? sqrt(dotv(w, h, r, r)) / r0 : 0.0;
  free(r); free(p); free(q);
  free_hier(&H);
  return it;
}

int pr_mgcg_blend_channels(const float *source, const float *target, const float *mask,
                           size_t channels, size_t width, size_t height, double lambda,
                           double rel_tol, uint32_t max_iterations, double *out_f64,
                           double *achieved, uint32_t *iterations) {
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
  int rc = 0;
  for (size_t ch = 0; ch < channels; ++ch) {
    for (size_t p = 0; p < count; ++p) {
      src[p] = (double)source[p * channels + ch];
      anchor[p] = (double)target[p * channels + ch];
      rhs[p] = 0.0;
    }
#pragma omp parallel for schedule(static)
    for (long row = 0; row < (long)height; ++row)
      for (size_t col = 0; col < width; ++col) {
        const size_t idx = (size_t)row * width + col;
        if (cells[idx] == PR_INTERIOR)
          rhs[idx] = pr_guidance_laplacian(src, col, (size_t)row, width, height);
      }
    const pr_system sys = {width, height, cells, rhs, anchor, lambda};
    double ach = 0.0;
    const int it = pr_mgcg_solve(&sys, rel_tol, max_iterations, NULL, field, &ach);
    if (it < 0) { rc = -1; break; }
    if (achieved) achieved[ch] = ach;
    if (iterations) iterations[ch] = (uint32_t)it;
    for (size_t p = 0; p < count; ++p) out_f64[p * channels + ch] = field[p];
  }
  free(cells); free(src); free(anchor); free(rhs); free(field);
  return rc;
}
