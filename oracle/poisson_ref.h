/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY. CPU restatement of paintop's Poisson
 * solver (crates/paintop-cpu/src/poisson.rs, poisson_blend.rs) and an FP64 CG
 * tight oracle on the same system. Not part of the product library.
 */
#ifndef PAINTOP_ORACLE_POISSON_REF_H
#define PAINTOP_ORACLE_POISSON_REF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { PR_BOUNDARY = 0, PR_INTERIOR = 1 };
/* SolverStopReason (crates/paintop-ir/src/resource.rs:1185-1194) */
enum { PR_CONVERGED = 0, PR_MAX_ITERATIONS = 1, PR_STALLED = 2 };

#define PR_MASK_THRESHOLD 0.5f

/* PoissonSystem (poisson.rs:105-121); all buffers row-major width*height. */
typedef struct {
  size_t width, height;
  const uint8_t *cells;
  const double *rhs;
  const double *anchor;
  double lambda;
} pr_system;

/* SolveControls (poisson.rs:145-154) */
typedef struct {
  uint32_t max_iterations;
  double tolerance;
  double omega;
} pr_controls;

/* SolveReport without the history vector (poisson.rs:126-141) */
typedef struct {
  uint32_t iterations;
  int32_t converged;
  int32_t stop_reason;
  double tolerance;
  double final_residual;
} pr_report;

void pr_classify_cells(const float *mask, size_t width, size_t height, uint8_t *cells);
double pr_guidance_laplacian(const double *field, size_t col, size_t row, size_t width,
                             size_t height);
double pr_residual_l2(const pr_system *s, const double *field);
/* field: width*height out; history: capacity max_iterations (may be NULL). */
void pr_solve(const pr_system *s, pr_controls c, double *field, double *history,
              pr_report *rep);
int pr_worse(const pr_report *a, const pr_report *b);
/* histories: channels * max_iterations (may be NULL). Returns 0 or -1 (OOM). */
int pr_blend_channels(const float *source, const float *target, const float *mask,
                      size_t channels, size_t width, size_t height, pr_controls c,
                      double lambda, float *out, pr_report *per_channel,
                      double *histories, int *worst_channel);

/* FP64 CG to ||r|| <= rel_tol * ||r(anchor)||. Returns iterations or -1. */
int pr_cg_solve(const pr_system *s, double rel_tol, uint32_t max_iterations, double *field,
                double *achieved);
int pr_cg_blend_channels(const float *source, const float *target, const float *mask,
                         size_t channels, size_t width, size_t height, double lambda,
                         double rel_tol, uint32_t max_iterations, double *out_f64,
                         double *achieved);

/* FP64 CG preconditioned by an aggregation multigrid V-cycle, to
 * ||r|| <= rel_tol * ||r(anchor)||; initial (nullable) seeds the interior.
 * Returns iterations or -1 (OOM). */
int pr_mgcg_solve(const pr_system *s, double rel_tol, uint32_t max_iterations,
                  const double *initial, double *field, double *achieved);
int pr_mgcg_blend_channels(const float *source, const float *target, const float *mask,
                           size_t channels, size_t width, size_t height, double lambda,
                           double rel_tol, uint32_t max_iterations, double *out_f64,
                           double *achieved, uint32_t *iterations);

/* FP64 red-black SOR (the GPU method in FP64): same controls and report. */
void pr_rb_solve(const pr_system *s, pr_controls c, double *field, double *history,
                 pr_report *rep);
int pr_rb_blend_channels(const float *source, const float *target, const float *mask,
                         size_t channels, size_t width, size_t height, pr_controls c,
                         double lambda, double *out_f64, pr_report *per_channel,
                         double *histories);

#ifdef __cplusplus
}
#endif
#endif
