/* mask_ref.c -- TEST INFRASTRUCTURE ONLY: a C restatement of the reference's
 * two mask generators, the checker for the device rasterisers.
 *
 *  or_mask_ellipse  mask.ellipse@1   crates/paintop-cpu/src/ellipse.rs
 *                   coverage (:168-201), feather (:208-218), rasterize (:545-565)
 *  or_mask_polygon  mask.polygon@1   crates/paintop-cpu/src/mask_polygon.rs
 *                   contains (:161-196), rasterize (:259-286), S = 4 (:77)
 *
 * Every `mul_add` of the Rust source is an explicit fma() and the file is built
 * with -ffp-contract=off, so the arithmetic is the Rust source's operation for
 * operation. The ellipse's sin_cos and hypot are libm's, as in the Rust build
 * on Linux. */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

/* ellipse.rs:208-218 */
static double feather(double sd, double half_width_px) {
  if (half_width_px <= 0.0) return sd <= 0.0 ? 1.0 : 0.0;
  double t = (sd + half_width_px) / (2.0 * half_width_px);
  if (t < 0.0) t = 0.0;
  if (t > 1.0) t = 1.0;
  const double smoothstep = t * t * fma(2.0, -t, 3.0);
  return 1.0 - smoothstep;
}

/* ellipse.rs:168-201; sin and cos are taken once by the caller */
static double ellipse_coverage(double cx, double cy, double rx, double ry, double sn, double cs,
                               double half_width_px, double x, double y) {
  const double off_x = x - cx, off_y = y - cy;
  const double local_u = fma(sn, off_y, cs * off_x);
  const double local_v = fma(cs, off_y, -sn * off_x);
  const double norm_x = local_u / rx, norm_y = local_v / ry;
  const double quadratic = fma(norm_x, norm_x, norm_y * norm_y);
  const double f = sqrt(quadratic);
  if (f == 0.0) return 1.0;
  const double grad_x = local_u / (rx * rx);
  const double grad_y = local_v / (ry * ry);
  const double grad = hypot(grad_x, grad_y);
  if (grad == 0.0) return 1.0;
  const double sd = (f - 1.0) * f / grad;
  return feather(sd, half_width_px);
}

void or_mask_ellipse(uint32_t width, uint32_t height, double cx, double cy, double rx, double ry,
                     double angle_rad, double half_width_px, float *out) {
  const double sn = sin(angle_rad), cs = cos(angle_rad);
  for (uint32_t j = 0; j < height; ++j) {
    const double y = (double)j + 0.5;
    for (uint32_t i = 0; i < width; ++i) {
      const double x = (double)i + 0.5;
      out[(size_t)j * width + i] = (float)ellipse_coverage(cx, cy, rx, ry, sn, cs, half_width_px, x, y);
    }
  }
}

/* mask_polygon.rs:161-196: half-open ray cast to +x; rule 0 nonzero, 1 even-odd */
static int polygon_contains(const double *pts, uint32_t n, int rule, double x, double y) {
  if (n < 3) return 0;
  int winding = 0, parity = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const double x0 = pts[2 * i], y0 = pts[2 * i + 1];
    const uint32_t k = (i + 1) % n;
    const double x1 = pts[2 * k], y1 = pts[2 * k + 1];
    const int below0 = y0 <= y, below1 = y1 <= y;
    if (below0 == below1) continue;
    const double t = (y - y0) / (y1 - y0);
    const double cross_x = fma(t, x1 - x0, x0);
    if (cross_x > x) {
      parity = !parity;
      winding += below0 ? 1 : -1;
    }
  }
  return rule == 0 ? winding != 0 : parity;
}

/* mask_polygon.rs:259-286 */
void or_mask_polygon(uint32_t width, uint32_t height, const double *pts, uint32_t n, int rule, float *out) {
  const uint32_t S = 4;
  const double step = 1.0 / (double)S, total = (double)(S * S);
  for (uint32_t j = 0; j < height; ++j)
    for (uint32_t i = 0; i < width; ++i) {
      uint32_t inside = 0;
      for (uint32_t t = 0; t < S; ++t) {
        const double sy = fma((double)t + 0.5, step, (double)j);
        for (uint32_t s = 0; s < S; ++s) {
          const double sx = fma((double)s + 0.5, step, (double)i);
          inside += (uint32_t)polygon_contains(pts, n, rule, sx, sy);
        }
      }
      out[(size_t)j * width + i] = (float)((double)inside / total);
    }
}
