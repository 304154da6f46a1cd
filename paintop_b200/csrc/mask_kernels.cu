// mask_kernels.cu -- device rasterisers of the reference's two mask generators,
// so a mask made by a plan node never leaves the GPU before the solve reads it.
//
//   pt_mask_ellipse  mask.ellipse@1  crates/paintop-cpu/src/ellipse.rs
//                    coverage :168-201, feather :208-218, rasterize :545-565
//   pt_mask_polygon  mask.polygon@1  crates/paintop-cpu/src/mask_polygon.rs
//                    contains :161-196, rasterize :259-286 (4 x 4 subsamples, :77)
//
// Ellipse: one thread per pixel evaluates the reference's formula in fp64 with
// its fused multiply-adds; sin and cos of the angle come from the host's libm
// once per call, like the reference's sin_cos, and sqrt is correctly rounded on
// the device. Only hypot may differ from the host's in the last bit (the op is
// declared tolerance-bounded for exactly that reason).
//
// Polygon: the reference tests every edge at every one of the 16 subsamples of
// every pixel. A subsample row's crossing abscissa t = (y - y0) / (y1 - y0),
// c = fma(t, x1 - x0, x0) depends on the row and the edge only, and a
// subsample column x_q = (q + 0.5) / 4 lies left of c exactly when
// q < ceil(4c - 0.5), an integer computed exactly from c. So a block owns a
// span of 1024 pixels of one pixel row; per subsample row it computes each
// edge's crossing once (edges in chunks of 256, one per thread), turns it into
// that integer, adds crossings right of the whole span to a span-wide winding,
// drops those left of it, and keeps the few inside the span; each thread then
// resolves its 4 pixels' 16 subsamples with integer compares. The arithmetic
// of every crossing is the reference's and winding sums and parities do not
// depend on the order crossings are visited in, so the mask is bit-identical
// to the reference's rasterize().
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/paintop_cuda.h"
#include "ctx.h"
#include "abi_guard.h"

namespace {

constexpr int kSub = 4;                    // subsamples per axis (mask_polygon.rs:77)
constexpr int kRowThreads = 256;           // threads of a polygon block
constexpr int kPix = 4;                    // pixels per thread (one float4 store)
constexpr int kSpan = kRowThreads * kPix;  // pixels of a row per polygon block

__device__ __forceinline__ double feather(double sd, double half_width_px) {
  if (half_width_px <= 0.0) return sd <= 0.0 ? 1.0 : 0.0;
  double t = (sd + half_width_px) / (2.0 * half_width_px);
  t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
  // rounded intrinsics: 1 - (t t) g must not contract into one fma
  const double smoothstep = __dmul_rn(__dmul_rn(t, t), fma(2.0, -t, 3.0));
  return __dsub_rn(1.0, smoothstep);
}

__global__ void k_mask_ellipse(int W, int H, double cx, double cy, double rx, double ry, double sn, double cs,
                               double half_width_px, float *out) {
  const long long n = (long long)W * H;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(p / W), i = (int)(p - (long long)j * W);
    const double off_x = ((double)i + 0.5) - cx, off_y = ((double)j + 0.5) - cy;
    const double local_u = fma(sn, off_y, cs * off_x);
    const double local_v = fma(cs, off_y, -sn * off_x);
    const double norm_x = local_u / rx, norm_y = local_v / ry;
    const double f = sqrt(fma(norm_x, norm_x, norm_y * norm_y));
    double cov = 1.0;
    if (f != 0.0) {
      const double grad = hypot(local_u / (rx * rx), local_v / (ry * ry));
      if (grad != 0.0) cov = feather((f - 1.0) * f / grad, half_width_px);
    }
    out[p] = (float)cov;
  }
}

// Subsample columns q >= 0 (x_q = (q + 0.5) / 4) strictly left of c, i.e. the
// q with c > x_q: q < ceil(4c - 0.5). Exact: clamping c to [-1, W + 1] keeps
// every comparison with the row's subsamples, 4c is a power-of-two scaling,
// and 4c - 0.5 is representable for |4c| <= 2^31.
__device__ __forceinline__ int columns_left_of(double c, int W) {
  const double cc = fmin(fmax(c, -1.0), (double)W + 1.0);
  const double z = ceil(__dsub_rn(__dmul_rn(4.0, cc), 0.5));
  return (int)fmin(fmax(z, 0.0), 4.0 * (double)W);
}

// Winding of this thread's 4 x kPix subsamples of one subsample row, applied
// to the fill rule and added to inside[]: wt is shared by all its columns,
// w[l] holds crossings that fall inside its columns.
__device__ __forceinline__ void add_row(int wt, const int (&w)[kPix * kSub], bool partial, int even_odd,
                                        int (&inside)[kPix]) {
  if (!partial) {
    const int n = even_odd ? (wt & 1) : (wt != 0);
    for (int p = 0; p < kPix; ++p) inside[p] += kSub * n;
  } else {
    for (int p = 0; p < kPix; ++p)
      for (int s = 0; s < kSub; ++s) {
        const int v = wt + w[p * kSub + s];
        inside[p] += even_odd ? (v & 1) : (v != 0);
      }
  }
}

// Polygons of at most 256 edges: a block loops over rows of its span. The
// (edge, subsample row) pairs are spread over all threads, crossings of a row
// land in one of three shared buffers (the row's position in the block's
// sequence, modulo 3), so one barrier per row orders them: the buffer written
// for the next row was last read two rows ago, and is cleared between the two
// barriers that follow that read.
// edges[k] = (x0, y0, x1, y1) of the edge from vertex k to vertex (k + 1) % n.
__device__ __forceinline__ void store_row(float *out, int W, int j, int px, int vec4, const int (&inside)[kPix]) {
  float cov[kPix];
  for (int p = 0; p < kPix; ++p) cov[p] = (float)inside[p] * (1.0f / (float)(kSub * kSub));  // k / 16, exact
  float *row = out + (long long)j * W;
  if (vec4 && px + kPix <= W) {
    *reinterpret_cast<float4 *>(row + px) = make_float4(cov[0], cov[1], cov[2], cov[3]);
  } else {
    for (int p = 0; p < kPix; ++p)
      if (px + p < W) row[px + p] = cov[p];
  }
}

__global__ void __launch_bounds__(kRowThreads, 4) k_mask_polygon_rows(int W, int H,
                                                                     const double4 *__restrict__ edges, int nedges,
                                                                     int even_odd, double ymin, double ymax,
                                                                     int vec4, float *__restrict__ out) {
  __shared__ double4 sedge[kRowThreads];
  __shared__ int cross_q[3][kSub][kRowThreads];
  __shared__ signed char cross_dir[3][kSub][kRowThreads];
  __shared__ int count[3][kSub];
  __shared__ int span_base[3][kSub];
  const int x0 = blockIdx.x * kSpan;
  const int q0 = 4 * x0, q1 = 4 * min(x0 + kSpan, W);
  const int px = x0 + threadIdx.x * kPix;
  const int qp = 4 * px;
  const double step = 1.0 / (double)kSub;
  if (threadIdx.x < 3 * kSub) {
    (&count[0][0])[threadIdx.x] = 0;
    (&span_base[0][0])[threadIdx.x] = 0;
  }
  if ((int)threadIdx.x < nedges) sedge[threadIdx.x] = edges[threadIdx.x];
  __syncthreads();
  int it = 0;
  for (int j = blockIdx.y; j < H; j += gridDim.y) {
    const double ylo = fma(0.5, step, (double)j), yhi = fma((double)kSub - 0.5, step, (double)j);
    int inside[kPix];
    for (int p = 0; p < kPix; ++p) inside[p] = 0;
    // a scanline below every vertex or at/above the highest one straddles no
    // edge (the half-open test compares y0 <= y and y1 <= y): coverage 0
    if (!(yhi < ymin || ylo >= ymax)) {
      const int b = it % 3;
      for (int task = threadIdx.x; task < nedges * kSub; task += kRowThreads) {
        const int e = task >> 2, t = task & 3;
        const double sy = fma((double)t + 0.5, step, (double)j);
        const double4 E = sedge[e];
        const bool below0 = E.y <= sy, below1 = E.w <= sy;
        if (below0 == below1) continue;
        const double tt = (sy - E.y) / (E.w - E.y);
        const int qc = columns_left_of(fma(tt, E.z - E.x, E.x), W);
        const int d = below0 ? 1 : -1;
        if (qc >= q1) {
          atomicAdd(&span_base[b][t], d);
        } else if (qc > q0) {  // (qc <= q0: no column of the span is left of it)
          const int k = atomicAdd(&count[b][t], 1);
          cross_q[b][t][k] = qc;
          cross_dir[b][t][k] = (signed char)d;
        }
      }
      __syncthreads();
      if (threadIdx.x < kSub) {
        const int c = (b + 2) % 3;  // last read two rows ago (before this barrier); next written for the next row
        count[c][threadIdx.x] = 0;
        span_base[c][threadIdx.x] = 0;
      }
      for (int t = 0; t < kSub; ++t) {
        int wt = span_base[b][t];
        int w[kPix * kSub];
        bool partial = false;
        const int m = count[b][t];
        for (int k = 0; k < m; ++k) {
          const int qc = cross_q[b][t][k];
          const int d = cross_dir[b][t][k];
          if (qc >= qp + kPix * kSub) {
            wt += d;
          } else if (qc > qp) {  // rare: a crossing among this thread's own columns
            if (!partial)
              for (int l = 0; l < kPix * kSub; ++l) w[l] = 0;
            partial = true;
            for (int l = 0; l < kPix * kSub; ++l) w[l] += qp + l < qc ? d : 0;
          }
        }
        add_row(wt, w, partial, even_odd, inside);
      }
      ++it;
    }
    store_row(out, W, j, px, vec4, inside);
  }
}

// More than 256 edges: edges in chunks of 256, one per thread, and every
// subsample row's windings held across chunks.
// edges[k] = (x0, y0, x1, y1) of the edge from vertex k to vertex (k + 1) % n.
__global__ void __launch_bounds__(kRowThreads) k_mask_polygon_chunked(int W, int H,
                                                                     const double4 *__restrict__ edges, int nedges,
                                                                     int even_odd, double ymin, double ymax,
                                                                     int vec4, float *__restrict__ out) {
  __shared__ int cross_q[kSub][kRowThreads];        // crossings inside the span: columns left of them
  __shared__ signed char cross_dir[kSub][kRowThreads];
  __shared__ int count[kSub];
  __shared__ int span_base[kSub];                   // winding of crossings right of the whole span
  const int x0 = blockIdx.x * kSpan;
  const int q0 = 4 * x0, q1 = 4 * min(x0 + kSpan, W);
  const int px = x0 + threadIdx.x * kPix;           // this thread's first pixel
  const int qp = 4 * px;                            // and its first subsample column
  const double step = 1.0 / (double)kSub;
  for (int j = blockIdx.y; j < H; j += gridDim.y) {
    double sy[kSub];
    for (int t = 0; t < kSub; ++t) sy[t] = fma((double)t + 0.5, step, (double)j);
    int inside[kPix];
    for (int p = 0; p < kPix; ++p) inside[p] = 0;
    if (!(sy[kSub - 1] < ymin || sy[0] >= ymax)) {
      int wt[kSub];
      int w[kSub][kPix * kSub];
      bool partial[kSub];
      for (int t = 0; t < kSub; ++t) {
        wt[t] = 0;
        partial[t] = false;
        for (int l = 0; l < kPix * kSub; ++l) w[t][l] = 0;
      }
      if (threadIdx.x < kSub) span_base[threadIdx.x] = 0;
      for (int e0 = 0; e0 < nedges; e0 += kRowThreads) {
        if (threadIdx.x < kSub) count[threadIdx.x] = 0;
        __syncthreads();
        const int e = e0 + threadIdx.x;
        if (e < nedges) {
          const double4 E = edges[e];
          for (int t = 0; t < kSub; ++t) {
            const bool below0 = E.y <= sy[t], below1 = E.w <= sy[t];
            if (below0 == below1) continue;
            const double tt = (sy[t] - E.y) / (E.w - E.y);
            const int qc = columns_left_of(fma(tt, E.z - E.x, E.x), W);
            const int d = below0 ? 1 : -1;
            if (qc >= q1) {
              atomicAdd(&span_base[t], d);
            } else if (qc > q0) {  // (qc <= q0: no column of the span is left of it)
              const int k = atomicAdd(&count[t], 1);
              cross_q[t][k] = qc;
              cross_dir[t][k] = (signed char)d;
            }
          }
        }
        __syncthreads();
        for (int t = 0; t < kSub; ++t) {
          const int m = count[t];
          for (int k = 0; k < m; ++k) {
            const int qc = cross_q[t][k];
            const int d = cross_dir[t][k];
            if (qc >= qp + kPix * kSub) {
              wt[t] += d;
            } else if (qc > qp) {
              partial[t] = true;
              for (int l = 0; l < kPix * kSub; ++l) w[t][l] += qp + l < qc ? d : 0;
            }
          }
        }
        __syncthreads();
      }
      for (int t = 0; t < kSub; ++t) add_row(wt[t] + span_base[t], w[t], partial[t], even_odd, inside);
      __syncthreads();  // span_base is reset for the next row only after every read
    }
    store_row(out, W, j, px, vec4, inside);
  }
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

pt_status mfail(pt_ctx *ctx, pt_status s, const std::string &msg) {
  if (ctx) ctx->last_error = msg;
  return s;
}

// Device output (the caller's, or the arena's first bytes for a host mask) and
// `extra` bytes of arena scratch after it.
pt_status mask_target(pt_ctx *ctx, size_t npx, bool device_out, float *mask, size_t extra, float **out,
                      char **scratch) {
  const size_t own = device_out ? 0 : align256(npx * sizeof(float));
  if (!ctx->reserve(own + align256(extra))) return mfail(ctx, PT_OOM, "device arena allocation failed");
  char *base = static_cast<char *>(ctx->arena);
  *out = device_out ? mask : reinterpret_cast<float *>(base);
  *scratch = base + own;
  return PT_OK;
}

// Events: ev[0] call start, ev[1]/ev[2] around the rasteriser, ev[3] call end
// (read back by pt_ctx_last_timing).
pt_status mask_begin(pt_ctx *ctx) {
  for (auto &e : ctx->ev)
    if (!e && cudaEventCreate(&e) != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, "event create");
  cudaEventRecord(ctx->ev[0], ctx->stream);
  return PT_OK;
}

pt_status mask_finish(pt_ctx *ctx, size_t npx, bool device_out, float *mask, const float *dev, int launches) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && !device_out)
    e = cudaMemcpyAsync(mask, dev, npx * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev[3], ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, std::string("mask: ") + cudaGetErrorString(e));
  float a = 0.f, b = 0.f;
  if (cudaEventElapsedTime(&a, ctx->ev[1], ctx->ev[2]) != cudaSuccess) a = -1.f;
  if (cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[3]) != cudaSuccess) b = -1.f;
  cudaGetLastError();
  ctx->last_solve_ms = a;
  ctx->last_call_ms = b;
  ctx->last_launches = launches;
  ctx->last_h2d = ctx->last_d2h = 0;  // not counted on this path
  return PT_OK;
}

}  // namespace

extern "C" pt_status pt_mask_ellipse(pt_ctx *ctx, uint32_t width, uint32_t height, double center_x,
                                     double center_y, double radius_x, double radius_y, double angle_rad,
                                     double half_width_px, float *mask, uint32_t flags) {
  return abi_guard(ctx, [&]() -> pt_status {
    if (!ctx) return PT_INVALID_ARG;
    const size_t npx = (size_t)width * height;
    if (npx && !mask) return mfail(ctx, PT_INVALID_ARG, "null mask buffer");
    // the checks of EllipseGeometry::resolve (ellipse.rs:119-158)
    if (!std::isfinite(center_x) || !std::isfinite(center_y) || !std::isfinite(angle_rad))
      return mfail(ctx, PT_INVALID_ARG, "non-finite ellipse center or angle");
    if (!(std::isfinite(radius_x) && radius_x > 0.0) || !(std::isfinite(radius_y) && radius_y > 0.0))
      return mfail(ctx, PT_INVALID_ARG, "ellipse radii must be finite and > 0");
    if (!std::isfinite(half_width_px) || half_width_px < 0.0)
      return mfail(ctx, PT_INVALID_ARG, "feather half-width must be finite and >= 0");
    if (npx == 0) return PT_OK;
    if (npx > (size_t)INT32_MAX * 4) return mfail(ctx, PT_INVALID_ARG, "mask too large");
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaError_t ce = cudaSetDevice(ctx->device);
    if (ce != cudaSuccess) return mfail(ctx, PT_NO_DEVICE, cudaGetErrorString(ce));
    const bool dev = (flags & PT_FLAG_DEVICE_POINTERS) != 0;
    float *out = nullptr;
    char *scratch = nullptr;
    pt_status st = mask_target(ctx, npx, dev, mask, 0, &out, &scratch);
    if (st != PT_OK) return st;
    if ((st = mask_begin(ctx)) != PT_OK) return st;
    const double sn = std::sin(angle_rad), cs = std::cos(angle_rad);
    const long long blocks = std::min<long long>(((long long)npx + 255) / 256, (long long)ctx->sms * 16);
    cudaEventRecord(ctx->ev[1], ctx->stream);
    k_mask_ellipse<<<(unsigned)blocks, 256, 0, ctx->stream>>>((int)width, (int)height, center_x, center_y,
                                                             radius_x, radius_y, sn, cs, half_width_px, out);
    cudaEventRecord(ctx->ev[2], ctx->stream);
    return mask_finish(ctx, npx, dev, mask, out, 1);
  });
}

extern "C" pt_status pt_mask_polygon(pt_ctx *ctx, uint32_t width, uint32_t height, const double *points_xy,
                                     uint32_t n_points, int32_t fill_rule, float *mask, uint32_t flags) {
  return abi_guard(ctx, [&]() -> pt_status {
    if (!ctx) return PT_INVALID_ARG;
    const size_t npx = (size_t)width * height;
    if (npx && !mask) return mfail(ctx, PT_INVALID_ARG, "null mask buffer");
    if (n_points && !points_xy) return mfail(ctx, PT_INVALID_ARG, "null points");
    if (fill_rule != PT_FILL_NONZERO && fill_rule != PT_FILL_EVEN_ODD)
      return mfail(ctx, PT_INVALID_ARG, "unknown fill rule");
    for (size_t k = 0; k < 2 * (size_t)n_points; ++k)
      if (!std::isfinite(points_xy[k])) return mfail(ctx, PT_INVALID_ARG, "non-finite polygon coordinate");
    if (npx == 0) return PT_OK;
    // subsample column indices (4 per pixel) are int32 in the kernel
    if (width > (1u << 28) || height > (uint32_t)INT32_MAX) return mfail(ctx, PT_INVALID_ARG, "mask too large");
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaError_t ce = cudaSetDevice(ctx->device);
    if (ce != cudaSuccess) return mfail(ctx, PT_NO_DEVICE, cudaGetErrorString(ce));
    const bool dev = (flags & PT_FLAG_DEVICE_POINTERS) != 0;
    float *out = nullptr;
    char *scratch = nullptr;
    pt_status st = mask_target(ctx, npx, dev, mask, (size_t)n_points * sizeof(double4), &out, &scratch);
    if (st != PT_OK) return st;
    if ((st = mask_begin(ctx)) != PT_OK) return st;
    if (n_points < 3) {  // contains() is false everywhere (mask_polygon.rs:162-165)
      cudaEventRecord(ctx->ev[1], ctx->stream);
      ce = cudaMemsetAsync(out, 0, npx * sizeof(float), ctx->stream);
      cudaEventRecord(ctx->ev[2], ctx->stream);
      if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, cudaGetErrorString(ce));
      return mask_finish(ctx, npx, dev, mask, out, 0);
    }
    std::vector<double4> edges(n_points);
    double ymin = points_xy[1], ymax = points_xy[1];
    for (uint32_t k = 0; k < n_points; ++k) {
      const uint32_t q = (k + 1) % n_points;
      edges[k] = make_double4(points_xy[2 * k], points_xy[2 * k + 1], points_xy[2 * q], points_xy[2 * q + 1]);
      ymin = std::min(ymin, points_xy[2 * k + 1]);
      ymax = std::max(ymax, points_xy[2 * k + 1]);
    }
    double4 *dedges = reinterpret_cast<double4 *>(scratch);
    ce = cudaMemcpyAsync(dedges, edges.data(), edges.size() * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream);
    if (ce != cudaSuccess) return mfail(ctx, PT_LAUNCH_FAILED, cudaGetErrorString(ce));
    const uint32_t spans = (width + kSpan - 1) / kSpan;
    const int vec4 = (width % 4 == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0) ? 1 : 0;
    const int even_odd = fill_rule == PT_FILL_EVEN_ODD ? 1 : 0;
    cudaEventRecord(ctx->ev[1], ctx->stream);
    if (n_points > (uint32_t)kRowThreads) {
      const dim3 grid(spans, std::min<uint32_t>(height, 65535u));
      k_mask_polygon_chunked<<<grid, kRowThreads, 0, ctx->stream>>>((int)width, (int)height, dedges,
                                                                    (int)n_points, even_odd, ymin, ymax, vec4, out);
    } else {
      // two waves of 4 resident blocks per SM, each block looping over rows of its span
      const uint32_t rows = std::max<uint32_t>(1u, (uint32_t)(ctx->sms * 8) / spans);
      const dim3 grid(spans, std::min<uint32_t>(std::min<uint32_t>(height, rows), 65535u));
      k_mask_polygon_rows<<<grid, kRowThreads, 0, ctx->stream>>>((int)width, (int)height, dedges, (int)n_points,
                                                                 even_odd, ymin, ymax, vec4, out);
    }
    cudaEventRecord(ctx->ev[2], ctx->stream);
    return mask_finish(ctx, npx, dev, mask, out, 1);
  });
}
