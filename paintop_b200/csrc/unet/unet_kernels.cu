// unet_kernels.cu -- sm_100a kernels of the learned warm start (a small U-Net)
// other than the 3x3 convolutions (conv_tma.cu): pooling, upsampling and their
// adjoints, the 1x1 head, the masked L2 loss, Adam, the bias and weight
// gradient reductions, the input features and the warm-start resampling.
//
// Activations are bf16 in the channel-blocked layout [B][C/8][H][W][8]
// (unet_kernels.h); every kernel here moves one 8-channel group of one pixel
// (16 bytes) per thread, so neighbouring threads touch neighbouring pixels of
// one plane. Every reduction is a fixed-order sum: training steps are
// deterministic.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "unet_kernels.h"

namespace unet {

__device__ __forceinline__ float bf2f(__nv_bfloat16 v) { return __bfloat162float(v); }

__device__ __forceinline__ void ld8(const __nv_bfloat16 *p, float (&v)[8]) {
  const uint4 q = *reinterpret_cast<const uint4 *>(p);
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float2 f = __bfloat1622float2(h[j]);
    v[2 * j] = f.x;
    v[2 * j + 1] = f.y;
  }
}
__device__ __forceinline__ void st8(__nv_bfloat16 *p, const float (&v)[8]) {
  uint4 q;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&q);
#pragma unroll
  for (int j = 0; j < 4; ++j) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
  *reinterpret_cast<uint4 *>(p) = q;
}

// Thread i of an elementwise kernel handles (image b, group g, row y, column x)
// with x fastest: i = ((b * groups + g) * H + y) * W + x.
struct Pix {
  int b, g, y, x;
};
__device__ __forceinline__ Pix pix_of(long long i, int groups, int H, int W) {
  Pix q;
  q.x = (int)(i % W);
  long long r = i / W;
  q.y = (int)(r % H);
  r /= H;
  q.g = (int)(r % groups);
  q.b = (int)(r / groups);
  return q;
}

// 2x2 average pooling: out (H/2 x W/2) from in (H x W)
__global__ void k_avgpool2(ActView in, ActView out, int B, int H, int W, int groups) {
  const int Ho = H / 2, Wo = W / 2;
  const long long total = (long long)B * groups * Ho * Wo;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const Pix q = pix_of(i, groups, Ho, Wo);
    const long long r0 = act_index(in, q.b, q.g, 2 * q.y, 2 * q.x, H, W);
    float v00[8], v01[8], v10[8], v11[8], o[8];
    ld8(in.p + r0, v00);
    ld8(in.p + r0 + 8, v01);
    ld8(in.p + r0 + (long long)W * 8, v10);
    ld8(in.p + r0 + (long long)W * 8 + 8, v11);
#pragma unroll
    for (int j = 0; j < 8; ++j) o[j] = 0.25f * (((v00[j] + v01[j]) + v10[j]) + v11[j]);
    st8(out.p + act_index(out, q.b, q.g, q.y, q.x, Ho, Wo), o);
  }
}

// Row-oriented elementwise kernels: threadIdx.y picks a row r = (b * groups +
// g) * H + y of one 8-channel plane (a grid-stride loop over rows),
// threadIdx.x the pixels x of the row; the row's plane and source rows are
// resolved once per row, and consecutive threads touch consecutive 16-byte
// pixels.
__device__ __forceinline__ void row_of(int r, int groups, int H, int &b, int &g, int &y) {
  y = r % H;
  const int bg = r / H;
  g = bg % groups;
  b = bg / groups;
}

// de = (dskip + unpool(dpool)) * (act > 0): the total gradient of a skip
// activation that feeds both the pooling and the decoder concatenation.
__global__ void k_unpool_add_mask(ActView dskip, ActView dpool, ActView act, ActView out, int B, int H, int W,
                                  int groups) {
  const int rows = B * groups * H;
  for (int r = blockIdx.x * blockDim.y + threadIdx.y; r < rows; r += gridDim.x * blockDim.y) {
    int b, g, y;
    row_of(r, groups, H, b, g, y);
    const __nv_bfloat16 *ds_row = dskip.p + act_index(dskip, b, g, y, 0, H, W);
    const __nv_bfloat16 *dp_row = dpool.p + act_index(dpool, b, g, y / 2, 0, H / 2, W / 2);
    const __nv_bfloat16 *av_row = act.p + act_index(act, b, g, y, 0, H, W);
    __nv_bfloat16 *o_row = out.p + act_index(out, b, g, y, 0, H, W);
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
      float ds[8], dp[8], av[8], o[8];
      ld8(ds_row + (long long)x * 8, ds);
      ld8(dp_row + (long long)(x / 2) * 8, dp);
      ld8(av_row + (long long)x * 8, av);
#pragma unroll
      for (int j = 0; j < 8; ++j) o[j] = av[j] > 0.0f ? ds[j] + 0.25f * dp[j] : 0.0f;
      st8(o_row + (long long)x * 8, o);
    }
  }
}

// Bilinear x2 upsampling, half-pixel centres (out y samples in at (y+0.5)/2-0.5),
// clamped at the border: out[2i] = 0.75 in[i] + 0.25 in[i-1], out[2i+1] = 0.75 in[i] + 0.25 in[i+1].
__device__ __forceinline__ void up_taps(int o, int n, int &i0, int &i1, float &w0, float &w1) {
  const int i = o >> 1;
  i0 = i;
  i1 = (o & 1) ? min(i + 1, n - 1) : max(i - 1, 0);
  w0 = 0.75f;
  w1 = 0.25f;
}
// One thread per input pixel x of input row y writes the 2x2 output block
// (2y .. 2y+1, 2x .. 2x+1): it loads the input's 3x3 neighbourhood once
// (clamped at the border), interpolates each of the three rows horizontally
// for output columns 2x and 2x+1, then those vertically. Every output is
// w0 (w0 a + w1 b) + w1 (w0 c + w1 d), the same expression as a per-output
// gather, so the result does not depend on the traversal.
__global__ void k_upsample2(ActView in, ActView out, int B, int Hi, int Wi, int groups) {
  const int Ho = 2 * Hi, Wo = 2 * Wi;
  const int rows = B * groups * Hi;
  constexpr float w0 = 0.75f, w1 = 0.25f;
  for (int r = blockIdx.x * blockDim.y + threadIdx.y; r < rows; r += gridDim.x * blockDim.y) {
    int b, g, y;
    row_of(r, groups, Hi, b, g, y);
    const __nv_bfloat16 *rm = in.p + act_index(in, b, g, max(y - 1, 0), 0, Hi, Wi);
    const __nv_bfloat16 *rc = in.p + act_index(in, b, g, y, 0, Hi, Wi);
    const __nv_bfloat16 *rp = in.p + act_index(in, b, g, min(y + 1, Hi - 1), 0, Hi, Wi);
    __nv_bfloat16 *o0 = out.p + act_index(out, b, g, 2 * y, 0, Ho, Wo);
    __nv_bfloat16 *o1 = out.p + act_index(out, b, g, 2 * y + 1, 0, Ho, Wo);
    for (int x = threadIdx.x; x < Wi; x += blockDim.x) {
      const int xl = max(x - 1, 0), xr = min(x + 1, Wi - 1);
      // horizontal: L = output column 2x (with x - 1), R = 2x + 1 (with x + 1)
      float mL[8], mR[8], cL[8], cR[8], pL[8], pR[8];
      {
        float v[8], l[8], rr[8];
        ld8(rm + x * 8, v); ld8(rm + xl * 8, l); ld8(rm + xr * 8, rr);
#pragma unroll
        for (int j = 0; j < 8; ++j) { mL[j] = w0 * v[j] + w1 * l[j]; mR[j] = w0 * v[j] + w1 * rr[j]; }
        ld8(rc + x * 8, v); ld8(rc + xl * 8, l); ld8(rc + xr * 8, rr);
#pragma unroll
        for (int j = 0; j < 8; ++j) { cL[j] = w0 * v[j] + w1 * l[j]; cR[j] = w0 * v[j] + w1 * rr[j]; }
        ld8(rp + x * 8, v); ld8(rp + xl * 8, l); ld8(rp + xr * 8, rr);
#pragma unroll
        for (int j = 0; j < 8; ++j) { pL[j] = w0 * v[j] + w1 * l[j]; pR[j] = w0 * v[j] + w1 * rr[j]; }
      }
      // vertical: output row 2y takes rows y, y - 1; row 2y + 1 rows y, y + 1
      float o[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) o[j] = w0 * cL[j] + w1 * mL[j];
      st8(o0 + (2 * x) * 8, o);
#pragma unroll
      for (int j = 0; j < 8; ++j) o[j] = w0 * cR[j] + w1 * mR[j];
      st8(o0 + (2 * x + 1) * 8, o);
#pragma unroll
      for (int j = 0; j < 8; ++j) o[j] = w0 * cL[j] + w1 * pL[j];
      st8(o1 + (2 * x) * 8, o);
#pragma unroll
      for (int j = 0; j < 8; ++j) o[j] = w0 * cR[j] + w1 * pR[j];
      st8(o1 + (2 * x + 1) * 8, o);
    }
  }
}
// Adjoint of k_upsample2 (a gather over the outputs that read each input),
// times the ReLU mask of the upsampled activation.
__global__ void k_upsample2_bwd(ActView dout, ActView act, ActView din, int B, int Hi, int Wi, int groups) {
  const int Ho = 2 * Hi, Wo = 2 * Wi;
  const int rows = B * groups * Hi;
  for (int r = blockIdx.x * blockDim.y + threadIdx.y; r < rows; r += gridDim.x * blockDim.y) {
    int b, g, y;
    row_of(r, groups, Hi, b, g, y);
    // output rows that read input row y: 2y, 2y+1 (weight 0.75), 2y-1 and 2y+2
    // (weight 0.25), plus the clamped border rows
    float wyv[4];
    int oy[4];
    int ny = 0;
    for (int o = max(2 * y - 1, 0); o <= min(2 * y + 2, Ho - 1); ++o) {
      int i0, i1;
      float w0, w1;
      up_taps(o, Hi, i0, i1, w0, w1);
      const float wgt = (i0 == y ? w0 : 0.0f) + (i1 == y ? w1 : 0.0f);
      if (wgt != 0.0f) { oy[ny] = o; wyv[ny] = wgt; ++ny; }
    }
    const __nv_bfloat16 *av_row = act.p + act_index(act, b, g, y, 0, Hi, Wi);
    __nv_bfloat16 *o_row = din.p + act_index(din, b, g, y, 0, Hi, Wi);
    for (int x = threadIdx.x; x < Wi; x += blockDim.x) {
      float wxv[4];
      int ox[4];
      int nx = 0;
      for (int o = max(2 * x - 1, 0); o <= min(2 * x + 2, Wo - 1); ++o) {
        int i0, i1;
        float w0, w1;
        up_taps(o, Wi, i0, i1, w0, w1);
        const float wgt = (i0 == x ? w0 : 0.0f) + (i1 == x ? w1 : 0.0f);
        if (wgt != 0.0f) { ox[nx] = o; wxv[nx] = wgt; ++nx; }
      }
      float s[8] = {0, 0, 0, 0, 0, 0, 0, 0}, v[8], av[8];
      for (int a1 = 0; a1 < ny; ++a1) {
        const __nv_bfloat16 *d_row = dout.p + act_index(dout, b, g, oy[a1], 0, Ho, Wo);
        for (int a2 = 0; a2 < nx; ++a2) {
          ld8(d_row + (long long)ox[a2] * 8, v);
          const float wgt = wyv[a1] * wxv[a2];
#pragma unroll
          for (int j = 0; j < 8; ++j) s[j] += wgt * v[j];
        }
      }
      ld8(av_row + (long long)x * 8, av);
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (!(av[j] > 0.0f)) s[j] = 0.0f;
      st8(o_row + (long long)x * 8, s);
    }
  }
}

// out[j] = sum_k part[k][j] in a fixed order: one warp per column, lane l sums
// k = l, l + 32, ..., then a fixed shuffle tree.
__global__ void k_colsum_reduce(const float *part, int nparts, int c, float *out) {
  const int j = blockIdx.x, lane = threadIdx.x;
  if (j >= c) return;
  float s = 0.0f;
  for (int k = lane; k < nparts; k += 32) s += part[(long long)k * c + j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) out[j] = s;
}

// ----------------------------------------------------------------------------
// head (1x1 conv 16 -> 1), loss, optimiser, input features
// ----------------------------------------------------------------------------
__global__ void k_head_fwd(ActView x, const float *w, const float *b, float *pred, int B, int H, int W) {
  const long long P = (long long)B * H * W;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const int bb = (int)(p / ((long long)H * W));
    const int r = (int)(p - (long long)bb * H * W), y = r / W, xx = r - y * W;
    float v0[8], v1[8];
    ld8(x.p + act_index(x, bb, 0, y, xx, H, W), v0);
    ld8(x.p + act_index(x, bb, 1, y, xx, H, W), v1);
    float s = b[0];
    for (int k = 0; k < 8; ++k) s += v0[k] * w[k];
    for (int k = 0; k < 8; ++k) s += v1[k] * w[8 + k];
    pred[p] = s;
  }
}

// Masked L2 loss: L = sum_m (pred - target)^2 / max(1, sum_m 1); dpred = 2 m (pred - target) / n.
// Per-block partial sums of the squared error and the mask count, then a
// fixed-order sum on the host side of the launch (k_loss_reduce).
__global__ void k_loss(const float *pred, const float *target, const float *mask, long long P, float *dpred,
                       double *part, const float *count) {
  __shared__ double sh[256];
  double acc = 0.0;
  const float n = fmaxf(*count, 1.0f);
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const float m = mask[p] > 0.5f ? 1.0f : 0.0f;
    const float d = (pred[p] - target[p]) * m;
    acc += (double)d * (double)d;
    dpred[p] = 2.0f * d / n;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
// Interior count: per-block partials over a fixed grid-stride partition, then
// one warp sums them in a fixed order.
__global__ void k_mask_count(const float *mask, long long P, float *part) {
  __shared__ float sh[256];
  float acc = 0.0f;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x)
    acc += mask[p] > 0.5f ? 1.0f : 0.0f;
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// head backward: dX[p][k] = dpred[p] * w[k] * (X[p][k] > 0) (bf16); per-block
// partials of dw[k] = sum_p dpred X and db = sum_p dpred.
__global__ void k_head_bwd(ActView x, const float *w, const float *dpred, ActView dx, int B, int H, int W,
                           float *part /* [blocks][17] */) {
  __shared__ float shw[256 * 17];
  float accw[16];
  float accb = 0.0f;
  for (int k = 0; k < 16; ++k) accw[k] = 0.0f;
  const long long P = (long long)B * H * W;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const int bb = (int)(p / ((long long)H * W));
    const int r = (int)(p - (long long)bb * H * W), y = r / W, xx = r - y * W;
    const float g = dpred[p];
    accb += g;
    for (int h = 0; h < 2; ++h) {
      float v[8], o[8];
      ld8(x.p + act_index(x, bb, h, y, xx, H, W), v);
      for (int k = 0; k < 8; ++k) {
        accw[8 * h + k] += g * v[k];
        o[k] = v[k] > 0.0f ? g * w[8 * h + k] : 0.0f;
      }
      st8(dx.p + act_index(dx, bb, h, y, xx, H, W), o);
    }
  }
  for (int k = 0; k < 16; ++k) shw[threadIdx.x * 17 + k] = accw[k];
  shw[threadIdx.x * 17 + 16] = accb;
  __syncthreads();
  if (threadIdx.x < 17) {
    float s = 0.0f;
    for (int t = 0; t < (int)blockDim.x; ++t) s += shw[t * 17 + threadIdx.x];
    part[(long long)blockIdx.x * 17 + threadIdx.x] = s;
  }
}

// Adam (Kingma & Ba): m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
// w -= lr * mhat / (sqrt(vhat) + eps); refreshes the bf16 copy.
__device__ __forceinline__ void adam_update(long long i, float gi, float *w, float *m, float *v, __nv_bfloat16 *wb,
                                            float lr, float b1, float b2, float eps, float bc1, float bc2) {
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
}

__global__ void k_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, long long n, float lr,
                       float b1, float b2, float eps, float bc1, float bc2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    adam_update(i, g[i], w, m, v, wb, lr, b1, b2, eps, bc1, bc2);
}

// Adam on the combination of `R` replicas' gradient records laid end to end,
// each n gradients of that replica's mean loss followed by its interior count
// c_r: g = (sum over r = 0 .. R-1, in order, of c_r g_r) / max(1, sum c_r),
// accumulated in fp64 (each product c_r g_r is exact there). Every replica
// that runs this on the same records takes the same step bit for bit; with
// one record g is that record's gradient exactly.
__global__ void k_adam_records(float *w, float *m, float *v, const float *rec, int R, __nv_bfloat16 *wb,
                               long long n, float lr, float b1, float b2, float eps, float bc1, float bc2) {
  double total = 0.0;
  for (int r = 0; r < R; ++r) total += (double)rec[(long long)r * (n + 1) + n];
  total = fmax(total, 1.0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int r = 0; r < R; ++r) {
      const float *q = rec + (long long)r * (n + 1);
      acc += (double)q[n] * (double)q[i];
    }
    adam_update(i, (float)(acc / total), w, m, v, wb, lr, b1, b2, eps, bc1, bc2);
  }
}

// fp32 master -> bf16 weights [co][tap][ci] and the flipped/transposed copy
// W'[ci][tap][co] = W[co][8 - tap][ci] used by the backward-data convolution.
__global__ void k_prep_weights(const float *w, int cout, int cin, __nv_bfloat16 *wb, __nv_bfloat16 *wt) {
  const int total = cout * 9 * cin;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int co = i / (9 * cin), r = i - co * 9 * cin, tap = r / cin, ci = r - tap * cin;
    const __nv_bfloat16 v = __float2bfloat16_rn(w[i]);
    wb[i] = v;
    if (wt) wt[((long long)ci * 9 + (8 - tap)) * cout + co] = v;
  }
}

// fp32 features (B x H x W x 4) -> the bf16 input, 16 channels (2 groups):
// group 0 = the 4 features then zeros, group 1 = zeros.
__global__ void k_features_to_input(const float *f, ActView x, int B, int H, int W) {
  const long long P = (long long)B * H * W;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const int bb = (int)(p / ((long long)H * W));
    const int r = (int)(p - (long long)bb * H * W), y = r / W, xx = r - y * W;
    float v[8] = {f[p * 4], f[p * 4 + 1], f[p * 4 + 2], f[p * 4 + 3], 0, 0, 0, 0};
    float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    st8(x.p + act_index(x, bb, 0, y, xx, H, W), v);
    st8(x.p + act_index(x, bb, 1, y, xx, H, W), z);
  }
}

// Input features of one image (single channel): masked divergence (the
// guidance Laplacian at interior cells, poisson.rs:364-373), boundary values
// of the correction the network predicts (anchor - guidance outside the
// interior: the solution is guidance + a harmonic correction with exactly
// these boundary values), the interior mask, and the distance to the nearest
// non-interior cell along the row/column (the minimum of the four
// straight-line distances, divided by 32 and clipped at 1).
__global__ void k_features(const float *guid, const float *anchor, const float *mask, int B, int H, int W,
                           float *f) {
  const long long P = (long long)B * H * W;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(p / ((long long)H * W));
    const int r = (int)(p - (long long)b * H * W), y = r / W, x = r - y * W;
    const long long base = (long long)b * H * W;
    auto interior = [&](int yy, int xx) {
      if (H < 3 || W < 3 || yy < 1 || xx < 1 || yy > H - 2 || xx > W - 2) return false;
      return mask[base + (long long)yy * W + xx] > 0.5f;
    };
    const bool in = interior(y, x);
    float div = 0.0f, dist = 0.0f;
    if (in) {
      const float c = guid[p];
      div = (guid[p - 1] + guid[p + 1] + guid[p - W] + guid[p + W]) - 4.0f * c;
      int d = 1;
      const int lim = 32;
      for (; d < lim; ++d)
        if (!interior(y, x - d) || !interior(y, x + d) || !interior(y - d, x) || !interior(y + d, x)) break;
      dist = (float)d / (float)lim;
    }
    f[p * 4 + 0] = div;
    f[p * 4 + 1] = in ? 0.0f : anchor[p] - guid[p];
    f[p * 4 + 2] = in ? 1.0f : 0.0f;
    f[p * 4 + 3] = dist;
  }
}

// ----------------------------------------------------------------------------
// warm-start guess at another resolution
// ----------------------------------------------------------------------------
// Pool channel ch of interleaved (H x W x C) guidance and anchor, and the mask,
// by `s` (area average over the block's in-image pixels) into image ch of a
// (C x Hc x Wc) batch; coarse cells with no in-image pixel get 0.
__global__ void k_pool_inputs(const float *g, const float *a, const float *m, int W, int H, int C, int s, int Wc,
                              int Hc, float *cg, float *ca, float *cm) {
  const long long total = (long long)C * Hc * Wc;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(i / ((long long)Hc * Wc));
    const int r = (int)(i - (long long)ch * Hc * Wc), cy = r / Wc, cx = r - cy * Wc;
    const int y0 = cy * s, x0 = cx * s, y1 = min(y0 + s, H), x1 = min(x0 + s, W);
    float sg = 0.0f, sa = 0.0f, sm = 0.0f;
    int cnt = 0;
    for (int y = y0; y < y1; ++y)
      for (int x = x0; x < x1; ++x) {
        const long long px = (long long)y * W + x;
        sg += g[px * C + ch];
        sa += a[px * C + ch];
        sm += m[px];
        ++cnt;
      }
    const float inv = cnt ? 1.0f / (float)cnt : 0.0f;
    cg[i] = sg * inv;
    ca[i] = sa * inv;
    cm[i] = sm * inv;
  }
}

// guess = guidance + the coarse correction upsampled bilinearly (half-pixel
// centres, clamped to the coarse cells that cover the image).
__global__ void k_compose_guess(const float *g, const float *corr, int W, int H, int C, int s, int Wc, int Hc,
                                float *guess) {
  const int hv = (H + s - 1) / s, wv = (W + s - 1) / s;  // coarse cells that touch the image
  const long long total = (long long)W * H * C;
  const float inv = 1.0f / (float)s;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(i % C);
    const long long px = i / C;
    const int y = (int)(px / W), x = (int)(px - (long long)y * W);
    const float fy = fminf(fmaxf(((float)y + 0.5f) * inv - 0.5f, 0.0f), (float)(hv - 1));
    const float fx = fminf(fmaxf(((float)x + 0.5f) * inv - 0.5f, 0.0f), (float)(wv - 1));
    const int iy = min((int)fy, hv - 1), ix = min((int)fx, wv - 1);
    const int jy = min(iy + 1, hv - 1), jx = min(ix + 1, wv - 1);
    const float wy = fy - (float)iy, wx = fx - (float)ix;
    const float *c = corr + (long long)ch * Hc * Wc;
    const float top = c[(long long)iy * Wc + ix] + wx * (c[(long long)iy * Wc + jx] - c[(long long)iy * Wc + ix]);
    const float bot = c[(long long)jy * Wc + ix] + wx * (c[(long long)jy * Wc + jx] - c[(long long)jy * Wc + ix]);
    guess[i] = g[i] + (top + wy * (bot - top));
  }
}

// ----------------------------------------------------------------------------
// launchers
// ----------------------------------------------------------------------------
// (the weight gradient's final sum, launched by launch_wgrad_reduce)
// Sum the per-chunk partials in chunk order: dW[co][tap][ci] (fp32), then,
// with db, db[co] from its [chunks][cout] partials. A block takes 32
// consecutive outputs (lane = output, so each warp's loads are coalesced);
// warp w forms the running sum over chunks w, w + 32, ... in chunk order, and
// warp 0 combines the 32 sums by the fixed tree s[l] += s[l + o], o = 16, 8,
// 4, 2, 1.
__global__ void __launch_bounds__(1024) k_wgrad_reduce(const float *part, int nchunks, int cout, int cin, float *dw,
                                                       const float *db_part, float *db) {
  __shared__ float sh[32][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long wtotal = (long long)cout * 9 * cin;
  const long long total = wtotal + (db ? cout : 0);
  for (long long i0 = blockIdx.x * 32LL; i0 < total; i0 += gridDim.x * 32LL) {
    const long long i = i0 + lane;
    float s = 0.0f;
    if (i < total) {
      const float *src;
      long long stride;
      if (i < wtotal) {
        const int co = (int)(i / (9 * cin)), r = (int)(i - (long long)co * 9 * cin), tap = r / cin, ci = r - tap * cin;
        src = part + ((long long)tap * cout + co) * cin + ci;
        stride = wtotal;
      } else {
        src = db_part + (i - wtotal);
        stride = cout;
      }
      for (int k = w; k < nchunks; k += 32) s += src[(long long)k * stride];
    }
    sh[w][lane] = s;
    __syncthreads();
    if (w == 0 && i < total) {
      float v[32];
#pragma unroll
      for (int l = 0; l < 32; ++l) v[l] = sh[l][lane];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int l = 0; l < o; ++l) v[l] += v[l + o];
      if (i < wtotal)
        dw[i] = v[0];
      else
        db[i - wtotal] = v[0];
    }
    __syncthreads();
  }
}

cudaError_t launch_wgrad_reduce(const float *part, int nchunks, int cout, int cin, float *dw, const float *db_part,
                                float *db, cudaStream_t st) {
  const long long total = (long long)cout * 9 * cin + (db ? cout : 0);
  long long blocks = (total + 31) / 32;
  if (blocks > 148 * 2) blocks = 148 * 2;
  k_wgrad_reduce<<<(unsigned)blocks, 1024, 0, st>>>(part, nchunks, cout, cin, dw, db_part, db);
  return cudaGetLastError();
}

// Row kernels: 256-thread blocks of row_threads(w) threads across a row (a
// multiple of 32, at most 256) times 256 / row_threads(w) rows, rows in a
// grid-stride loop over a fixed number of blocks.
static dim3 row_threads(int w) {
  const unsigned tx = (unsigned)std::min(256, std::max(32, (w + 31) / 32 * 32));
  return dim3(tx, 256 / tx);
}
static unsigned row_blocks(long long rows, int w) {
  const long long per = 256 / row_threads(w).x;
  return (unsigned)std::min<long long>(std::max<long long>((rows + per - 1) / per, 1), 148 * 16);
}

static unsigned blocks_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 148 * 32) b = 148 * 32;
  return (unsigned)(b < 1 ? 1 : b);
}

cudaError_t launch_reduce_rows(const float *part, int nparts, int c, float *out, cudaStream_t st) {
  k_colsum_reduce<<<c, 32, 0, st>>>(part, nparts, c, out);
  return cudaGetLastError();
}

cudaError_t launch_avgpool2(const ActView &in, const ActView &out, int B, int H, int W, int groups,
                            cudaStream_t st) {
  k_avgpool2<<<blocks_for((long long)B * groups * H * W / 4, 256), 256, 0, st>>>(in, out, B, H, W, groups);
  return cudaGetLastError();
}
cudaError_t launch_unpool_add_mask(const ActView &dskip, const ActView &dpool, const ActView &act,
                                   const ActView &out, int B, int H, int W, int groups, cudaStream_t st) {
  k_unpool_add_mask<<<row_blocks((long long)B * groups * H, W), row_threads(W), 0, st>>>(dskip, dpool, act, out, B, H,
                                                                                       W, groups);
  return cudaGetLastError();
}
cudaError_t launch_upsample2(const ActView &in, const ActView &out, int B, int Hi, int Wi, int groups,
                             cudaStream_t st) {
  k_upsample2<<<row_blocks((long long)B * groups * Hi, Wi), row_threads(Wi), 0, st>>>(in, out, B, Hi, Wi, groups);
  return cudaGetLastError();
}
cudaError_t launch_upsample2_bwd(const ActView &dout, const ActView &act, const ActView &din, int B, int Hi,
                                 int Wi, int groups, cudaStream_t st) {
  k_upsample2_bwd<<<row_blocks((long long)B * groups * Hi, Wi), row_threads(Wi), 0, st>>>(dout, act, din, B, Hi, Wi,
                                                                                    groups);
  return cudaGetLastError();
}
cudaError_t launch_head_fwd(const ActView &x, const float *w, const float *b, float *pred, int B, int H, int W,
                            cudaStream_t st) {
  k_head_fwd<<<blocks_for((long long)B * H * W, 256), 256, 0, st>>>(x, w, b, pred, B, H, W);
  return cudaGetLastError();
}
int head_bwd_blocks(long long P) { return (int)blocks_for(P, 256); }
cudaError_t launch_head_bwd(const ActView &x, const float *w, const float *dpred, const ActView &dx, int B, int H,
                            int W, float *part, cudaStream_t st) {
  const int nb = head_bwd_blocks((long long)B * H * W);
  k_head_bwd<<<nb, 256, 0, st>>>(x, w, dpred, dx, B, H, W, part);
  return cudaGetLastError();
}
int loss_blocks(long long P) { return (int)blocks_for(P, 256) > 1024 ? 1024 : (int)blocks_for(P, 256); }
cudaError_t launch_loss(const float *pred, const float *target, const float *mask, long long P, float *dpred,
                        double *part, float *count, cudaStream_t st) {
  // count[0] = the interior count, count[1 ..] the per-block partials
  const int nb = loss_blocks(P);
  k_mask_count<<<nb, 256, 0, st>>>(mask, P, count + 1);
  k_colsum_reduce<<<1, 32, 0, st>>>(count + 1, nb, 1, count);
  k_loss<<<nb, 256, 0, st>>>(pred, target, mask, P, dpred, part, count);
  return cudaGetLastError();
}
cudaError_t launch_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, long long n, float lr,
                        int step, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
  k_adam<<<blocks_for(n, 256), 256, 0, st>>>(w, m, v, g, wb, n, lr, b1, b2, eps, bc1, bc2);
  return cudaGetLastError();
}
cudaError_t launch_adam_records(float *w, float *m, float *v, const float *records, int replicas, long long n,
                                float lr, int step, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
  k_adam_records<<<blocks_for(n, 256), 256, 0, st>>>(w, m, v, records, replicas, nullptr, n, lr, b1, b2, eps, bc1,
                                                     bc2);
  return cudaGetLastError();
}
cudaError_t launch_prep_weights(const float *w, int cout, int cin, __nv_bfloat16 *wb, __nv_bfloat16 *wt,
                                cudaStream_t st) {
  k_prep_weights<<<blocks_for((long long)cout * 9 * cin, 256), 256, 0, st>>>(w, cout, cin, wb, wt);
  return cudaGetLastError();
}
cudaError_t launch_features_to_input(const float *f, const ActView &x, int B, int H, int W, cudaStream_t st) {
  k_features_to_input<<<blocks_for((long long)B * H * W, 256), 256, 0, st>>>(f, x, B, H, W);
  return cudaGetLastError();
}
cudaError_t launch_features(const float *guid, const float *anchor, const float *mask, int B, int H, int W,
                            float *f, cudaStream_t st) {
  k_features<<<blocks_for((long long)B * H * W, 256), 256, 0, st>>>(guid, anchor, mask, B, H, W, f);
  return cudaGetLastError();
}

cudaError_t launch_pool_inputs(const float *g, const float *a, const float *m, int W, int H, int C, int s, int Wc,
                               int Hc, float *cg, float *ca, float *cm, cudaStream_t st) {
  k_pool_inputs<<<blocks_for((long long)C * Hc * Wc, 256), 256, 0, st>>>(g, a, m, W, H, C, s, Wc, Hc, cg, ca, cm);
  return cudaGetLastError();
}
cudaError_t launch_compose_guess(const float *g, const float *corr, int W, int H, int C, int s, int Wc, int Hc,
                                 float *guess, cudaStream_t st) {
  k_compose_guess<<<blocks_for((long long)W * H * C, 256), 256, 0, st>>>(g, corr, W, H, C, s, Wc, Hc, guess);
  return cudaGetLastError();
}

}  // namespace unet
