// unet_kernels.cu -- sm_100a kernels of the learned warm start (a small U-Net).
//
// Tensors are NHWC. Activations and activation gradients are bf16; weights are
// bf16 copies of fp32 master weights; every product is accumulated in fp32 on
// the tensor core (tcgen05.mma, accumulator in TMEM).
//
// 3x3 convolutions (stride 1, zero padding 1) are implicit GEMMs:
//   forward   Y[p][co]  = sum_{tap,ci} X[p + off(tap)][ci] * W[co][tap][ci]
//   bwd data  dX[q][ci] = sum_{tap,co} dY[q + off(tap)][co] * W'[ci][tap][co],
//             W'[ci][tap][co] = W[co][8 - tap][ci]   (the same kernel)
//   bwd wts   dW[co][tap][ci] = sum_p dY[p][co] * X[p + off(tap)][ci]
// with off(tap) = (tap / 3 - 1, tap % 3 - 1). The GEMM rows are 128 pixels, the
// columns the output channels; operand tiles are gathered (im2col on the fly)
// into shared memory with cp.async, in the canonical no-swizzle core-matrix
// layout that the tensor core reads through shared-memory descriptors.
#include <cuda_bf16.h>

#include <cstdint>

#include "tc.cuh"
#include "unet_kernels.h"

namespace unet {

constexpr uint32_t kWaitPolls = 1u << 26;  // bounded mbarrier waits (seconds at most)

__device__ __forceinline__ uint32_t tmem_cols_for(int n) {
  return n <= 32 ? 32u : (n <= 64 ? 64u : (n <= 128 ? 128u : 256u));
}

__device__ __forceinline__ float bf2f(__nv_bfloat16 v) { return __bfloat162float(v); }

// ----------------------------------------------------------------------------
// 3x3 convolution, forward and backward-data (implicit GEMM on tcgen05)
// ----------------------------------------------------------------------------
// The reduction axis (tap, channel) is cut into pipeline chunks: the channels
// into cpt equal parts of kc (kc <= 128, a multiple of 16), and up to tpc taps
// of one part share a chunk (tpc * kc <= 144), so a 16-channel layer runs all
// nine taps as one chunk. Chunk c covers taps [tg * tpc, tg * tpc + ntap) of
// channel part c % cpt, tg = c / cpt. Shared memory per stage: A = 128 pixels
// x kmax, B = N x kmax, both K-major; kk = tap_local * kc / 8 + j indexes the
// 8-element K groups of a chunk.
__host__ __device__ inline ConvChunking conv_chunking(int cin) {
  ConvChunking c;
  c.cpt = (cin + 127) / 128;
  c.kc = cin / c.cpt;
  c.tpc = c.kc >= 144 ? 1 : 144 / c.kc;
  if (c.tpc > 9) c.tpc = 9;
  c.ntg = (9 + c.tpc - 1) / c.tpc;
  c.nchunks = c.ntg * c.cpt;
  c.kmax = c.tpc * c.kc;
  c.stages = c.nchunks > 1 ? 2 : 1;
  return c;
}

template <int N>
__global__ void __launch_bounds__(128) k_conv3x3(ConvArgs a) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t mbar[2];
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ncols = tmem_cols_for(N);
  const ConvChunking ck = conv_chunking(a.cin);
  const int A_BYTES = 128 * ck.kmax * 2;
  const int STAGE = (128 + N) * ck.kmax * 2;

  if (warp == 0) tmem_alloc(&tbase, ncols);
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
  }
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t tm = tbase;

  const long long P = (long long)a.B * a.H * a.W;
  const long long p = (long long)blockIdx.x * 128 + tid;  // this thread's pixel (GEMM row)
  int pb = 0, py = 0, px = 0;
  if (p < P) {
    pb = (int)(p / ((long long)a.H * a.W));
    const int r = (int)(p - (long long)pb * a.H * a.W);
    py = r / a.W;
    px = r - py * a.W;
  }
  const uint32_t idesc = instr_desc_bf16(128, N, false, false);
  const int g8 = ck.kc / 8;  // 8-channel groups per tap in a chunk

  auto load_chunk = [&](int c, int stage) {
    const int tap0 = (c / ck.cpt) * ck.tpc, c0 = (c % ck.cpt) * ck.kc;
    const int ntap = min(ck.tpc, 9 - tap0);
    unsigned char *sA = sm + stage * STAGE;
    unsigned char *sB = sA + A_BYTES;
    for (int t = 0; t < ntap; ++t) {
      const int tap = tap0 + t;
      const int yy = py + tap / 3 - 1, xx = px + tap % 3 - 1;
      const bool in = p < P && yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
      const __nv_bfloat16 *src =
          a.x + (((long long)pb * a.H + (in ? yy : 0)) * a.W + (in ? xx : 0)) * a.ldx + a.x_off + c0;
      for (int j = 0; j < g8; ++j) cp16(sA + kmajor_off(tid, t * g8 + j, 16), src + j * 8, in);
    }
    const int per = ntap * g8;
    for (int idx = tid; idx < N * per; idx += 128) {
      const int n = idx / per, kk = idx - n * per, t = kk / g8, j = kk - t * g8;
      cp16(sB + kmajor_off(n, kk, N / 8), a.w + ((long long)n * 9 + tap0 + t) * a.cin + c0 + j * 8, true);
    }
  };

  bool ok = true;
  load_chunk(0, 0);
  cp_commit();
  for (int c = 0; c < ck.nchunks; ++c) {
    const int s = c & 1;
    bool w = true;
    if (c + 1 < ck.nchunks) {
      // the MMAs of chunk c-1 read stage s^1: wait for them before refilling it
      if (c >= 1) w = mbar_wait(&mbar[s ^ 1], ((c - 1) >> 1) & 1, kWaitPolls);
      if (w) load_chunk(c + 1, s ^ 1);
      cp_commit();
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    fence_async_smem();
    tc_fence_before_sync();
    if (!__syncthreads_and(w)) { ok = false; break; }
    if (tid == 0) {
      tc_fence_after_sync();
      const int ntap = min(ck.tpc, 9 - (c / ck.cpt) * ck.tpc);
      const uint32_t aB = smem_u32(sm + s * STAGE), bB = aB + A_BYTES;
      for (int ks = 0; ks < ntap * ck.kc / 16; ++ks) {
        const uint64_t ad = smem_desc(aB + ks * 2 * 16 * 128, 16 * 128, 128);
        const uint64_t bd = smem_desc(bB + ks * 2 * (N / 8) * 128, (N / 8) * 128, 128);
        mma_bf16(tm, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
      }
      mma_commit(&mbar[s]);
    }
  }
  if (ok) ok = mbar_wait(&mbar[(ck.nchunks - 1) & 1], ((ck.nchunks - 1) >> 1) & 1, kWaitPolls);
  cp_wait<0>();
  tc_fence_before_sync();
  ok = __syncthreads_and(ok);
  tc_fence_after_sync();
  if (!ok && tid == 0) atomicExch(a.err, 1);

  if (ok) {
    // epilogue: warp w owns TMEM lanes 32w..32w+31 = GEMM rows = pixels
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    for (int c16 = 0; c16 < N / 16; ++c16) {
      uint32_t r[16];
      tmem_ld16(tm + lane_base + c16 * 16, r);
      if (p < P) {
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          float f = __uint_as_float(r[j]);
          if (a.bias) f += a.bias[c16 * 16 + j];
          if (a.relu) f = fmaxf(f, 0.0f);
          v[j] = f;
        }
        if (a.mask) {
          const __nv_bfloat16 *m = a.mask + p * a.ldm + a.m_off + c16 * 16;
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (!(bf2f(m[j]) > 0.0f)) v[j] = 0.0f;
        }
        __align__(16) __nv_bfloat16 o[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) o[j] = __float2bfloat16_rn(v[j]);
        uint4 *dst = reinterpret_cast<uint4 *>(a.y + p * a.ldy + a.y_off + c16 * 16);
        dst[0] = reinterpret_cast<const uint4 *>(o)[0];
        dst[1] = reinterpret_cast<const uint4 *>(o)[1];
      }
    }
  }
  tc_fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after_sync();
    tmem_dealloc(tm, ncols);
  }
}

// ----------------------------------------------------------------------------
// 3x3 convolution, backward-weights (tcgen05, both operands MN-major)
// ----------------------------------------------------------------------------
// One CTA: one tap, one chunk of kWgPix pixels. GEMM rows = output channels
// (padded to 128 with zero rows), columns = input channels, reduction = the
// chunk's pixels. Partial sums go to part[chunk][tap][co][ci] (fp32) and are
// reduced over chunks in chunk order by k_wgrad_reduce.
constexpr int kWgPix = 2048;  // pixels per CTA
constexpr int KP = 64;        // pixels per pipeline stage

// MN-major core-matrix tile offset: element (mn, k) of an MN x K tile with
// mn8 = MN / 8 groups: ((k / 8) * mn8 + mn / 8) * 128 + (k % 8) * 16 + (mn % 8) * 2.
__host__ __device__ constexpr uint32_t mnmajor_off(uint32_t g8, uint32_t k, uint32_t mn8) {
  return ((k >> 3) * mn8 + g8) * 128u + (k & 7u) * 16u;
}

template <int N>
__global__ void __launch_bounds__(128) k_wgrad(WgradArgs a) {
  constexpr int M = 128;
  constexpr int A_BYTES = M * KP * 2;
  constexpr int B_BYTES = N * KP * 2;
  constexpr int STAGE = A_BYTES + B_BYTES;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t mbar[2];
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = tmem_cols_for(N);
  const int tap = blockIdx.y;
  const long long P = (long long)a.B * a.H * a.W;
  const long long p0 = (long long)blockIdx.x * kWgPix;
  const int npix = (int)min((long long)kWgPix, P - p0);
  const int nsub = (npix + KP - 1) / KP;

  if (warp == 0) tmem_alloc(&tbase, ncols);
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
  }
  // rows >= cout of A stay zero in both stages: clear both stages once
  for (int k = tid * 16; k < 2 * STAGE; k += 128 * 16)
    *reinterpret_cast<uint4 *>(sm + k) = make_uint4(0, 0, 0, 0);
  fence_async_smem();
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t tm = tbase;
  const uint32_t idesc = instr_desc_bf16(M, N, true, true);
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;

  auto load_sub = [&](int sidx, int stage) {
    unsigned char *sA = sm + stage * STAGE;
    unsigned char *sB = sA + A_BYTES;
    // 64 pixels of this sub-chunk; A rows: cout/8 groups, B rows: cin/8 groups
    const int ga = a.cout / 8, gb = N / 8;
    for (int idx = tid; idx < KP * (ga + gb); idx += 128) {
      const int k = idx / (ga + gb), g = idx - k * (ga + gb);
      const long long p = p0 + (long long)sidx * KP + k;
      const bool pin = (long long)sidx * KP + k < npix;
      if (g < ga) {
        const __nv_bfloat16 *src = a.dy + (pin ? p : 0) * a.lddy + a.dy_off + g * 8;
        cp16(sA + mnmajor_off(g, k, M / 8), src, pin);
      } else {
        const int gg = g - ga;
        int b = 0, y = 0, x = 0;
        bool in = false;
        if (pin) {
          b = (int)(p / ((long long)a.H * a.W));
          const int r = (int)(p - (long long)b * a.H * a.W);
          y = r / a.W + dy;
          x = r % a.W + dx;
          in = y >= 0 && y < a.H && x >= 0 && x < a.W;
        }
        const __nv_bfloat16 *src =
            a.x + (((long long)b * a.H + (in ? y : 0)) * a.W + (in ? x : 0)) * a.ldx + a.x_off + gg * 8;
        cp16(sB + mnmajor_off(gg, k, gb), src, in);
      }
    }
  };

  bool ok = true;
  if (nsub > 0) load_sub(0, 0);
  cp_commit();
  for (int c = 0; c < nsub; ++c) {
    const int s = c & 1;
    bool w = true;
    if (c + 1 < nsub) {
      if (c >= 1) w = mbar_wait(&mbar[s ^ 1], ((c - 1) >> 1) & 1, kWaitPolls);
      if (w) load_sub(c + 1, s ^ 1);
      cp_commit();
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    fence_async_smem();
    tc_fence_before_sync();
    if (!__syncthreads_and(w)) { ok = false; break; }
    if (tid == 0) {
      tc_fence_after_sync();
      const uint32_t aB = smem_u32(sm + s * STAGE), bB = aB + A_BYTES;
      for (int ks = 0; ks < KP / 16; ++ks) {
        const uint64_t ad = smem_desc(aB + ks * 2 * (M / 8) * 128, (M / 8) * 128, 128);
        const uint64_t bd = smem_desc(bB + ks * 2 * (N / 8) * 128, (N / 8) * 128, 128);
        mma_bf16(tm, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
      }
      mma_commit(&mbar[s]);
    }
  }
  if (ok && nsub > 0) ok = mbar_wait(&mbar[(nsub - 1) & 1], ((nsub - 1) >> 1) & 1, kWaitPolls);
  cp_wait<0>();
  tc_fence_before_sync();
  ok = __syncthreads_and(ok);
  tc_fence_after_sync();
  if (!ok && tid == 0) atomicExch(a.err, 1);
  if (ok) {
    const int co = 32 * warp + lane;
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    float *dst = a.part + (((long long)blockIdx.x * 9 + tap) * a.cout + co) * N;
    for (int c16 = 0; c16 < N / 16; ++c16) {
      uint32_t r[16];
      tmem_ld16(tm + lane_base + c16 * 16, r);
      if (co < a.cout) {
#pragma unroll
        for (int j = 0; j < 16; ++j) dst[c16 * 16 + j] = nsub > 0 ? __uint_as_float(r[j]) : 0.0f;
      }
    }
  }
  tc_fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after_sync();
    tmem_dealloc(tm, ncols);
  }
}

// Sum the per-chunk partials in chunk order: dW[co][tap][ci] (fp32).
__global__ void k_wgrad_reduce(const float *part, int nchunks, int cout, int cin, float *dw) {
  const int total = cout * 9 * cin;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int co = i / (9 * cin), r = i - co * 9 * cin, tap = r / cin, ci = r - tap * cin;
    float s = 0.0f;
    for (int k = 0; k < nchunks; ++k) s += part[(((long long)k * 9 + tap) * cout + co) * cin + ci];
    dw[i] = s;
  }
}

// db[co] = sum_p dY[p][co]: block k sums pixels [k * chunk, (k + 1) * chunk)
// with blockDim / c pixel lanes per channel, lanes combined in lane order;
// k_colsum_reduce then sums the block partials in block order.
__global__ void k_colsum(const __nv_bfloat16 *dy, int ld, int off, int c, long long P, int chunk,
                         float *part) {
  __shared__ float sh[256];
  const int lanes = blockDim.x / c;
  const int co = threadIdx.x % c, ln = threadIdx.x / c;
  const long long p0 = (long long)blockIdx.x * chunk;
  const long long p1 = min(p0 + chunk, P);
  float s = 0.0f;
  if (ln < lanes)
    for (long long p = p0 + ln; p < p1; p += lanes) s += bf2f(dy[p * ld + off + co]);
  sh[threadIdx.x] = s;
  __syncthreads();
  if ((int)threadIdx.x < c) {
    float t = 0.0f;
    for (int l = 0; l < lanes; ++l) t += sh[l * c + threadIdx.x];
    part[(long long)blockIdx.x * c + threadIdx.x] = t;
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
// pooling, upsampling, masks
// ----------------------------------------------------------------------------
// The elementwise kernels below move 8 channels (16 bytes) per thread: every
// channel count, pitch and slice offset of the network is a multiple of 8.
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

// 2x2 average pooling: out (H/2 x W/2 x c at ldo, ooff) from in (H x W x c at ldi, ioff)
__global__ void k_avgpool2(const __nv_bfloat16 *in, int ldi, int ioff, __nv_bfloat16 *out, int ldo, int ooff,
                           int B, int H, int W, int c) {
  const int Ho = H / 2, Wo = W / 2, c8 = c / 8;
  const long long total = (long long)B * Ho * Wo * c8;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(i % c8) * 8;
    const long long q = i / c8;
    const int x = (int)(q % Wo), y = (int)((q / Wo) % Ho), b = (int)(q / ((long long)Wo * Ho));
    const long long r0 = ((long long)b * H + 2 * y) * W + 2 * x;
    float v00[8], v01[8], v10[8], v11[8], o[8];
    ld8(in + r0 * ldi + ioff + ch, v00);
    ld8(in + (r0 + 1) * ldi + ioff + ch, v01);
    ld8(in + (r0 + W) * ldi + ioff + ch, v10);
    ld8(in + (r0 + W + 1) * ldi + ioff + ch, v11);
#pragma unroll
    for (int j = 0; j < 8; ++j) o[j] = 0.25f * (((v00[j] + v01[j]) + v10[j]) + v11[j]);
    st8(out + q * ldo + ooff + ch, o);
  }
}

// de = (dskip + unpool(dpool)) * (act > 0): the total gradient of a skip
// activation that feeds both the pooling and the decoder concatenation.
__global__ void k_unpool_add_mask(const __nv_bfloat16 *dskip, int lds, int soff, const __nv_bfloat16 *dpool,
                                  int ldp, int poff, const __nv_bfloat16 *act, int lda, int aoff,
                                  __nv_bfloat16 *out, int ldo, int ooff, int B, int H, int W, int c) {
  const int c8 = c / 8;
  const long long total = (long long)B * H * W * c8;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(i % c8) * 8;
    const long long q = i / c8;
    const int x = (int)(q % W), y = (int)((q / W) % H), b = (int)(q / ((long long)W * H));
    const long long pq = ((long long)b * (H / 2) + y / 2) * (W / 2) + x / 2;
    float ds[8], dp[8], av[8], o[8];
    ld8(dskip + q * lds + soff + ch, ds);
    ld8(dpool + pq * ldp + poff + ch, dp);
    ld8(act + q * lda + aoff + ch, av);
#pragma unroll
    for (int j = 0; j < 8; ++j) o[j] = av[j] > 0.0f ? ds[j] + 0.25f * dp[j] : 0.0f;
    st8(out + q * ldo + ooff + ch, o);
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
__global__ void k_upsample2(const __nv_bfloat16 *in, int ldi, int ioff, __nv_bfloat16 *out, int ldo, int ooff,
                            int B, int Hi, int Wi, int c) {
  const int Ho = 2 * Hi, Wo = 2 * Wi, c8 = c / 8;
  const long long total = (long long)B * Ho * Wo * c8;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(i % c8) * 8;
    const long long q = i / c8;
    const int x = (int)(q % Wo), y = (int)((q / Wo) % Ho), b = (int)(q / ((long long)Wo * Ho));
    int y0, y1, x0, x1;
    float wy0, wy1, wx0, wx1;
    up_taps(y, Hi, y0, y1, wy0, wy1);
    up_taps(x, Wi, x0, x1, wx0, wx1);
    const __nv_bfloat16 *base = in + ioff + ch;
    float a00[8], a01[8], a10[8], a11[8], o[8];
    ld8(base + (((long long)b * Hi + y0) * Wi + x0) * ldi, a00);
    ld8(base + (((long long)b * Hi + y0) * Wi + x1) * ldi, a01);
    ld8(base + (((long long)b * Hi + y1) * Wi + x0) * ldi, a10);
    ld8(base + (((long long)b * Hi + y1) * Wi + x1) * ldi, a11);
#pragma unroll
    for (int j = 0; j < 8; ++j)
      o[j] = wy0 * (wx0 * a00[j] + wx1 * a01[j]) + wy1 * (wx0 * a10[j] + wx1 * a11[j]);
    st8(out + q * ldo + ooff + ch, o);
  }
}
// Adjoint of k_upsample2 (a gather over the outputs that read each input),
// times the ReLU mask of the upsampled activation.
__global__ void k_upsample2_bwd(const __nv_bfloat16 *dout, int ldd, int doff, const __nv_bfloat16 *act, int lda,
                                int aoff, __nv_bfloat16 *din, int ldo, int ooff, int B, int Hi, int Wi, int c) {
  const int Ho = 2 * Hi, Wo = 2 * Wi, c8 = c / 8;
  const long long total = (long long)B * Hi * Wi * c8;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(i % c8) * 8;
    const long long q = i / c8;
    const int x = (int)(q % Wi), y = (int)((q / Wi) % Hi), b = (int)(q / ((long long)Wi * Hi));
    // output rows that read input row y: 2y, 2y+1 (weight 0.75), 2y-1 and 2y+2
    // (weight 0.25), plus the clamped border rows
    float wyv[4], wxv[4];
    int oy[4], ox[4];
    int ny = 0, nx = 0;
    for (int o = max(2 * y - 1, 0); o <= min(2 * y + 2, Ho - 1); ++o) {
      int i0, i1;
      float w0, w1;
      up_taps(o, Hi, i0, i1, w0, w1);
      const float wgt = (i0 == y ? w0 : 0.0f) + (i1 == y ? w1 : 0.0f);
      if (wgt != 0.0f) { oy[ny] = o; wyv[ny] = wgt; ++ny; }
    }
    for (int o = max(2 * x - 1, 0); o <= min(2 * x + 2, Wo - 1); ++o) {
      int i0, i1;
      float w0, w1;
      up_taps(o, Wi, i0, i1, w0, w1);
      const float wgt = (i0 == x ? w0 : 0.0f) + (i1 == x ? w1 : 0.0f);
      if (wgt != 0.0f) { ox[nx] = o; wxv[nx] = wgt; ++nx; }
    }
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0}, v[8], av[8];
    for (int a1 = 0; a1 < ny; ++a1)
      for (int a2 = 0; a2 < nx; ++a2) {
        ld8(dout + (((long long)b * Ho + oy[a1]) * Wo + ox[a2]) * ldd + doff + ch, v);
        const float wgt = wyv[a1] * wxv[a2];
#pragma unroll
        for (int j = 0; j < 8; ++j) s[j] += wgt * v[j];
      }
    ld8(act + q * lda + aoff + ch, av);
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (!(av[j] > 0.0f)) s[j] = 0.0f;
    st8(din + q * ldo + ooff + ch, s);
  }
}

// ----------------------------------------------------------------------------
// head (1x1 conv c -> 1), loss, optimiser, input features
// ----------------------------------------------------------------------------
__global__ void k_head_fwd(const __nv_bfloat16 *x, int ldx, int c, const float *w, const float *b, float *pred,
                           long long P) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    float s = b[0];
    for (int k = 0; k < c; ++k) s += bf2f(x[p * ldx + k]) * w[k];
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
__global__ void k_head_bwd(const __nv_bfloat16 *x, int ldx, int c, const float *w, const float *dpred, long long P,
                           __nv_bfloat16 *dx, int lddx, float *part /* [blocks][c+1] */) {
  extern __shared__ float shw[];  // blockDim.x * (c + 1)
  float accw[16];
  float accb = 0.0f;
  for (int k = 0; k < 16; ++k) accw[k] = 0.0f;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const float g = dpred[p];
    accb += g;
    for (int k = 0; k < c; ++k) {
      const float xv = bf2f(x[p * ldx + k]);
      accw[k] += g * xv;
      dx[p * lddx + k] = __float2bfloat16_rn(xv > 0.0f ? g * w[k] : 0.0f);
    }
  }
  for (int k = 0; k < c; ++k) shw[threadIdx.x * (c + 1) + k] = accw[k];
  shw[threadIdx.x * (c + 1) + c] = accb;
  __syncthreads();
  if (threadIdx.x <= (unsigned)c) {
    float s = 0.0f;
    for (int t = 0; t < (int)blockDim.x; ++t) s += shw[t * (c + 1) + threadIdx.x];
    part[(long long)blockIdx.x * (c + 1) + threadIdx.x] = s;
  }
}

// Adam (Kingma & Ba): m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
// w -= lr * mhat / (sqrt(vhat) + eps); refreshes the bf16 copy.
__global__ void k_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, long long n, float lr,
                       float b1, float b2, float eps, float bc1, float bc2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
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

// fp32 features (B x H x W x 4) -> bf16 input tensor padded to 16 channels.
__global__ void k_features_to_input(const float *f, __nv_bfloat16 *x, long long P) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P * 16;
       i += (long long)gridDim.x * blockDim.x) {
    const long long p = i / 16;
    const int c = (int)(i % 16);
    x[i] = __float2bfloat16_rn(c < 4 ? f[p * 4 + c] : 0.0f);
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
template <int N>
static cudaError_t launch_conv_t(const ConvArgs &a, cudaStream_t st) {
  const ConvChunking ck = conv_chunking(a.cin);
  if (a.cin % 16 != 0 || ck.kc % 16 != 0 || ck.kc * ck.cpt != a.cin) return cudaErrorInvalidValue;
  const int smem_raw = ck.stages * (128 + N) * ck.kmax * 2;
  // cap the CTAs per SM so that their TMEM columns always fit the SM's 512
  constexpr int cols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  constexpr int min_smem = cols >= 256 ? 80 * 1024 : (cols >= 128 ? 60 * 1024 : (cols >= 64 ? 30 * 1024 : 0));
  const int smem = smem_raw > min_smem ? smem_raw : min_smem;
  cudaError_t e = cudaFuncSetAttribute(k_conv3x3<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  const long long P = (long long)a.B * a.H * a.W;
  k_conv3x3<N><<<(unsigned)((P + 127) / 128), 128, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_conv3x3(const ConvArgs &a, int n, cudaStream_t st) {
  switch (n) {
    case 16: return launch_conv_t<16>(a, st);
    case 32: return launch_conv_t<32>(a, st);
    case 48: return launch_conv_t<48>(a, st);
    case 64: return launch_conv_t<64>(a, st);
    case 96: return launch_conv_t<96>(a, st);
    case 128: return launch_conv_t<128>(a, st);
    case 192: return launch_conv_t<192>(a, st);
    default: return cudaErrorInvalidValue;
  }
}

template <int N>
static cudaError_t launch_wgrad_t(const WgradArgs &a, cudaStream_t st, int nchunks) {
  constexpr int smem_raw = 2 * (128 * KP * 2 + N * KP * 2);
  constexpr int cols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  constexpr int min_smem = cols >= 256 ? 80 * 1024 : (cols >= 128 ? 60 * 1024 : (cols >= 64 ? 30 * 1024 : 0));
  constexpr int smem = smem_raw > min_smem ? smem_raw : min_smem;
  cudaError_t e = cudaFuncSetAttribute(k_wgrad<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_wgrad<N><<<dim3(nchunks, 9), 128, smem, st>>>(a);
  return cudaGetLastError();
}

int wgrad_chunks(int B, int H, int W) {
  const long long P = (long long)B * H * W;
  return (int)((P + kWgPix - 1) / kWgPix);
}

cudaError_t launch_wgrad(const WgradArgs &a, int cin, cudaStream_t st) {
  if (a.cout > 128 || a.cout % 8 != 0) return cudaErrorInvalidValue;
  const int nch = wgrad_chunks(a.B, a.H, a.W);
  cudaError_t e;
  switch (cin) {
    case 16: e = launch_wgrad_t<16>(a, st, nch); break;
    case 32: e = launch_wgrad_t<32>(a, st, nch); break;
    case 48: e = launch_wgrad_t<48>(a, st, nch); break;
    case 64: e = launch_wgrad_t<64>(a, st, nch); break;
    case 96: e = launch_wgrad_t<96>(a, st, nch); break;
    case 128: e = launch_wgrad_t<128>(a, st, nch); break;
    case 192: e = launch_wgrad_t<192>(a, st, nch); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  k_wgrad_reduce<<<256, 256, 0, st>>>(a.part, nch, a.cout, cin, a.dw);
  return cudaGetLastError();
}

cudaError_t launch_wgrad_reduce(const float *part, int nchunks, int cout, int cin, float *dw, cudaStream_t st) {
  k_wgrad_reduce<<<256, 256, 0, st>>>(part, nchunks, cout, cin, dw);
  return cudaGetLastError();
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

constexpr int kColsumChunk = 1024;  // pixels per bias-gradient block
cudaError_t launch_colsum(const __nv_bfloat16 *dy, int ld, int off, int c, long long P, float *part,
                          float *out, cudaStream_t st) {
  if (c > 256 || 256 % c != 0) return cudaErrorInvalidValue;
  const int nparts = colsum_parts(P);
  k_colsum<<<nparts, 256, 0, st>>>(dy, ld, off, c, P, kColsumChunk, part);
  k_colsum_reduce<<<c, 32, 0, st>>>(part, nparts, c, out);
  return cudaGetLastError();
}
int colsum_parts(long long P) { return (int)((P + kColsumChunk - 1) / kColsumChunk); }

cudaError_t launch_avgpool2(const __nv_bfloat16 *in, int ldi, int ioff, __nv_bfloat16 *out, int ldo, int ooff,
                            int B, int H, int W, int c, cudaStream_t st) {
  if (c % 8 || ldi % 8 || ioff % 8 || ldo % 8 || ooff % 8) return cudaErrorInvalidValue;
  k_avgpool2<<<blocks_for((long long)B * H * W * c / 32, 256), 256, 0, st>>>(in, ldi, ioff, out, ldo, ooff, B, H,
                                                                           W, c);
  return cudaGetLastError();
}
cudaError_t launch_unpool_add_mask(const __nv_bfloat16 *dskip, int lds, int soff, const __nv_bfloat16 *dpool,
                                   int ldp, int poff, const __nv_bfloat16 *act, int lda, int aoff,
                                   __nv_bfloat16 *out, int ldo, int ooff, int B, int H, int W, int c,
                                   cudaStream_t st) {
  if (c % 8 || lds % 8 || soff % 8 || ldp % 8 || poff % 8 || lda % 8 || aoff % 8 || ldo % 8 || ooff % 8)
    return cudaErrorInvalidValue;
  k_unpool_add_mask<<<blocks_for((long long)B * H * W * c / 8, 256), 256, 0, st>>>(
      dskip, lds, soff, dpool, ldp, poff, act, lda, aoff, out, ldo, ooff, B, H, W, c);
  return cudaGetLastError();
}
cudaError_t launch_upsample2(const __nv_bfloat16 *in, int ldi, int ioff, __nv_bfloat16 *out, int ldo, int ooff,
                             int B, int Hi, int Wi, int c, cudaStream_t st) {
  if (c % 8 || ldi % 8 || ioff % 8 || ldo % 8 || ooff % 8) return cudaErrorInvalidValue;
  k_upsample2<<<blocks_for((long long)B * Hi * Wi * 4 * c / 8, 256), 256, 0, st>>>(in, ldi, ioff, out, ldo, ooff, B,
                                                                               Hi, Wi, c);
  return cudaGetLastError();
}
cudaError_t launch_upsample2_bwd(const __nv_bfloat16 *dout, int ldd, int doff, const __nv_bfloat16 *act, int lda,
                                 int aoff, __nv_bfloat16 *din, int ldo, int ooff, int B, int Hi, int Wi, int c,
                                 cudaStream_t st) {
  if (c % 8 || ldd % 8 || doff % 8 || lda % 8 || aoff % 8 || ldo % 8 || ooff % 8) return cudaErrorInvalidValue;
  k_upsample2_bwd<<<blocks_for((long long)B * Hi * Wi * c / 8, 256), 256, 0, st>>>(dout, ldd, doff, act, lda, aoff,
                                                                               din, ldo, ooff, B, Hi, Wi, c);
  return cudaGetLastError();
}
cudaError_t launch_head_fwd(const __nv_bfloat16 *x, int ldx, int c, const float *w, const float *b, float *pred,
                            long long P, cudaStream_t st) {
  k_head_fwd<<<blocks_for(P, 256), 256, 0, st>>>(x, ldx, c, w, b, pred, P);
  return cudaGetLastError();
}
int head_bwd_blocks(long long P) { return (int)blocks_for(P, 256); }
cudaError_t launch_head_bwd(const __nv_bfloat16 *x, int ldx, int c, const float *w, const float *dpred,
                            long long P, __nv_bfloat16 *dx, int lddx, float *part, cudaStream_t st) {
  if (c > 16) return cudaErrorInvalidValue;
  const int nb = head_bwd_blocks(P);
  k_head_bwd<<<nb, 256, 256 * (c + 1) * sizeof(float), st>>>(x, ldx, c, w, dpred, P, dx, lddx, part);
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
cudaError_t launch_prep_weights(const float *w, int cout, int cin, __nv_bfloat16 *wb, __nv_bfloat16 *wt,
                                cudaStream_t st) {
  k_prep_weights<<<blocks_for((long long)cout * 9 * cin, 256), 256, 0, st>>>(w, cout, cin, wb, wt);
  return cudaGetLastError();
}
cudaError_t launch_features_to_input(const float *f, __nv_bfloat16 *x, long long P, cudaStream_t st) {
  k_features_to_input<<<blocks_for(P * 16, 256), 256, 0, st>>>(f, x, P);
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
