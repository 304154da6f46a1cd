// conv_tma.cu -- persistent, warp-specialised 3x3 convolutions on tcgen05 with
// TMA halo loads, for layers whose width is a multiple of 128 pixels.
//
// Tiling. A tile is one 128-pixel segment of one image row. For channel group j
// (8 channels) TMA loads the halo box {8 channels, 130 pixels, 3 rows}
// starting at (x0 - 1, y0 - 1); out-of-image pixels read as zero, which is the
// convolution's zero padding. The box lands in shared memory as 390 rows of 16
// bytes (row = pixel, 8 channels), so pixel (r, c) of the halo sits at row
// r * 130 + c. In the canonical no-swizzle layout consecutive rows are
// consecutive core-matrix rows along M (K-major operand) or K (MN-major
// operand), so the operand of tap (dy, dx) for output pixel m is row
// (1 + dy) * 130 + 1 + dx + m: a shift of the descriptor's start address by
// 16 bytes per pixel. One halo tile therefore feeds all nine taps.
//
// k_conv_tma<N> (forward / backward-data): GEMM rows = the segment's 128
// pixels, columns = N output channels, K = (tap, channel). The weights stay
// resident in shared memory (K-major, loaded once per CTA). Roles: warp 4 lane
// 0 issues the TMA loads into a ring of stages (full/empty mbarriers), warp 5
// allocates TMEM and its lane 0 issues the MMAs into one of two TMEM
// accumulators, warps 0-3 run the epilogue of the other accumulator (bias,
// ReLU, ReLU mask -> bf16 stores).
//
// k_wgrad_tma<CIN> (backward-weights): D[co][tap][ci] += sum over the
// segment's pixels of dY[p][co] X[p + off(tap)][ci]; GEMM rows = output
// channels (padded to 128: rows past cout read whatever follows in shared
// memory and their accumulators are never stored), columns = input channels,
// K = pixels. A is the dY segment (MN-major, one box {8, 128, 1} per channel
// group), B the X halo (MN-major). Each CTA accumulates its taps over a fixed
// range of segments in TMEM and writes one fp32 partial per (tap, co, ci);
// the partials are summed in chunk order by k_wgrad_reduce.
//
// Every wait is bounded in time; a CTA whose wait expires sets the error word,
// stops issuing, drains its copies and MMAs (bounded), frees its TMEM and
// returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "tc.cuh"
#include "unet_kernels.h"

namespace unet {

constexpr int kSeg = 128;              // pixels per tile
constexpr int kHaloW = kSeg + 2;       // halo pixels per row
constexpr int kHaloRows = 3 * kHaloW;  // 390
constexpr int kHaloBytes = 6272;       // 390 rows x 16 B, padded to a multiple of 128
constexpr int kSegBytes = kSeg * 16;   // one channel group of a segment (dY box)
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait on an mbarrier phase (wall-clock limit).
__device__ __forceinline__ bool wait_phase(uint64_t *mbar, uint32_t parity) {
  const unsigned long long t0 = now_ns();
  while (true) {
    if (mbar_wait(mbar, parity, 64)) return true;
    if (now_ns() - t0 > kWaitNs) return false;
  }
}
__device__ __forceinline__ uint32_t pow2_cols(int n) {
  uint32_t c = 32;
  while ((int)c < n) c <<= 1;
  return c;
}

// --------------------------------------------------------------------------
// forward / backward-data
// --------------------------------------------------------------------------
struct ConvTmaGeom {
  int segs_x, ntiles;   // segments per row (W / 128), tiles = B * H * segs_x
  int nst;              // pipeline stages
  int w_bytes;          // resident weight bytes (N * 9 * cin * 2, rounded to 1024)
};

template <int N>
__global__ void __launch_bounds__(192, 1)
    k_conv_tma(const __grid_constant__ CUtensorMap xmap, ConvArgs a, ConvTmaGeom g) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t full[4], empty[4], tfull[2], tempty[2], drain;
  __shared__ uint32_t tbase;
  __shared__ int s_abort, s_issued, s_consumed;
  __shared__ float sbias[N];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g8 = a.cin / 8;           // channel groups of the input
  const int KK = 9 * g8;              // 8-element K groups of the weights
  const int stage_bytes = g8 * kHaloBytes;
  unsigned char *sW = sm;
  unsigned char *sA = sm + g.w_bytes;
  const uint32_t acc_cols = pow2_cols(N);
  const uint32_t ncols = 2 * acc_cols;

  if (warp == 5) tmem_alloc(&tbase, ncols);
  if (tid == 0) {
    for (int s = 0; s < g.nst; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int k = 0; k < 2; ++k) {
      mbar_init(&tfull[k], 1);
      mbar_init(&tempty[k], 4);
    }
    mbar_init(&drain, 1);
    s_abort = 0;
    s_issued = 0;
    s_consumed = 0;
  }
  // resident weights, K-major core matrices: row n, K group kk = tap * g8 + j
  for (int idx = tid; idx < N * KK; idx += blockDim.x) {
    const int n = idx / KK, kk = idx - n * KK;
    cp16(sW + kmajor_off(n, kk, N / 8), a.w + (long long)n * 9 * a.cin + kk * 8, true);
  }
  cp_commit();
  for (int n = tid; n < N; n += blockDim.x) sbias[n] = a.bias ? a.bias[n] : 0.0f;
  cp_wait<0>();
  fence_async_smem();
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t tm = tbase;
  const int HW = a.H * g.segs_x;  // tiles per image

  if (warp == 4) {
    // ---------------- producer ----------------
    if (lane == 0) {
      int it = 0;
      for (int tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x, ++it) {
        const int s = it % g.nst;
        if (!wait_phase(&empty[s], ((it / g.nst) & 1) ^ 1) || *(volatile int *)&s_abort) {
          atomicExch(&s_abort, 1);
          break;
        }
        const int b = tile / HW, r = tile - b * HW, y = r / g.segs_x, x0 = (r - y * g.segs_x) * kSeg;
        mbar_arrive_expect_tx(&full[s], (uint32_t)(g8 * kHaloRows * 16));
        for (int j = 0; j < g8; ++j)
          tma_load_4d(sA + s * stage_bytes + j * kHaloBytes, &xmap, a.x_off + j * 8, x0 - 1, y - 1, b, &full[s]);
        s_issued = it + 1;
      }
    }
  } else if (warp == 5) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = instr_desc_bf16(128, N, false, false);
      int it = 0;
      for (int tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x, ++it) {
        const int s = it % g.nst, acc = it & 1;
        if (!wait_phase(&tempty[acc], ((it >> 1) & 1) ^ 1) || !wait_phase(&full[s], (it / g.nst) & 1) ||
            *(volatile int *)&s_abort) {
          atomicExch(&s_abort, 1);
          break;
        }
        tc_fence_after_sync();
        const uint32_t a0 = smem_u32(sA + s * stage_bytes), b0 = smem_u32(sW);
        const uint32_t d = tm + acc * acc_cols;
        bool first = true;
        for (int tap = 0; tap < 9; ++tap) {
          const int dy = tap / 3 - 1, dx = tap % 3 - 1;
          const uint32_t arow = a0 + (uint32_t)(((1 + dy) * kHaloW + 1 + dx) * 16);
          for (int j = 0; j < g8; j += 2) {
            const uint64_t ad = smem_desc(arow + j * kHaloBytes, kHaloBytes, 128);
            const uint64_t bd = smem_desc(b0 + (tap * g8 + j) * (N / 8) * 128, (N / 8) * 128, 128);
            mma_bf16(d, ad, bd, idesc, first ? 0u : 1u);
            first = false;
          }
        }
        mma_commit(&empty[s]);
        mma_commit(&tfull[acc]);
        s_consumed = it + 1;
      }
    }
  } else {
    // ---------------- epilogue (warps 0-3: TMEM lanes 32w..32w+31) ----------------
    int it = 0;
    for (int tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x, ++it) {
      const int acc = it & 1;
      // lane 0 decides for the warp: tmem loads below are warp-collective
      int go = 0;
      if (lane == 0) {
        go = wait_phase(&tfull[acc], (it >> 1) & 1) && !*(volatile int *)&s_abort;
        if (!go) atomicExch(&s_abort, 1);
      }
      if (!__shfl_sync(0xffffffffu, go, 0)) break;
      __syncwarp();
      tc_fence_after_sync();
      const int b = tile / HW, r = tile - b * HW, y = r / g.segs_x, x = (r - y * g.segs_x) * kSeg + 32 * warp + lane;
      const long long p = ((long long)b * a.H + y) * a.W + x;
      const uint32_t taddr = tm + acc * acc_cols + ((uint32_t)(32 * warp) << 16);
#pragma unroll 1
      for (int c16 = 0; c16 < N / 16; ++c16) {
        uint32_t rr[16];
        tmem_ld16(taddr + c16 * 16, rr);
        float v[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          float f = __uint_as_float(rr[k]) + sbias[c16 * 16 + k];
          if (a.relu) f = fmaxf(f, 0.0f);
          v[k] = f;
        }
        if (a.mask) {
          const __nv_bfloat16 *m = a.mask + p * a.ldm + a.m_off + c16 * 16;
#pragma unroll
          for (int k = 0; k < 16; ++k)
            if (!(__bfloat162float(m[k]) > 0.0f)) v[k] = 0.0f;
        }
        __align__(16) __nv_bfloat16 o[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) o[k] = __float2bfloat16_rn(v[k]);
        uint4 *dst = reinterpret_cast<uint4 *>(a.y + p * a.ldy + a.y_off + c16 * 16);
        dst[0] = reinterpret_cast<const uint4 *>(o)[0];
        dst[1] = reinterpret_cast<const uint4 *>(o)[1];
      }
      tc_fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[acc]);
    }
  }

  __syncthreads();
  if (s_abort && tid == 0) atomicExch(a.err, 1);
  if (warp == 5 && lane == 0) {
    // drain: loads issued but never consumed (only after an abort), then
    // every MMA issued and the barrier arrivals they signal
    for (int it = s_consumed; it < s_issued; ++it) wait_phase(&full[it % g.nst], (it / g.nst) & 1);
    mma_commit(&drain);
    wait_phase(&drain, 0);
  }
  tc_fence_before_sync();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after_sync();
    tmem_dealloc(tm, ncols);
  }
}

// --------------------------------------------------------------------------
// backward-weights
// --------------------------------------------------------------------------
struct WgradTmaGeom {
  int segs_x, nseg;     // segments per row, segments in total
  int seg_per_chunk;    // consecutive segments per CTA (blockIdx.x)
  int tpc;              // taps per CTA (blockIdx.y selects the group)
  int nst;
  int a_bytes;          // dY bytes of one stage (cout / 8 groups)
};

template <int CIN>
__global__ void __launch_bounds__(192, 1)
    k_wgrad_tma(const __grid_constant__ CUtensorMap dymap, const __grid_constant__ CUtensorMap xmap, WgradArgs a,
                WgradTmaGeom g) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t full[4], empty[4], done, drain;
  __shared__ uint32_t tbase;
  __shared__ int s_abort, s_issued, s_consumed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int G8 = CIN / 8;
  const int ga = a.cout / 8;
  const int stage_bytes = g.a_bytes + G8 * kHaloBytes;
  const int tap0 = blockIdx.y * g.tpc, ntap = min(g.tpc, 9 - tap0);
  const uint32_t ncols = pow2_cols(g.tpc * CIN);
  const int seg0 = blockIdx.x * g.seg_per_chunk;
  const int nitems = max(0, min(g.seg_per_chunk, g.nseg - seg0));
  const int HW = a.H * g.segs_x;

  if (warp == 5) tmem_alloc(&tbase, ncols);
  if (tid == 0) {
    for (int s = 0; s < g.nst; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    mbar_init(&drain, 1);
    s_abort = 0;
    s_issued = 0;
    s_consumed = 0;
  }
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t tm = tbase;

  if (warp == 4) {
    if (lane == 0) {
      for (int it = 0; it < nitems; ++it) {
        const int s = it % g.nst;
        if (!wait_phase(&empty[s], ((it / g.nst) & 1) ^ 1) || *(volatile int *)&s_abort) {
          atomicExch(&s_abort, 1);
          break;
        }
        const int seg = seg0 + it;
        const int b = seg / HW, r = seg - b * HW, y = r / g.segs_x, x0 = (r - y * g.segs_x) * kSeg;
        unsigned char *st = sm + s * stage_bytes;
        mbar_arrive_expect_tx(&full[s], (uint32_t)(ga * kSegBytes + G8 * kHaloRows * 16));
        for (int j = 0; j < ga; ++j)
          tma_load_4d(st + j * kSegBytes, &dymap, a.dy_off + j * 8, x0, y, b, &full[s]);
        for (int j = 0; j < G8; ++j)
          tma_load_4d(st + g.a_bytes + j * kHaloBytes, &xmap, a.x_off + j * 8, x0 - 1, y - 1, b, &full[s]);
        s_issued = it + 1;
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      const uint32_t idesc = instr_desc_bf16(128, CIN, true, true);
      int it = 0;
      for (; it < nitems; ++it) {
        const int s = it % g.nst;
        if (!wait_phase(&full[s], (it / g.nst) & 1) || *(volatile int *)&s_abort) {
          atomicExch(&s_abort, 1);
          break;
        }
        tc_fence_after_sync();
        const uint32_t a0 = smem_u32(sm + s * stage_bytes), b0 = a0 + g.a_bytes;
        for (int t = 0; t < ntap; ++t) {
          const int tap = tap0 + t, dy = tap / 3 - 1, dx = tap % 3 - 1;
          const uint32_t brow = b0 + (uint32_t)(((1 + dy) * kHaloW + 1 + dx) * 16);
          for (int k = 0; k < kSeg / 16; ++k) {
            // A: co groups at kSegBytes, pixel groups at 128; B: ci groups at
            // kHaloBytes, pixel groups at 128
            const uint64_t ad = smem_desc(a0 + k * 256, 128, kSegBytes);
            const uint64_t bd = smem_desc(brow + k * 256, 128, kHaloBytes);
            mma_bf16(tm + t * CIN, ad, bd, idesc, (it > 0 || k > 0) ? 1u : 0u);
          }
        }
        mma_commit(&empty[s]);
        s_consumed = it + 1;
      }
      if (!s_abort) mma_commit(&done);
    }
  }
  __syncthreads();
  bool ok = !s_abort;
  if (ok && nitems > 0) {
    if (warp < 4) {
      bool w = lane == 0 ? wait_phase(&done, 0) : true;
      w = __shfl_sync(0xffffffffu, w ? 1 : 0, 0) != 0;
      if (!w && lane == 0) atomicExch(&s_abort, 1);
    }
  }
  __syncthreads();
  ok = !s_abort;
  if (ok && warp < 4) {
    tc_fence_after_sync();
    const int co = 32 * warp + lane;
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    for (int t = 0; t < ntap; ++t) {
      float *dst = a.part + (((long long)blockIdx.x * 9 + tap0 + t) * a.cout + co) * CIN;
#pragma unroll 1
      for (int c16 = 0; c16 < CIN / 16; ++c16) {
        uint32_t rr[16];
        tmem_ld16(tm + lane_base + t * CIN + c16 * 16, rr);
        if (co < a.cout) {
#pragma unroll
          for (int k = 0; k < 16; ++k) dst[c16 * 16 + k] = nitems > 0 ? __uint_as_float(rr[k]) : 0.0f;
        }
      }
    }
  }
  if (!ok && tid == 0) atomicExch(a.err, 1);
  if (warp == 5 && lane == 0) {
    for (int it = s_consumed; it < s_issued; ++it) wait_phase(&full[it % g.nst], (it / g.nst) & 1);
    mma_commit(&drain);
    wait_phase(&drain, 0);
  }
  tc_fence_before_sync();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after_sync();
    tmem_dealloc(tm, ncols);
  }
}

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// NHWC bf16 activation (pitch ld channels) as a 4-D tensor map {ld, W, H, B}
// with box {8, box_w, box_h, 1}.
static bool act_map(CUtensorMap *m, const void *base, int B, int H, int W, int ld, int box_w, int box_h) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)ld, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
  const cuuint64_t strides[3] = {(cuuint64_t)ld * 2, (cuuint64_t)W * ld * 2, (cuuint64_t)H * W * ld * 2};
  const cuuint32_t box[4] = {8, (cuuint32_t)box_w, (cuuint32_t)box_h, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

constexpr int kSmemCap = 227 * 1024;

static int pow2_host(int n) {
  int c = 32;
  while (c < n) c <<= 1;
  return c;
}

bool conv_tma_ok(const ConvArgs &a, int n) {
  if (a.W % kSeg != 0 || a.cin % 16 != 0 || a.cin > 128) return false;
  if (n != 16 && n != 32 && n != 48 && n != 64 && n != 96) return false;
  const int w_bytes = (n * 9 * a.cin * 2 + 1023) / 1024 * 1024;
  const int stage = a.cin / 8 * kHaloBytes;
  return w_bytes + 2 * stage <= kSmemCap - 4096 && encode_fn() != nullptr;
}

template <int N>
static cudaError_t launch_conv_tma_t(const ConvArgs &a, cudaStream_t st) {
  CUtensorMap xm;
  if (!act_map(&xm, a.x, a.B, a.H, a.W, a.ldx, kHaloW, 3)) return cudaErrorNotSupported;
  ConvTmaGeom g{};
  g.segs_x = a.W / kSeg;
  g.ntiles = a.B * a.H * g.segs_x;
  g.w_bytes = (N * 9 * a.cin * 2 + 1023) / 1024 * 1024;
  const int stage = a.cin / 8 * kHaloBytes;
  g.nst = 4;
  while (g.nst > 2 && g.w_bytes + g.nst * stage > kSmemCap - 4096) --g.nst;
  const int smem = g.w_bytes + g.nst * stage;
  cudaError_t e = cudaFuncSetAttribute(k_conv_tma<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  const int grid = g.ntiles < num_sms() ? g.ntiles : num_sms();
  k_conv_tma<N><<<grid, 192, smem, st>>>(xm, a, g);
  return cudaGetLastError();
}

cudaError_t launch_conv_tma(const ConvArgs &a, int n, cudaStream_t st) {
  switch (n) {
    case 16: return launch_conv_tma_t<16>(a, st);
    case 32: return launch_conv_tma_t<32>(a, st);
    case 48: return launch_conv_tma_t<48>(a, st);
    case 64: return launch_conv_tma_t<64>(a, st);
    case 96: return launch_conv_tma_t<96>(a, st);
    default: return cudaErrorInvalidValue;
  }
}

// Partial-sum chunks of the TMA weight-gradient path: a fixed count, so the
// order of the final sum does not depend on the device.
constexpr int kWgChunks = 296;

int wgrad_tma_chunks(int B, int H, int W) {
  const int nseg = B * H * (W / kSeg);
  const int per = (nseg + kWgChunks - 1) / kWgChunks;
  return (nseg + per - 1) / per;
}

bool wgrad_tma_ok(const WgradArgs &a, int cin) {
  if (a.W % kSeg != 0 || a.cout % 8 != 0 || a.cout > 128) return false;
  if (cin != 16 && cin != 32 && cin != 48 && cin != 64 && cin != 96 && cin != 128) return false;
  return encode_fn() != nullptr;
}

template <int CIN>
static cudaError_t launch_wgrad_tma_t(const WgradArgs &a, cudaStream_t st, int *chunks) {
  CUtensorMap dym, xm;
  if (!act_map(&dym, a.dy, a.B, a.H, a.W, a.lddy, kSeg, 1) || !act_map(&xm, a.x, a.B, a.H, a.W, a.ldx, kHaloW, 3))
    return cudaErrorNotSupported;
  WgradTmaGeom g{};
  g.segs_x = a.W / kSeg;
  g.nseg = a.B * a.H * g.segs_x;
  g.seg_per_chunk = (g.nseg + kWgChunks - 1) / kWgChunks;
  const int nchunks = (g.nseg + g.seg_per_chunk - 1) / g.seg_per_chunk;
  int tpc = 256 / CIN;
  if (tpc > 9) tpc = 9;
  const int ngroups = (9 + tpc - 1) / tpc;
  g.tpc = (9 + ngroups - 1) / ngroups;
  g.a_bytes = a.cout / 8 * kSegBytes;
  // A rows past cout address the bytes that follow the dY groups: keep the
  // full 128-row span (16 groups) inside the allocation
  const int stage = g.a_bytes + CIN / 8 * kHaloBytes;
  const int tail = 16 * kSegBytes - g.a_bytes;
  g.nst = 4;
  while (g.nst > 2 && g.nst * stage + tail > 110 * 1024) --g.nst;
  int smem = g.nst * stage + (tail > 0 ? tail : 0);
  // at most two CTAs per SM when each holds 256 TMEM columns
  if (pow2_host(g.tpc * CIN) >= 256 && smem < 80 * 1024) smem = 80 * 1024;
  if (smem > kSmemCap - 4096) return cudaErrorNotSupported;
  cudaError_t e = cudaFuncSetAttribute(k_wgrad_tma<CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_wgrad_tma<CIN><<<dim3(nchunks, ngroups), 192, smem, st>>>(dym, xm, a, g);
  *chunks = nchunks;
  return cudaGetLastError();
}

cudaError_t launch_wgrad_tma(const WgradArgs &a, int cin, cudaStream_t st, int *chunks) {
  switch (cin) {
    case 16: return launch_wgrad_tma_t<16>(a, st, chunks);
    case 32: return launch_wgrad_tma_t<32>(a, st, chunks);
    case 48: return launch_wgrad_tma_t<48>(a, st, chunks);
    case 64: return launch_wgrad_tma_t<64>(a, st, chunks);
    case 96: return launch_wgrad_tma_t<96>(a, st, chunks);
    case 128: return launch_wgrad_tma_t<128>(a, st, chunks);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace unet
