// conv_tma.cu -- persistent, warp-specialised 3x3 convolutions on tcgen05 with
// TMA halo loads, on activations in the channel-blocked layout
// [B][C/8][H][W][8] (unet_kernels.h).
//
// Tiling. A tile is R output rows (R = 1, 2 or 4) of one segment of SW pixels:
// SW = 128, or W rounded up to 16 for narrower images; a row's last segment
// may reach past W and the last row group past H (those pixels load as zero
// and are never stored). TMA sees a buffer as the 5-D tensor {CW * 8 elements,
// W / CW chunks, H rows, C/8 planes, B}: a plane row in chunks of CW pixels
// (CW = 16, or the largest power of two dividing W). One box {CW * 8, HP / CW
// chunks, R + 2 rows, planes, 1} starting one chunk left of the segment and
// one row above it brings the tile's whole halo: in shared memory, for each
// channel group g and halo row h, a row of HP 16-byte entries (one entry =
// one pixel's 8 channels) at entry (g * (R + 2) + h) * HP, entry CW being
// pixel x0. Pixels outside the image read as zero, the convolution's zero
// padding. In the canonical no-swizzle layout consecutive 16-byte entries are
// consecutive core-matrix rows along M (K-major operand) or K (MN-major
// operand), so the operand of tap (dy, dx) for output row r and pixel m is
// entry (g * (R + 2) + r + 1 + dy) * HP + CW + dx + m: a shift of the
// descriptor's start address by 16 bytes per pixel. One halo tile feeds all
// nine taps of all R rows.
//
// k_conv_tma<N> (forward / backward-data): per output row, GEMM rows = the
// segment's pixels (M = 128, or 64 when SW <= 64; rows past SW are never
// stored), columns = N
// output channels (the CTA's part [n0, n0 + N) of them: blockIdx.y), K = (tap,
// channel) taken in chunks of cg channel groups (chosen per layer, at most
// 64 channels) per pipeline stage: K groups (g, g+1) of one tap are (R + 2) *
// HP entries apart. The CTA's weights stay resident in shared memory. Roles:
// one warp's lane 0 issues TMA loads into a ring of stages (full/empty
// mbarriers); up to four issuer warps (lane 0 of each) issue the MMAs into
// one buffer per epilogue warpgroup, issuer i taking the accumulators of
// output rows i, i + nis, ... (nis = min(4, R); the first issuer also
// allocates TMEM); two warpgroups take alternate tiles through the epilogue
// (bias, ReLU, ReLU mask -> bf16).
//
// k_wgrad_tma<CP> (backward-weights, R = 1): D[co][tap][ci] += sum over the
// segment's pixels of dY[p][co] X[p + off(tap)][ci]. GEMM rows = output
// channels (padded to 128: rows past cout read whatever follows in shared
// memory and are never stored), K = pixels, and columns = (channel group, dy,
// channel): with one output row the halo rows of one part of CP channels are
// 3 * CP / 8 groups of 8 columns at a constant stride of HP entries, so one
// MMA covers the three dy taps of that part (N = 3 CP) and dx selects the
// start entry. A CTA owns a fixed
// range of segments, one part of the channels and one or all three dx values,
// accumulates in TMEM and writes one fp32 partial per (tap, co, ci); the
// partials are summed in chunk order by k_wgrad_reduce. The transposed form
// (cout <= 32) issues the three dx accumulators from three warps and, with 16
// channels per part (48 GEMM rows), uses M = 64 MMAs. The CTAs of the
// first channel part also sum dY over their segments for the bias gradient
// (one partial per chunk and output channel, summed by the same reduce).
//
// Every wait is bounded in time; a CTA whose wait expires sets the error word,
// stops issuing, drains its copies and MMAs (bounded), frees its TMEM and
// returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "tc.cuh"
#include "unet_kernels.h"

namespace unet {

constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s per wait
constexpr int kMaxStages = 8;                           // depth of the TMA ring
constexpr int kTail = 4096;                             // slack past the last stage (see the M/N spans)

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait on an mbarrier phase (wall-clock limit, kWaitNs by default).
// The clock is read only once a first round of polls has missed: most waits
// in the pipelines find their phase complete, and a global-timer read costs
// far more than a poll.
__device__ __forceinline__ bool wait_phase(uint64_t *mbar, uint32_t parity,
                                           unsigned long long limit_ns = kWaitNs) {
  if (mbar_wait(mbar, parity, 8)) return true;
  const unsigned long long t0 = now_ns();
  while (true) {
    if (mbar_wait(mbar, parity, 64)) return true;
    if (now_ns() - t0 > limit_ns) return false;
  }
}
__host__ __device__ inline uint32_t pow2_cols(int n) {
  uint32_t c = 32;
  while ((int)c < n) c <<= 1;
  return c;
}

// Segment geometry shared by both kernels.
struct SegGeom {
  int SW, CW, HP;       // segment width, TMA chunk width, halo row pitch (pixels)
  int R;                // output rows per tile
  int segs_x, ngr;      // segments per row, row groups per image
  int nseg;             // tiles in total: B * ngr * segs_x
  int nst;              // pipeline stages
};

// --------------------------------------------------------------------------
// forward / backward-data
// --------------------------------------------------------------------------
struct ConvTmaGeom {
  SegGeom s;
  int w_bytes;          // resident weight bytes of the CTA's part (rounded to 1024)
  int cg;               // channel groups per K chunk (pipeline stage): even, <= kMaxChunkGroups
};

constexpr int kEpiGroups = 2;  // epilogue warpgroups (one accumulator each)
// MMA issuers: one thread issues a tcgen05.mma about every 156 cycles
// whatever its shape, while the tensor core takes an M = 128, K = 16 MMA of
// N <= 32 every ~37 cycles (its 4 KB A operand read from shared memory); one
// issuer per output row of a tile (up to four per CTA) keeps the small-N
// layers on the tensor core's bound instead of the issue rate.
constexpr int kIssuers = 4;
constexpr int kConvThreads = 32 * (4 * kEpiGroups + 1 + kIssuers);  // + producer warp + issuers
constexpr int kProdWarp = 4 * kEpiGroups, kMmaWarp = 4 * kEpiGroups + 1;  // first issuer

constexpr int kMaxChunkGroups = 8;  // channel groups (64 channels) per pipeline stage, at most

template <int N>
__global__ void __launch_bounds__(kConvThreads, 2)
    k_conv_tma(const __grid_constant__ CUtensorMap xmap, ConvArgs a, ConvTmaGeom g) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t full[kMaxStages], empty[kMaxStages], tfull[kEpiGroups], tempty[kEpiGroups], drain;
  __shared__ uint32_t tbase;
  __shared__ int s_abort, s_issued, s_consumed[kIssuers];
  __shared__ float sbias[N];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g8 = a.cin / 8;           // channel groups of the input
  const int KK = 9 * g8;              // 8-element K groups of the weights
  const int CG = g.cg;                 // channel groups per K chunk
  const int nkc = (g8 + CG - 1) / CG;  // K chunks per tile
  const int SW = g.s.SW, HP = g.s.HP, CW = g.s.CW, R = g.s.R, nst = g.s.nst, ntiles = g.s.nseg;
  const int GB = min(g8, CG);            // planes per chunk box
  const int gstride = (R + 2) * HP;      // entries between channel groups of a stage
  const int stage_bytes = GB * gstride * 16;
  const int n0 = blockIdx.y * N;      // the CTA's output channels
  const int nis = min(kIssuers, R);   // issuers with rows: issuer i takes rows i, i + nis, ...
  // GEMM rows per MMA: 64 when the segment has at most 64 pixels (half the A
  // operand read per MMA); the accumulator's row m then sits in TMEM lane
  // (m % 16) + 32 (m / 16)
  const int MT = g.s.SW <= 64 ? 64 : 128;
  const unsigned long long wait_ns = a.wait_ns ? a.wait_ns : kWaitNs;
  unsigned char *sW = sm;
  unsigned char *sA = sm + g.w_bytes;
  const uint32_t acc_cols = pow2_cols(N);
  const uint32_t buf_cols = R * acc_cols;  // one accumulator per output row
  const uint32_t ncols = pow2_cols(kEpiGroups * buf_cols);

  if (warp == kMmaWarp) tmem_alloc(&tbase, ncols);
  if (tid == 0) {
    for (int s = 0; s < nst; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], nis);  // one commit per issuer
    }
    for (int k = 0; k < kEpiGroups; ++k) {
      mbar_init(&tfull[k], nis);
      mbar_init(&tempty[k], 4);
    }
    mbar_init(&drain, nis);
    s_abort = 0;
    s_issued = 0;
    for (int i = 0; i < kIssuers; ++i) s_consumed[i] = 0;
  }
  // resident weights of rows n0 .. n0+N-1, K-major core matrices: row n, K group kk = tap * g8 + j
  for (int idx = tid; idx < N * KK; idx += blockDim.x) {
    const int n = idx / KK, kk = idx - n * KK;
    cp16(sW + kmajor_off(n, kk, N / 8), a.w + (long long)(n0 + n) * 9 * a.cin + kk * 8, true);
  }
  cp_commit();
  for (int n = tid; n < N; n += blockDim.x) sbias[n] = a.bias ? a.bias[n0 + n] : 0.0f;
  cp_wait<0>();
  fence_async_smem();
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t tm = tbase;
  const int HW = g.s.ngr * g.s.segs_x;  // tiles per image

  if (warp == kProdWarp) {
    // ---------------- producer: one item = (tile, K chunk) ----------------
    if (lane == 0) {
      int it = 0;
      bool stop = false;
      for (int tile = blockIdx.x; tile < ntiles && !stop; tile += gridDim.x) {
        const int b = tile / HW, r = tile - b * HW, rg = r / g.s.segs_x, x0 = (r - rg * g.s.segs_x) * SW;
        for (int c = 0; c < nkc; ++c, ++it) {
          const int s = it % nst;
          if (!wait_phase(&empty[s], ((it / nst) & 1) ^ 1, wait_ns) || *(volatile int *)&s_abort) {
            atomicExch(&s_abort, 1);
            stop = true;
            break;
          }
          // the box is GB planes; planes past the buffer read as zero
          mbar_arrive_expect_tx(&full[s], (uint32_t)stage_bytes);
          tma_load_5d(sA + s * stage_bytes, &xmap, 0, x0 / CW - 1, rg * R - 1, a.x.g0 + c * CG, b,
                      &full[s]);
          s_issued = it + 1;
        }
      }
    }
  } else if (warp >= kMmaWarp) {
    // ---------------- MMA issuers: each owns the accumulators of its rows ----------------
    const int issuer = warp - kMmaWarp;
    if (lane == 0 && issuer < nis) {
      const uint32_t idesc = instr_desc_bf16(MT, N, false, false);
      // descriptors advance by adding (bytes >> 4) to their address field
      const uint64_t bdesc0 = smem_desc(smem_u32(sW), (N / 8) * 128, 128);
      const uint32_t bgrp = (uint32_t)((N / 8) * 128) >> 4;   // one K group of the weights
      const uint32_t astep = (uint32_t)(2 * gstride);          // two channel groups of the halo (entries)
      int it = 0, ti = 0;
      bool stop = false;
      // test knob (a.stall): wait first on a phase that nothing completes before
      // the drain below, so the wait runs out and the CTA takes the abort path
      if (a.stall && issuer == 0 && !wait_phase(&drain, 0, wait_ns)) {
        atomicExch(&s_abort, 1);
        stop = true;
      }
      for (int tile = blockIdx.x; tile < ntiles && !stop; tile += gridDim.x, ++ti) {
        const int acc = ti % kEpiGroups;
        if (!wait_phase(&tempty[acc], ((ti / kEpiGroups) & 1) ^ 1, wait_ns)) {
          atomicExch(&s_abort, 1);
          break;
        }
        for (int c = 0; c < nkc; ++c, ++it) {
          const int s = it % nst;
          if (!wait_phase(&full[s], (it / nst) & 1, wait_ns) || *(volatile int *)&s_abort) {
            atomicExch(&s_abort, 1);
            stop = true;
            break;
          }
          tc_fence_after_sync();
          const int gcn = min(CG, g8 - c * CG);
          const uint64_t adesc0 = smem_desc(smem_u32(sA + s * stage_bytes), gstride * 16, 128);
#pragma unroll 1
          for (int rr = issuer; rr < R; rr += nis) {
            const uint32_t d = tm + acc * buf_cols + rr * acc_cols;
            uint32_t accumulate = c > 0 ? 1u : 0u;
            for (int tap = 0; tap < 9; ++tap) {
              // entries of 16 bytes
              uint64_t ad = adesc0 + (uint32_t)((rr + tap / 3) * HP + CW - 1 + (tap % 3));
              uint64_t bd = bdesc0 + (uint32_t)(tap * g8 + c * CG) * bgrp;
              for (int j = 0; j < gcn; j += 2) {
                mma_bf16(d, ad, bd, idesc, accumulate);
                accumulate = 1;
                ad += astep;
                bd += 2 * bgrp;
              }
            }
          }
          mma_commit(&empty[s]);
          s_consumed[issuer] = it + 1;
        }
        if (stop) break;
        mma_commit(&tfull[acc]);
      }
    }
  } else {
    // ------- epilogue: warpgroup wg takes tiles wg, wg + kEpiGroups, ...;
    //         warp w reads TMEM lanes 32 (w % 4) .. + 31 -------
    const int wg = warp / 4, q = warp % 4;
    // GEMM row = pixel m of the segment; warp q reads TMEM lanes 32 q .. 32 q +
    // 31, which hold rows 32 q + lane (M = 128) or, for lanes below 16, rows
    // 16 q + lane (M = 64)
    const int m = MT == 64 ? 16 * q + lane : 32 * q + lane;
    const bool row_here = MT == 128 || lane < 16;
    int k = 0;
    for (int tile = blockIdx.x + wg * gridDim.x; tile < ntiles; tile += kEpiGroups * gridDim.x, ++k) {
      // lane 0 decides for the warp: tmem loads below are warp-collective
      int go = 0;
      if (lane == 0) {
        go = wait_phase(&tfull[wg], k & 1, wait_ns) && !*(volatile int *)&s_abort;
        if (!go) atomicExch(&s_abort, 1);
      }
      if (!__shfl_sync(0xffffffffu, go, 0)) break;
      tc_fence_after_sync();
      const int b = tile / HW, r = tile - b * HW, rg = r / g.s.segs_x, x = (r - rg * g.s.segs_x) * SW + m;
      const bool valid = row_here && m < SW && x < a.W;
#pragma unroll 1
      for (int orow = 0; orow < R; ++orow) {
      const int y = rg * R + orow;
      if (y >= a.H) break;  // uniform across the warp
      const uint32_t taddr = tm + wg * buf_cols + orow * acc_cols + ((uint32_t)(32 * q) << 16);
#pragma unroll 1
      for (int c16 = 0; c16 < N / 16; ++c16) {
        uint32_t rr[16];
        tmem_ld16(taddr + c16 * 16, rr);
        if (valid) {
          float v[16];
#pragma unroll
          for (int kk = 0; kk < 16; ++kk) {
            float f = __uint_as_float(rr[kk]) + sbias[c16 * 16 + kk];
            if (a.relu) f = fmaxf(f, 0.0f);
            v[kk] = f;
          }
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int grp = n0 / 8 + 2 * c16 + h;  // group of the output slice
            if (a.mask.p) {
              const uint4 mq = *reinterpret_cast<const uint4 *>(a.mask.p + act_index(a.mask, b, grp, y, x, a.H, a.W));
              const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(&mq);
#pragma unroll
              for (int kk = 0; kk < 8; ++kk)
                if (!(__bfloat162float(mb[kk]) > 0.0f)) v[8 * h + kk] = 0.0f;
            }
            __align__(16) __nv_bfloat16 o[8];
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) o[kk] = __float2bfloat16_rn(v[8 * h + kk]);
            *reinterpret_cast<uint4 *>(a.y.p + act_index(a.y, b, grp, y, x, a.H, a.W)) =
                *reinterpret_cast<const uint4 *>(o);
          }
        }
      }
      }
      tc_fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[wg]);
    }
  }

  __syncthreads();
  if (s_abort && tid == 0) atomicExch(a.err, 1);
  if (warp >= kMmaWarp && warp - kMmaWarp < nis && lane == 0) {
    // drain: loads issued but not consumed by every issuer (only after an
    // abort), then every MMA each issuer issued and the barrier arrivals
    // they signal
    if (warp == kMmaWarp) {
      int lo = s_issued;
      for (int i = 0; i < nis; ++i) lo = min(lo, s_consumed[i]);
      for (int it = lo; it < s_issued; ++it) wait_phase(&full[it % nst], (it / nst) & 1);
    }
    mma_commit(&drain);
    if (warp == kMmaWarp) wait_phase(&drain, 0);
  }
  tc_fence_before_sync();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after_sync();
    tmem_dealloc(tm, ncols);
  }
}

// --------------------------------------------------------------------------
// backward-weights
// --------------------------------------------------------------------------
struct WgradTmaGeom {
  SegGeom s;
  int seg_per_chunk;    // consecutive segments per CTA (blockIdx.x)
  int ndx;              // dx values per CTA (3, or 1: blockIdx.y % 3 picks it)
  int a_bytes;          // dY bytes of one stage (cout / 8 groups of SW rows)
};

// T = false: D[co][(group, dy, channel)] as described above. T = true (used
// when cout <= 32): the transposed product D[(group, dy, channel)][co], GEMM
// rows = the halo's 3 * CP / 8 (group, dy) groups (padded to 128 the same
// way), columns = the output channels: the same MMA count with N = cout
// instead of 3 * CP, a third of the tensor work when cout = 16 = CP.
// Warps: 0-3 epilogue, 4 producer, 5.. MMA issuers. With T the three dx
// accumulators are independent and each gets its own issuer (N = cout is
// small, so one issuer would bound the tensor core); without T, N = 3 CP is
// wide enough for one.
constexpr int kWgIssuers = 3;
constexpr int kWgThreads = 32 * (5 + kWgIssuers);

template <int CP, bool T>
__global__ void __launch_bounds__(kWgThreads, 2)
    k_wgrad_tma(const __grid_constant__ CUtensorMap dymap, const __grid_constant__ CUtensorMap xmap, WgradArgs a,
                WgradTmaGeom g) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t full[kMaxStages], empty[kMaxStages], done, drain;
  __shared__ uint32_t tbase;
  __shared__ int s_abort, s_issued, s_consumed[kWgIssuers];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int G8 = CP / 8;          // channel groups of the part
  constexpr int NC = 3 * CP;          // GEMM columns per dx: (group, dy, channel)
  // GEMM rows: with T and 3 CP <= 64 an M = 64 MMA (half the A operand read
  // per MMA); its accumulator row m sits in TMEM lane (m % 16) + 32 (m / 16)
  constexpr int kMT = (T && 3 * CP <= 64) ? 64 : 128;
  const int SW = g.s.SW, HP = g.s.HP, CW = g.s.CW, nst = g.s.nst;
  const int rowb = HP * 16;
  const int ga = a.cout / 8;
  const int stage_bytes = g.a_bytes + 3 * G8 * rowb;
  const int part = (g.ndx == 3) ? blockIdx.y : blockIdx.y / 3;
  const int dx0 = (g.ndx == 3) ? 0 : blockIdx.y % 3;  // index 0..2 of dx = -1..1
  const int c0 = part * CP;
  const int dcols = T ? a.cout : NC;  // accumulator columns per dx
  const uint32_t ncols = pow2_cols(g.ndx * dcols);
  const int seg0 = blockIdx.x * g.seg_per_chunk;
  const int nitems = max(0, min(g.seg_per_chunk, g.s.nseg - seg0));
  const int HW = a.H * g.s.segs_x;  // R = 1: one tile per row and segment
  const int nis = T ? min(kWgIssuers, g.ndx) : 1;  // issuer i takes dx t = i, i + nis, ...
  // the first CTA of each segment chunk also sums dY for the bias gradient
  // (warps 0-3, from the stages the MMAs read, while the MMAs run)
  const bool colsum = a.db != nullptr && blockIdx.y == 0;

  if (warp == 5) tmem_alloc(&tbase, ncols);
  if (tid == 0) {
    for (int s = 0; s < nst; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], nis + (colsum ? 4 : 0));  // one commit per issuer (+ the summing warps)
    }
    mbar_init(&done, nis);
    mbar_init(&drain, nis);
    s_abort = 0;
    s_issued = 0;
    for (int i = 0; i < kWgIssuers; ++i) s_consumed[i] = 0;
  }
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t tm = tbase;

  if (warp == 4) {
    if (lane == 0) {
      for (int it = 0; it < nitems; ++it) {
        const int s = it % nst;
        if (!wait_phase(&empty[s], ((it / nst) & 1) ^ 1) || *(volatile int *)&s_abort) {
          atomicExch(&s_abort, 1);
          break;
        }
        const int seg = seg0 + it;
        const int b = seg / HW, r = seg - b * HW, y = r / g.s.segs_x, x0 = (r - y * g.s.segs_x) * SW;
        unsigned char *st = sm + s * stage_bytes;
        mbar_arrive_expect_tx(&full[s], (uint32_t)(ga * SW * 16 + 3 * G8 * rowb));
        tma_load_5d(st, &dymap, 0, x0 / CW, y, a.dy.g0, b, &full[s]);
        tma_load_5d(st + g.a_bytes, &xmap, 0, x0 / CW - 1, y - 1, a.x.g0 + c0 / 8, b, &full[s]);
        s_issued = it + 1;
      }
    }
  } else if (warp >= 5) {
    const int issuer = warp - 5;
    if (lane == 0 && issuer < nis) {
      const uint32_t idesc = instr_desc_bf16(kMT, T ? a.cout : NC, true, true);
      for (int it = 0; it < nitems; ++it) {
        const int s = it % nst;
        if (!wait_phase(&full[s], (it / nst) & 1) || *(volatile int *)&s_abort) {
          atomicExch(&s_abort, 1);
          break;
        }
        tc_fence_after_sync();
        const uint32_t a0 = smem_u32(sm + s * stage_bytes), b0 = a0 + g.a_bytes;
        // A: co groups at SW rows, pixel groups at 128 bytes; B: (group, dy)
        // column groups at HP rows, pixel groups at 128 bytes. 16 pixels =
        // 256 bytes = 16 in the descriptors' address field.
        const uint64_t ydesc = smem_desc(a0, 128, SW * 16);
        for (int t = issuer; t < g.ndx; t += nis) {
          const uint64_t xdesc = smem_desc(b0 + (uint32_t)((CW - 1 + dx0 + t) * 16), 128, rowb);
          const uint64_t adesc0 = T ? xdesc : ydesc, bdesc0 = T ? ydesc : xdesc;
          const uint32_t d = tm + t * dcols;
          mma_bf16(d, adesc0, bdesc0, idesc, it > 0 ? 1u : 0u);
          for (int k = 1; k < SW / 16; ++k) mma_bf16(d, adesc0 + 16 * k, bdesc0 + 16 * k, idesc, 1u);
        }
        mma_commit(&empty[s]);
        s_consumed[issuer] = it + 1;
      }
      if (!s_abort) mma_commit(&done);
    }
  } else if (colsum) {
    // db partial of this chunk: warp w sums channel groups w, w + 4, ...;
    // lane l pixels l, l + 32, ... of each segment, segments in order, then
    // a fixed shuffle tree over the lanes. Stage layout: group g's SW pixels
    // of 8 channels at (g * SW + p) * 16 bytes; pixels past W load as zero.
    const int G = a.cout / 8;
    float acc[4][8];
#pragma unroll
    for (int gi = 0; gi < 4; ++gi)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[gi][j] = 0.0f;
    bool sum_ok = true;
    for (int it = 0; it < nitems; ++it) {
      const int s = it % nst;
      int go = 0;
      if (lane == 0) {
        go = wait_phase(&full[s], (it / nst) & 1) && !*(volatile int *)&s_abort;
        if (!go) atomicExch(&s_abort, 1);
      }
      if (!__shfl_sync(0xffffffffu, go, 0)) {
        sum_ok = false;
        break;
      }
      const unsigned char *st = sm + s * stage_bytes;
#pragma unroll
      for (int gi = 0; gi < 4; ++gi) {
        const int grp = warp + 4 * gi;
        if (grp < G)
          for (int p = lane; p < SW; p += 32) {
            const uint4 q = *reinterpret_cast<const uint4 *>(st + ((size_t)grp * SW + p) * 16);
            const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const float2 f = __bfloat1622float2(h[k]);
              acc[gi][2 * k] += f.x;
              acc[gi][2 * k + 1] += f.y;
            }
          }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
    if (sum_ok) {
#pragma unroll
      for (int gi = 0; gi < 4; ++gi) {
        const int grp = warp + 4 * gi;
        if (grp < G) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            float v = acc[gi][j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) a.db_part[(long long)blockIdx.x * a.cout + grp * 8 + j] = v;
          }
        }
      }
    }
  }
  __syncthreads();
  bool ok = !s_abort;
  if (ok && nitems > 0 && warp < 4) {
    bool w = lane == 0 ? wait_phase(&done, 0) : true;
    w = __shfl_sync(0xffffffffu, w ? 1 : 0, 0) != 0;
    if (!w && lane == 0) atomicExch(&s_abort, 1);
  }
  __syncthreads();
  ok = !s_abort;
  if (ok && warp < 4 && T) {
    tc_fence_after_sync();
    // GEMM row m: halo group k = m / 8 = 3 * group + (dy + 1), channel m % 8;
    // warp w reads TMEM lanes 32 w .. 32 w + 31, which hold rows 32 w + lane
    // (M = 128) or, for lanes below 16, rows 16 w + lane (M = 64)
    const int m = kMT == 64 ? 16 * warp + lane : 32 * warp + lane;
    const bool row_here = kMT == 128 || lane < 16;
    const int k = m >> 3, grp = k / 3, dyi = k - 3 * grp;
    const int ci = c0 + 8 * grp + (m & 7);
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    for (int t = 0; t < g.ndx; ++t) {
      const int tap = dyi * 3 + dx0 + t;
#pragma unroll 1
      for (int c16 = 0; c16 < a.cout / 16; ++c16) {
        uint32_t rr[16];
        tmem_ld16(tm + lane_base + t * dcols + c16 * 16, rr);
        if (row_here && m < 3 * CP) {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            a.part[(((long long)blockIdx.x * 9 + tap) * a.cout + c16 * 16 + j) * a.cin + ci] =
                nitems > 0 ? __uint_as_float(rr[j]) : 0.0f;
        }
      }
    }
  } else if (ok && warp < 4) {
    tc_fence_after_sync();
    const int co = 32 * warp + lane;
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    for (int t = 0; t < g.ndx; ++t) {
      const int dxi = dx0 + t;
#pragma unroll 1
      for (int c16 = 0; c16 < NC / 16; ++c16) {
        uint32_t rr[16];
        tmem_ld16(tm + lane_base + t * NC + c16 * 16, rr);
        if (co < a.cout) {
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            // column n = (3 j + dyi) * 8 + i: channel c0 + 8 j + i, tap dyi * 3 + dxi
            const int n = c16 * 16 + k, grp = n >> 3, j = grp / 3, dyi = grp - 3 * j;
            const int tap = dyi * 3 + dxi, ci = c0 + 8 * j + (n & 7);
            a.part[(((long long)blockIdx.x * 9 + tap) * a.cout + co) * a.cin + ci] =
                nitems > 0 ? __uint_as_float(rr[k]) : 0.0f;
          }
        }
      }
    }
  }
  if (!ok && tid == 0) atomicExch(a.err, 1);
  if (warp >= 5 && warp - 5 < nis && lane == 0) {
    if (warp == 5) {
      int lo = s_issued;
      for (int i = 0; i < nis; ++i) lo = min(lo, s_consumed[i]);
      for (int it = lo; it < s_issued; ++it) wait_phase(&full[it % nst], (it / nst) & 1);
    }
    mma_commit(&drain);
    if (warp == 5) wait_phase(&drain, 0);
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

// A blocked activation buffer as the 5-D tensor {CW * 8 elements, W / CW
// chunks, H rows, CG planes, B} with box {CW * 8, box_chunks, box_rows,
// box_planes, 1}.
static bool act_map(CUtensorMap *m, const ActView &v, int B, int H, int W, int CW, int box_chunks, int box_rows,
                    int box_planes) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[5] = {(cuuint64_t)CW * 8, (cuuint64_t)(W / CW), (cuuint64_t)H, (cuuint64_t)v.cg,
                              (cuuint64_t)B};
  const cuuint64_t strides[4] = {(cuuint64_t)CW * 16, (cuuint64_t)W * 16, (cuuint64_t)H * W * 16,
                                 (cuuint64_t)v.cg * H * W * 16};
  const cuuint32_t box[5] = {(cuuint32_t)CW * 8, (cuuint32_t)box_chunks, (cuuint32_t)box_rows,
                             (cuuint32_t)box_planes, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, v.p, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
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

constexpr int kSmemCap = 227 * 1024 - 4096;  // dynamic shared memory a CTA may take
constexpr int kHalfSm = 110 * 1024;          // two CTAs per SM

// Segments: 128 pixels, or the whole row rounded up to 16 for narrower
// images. Chunks: 16 pixels, or the largest power of two dividing W. The halo
// row spans one chunk left of the segment to at least one pixel past it,
// rounded up to 8 entries so that every row starts on a 128-byte boundary.
static SegGeom seg_geom(int B, int H, int W, int R) {
  SegGeom s{};
  s.SW = W >= 128 ? 128 : (W + 15) / 16 * 16;
  s.CW = 16;
  while (W % s.CW) s.CW >>= 1;
  s.HP = (s.SW + 2 * s.CW + 7) / 8 * 8;
  s.R = R;
  s.segs_x = (W + s.SW - 1) / s.SW;
  s.ngr = (H + R - 1) / R;
  s.nseg = B * s.ngr * s.segs_x;
  return s;
}

// Output channels per CTA: the largest part (a multiple of 16 dividing N, at
// most 96) whose resident weights fit in 110 KB and still leave shared memory
// for two one-row pipeline stages at this width. Wider parts mean fewer,
// larger MMAs and fewer reloads of the input halo.
static int conv_part(int n, int cin, int W) {
  const int HP = seg_geom(1, 1, W, 1).HP;
  const int stage1 = std::min(cin / 8, kMaxChunkGroups) * 3 * HP * 16;
  for (int p = n; p >= 16; p -= 16) {
    const int w_bytes = (p * 9 * cin * 2 + 1023) / 1024 * 1024;
    if (n % p == 0 && p <= 96 && p * 9 * cin * 2 <= 110 * 1024 && w_bytes + 2 * stage1 + kTail <= kSmemCap)
      return p;
  }
  return 0;
}

template <int NP>
static cudaError_t launch_conv_tma_t(const ConvArgs &a, int parts, cudaStream_t st) {
  ConvTmaGeom g{};
  g.w_bytes = (NP * 9 * a.cin * 2 + 1023) / 1024 * 1024;
  const int g8 = a.cin / 8;
  // Geometry: CTAs per SM (2 or 1), rows per tile R (TMEM: two buffers of R
  // accumulators within the CTA's share, 256 columns with two CTAs per SM
  // and 512 with one; at most 4) and channel groups per K chunk, with at
  // least 3 stages in the ring. Preferred: the most MMA issuers per SM (CTAs
  // x min(issuers, R)), then the larger R (fewer halo rows re-read), then the
  // larger chunk (fewer barrier round trips).
  int best_score = -1, per_sm = 1;
  for (int ps = 2; ps >= 1; --ps) {
    int rmax = (ps == 2 ? 256 : 512) / (2 * (int)pow2_cols(NP));
    if (rmax > 4) rmax = 4;
    const int budget = (ps == 2 ? kHalfSm : kSmemCap) - kTail - g.w_bytes;
    for (int R = rmax; R >= 1; R >>= 1) {
      const int HP = seg_geom(a.B, a.H, a.W, R).HP;
      for (int cg = std::min(g8, kMaxChunkGroups); cg >= 2; cg -= 2) {
        if (g8 % cg != 0 && cg != std::min(g8, kMaxChunkGroups)) continue;  // whole chunks, or the widest
        const int stage = cg * (R + 2) * HP * 16;
        if (budget / stage < 3) continue;
        const int score = (ps * std::min(kIssuers, R)) * 1000 + R * 100 + cg;
        if (score > best_score) best_score = score, per_sm = ps, g.s.R = R, g.cg = cg;
        break;  // the widest chunk that fits at this R
      }
    }
  }
  if (best_score < 0) return cudaErrorInvalidValue;
  const int R = g.s.R, GB = g.cg;
  g.s = seg_geom(a.B, a.H, a.W, R);
  CUtensorMap xm;
  if (!act_map(&xm, a.x, a.B, a.H, a.W, g.s.CW, g.s.HP / g.s.CW, R + 2, GB)) return cudaErrorInvalidValue;
  const int stage = GB * (R + 2) * g.s.HP * 16;
  const int budget = per_sm == 2 ? kHalfSm - kTail : kSmemCap - kTail;
  g.s.nst = (budget - g.w_bytes) / stage;
  if (g.s.nst > kMaxStages) g.s.nst = kMaxStages;
  if (g.s.nst < 2) return cudaErrorInvalidValue;
  int smem = g.w_bytes + g.s.nst * stage + kTail;
  // one CTA per SM: take enough shared memory that a second cannot share the
  // SM (and its TMEM)
  if (per_sm == 1 && smem < kHalfSm + 8 * 1024) smem = kHalfSm + 8 * 1024;
  cudaError_t e = cudaFuncSetAttribute(k_conv_tma<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  int gx = per_sm * num_sms() / parts;
  if (gx > g.s.nseg) gx = g.s.nseg;
  if (gx < 1) gx = 1;
  k_conv_tma<NP><<<dim3(gx, parts), kConvThreads, smem, st>>>(xm, a, g);
  return cudaGetLastError();
}

cudaError_t launch_conv3x3(const ConvArgs &a, int n, cudaStream_t st) {
  if (a.cin % 16 != 0 || a.cin > 256 || a.W < 1 || a.H < 1 || a.B < 1) return cudaErrorInvalidValue;
  const int p = conv_part(n, a.cin, a.W);
  switch (p) {
    case 16: return launch_conv_tma_t<16>(a, n / p, st);
    case 32: return launch_conv_tma_t<32>(a, n / p, st);
    case 48: return launch_conv_tma_t<48>(a, n / p, st);
    case 64: return launch_conv_tma_t<64>(a, n / p, st);
    case 96: return launch_conv_tma_t<96>(a, n / p, st);
    default: return cudaErrorInvalidValue;
  }
}

// Partial-sum chunks of the weight gradient: at most a fixed count (divided by
// the CTAs a chunk already spans), so the order of the final sum does not
// depend on the device; wgrad_chunks bounds it for buffer sizing.
constexpr int kWgChunks = 296;

int wgrad_chunks(int B, int H, int W) {
  const SegGeom s = seg_geom(B, H, W, 1);
  const int per = (s.nseg + kWgChunks - 1) / kWgChunks;
  return (s.nseg + per - 1) / per;
}

// Channels per part of the weight-gradient columns.
static int wgrad_part(int cin) {
  if (cin <= 64) return cin;
  for (int p = 64; p >= 16; p -= 16)
    if (cin % p == 0) return p;
  return 0;
}

template <int CP, bool T>
static cudaError_t launch_wgrad_tma_t(const WgradArgs &a, cudaStream_t st, int *chunks) {
  WgradTmaGeom g{};
  g.s = seg_geom(a.B, a.H, a.W, 1);
  CUtensorMap dym, xm;
  if (!act_map(&dym, a.dy, a.B, a.H, a.W, g.s.CW, g.s.SW / g.s.CW, 1, a.cout / 8) ||
      !act_map(&xm, a.x, a.B, a.H, a.W, g.s.CW, g.s.HP / g.s.CW, 3, CP / 8))
    return cudaErrorInvalidValue;
  g.ndx = (T || 9 * CP <= 256) ? 3 : 1;
  const int nparts = a.cin / CP;
  const int gy = nparts * (g.ndx == 3 ? 1 : 3);
  // about kWgChunks CTAs in all: fewer segment chunks when the channels and
  // dx already split the work (fewer partials to write and sum)
  const int target = std::max(1, kWgChunks / gy);
  g.seg_per_chunk = (g.s.nseg + target - 1) / target;
  const int nchunks = (g.s.nseg + g.seg_per_chunk - 1) / g.seg_per_chunk;
  g.a_bytes = a.cout / 8 * g.s.SW * 16;
  // GEMM rows past the real ones address the bytes that follow their groups:
  // keep the full 128-row span (16 groups) inside the allocation
  const int stage = g.a_bytes + 3 * (CP / 8) * g.s.HP * 16;
  int tail = T ? (16 - 3 * CP / 8) * g.s.HP * 16 + 512 : 16 * g.s.SW * 16 - g.a_bytes;
  if (tail < kTail) tail = kTail;
  g.s.nst = (kHalfSm - tail) / stage;
  if (g.s.nst < 3) g.s.nst = (kSmemCap - tail) / stage;
  if (g.s.nst > kMaxStages) g.s.nst = kMaxStages;
  if (g.s.nst < 2) return cudaErrorInvalidValue;
  int smem = g.s.nst * stage + tail;
  // at most two CTAs per SM when each holds 256 TMEM columns
  if (pow2_cols(g.ndx * (T ? a.cout : 3 * CP)) >= 256 && smem < 80 * 1024) smem = 80 * 1024;
  cudaError_t e = cudaFuncSetAttribute(k_wgrad_tma<CP, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_wgrad_tma<CP, T><<<dim3(nchunks, gy), kWgThreads, smem, st>>>(dym, xm, a, g);
  *chunks = nchunks;
  return cudaGetLastError();
}

cudaError_t launch_wgrad(const WgradArgs &a, cudaStream_t st) {
  if (a.cout % 8 != 0 || a.cout > 128 || a.cin % 16 != 0 || a.W < 1) return cudaErrorInvalidValue;
  int chunks = 0;
  cudaError_t e;
  if (a.cout <= 32) {
    // transposed product: parts of at most 32 channels (3 * 32 GEMM rows)
    const int cp = a.cin % 32 == 0 ? 32 : 16;
    e = cp == 32 ? launch_wgrad_tma_t<32, true>(a, st, &chunks) : launch_wgrad_tma_t<16, true>(a, st, &chunks);
  } else {
    switch (wgrad_part(a.cin)) {
      case 16: e = launch_wgrad_tma_t<16, false>(a, st, &chunks); break;
      case 32: e = launch_wgrad_tma_t<32, false>(a, st, &chunks); break;
      case 48: e = launch_wgrad_tma_t<48, false>(a, st, &chunks); break;
      case 64: e = launch_wgrad_tma_t<64, false>(a, st, &chunks); break;
      default: return cudaErrorInvalidValue;
    }
  }
  if (e != cudaSuccess) return e;
  return launch_wgrad_reduce(a.part, chunks, a.cout, a.cin, a.dw, a.db ? a.db_part : nullptr, a.db, st);
}

}  // namespace unet
