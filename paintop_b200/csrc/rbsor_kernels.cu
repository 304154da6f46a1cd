// rbsor_kernels.cu -- device kernels of the red-black SOR solver (sm_100a).
// See rbsor.cuh for the method, the HBM layout and the control scheme.
#include "rbsor.cuh"
#include "rbsor_launch.h"

#include <cmath>
#include <cstdio>

namespace ptk {

// ----------------------------------------------------------------------------
// small device helpers
// ----------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_vol(const int *p) { return *reinterpret_cast<const volatile int *>(p); }

// Asynchronous global -> shared copies (Ampere+ cp.async). `in == false` copies
// no bytes and zero-fills the destination.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src, bool in) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(gmem_src),
               "r"(in ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem_dst, const void *gmem_src, bool in) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(gmem_src),
               "r"(in ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Deterministic block sum: fixed xor-butterfly inside each warp, then warps in
// index order. The total is valid in thread 0. Uses sred[0 .. blockDim.x/32).
__device__ __forceinline__ double block_sum(double v, double *sred) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) sred[warp] = v;
  __syncthreads();
  double tot = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sred[w];
  __syncthreads();
  return tot;
}

__device__ __forceinline__ long long plane_index(const SysDesc &d, int c, int y, int i) {
  return d.off + (long long)c * d.plane + (long long)y * d.pw + i;
}

// ----------------------------------------------------------------------------
// geometry of one tile configuration
// ----------------------------------------------------------------------------
template <int S, int TH>
struct Geo {
  static constexpr int H = halo_y(S);
  static constexpr int HX = halo_x(S);
  static constexpr int TW = tile_w(S);
  static constexpr int LH = TH + 2 * H;
  static constexpr int PLANE = LH * kPWL;  // elements per shared plane
  static constexpr int XOFF = HX - H;      // unused loaded columns on each side
  static_assert(HX >= H, "x halo must cover the sweep halo");
  static_assert(TW > 0 && TW % 8 == 0, "tile width must keep plane loads 16-byte aligned");
  static constexpr size_t kSmem = (size_t)2 * PLANE * sizeof(float)   // e
                                  + (size_t)2 * PLANE * sizeof(float) // g
                                  + (size_t)2 * PLANE                 // cell
                                  + kWarps * sizeof(double);          // reduction scratch
};

// ----------------------------------------------------------------------------
// assembly kernels
// ----------------------------------------------------------------------------
__device__ __forceinline__ bool interior_at(const SysDesc &d, int x, int y) {
  if (d.W < 3 || d.H < 3) return false;                  // poisson.rs:342-345
  if (x < 1 || y < 1 || x > d.W - 2 || y > d.H - 2) return false;
  return d.mask[(long long)y * d.W + x] > 0.5f;           // poisson.rs:349 (strict >)
}

// Interior cells per tile (owned region only) and their bounding box. min/max
// are order-independent, so the box is deterministic.
// The channels of an image share its mask, so only channel 0's blocks count;
// they store the count and box for every channel's copy of the tile.
__global__ void k_tile_count(KParams P, int TW, int TH) {
  const Tile tl = P.tiles[blockIdx.x];
  const SysDesc d = P.sys[tl.sys];
  if (d.chan != 0) return;
  __shared__ int s[32];
  __shared__ int sb[4];
  if (threadIdx.x < 4) sb[threadIdx.x] = (threadIdx.x < 2) ? 0x7fffffff : -1;
  __syncthreads();
  int n = 0, x0m = 0x7fffffff, y0m = 0x7fffffff, x1m = -1, y1m = -1;
  const int x0 = tl.tx * TW, y0 = tl.ty * TH;
  for (int k = threadIdx.x; k < TW * TH; k += blockDim.x) {
    const int x = x0 + k % TW, y = y0 + k / TW;
    if (x < d.W && y < d.H && interior_at(d, x, y)) {
      ++n;
      x0m = min(x0m, x); y0m = min(y0m, y); x1m = max(x1m, x); y1m = max(y1m, y);
    }
  }
  for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = n;
  if (x1m >= 0) {
    atomicMin(&sb[0], x0m); atomicMin(&sb[1], y0m); atomicMax(&sb[2], x1m); atomicMax(&sb[3], y1m);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    const int4 box = make_int4(sb[0], sb[1], sb[2], sb[3]);
    const int local = (int)blockIdx.x - d.tile0;  // the tile's index within its system
    for (int c = 0; c < d.C; ++c) {
      const int tt = P.sys[tl.sys + c].tile0 + local;
      P.tcount[tt] = t;
      P.tbox[tt] = box;
    }
  }
}

__device__ __forceinline__ bool tile_support(const KParams &P, const SysDesc &d, int tx, int ty) {
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      const int x = tx + dx, y = ty + dy;
      if (x < 0 || y < 0 || x >= d.ntx || y >= d.nty) continue;
      if (P.tcount[d.tile0 + y * d.ntx + x] > 0) return true;
    }
  return false;
}

// r(anchor) at an interior pixel: (4 + lambda) a - (sum of the four anchor
// neighbours) against b' (poisson.rs:315-321), in this operand order.
__device__ __forceinline__ double anchor_residual(const SysDesc &d, long long px, double a, double bp) {
  const int C = d.C, ch = d.chan;
  const double na = (((double)d.tgt[(px - 1) * C + ch] + (double)d.tgt[(px + 1) * C + ch]) +
                     (double)d.tgt[(px - d.W) * C + ch]) + (double)d.tgt[(px + d.W) * C + ch];
  return fma(d.lambda + 4.0, -a, na) - bp;
}

// Assemble one tile of one system (owned cells only). Writes cell, bp, u, g and
// zeroes e0/e1; accumulates ||r(anchor)||^2 and ||r(u_init)||^2 partials.
// Arithmetic of b and r follows poisson.rs:364-373 (guidance_laplacian) and
// poisson.rs:315-321 (residual), operand for operand.
__global__ void __launch_bounds__(kThreads) k_assemble(KParams P, int TW, int TH) {
  __shared__ double sred[kWarps];
  // Block order: within each image, its channels' copies of a tile come one
  // after another, so the interleaved source and target pixels a tile reads
  // are still in L2 for the other channels' blocks. The tiles of an image are
  // channel 0's, then channel 1's, ...; block b of the image takes channel
  // b % C's tile b / C.
  int t = blockIdx.x;
  {
    const SysDesc &d0 = P.sys[P.tiles[t].sys];
    const int base = d0.tile0 - d0.chan * d0.ntiles;  // the image's first tile
    const int local = t - base;
    t = base + (local % d0.C) * d0.ntiles + local / d0.C;
  }
  const Tile tl = P.tiles[t];
  const SysDesc d = P.sys[tl.sys];
  if (!tile_support(P, d, tl.tx, tl.ty)) return;
  const int C = d.C, ch = d.chan;
  const double lam = d.lambda;
  double acc_a = 0.0, acc_u = 0.0;
  const int half = TW / 2;
  for (int k = threadIdx.x; k < 2 * TH * half; k += blockDim.x) {
    const int c = k / (TH * half);
    const int r = k - c * (TH * half);
    const int y = tl.ty * TH + r / half;
    const int i = tl.tx * half + r % half;
    if (y >= d.H || i >= d.pw) continue;
    const int x = 2 * i + ((c + y) & 1);
    const long long o = plane_index(d, c, y, i);
    P.e0[o] = 0.0f;
    P.e1[o] = 0.0f;
    if (x >= d.W) {  // padding column beyond the image
      P.cell[o] = 0; P.bp[o] = 0.0; P.u[o] = 0.0; P.g[o] = 0.0f;
      continue;
    }
    const long long px = (long long)y * d.W + x;
    const double a = (double)d.tgt[px * C + ch];
    if (!interior_at(d, x, y)) {
      P.cell[o] = 0; P.bp[o] = 0.0; P.u[o] = a; P.g[o] = 0.0f;
      continue;
    }
    // interior: all four neighbours are inside the image
    const long long pl = px - 1, pr = px + 1, pu = px - d.W, pd = px + d.W;
    const double sc = (double)d.src[px * C + ch];
    const double ns = (((double)d.src[pl * C + ch] + (double)d.src[pr * C + ch]) +
                       (double)d.src[pu * C + ch]) + (double)d.src[pd * C + ch];
    const double b = fma(4.0, -sc, ns);
    const double bp = fma(lam, -a, b);
    const double ra = anchor_residual(d, px, a, bp);
    acc_a = fma(ra, ra, acc_a);
    double uc = a, ru = ra;
    if (d.warm) {
      auto guess_or_anchor = [&](long long q, int qx, int qy) -> double {
        return interior_at(d, qx, qy) ? (double)d.guess[q * C + ch] : (double)d.tgt[q * C + ch];
      };
      uc = (double)d.guess[px * C + ch];
      const double nu = ((guess_or_anchor(pl, x - 1, y) + guess_or_anchor(pr, x + 1, y)) +
                         guess_or_anchor(pu, x, y - 1)) + guess_or_anchor(pd, x, y + 1);
      ru = fma(lam + 4.0, -uc, nu) - bp;
    }
    acc_u = fma(ru, ru, acc_u);
    P.cell[o] = 1;
    P.bp[o] = bp;
    P.u[o] = uc;
    P.g[o] = (float)(-ru);
  }
  acc_a = block_sum(acc_a, sred);
  acc_u = block_sum(acc_u, sred);
  if (threadIdx.x == 0) {
    P.fpart[t] = acc_a;
    P.fpart[P.ntiles + t] = acc_u;
  }
}

// ---- connected interior regions (automatic omega) --------------------------
// A union-find over the pixels of each labelled image (4-neighbour
// connectivity): every label points at itself (a root) or at a smaller index
// of the same region, so a root search walks strictly decreasing indices and
// ends; unions lower a root with atomicMin, so each retry sees a smaller
// label and ends too. The final labels are the regions' smallest pixel
// indices whatever the order of the unions, so the result is deterministic.
__device__ __forceinline__ int region_of(const KParams &P, long long gp) {
  int lo = 0, hi = P.nregions - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (P.regions[mid].lab_off <= gp) lo = mid; else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ int label_root(int *L, int x) {
  const volatile int *vl = L;
  const int x0 = x;
  for (int k = x; k >= 0; --k) {  // at most x + 1 steps: labels only decrease
    const int y = vl[x];
    if (y == x) break;
    x = y;
  }
  if (x != x0) atomicMin(&L[x0], x);  // shorten the chain; never raises a label
  return x;
}
__device__ void label_unite(int *L, int a, int b) {
  for (int k = a + b + 2; k > 0; --k) {  // each retry lowers a or b
    a = label_root(L, a);
    b = label_root(L, b);
    if (a == b) return;
    if (a < b) {
      const int old = atomicMin(&L[b], a);
      if (old == b) return;
      b = old;
    } else {
      const int old = atomicMin(&L[a], b);
      if (old == a) return;
      a = old;
    }
  }
}
__global__ void k_label_init(KParams P) {
  for (long long gp = blockIdx.x * (long long)blockDim.x + threadIdx.x; gp < P.rpix;
       gp += (long long)gridDim.x * blockDim.x) {
    const RegionDesc r = P.regions[region_of(P, gp)];
    const int p = (int)(gp - r.lab_off), y = p / r.W, x = p - y * r.W;
    P.label[gp] = interior_at(P.sys[r.sys0], x, y) ? p : -1;
  }
}
__global__ void k_label_link(KParams P) {
  for (long long gp = blockIdx.x * (long long)blockDim.x + threadIdx.x; gp < P.rpix;
       gp += (long long)gridDim.x * blockDim.x) {
    if (P.label[gp] < 0) continue;
    const RegionDesc r = P.regions[region_of(P, gp)];
    int *L = P.label + r.lab_off;
    const int p = (int)(gp - r.lab_off), y = p / r.W, x = p - y * r.W;
    if (x > 0 && L[p - 1] >= 0) label_unite(L, p, p - 1);
    if (y > 0 && L[p - r.W] >= 0) label_unite(L, p, p - r.W);
  }
}
__global__ void k_label_count(KParams P) {
  for (long long gp = blockIdx.x * (long long)blockDim.x + threadIdx.x; gp < P.rpix;
       gp += (long long)gridDim.x * blockDim.x) {
    if (P.label[gp] < 0) continue;
    const RegionDesc r = P.regions[region_of(P, gp)];
    const int root = label_root(P.label + r.lab_off, (int)(gp - r.lab_off));
    atomicAdd(&P.rsize[r.lab_off + root], 1);
  }
}
__global__ void k_label_max(KParams P) {
  for (long long gp = blockIdx.x * (long long)blockDim.x + threadIdx.x; gp < P.rpix;
       gp += (long long)gridDim.x * blockDim.x) {
    const int n = P.rsize[gp];
    if (n > 0) atomicMax(&P.rmax[region_of(P, gp)], n);
  }
}

// Per-system initial state from the assembly partials (tile order).
__global__ void k_init(KParams P) {
  __shared__ double sred[kWarps];
  const int sys = blockIdx.x;
  const SysDesc d = P.sys[sys];
  double sa = 0.0, su = 0.0;
  int nact = 0;
  for (int k = threadIdx.x; k < d.ntiles; k += blockDim.x) {
    const int t = d.tile0 + k;
    if (P.tcount[t] == 0) continue;
    sa += P.fpart[t];
    su += P.fpart[P.ntiles + t];
    ++nact;
  }
  sa = block_sum(sa, sred);
  su = block_sum(su, sred);
  for (int o = 16; o > 0; o >>= 1) nact += __shfl_xor_sync(0xffffffffu, nact, o);
  __shared__ int sn[kWarps];
  if ((threadIdx.x & 31) == 0) sn[threadIdx.x >> 5] = nact;
  __syncthreads();
  if (threadIdx.x != 0) return;
  int n = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) n += sn[w];
  SysState s;
  s.mode = M_SWEEP; s.s = 0; s.iterations = 0; s.cur = 0;
  s.pending = P_NONE; s.status = -1; s.refinements = 0; s.since = 0;
  s.isince = 0; s.nact = n; s.out_anchor = 0; s.steps = 0;
  s.warm_used = 0; s.pad1 = 0;
  s.r0 = sqrt(sa); s.outer = sqrt(su);
  if (d.warm) {
    // The plain start is the fallback: a guess whose residual is not below the
    // anchor's (or not finite) is replaced by the anchor (k_warm_fallback).
    if (s.outer < s.r0) s.warm_used = 1;
    else s.outer = s.r0;
  }
  s.best = INFINITY; s.ibest = INFINITY; s.last = 1.0; s.ibase = s.outer;
  s.omega = d.omega;
  s.stall_window = (int)kStallWindow;  // poisson.rs:80
  s.pad2 = 0;
  if (d.omega < 0.0f) {
    // automatic SOR factor: Young's optimum for red-black SOR with the Jacobi
    // spectral radius of (4+lambda)I - N on the region's bounding box (a x b
    // cells including the boundary ring): (2cos(pi/a) + 2cos(pi/b)) / (4+lambda)
    int bx0 = 0x7fffffff, by0 = 0x7fffffff, bx1 = -1, by1 = -1;
    for (int k = 0; k < d.ntiles; ++k) {
      const int t = d.tile0 + k;
      if (P.tcount[t] == 0) continue;
      const int4 b = P.tbox[t];
      bx0 = min(bx0, b.x); by0 = min(by0, b.y); bx1 = max(bx1, b.z); by1 = max(by1, b.w);
    }
    double om = 1.0;
    if (bx1 >= 0) {
      const double a = (double)(bx1 - bx0 + 2), b = (double)(by1 - by0 + 2);
      const double pi = 3.141592653589793;
      double rho = (2.0 * cos(pi / a) + 2.0 * cos(pi / b)) / (4.0 + d.lambda);
      // Several regions share one box: bound the largest region's smallest
      // eigenvalue from its area instead (Faber-Krahn: no region of that area
      // has a smaller one than the disk, pi j0^2 / area), with the area grown
      // to (sqrt(n) + 1)^2 for the half-cell margin of the discrete boundary.
      // Both are upper bounds on the Jacobi spectral radius; take the smaller.
      if (d.region1 > 0) {
        const int nmax = P.rmax[d.region1 - 1];
        if (nmax > 0) {
          const double area = (sqrt((double)nmax) + 1.0) * (sqrt((double)nmax) + 1.0);
          const double j0 = 2.404825557695773;  // first zero of the Bessel function J0
          const double pij0sq = 3.141592653589793 * (j0 * j0);
          rho = fmin(rho, (4.0 - pij0sq / area) / (4.0 + d.lambda));
        }
      }
      rho = fmin(fmax(rho, 0.0), 1.0 - 1e-15);
      om = 2.0 / (1.0 + sqrt(1.0 - rho * rho));
    }
    s.omega = om;
    const_cast<SysDesc *>(P.sys)[sys].omega = (float)om;
    // Near the optimum the residual norm of red-black SOR rises and falls on a
    // time scale of 1/(2 - omega) sweeps (its asymptotic decay time) before it
    // settles; a window of twice that many sweeps keeps the stall rule a test
    // for lost progress rather than for that transient.
    s.stall_window = max((int)kStallWindow, (int)ceil(2.0 / fmax(2.0 - om, 1e-6)));
  }
  // poisson.rs:172-189: no unknowns or a satisfied system -> 0 iterations, converged.
  if (n == 0 || s.r0 == 0.0) {
    s.mode = M_DONE; s.status = STOP_CONVERGED; s.last = 0.0; s.out_anchor = 1;
    atomicAdd(P.bar + 2, 1u);
  } else if (d.max_it <= 0) {
    // poisson.rs:202: an empty sweep loop reports the cap with last_relative = 1.
    s.mode = M_DONE; s.status = STOP_MAX; s.last = 1.0; s.out_anchor = 1;
    atomicAdd(P.bar + 2, 1u);
  } else {
    s.s = d.max_it < P.S ? d.max_it : P.S;
  }
  P.st[sys] = s;
  P.arrive[sys] = 0;
  P.claim[sys] = s.mode == M_DONE ? (unsigned long long)kClaimDone : 0ull;
}

// Restore the anchor start (u = anchor, g = -r(anchor), as k_assemble writes
// without a guess) in the systems whose guess k_init rejected.
__global__ void __launch_bounds__(kThreads) k_warm_fallback(KParams P, int TW, int TH) {
  const int t = blockIdx.x;
  const Tile tl = P.tiles[t];
  const SysDesc d = P.sys[tl.sys];
  if (!d.warm || P.st[tl.sys].warm_used || !tile_support(P, d, tl.tx, tl.ty)) return;
  const int half = TW / 2;
  for (int k = threadIdx.x; k < 2 * TH * half; k += blockDim.x) {
    const int c = k / (TH * half);
    const int r = k - c * (TH * half);
    const int y = tl.ty * TH + r / half;
    const int i = tl.tx * half + r % half;
    if (y >= d.H || i >= d.pw) continue;
    const int x = 2 * i + ((c + y) & 1);
    if (x >= d.W || !interior_at(d, x, y)) continue;
    const long long o = plane_index(d, c, y, i);
    const long long px = (long long)y * d.W + x;
    const double a = (double)d.tgt[px * d.C + d.chan];
    P.u[o] = a;
    P.g[o] = (float)(-anchor_residual(d, px, a, P.bp[o]));
  }
}

// Per system, the tiles with interior cells in index order (one block per
// system; a block-wide exclusive scan keeps the order fixed).
__global__ void k_compact(KParams P) {
  __shared__ int sw[32];
  __shared__ int s_base;
  const SysDesc d = P.sys[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (int k0 = 0; k0 < d.ntiles; k0 += blockDim.x) {
    const int k = k0 + threadIdx.x;
    const int flag = (k < d.ntiles && P.tcount[d.tile0 + k] > 0) ? 1 : 0;
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    const int before = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) sw[warp] = __popc(m);
    __syncthreads();
    int off = s_base;
    for (int w = 0; w < warp; ++w) off += sw[w];
    if (flag) P.act[d.tile0 + off + before] = d.tile0 + k;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < nw; ++w) tot += sw[w];
      s_base += tot;
    }
    __syncthreads();
  }
}

// Interleave the result: interior cells take (float)u (the reference's `as f32`,
// poisson_blend.rs:211-219); every other pixel copies the target bit for bit.
__global__ void k_emit(KParams P, int sys0, int TW, int TH) {
  const SysDesc d0 = P.sys[sys0];
  const long long npx = (long long)d0.W * d0.H;
  const int C = d0.C;
  // four channels with 16-byte aligned images: one vector load and store per pixel
  const bool vec4 = C == 4 && ((reinterpret_cast<uintptr_t>(d0.tgt) | reinterpret_cast<uintptr_t>(d0.out)) & 15) == 0;
  for (long long px = blockIdx.x * (long long)blockDim.x + threadIdx.x; px < npx;
       px += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(px / d0.W), x = (int)(px - (long long)y * d0.W);
    const int tx = x / TW, ty = y / TH;
    const int c = (x + y) & 1, i = x >> 1;
    // the channels share the tile counts (k_tile_count stores one per channel)
    const bool active = P.tcount[d0.tile0 + ty * d0.ntx + tx] > 0;
    if (vec4) {
      float4 v = *reinterpret_cast<const float4 *>(d0.tgt + px * 4);
      if (active) {
        float *vv = reinterpret_cast<float *>(&v);
#pragma unroll
        for (int ch = 0; ch < 4; ++ch) {
          if (P.st[sys0 + ch].out_anchor) continue;
          const long long o = plane_index(P.sys[sys0 + ch], c, y, i);
          if (P.cell[o]) vv[ch] = (float)P.u[o];
        }
      }
      *reinterpret_cast<float4 *>(d0.out + px * 4) = v;
      continue;
    }
    for (int ch = 0; ch < C; ++ch) {
      const SysDesc &d = P.sys[sys0 + ch];
      float v = d.tgt[px * C + ch];
      if (active && !P.st[sys0 + ch].out_anchor) {
        const long long o = plane_index(d, c, y, i);
        if (P.cell[o]) v = (float)P.u[o];
      }
      d.out[px * C + ch] = v;
    }
  }
}

// Per row band of tiles of image sys0: the first and last tile column holding
// interior cells, or -1, -1 when the band holds none (two ints per band). The
// solve reads the image's source and target only in those spans, one pixel
// and one row around; the rest of the output is the target, bit for bit
// (k_emit).
__global__ void k_band_flags(KParams P, int sys0, int *spans) {
  const SysDesc d = P.sys[sys0];
  for (int ty = threadIdx.x; ty < d.nty; ty += blockDim.x) {
    int lo = -1, hi = -1;
    for (int tx = 0; tx < d.ntx; ++tx)
      if (P.tcount[d.tile0 + ty * d.ntx + tx] > 0) {
        if (lo < 0) lo = tx;
        hi = tx;
      }
    spans[2 * ty] = lo;
    spans[2 * ty + 1] = hi;
  }
}

// ----------------------------------------------------------------------------
// the persistent solve kernel
// ----------------------------------------------------------------------------
// Cell-flag rows are stored in slot ly ^ ((ly >> 1) & 1): the two rows a warp
// reads (two apart, one per half-warp) then sit an odd number of 64-byte rows
// apart, in different shared-memory banks (rows two apart would share all 16).
__host__ __device__ constexpr int cell_slot(int ly) { return ly ^ ((ly >> 1) & 1); }

template <int S, int TH>
__device__ void sweep_tile(const KParams &P, const SysDesc &d, int t, const Tile &tl, int s,
                           int cur, float *sE, float *sG, uint8_t *sC, double *sred) {
  using G = Geo<S, TH>;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int X0 = tl.tx * G::TW - G::HX;  // loaded column 0, a multiple of 8
  const int Y0 = tl.ty * TH - G::H;
  const int gi0 = X0 >> 1;                // plane index of loaded column 0, a multiple of 4
  const float *__restrict__ ein = cur ? P.e1 : P.e0;
  float *__restrict__ eout = cur ? P.e0 : P.e1;

  // ---- load tile + halo straight into shared memory with cp.async (L2 only:
  // other blocks wrote these planes). Outside the image the copy reads nothing
  // and zero-fills, which is exactly a boundary cell (e = 0, g = 0, cell = 0).
  constexpr int V = kPWL / 4;
  for (int k = tid; k < 2 * G::LH * V; k += kThreads) {
    const int c = k / (G::LH * V);
    const int r = k - c * (G::LH * V);
    const int ly = r / V, v = r - ly * V;
    const int gy = Y0 + ly, gi = gi0 + 4 * v;
    const bool in = gy >= 0 && gy < d.H && gi >= 0 && gi < d.pw;
    const long long o = in ? plane_index(d, c, gy, gi) : d.off;  // a valid address either way
    const int so = c * G::PLANE + ly * kPWL + 4 * v;
    cp_async16(sE + so, ein + o, in);
    cp_async16(sG + so, P.g + o, in);
    cp_async4(sC + c * G::PLANE + cell_slot(ly) * kPWL + 4 * v, P.cell + o, in);
  }
  cp_async_wait_all();
  __syncthreads();

  const int pl = Y0 & 1;  // colour parity of loaded row 0 (column 0 is even)
  const float w = d.omega, inv = d.inv_denom;
  const double dd = 4.0 + d.lambda;
  constexpr int OX0 = G::HX, OX1 = G::HX + G::TW;  // owned loaded columns
  constexpr int OY0 = G::H, OY1 = G::H + TH;       // owned loaded rows
  constexpr int RQ = kPWL / 4;                      // float4 per plane row (16 lanes)
  static_assert((G::LH - 2) % 32 == 0, "rows 1..LH-2 must split evenly over the warps");
  static_assert(TH % 4 == 0, "owned rows come in groups of four");
  static_assert(OX0 % 8 == 0 && OX1 % 8 == 0, "owned columns come in whole lanes");
  static_assert(G::LH % 4 == 0 || G::LH % 4 == 2, "cell slots stay inside the plane");
  constexpr int LO = OX0 / 8, LE = OX1 / 8;         // lanes (l16) whose cells are owned
  constexpr int kRowPairs = (G::LH - 2) / 2;
  // Each lane owns four consecutive plane entries (four cells of one colour) of
  // a row; the two half-warps take rows two apart, so both rows of a warp have
  // the same colour parity. Every half-sweep relaxes all rows 1..LH-2 and all
  // columns: cells outside the window that a whole-grid sweep would reproduce
  // get values nobody reads (they never reach the owned region before the tile
  // is written back), which keeps the work of every warp identical.
  const int hw = lane >> 4, l16 = lane & 15;
  double acc[S];
#pragma unroll
  for (int j = 0; j < S; ++j) acc[j] = 0.0;

  // the four cells of a lane together: each square added in cell order as
  // fma(r, r, part); a cell that is not interior adds fma(0, 0, part) = part,
  // bit for bit what skipping it gives
  auto rval = [&](float l, float r, float u, float dn, float e, float g) -> double {
    const double ns = (((double)l + (double)r) + (double)u) + (double)dn;
    return fma(-dd, (double)e, ns) - (double)g;
  };
  auto resid4 = [&](double &part, uint32_t cc, float L0, float R0, float L1, float R1, float L2, float R2,
                    float L3, float R3, const float4 &up, const float4 &dn, const float4 &e, const float4 &g) {
    double r0 = rval(L0, R0, up.x, dn.x, e.x, g.x), r1 = rval(L1, R1, up.y, dn.y, e.y, g.y),
           r2 = rval(L2, R2, up.z, dn.z, e.z, g.z), r3 = rval(L3, R3, up.w, dn.w, e.w, g.w);
    r0 = (cc & 0xffu) ? r0 : 0.0;
    r1 = (cc & 0xff00u) ? r1 : 0.0;
    r2 = (cc & 0xff0000u) ? r2 : 0.0;
    r3 = (cc & 0xff000000u) ? r3 : 0.0;
    part = fma(r0, r0, part);
    part = fma(r1, r1, part);
    part = fma(r2, r2, part);
    part = fma(r3, r3, part);
  };

#pragma unroll
  for (int j = 0; j < S; ++j) {
    if (j >= s) break;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float4 *Ec = reinterpret_cast<float4 *>(sE + h * G::PLANE);
      const float4 *Eo = reinterpret_cast<const float4 *>(sE + (1 - h) * G::PLANE);
      const float4 *Gc = reinterpret_cast<const float4 *>(sG + h * G::PLANE);
      const uint32_t *Cc = reinterpret_cast<const uint32_t *>(sC + h * G::PLANE);
      const bool duty = (h == 1) || (j > 0);  // residual of black state j / red state j-1
      double part = 0.0;
      for (int rp = warp; rp < kRowPairs; rp += kWarps) {
        const int base = 1 + 4 * (rp >> 1) + (rp & 1);
        const int ly = base + 2 * hw;
        const int q = (h + base + pl) & 1;  // same for both rows of the warp
        const int r4 = ly * RQ + l16;
        const float4 up = Eo[r4 - RQ], dn = Eo[r4 + RQ], ct = Eo[r4];
        const float4 gc = Gc[r4];
        const float4 ec = Ec[r4];
        const uint32_t cc = Cc[cell_slot(ly) * RQ + l16];
        const float prev = __shfl_up_sync(0xffffffffu, ct.w, 1, 16);
        const float next = __shfl_down_sync(0xffffffffu, ct.x, 1, 16);
        float L0, R0, L1, R1, L2, R2, L3, R3;
        if (q == 0) {
          L0 = prev; R0 = ct.x; L1 = ct.x; R1 = ct.y; L2 = ct.y; R2 = ct.z; L3 = ct.z; R3 = ct.w;
        } else {
          L0 = ct.x; R0 = ct.y; L1 = ct.y; R1 = ct.z; L2 = ct.z; R2 = ct.w; L3 = ct.w; R3 = next;
        }
        float4 ne = ec;
        if (cc & 0xffu) ne.x = fmaf(w, ((((L0 + R0) + up.x) + dn.x) - gc.x) * inv - ec.x, ec.x);
        if (cc & 0xff00u) ne.y = fmaf(w, ((((L1 + R1) + up.y) + dn.y) - gc.y) * inv - ec.y, ec.y);
        if (cc & 0xff0000u) ne.z = fmaf(w, ((((L2 + R2) + up.z) + dn.z) - gc.z) * inv - ec.z, ec.z);
        if (cc & 0xff000000u) ne.w = fmaf(w, ((((L3 + R3) + up.w) + dn.w) - gc.w) * inv - ec.w, ec.w);
        // a lane's four residuals together behind one lane-level test, so their
        // conversion and FP64 chains interleave (the owned columns come in whole
        // lanes: HX and TW are multiples of 8)
        if (duty && ly >= OY0 && ly < OY1 && l16 >= LO && l16 < LE && cc != 0u)
          resid4(part, cc, L0, R0, L1, R1, L2, R2, L3, R3, up, dn, h ? ne : ec, gc);
        Ec[r4] = ne;
      }
      if (h == 1) acc[j] += part;
      else if (j > 0) acc[j - 1] += part;
      __syncthreads();
    }
  }
  // red cells' residual of the final state
  {
    const float4 *Er = reinterpret_cast<const float4 *>(sE);
    const float4 *Eb = reinterpret_cast<const float4 *>(sE + G::PLANE);
    const float4 *Gr = reinterpret_cast<const float4 *>(sG);
    const uint32_t *Cr = reinterpret_cast<const uint32_t *>(sC);
    double part = 0.0;
    for (int rp = warp; rp < TH / 2; rp += kWarps) {
      const int base = OY0 + 4 * (rp >> 1) + (rp & 1);
      const int ly = base + 2 * hw;
      const int q = (base + pl) & 1;
      const int r4 = ly * RQ + l16;
      const float4 up = Eb[r4 - RQ], dn = Eb[r4 + RQ], ct = Eb[r4];
      const float4 gc = Gr[r4], ec = Er[r4];
      const uint32_t cc = Cr[cell_slot(ly) * RQ + l16];
      const float prev = __shfl_up_sync(0xffffffffu, ct.w, 1, 16);
      const float next = __shfl_down_sync(0xffffffffu, ct.x, 1, 16);
      float L0, R0, L1, R1, L2, R2, L3, R3;
      if (q == 0) {
        L0 = prev; R0 = ct.x; L1 = ct.x; R1 = ct.y; L2 = ct.y; R2 = ct.z; L3 = ct.z; R3 = ct.w;
      } else {
        L0 = ct.x; R0 = ct.y; L1 = ct.y; R1 = ct.z; L2 = ct.z; R2 = ct.w; L3 = ct.w; R3 = next;
      }
      if (l16 >= LO && l16 < LE && cc != 0u) resid4(part, cc, L0, R0, L1, R1, L2, R2, L3, R3, up, dn, ec, gc);
    }
#pragma unroll
    for (int j = 0; j < S; ++j)
      if (j == s - 1) acc[j] += part;
  }
  // The S tile partials in one pass, each with block_sum's order (a warp's
  // xor butterfly, then the warps in index order): one barrier instead of two
  // per sweep. The scratch is the black plane of g, which nothing reads after
  // the half-sweeps (the pass above reads only the red plane).
  {
    double *sr = reinterpret_cast<double *>(sG + G::PLANE);
#pragma unroll
    for (int j = 0; j < S; ++j) {
      if (j >= s) break;
      double v = acc[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) sr[j * kWarps + warp] = v;
    }
    __syncthreads();
    if (tid < s) {
      double tot = 0.0;
      for (int w = 0; w < kWarps; ++w) tot += sr[tid * kWarps + w];
      P.partial[(long long)tid * P.ntiles + t] = tot;
    }
  }

  // ---- write the owned cells
  constexpr int OV = G::TW / 8;  // float4 per owned plane row
  for (int k = tid; k < 2 * TH * OV; k += kThreads) {
    const int c = k / (TH * OV);
    const int r = k - c * (TH * OV);
    const int ly = G::H + r / OV, v = G::HX / 8 + r % OV;
    const int gy = Y0 + ly, gi = gi0 + 4 * v;
    if (gy < d.H && gi < d.pw) {
      const int so = c * G::PLANE + ly * kPWL + 4 * v;
      *reinterpret_cast<float4 *>(eout + plane_index(d, c, gy, gi)) =
          *reinterpret_cast<const float4 *>(sE + so);
    }
  }
}

// u += e on interior cells; e = 0 (owned cells of the tile).
template <int S, int TH>
__device__ void fold_tile(const KParams &P, const SysDesc &d, const Tile &tl, int cur) {
  using G = Geo<S, TH>;
  float *ec = cur ? P.e1 : P.e0;
  constexpr int OV = G::TW / 8;
  for (int k = threadIdx.x; k < 2 * TH * OV; k += kThreads) {
    const int c = k / (TH * OV);
    const int r = k - c * (TH * OV);
    const int gy = tl.ty * TH + r / OV;
    const int gi = tl.tx * (G::TW / 2) + 4 * (r % OV);
    if (gy >= d.H || gi >= d.pw) continue;
    const long long o = plane_index(d, c, gy, gi);
    const float4 e = __ldcg(reinterpret_cast<const float4 *>(ec + o));
    const uint32_t cv = __ldg(reinterpret_cast<const uint32_t *>(P.cell + o));
    double2 u01 = __ldcg(reinterpret_cast<const double2 *>(P.u + o));
    double2 u23 = __ldcg(reinterpret_cast<const double2 *>(P.u + o + 2));
    if (cv & 0xffu) u01.x += (double)e.x;
    if (cv & 0xff00u) u01.y += (double)e.y;
    if (cv & 0xff0000u) u23.x += (double)e.z;
    if (cv & 0xff000000u) u23.y += (double)e.w;
    *reinterpret_cast<double2 *>(P.u + o) = u01;
    *reinterpret_cast<double2 *>(P.u + o + 2) = u23;
    *reinterpret_cast<float4 *>(ec + o) = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// g = -r(u) with r in FP64 exactly as residual_l2 (poisson.rs:315-321); partial ||r||^2.
template <int S, int TH>
__device__ void resid_tile(const KParams &P, const SysDesc &d, int t, const Tile &tl, double *sred) {
  using G = Geo<S, TH>;
  constexpr int half = G::TW / 2;
  const double lam4 = d.lambda + 4.0;
  double acc = 0.0;
  for (int k = threadIdx.x; k < 2 * TH * half; k += kThreads) {
    const int c = k / (TH * half);
    const int r = k - c * (TH * half);
    const int gy = tl.ty * TH + r / half;
    const int gi = tl.tx * half + r % half;
    if (gy >= d.H || gi >= d.pw) continue;
    const long long o = plane_index(d, c, gy, gi);
    if (!__ldg(P.cell + o)) continue;
    const int q = (c + gy) & 1;
    const long long oo = d.off + (long long)(1 - c) * d.plane;
    const double L = __ldcg(P.u + oo + (long long)gy * d.pw + gi - 1 + q);
    const double R = __ldcg(P.u + oo + (long long)gy * d.pw + gi + q);
    const double U = __ldcg(P.u + oo + (long long)(gy - 1) * d.pw + gi);
    const double D = __ldcg(P.u + oo + (long long)(gy + 1) * d.pw + gi);
    const double lhs = fma(lam4, -__ldcg(P.u + o), ((L + R) + U) + D);
    const double res = lhs - __ldg(P.bp + o);
    P.g[o] = (float)(-res);
    acc = fma(res, res, acc);
  }
  acc = block_sum(acc, sred);
  if (threadIdx.x == 0) P.partial[t] = acc;
}

__device__ __forceinline__ void apply_stall(SysState &s, double rel, int &done) {
  // poisson.rs:219-228 (window 16 for a given omega; see k_init for automatic omega)
  if (rel < s.best * (1.0 - kStallImprovement)) {
    s.best = rel;
    s.since = 0;
  } else {
    s.since += 1;
    if (s.since >= s.stall_window) done = 1;
  }
}

__device__ SysState load_state(const SysState *p) {
  SysState s;
  const int *pi = reinterpret_cast<const int *>(p);
  int *si = reinterpret_cast<int *>(&s);
  for (int k = 0; k < (int)(sizeof(SysState) / sizeof(int)); ++k) si[k] = __ldcg(pi + k);
  return s;
}

// The state machine step run by the last tile of a system to finish a step
// (thread 0 only). sums[j] = sum of the tile partials of sweep j (tile order).
__device__ void advance(const KParams &P, const SysDesc &d, SysState *stp, int mode,
                        const double *sums) {
  SysState s = load_state(stp);
  double *hist = P.hist + d.hist_off;
  const int cap = P.S;
  switch (mode) {
    case M_SWEEP: {
      int kind = P_NONE, stop_j = -1;
      bool refine = false;
      for (int j = 0; j < s.s; ++j) {
        const double nrm = sqrt(sums[j]);
        const double rel = nrm / s.r0;  // poisson.rs:206
        s.iterations += 1;
        hist[s.iterations - 1] = rel;
        s.last = rel;
        if (rel <= d.tol) { kind = P_CONV; stop_j = j; break; }  // poisson.rs:210-214
        int stalled = 0;
        apply_stall(s, rel, stalled);
        if (stalled) { kind = P_STALL; stop_j = j; break; }
        if (s.iterations >= d.max_it) { kind = P_MAX; stop_j = j; break; }
        // residual-correction trigger (does not change the iterate, only when
        // the FP64 fold happens, so it waits for the end of the block)
        if (nrm <= kRefineFactor * s.ibase) refine = true;
        if (nrm < s.ibest * kInnerGain) { s.ibest = nrm; s.isince = 0; }
        else if (++s.isince >= kInnerWindow) refine = true;
      }
      if (kind == P_NONE) {
        s.cur ^= 1;
        if (refine) { s.pending = P_REFINE; s.mode = M_FOLD; }
        else { s.mode = M_SWEEP; s.s = min(cap, d.max_it - s.iterations); }
      } else if (stop_j == s.s - 1) {
        s.cur ^= 1; s.pending = kind; s.mode = M_FOLD;
      } else {
        // stop inside the block: re-run the block from the same start with
        // exactly stop_j+1 sweeps (identical arithmetic), so the iterate kept is
        // the one after the reported sweep.
        s.pending = kind; s.mode = M_REDO; s.s = stop_j + 1;
      }
    } break;
    case M_REDO:
      s.cur ^= 1;
      s.mode = M_FOLD;
      break;
    case M_FOLD:
      s.mode = M_RESID;
      break;
    case M_RESID: {
      const double nrm = sqrt(sums[0]);
      const double rel = nrm / s.r0;
      s.outer = nrm;
      s.ibase = nrm;
      s.ibest = INFINITY;
      s.isince = 0;
      s.refinements += 1;
      if (s.iterations > 0) { hist[s.iterations - 1] = rel; s.last = rel; }
      int stop = -1;
      if (rel <= d.tol) stop = STOP_CONVERGED;
      else if (s.pending == P_STALL) stop = STOP_STALLED;
      else if (s.pending == P_MAX || s.iterations >= d.max_it) stop = STOP_MAX;
      else if (s.pending == P_CONV) {
        // the per-sweep estimate met the tolerance but the FP64 residual does
        // not: apply the stall rule the estimate skipped, then keep sweeping
        int stalled = 0;
        apply_stall(s, rel, stalled);
        if (stalled) stop = STOP_STALLED;
      }
      s.pending = P_NONE;
      if (stop >= 0) {
        s.mode = M_DONE;
        s.status = stop;
        atomicAdd(P.bar + 2, 1u);
      } else {
        s.mode = M_SWEEP;
        s.s = min(cap, d.max_it - s.iterations);
      }
    } break;
    default:
      break;
  }
  s.steps += 1;
  *stp = s;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Thread 0: claim the next open tile of any system, starting at system `rot`.
// Returns the system (or -1 when every system is done, an error was raised or
// the wait for work exceeded its bound) and sets *idx, *gen.
__device__ int claim_tile(const KParams &P, int rot, int *idx, unsigned *gen,
                          unsigned long long t_start) {
  unsigned long long idle_from = 0;
  for (;;) {
    // an error anywhere or the wall budget ends every block at its next claim
    if (ld_vol(P.err) != 0) return -1;
    if (gtimer() - t_start > P.budget_ns) {
      atomicCAS(P.err, 0, KERR_DEADLINE);
      return -1;
    }
    for (int k = 0; k < P.nsys; ++k) {
      int c = rot + k;
      if (c >= P.nsys) c -= P.nsys;
      const unsigned nact = (unsigned)__ldcg(&P.st[c].nact);
      if ((unsigned)ld_acquire_u64(P.claim + c) >= nact) continue;  // step fully handed out
      const unsigned long long cw = atomicAdd(P.claim + c, 1ull);
      if ((unsigned)cw < nact) {
        *idx = (int)(unsigned)cw;
        *gen = (unsigned)(cw >> 32);
        __threadfence();  // the claimed generation's state was published before its claim word
        return c;
      }
    }
    if (ld_acquire(P.bar + 2) >= (unsigned)P.nsys) return -1;
    const unsigned long long now = gtimer();
    // every open step is handed out and being finished by other blocks; a
    // step takes milliseconds at most, so 20 s without work is a fault
    if (!idle_from) idle_from = now;
    else if (now - idle_from > 20ull * 1000000000ull) {
      atomicCAS(P.err, 0, KERR_STALLED);
      return -1;
    }
    __nanosleep(64);
  }
}

template <int S, int TH>
__global__ void __launch_bounds__(kThreads, 2) k_solve(KParams P) {
  using G = Geo<S, TH>;
  extern __shared__ __align__(16) unsigned char smem[];
  float *sE = reinterpret_cast<float *>(smem);
  float *sG = sE + 2 * G::PLANE;
  uint8_t *sC = reinterpret_cast<uint8_t *>(sG + 2 * G::PLANE);
  double *sred = reinterpret_cast<double *>(sC + 2 * G::PLANE);
  __shared__ int s_last, s_sys, s_idx;
  __shared__ unsigned s_gen;
  const unsigned long long t_start = gtimer();
  int rot = P.nsys > 0 ? (int)(blockIdx.x % (unsigned)P.nsys) : 0;

  for (;;) {
    if (threadIdx.x == 0) {
      int idx = 0;
      unsigned gen = 0;
      const int sys = claim_tile(P, rot, &idx, &gen, t_start);
      s_sys = sys;
      s_idx = idx;
      s_gen = gen;
    }
    __syncthreads();
    const int sys = s_sys, idx = s_idx;
    const unsigned gen = s_gen;
    __syncthreads();
    if (sys < 0) break;
    rot = sys;
    const SysDesc d = P.sys[sys];
    const int t = __ldcg(P.act + d.tile0 + idx);
    const Tile tl = P.tiles[t];
    SysState *stp = P.st + sys;
    const int mode = __ldcg(&stp->mode);
    const int s = __ldcg(&stp->s);
    const int cur = __ldcg(&stp->cur);
    if (mode == M_SWEEP || mode == M_REDO) {
      sweep_tile<S, TH>(P, d, t, tl, s, cur, sE, sG, sC, sred);
    } else if (mode == M_FOLD) {
      fold_tile<S, TH>(P, d, tl, cur);
    } else {
      resid_tile<S, TH>(P, d, t, tl, sred);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned a = atomicAdd(P.arrive + sys, 1u);
      s_last = (a == (unsigned)__ldcg(&stp->nact) - 1u);
      __threadfence();
    }
    __syncthreads();
    if (s_last) {
      // the system's step is complete: reduce its partials in tile order,
      // advance its state machine and open its next step
      double part[S];
#pragma unroll
      for (int j = 0; j < S; ++j) part[j] = 0.0;
      const int nsum = (mode == M_SWEEP) ? s : (mode == M_RESID ? 1 : 0);
      const int nact = __ldcg(&stp->nact);
      if (nsum > 0) {
        for (int k = threadIdx.x; k < nact; k += kThreads) {
          const int tk = __ldcg(P.act + d.tile0 + k);
#pragma unroll
          for (int j = 0; j < S; ++j)
            if (j < nsum) part[j] += __ldcg(P.partial + (long long)j * P.ntiles + tk);
        }
#pragma unroll
        for (int j = 0; j < S; ++j)
          if (j < nsum) part[j] = block_sum(part[j], sred);
      }
      if (threadIdx.x == 0) {
        advance(P, d, stp, mode, part);
        P.arrive[sys] = 0;
        __threadfence();
        const unsigned long long next = (unsigned long long)(gen + 1u) << 32;
        atomicExch(P.claim + sys, __ldcg(&stp->mode) == M_DONE ? (next | kClaimDone) : next);
      }
      __syncthreads();
    }
  }
}

// ----------------------------------------------------------------------------
// launch entry points (host)
// ----------------------------------------------------------------------------
template <int S, int TH>
static cudaError_t prepare_solve_t(const KParams &P, int sms, int *grid_out) {
  using G = Geo<S, TH>;
  cudaError_t e = cudaFuncSetAttribute(k_solve<S, TH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)G::kSmem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve<S, TH>, kThreads, G::kSmem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int grid = per_sm * sms;
  if (grid > P.ntiles) grid = P.ntiles > 0 ? P.ntiles : 1;
  *grid_out = grid;
  return cudaSuccess;
}

template <int S, int TH>
static cudaError_t launch_prepared_t(const KParams &P, int grid, cudaStream_t stream) {
  using G = Geo<S, TH>;
  KParams Pc = P;
  Pc.S = S;
  // No block waits for a particular other block (work is claimed, never
  // assigned), so an ordinary launch suffices; the grid fills the GPU once.
  k_solve<S, TH><<<grid, kThreads, G::kSmem, stream>>>(Pc);
  return cudaGetLastError();
}

int tile_config_count() { return 5; }

// (sweeps per step S, owned tile height TH); every loaded height TH + 2(2S+1)
// leaves rows 1..LH-2 a multiple of 32.
TileConfig tile_config(int idx) {
  switch (idx) {
    case 0: return {1, 60, tile_w(1)};
    case 1: return {2, 88, tile_w(2)};
    case 2: return {3, 84, tile_w(3)};
    case 3: return {3, 52, tile_w(3)};
    default: return {4, 80, tile_w(4)};
  }
}

size_t tile_config_smem(int idx) {
  switch (idx) {
    case 0: return Geo<1, 60>::kSmem;
    case 1: return Geo<2, 88>::kSmem;
    case 2: return Geo<3, 84>::kSmem;
    case 3: return Geo<3, 52>::kSmem;
    default: return Geo<4, 80>::kSmem;
  }
}

cudaError_t launch_assembly(const KParams &P, const TileConfig &tc, cudaStream_t stream, bool any_warm) {
  if (P.ntiles <= 0) return cudaSuccess;
  if (P.nregions > 0) {
    cudaError_t e = cudaMemsetAsync(P.rsize, 0, P.rpix * sizeof(int), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(P.rmax, 0, P.nregions * sizeof(int), stream);
    if (e != cudaSuccess) return e;
    long long nb = (P.rpix + 255) / 256;
    const unsigned blocks = (unsigned)(nb > 148 * 16 ? 148 * 16 : (nb < 1 ? 1 : nb));
    k_label_init<<<blocks, 256, 0, stream>>>(P);
    k_label_link<<<blocks, 256, 0, stream>>>(P);
    k_label_count<<<blocks, 256, 0, stream>>>(P);
    k_label_max<<<blocks, 256, 0, stream>>>(P);
  }
  k_tile_count<<<P.ntiles, 256, 0, stream>>>(P, tc.tw, tc.th);
  k_compact<<<P.nsys, 256, 0, stream>>>(P);
  k_assemble<<<P.ntiles, kThreads, 0, stream>>>(P, tc.tw, tc.th);
  k_init<<<P.nsys, 256, 0, stream>>>(P);
  if (any_warm) k_warm_fallback<<<P.ntiles, kThreads, 0, stream>>>(P, tc.tw, tc.th);
  return cudaGetLastError();
}

cudaError_t prepare_solve(const KParams &P, int cfg, int sms, int *grid) {
  switch (cfg) {
    case 0: return prepare_solve_t<1, 60>(P, sms, grid);
    case 1: return prepare_solve_t<2, 88>(P, sms, grid);
    case 2: return prepare_solve_t<3, 84>(P, sms, grid);
    case 3: return prepare_solve_t<3, 52>(P, sms, grid);
    default: return prepare_solve_t<4, 80>(P, sms, grid);
  }
}

cudaError_t launch_prepared(const KParams &P, int cfg, int grid, cudaStream_t stream) {
  switch (cfg) {
    case 0: return launch_prepared_t<1, 60>(P, grid, stream);
    case 1: return launch_prepared_t<2, 88>(P, grid, stream);
    case 2: return launch_prepared_t<3, 84>(P, grid, stream);
    case 3: return launch_prepared_t<3, 52>(P, grid, stream);
    default: return launch_prepared_t<4, 80>(P, grid, stream);
  }
}

cudaError_t launch_solve(const KParams &P, int cfg, int sms, cudaStream_t stream, int *grid) {
  cudaError_t e = prepare_solve(P, cfg, sms, grid);
  if (e != cudaSuccess) return e;
  return launch_prepared(P, cfg, *grid, stream);
}

cudaError_t launch_tile_count(const KParams &P, const TileConfig &tc, cudaStream_t stream) {
  if (P.ntiles <= 0) return cudaSuccess;
  k_tile_count<<<P.ntiles, 256, 0, stream>>>(P, tc.tw, tc.th);
  return cudaGetLastError();
}

cudaError_t launch_band_flags(const KParams &P, int sys0, int *spans, cudaStream_t stream) {
  k_band_flags<<<1, 256, 0, stream>>>(P, sys0, spans);
  return cudaGetLastError();
}

cudaError_t launch_emit(const KParams &P, int sys0, const TileConfig &tc, long long npx,
                        cudaStream_t stream) {
  if (npx <= 0) return cudaSuccess;
  long long blocks = (npx + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_emit<<<(int)blocks, 256, 0, stream>>>(P, sys0, tc.tw, tc.th);
  return cudaGetLastError();
}

}  // namespace ptk
