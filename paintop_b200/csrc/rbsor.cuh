// rbsor.cuh -- device side of the B200 red-black SOR Poisson / screened-Poisson
// solver (sm_100a).
//
// Method. The reference relaxes each channel with row-major SOR in f64
// (crates/paintop-cpu/src/poisson.rs:244-265) and records ||r_k|| / ||r_0|| after
// every sweep (poisson.rs:202-229). This solver keeps the same discrete system,
// stopping rule, stall rule and report, and changes how the iterate is computed:
//
//   * the iterate is u = u64 + e: u64 an FP64 field, e an FP32 correction;
//   * sweeps are red-black SOR in FP32 on the correction equation
//       nsum(e) - (4 + lambda) e = g,   g = -r(u64)   (e = 0 on boundary cells);
//   * after every sweep the residual of u64 + e, rho = nsum(e) - (4+lambda) e - g,
//     is evaluated in FP64 and summed in FP64, giving the history entry;
//   * a FOLD step (u64 += e, e = 0) followed by a RESID step (g = -r(u64), with
//     r computed entirely in FP64 from u64) is the FP64 residual-correction
//     (iterative refinement) outer loop. It runs when the correction has reduced
//     the residual by a fixed factor, and before every stop, so every stop
//     decision and every final_residual is a true FP64 residual.
//
// Layout in HBM. Every channel of every image is one "system". Its fields are
// stored over the whole image in a red-black split layout: plane c (c = (x+y)&1)
// holds row y's cells of that colour, plane index i = x >> 1, with a row pitch
// of `pw` floats (a multiple of 4, so rows start 16-byte aligned). The planes
// are e0/e1 (ping-pong f32 correction), g (f32), cell (u8, 1 = interior),
// u (f64 iterate) and bp (f64, b - lambda*anchor).
//
// Tiles. The image is cut into tiles of TW x TH owned cells. A SWEEP step loads
// a tile with a halo of H = 2S+1 rows (Hx >= H columns, a multiple of 8 so plane
// loads stay 16-byte aligned) into shared memory, runs s <= S red-black sweeps
// on a window that shrinks by one cell per half-sweep (so every value it keeps
// equals the value a whole-grid sweep would produce), evaluates the FP64
// residual of the owned cells after every sweep, and writes the owned cells to
// the other ping-pong buffer. Tiles without interior cells are never swept.
//
// Control. One persistent kernel runs all steps of all systems as a dataflow:
// each system publishes its current step through a claim word (generation,
// next tile); any block takes the next tile of any system whose step is open.
// The last tile of a system to finish a step (per-system arrival counter) sums
// that system's per-tile partials in tile order -- a fixed order that depends
// on nothing but the tile grid, so reruns are byte-identical -- advances the
// system's state machine (record history, test tolerance, stall, cap; choose
// the next mode) and publishes the next generation. Systems therefore advance
// independently; no block ever waits for a particular other block, and an
// idle block's wait for work is bounded by a watchdog.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ptk {

constexpr int kLW = 128;          // loaded tile width in cells
constexpr int kPWL = kLW / 2;     // plane row width in shared memory (floats)
constexpr int kThreads = 512;     // threads per block of the tile kernels
constexpr int kWarps = kThreads / 32;

__host__ __device__ constexpr int halo_y(int S) { return 2 * S + 1; }
__host__ __device__ constexpr int halo_x(int S) { return ((2 * S + 1) + 7) / 8 * 8; }
__host__ __device__ constexpr int tile_w(int S) { return kLW - 2 * halo_x(S); }

// State machine modes.
enum Mode : int { M_SWEEP = 0, M_REDO = 1, M_FOLD = 2, M_RESID = 3, M_DONE = 4 };
// Why a system left the plain sweep loop.
enum Pending : int { P_NONE = 0, P_CONV = 1, P_STALL = 2, P_MAX = 3, P_REFINE = 4 };
// Stop reasons (SolverStopReason order).
enum Stop : int { STOP_CONVERGED = 0, STOP_MAX = 1, STOP_STALLED = 2 };

// Error codes written to the kernel error word.
enum KErr : int { KERR_NONE = 0, KERR_STALLED = 1, KERR_DEADLINE = 2 };

// poisson.rs:80,85 -- stall window and improvement fraction.
constexpr unsigned kStallWindow = 16;
constexpr double kStallImprovement = 1e-12;
// Residual-correction trigger: refine once the correction has reduced the
// residual of the current outer step by this factor ...
constexpr double kRefineFactor = 1e-3;
// ... or once its residual has not improved by at least 0.1% for kInnerWindow
// sweeps (the FP32 correction has reached its rounding floor). Refinement does
// not change the iterate (SOR is a stationary method: restarting it on the
// residual equation at a sweep boundary continues the same iteration), so an
// early trigger costs two cheap steps and nothing else.
constexpr double kInnerGain = 0.999;
constexpr int kInnerWindow = 16;

struct SysDesc {
  int inst, chan;          // image index in the batch, channel
  int W, H, C;             // image extent and channel count
  int pw;                  // plane pitch (floats), multiple of 4
  int ntx, nty;            // tile grid
  long long off;           // element offset of plane 0 in the cell pools
  long long plane;         // elements per plane (H * pw)
  int tile0, ntiles;       // range in the tile list
  const float *src;        // interleaved source / guidance image (W*H*C)
  const float *tgt;        // interleaved target / anchor image (W*H*C)
  const float *guess;      // interleaved initial guess or nullptr
  const float *mask;       // coverage mask (W*H)
  float *out;              // interleaved candidate (W*H*C)
  long long hist_off;      // offset of this system's history
  float omega, inv_denom;  // SOR factor (negative: choose it on device), 1 / (4 + lambda)
  double lambda;
  double tol;
  int max_it;
  int warm;                // 1 if an initial guess is staged
  int region1;             // 1 + index of the image's RegionDesc (automatic omega), 0: none
  int pad;
};

// Connected interior regions of one image, for the automatic SOR factor. The
// channels of an image share its mask, so each image is labelled once.
struct RegionDesc {
  long long lab_off;       // offset of the image's pixels in the label / size arrays
  int W, H;
  int sys0;                // the image's first system (its mask and extent)
  int pad;
};

struct SysState {
  int mode, s, iterations, cur;
  int pending, status, refinements, since;
  int isince, nact, out_anchor, steps;
  int warm_used;           // 1: the sweeps start from the caller's guess
  int pad1;
  double r0, outer, best, ibest, last, ibase;
  double omega;            // the SOR factor the sweeps use (chosen on device when automatic)
  int stall_window;        // sweeps without a new best that end the solve as stalled
  int pad2;
};

// Control words of the persistent kernel: [2] systems done. The host zeroes
// them before every launch.
constexpr int kBarWords = 16;
// A claim word's low half once its system is done: never below any tile count,
// and far from overflowing into the generation half however often it is bumped.
constexpr unsigned kClaimDone = 0x7fffffffu;

struct Tile {
  int sys, tx, ty, pad;
};

struct KParams {
  const SysDesc *sys;
  SysState *st;
  const Tile *tiles;
  int *tcount;             // interior cells per tile
  int4 *tbox;              // per tile: interior bounding box (min x, min y, max x, max y)
  int ntiles, nsys;
  float *e0, *e1, *g;
  uint8_t *cell;
  double *u, *bp;
  double *partial;         // [S][ntiles]
  double *fpart;           // [2][ntiles] assembly partials
  double *hist;
  int *act;                // per system, its tiles with interior cells, in index order
                           // (stored at the system's tile range)
  unsigned long long *claim;  // per system: generation << 32 | next tile to hand out
  unsigned *arrive;        // per system: tiles finished in the current generation
  unsigned *bar;           // control words, kBarWords of them
  int *err;
  unsigned long long budget_ns;
  int S;                   // sweeps per step of this launch
  // connected regions (automatic omega); nregions = 0 skips the labelling
  const RegionDesc *regions;
  int nregions;
  long long rpix;          // pixels of all labelled images
  int *label;              // per pixel: region root (local pixel index) or -1
  int *rsize;              // per pixel: region size, at the root
  int *rmax;               // per RegionDesc: largest region size
};

}  // namespace ptk
