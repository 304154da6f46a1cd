/*
 * paintop_cuda.h -- C ABI of the B200 `cuda` backend for paintop's Poisson /
 * screened-Poisson ops (`repair.poisson_blend@1`, `repair.screened_poisson@1`).
 *
 * This is the seam a Rust FFI crate binds. In the reference, an op backend is a
 * Rust `OpImplementation` (crates/paintop-core/src/executor/op_impl.rs:51-70)
 * registered with `ImplRegistry::register_backend`
 * (crates/paintop-core/src/executor/op_impl.rs:142-172); its compute() calls
 * `blend_channels` (crates/paintop-cpu/src/poisson_blend.rs:168-236), which calls
 * `poisson::solve` (crates/paintop-cpu/src/poisson.rs:167-240) per channel. The
 * entry points below replace that chain:
 *
 *   pt_poisson_solve        replaces blend_channels + solve for one image
 *                           (poisson_blend.rs:168-246, poisson.rs:167-240)
 *   pt_poisson_solve_batch  many independent images in one persistent launch
 *                           (no reference counterpart: the reference solves one
 *                           image per op call)
 *   pt_op_compute           replaces PoissonBlend::compute / ScreenedPoisson::compute
 *                           (poisson_blend.rs:534-600, screened_poisson.rs:361-430)
 *                           including resolve_controls / check_shapes validation
 *                           (poisson_blend.rs:102-139,417-445; screened_poisson.rs:66-112),
 *                           and EllipseMask::compute / PolygonMask::compute
 *                           (ellipse.rs:506-540, mask_polygon.rs:427-452)
 *   pt_op_compute_ex        the same ops with solve flags: PT_FLAG_MULTIGRID is a
 *                           second implementation of the two Poisson ops
 *   pt_mask_ellipse         replaces ellipse.rs rasterize (:545-565)
 *   pt_mask_polygon         replaces mask_polygon.rs rasterize (:259-286)
 *   pt_status_str           message for a status code (the reference's typed
 *                           errors: crates/paintop-ir/src/error.rs:23-114)
 *
 * Conventions: plain C types only; all image buffers are row-major,
 * channel-interleaved f32 (the reference's ResourceValue samples,
 * crates/paintop-core/src/executor/value.rs:35-69). Unless PT_FLAG_DEVICE_POINTERS
 * is set, every pointer is a host pointer owned by the caller. The library owns
 * device memory inside the context (reused across calls, grown to a high-water
 * mark). No function aborts, throws or panics across the ABI. A context is
 * internally serialised by a mutex; distinct contexts are independent, so the
 * library is reentrant across contexts. Results are deterministic: a rerun on the
 * same device with the same inputs is byte-identical.
 */
#ifndef PAINTOP_CUDA_H
#define PAINTOP_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. Mapping to the reference's error classes
 * (crates/paintop-ir/src/error.rs:23-114): PT_NO_DEVICE -> Policy (exit 4,
 * mirrors E_GPU_UNAVAILABLE in crates/paintop-wgpu/src/gpu/error.rs:17);
 * PT_INVALID_ARG -> Schema/Semantic as reported in pt_error; the rest ->
 * Execution (exit 5). No C++ exception leaves any entry point: a host
 * allocation failure inside a call returns PT_OOM, any other host-side
 * exception PT_INTERNAL, with the message in pt_ctx_last_error. */
typedef enum pt_status {
  PT_OK = 0,
  PT_NO_DEVICE = 1,     /* no CUDA device / driver, or the device is not sm_100 */
  PT_INVALID_ARG = 2,   /* a null pointer, a bad size, or an out-of-range control */
  PT_LAUNCH_FAILED = 3, /* a CUDA launch or copy failed */
  PT_TIMEOUT = 4,       /* the device watchdog expired (bounded waits, wall budget) */
  PT_OOM = 5,           /* device or host allocation failed */
  PT_INTERNAL = 6       /* any other failure */
} pt_status;

/* pt_problem.flags */
#define PT_FLAG_WARM_START 0x1u      /* initial_guess holds the interior start values */
#define PT_FLAG_DEVICE_POINTERS 0x2u /* every buffer (inputs, outputs, history) is device memory */
#define PT_FLAG_OMEGA_AUTO 0x4u      /* ignore `omega`; pick the red-black optimum per channel */
#define PT_FLAG_MULTIGRID 0x8u       /* solve by multigrid-preconditioned CG (FP32) inside FP64
                                        refinement instead of red-black SOR: the same system,
                                        bar and report fields; iterations count CG iterations,
                                        omega is ignored. Every problem of a batch must agree. */

/* Stop reasons: the kebab-case SolverStopReason of
 * crates/paintop-ir/src/resource.rs:1185-1194 in declaration order. */
#define PT_STOP_CONVERGED 0
#define PT_STOP_MAX_ITERATIONS 1
#define PT_STOP_STALLED 2

typedef struct pt_ctx pt_ctx;

/* One image to solve: the arguments of blend_channels (poisson_blend.rs:168-175)
 * plus the SolveControls (poisson.rs:145-154). For poisson_blend,
 * source_or_guidance = source and target_or_anchor = target; for
 * screened_poisson, guidance and anchor (screened_poisson.rs:394-401). */
typedef struct pt_problem {
  uint32_t width, height, channels;
  const float *source_or_guidance; /* width*height*channels */
  const float *target_or_anchor;   /* width*height*channels */
  const float *mask;               /* width*height coverage; > 0.5 is interior */
  double lambda;                   /* >= 0, finite */
  uint32_t max_iterations;         /* sweeps per channel */
  double tolerance;                /* relative residual ||r_k|| / ||r(anchor)|| */
  double omega;                    /* SOR factor in (0, 2); the op uses 1.8 */
  uint32_t flags;                  /* PT_FLAG_* */
  const float *initial_guess;      /* width*height*channels or NULL */
} pt_problem;

/* SolveReport (poisson.rs:126-141) without the history vector, plus what the
 * GPU method adds. */
typedef struct pt_report {
  uint32_t iterations;  /* sweeps run (the last block is clipped exactly) */
  int32_t converged;    /* 1 iff stop_reason == PT_STOP_CONVERGED */
  int32_t stop_reason;  /* PT_STOP_* */
  double tolerance;     /* the requested tolerance */
  double final_residual;/* == history[iterations-1], an FP64 residual; 0 if none */
  uint32_t history_len; /* == iterations */
  double omega_used;    /* the SOR factor the sweeps used */
  uint32_t refinements; /* FP64 residual-correction steps (incl. the final check) */
  int32_t channel;      /* the channel index (for the worst entry: which channel) */
  double initial_residual; /* ||r(anchor)||, the FP64 normaliser of every relative residual */
  int32_t warm_start;   /* 1: the sweeps started from initial_guess; 0: from the anchor
                           (no guess, or a guess whose FP64 residual norm was not below
                           ||r(anchor)||, which falls back to the plain start) */
} pt_report;

pt_status pt_ctx_create(int device, pt_ctx **out);
pt_status pt_ctx_destroy(pt_ctx *ctx);

/* Solve one image, every channel independently.
 *   out_candidate: width*height*channels f32 (caller-owned); equals the target
 *                  bit for bit at every non-interior pixel.
 *   reports:       channels + 1 entries: one per channel, then the worst channel
 *                  by (iterations, final_residual) as worse_of (poisson_blend.rs:240-246).
 *   history:       channels * max_iterations doubles, channel-major (may be NULL).
 */
pt_status pt_poisson_solve(pt_ctx *ctx, const pt_problem *p, float *out_candidate,
                           pt_report *reports, double *history);

/* Solve n independent images in one persistent launch. outs[i], reports[i]
 * (channels_i + 1 entries) and histories[i] (channels_i * max_iterations_i, or
 * NULL; `histories` itself may be NULL) follow pt_poisson_solve. Without
 * PT_FLAG_MULTIGRID, PT_FLAG_DEVICE_POINTERS must agree across the batch. With
 * PT_FLAG_MULTIGRID (on every problem), all images share each launch of the
 * multigrid-CG iteration, may mix host and device buffers, extents, channels,
 * lambda, tolerance and caps, and each image's output, reports and history are
 * bit for bit those of pt_poisson_solve on it alone. */
pt_status pt_poisson_solve_batch(pt_ctx *ctx, const pt_problem *ps, uint32_t n,
                                 float *const *outs, pt_report *const *reports,
                                 double *const *histories);

/* ---- mask generators (mask.ellipse@1, mask.polygon@1) ---------------------
 * The masks the solve consumes, made on the device so that a mask produced by
 * a plan node needs no host round trip. `mask` is width*height f32 coverage,
 * row-major; a device pointer when flags has PT_FLAG_DEVICE_POINTERS, else
 * host memory. Geometry is in pixel coordinates, pixel (i, j) spanning
 * [i, i+1) x [j, j+1). Non-finite geometry, a radius <= 0 or a negative
 * half-width is PT_INVALID_ARG (the op layer, pt_op_compute, reports the
 * reference's messages for them). */

/* mask.ellipse@1 (crates/paintop-cpu/src/ellipse.rs:168-218,545-565): the
 * analytic coverage at each pixel centre, a smoothstep feather of half-width
 * half_width_px about the first-order signed distance (0: hard, half-open
 * edge). Within the reference's tolerance (its hypot's last bit may differ). */
pt_status pt_mask_ellipse(pt_ctx *ctx, uint32_t width, uint32_t height, double center_x,
                          double center_y, double radius_x, double radius_y, double angle_rad,
                          double half_width_px, float *mask, uint32_t flags);

#define PT_FILL_NONZERO 0
#define PT_FILL_EVEN_ODD 1

/* mask.polygon@1 (crates/paintop-cpu/src/mask_polygon.rs:161-196,259-286): the
 * fraction of each pixel's 4 x 4 subsamples inside the polygon (vertices
 * points_xy[2k], points_xy[2k+1], closed implicitly) by the half-open +x ray
 * cast under fill_rule (PT_FILL_*). Fewer than 3 vertices give an all-zero
 * mask. Bit-identical to the reference. */
pt_status pt_mask_polygon(pt_ctx *ctx, uint32_t width, uint32_t height, const double *points_xy,
                          uint32_t n_points, int32_t fill_rule, float *mask, uint32_t flags);

/* ---- op-level entry (the OpImplementation::compute seam) ------------------ */

/* Resource kinds of an input port (crates/paintop-ir ResourceKind). */
#define PT_KIND_IMAGE 0
#define PT_KIND_MASK 1

typedef struct pt_port {
  const char *name;      /* "source"/"target"/"mask" or "guidance"/"anchor"/"mask" */
  uint32_t kind;         /* PT_KIND_* */
  uint32_t width, height;
  uint32_t channels;     /* channel count of the layout (mask: 1) */
  const float *samples;  /* width*height*channels, host memory */
  size_t sample_count;   /* length of samples */
} pt_port;

/* The reference's Error (crates/paintop-ir/src/error.rs): class token
 * ("schema", "reference", "type", "semantic", "policy", "execution"), stable
 * code (e.g. "E_POISSON_BLEND_PARAM") and message. */
typedef struct pt_error {
  char error_class[16];
  char code[40];
  char message[256];
  char actual[96];
} pt_error;

/* SolverData (crates/paintop-ir/src/resource.rs:1130-1178) built as
 * solver_data() does (poisson_blend.rs:249-266). */
typedef struct pt_solver_data {
  char kind[24];          /* "poisson" or "screened-poisson" */
  uint32_t steps;
  double stability_number;
  double stability_limit;
  int32_t stable;
  double total_energy;
  uint32_t iterations;
  int32_t stop_reason;    /* PT_STOP_* */
  int32_t converged;
  double tolerance;
  double final_residual;
  uint32_t history_len;   /* residual_history length */
} pt_solver_data;

/* Run the op (ctx may be NULL: the inputs and params are then validated and,
 * if valid, PT_NO_DEVICE is returned with E_CUDA_UNAVAILABLE). op_id is
 * "repair.poisson_blend@1" or "repair.screened_poisson@1";
 * params_json the op's JSON params object (e.g. {"tolerance":1e-6}). On PT_OK,
 * candidate (width*height*channels f32, caller-owned) and *solver are filled,
 * residual_history receives min(history_len, history_cap) entries and
 * *all_finite the report's all_finite flag. On PT_INVALID_ARG, *err carries the
 * reference's error class, code and message. */
pt_status pt_op_compute(pt_ctx *ctx, const char *op_id, const pt_port *inputs,
                        uint32_t n_inputs, const char *params_json, float *candidate,
                        size_t candidate_count, pt_solver_data *solver,
                        double *residual_history, uint32_t history_cap,
                        int32_t *all_finite, pt_error *err);

/* pt_op_compute with flags for the op's solve, for a backend implementation
 * registered beside the default one (a plan picks it by implementation id):
 * 0 is pt_op_compute exactly (red-black SOR); PT_FLAG_MULTIGRID solves the same
 * system to the same bar by multigrid-preconditioned CG, SolverData.steps and
 * .iterations then counting CG iterations. Any other bit is PT_INVALID_ARG
 * (E_CUDA_SOLVE_FLAGS). The mask generators ignore the flags. */
pt_status pt_op_compute_ex(pt_ctx *ctx, const char *op_id, const pt_port *inputs,
                           uint32_t n_inputs, const char *params_json, float *candidate,
                           size_t candidate_count, pt_solver_data *solver,
                           double *residual_history, uint32_t history_cap,
                           int32_t *all_finite, pt_error *err, uint32_t solve_flags);

const char *pt_status_str(pt_status s);

/* Last CUDA / watchdog detail recorded on this context ("" if none). */
const char *pt_ctx_last_error(const pt_ctx *ctx);

/* Wall budget of one persistent solve in seconds (default 600). A solve that
 * exceeds it stops at the next step boundary and returns PT_TIMEOUT; the
 * context stays usable. */
pt_status pt_ctx_set_budget(pt_ctx *ctx, double seconds);

/* The context's CUDA stream (a cudaStream_t), for callers that order their own
 * work or events with the library's. */
void *pt_ctx_stream(const pt_ctx *ctx);

/* Timing of the context's last solve or mask call, from CUDA events on its
 * stream: its main kernel alone (the persistent solve kernel, or the mask
 * rasteriser), the whole call (first upload to last download), and the number
 * of kernels the call launched. */
pt_status pt_ctx_last_timing(const pt_ctx *ctx, double *solve_kernel_ms, double *call_ms,
                             int64_t *kernel_launches);

/* Bytes the context's last red-black solve call (pt_poisson_solve or
 * pt_poisson_solve_batch without PT_FLAG_MULTIGRID) moved between host and
 * device. With host buffers a solve uploads the masks, then source, target
 * and guess only in the tile row bands that hold interior cells, each band as
 * one rectangle (its span of interior tile columns, one pixel and one row
 * either side: the part the solve reads), and downloads only the bands'
 * spans of the output; the rest of the output is the target, copied on the
 * host. Other calls set both counts to 0 (not counted). */
pt_status pt_ctx_last_transfer(const pt_ctx *ctx, uint64_t *h2d_bytes, uint64_t *d2h_bytes);

/* ---- tile configurations and the autotuner (no reference counterpart: the
 * reference has a single sequential sweep) -------------------------------- */

/* Number of compiled tile configurations (sweeps per step S, tile shape). */
uint32_t pt_tile_config_count(void);
pt_status pt_tile_config_info(uint32_t idx, int32_t *sweeps_per_step, int32_t *tile_w,
                              int32_t *tile_h);
/* Force a configuration for this context's solves (-1: use the tuned table). */
pt_status pt_ctx_set_config(pt_ctx *ctx, int32_t cfg);
/* The configuration the context's last solve used. */
int32_t pt_ctx_last_config(const pt_ctx *ctx);
/* Time every configuration on this batch, store the fastest in the shape-keyed
 * table (persisted to $PAINTOP_CUDA_TUNE_TABLE when set) and report it. Later
 * solves of the same shape read the table; they never re-time. */
pt_status pt_autotune(pt_ctx *ctx, const pt_problem *ps, uint32_t n, uint32_t repeats,
                      float *const *outs, pt_report *const *reports, int32_t *chosen,
                      double *ms_per_config);

/* ---- solving without allocating (no counterpart in the reference) -------- */

/* Size of the fixed device scratch array behind pt_poisson_solve_noalloc.
 * Every GPU that loads the library holds this much device memory until the
 * process exits. 64 MiB fits one 1024x1024 single-channel image or one 512x512
 * RGBA image with 2000 sweeps of history. */
#define PT_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)

/* pt_poisson_solve for callers that may not allocate memory: hosts whose device
 * memory belongs to another allocator (a plugin inside a framework's caching
 * pool must not call cudaMalloc/cudaFree behind it) and latency-critical threads
 * that cannot take the device synchronisation cudaMalloc/cudaFree may cause. It
 * needs no pt_ctx and makes no allocation call of any kind: its working memory
 * is a file-scope device array of PT_NOALLOC_SCRATCH_BYTES.
 *   p:         PT_FLAG_DEVICE_POINTERS must be set (inputs are the caller's
 *              device buffers); PT_FLAG_WARM_START and PT_FLAG_OMEGA_AUTO are
 *              not supported; at most 8 channels.
 *   out_candidate: device buffer, width*height*channels f32.
 *   reports:   host array of channels + 1 entries, as pt_poisson_solve.
 *   history:   device buffer of channels * max_iterations doubles, or NULL.
 *   stream:    the caller's cudaStream_t (NULL: the legacy default stream); the
 *              call returns after that stream has finished the solve.
 * Returns PT_OOM, before touching the GPU, when the problem needs more scratch
 * than PT_NOALLOC_SCRATCH_BYTES, and PT_INVALID_ARG for the same image limits
 * as pt_poisson_solve (width and height 1..2^30, at most 2^31 pixels and 2^34
 * values). The first call on each device (made with that device current) looks
 * up the array's device address once; make that first call before any stream
 * capture. The CUDA runtime loads modules lazily, so that first call is also
 * when the library's kernels and the array are placed on the device: the
 * guarantee of no allocation begins with the second call on each device. The
 * cached address is stale after cudaDeviceReset; calls after a reset are not
 * supported. A stream that is capturing is refused with PT_INVALID_ARG, since
 * the call copies from host memory and waits for its stream. All calls share
 * the one array and leave their contents in it; calls whose GPU work overlapped
 * would race on it, so each call holds a process-wide lock and waits for its
 * stream before returning. Uses the built-in tile configuration, never the
 * tuned table. */
pt_status pt_poisson_solve_noalloc(const pt_problem *p, float *out_candidate, pt_report *reports,
                                   double *history, void *stream);

/* ---- learned warm start (no counterpart in the reference) ----------------
 *
 * A small U-Net (4 levels of 16-32-64-128 channels, two 3x3 convolutions +
 * ReLU per level, 2x2 average pooling, bilinear x2 upsampling, skip
 * concatenation, 1x1 head) that predicts a solve's result from four per-pixel
 * features; its prediction seeds pt_poisson_solve through PT_FLAG_WARM_START.
 * Convolutions run on the tensor cores in bf16 with fp32 accumulation; the
 * parameters are fp32 masters trained with Adam (beta1 0.9, beta2 0.999, eps
 * 1e-8). Training steps are deterministic (fixed-order reductions).
 * All image buffers of these calls are DEVICE pointers: batch x h x w f32
 * (features: batch x h x w x 4). h and w must be multiples of 8. Calls on a
 * network take its context's lock and run on the context's stream. */
typedef struct pt_unet pt_unet;

/* He-normal initialisation from a SplitMix64 stream seeded with `seed`. */
pt_status pt_unet_create(pt_ctx *ctx, uint64_t seed, pt_unet **out);
pt_status pt_unet_destroy(pt_unet *net);
/* Number of fp32 parameters: per 3x3 layer W[cout][3][3][cin] then b[cout]
 * (the first layer's cin is 16, of which 4 are real inputs), then the head's
 * w[16] and b[1]. */
uint64_t pt_unet_param_count(const pt_unet *net);
pt_status pt_unet_get_params(pt_unet *net, float *host);
pt_status pt_unet_set_params(pt_unet *net, const float *host);
/* Features of single-channel images: 0 the guidance Laplacian at interior
 * cells (0 elsewhere), 1 anchor - guidance outside the interior (0 inside), 2
 * the interior mask, 3 the distance to the nearest non-interior cell along the
 * row and column, divided by 32 and clipped at 1 (0 outside). Interior = mask >
 * 0.5 and not on the image border (the reference's rule, poisson.rs:86-103).
 * The network predicts the correction u - guidance (harmonic inside the
 * interior for Poisson blending, with boundary values feature 1); the warm
 * start is guidance + prediction. */
pt_status pt_unet_features(pt_unet *net, const float *guidance, const float *anchor,
                           const float *mask, uint32_t batch, uint32_t h, uint32_t w,
                           float *features);
/* pred = network(features). */
pt_status pt_unet_forward(pt_unet *net, const float *features, uint32_t batch, uint32_t h,
                          uint32_t w, float *pred);
/* The masked mean squared error over pixels with loss_mask > 0.5 and, when
 * grad_host is not NULL, its gradient with respect to every parameter (host
 * array of pt_unet_param_count floats). Does not update the parameters. */
pt_status pt_unet_loss_grad(pt_unet *net, const float *features, const float *target,
                            const float *loss_mask, uint32_t batch, uint32_t h, uint32_t w,
                            double *loss, float *grad_host);
/* One Adam step on the masked mean squared error; *loss receives the loss of
 * the parameters before the step. */
pt_status pt_unet_train_step(pt_unet *net, const float *features, const float *target,
                             const float *loss_mask, uint32_t batch, uint32_t h, uint32_t w,
                             float lr, double *loss);
/* Data-parallel training, one replica per GPU. A replica's share of a step is
 * its gradient record: the gradient of the masked mean squared error over its
 * own part of the batch (pt_unet_param_count floats) followed by that part's
 * interior-pixel count, written to `record` (device memory, param_count + 1
 * floats). Does not update the parameters; *loss as in pt_unet_loss_grad. */
pt_status pt_unet_grad_record(pt_unet *net, const float *features, const float *target,
                              const float *loss_mask, uint32_t batch, uint32_t h, uint32_t w,
                              double *loss, float *record);
/* One Adam step on `replicas` gradient records laid end to end in device
 * memory (replica-major): each gradient weighted by its share of the interior
 * pixels and summed in replica order in fp64, which is the gradient of the
 * whole batch's masked mean squared error. Replicas that apply the same
 * records from the same state stay bit-identical; one record reproduces
 * pt_unet_train_step exactly. */
pt_status pt_unet_apply_records(pt_unet *net, const float *records, uint32_t replicas, float lr);
/* The warm start of one pt_poisson_solve problem (device pointers; images
 * width x height x channels interleaved, mask width x height): every channel
 * is pooled by `scale` (area average, 1 = full resolution), the network
 * predicts each channel's correction at that resolution, and
 *   guess = guidance + bilinear upsampling of the correction
 * is written to `guess` (width x height x channels), ready for
 * PT_FLAG_WARM_START. Pooling brings large regions to the size the network was
 * trained on (its receptive field is about 100 pixels). */
pt_status pt_unet_guess(pt_unet *net, const float *guidance, const float *anchor,
                        const float *mask, uint32_t width, uint32_t height, uint32_t channels,
                        uint32_t scale, float *guess);
/* Parameters and Adam moments to / from a file (little-endian, versioned). */
pt_status pt_unet_save(pt_unet *net, const char *path);
pt_status pt_unet_load(pt_unet *net, const char *path);

#ifdef __cplusplus
}
#endif
#endif /* PAINTOP_CUDA_H */
