// unet_kernels.h -- launch interface of the U-Net kernels (unet_kernels.cu,
// conv_tma.cu).
//
// Activations are bf16 in a channel-blocked layout [B][C/8][H][W][8]: one
// plane per group of 8 channels, so a row of one plane is contiguous (16
// bytes per pixel) and the tensor-memory-accelerator (TMA) loads a run of
// pixels of one plane as a single wide line. A channel slice of a buffer (the
// decoder's concatenations write into slices) is a range of planes.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace unet {

// A channel slice of a blocked activation buffer.
struct ActView {
  __nv_bfloat16 *p;  // buffer base
  int cg;            // 8-channel groups of the whole buffer
  int g0;            // first group of the slice
};

// Element index of (image b, slice group g, row y, column x, channel 0 of the group).
__host__ __device__ __forceinline__ long long act_index(const ActView &v, int b, int g, int y, int x, int H,
                                                        int W) {
  return ((((long long)b * v.cg + v.g0 + g) * H + y) * W + x) * 8;
}

// 3x3 convolution (forward, or backward-data with flipped weights).
struct ConvArgs {
  ActView x;               // input slice
  int cin;                 // its channels (multiple of 16)
  const __nv_bfloat16 *w;  // [N][9][cin] bf16
  const float *bias;       // [N] or nullptr
  ActView y;               // output slice (N channels)
  int relu;                // apply max(0, .) after the bias
  ActView mask;            // mask.p != nullptr: zero outputs where mask <= 0 (ReLU backward)
  int B, H, W;
  int *err;                // set to 1 if a bounded wait gave up
  unsigned long long wait_ns;  // limit of each pipeline wait (0: the 2 s default)
  int stall;               // test knob: the MMA warp first waits on a phase nothing completes
};

// 3x3 convolution backward-weights.
struct WgradArgs {
  ActView dy;               // output gradient (pre-activation)
  int cout;                 // cout <= 128, multiple of 8
  ActView x;                // forward input
  int cin;                  // multiple of 16
  int B, H, W;
  float *part;              // [chunks][9][cout][cin] partials
  float *dw;                // [cout][9][cin] result
  float *db_part;           // [chunks][cout] bias-gradient partials (with db)
  float *db;                // [cout] bias gradient sum_p dY[p][co], or nullptr
  int *err;
};

// conv_tma.cu
cudaError_t launch_conv3x3(const ConvArgs &a, int n, cudaStream_t st);
int wgrad_chunks(int B, int H, int W);  // partial-sum chunks launch_wgrad writes
cudaError_t launch_wgrad(const WgradArgs &a, cudaStream_t st);

// unet_kernels.cu
// out[j] = sum over k = 0 .. nparts-1 (in order) of part[k][j], j < c
cudaError_t launch_reduce_rows(const float *part, int nparts, int c, float *out, cudaStream_t st);
cudaError_t launch_wgrad_reduce(const float *part, int nchunks, int cout, int cin, float *dw, const float *db_part,
                                float *db, cudaStream_t st);
cudaError_t launch_avgpool2(const ActView &in, const ActView &out, int B, int H, int W, int groups,
                            cudaStream_t st);
cudaError_t launch_unpool_add_mask(const ActView &dskip, const ActView &dpool, const ActView &act,
                                   const ActView &out, int B, int H, int W, int groups, cudaStream_t st);
cudaError_t launch_upsample2(const ActView &in, const ActView &out, int B, int Hi, int Wi, int groups,
                             cudaStream_t st);
cudaError_t launch_upsample2_bwd(const ActView &dout, const ActView &act, const ActView &din, int B, int Hi,
                                 int Wi, int groups, cudaStream_t st);
// 1x1 head on 16 channels (2 groups)
cudaError_t launch_head_fwd(const ActView &x, const float *w, const float *b, float *pred, int B, int H, int W,
                            cudaStream_t st);
int head_bwd_blocks(long long P);
cudaError_t launch_head_bwd(const ActView &x, const float *w, const float *dpred, const ActView &dx, int B, int H,
                            int W, float *part, cudaStream_t st);
int loss_blocks(long long P);
// count: 1 + loss_blocks(P) floats of scratch; count[0] receives the interior count
cudaError_t launch_loss(const float *pred, const float *target, const float *mask, long long P, float *dpred,
                        double *part, float *count, cudaStream_t st);
cudaError_t launch_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, long long n, float lr,
                        int step, cudaStream_t st);
// Adam on the fixed-order combination of `replicas` gradient records (n
// gradients + the interior count each, replica-major).
cudaError_t launch_adam_records(float *w, float *m, float *v, const float *records, int replicas, long long n,
                                float lr, int step, cudaStream_t st);
cudaError_t launch_prep_weights(const float *w, int cout, int cin, __nv_bfloat16 *wb, __nv_bfloat16 *wt,
                                cudaStream_t st);
// fp32 features (B x H x W x 4) -> the 16-channel input (2 groups, channels 4..15 zero)
cudaError_t launch_features_to_input(const float *f, const ActView &x, int B, int H, int W, cudaStream_t st);
cudaError_t launch_features(const float *guid, const float *anchor, const float *mask, int B, int H, int W,
                            float *f, cudaStream_t st);
// Warm start at another resolution: pool interleaved inputs by s into a
// (C x Hc x Wc) batch; compose guess = guidance + bilinear upsampling of the
// (C x Hc x Wc) correction.
cudaError_t launch_pool_inputs(const float *g, const float *a, const float *m, int W, int H, int C, int s, int Wc,
                               int Hc, float *cg, float *ca, float *cm, cudaStream_t st);
cudaError_t launch_compose_guess(const float *g, const float *corr, int W, int H, int C, int s, int Wc, int Hc,
                                 float *guess, cudaStream_t st);

}  // namespace unet
