// unet_kernels.h -- launch interface of the U-Net kernels (unet_kernels.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace unet {

// 3x3 convolution (forward, or backward-data with flipped weights).
struct ConvArgs {
  const __nv_bfloat16 *x;  // input, NHWC, row pitch ldx channels, first channel x_off
  int ldx, x_off, cin;     // cin: channels read (multiple of 16)
  const __nv_bfloat16 *w;  // [N][9][cin] bf16
  const float *bias;       // [N] or nullptr
  __nv_bfloat16 *y;        // output, NHWC, pitch ldy, first channel y_off
  int ldy, y_off;
  int relu;                // apply max(0, .) after the bias
  const __nv_bfloat16 *mask;  // optional: zero outputs where mask <= 0 (ReLU backward)
  int ldm, m_off;
  int B, H, W;
  int *err;                // set to 1 if a bounded wait gave up
};

// How a convolution's reduction axis (9 taps x cin channels) is cut into
// pipeline chunks (unet_kernels.cu states the rule).
struct ConvChunking {
  int kc;       // channels per part
  int cpt;      // channel parts
  int tpc;      // taps per chunk
  int ntg;      // tap groups
  int nchunks;  // ntg * cpt
  int kmax;     // K elements of the largest chunk
  int stages;   // pipeline stages in shared memory
};

// 3x3 convolution backward-weights.
struct WgradArgs {
  const __nv_bfloat16 *dy;  // output gradient (pre-activation), pitch lddy, offset dy_off
  int lddy, dy_off, cout;   // cout <= 128, multiple of 8
  const __nv_bfloat16 *x;   // forward input, pitch ldx, offset x_off
  int ldx, x_off;
  int cin;                  // input channels (the TMA path reads it; the gather path takes it as an argument)
  int B, H, W;
  float *part;              // [chunks][9][cout][cin] partials
  float *dw;                // [cout][9][cin] result
  int *err;
};

cudaError_t launch_conv3x3(const ConvArgs &a, int n, cudaStream_t st);
// TMA halo path (conv_tma.cu) for widths that are multiples of 128; the
// launchers return cudaErrorNotSupported when a tensor map cannot be built.
bool conv_tma_ok(const ConvArgs &a, int n);
cudaError_t launch_conv_tma(const ConvArgs &a, int n, cudaStream_t st);
bool wgrad_tma_ok(const WgradArgs &a, int cin);
int wgrad_tma_chunks(int B, int H, int W);
cudaError_t launch_wgrad_tma(const WgradArgs &a, int cin, cudaStream_t st, int *chunks);
cudaError_t launch_wgrad_reduce(const float *part, int nchunks, int cout, int cin, float *dw, cudaStream_t st);
int wgrad_chunks(int B, int H, int W);
cudaError_t launch_wgrad(const WgradArgs &a, int cin, cudaStream_t st);
int colsum_parts(long long P);
// out[j] = sum over k = 0 .. nparts-1 (in order) of part[k][j], j < c
cudaError_t launch_reduce_rows(const float *part, int nparts, int c, float *out, cudaStream_t st);
cudaError_t launch_colsum(const __nv_bfloat16 *dy, int ld, int off, int c, long long P, float *part,
                          float *out, cudaStream_t st);
cudaError_t launch_avgpool2(const __nv_bfloat16 *in, int ldi, int ioff, __nv_bfloat16 *out, int ldo, int ooff,
                            int B, int H, int W, int c, cudaStream_t st);
cudaError_t launch_unpool_add_mask(const __nv_bfloat16 *dskip, int lds, int soff, const __nv_bfloat16 *dpool,
                                   int ldp, int poff, const __nv_bfloat16 *act, int lda, int aoff,
                                   __nv_bfloat16 *out, int ldo, int ooff, int B, int H, int W, int c,
                                   cudaStream_t st);
cudaError_t launch_upsample2(const __nv_bfloat16 *in, int ldi, int ioff, __nv_bfloat16 *out, int ldo, int ooff,
                             int B, int Hi, int Wi, int c, cudaStream_t st);
cudaError_t launch_upsample2_bwd(const __nv_bfloat16 *dout, int ldd, int doff, const __nv_bfloat16 *act, int lda,
                                 int aoff, __nv_bfloat16 *din, int ldo, int ooff, int B, int Hi, int Wi, int c,
                                 cudaStream_t st);
cudaError_t launch_head_fwd(const __nv_bfloat16 *x, int ldx, int c, const float *w, const float *b, float *pred,
                            long long P, cudaStream_t st);
int head_bwd_blocks(long long P);
cudaError_t launch_head_bwd(const __nv_bfloat16 *x, int ldx, int c, const float *w, const float *dpred,
                            long long P, __nv_bfloat16 *dx, int lddx, float *part, cudaStream_t st);
int loss_blocks(long long P);
// count: 1 + loss_blocks(P) floats of scratch; count[0] receives the interior count
cudaError_t launch_loss(const float *pred, const float *target, const float *mask, long long P, float *dpred,
                        double *part, float *count, cudaStream_t st);
cudaError_t launch_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, long long n, float lr,
                        int step, cudaStream_t st);
cudaError_t launch_prep_weights(const float *w, int cout, int cin, __nv_bfloat16 *wb, __nv_bfloat16 *wt,
                                cudaStream_t st);
cudaError_t launch_features_to_input(const float *f, __nv_bfloat16 *x, long long P, cudaStream_t st);
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
