// unet.cu -- the learned warm start: network definition, training step and the
// pt_unet_* C ABI.
//
// Architecture: a 4-level U-Net with 16-32-64-128 channels,
// two 3x3 convolutions + ReLU per level, 2x2 average pooling down, bilinear x2
// upsampling up, skip concatenation (decoder input = [upsampled, skip]), and a
// 1x1 head to one output channel. Inputs: 4 feature channels (masked guidance
// divergence, boundary values, interior mask, distance to the boundary),
// zero-padded to 16 for the tensor core. The head predicts the solution at
// every pixel; the loss is the mean squared error over interior pixels.
//
// Parameters are fp32 master copies (flat, layer by layer: W[cout][3][3][cin]
// then b[cout]; the 1x1 head's w[16], b last) with bf16 copies for the tensor
// core, trained with Adam. Every reduction (weight gradients over pixels, bias
// gradients, loss) is a fixed-order sum, so a training step is deterministic.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../../include/paintop_cuda.h"
#include "../ctx.h"
#include "unet_kernels.h"
#include "../abi_guard.h"

using namespace unet;

namespace {

struct LayerSpec {
  int cout, cin;
};
// enc0a enc0b | enc1a enc1b | enc2a enc2b | bott a, b | dec2a dec2b | dec1a dec1b | dec0a dec0b
constexpr LayerSpec kLayers[14] = {{16, 16},  {16, 16},  {32, 16}, {32, 32}, {64, 32},
                                   {64, 64},  {128, 64}, {128, 128}, {64, 192}, {64, 64},
                                   {32, 96},  {32, 32},  {16, 48},  {16, 16}};
constexpr int kInReal = 4;   // real input channels of layer 0 (padded to 16)
constexpr int kHeadIn = 16;

struct Act {  // one bf16 NHWC tensor
  __nv_bfloat16 *p = nullptr;
  int c = 0;   // channels (row pitch)
  int level = 0;
};

}  // namespace

struct pt_unet {
  pt_ctx *ctx = nullptr;
  size_t nparam = 0;
  size_t w_off[14], b_off[14], head_w = 0, head_b = 0;
  size_t wb_off[14], wt_off[14];
  float *params = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
  __nv_bfloat16 *wbf = nullptr;  // bf16 weights and their flipped copies
  int step = 0;
  // activations, sized for (B, H, W)
  int B = 0, H = 0, W = 0;
  void *act_mem = nullptr;
  size_t act_bytes = 0;
  Act X0, E0a, CAT0, P1, E1a, CAT1, P2, E2a, CAT2, P3, E3a, E3, D2a, D2, D1a, D1, D0a, D0;
  Act dD0, dD0a, dCAT0, dD1, dD1a, dCAT1, dD2, dD2a, dCAT2, dE3, dE3a, dP3, de2, dE2a, dP2, de1, dE1a, dP1,
      de0, dE0a;
  float *pred = nullptr, *dpred = nullptr, *wpart = nullptr, *cpart = nullptr, *count = nullptr;
  double *lpart = nullptr;
  int *err = nullptr;
  float *gmem = nullptr;  // scratch of pt_unet_guess, grown to a high-water mark
  size_t gmem_bytes = 0;
  std::mutex mu;
};

namespace {

uint64_t splitmix(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uniform01(uint64_t &s) { return ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
double normal(uint64_t &s) {  // Box-Muller
  const double u1 = uniform01(s), u2 = uniform01(s);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

pt_status cfail(pt_unet *n, cudaError_t e, const char *what) {
  if (n && n->ctx) n->ctx->last_error = std::string(what) + ": " + cudaGetErrorName(e);
  if (e == cudaErrorMemoryAllocation) return PT_OOM;
  return PT_LAUNCH_FAILED;
}

#define CK(expr, what)                          \
  do {                                          \
    cudaError_t _e = (expr);                    \
    if (_e != cudaSuccess) return cfail(n, _e, what); \
  } while (0)

long long npix(const pt_unet *n, int level) {
  return (long long)n->B * (n->H >> level) * (n->W >> level);
}

// (Re)size the activation buffers for a batch shape.
pt_status ensure_acts(pt_unet *n, int B, int H, int W) {
  if (n->act_mem && n->B == B && n->H == H && n->W == W)
    // a wait that gave up in an earlier call must not fail this one
    return cudaMemsetAsync(n->err, 0, sizeof(int), n->ctx->stream) == cudaSuccess ? PT_OK : PT_LAUNCH_FAILED;
  struct Item { Act *a; int c; int level; };
  Item items[] = {{&n->X0, 16, 0},  {&n->E0a, 16, 0}, {&n->CAT0, 48, 0}, {&n->P1, 16, 1},   {&n->E1a, 32, 1},
                  {&n->CAT1, 96, 1}, {&n->P2, 32, 2},  {&n->E2a, 64, 2},  {&n->CAT2, 192, 2}, {&n->P3, 64, 3},
                  {&n->E3a, 128, 3}, {&n->E3, 128, 3}, {&n->D2a, 64, 2},  {&n->D2, 64, 2},    {&n->D1a, 32, 1},
                  {&n->D1, 32, 1},   {&n->D0a, 16, 0}, {&n->D0, 16, 0},   {&n->dD0, 16, 0},   {&n->dD0a, 16, 0},
                  {&n->dCAT0, 48, 0}, {&n->dD1, 32, 1}, {&n->dD1a, 32, 1}, {&n->dCAT1, 96, 1}, {&n->dD2, 64, 2},
                  {&n->dD2a, 64, 2}, {&n->dCAT2, 192, 2}, {&n->dE3, 128, 3}, {&n->dE3a, 128, 3},
                  {&n->dP3, 64, 3},  {&n->de2, 64, 2},  {&n->dE2a, 64, 2}, {&n->dP2, 32, 2},  {&n->de1, 32, 1},
                  {&n->dE1a, 32, 1}, {&n->dP1, 16, 1},  {&n->de0, 16, 0},  {&n->dE0a, 16, 0}};
  const long long P0 = (long long)B * H * W;
  size_t total = 0;
  auto al = [](size_t v) { return (v + 255) / 256 * 256; };
  for (auto &it : items) total += al((size_t)P0 / (1ull << (2 * it.level)) * it.c * 2);
  // fp32/double scratch
  size_t maxch = 0, maxdb = 0;
  for (int l = 0; l < 14; ++l) {
    const int lev = (l <= 1 || l >= 12) ? 0 : (l <= 3 || l >= 10) ? 1 : (l <= 5 || l >= 8) ? 2 : 3;
    const int ch = wgrad_chunks(B, H >> lev, W >> lev);
    const size_t need = (size_t)ch * 9 * kLayers[l].cout * kLayers[l].cin;
    if (need > maxch) maxch = need;
    if ((size_t)ch * kLayers[l].cout > maxdb) maxdb = (size_t)ch * kLayers[l].cout;
  }
  const size_t f_pred = al(P0 * 4), f_dpred = al(P0 * 4), f_w = al((size_t)maxch * 4),
               f_c = al(std::max(maxdb, (size_t)head_bwd_blocks(P0) * (kHeadIn + 1)) * 4), f_cnt = al(1025 * 4),
               f_l = al(1024 * 8), f_err = 256;
  total += f_pred + f_dpred + f_w + f_c + f_cnt + f_l + f_err;
  if (n->act_mem) { cudaFree(n->act_mem); n->act_mem = nullptr; }
  if (cudaMalloc(&n->act_mem, total) != cudaSuccess) { cudaGetLastError(); n->B = 0; return PT_OOM; }
  n->act_bytes = total;
  char *q = static_cast<char *>(n->act_mem);
  for (auto &it : items) {
    it.a->p = reinterpret_cast<__nv_bfloat16 *>(q);
    it.a->c = it.c;
    it.a->level = it.level;
    q += al((size_t)P0 / (1ull << (2 * it.level)) * it.c * 2);
  }
  n->pred = reinterpret_cast<float *>(q); q += f_pred;
  n->dpred = reinterpret_cast<float *>(q); q += f_dpred;
  n->wpart = reinterpret_cast<float *>(q); q += f_w;
  n->cpart = reinterpret_cast<float *>(q); q += f_c;
  n->count = reinterpret_cast<float *>(q); q += f_cnt;
  n->lpart = reinterpret_cast<double *>(q); q += f_l;
  n->err = reinterpret_cast<int *>(q);
  n->B = B; n->H = H; n->W = W;
  return cudaMemset(n->err, 0, sizeof(int)) == cudaSuccess ? PT_OK : PT_LAUNCH_FAILED;
}

// A channel slice [off, ...) of a buffer (off a multiple of 8).
ActView view(const Act &t, int off = 0) { return ActView{t.p, t.c / 8, off / 8}; }

// Host fault injection for tests of the bounded waits (no GPU fault involved):
// PAINTOP_CUDA_FAULT=unet-stall makes the first convolution of a forward pass
// wait on a barrier phase that nothing completes, under a 0.1 s limit. The
// wait runs out, the kernel takes its abort path, and the call returns
// PT_TIMEOUT; the next call runs normally.
bool stall_injected() {
  const char *f = std::getenv("PAINTOP_CUDA_FAULT");
  return f && !std::strcmp(f, "unet-stall");
}

pt_status conv(pt_unet *n, int l, const Act &x, int x_off, const Act &y, int y_off, bool relu,
               bool stall = false) {
  ConvArgs a{};
  if (stall) {
    a.stall = 1;
    a.wait_ns = 100000000ull;
  }
  a.x = view(x, x_off); a.cin = kLayers[l].cin;
  a.w = n->wbf + n->wb_off[l];
  a.bias = n->params + n->b_off[l];
  a.y = view(y, y_off); a.relu = relu ? 1 : 0;
  a.B = n->B; a.H = n->H >> x.level; a.W = n->W >> x.level; a.err = n->err;
  CK(launch_conv3x3(a, kLayers[l].cout, n->ctx->stream), "conv forward");
  return PT_OK;
}

// dX = conv(dY, W') (times the ReLU mask of X when `mask` is given)
pt_status dgrad(pt_unet *n, int l, const Act &dy, const Act &dx, int dx_off, const Act *mask, int m_off) {
  ConvArgs a{};
  a.x = view(dy); a.cin = kLayers[l].cout;
  a.w = n->wbf + n->wt_off[l];
  a.bias = nullptr;
  a.y = view(dx, dx_off); a.relu = 0;
  if (mask) a.mask = view(*mask, m_off);
  a.B = n->B; a.H = n->H >> dy.level; a.W = n->W >> dy.level; a.err = n->err;
  CK(launch_conv3x3(a, kLayers[l].cin, n->ctx->stream), "conv backward-data");
  return PT_OK;
}

// dW and db (into grad) from dY (pre-activation) and the forward input x;
// db[co] = sum over pixels of dY[p][co], summed by the same kernel
pt_status wgrad(pt_unet *n, int l, const Act &dy, const Act &x, int x_off) {
  WgradArgs a{};
  a.dy = view(dy); a.cout = kLayers[l].cout;
  a.x = view(x, x_off); a.cin = kLayers[l].cin;
  a.B = n->B; a.H = n->H >> dy.level; a.W = n->W >> dy.level;
  a.part = n->wpart; a.dw = n->grad + n->w_off[l]; a.err = n->err;
  a.db_part = n->cpart; a.db = n->grad + n->b_off[l];
  CK(launch_wgrad(a, n->ctx->stream), "conv backward-weights");
  return PT_OK;
}

#define RET(expr)                     \
  do {                                \
    pt_status _s = (expr);            \
    if (_s != PT_OK) return _s;       \
  } while (0)

pt_status forward(pt_unet *n, const float *features) {
  cudaStream_t st = n->ctx->stream;
  const long long P0 = npix(n, 0);
  (void)P0;
  CK(launch_features_to_input(features, view(n->X0), n->B, n->H, n->W, st), "input");
  RET(conv(n, 0, n->X0, 0, n->E0a, 0, true, stall_injected()));
  RET(conv(n, 1, n->E0a, 0, n->CAT0, 32, true));  // e0 -> skip slice
  CK(launch_avgpool2(view(n->CAT0, 32), view(n->P1), n->B, n->H, n->W, 2, st), "pool");
  RET(conv(n, 2, n->P1, 0, n->E1a, 0, true));
  RET(conv(n, 3, n->E1a, 0, n->CAT1, 64, true));  // e1
  CK(launch_avgpool2(view(n->CAT1, 64), view(n->P2), n->B, n->H >> 1, n->W >> 1, 4, st), "pool");
  RET(conv(n, 4, n->P2, 0, n->E2a, 0, true));
  RET(conv(n, 5, n->E2a, 0, n->CAT2, 128, true));  // e2
  CK(launch_avgpool2(view(n->CAT2, 128), view(n->P3), n->B, n->H >> 2, n->W >> 2, 8, st), "pool");
  RET(conv(n, 6, n->P3, 0, n->E3a, 0, true));
  RET(conv(n, 7, n->E3a, 0, n->E3, 0, true));
  CK(launch_upsample2(view(n->E3), view(n->CAT2), n->B, n->H >> 3, n->W >> 3, 16, st), "up");
  RET(conv(n, 8, n->CAT2, 0, n->D2a, 0, true));
  RET(conv(n, 9, n->D2a, 0, n->D2, 0, true));
  CK(launch_upsample2(view(n->D2), view(n->CAT1), n->B, n->H >> 2, n->W >> 2, 8, st), "up");
  RET(conv(n, 10, n->CAT1, 0, n->D1a, 0, true));
  RET(conv(n, 11, n->D1a, 0, n->D1, 0, true));
  CK(launch_upsample2(view(n->D1), view(n->CAT0), n->B, n->H >> 1, n->W >> 1, 4, st), "up");
  RET(conv(n, 12, n->CAT0, 0, n->D0a, 0, true));
  RET(conv(n, 13, n->D0a, 0, n->D0, 0, true));
  CK(launch_head_fwd(view(n->D0), n->params + n->head_w, n->params + n->head_b, n->pred, n->B, n->H, n->W, st),
     "head");
  return PT_OK;
}

pt_status backward(pt_unet *n, const float *target, const float *mask, double *loss) {
  cudaStream_t st = n->ctx->stream;
  const long long P0 = npix(n, 0);
  const int nlb = loss_blocks(P0);
  CK(launch_loss(n->pred, target, mask, P0, n->dpred, n->lpart, n->count, st), "loss");
  // head
  CK(launch_head_bwd(view(n->D0), n->params + n->head_w, n->dpred, view(n->dD0), n->B, n->H, n->W, n->cpart, st),
     "head backward");
  // the head partials [blocks][17], in block order, into grad[head_w .. head_b]
  CK(launch_reduce_rows(n->cpart, head_bwd_blocks(P0), kHeadIn + 1, n->grad + n->head_w, st), "head reduce");
  const int B = n->B, H = n->H, W = n->W;
  // decoder level 0
  RET(wgrad(n, 13, n->dD0, n->D0a, 0));
  RET(dgrad(n, 13, n->dD0, n->dD0a, 0, &n->D0a, 0));
  RET(wgrad(n, 12, n->dD0a, n->CAT0, 0));
  RET(dgrad(n, 12, n->dD0a, n->dCAT0, 0, nullptr, 0));
  CK(launch_upsample2_bwd(view(n->dCAT0), view(n->D1), view(n->dD1), B, H >> 1, W >> 1, 4, st), "up bwd");
  // decoder level 1
  RET(wgrad(n, 11, n->dD1, n->D1a, 0));
  RET(dgrad(n, 11, n->dD1, n->dD1a, 0, &n->D1a, 0));
  RET(wgrad(n, 10, n->dD1a, n->CAT1, 0));
  RET(dgrad(n, 10, n->dD1a, n->dCAT1, 0, nullptr, 0));
  CK(launch_upsample2_bwd(view(n->dCAT1), view(n->D2), view(n->dD2), B, H >> 2, W >> 2, 8, st), "up bwd");
  // decoder level 2
  RET(wgrad(n, 9, n->dD2, n->D2a, 0));
  RET(dgrad(n, 9, n->dD2, n->dD2a, 0, &n->D2a, 0));
  RET(wgrad(n, 8, n->dD2a, n->CAT2, 0));
  RET(dgrad(n, 8, n->dD2a, n->dCAT2, 0, nullptr, 0));
  CK(launch_upsample2_bwd(view(n->dCAT2), view(n->E3), view(n->dE3), B, H >> 3, W >> 3, 16, st), "up bwd");
  // bottleneck
  RET(wgrad(n, 7, n->dE3, n->E3a, 0));
  RET(dgrad(n, 7, n->dE3, n->dE3a, 0, &n->E3a, 0));
  RET(wgrad(n, 6, n->dE3a, n->P3, 0));
  RET(dgrad(n, 6, n->dE3a, n->dP3, 0, nullptr, 0));
  CK(launch_unpool_add_mask(view(n->dCAT2, 128), view(n->dP3), view(n->CAT2, 128), view(n->de2), B, H >> 2,
                            W >> 2, 8, st),
     "unpool");
  // encoder level 2
  RET(wgrad(n, 5, n->de2, n->E2a, 0));
  RET(dgrad(n, 5, n->de2, n->dE2a, 0, &n->E2a, 0));
  RET(wgrad(n, 4, n->dE2a, n->P2, 0));
  RET(dgrad(n, 4, n->dE2a, n->dP2, 0, nullptr, 0));
  CK(launch_unpool_add_mask(view(n->dCAT1, 64), view(n->dP2), view(n->CAT1, 64), view(n->de1), B, H >> 1,
                            W >> 1, 4, st),
     "unpool");
  // encoder level 1
  RET(wgrad(n, 3, n->de1, n->E1a, 0));
  RET(dgrad(n, 3, n->de1, n->dE1a, 0, &n->E1a, 0));
  RET(wgrad(n, 2, n->dE1a, n->P1, 0));
  RET(dgrad(n, 2, n->dE1a, n->dP1, 0, nullptr, 0));
  CK(launch_unpool_add_mask(view(n->dCAT0, 32), view(n->dP1), view(n->CAT0, 32), view(n->de0), B, H, W, 2, st),
     "unpool");
  // encoder level 0
  RET(wgrad(n, 1, n->de0, n->E0a, 0));
  RET(dgrad(n, 1, n->de0, n->dE0a, 0, &n->E0a, 0));
  RET(wgrad(n, 0, n->dE0a, n->X0, 0));
  // loss value: fixed-order sum of the block partials on the host
  std::vector<double> lp(nlb);
  float cnt = 0.0f;
  int kerr = 0;
  CK(cudaMemcpyAsync(lp.data(), n->lpart, nlb * sizeof(double), cudaMemcpyDeviceToHost, st), "loss copy");
  CK(cudaMemcpyAsync(&cnt, n->count, sizeof(float), cudaMemcpyDeviceToHost, st), "count copy");
  CK(cudaMemcpyAsync(&kerr, n->err, sizeof(int), cudaMemcpyDeviceToHost, st), "err copy");
  CK(cudaStreamSynchronize(st), "sync");
  if (kerr) {
    n->ctx->last_error = "a tensor-core pipeline wait gave up";
    return PT_TIMEOUT;
  }
  double s = 0.0;
  for (double v : lp) s += v;
  if (loss) *loss = s / std::max(1.0f, cnt);
  return PT_OK;
}

pt_status refresh_weights(pt_unet *n) {
  for (int l = 0; l < 14; ++l)
    CK(launch_prep_weights(n->params + n->w_off[l], kLayers[l].cout, kLayers[l].cin, n->wbf + n->wb_off[l],
                           n->wbf + n->wt_off[l], n->ctx->stream),
       "weights");
  return PT_OK;
}

pt_status check_shape(uint32_t B, uint32_t H, uint32_t W) {
  if (B == 0 || H < 8 || W < 8 || H % 8 || W % 8) return PT_INVALID_ARG;
  if ((unsigned long long)B * H * W > (1ull << 31)) return PT_INVALID_ARG;
  return PT_OK;
}

}  // namespace

extern "C" {

pt_status pt_unet_create(pt_ctx *ctx, uint64_t seed, pt_unet **out) {
  return abi_guard(ctx, [&]() -> pt_status {
    if (!ctx || !out) return PT_INVALID_ARG;
    *out = nullptr;
    pt_unet *n = new (std::nothrow) pt_unet();
    if (!n) return PT_OOM;
    n->ctx = ctx;
    size_t off = 0, boff = 0;
    for (int l = 0; l < 14; ++l) {
      n->w_off[l] = off;
      off += (size_t)kLayers[l].cout * 9 * kLayers[l].cin;
      n->b_off[l] = off;
      off += kLayers[l].cout;
      n->wb_off[l] = boff;
      boff += (size_t)kLayers[l].cout * 9 * kLayers[l].cin;
      n->wt_off[l] = boff;
      boff += (size_t)kLayers[l].cout * 9 * kLayers[l].cin;
    }
    n->head_w = off;
    off += kHeadIn;
    n->head_b = off;
    off += 1;
    n->nparam = off;
    // He-normal initialisation (std sqrt(2 / fan_in)) from a seeded SplitMix64;
    // biases zero; padded input channels of layer 0 zero.
    std::vector<float> h(off, 0.0f);
    uint64_t s = seed ^ 0x5eed5eed5eedull;
    for (int l = 0; l < 14; ++l) {
      const int ci_real = l == 0 ? kInReal : kLayers[l].cin;
      const double sd = std::sqrt(2.0 / (9.0 * ci_real));
      for (int co = 0; co < kLayers[l].cout; ++co)
        for (int t = 0; t < 9; ++t)
          for (int ci = 0; ci < kLayers[l].cin; ++ci)
            h[n->w_off[l] + ((size_t)co * 9 + t) * kLayers[l].cin + ci] = ci < ci_real ? (float)(sd * normal(s)) : 0.0f;
    }
    for (int k = 0; k < kHeadIn; ++k) h[n->head_w + k] = (float)(std::sqrt(1.0 / kHeadIn) * normal(s));
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    bool okm = cudaMalloc(&n->params, off * 4) == cudaSuccess && cudaMalloc(&n->m, off * 4) == cudaSuccess &&
               cudaMalloc(&n->v, off * 4) == cudaSuccess && cudaMalloc(&n->grad, off * 4) == cudaSuccess &&
               cudaMalloc(&n->wbf, boff * 2) == cudaSuccess;
    if (!okm) {
      cudaGetLastError();
      cudaFree(n->params); cudaFree(n->m); cudaFree(n->v); cudaFree(n->grad); cudaFree(n->wbf);
      delete n;
      return PT_OOM;
    }
    cudaMemcpy(n->params, h.data(), off * 4, cudaMemcpyHostToDevice);
    cudaMemset(n->m, 0, off * 4);
    cudaMemset(n->v, 0, off * 4);
    cudaMemset(n->grad, 0, off * 4);
    if (refresh_weights(n) != PT_OK || cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      pt_unet_destroy(n);
      return PT_LAUNCH_FAILED;
    }
    *out = n;
    return PT_OK;
  });
}

pt_status pt_unet_destroy(pt_unet *n) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n) return PT_OK;
    if (n->ctx) {
      std::lock_guard<std::mutex> lock(n->ctx->mu);
      cudaSetDevice(n->ctx->device);
      cudaStreamSynchronize(n->ctx->stream);
      cudaFree(n->params); cudaFree(n->m); cudaFree(n->v); cudaFree(n->grad); cudaFree(n->wbf);
      cudaFree(n->act_mem);
      cudaFree(n->gmem);
    }
    delete n;
    return PT_OK;
  });
}

uint64_t pt_unet_param_count(const pt_unet *n) { return n ? n->nparam : 0; }

pt_status pt_unet_get_params(pt_unet *n, float *host) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !host) return PT_INVALID_ARG;
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    CK(cudaMemcpy(host, n->params, n->nparam * 4, cudaMemcpyDeviceToHost), "get params");
    return PT_OK;
  });
}

pt_status pt_unet_set_params(pt_unet *n, const float *host) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !host) return PT_INVALID_ARG;
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    CK(cudaMemcpy(n->params, host, n->nparam * 4, cudaMemcpyHostToDevice), "set params");
    RET(refresh_weights(n));
    CK(cudaStreamSynchronize(n->ctx->stream), "sync");
    return PT_OK;
  });
}

pt_status pt_unet_features(pt_unet *n, const float *guidance, const float *anchor, const float *mask,
                           uint32_t batch, uint32_t h, uint32_t w, float *features) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !guidance || !anchor || !mask || !features || !batch || !h || !w) return PT_INVALID_ARG;
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    CK(launch_features(guidance, anchor, mask, (int)batch, (int)h, (int)w, features, n->ctx->stream), "features");
    CK(cudaStreamSynchronize(n->ctx->stream), "sync");
    return PT_OK;
  });
}

pt_status pt_unet_forward(pt_unet *n, const float *features, uint32_t batch, uint32_t h, uint32_t w, float *pred) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !features || !pred) return PT_INVALID_ARG;
    RET(check_shape(batch, h, w));
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    cudaSetDevice(n->ctx->device);
    RET(ensure_acts(n, (int)batch, (int)h, (int)w));
    RET(forward(n, features));
    const long long P0 = npix(n, 0);
    CK(cudaMemcpyAsync(pred, n->pred, P0 * 4, cudaMemcpyDeviceToDevice, n->ctx->stream), "pred copy");
    int kerr = 0;
    CK(cudaMemcpyAsync(&kerr, n->err, sizeof(int), cudaMemcpyDeviceToHost, n->ctx->stream), "err copy");
    CK(cudaStreamSynchronize(n->ctx->stream), "sync");
    if (kerr) {
      n->ctx->last_error = "a tensor-core pipeline wait gave up";
      return PT_TIMEOUT;
    }
    return PT_OK;
  });
}

pt_status pt_unet_loss_grad(pt_unet *n, const float *features, const float *target, const float *loss_mask,
                            uint32_t batch, uint32_t h, uint32_t w, double *loss, float *grad_host) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !features || !target || !loss_mask) return PT_INVALID_ARG;
    RET(check_shape(batch, h, w));
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    cudaSetDevice(n->ctx->device);
    RET(ensure_acts(n, (int)batch, (int)h, (int)w));
    RET(forward(n, features));
    RET(backward(n, target, loss_mask, loss));
    if (grad_host) CK(cudaMemcpy(grad_host, n->grad, n->nparam * 4, cudaMemcpyDeviceToHost), "grad copy");
    return PT_OK;
  });
}

pt_status pt_unet_train_step(pt_unet *n, const float *features, const float *target, const float *loss_mask,
                             uint32_t batch, uint32_t h, uint32_t w, float lr, double *loss) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !features || !target || !loss_mask || !(lr > 0.0f)) return PT_INVALID_ARG;
    RET(check_shape(batch, h, w));
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    cudaSetDevice(n->ctx->device);
    RET(ensure_acts(n, (int)batch, (int)h, (int)w));
    RET(forward(n, features));
    RET(backward(n, target, loss_mask, loss));
    n->step += 1;
    CK(launch_adam(n->params, n->m, n->v, n->grad, nullptr, (long long)n->nparam, lr, n->step, n->ctx->stream),
       "adam");
    RET(refresh_weights(n));
    return PT_OK;
  });
}

pt_status pt_unet_grad_record(pt_unet *n, const float *features, const float *target, const float *loss_mask,
                              uint32_t batch, uint32_t h, uint32_t w, double *loss, float *record) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !features || !target || !loss_mask || !record) return PT_INVALID_ARG;
    RET(check_shape(batch, h, w));
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    cudaSetDevice(n->ctx->device);
    RET(ensure_acts(n, (int)batch, (int)h, (int)w));
    RET(forward(n, features));
    RET(backward(n, target, loss_mask, loss));
    cudaStream_t st = n->ctx->stream;
    CK(cudaMemcpyAsync(record, n->grad, n->nparam * 4, cudaMemcpyDeviceToDevice, st), "record copy");
    CK(cudaMemcpyAsync(record + n->nparam, n->count, 4, cudaMemcpyDeviceToDevice, st), "count copy");
    CK(cudaStreamSynchronize(st), "sync");
    return PT_OK;
  });
}

pt_status pt_unet_apply_records(pt_unet *n, const float *records, uint32_t replicas, float lr) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !records || replicas == 0 || !(lr > 0.0f)) return PT_INVALID_ARG;
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    cudaSetDevice(n->ctx->device);
    n->step += 1;
    CK(launch_adam_records(n->params, n->m, n->v, records, (int)replicas, (long long)n->nparam, lr, n->step,
                           n->ctx->stream),
       "adam");
    RET(refresh_weights(n));
    CK(cudaStreamSynchronize(n->ctx->stream), "sync");
    return PT_OK;
  });
}

pt_status pt_unet_guess(pt_unet *n, const float *guidance, const float *anchor, const float *mask,
                        uint32_t width, uint32_t height, uint32_t channels, uint32_t scale, float *guess) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !guidance || !anchor || !mask || !guess || !width || !height || !channels || !scale)
      return PT_INVALID_ARG;
    if (scale > 64 || channels > 64) return PT_INVALID_ARG;
    const int W = (int)width, H = (int)height, C = (int)channels, s = (int)scale;
    const int hv = (H + s - 1) / s, wv = (W + s - 1) / s;
    const int Hc = (std::max(hv, 8) + 7) / 8 * 8, Wc = (std::max(wv, 8) + 7) / 8 * 8;
    RET(check_shape((uint32_t)C, (uint32_t)Hc, (uint32_t)Wc));
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    cudaSetDevice(n->ctx->device);
    const size_t cells = (size_t)C * Hc * Wc, need = cells * 7 * sizeof(float);
    if (need > n->gmem_bytes) {
      cudaFree(n->gmem);
      n->gmem = nullptr;
      n->gmem_bytes = 0;
      if (cudaMalloc(&n->gmem, need) != cudaSuccess) {
        cudaGetLastError();
        n->gmem = nullptr;
        return PT_OOM;
      }
      n->gmem_bytes = need;
    }
    float *cg = n->gmem, *ca = cg + cells, *cm = ca + cells, *feat = cm + cells;
    cudaStream_t st = n->ctx->stream;
    CK(launch_pool_inputs(guidance, anchor, mask, W, H, C, s, Wc, Hc, cg, ca, cm, st), "pool inputs");
    CK(launch_features(cg, ca, cm, C, Hc, Wc, feat, st), "features");
    RET(ensure_acts(n, C, Hc, Wc));
    RET(forward(n, feat));
    CK(launch_compose_guess(guidance, n->pred, W, H, C, s, Wc, Hc, guess, st), "compose guess");
    int kerr = 0;
    CK(cudaMemcpyAsync(&kerr, n->err, sizeof(int), cudaMemcpyDeviceToHost, st), "err copy");
    CK(cudaStreamSynchronize(st), "sync");
    if (kerr) {
      n->ctx->last_error = "a tensor-core pipeline wait gave up";
      return PT_TIMEOUT;
    }
    return PT_OK;
  });
}

pt_status pt_unet_save(pt_unet *n, const char *path) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !path) return PT_INVALID_ARG;
    std::vector<float> h(n->nparam * 3);
    {
      std::lock_guard<std::mutex> lock(n->ctx->mu);
      CK(cudaMemcpy(h.data(), n->params, n->nparam * 4, cudaMemcpyDeviceToHost), "save");
      CK(cudaMemcpy(h.data() + n->nparam, n->m, n->nparam * 4, cudaMemcpyDeviceToHost), "save");
      CK(cudaMemcpy(h.data() + 2 * n->nparam, n->v, n->nparam * 4, cudaMemcpyDeviceToHost), "save");
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return PT_INVALID_ARG;
    const uint64_t hdr[3] = {0x70746e6574763031ull, n->nparam, (uint64_t)n->step};
    const bool ok = std::fwrite(hdr, sizeof(hdr), 1, f) == 1 && std::fwrite(h.data(), 4, h.size(), f) == h.size();
    std::fclose(f);
    return ok ? PT_OK : PT_INTERNAL;
  });
}

pt_status pt_unet_load(pt_unet *n, const char *path) {
  return abi_guard(n ? n->ctx : nullptr, [&]() -> pt_status {
    if (!n || !path) return PT_INVALID_ARG;
    FILE *f = std::fopen(path, "rb");
    if (!f) return PT_INVALID_ARG;
    uint64_t hdr[3] = {0, 0, 0};
    std::vector<float> h(n->nparam * 3);
    const bool ok = std::fread(hdr, sizeof(hdr), 1, f) == 1 && hdr[0] == 0x70746e6574763031ull &&
                    hdr[1] == n->nparam && std::fread(h.data(), 4, h.size(), f) == h.size();
    std::fclose(f);
    if (!ok) return PT_INVALID_ARG;
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    CK(cudaMemcpy(n->params, h.data(), n->nparam * 4, cudaMemcpyHostToDevice), "load");
    CK(cudaMemcpy(n->m, h.data() + n->nparam, n->nparam * 4, cudaMemcpyHostToDevice), "load");
    CK(cudaMemcpy(n->v, h.data() + 2 * n->nparam, n->nparam * 4, cudaMemcpyHostToDevice), "load");
    n->step = (int)hdr[2];
    RET(refresh_weights(n));
    CK(cudaStreamSynchronize(n->ctx->stream), "sync");
    return PT_OK;
  });
}

}  // extern "C"
