"""CPU oracle of the learned warm start's network (test infrastructure only).

The reference has no learned component, so this file is not a restatement of
reference code: it is the float64 numpy statement of the network that the CUDA
kernels in ``paintop_b200/csrc/unet`` implement, used by the tests to check the
GPU forward pass, loss and parameter gradients. The backward pass here is
itself pinned by central finite differences (``tests/test_unet_oracle.py``).

With ``emulate_bf16=True`` every value the GPU stores in bf16 (activations,
activation gradients, the convolution weights) is rounded to bf16
(round-to-nearest-even) at the same points, so the GPU and this oracle differ
only by fp32-vs-fp64 accumulation order. With ``emulate_bf16=False`` it is the
exact float64 network, the one finite differences check.

Layout (matches ``pt_unet_get_params``): for each of the 14 3x3 layers
W[cout][9][cin] (tap = 3 * (dy + 1) + (dx + 1)) then b[cout]; then the 1x1
head's w[16] and b[1]. Tensors are NHWC.
"""
from __future__ import annotations

import numpy as np

LAYERS = [(16, 16), (16, 16), (32, 16), (32, 32), (64, 32), (64, 64), (128, 64), (128, 128),
          (64, 192), (64, 64), (32, 96), (32, 32), (16, 48), (16, 16)]  # (cout, cin)
IN_REAL = 4
HEAD_IN = 16


def param_layout():
    """[(w_off, b_off, cout, cin)] for the 3x3 layers, head_w offset, total count."""
    out, off = [], 0
    for co, ci in LAYERS:
        w = off
        off += co * 9 * ci
        out.append((w, off, co, ci))
        off += co
    head_w = off
    off += HEAD_IN + 1
    return out, head_w, off


def bf16(x):
    """Round to the nearest bf16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def split_params(params):
    layout, head_w, n = param_layout()
    params = np.asarray(params, dtype=np.float64)
    assert params.size == n
    Ws = [params[w:b].reshape(co, 9, ci) for (w, b, co, ci) in layout]
    bs = [params[b:b + co] for (w, b, co, ci) in layout]
    return Ws, bs, params[head_w:head_w + HEAD_IN], params[head_w + HEAD_IN]


def _shift(x, dy, dx):
    """out[b, y, x] = x[b, y + dy, x + dx] (zero outside)."""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C), dtype=x.dtype)
    xp[:, 1:H + 1, 1:W + 1] = x
    return xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]


def conv3x3(x, W):
    """y[p][co] = sum_tap x[p + off(tap)] . W[co][tap] (no bias)."""
    y = 0.0
    for t in range(9):
        y = y + _shift(x, t // 3 - 1, t % 3 - 1) @ W[:, t, :].T
    return y


def conv3x3_dgrad(dy, W):
    """dx[q] = sum_tap dy[q - off(tap)] . W[:, tap, :]."""
    dx = 0.0
    for t in range(9):
        dx = dx + _shift(dy, -(t // 3 - 1), -(t % 3 - 1)) @ W[:, t, :]
    return dx


def conv3x3_wgrad(dy, x):
    B, H, Wd, co = dy.shape
    ci = x.shape[-1]
    g = np.zeros((co, 9, ci))
    d2 = dy.reshape(-1, co)
    for t in range(9):
        g[:, t, :] = d2.T @ _shift(x, t // 3 - 1, t % 3 - 1).reshape(-1, ci)
    return g


def pool(x):
    B, H, W, C = x.shape
    return 0.25 * x.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def unpool(d):
    return 0.25 * np.repeat(np.repeat(d, 2, axis=1), 2, axis=2)


def _up_matrix(n):
    """Bilinear x2 with half-pixel centres, clamped: out[2i] = .75 in[i] + .25 in[i-1],
    out[2i+1] = .75 in[i] + .25 in[i+1]."""
    U = np.zeros((2 * n, n))
    for i in range(n):
        U[2 * i, i] += 0.75
        U[2 * i, max(i - 1, 0)] += 0.25
        U[2 * i + 1, i] += 0.75
        U[2 * i + 1, min(i + 1, n - 1)] += 0.25
    return U


def upsample(x):
    B, H, W, C = x.shape
    return np.einsum("yi,xj,bijc->byxc", _up_matrix(H), _up_matrix(W), x, optimize=True)


def upsample_adj(d):
    B, H2, W2, C = d.shape
    return np.einsum("yi,xj,byxc->bijc", _up_matrix(H2 // 2), _up_matrix(W2 // 2), d, optimize=True)


class Net:
    """Forward and backward of the network for one batch."""

    def __init__(self, params, emulate_bf16=True):
        self.q = bf16 if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
        self.Ws, self.bs, self.hw, self.hb = split_params(params)
        self.Wq = [self.q(W) for W in self.Ws]

    def _conv(self, l, x):
        return self.q(np.maximum(conv3x3(x, self.Wq[l]) + self.bs[l], 0.0))

    def forward(self, features):
        q = self.q
        B, H, W, _ = features.shape
        x0 = np.zeros((B, H, W, 16))
        x0[..., :IN_REAL] = q(features)
        a = {"x0": x0}
        a["e0a"] = self._conv(0, x0)
        a["e0"] = self._conv(1, a["e0a"])
        a["p1"] = q(pool(a["e0"]))
        a["e1a"] = self._conv(2, a["p1"])
        a["e1"] = self._conv(3, a["e1a"])
        a["p2"] = q(pool(a["e1"]))
        a["e2a"] = self._conv(4, a["p2"])
        a["e2"] = self._conv(5, a["e2a"])
        a["p3"] = q(pool(a["e2"]))
        a["e3a"] = self._conv(6, a["p3"])
        a["e3"] = self._conv(7, a["e3a"])
        a["cat2"] = np.concatenate([q(upsample(a["e3"])), a["e2"]], axis=-1)
        a["d2a"] = self._conv(8, a["cat2"])
        a["d2"] = self._conv(9, a["d2a"])
        a["cat1"] = np.concatenate([q(upsample(a["d2"])), a["e1"]], axis=-1)
        a["d1a"] = self._conv(10, a["cat1"])
        a["d1"] = self._conv(11, a["d1a"])
        a["cat0"] = np.concatenate([q(upsample(a["d1"])), a["e0"]], axis=-1)
        a["d0a"] = self._conv(12, a["cat0"])
        a["d0"] = self._conv(13, a["d0a"])
        a["pred"] = a["d0"] @ self.hw + self.hb
        self.a = a
        return a["pred"]

    def loss_grad(self, features, target, loss_mask):
        """Masked mean squared error and the flat gradient (float64)."""
        q = self.q
        pred = self.forward(features)
        a = self.a
        m = (np.asarray(loss_mask) > 0.5).astype(np.float64)
        n = max(1.0, m.sum())
        d = (pred - target) * m
        loss = float((d * d).sum() / n)
        dpred = 2.0 * d / n
        layout, head_w, total = param_layout()
        g = np.zeros(total)
        g[head_w:head_w + HEAD_IN] = (a["d0"] * dpred[..., None]).reshape(-1, HEAD_IN).sum(0)
        g[head_w + HEAD_IN] = dpred.sum()

        def grads(l, dy, x):
            w, b, co, ci = layout[l]
            g[w:b] = conv3x3_wgrad(dy, x).reshape(-1)
            g[b:b + co] = dy.reshape(-1, co).sum(0)

        relu = lambda v: (v > 0).astype(np.float64)
        dd0 = q(dpred[..., None] * self.hw * relu(a["d0"]))
        grads(13, dd0, a["d0a"])
        dd0a = q(conv3x3_dgrad(dd0, self.Wq[13]) * relu(a["d0a"]))
        grads(12, dd0a, a["cat0"])
        dcat0 = q(conv3x3_dgrad(dd0a, self.Wq[12]))
        dd1 = q(upsample_adj(dcat0[..., :32]) * relu(a["d1"]))
        grads(11, dd1, a["d1a"])
        dd1a = q(conv3x3_dgrad(dd1, self.Wq[11]) * relu(a["d1a"]))
        grads(10, dd1a, a["cat1"])
        dcat1 = q(conv3x3_dgrad(dd1a, self.Wq[10]))
        dd2 = q(upsample_adj(dcat1[..., :64]) * relu(a["d2"]))
        grads(9, dd2, a["d2a"])
        dd2a = q(conv3x3_dgrad(dd2, self.Wq[9]) * relu(a["d2a"]))
        grads(8, dd2a, a["cat2"])
        dcat2 = q(conv3x3_dgrad(dd2a, self.Wq[8]))
        de3 = q(upsample_adj(dcat2[..., :128]) * relu(a["e3"]))
        grads(7, de3, a["e3a"])
        de3a = q(conv3x3_dgrad(de3, self.Wq[7]) * relu(a["e3a"]))
        grads(6, de3a, a["p3"])
        dp3 = q(conv3x3_dgrad(de3a, self.Wq[6]))
        de2 = q((dcat2[..., 128:] + unpool(dp3)) * relu(a["e2"]))
        grads(5, de2, a["e2a"])
        de2a = q(conv3x3_dgrad(de2, self.Wq[5]) * relu(a["e2a"]))
        grads(4, de2a, a["p2"])
        dp2 = q(conv3x3_dgrad(de2a, self.Wq[4]))
        de1 = q((dcat1[..., 64:] + unpool(dp2)) * relu(a["e1"]))
        grads(3, de1, a["e1a"])
        de1a = q(conv3x3_dgrad(de1, self.Wq[3]) * relu(a["e1a"]))
        grads(2, de1a, a["p1"])
        dp1 = q(conv3x3_dgrad(de1a, self.Wq[2]))
        de0 = q((dcat0[..., 32:] + unpool(dp1)) * relu(a["e0"]))
        grads(1, de0, a["e0a"])
        de0a = q(conv3x3_dgrad(de0, self.Wq[1]) * relu(a["e0a"]))
        grads(0, de0a, a["x0"])
        return loss, g


def init_params(seed: int) -> np.ndarray:
    """A He-normal parameter vector for oracle-only tests (not the library's stream)."""
    rng = np.random.default_rng(seed)
    layout, head_w, total = param_layout()
    p = np.zeros(total)
    for l, (w, b, co, ci) in enumerate(layout):
        ci_real = IN_REAL if l == 0 else ci
        W = rng.normal(0.0, np.sqrt(2.0 / (9 * ci_real)), (co, 9, ci))
        W[:, :, ci_real:] = 0.0
        p[w:b] = W.reshape(-1)
        p[b:b + co] = rng.normal(0.0, 0.05, co)
    p[head_w:head_w + HEAD_IN] = rng.normal(0.0, 0.25, HEAD_IN)
    p[head_w + HEAD_IN] = 0.1
    return p


def features(guidance, anchor, mask):
    """The four input features of single-channel images (B, H, W) -> (B, H, W, 4),
    float32 arithmetic in the GPU's order: 0 the guidance Laplacian at interior
    cells, 1 anchor - guidance outside the interior (the boundary values of the
    correction u - g that the network predicts), 2 the interior mask, 3 the
    distance to the nearest non-interior cell along the row or column / 32,
    clipped at 1."""
    g = np.asarray(guidance, dtype=np.float32)
    an = np.asarray(anchor, dtype=np.float32)
    B, H, W = g.shape
    inter = np.asarray(mask, dtype=np.float32) > 0.5
    inter[:, 0, :] = inter[:, -1, :] = False
    inter[:, :, 0] = inter[:, :, -1] = False
    if H < 3 or W < 3:
        inter[:] = False
    f = np.zeros((B, H, W, 4), dtype=np.float32)
    lap = np.zeros_like(g)
    lap[:, 1:-1, 1:-1] = (((g[:, 1:-1, :-2] + g[:, 1:-1, 2:]) + g[:, :-2, 1:-1]) + g[:, 2:, 1:-1]) \
        - np.float32(4.0) * g[:, 1:-1, 1:-1]
    f[..., 0] = np.where(inter, lap, 0.0)
    f[..., 1] = np.where(inter, np.float32(0.0), an - g)
    f[..., 2] = inter
    pad = np.zeros((B, H + 64, W + 64), dtype=bool)
    pad[:, 32:32 + H, 32:32 + W] = inter
    dist = np.full((B, H, W), 32, dtype=np.int32)
    for d in range(31, 0, -1):
        hit = ~(pad[:, 32:32 + H, 32 - d:32 - d + W] & pad[:, 32:32 + H, 32 + d:32 + d + W]
                & pad[:, 32 - d:32 - d + H, 32:32 + W] & pad[:, 32 + d:32 + d + H, 32:32 + W])
        dist = np.where(hit, d, dist)
    f[..., 3] = np.where(inter, dist.astype(np.float32) / np.float32(32.0), 0.0)
    return f
