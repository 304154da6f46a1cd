"""Seeded synthetic inputs for the Poisson workloads (no dataset is involved).

Images: a sum of 8 random 2-D sinusoids (frequency 1-16 cycles per image, random
orientation and phase, amplitude U[0.05, 0.2]) + 0.5 + N(0, 0.02^2) noise,
clamped to [0, 1]; one independent field per channel.

Masks follow paintop's mask ops: a hard ellipse samples each pixel centre
(x + 0.5, y + 0.5) against the implicit form (crates/paintop-cpu/src/ellipse.rs,
half-width 0: a centre on the boundary is covered); a polygon is rasterised with
4 x 4 subsamples per pixel at offsets ((s + 0.5)/4, (t + 0.5)/4), a half-open
(+x) crossing test and the nonzero fill rule (crates/paintop-cpu/src/mask_polygon.rs:1-50),
so coverage is k/16.

Workloads:
  clone_512      512x512 RGB, ellipse (256,256) radii 150x110, omega 1.9, tol 1e-5
  screened_2048  2048x2048 RGBA, lambda 0.01, random 12-vertex star ~30% +-2%, tol 1e-6
  batch_uneven   256 RGB instances, side log-uniform [64,1024], aspect U[0.5,2],
                 ellipse covering 20-60%, tol 1e-6
  train_256      single-channel 256x256, random ellipse or polygon, tol 1e-7
  multi_4096     4096x4096 RGB, 8 non-overlapping random polygons, each 3-10%
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

SUPERSAMPLE = 4


def sinusoid_image(rng: np.random.Generator, width: int, height: int, channels: int,
                   n_waves: int = 8, noise: float = 0.02) -> np.ndarray:
    """Interleaved f32 image (height, width, channels) in [0, 1]."""
    out = np.empty((height, width, channels), dtype=np.float32)
    y = (np.arange(height, dtype=np.float64) + 0.5) / height
    x = (np.arange(width, dtype=np.float64) + 0.5) / width
    for c in range(channels):
        acc = np.full((height, width), 0.5, dtype=np.float64)
        for _ in range(n_waves):
            f = rng.uniform(1.0, 16.0)
            th = rng.uniform(0.0, 2.0 * math.pi)
            ph = rng.uniform(0.0, 2.0 * math.pi)
            a = rng.uniform(0.05, 0.2)
            kx, ky = 2.0 * math.pi * f * math.cos(th), 2.0 * math.pi * f * math.sin(th)
            # separable evaluation: sin(kx x + ky y + ph) = sin(A)cos(B) + cos(A)sin(B)
            ax = kx * x + ph
            by = ky * y
            acc += a * (np.sin(ax)[None, :] * np.cos(by)[:, None] +
                        np.cos(ax)[None, :] * np.sin(by)[:, None])
        acc += rng.normal(0.0, noise, size=(height, width))
        out[:, :, c] = np.clip(acc, 0.0, 1.0)
    return out


def ellipse_mask(width: int, height: int, cx: float, cy: float, rx: float, ry: float,
                 angle: float = 0.0) -> np.ndarray:
    """Hard ellipse coverage (height, width): 1 where the pixel centre is inside."""
    y = np.arange(height, dtype=np.float64)[:, None] + 0.5 - cy
    x = np.arange(width, dtype=np.float64)[None, :] + 0.5 - cx
    ca, sa = math.cos(angle), math.sin(angle)
    u = x * ca + y * sa
    v = -x * sa + y * ca
    q = (u / rx) ** 2 + (v / ry) ** 2
    return (q <= 1.0).astype(np.float32)


def polygon_mask(width: int, height: int, points) -> np.ndarray:
    """Supersampled nonzero-rule polygon coverage (height, width), values k/16."""
    pts = np.asarray(points, dtype=np.float64)
    p0 = pts
    p1 = np.roll(pts, -1, axis=0)
    S = SUPERSAMPLE
    cov = np.zeros((height, width), dtype=np.int32)
    sub = (np.arange(S) + 0.5) / S
    xs = (np.arange(width)[:, None] + sub[None, :]).reshape(-1)  # all subsample x, sorted
    ymin, ymax = pts[:, 1].min(), pts[:, 1].max()
    r0 = max(0, int(math.floor(ymin)) - 1)
    r1 = min(height, int(math.ceil(ymax)) + 1)
    for row in range(r0, r1):
        for t in range(S):
            yy = row + sub[t]
            straddle = (p0[:, 1] <= yy) != (p1[:, 1] <= yy)
            if not straddle.any():
                continue
            a, b = p0[straddle], p1[straddle]
            xc = a[:, 0] + (yy - a[:, 1]) * (b[:, 0] - a[:, 0]) / (b[:, 1] - a[:, 1])
            wdir = np.where(b[:, 1] > a[:, 1], 1, -1)
            order = np.argsort(xc, kind="stable")
            xc, wdir = xc[order], wdir[order]
            # winding number of a point = sum of dirs of crossings strictly to its right
            suffix = np.concatenate([np.cumsum(wdir[::-1])[::-1], [0]])
            idx = np.searchsorted(xc, xs, side="right")
            inside = suffix[idx] != 0
            cov[row] += inside.reshape(width, S).sum(axis=1)
    return (cov.astype(np.float32) / float(S * S))


def star_polygon(cx, cy, r_out, r_in, n_vertices=12, rot=0.0):
    pts = []
    for k in range(n_vertices):
        r = r_out if k % 2 == 0 else r_in
        a = rot + 2.0 * math.pi * k / n_vertices
        pts.append((cx + r * math.cos(a), cy + r * math.sin(a)))
    return pts


def random_blob_polygon(rng, cx, cy, mean_r, n_vertices, jitter=0.25, stretch=(1.0, 1.0)):
    angles = np.sort(rng.uniform(0, 2 * math.pi, n_vertices))
    radii = mean_r * (1.0 + rng.uniform(-jitter, jitter, n_vertices))
    return [(cx + stretch[0] * r * math.cos(a), cy + stretch[1] * r * math.sin(a))
            for r, a in zip(radii, angles)]


def polygon_area(points) -> float:
    p = np.asarray(points, dtype=np.float64)
    x, y = p[:, 0], p[:, 1]
    return 0.5 * abs(np.dot(x, np.roll(y, -1)) - np.dot(y, np.roll(x, -1)))


@dataclass
class Instance:
    width: int
    height: int
    channels: int
    source: np.ndarray   # (h, w, c) f32
    target: np.ndarray   # (h, w, c) f32
    mask: np.ndarray     # (h, w) f32
    lam: float = 0.0
    tolerance: float = 1e-6
    max_iterations: int = 2000
    omega: float = 1.8
    polygons: list = None  # the polygons (vertex lists) the mask was drawn from

    def problem(self, **over) -> dict:
        d = dict(source=self.source, target=self.target, mask=self.mask, width=self.width,
                 height=self.height, channels=self.channels, lam=self.lam,
                 tolerance=self.tolerance, max_iterations=self.max_iterations, omega=self.omega)
        d.update(over)
        return d


def clone_512(seed: int = 1) -> Instance:
    rng = np.random.default_rng(seed)
    w = h = 512
    src = sinusoid_image(rng, w, h, 3)
    tgt = sinusoid_image(rng, w, h, 3)
    mask = ellipse_mask(w, h, 256, 256, 150, 110)
    return Instance(w, h, 3, src, tgt, mask, 0.0, 1e-5, 5000, 1.9)


def screened_2048(seed: int = 1, size: int = 2048) -> Instance:
    rng = np.random.default_rng(seed)
    w = h = size
    src = sinusoid_image(rng, w, h, 4)
    tgt = sinusoid_image(rng, w, h, 4)
    ratio = rng.uniform(0.5, 0.8)
    # a 12-vertex star with alternating radii has area 3 * r_out * r_in
    area = 0.30 * w * h
    r_out = math.sqrt(area / (3.0 * ratio))
    pts = star_polygon(w / 2, h / 2, r_out, ratio * r_out, 12, rng.uniform(0, math.pi / 6))
    mask = polygon_mask(w, h, pts)
    return Instance(w, h, 4, src, tgt, mask, 0.01, 1e-6, 2000, 1.8, [pts])


def uneven_instance(rng: np.random.Generator, tol: float = 1e-6) -> Instance:
    s = math.exp(rng.uniform(math.log(64), math.log(1024)))
    a = rng.uniform(0.5, 2.0)
    w = max(8, int(round(s * math.sqrt(a))))
    h = max(8, int(round(s / math.sqrt(a))))
    frac = rng.uniform(0.2, 0.6)
    k = math.sqrt(4.0 * frac / math.pi)
    rx, ry = 0.5 * w * k, 0.5 * h * k
    cx = w / 2 + rng.uniform(-1, 1) * max(0.0, w / 2 - rx - 1)
    cy = h / 2 + rng.uniform(-1, 1) * max(0.0, h / 2 - ry - 1)
    src = sinusoid_image(rng, w, h, 3)
    tgt = sinusoid_image(rng, w, h, 3)
    mask = ellipse_mask(w, h, cx, cy, rx, ry)
    return Instance(w, h, 3, src, tgt, mask, 0.0, tol, 100000, 1.8)


def batch_uneven(seed: int = 1, n: int = 256) -> list:
    rng = np.random.default_rng(seed)
    return [uneven_instance(rng) for _ in range(n)]


def train_instance(rng: np.random.Generator, size: int = 256) -> Instance:
    w = h = size
    src = sinusoid_image(rng, w, h, 1)
    tgt = sinusoid_image(rng, w, h, 1)
    if rng.uniform() < 0.5:
        rx, ry = rng.uniform(0.15, 0.4) * w, rng.uniform(0.15, 0.4) * h
        mask = ellipse_mask(w, h, w / 2 + rng.uniform(-0.08, 0.08) * w,
                            h / 2 + rng.uniform(-0.08, 0.08) * h, rx, ry,
                            rng.uniform(0, math.pi))
    else:
        pts = random_blob_polygon(rng, w / 2, h / 2, rng.uniform(0.2, 0.38) * w,
                                  int(rng.integers(5, 13)))
        mask = polygon_mask(w, h, pts)
    return Instance(w, h, 1, src, tgt, mask, 0.0, 1e-7, 100000, 1.8)


def multi_4096(seed: int = 1, size: int = 4096) -> Instance:
    rng = np.random.default_rng(seed)
    w = h = size
    src = sinusoid_image(rng, w, h, 3)
    tgt = sinusoid_image(rng, w, h, 3)
    mask = np.zeros((h, w), dtype=np.float32)
    polys = []
    cw, ch = w // 4, h // 2           # 8 cells, one polygon each: never overlapping
    for k in range(8):
        gx, gy = k % 4, k // 4
        cx, cy = (gx + 0.5) * cw, (gy + 0.5) * ch
        target_area = rng.uniform(0.03, 0.10) * w * h
        pts = random_blob_polygon(rng, cx, cy, 1.0, int(rng.integers(7, 14)), 0.2, (1.0, 1.6))
        scale = math.sqrt(target_area / polygon_area(pts))
        pts = [(cx + (px - cx) * scale, cy + (py - cy) * scale) for px, py in pts]
        # keep inside the cell with a margin
        xs, ys = [p[0] for p in pts], [p[1] for p in pts]
        fx = (0.5 * cw - 2) / max(max(xs) - cx, cx - min(xs))
        fy = (0.5 * ch - 2) / max(max(ys) - cy, cy - min(ys))
        f = min(1.0, fx, fy)
        pts = [(cx + (px - cx) * f, cy + (py - cy) * f) for px, py in pts]
        polys.append(pts)
        mask = np.maximum(mask, polygon_mask(w, h, pts))
    return Instance(w, h, 3, src, tgt, mask, 0.0, 1e-6, 100000, 1.8, polys)
