"""Generate tests/golden/poisson_cases.npz from the pinned oracle.

The reference publishes no golden arrays for this path, so the fixtures are the
outputs of the C restatement of crates/paintop-cpu/src/poisson.rs (oracle/),
which is itself pinned bit for bit to an independent pure-Python restatement
and to the reference's analytic tests. Each case stores its seeded inputs, the
controls and the oracle's interleaved f32 output, per-channel reports and
histories. Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

# name, width, height, channels, lambda, omega, max_iterations, tolerance, mask kind
CASES = [
    ("square_rgb", 16, 12, 3, 0.0, 1.8, 2000, 1e-6, "square"),
    ("ellipse_gray", 24, 24, 1, 0.0, 1.9, 5000, 1e-10, "ellipse"),
    ("screened_rgba", 33, 17, 4, 0.5, 1.8, 300, 1e-8, "random"),
    ("capped", 20, 20, 2, 0.0, 1.0, 7, 1e-30, "square"),
    ("thin_strip", 2, 9, 1, 0.0, 1.8, 50, 1e-6, "full"),
    ("empty_mask", 10, 8, 3, 0.0, 1.8, 50, 1e-6, "empty"),
    ("border_touching", 15, 11, 2, 0.2, 1.7, 500, 1e-9, "full"),
]


def make_mask(kind, w, h, rng):
    yy, xx = np.mgrid[0:h, 0:w]
    if kind == "square":
        m = ((xx >= w // 4) & (xx < w - w // 4) & (yy >= h // 4) & (yy < h - h // 4))
    elif kind == "ellipse":
        m = ((xx + 0.5 - w / 2) / (0.35 * w)) ** 2 + ((yy + 0.5 - h / 2) / (0.3 * h)) ** 2 <= 1
    elif kind == "random":
        m = rng.random((h, w)) < 0.7
    elif kind == "full":
        m = np.ones((h, w), bool)
    else:
        m = np.zeros((h, w), bool)
    return m.astype(np.float32).reshape(-1)


def build():
    arrays = {}
    for k, (name, w, h, c, lam, omega, max_it, tol, kind) in enumerate(CASES):
        rng = np.random.default_rng(1000 + k)
        src = rng.random(w * h * c).astype(np.float32)
        tgt = rng.random(w * h * c).astype(np.float32)
        mask = make_mask(kind, w, h, rng)
        out, worst, per = O.blend_channels(src, tgt, mask, c, w, h, max_it, tol, lam, omega)
        arrays[f"{name}/source"] = src
        arrays[f"{name}/target"] = tgt
        arrays[f"{name}/mask"] = mask
        arrays[f"{name}/controls"] = np.array([w, h, c, lam, omega, max_it, tol], np.float64)
        arrays[f"{name}/out"] = out
        arrays[f"{name}/iterations"] = np.array([p.iterations for p in per], np.int64)
        arrays[f"{name}/stop"] = np.array([("converged", "max-iterations", "stalled").index(
            p.stop_reason) for p in per], np.int64)
        arrays[f"{name}/final_residual"] = np.array([p.final_residual for p in per], np.float64)
        hist = np.full((c, max(max_it, 1)), np.nan)
        for i, p in enumerate(per):
            hist[i, :len(p.residual_history)] = p.residual_history
        arrays[f"{name}/history"] = hist
    return arrays


if __name__ == "__main__":
    O.build()
    a = build()
    np.savez_compressed(os.path.join(HERE, "poisson_cases.npz"), **a)
    print(f"wrote {len(CASES)} cases")
