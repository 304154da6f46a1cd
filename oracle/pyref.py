"""Pure-Python restatement of paintop's Poisson solver -- TEST INFRASTRUCTURE ONLY.

An independent second restatement of crates/paintop-cpu/src/poisson.rs:167-373
and poisson_blend.rs:153-246, written with plain Python floats (IEEE-754
binary64, round to nearest even) and an exactly-rounded fused multiply-add
built from rational arithmetic (``Fraction`` -> ``float`` is correctly
rounded). It exists to pin the C oracle bit for bit on small grids; it is far
too slow for anything else.
"""
from __future__ import annotations

import math
from fractions import Fraction

CENTRE_WEIGHT = 4.0          # poisson.rs:73
STALL_WINDOW = 16            # poisson.rs:80
STALL_IMPROVEMENT = 1e-12    # poisson.rs:85
MASK_THRESHOLD = 0.5         # poisson.rs:329


def fma(a: float, b: float, c: float) -> float:
    """Correctly rounded a*b+c (Rust ``f64::mul_add``) for finite operands."""
    if not (math.isfinite(a) and math.isfinite(b) and math.isfinite(c)):
        return a * b + c
    exact = Fraction(a) * Fraction(b) + Fraction(c)
    if exact == 0:
        # IEEE sign of an exact zero sum under round-to-nearest
        p = a * b
        if p == 0 and c == 0:
            return p + c
        return 0.0
    return float(exact)


def f32(x: float) -> float:
    """Round a binary64 value to binary32 (nearest even), returned as a float."""
    import struct
    return struct.unpack("<f", struct.pack("<f", x))[0]


def neighbour_sum(field, col, row, width, height):
    """poisson.rs:275-298."""
    centre = field[row * width + col]
    left = centre if col == 0 else field[row * width + col - 1]
    right = centre if col + 1 == width else field[row * width + col + 1]
    up = centre if row == 0 else field[(row - 1) * width + col]
    down = centre if row + 1 == height else field[(row + 1) * width + col]
    return left + right + up + down


def classify_cells(mask, width, height):
    """poisson.rs:340-355 (1 = Interior, 0 = Boundary)."""
    cells = [0] * (width * height)
    if width < 3 or height < 3:
        return cells
    for row in range(1, height - 1):
        for col in range(1, width - 1):
            idx = row * width + col
            if f32(mask[idx]) > MASK_THRESHOLD:
                cells[idx] = 1
    return cells


def guidance_laplacian(field, col, row, width, height):
    """poisson.rs:364-373."""
    centre = field[row * width + col]
    return fma(CENTRE_WEIGHT, -centre, neighbour_sum(field, col, row, width, height))


def _sweep_once(width, height, cells, rhs, anchor, lam, field, denom, omega):
    """poisson.rs:244-265."""
    for row in range(height):
        for col in range(width):
            idx = row * width + col
            if cells[idx] != 1:
                continue
            nsum = neighbour_sum(field, col, row, width, height)
            target = fma(lam, anchor[idx], nsum - rhs[idx]) / denom
            field[idx] = fma(omega, target - field[idx], field[idx])


def _residual_l2(width, height, cells, rhs, anchor, lam, field):
    """poisson.rs:305-325."""
    s = 0.0
    for row in range(height):
        for col in range(width):
            idx = row * width + col
            if cells[idx] != 1:
                continue
            nsum = neighbour_sum(field, col, row, width, height)
            lhs = fma(lam + CENTRE_WEIGHT, -field[idx], nsum)
            rr = fma(lam, -anchor[idx], rhs[idx])
            r = lhs - rr
            s = fma(r, r, s)
    return math.sqrt(s)


def solve(width, height, cells, rhs, anchor, lam, max_iterations, tolerance, omega):
    """poisson.rs:167-240 -> (field, dict report)."""
    field = list(anchor)
    r0 = _residual_l2(width, height, cells, rhs, anchor, lam, field)
    if r0 == 0.0:
        return field, dict(iterations=0, converged=True, stop_reason="converged",
                           tolerance=tolerance, final_residual=0.0, residual_history=[])
    denom = CENTRE_WEIGHT + lam
    hist = []
    converged = False
    stop = "max-iterations"
    last = 1.0
    iterations = 0
    best = math.inf
    since = 0
    for sweep in range(max_iterations):
        _sweep_once(width, height, cells, rhs, anchor, lam, field, denom, omega)
        iterations = sweep + 1
        rel = _residual_l2(width, height, cells, rhs, anchor, lam, field) / r0
        hist.append(rel)
        last = rel
        if rel <= tolerance:
            converged = True
            stop = "converged"
            break
        if rel < best * (1.0 - STALL_IMPROVEMENT):
            best = rel
            since = 0
        else:
            since += 1
            if since >= STALL_WINDOW:
                stop = "stalled"
                break
    return field, dict(iterations=iterations, converged=converged, stop_reason=stop,
                       tolerance=tolerance, final_residual=last, residual_history=hist)


def blend_channels(source, target, mask, channels, width, height, max_iterations, tolerance,
                   lam, omega):
    """poisson_blend.rs:168-246 -> (out f32 list, worst report dict)."""
    count = width * height
    cells = classify_cells(mask, width, height)
    out = [0.0] * (count * channels)
    worst = None
    for ch in range(channels):
        src = [float(f32(source[p * channels + ch])) for p in range(count)]
        anchor = [float(f32(target[p * channels + ch])) for p in range(count)]
        rhs = [0.0] * count
        for row in range(height):
            for col in range(width):
                idx = row * width + col
                if cells[idx] == 1:
                    rhs[idx] = guidance_laplacian(src, col, row, width, height)
        field, rep = solve(width, height, cells, rhs, anchor, lam, max_iterations, tolerance,
                           omega)
        for p in range(count):
            out[p * channels + ch] = f32(field[p])
        if worst is None or (rep["iterations"], rep["final_residual"]) > (
                worst["iterations"], worst["final_residual"]):
            worst = rep
    if worst is None:
        worst = dict(iterations=0, converged=True, stop_reason="converged", tolerance=tolerance,
                     final_residual=0.0, residual_history=[])
    return out, worst
