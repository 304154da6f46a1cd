"""ctypes wrapper over the C oracle -- TEST INFRASTRUCTURE ONLY.

Wraps ``oracle/_build/libpaintop_oracle.so`` (built by ``oracle/Makefile``):

* :func:`solve` -- ``poisson::solve`` (crates/paintop-cpu/src/poisson.rs:167-240)
  on an assembled system (cells, rhs, anchor, lambda) with explicit controls.
* :func:`blend_channels` -- ``blend_channels`` + ``worse_of``
  (crates/paintop-cpu/src/poisson_blend.rs:168-246) on interleaved f32 images.
* :func:`cg_blend_channels` -- the FP64 CG tight oracle on the same system.
* :func:`rb_blend_channels` -- FP64 red-black SOR: the GPU method in FP64.
* :func:`mask_ellipse`, :func:`mask_polygon` -- the ``mask.ellipse@1`` and
  ``mask.polygon@1`` generators (``oracle/mask_ref.c``).

The C restatement is checked bit-for-bit against the pure-Python restatement in
``oracle/pyref.py`` and against the reference's analytic known-answer tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libpaintop_oracle.so")

PR_BOUNDARY, PR_INTERIOR = 0, 1
STOP_REASONS = ("converged", "max-iterations", "stalled")


class _System(C.Structure):
    _fields_ = [
        ("width", C.c_size_t),
        ("height", C.c_size_t),
        ("cells", C.POINTER(C.c_uint8)),
        ("rhs", C.POINTER(C.c_double)),
        ("anchor", C.POINTER(C.c_double)),
        ("lambda_", C.c_double),
    ]


class _Controls(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_uint32),
        ("tolerance", C.c_double),
        ("omega", C.c_double),
    ]


class _Report(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32),
        ("converged", C.c_int32),
        ("stop_reason", C.c_int32),
        ("tolerance", C.c_double),
        ("final_residual", C.c_double),
    ]


@dataclass
class SolveReport:
    """Mirror of ``SolveReport`` (crates/paintop-cpu/src/poisson.rs:126-141)."""

    iterations: int
    converged: bool
    stop_reason: str
    tolerance: float
    final_residual: float
    residual_history: list = field(default_factory=list)


_lib = None


def build() -> None:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.exists(os.path.join(_HERE, "Makefile")):
            build()  # a no-op when the library is newer than every source
        L = C.CDLL(_LIB_PATH)
        L.pr_classify_cells.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p]
        L.pr_classify_cells.restype = None
        L.pr_solve.argtypes = [C.POINTER(_System), _Controls, C.c_void_p, C.c_void_p,
                               C.POINTER(_Report)]
        L.pr_solve.restype = None
        L.pr_residual_l2.argtypes = [C.POINTER(_System), C.c_void_p]
        L.pr_residual_l2.restype = C.c_double
        L.pr_blend_channels.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.c_size_t, C.c_size_t, _Controls, C.c_double,
                                        C.c_void_p, C.POINTER(_Report), C.c_void_p,
                                        C.POINTER(C.c_int)]
        L.pr_blend_channels.restype = C.c_int
        L.pr_cg_solve.argtypes = [C.POINTER(_System), C.c_double, C.c_uint32, C.c_void_p,
                                  C.POINTER(C.c_double)]
        L.pr_cg_solve.restype = C.c_int
        L.pr_cg_blend_channels.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                           C.c_size_t, C.c_size_t, C.c_double, C.c_double,
                                           C.c_uint32, C.c_void_p, C.c_void_p]
        L.pr_cg_blend_channels.restype = C.c_int
        L.pr_mgcg_blend_channels.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                             C.c_size_t, C.c_size_t, C.c_double, C.c_double,
                                             C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.pr_mgcg_blend_channels.restype = C.c_int
        L.pr_rb_blend_channels.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                           C.c_size_t, C.c_size_t, _Controls, C.c_double,
                                           C.c_void_p, C.POINTER(_Report), C.c_void_p]
        L.pr_rb_blend_channels.restype = C.c_int
        L.or_mask_ellipse.argtypes = [C.c_uint32, C.c_uint32] + [C.c_double] * 6 + [C.c_void_p]
        L.or_mask_ellipse.restype = None
        L.or_mask_polygon.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]
        L.or_mask_polygon.restype = None
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def classify_cells(mask: np.ndarray, width: int, height: int) -> np.ndarray:
    mask = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1)
    cells = np.zeros(width * height, dtype=np.uint8)
    lib().pr_classify_cells(_p(mask), width, height, _p(cells))
    return cells


def _system(width, height, cells, rhs, anchor, lam):
    cells = np.ascontiguousarray(cells, dtype=np.uint8).reshape(-1)
    rhs = np.ascontiguousarray(rhs, dtype=np.float64).reshape(-1)
    anchor = np.ascontiguousarray(anchor, dtype=np.float64).reshape(-1)
    s = _System(width, height, cells.ctypes.data_as(C.POINTER(C.c_uint8)),
                rhs.ctypes.data_as(C.POINTER(C.c_double)),
                anchor.ctypes.data_as(C.POINTER(C.c_double)), float(lam))
    return s, (cells, rhs, anchor)


def solve(width, height, cells, rhs, anchor, lam, max_iterations, tolerance, omega):
    """``poisson::solve`` -> (field f64 [h*w], SolveReport)."""
    s, keep = _system(width, height, cells, rhs, anchor, lam)
    field_ = np.empty(width * height, dtype=np.float64)
    hist = np.zeros(max(int(max_iterations), 1), dtype=np.float64)
    rep = _Report()
    lib().pr_solve(C.byref(s), _Controls(int(max_iterations), float(tolerance), float(omega)),
                   _p(field_), _p(hist), C.byref(rep))
    del keep
    return field_, SolveReport(rep.iterations, bool(rep.converged), STOP_REASONS[rep.stop_reason],
                               rep.tolerance, rep.final_residual,
                               hist[: rep.iterations].tolist())


def residual_l2(width, height, cells, rhs, anchor, lam, field_):
    s, keep = _system(width, height, cells, rhs, anchor, lam)
    f = np.ascontiguousarray(field_, dtype=np.float64).reshape(-1)
    r = lib().pr_residual_l2(C.byref(s), _p(f))
    del keep
    return r


def blend_channels(source, target, mask, channels, width, height, max_iterations=2000,
                   tolerance=1e-6, lam=0.0, omega=1.8):
    """``blend_channels`` -> (out f32 interleaved, worst SolveReport, per-channel reports)."""
    source = np.ascontiguousarray(source, dtype=np.float32).reshape(-1)
    target = np.ascontiguousarray(target, dtype=np.float32).reshape(-1)
    mask = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1)
    n = width * height
    assert source.size == n * channels and target.size == n * channels and mask.size == n
    out = np.empty(n * channels, dtype=np.float32)
    reps = (_Report * max(channels, 1))()
    hist = np.zeros(max(channels, 1) * max(int(max_iterations), 1), dtype=np.float64)
    worst = C.c_int(-1)
    rc = lib().pr_blend_channels(_p(source), _p(target), _p(mask), channels, width, height,
                                 _Controls(int(max_iterations), float(tolerance), float(omega)),
                                 float(lam), _p(out), reps, _p(hist), C.byref(worst))
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    per = []
    for c in range(channels):
        r = reps[c]
        h = hist[c * max_iterations: c * max_iterations + r.iterations].tolist()
        per.append(SolveReport(r.iterations, bool(r.converged), STOP_REASONS[r.stop_reason],
                               r.tolerance, r.final_residual, h))
    if channels == 0:
        worst_rep = SolveReport(0, True, "converged", float(tolerance), 0.0, [])
    else:
        worst_rep = per[worst.value]
    return out, worst_rep, per


def rb_blend_channels(source, target, mask, channels, width, height, max_iterations=2000,
                      tolerance=1e-6, lam=0.0, omega=1.8):
    """FP64 red-black SOR (the GPU method in FP64) -> (field f64 interleaved, per-channel reports)."""
    source = np.ascontiguousarray(source, dtype=np.float32).reshape(-1)
    target = np.ascontiguousarray(target, dtype=np.float32).reshape(-1)
    mask = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1)
    n = width * height
    out = np.empty(n * channels, dtype=np.float64)
    reps = (_Report * max(channels, 1))()
    hist = np.zeros(max(channels, 1) * max(int(max_iterations), 1), dtype=np.float64)
    rc = lib().pr_rb_blend_channels(_p(source), _p(target), _p(mask), channels, width, height,
                                    _Controls(int(max_iterations), float(tolerance), float(omega)),
                                    float(lam), _p(out), reps, _p(hist))
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    per = []
    for c in range(channels):
        r = reps[c]
        h = hist[c * max_iterations: c * max_iterations + r.iterations].tolist()
        per.append(SolveReport(r.iterations, bool(r.converged), STOP_REASONS[r.stop_reason],
                               r.tolerance, r.final_residual, h))
    return out, per


def cg_blend_channels(source, target, mask, channels, width, height, lam=0.0, rel_tol=1e-12,
                      max_iterations=200000):
    """FP64 CG tight oracle -> (field f64 interleaved, achieved rel-res per channel)."""
    source = np.ascontiguousarray(source, dtype=np.float32).reshape(-1)
    target = np.ascontiguousarray(target, dtype=np.float32).reshape(-1)
    mask = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1)
    n = width * height
    out = np.empty(n * channels, dtype=np.float64)
    ach = np.zeros(max(channels, 1), dtype=np.float64)
    it = lib().pr_cg_blend_channels(_p(source), _p(target), _p(mask), channels, width, height,
                                    float(lam), float(rel_tol), int(max_iterations), _p(out),
                                    _p(ach))
    if it < 0:
        raise MemoryError("oracle allocation failed")
    return out, ach[:channels]


def mgcg_blend_channels(source, target, mask, channels, width, height, lam=0.0, rel_tol=1e-12,
                        max_iterations=2000):
    """FP64 multigrid-preconditioned CG tight oracle for large systems (mgcg_ref.c)
    -> (field f64 interleaved, achieved rel-res per channel, iterations per channel)."""
    source = np.ascontiguousarray(source, dtype=np.float32).reshape(-1)
    target = np.ascontiguousarray(target, dtype=np.float32).reshape(-1)
    mask = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1)
    n = width * height
    out = np.empty(n * channels, dtype=np.float64)
    ach = np.zeros(max(channels, 1), dtype=np.float64)
    its = np.zeros(max(channels, 1), dtype=np.uint32)
    rc = lib().pr_mgcg_blend_channels(_p(source), _p(target), _p(mask), channels, width, height,
                                      float(lam), float(rel_tol), int(max_iterations), _p(out),
                                      _p(ach), _p(its))
    if rc < 0:
        raise MemoryError("oracle allocation failed")
    return out, ach[:channels], its[:channels]


def mask_ellipse(width, height, center, radii, angle_rad=0.0, half_width_px=0.0) -> np.ndarray:
    """``mask.ellipse@1`` coverage (height, width) f32 (ellipse.rs:168-218,545-565)."""
    out = np.empty((height, width), dtype=np.float32)
    lib().or_mask_ellipse(width, height, float(center[0]), float(center[1]), float(radii[0]),
                          float(radii[1]), float(angle_rad), float(half_width_px), _p(out))
    return out


def mask_polygon(width, height, points, fill_rule="nonzero") -> np.ndarray:
    """``mask.polygon@1`` coverage (height, width) f32, 4x4 supersampled, half-open
    (mask_polygon.rs:161-196,259-286)."""
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 2))
    out = np.empty((height, width), dtype=np.float32)
    rule = {"nonzero": 0, "even-odd": 1}[fill_rule]
    lib().or_mask_polygon(width, height, _p(pts), pts.shape[0], rule, _p(out))
    return out
