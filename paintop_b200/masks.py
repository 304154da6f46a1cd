"""Device mask generators: ``mask.ellipse@1`` and ``mask.polygon@1`` rasterised
on the GPU (``pt_mask_ellipse`` / ``pt_mask_polygon``) straight into device
memory, ready to be a solve's mask without a host round trip.

The semantics are the reference's: pixel (i, j) spans [i, i+1) x [j, j+1); the
ellipse is sampled at pixel centres with an optional smoothstep feather
(crates/paintop-cpu/src/ellipse.rs:168-218); the polygon's coverage is the
fraction of a 4 x 4 subsample grid inside it by a half-open +x ray cast under
the nonzero or even-odd rule (crates/paintop-cpu/src/mask_polygon.rs:161-196,
259-286), bit-identical to the reference.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

FILL_RULES = {"nonzero": 0, "even-odd": 1}


def _check(ctx, st, what):
    if st != _lib.PT_OK:
        raise _lib.CudaError(st, f"{what}: {ctx.last_error()}")


def _target(out, width, height, device):
    import torch
    if out is None:
        return torch.empty((height, width), dtype=torch.float32, device=device)
    if not (out.is_cuda and out.dtype == torch.float32 and out.is_contiguous() and out.numel() == width * height):
        raise ValueError("out must be a contiguous float32 CUDA tensor of width*height elements")
    return out


def ellipse(ctx, width: int, height: int, center, radii, angle_rad: float = 0.0, half_width_px: float = 0.0,
            out=None, device="cuda"):
    """Ellipse coverage (height, width) on the device."""
    import torch
    out = _target(out, width, height, device)
    torch.cuda.synchronize()
    _check(ctx, _lib.lib().pt_mask_ellipse(ctx.h, width, height, float(center[0]), float(center[1]),
                                           float(radii[0]), float(radii[1]), float(angle_rad),
                                           float(half_width_px), out.data_ptr(), _lib.PT_FLAG_DEVICE_POINTERS),
           "mask.ellipse")
    return out


def polygon(ctx, width: int, height: int, points, fill_rule: str = "nonzero", out=None, device="cuda"):
    """Polygon coverage (height, width) on the device; values are k / 16."""
    import torch
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 2))
    out = _target(out, width, height, device)
    torch.cuda.synchronize()
    _check(ctx, _lib.lib().pt_mask_polygon(ctx.h, width, height, pts.ctypes.data_as(C.c_void_p), pts.shape[0],
                                           FILL_RULES[fill_rule], out.data_ptr(), _lib.PT_FLAG_DEVICE_POINTERS),
           "mask.polygon")
    return out


def polygon_host(ctx, width: int, height: int, points, fill_rule: str = "nonzero") -> np.ndarray:
    """Polygon coverage into host memory (the library stages it on the device)."""
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 2))
    out = np.empty((height, width), dtype=np.float32)
    _check(ctx, _lib.lib().pt_mask_polygon(ctx.h, width, height, pts.ctypes.data_as(C.c_void_p), pts.shape[0],
                                           FILL_RULES[fill_rule], out.ctypes.data_as(C.c_void_p), 0),
           "mask.polygon")
    return out


def ellipse_host(ctx, width: int, height: int, center, radii, angle_rad: float = 0.0,
                 half_width_px: float = 0.0) -> np.ndarray:
    """Ellipse coverage into host memory."""
    out = np.empty((height, width), dtype=np.float32)
    _check(ctx, _lib.lib().pt_mask_ellipse(ctx.h, width, height, float(center[0]), float(center[1]),
                                           float(radii[0]), float(radii[1]), float(angle_rad),
                                           float(half_width_px), out.ctypes.data_as(C.c_void_p), 0),
           "mask.ellipse")
    return out
