"""The ``cuda.poisson@1`` implementation of ``repair.poisson_blend@1`` and
``repair.screened_poisson@1``, and of the mask generators ``mask.ellipse@1``
and ``mask.polygon@1`` that feed them, as seen from Python.

Mirrors the reference's operator interface: ``compute(inputs, params)`` takes a
map of port name -> resource value and the op's JSON params and returns the
``candidate`` image plus the ``report`` carrying ``SolverData``
(crates/paintop-core/src/executor/op_impl.rs:51-70;
crates/paintop-cpu/src/poisson_blend.rs:534-600;
crates/paintop-cpu/src/screened_poisson.rs:361-430). Validation, defaults, error
classes, codes and messages live in the C++ host layer behind ``pt_op_compute``;
this module only marshals values across the C ABI. Errors surface as
:class:`PaintopError` with the reference's class/code/message.
"""
from __future__ import annotations

import json
import threading
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib

IMPLEMENTATION_ID = "cuda.poisson@1"
# The second implementation of the two Poisson ops: the same contract solved by
# multigrid-preconditioned CG (pt_op_compute_ex with PT_FLAG_MULTIGRID).
MULTIGRID_IMPLEMENTATION_ID = "cuda.multigrid@1"


class PaintopError(Exception):
    """The reference's structured error: class token, stable code, message."""

    def __init__(self, error_class: str, code: str, message: str, actual: str = ""):
        super().__init__(f"[{error_class}/{code}] {message}")
        self.error_class = error_class
        self.code = code
        self.message = message
        self.actual = actual

    # crates/paintop-ir/src/error.rs:103-114
    @property
    def exit_code(self) -> int:
        return {"parse": 2, "schema": 2, "reference": 2, "type": 3, "semantic": 3, "policy": 4,
                "execution": 5}.get(self.error_class, 5)


@dataclass
class SolverData:
    """crates/paintop-ir/src/resource.rs:1130-1178."""

    kind: str
    steps: int
    stability_number: float
    stability_limit: float
    stable: bool
    residual_history: list
    total_energy: float
    iterations: Optional[int]
    stop_reason: Optional[str]
    converged: Optional[bool]
    tolerance: Optional[float]
    final_residual: Optional[float]


@dataclass
class Report:
    width: int
    height: int
    channels: int
    all_finite: bool
    solver: Optional[SolverData] = None

    def to_json(self) -> str:
        """The canonical JSON an evidence bundle stores for this report
        (:mod:`paintop_b200.report_json`)."""
        from .report_json import report_json
        return report_json(self)


@dataclass
class ResourceValue:
    """A resource value: an image or mask (row-major interleaved f32) or a report."""

    kind: str                 # "image" | "mask" | "report"
    width: int
    height: int
    channels: int
    samples: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    report: Optional[Report] = None

    def as_report(self) -> Optional[Report]:
        return self.report


def image_value(width: int, height: int, channels: int, samples) -> ResourceValue:
    return ResourceValue("image", int(width), int(height), int(channels),
                         np.ascontiguousarray(samples, dtype=np.float32).reshape(-1))


def gray_image(width: int, height: int, samples) -> ResourceValue:
    return image_value(width, height, 1, samples)


def mask_value(width: int, height: int, samples) -> ResourceValue:
    return ResourceValue("mask", int(width), int(height), 1,
                         np.ascontiguousarray(samples, dtype=np.float32).reshape(-1))


_ctx = None
_ctx_lock = threading.Lock()


def context() -> _lib.Context:
    """The process-wide context on device 0 (created on first use)."""
    global _ctx
    with _ctx_lock:
        if _ctx is None:
            _ctx = _lib.Context(0)
        return _ctx


class _PoissonOp:
    OP_ID = ""
    PORTS = ("", "", "mask")

    def __init__(self, multigrid: bool = False):
        """multigrid=False: ``cuda.poisson@1`` (red-black SOR). multigrid=True:
        ``cuda.multigrid@1``, the same inputs, params, validation, stopping bar
        and report, solved by multigrid-preconditioned CG; ``steps`` and
        ``iterations`` then count CG iterations."""
        self.solve_flags = _lib.PT_FLAG_MULTIGRID if multigrid else 0
        self.implementation_id = MULTIGRID_IMPLEMENTATION_ID if multigrid else IMPLEMENTATION_ID

    def compute(self, inputs: dict, params) -> dict:
        ctx = context()
        ports = {}
        for name, v in inputs.items():
            kind = _lib.PT_KIND_MASK if v.kind == "mask" else _lib.PT_KIND_IMAGE
            if v.kind == "report":
                kind = 7  # neither an image nor a mask: a Type error in the host layer
            ports[name] = (kind, v.width, v.height, v.channels, v.samples)
        pj = json.dumps(params) if not isinstance(params, str) else params
        st, cand, sd, hist, all_finite, err = ctx.op_compute(self.OP_ID, ports, pj, solve_flags=self.solve_flags)
        if st != _lib.PT_OK:
            if err.code:
                raise PaintopError(err.error_class.decode(), err.code.decode(),
                                   err.message.decode(), err.actual.decode())
            raise _lib.CudaError(st, ctx.last_error())
        target = inputs[self.PORTS[1]]
        solver = SolverData(
            kind=sd.kind.decode(), steps=int(sd.steps), stability_number=sd.stability_number,
            stability_limit=sd.stability_limit, stable=bool(sd.stable), residual_history=hist,
            total_energy=sd.total_energy, iterations=int(sd.iterations),
            stop_reason=_lib.STOP_REASONS[sd.stop_reason], converged=bool(sd.converged),
            tolerance=sd.tolerance, final_residual=sd.final_residual)
        rep = Report(target.width, target.height, target.channels, all_finite, solver)
        return {
            "candidate": image_value(target.width, target.height, target.channels, cand),
            "report": ResourceValue("report", target.width, target.height, 0, report=rep),
        }


class PoissonBlend(_PoissonOp):
    """``repair.poisson_blend@1`` on the ``cuda`` backend."""

    OP_ID = "repair.poisson_blend@1"
    PORTS = ("source", "target", "mask")


class ScreenedPoisson(_PoissonOp):
    """``repair.screened_poisson@1`` on the ``cuda`` backend."""

    OP_ID = "repair.screened_poisson@1"
    PORTS = ("guidance", "anchor", "mask")


class _MaskOp:
    """A mask generator: ``compute({"extent_from": value}, params)`` returns
    ``{"mask": mask value}`` sized to the input's extent."""

    OP_ID = ""

    def compute(self, inputs: dict, params) -> dict:
        ctx = context()
        ports = {}
        for name, v in inputs.items():
            kind = _lib.PT_KIND_MASK if v.kind == "mask" else _lib.PT_KIND_IMAGE
            ports[name] = (kind, v.width, v.height, v.channels, v.samples)
        pj = json.dumps(params) if not isinstance(params, str) else params
        st, out, _, _, _, err = ctx.op_compute(self.OP_ID, ports, pj)
        if st != _lib.PT_OK:
            if err.code:
                raise PaintopError(err.error_class.decode(), err.code.decode(),
                                   err.message.decode(), err.actual.decode())
            raise _lib.CudaError(st, ctx.last_error())
        src = inputs["extent_from"]
        return {"mask": mask_value(src.width, src.height, out)}


class EllipseMask(_MaskOp):
    """``mask.ellipse@1`` on the ``cuda`` backend (crates/paintop-cpu/src/ellipse.rs:506-540)."""

    OP_ID = "mask.ellipse@1"


class PolygonMask(_MaskOp):
    """``mask.polygon@1`` on the ``cuda`` backend (crates/paintop-cpu/src/mask_polygon.rs:427-452)."""

    OP_ID = "mask.polygon@1"
