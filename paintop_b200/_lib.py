"""ctypes binding of ``libpaintop_cuda.so`` (the C ABI declared in include/paintop_cuda.h).

This module is plumbing: it loads the in-tree CUDA library and exposes its
entry points with numpy arrays. There is no fallback: if the library is
missing, importing :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpaintop_cuda.so")

PT_OK, PT_NO_DEVICE, PT_INVALID_ARG, PT_LAUNCH_FAILED, PT_TIMEOUT, PT_OOM, PT_INTERNAL = range(7)
PT_FLAG_WARM_START = 0x1
PT_FLAG_DEVICE_POINTERS = 0x2
PT_FILL_NONZERO, PT_FILL_EVEN_ODD = 0, 1
PT_FLAG_OMEGA_AUTO = 0x4
PT_FLAG_MULTIGRID = 0x8
PT_KIND_IMAGE, PT_KIND_MASK = 0, 1
STOP_REASONS = ("converged", "max-iterations", "stalled")

# Every symbol include/paintop_cuda.h declares.
EXPORTED = (
    "pt_ctx_create", "pt_ctx_destroy", "pt_poisson_solve", "pt_poisson_solve_batch",
    "pt_op_compute", "pt_op_compute_ex", "pt_status_str", "pt_ctx_last_error", "pt_tile_config_count",
    "pt_tile_config_info", "pt_ctx_set_config", "pt_ctx_last_config", "pt_autotune",
    "pt_ctx_set_budget", "pt_ctx_stream", "pt_ctx_last_timing", "pt_ctx_last_transfer", "pt_poisson_solve_noalloc",
    "pt_unet_create", "pt_unet_destroy", "pt_unet_param_count", "pt_unet_get_params",
    "pt_unet_set_params", "pt_unet_features", "pt_unet_forward", "pt_unet_loss_grad",
    "pt_unet_train_step", "pt_unet_save", "pt_unet_load", "pt_unet_guess", "pt_unet_grad_record",
    "pt_unet_apply_records", "pt_mask_ellipse", "pt_mask_polygon",
)
PT_NOALLOC_SCRATCH_BYTES = 64 * 1024 * 1024


class PtProblem(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32), ("channels", C.c_uint32),
        ("source_or_guidance", C.c_void_p), ("target_or_anchor", C.c_void_p),
        ("mask", C.c_void_p), ("lambda_", C.c_double), ("max_iterations", C.c_uint32),
        ("tolerance", C.c_double), ("omega", C.c_double), ("flags", C.c_uint32),
        ("initial_guess", C.c_void_p),
    ]


class PtReport(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32), ("converged", C.c_int32), ("stop_reason", C.c_int32),
        ("tolerance", C.c_double), ("final_residual", C.c_double), ("history_len", C.c_uint32),
        ("omega_used", C.c_double), ("refinements", C.c_uint32), ("channel", C.c_int32),
        ("initial_residual", C.c_double), ("warm_start", C.c_int32),
    ]

    def as_dict(self, history=None):
        d = dict(iterations=int(self.iterations), converged=bool(self.converged),
                 stop_reason=STOP_REASONS[self.stop_reason] if 0 <= self.stop_reason < 3 else "?",
                 tolerance=float(self.tolerance), final_residual=float(self.final_residual),
                 history_len=int(self.history_len), omega_used=float(self.omega_used),
                 refinements=int(self.refinements), channel=int(self.channel),
                 initial_residual=float(self.initial_residual),
                 warm_start=bool(self.warm_start))
        if history is not None:
            d["residual_history"] = history
        return d


class PtPort(C.Structure):
    _fields_ = [
        ("name", C.c_char_p), ("kind", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
        ("channels", C.c_uint32), ("samples", C.c_void_p), ("sample_count", C.c_size_t),
    ]


class PtError(C.Structure):
    _fields_ = [
        ("error_class", C.c_char * 16), ("code", C.c_char * 40), ("message", C.c_char * 256),
        ("actual", C.c_char * 96),
    ]


class PtSolverData(C.Structure):
    _fields_ = [
        ("kind", C.c_char * 24), ("steps", C.c_uint32), ("stability_number", C.c_double),
        ("stability_limit", C.c_double), ("stable", C.c_int32), ("total_energy", C.c_double),
        ("iterations", C.c_uint32), ("stop_reason", C.c_int32), ("converged", C.c_int32),
        ("tolerance", C.c_double), ("final_residual", C.c_double), ("history_len", C.c_uint32),
    ]


_lib = None


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m paintop_b200.build` "
            "(the cuda backend has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, u32, i32 = C.c_void_p, C.c_uint32, C.c_int32
    L.pt_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.pt_ctx_create.restype = C.c_int
    L.pt_ctx_destroy.argtypes = [vp]
    L.pt_ctx_destroy.restype = C.c_int
    L.pt_poisson_solve.argtypes = [vp, C.POINTER(PtProblem), vp, C.POINTER(PtReport), vp]
    L.pt_poisson_solve.restype = C.c_int
    L.pt_poisson_solve_batch.argtypes = [vp, C.POINTER(PtProblem), u32, C.POINTER(vp),
                                         C.POINTER(C.POINTER(PtReport)), C.POINTER(vp)]
    L.pt_poisson_solve_batch.restype = C.c_int
    L.pt_op_compute.argtypes = [vp, C.c_char_p, C.POINTER(PtPort), u32, C.c_char_p, vp, C.c_size_t,
                                C.POINTER(PtSolverData), vp, u32, C.POINTER(i32), C.POINTER(PtError)]
    L.pt_op_compute.restype = C.c_int
    L.pt_op_compute_ex.argtypes = list(L.pt_op_compute.argtypes) + [u32]
    L.pt_op_compute_ex.restype = C.c_int
    L.pt_status_str.argtypes = [C.c_int]
    L.pt_status_str.restype = C.c_char_p
    L.pt_ctx_last_error.argtypes = [vp]
    L.pt_ctx_last_error.restype = C.c_char_p
    L.pt_tile_config_count.argtypes = []
    L.pt_tile_config_count.restype = u32
    L.pt_tile_config_info.argtypes = [u32, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    L.pt_tile_config_info.restype = C.c_int
    L.pt_ctx_set_config.argtypes = [vp, i32]
    L.pt_ctx_set_config.restype = C.c_int
    L.pt_ctx_last_config.argtypes = [vp]
    L.pt_ctx_last_config.restype = i32
    L.pt_autotune.argtypes = [vp, C.POINTER(PtProblem), u32, u32, C.POINTER(vp),
                              C.POINTER(C.POINTER(PtReport)), C.POINTER(i32), vp]
    L.pt_autotune.restype = C.c_int
    L.pt_ctx_set_budget.argtypes = [vp, C.c_double]
    L.pt_ctx_set_budget.restype = C.c_int
    L.pt_ctx_stream.argtypes = [vp]
    L.pt_ctx_stream.restype = vp
    L.pt_ctx_last_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.POINTER(C.c_int64)]
    L.pt_ctx_last_timing.restype = C.c_int
    L.pt_ctx_last_transfer.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.pt_ctx_last_transfer.restype = C.c_int
    L.pt_poisson_solve_noalloc.argtypes = [C.POINTER(PtProblem), vp, C.POINTER(PtReport), vp, vp]
    L.pt_poisson_solve_noalloc.restype = C.c_int
    u64, f32 = C.c_uint64, C.c_float
    L.pt_unet_create.argtypes = [vp, u64, C.POINTER(vp)]
    L.pt_unet_destroy.argtypes = [vp]
    L.pt_unet_param_count.argtypes = [vp]
    L.pt_unet_param_count.restype = u64
    L.pt_unet_get_params.argtypes = [vp, vp]
    L.pt_unet_set_params.argtypes = [vp, vp]
    L.pt_unet_features.argtypes = [vp, vp, vp, vp, u32, u32, u32, vp]
    L.pt_unet_forward.argtypes = [vp, vp, u32, u32, u32, vp]
    L.pt_unet_loss_grad.argtypes = [vp, vp, vp, vp, u32, u32, u32, C.POINTER(C.c_double), vp]
    L.pt_unet_train_step.argtypes = [vp, vp, vp, vp, u32, u32, u32, f32, C.POINTER(C.c_double)]
    L.pt_unet_guess.argtypes = [vp, vp, vp, vp, u32, u32, u32, u32, vp]
    d = C.c_double
    L.pt_mask_ellipse.argtypes = [vp, u32, u32, d, d, d, d, d, d, vp, u32]
    L.pt_mask_ellipse.restype = C.c_int
    L.pt_mask_polygon.argtypes = [vp, u32, u32, vp, u32, C.c_int32, vp, u32]
    L.pt_mask_polygon.restype = C.c_int
    L.pt_unet_grad_record.argtypes = [vp, vp, vp, vp, u32, u32, u32, C.POINTER(C.c_double), vp]
    L.pt_unet_apply_records.argtypes = [vp, vp, u32, f32]
    L.pt_unet_save.argtypes = [vp, C.c_char_p]
    L.pt_unet_load.argtypes = [vp, C.c_char_p]
    for name in ("pt_unet_create", "pt_unet_destroy", "pt_unet_get_params", "pt_unet_set_params",
                 "pt_unet_features", "pt_unet_forward", "pt_unet_loss_grad", "pt_unet_train_step",
                 "pt_unet_save", "pt_unet_load", "pt_unet_guess", "pt_unet_grad_record",
                 "pt_unet_apply_records"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


class CudaError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        msg = lib().pt_status_str(status).decode()
        super().__init__(f"{msg} (status {status}){': ' + detail if detail else ''}")


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a)  # a raw device pointer


class Context:
    """A library context (one CUDA stream, a device arena) on one GPU."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = lib().pt_ctx_create(device, C.byref(h))
        if st != PT_OK:
            raise CudaError(st, "pt_ctx_create")
        self.h = h
        self.device = int(device)
        self._children = weakref.WeakSet()  # objects whose C handles point into this context

    def adopt(self, child) -> None:
        """Register an object with a close() that must run before the context is destroyed."""
        self._children.add(child)

    def close(self):
        if getattr(self, "h", None):
            for child in list(self._children):
                child.close()
            lib().pt_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def last_error(self) -> str:
        return lib().pt_ctx_last_error(self.h).decode()

    def set_config(self, cfg: int):
        st = lib().pt_ctx_set_config(self.h, int(cfg))
        if st != PT_OK:
            raise CudaError(st)

    def set_budget(self, seconds: float):
        st = lib().pt_ctx_set_budget(self.h, float(seconds))
        if st != PT_OK:
            raise CudaError(st)

    def stream(self) -> int:
        return int(lib().pt_ctx_stream(self.h) or 0)

    def last_timing(self):
        """(persistent solve kernel ms, whole call ms, kernels launched) of the last solve."""
        a, b, n = C.c_double(), C.c_double(), C.c_int64()
        lib().pt_ctx_last_timing(self.h, C.byref(a), C.byref(b), C.byref(n))
        return a.value, b.value, int(n.value)

    def last_transfer(self):
        """(host->device bytes, device->host bytes) of the last red-black solve call."""
        a, b = C.c_uint64(), C.c_uint64()
        lib().pt_ctx_last_transfer(self.h, C.byref(a), C.byref(b))
        return int(a.value), int(b.value)

    def last_config(self) -> int:
        return int(lib().pt_ctx_last_config(self.h))

    # -- solves ------------------------------------------------------------
    @staticmethod
    def make_problem(source, target, mask, width, height, channels, lam=0.0, max_iterations=2000,
                     tolerance=1e-6, omega=1.8, flags=0, initial_guess=None) -> PtProblem:
        return PtProblem(int(width), int(height), int(channels), _ptr(source), _ptr(target),
                         _ptr(mask), float(lam), int(max_iterations), float(tolerance),
                         float(omega), int(flags | (PT_FLAG_WARM_START if initial_guess is not None
                                                    else 0)), _ptr(initial_guess))

    def solve(self, source, target, mask, width, height, channels, *, lam=0.0, max_iterations=2000,
              tolerance=1e-6, omega=1.8, flags=0, initial_guess=None, want_history=True):
        """pt_poisson_solve with host numpy arrays -> (out f32, [per-channel reports], worst)."""
        source = np.ascontiguousarray(source, dtype=np.float32)
        target = np.ascontiguousarray(target, dtype=np.float32)
        mask = np.ascontiguousarray(mask, dtype=np.float32)
        if initial_guess is not None:
            initial_guess = np.ascontiguousarray(initial_guess, dtype=np.float32)
        n = int(width) * int(height) * int(channels)
        assert source.size == n and target.size == n and mask.size == int(width) * int(height)
        out = np.empty(n, dtype=np.float32)
        reps = (PtReport * (int(channels) + 1))()
        hist = np.zeros(max(int(channels) * int(max_iterations), 1), dtype=np.float64) \
            if want_history else None
        p = self.make_problem(source, target, mask, width, height, channels, lam, max_iterations,
                              tolerance, omega, flags, initial_guess)
        st = lib().pt_poisson_solve(self.h, C.byref(p), out.ctypes.data, reps,
                                    hist.ctypes.data if hist is not None else None)
        if st != PT_OK:
            raise CudaError(st, self.last_error())
        per = []
        for c in range(int(channels)):
            h = None
            if hist is not None:
                k = reps[c].history_len
                h = hist[c * max_iterations: c * max_iterations + k].tolist()
            per.append(reps[c].as_dict(h))
        worst = reps[int(channels)].as_dict(
            per[reps[int(channels)].channel]["residual_history"]
            if channels and hist is not None and reps[int(channels)].channel >= 0 else
            ([] if hist is not None else None))
        return out, per, worst

    def solve_batch(self, problems, want_history=False):
        """pt_poisson_solve_batch. problems: list of dicts with the solve() arguments."""
        n = len(problems)
        keep = []
        arr = (PtProblem * n)()
        outs = (C.c_void_p * n)()
        rep_arrays = []
        rep_ptrs = (C.POINTER(PtReport) * n)()
        hist_ptrs = (C.c_void_p * n)()
        results = []
        for i, pr in enumerate(problems):
            src = np.ascontiguousarray(pr["source"], dtype=np.float32)
            tgt = np.ascontiguousarray(pr["target"], dtype=np.float32)
            msk = np.ascontiguousarray(pr["mask"], dtype=np.float32)
            guess = pr.get("initial_guess")
            if guess is not None:
                guess = np.ascontiguousarray(guess, dtype=np.float32)
            w, h, c = int(pr["width"]), int(pr["height"]), int(pr["channels"])
            out = np.empty(w * h * c, dtype=np.float32)
            reps = (PtReport * (c + 1))()
            mi = int(pr.get("max_iterations", 2000))
            hist = np.zeros(max(c * mi, 1), dtype=np.float64) if want_history else None
            keep += [src, tgt, msk, guess, out, reps, hist]
            arr[i] = self.make_problem(src, tgt, msk, w, h, c, pr.get("lam", 0.0), mi,
                                       pr.get("tolerance", 1e-6), pr.get("omega", 1.8),
                                       pr.get("flags", 0), guess)
            outs[i] = out.ctypes.data
            rep_ptrs[i] = C.cast(reps, C.POINTER(PtReport))
            hist_ptrs[i] = hist.ctypes.data if hist is not None else None
            rep_arrays.append(reps)
            results.append((out, reps, hist, c, mi))
        st = lib().pt_poisson_solve_batch(self.h, arr, n, outs, rep_ptrs,
                                          hist_ptrs if want_history else None)
        if st != PT_OK:
            raise CudaError(st, self.last_error())
        ret = []
        for out, reps, hist, c, mi in results:
            per = []
            for k in range(c):
                hh = None
                if hist is not None:
                    hh = hist[k * mi: k * mi + reps[k].history_len].tolist()
                per.append(reps[k].as_dict(hh))
            ret.append((out, per, reps[c].as_dict()))
        return ret

    def op_compute(self, op_id: str, inputs: dict, params_json: str, history_cap: int = 100000,
                   solve_flags: int = 0):
        """pt_op_compute (pt_op_compute_ex when solve_flags is not 0). inputs:
        name -> (kind, width, height, channels, samples f32)."""
        ports = (PtPort * len(inputs))()
        keep = []
        out_shape = None
        for k, (name, (kind, w, h, c, samples)) in enumerate(inputs.items()):
            s = np.ascontiguousarray(samples, dtype=np.float32).reshape(-1)
            keep.append(s)
            nm = name.encode()
            keep.append(nm)
            ports[k] = PtPort(nm, kind, w, h, c, s.ctypes.data, s.size)
        # output is the target/anchor descriptor (a mask generator's: extent_from's extent)
        for name in ("target", "anchor"):
            if name in inputs:
                _, w, h, c, _ = inputs[name]
                out_shape = (w, h, c)
        if op_id.startswith("mask.") and "extent_from" in inputs:
            _, w, h, _, _ = inputs["extent_from"]
            out_shape = (w, h, 1)
        count = out_shape[0] * out_shape[1] * out_shape[2] if out_shape else 0
        cand = np.empty(max(count, 1), dtype=np.float32)
        sd = PtSolverData()
        hist = np.zeros(max(history_cap, 1), dtype=np.float64)
        fin = C.c_int32(0)
        err = PtError()
        args = (self.h, op_id.encode(), ports, len(inputs), params_json.encode(), cand.ctypes.data, count,
                C.byref(sd), hist.ctypes.data, history_cap, C.byref(fin), C.byref(err))
        st = lib().pt_op_compute_ex(*args, solve_flags) if solve_flags else lib().pt_op_compute(*args)
        return st, cand[:count], sd, hist[: min(sd.history_len, history_cap)].tolist(), \
            bool(fin.value), err
