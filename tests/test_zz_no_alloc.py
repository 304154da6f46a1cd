"""pt_poisson_solve_noalloc: the solve for callers that may not allocate.

Hosts whose device memory belongs to another allocator (a plugin inside a
framework's caching pool) or that run on latency-critical threads cannot call
cudaMalloc/cudaFree; this entry point works from a fixed device array inside the
library instead. The test drives it through the C ABI twice in a row (the array
keeps the first call's contents, so the second call shows that everything that
must start at zero is cleared) and compares each result with pt_poisson_solve on
the same device buffers. This file sorts last so that a stop-at-first-failure run
has already run every other test. The argument checks run on the CPU: every
rejection returns before the call touches the CUDA runtime.
"""
import ctypes as C

import numpy as np
import pytest

TOL_ABS = 1e-6  # the agreement the other GPU parity tests require between solvers


def _inputs(seed, size, channels):
    from paintop_b200 import synth
    inst = synth.screened_2048(seed, size=size)
    src = inst.source[:, :, :channels].reshape(-1).copy()
    tgt = inst.target[:, :, :channels].reshape(-1).copy()
    return src, tgt, inst.mask.reshape(-1).copy()


@pytest.mark.gpu
def test_noalloc_matches_solve_on_two_calls_in_a_row(cuda_lib):
    import torch
    from paintop_b200 import _lib

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ctx = _lib.Context(0)
    try:
        for call, (seed, size, ch, lam) in enumerate([(11, 256, 4, 0.01), (12, 200, 3, 0.0)]):
            src, tgt, mask = _inputs(seed, size, ch)
            W = H = size
            d_src = torch.from_numpy(src).to(dev)
            d_tgt = torch.from_numpy(tgt).to(dev)
            d_mask = torch.from_numpy(mask).to(dev)
            max_it = 2000
            p = _lib.PtProblem(W, H, ch, d_src.data_ptr(), d_tgt.data_ptr(), d_mask.data_ptr(),
                               lam, max_it, 1e-6, 1.8, _lib.PT_FLAG_DEVICE_POINTERS, None)

            out_na = torch.full((W * H * ch,), float("nan"), device=dev)
            hist_na = torch.zeros(ch * max_it, dtype=torch.float64, device=dev)
            rep_na = (_lib.PtReport * (ch + 1))()
            torch.cuda.synchronize()
            st = L.pt_poisson_solve_noalloc(C.byref(p), out_na.data_ptr(), rep_na,
                                            hist_na.data_ptr(), None)
            assert st == _lib.PT_OK, f"call {call}: status {st}"

            out_ref = torch.empty(W * H * ch, device=dev)
            hist_ref = torch.zeros(ch * max_it, dtype=torch.float64, device=dev)
            rep_ref = (_lib.PtReport * (ch + 1))()
            st = L.pt_poisson_solve(ctx.h, C.byref(p), out_ref.data_ptr(), rep_ref,
                                    hist_ref.data_ptr())
            assert st == _lib.PT_OK, ctx.last_error()

            a, b = out_na.cpu().numpy(), out_ref.cpu().numpy()
            assert np.isfinite(a).all()
            assert np.abs(a - b).max() <= TOL_ABS
            for c in range(ch + 1):
                assert rep_na[c].converged == rep_ref[c].converged == 1
                assert rep_na[c].stop_reason == rep_ref[c].stop_reason
                assert abs(int(rep_na[c].iterations) - int(rep_ref[c].iterations)) <= 3
                assert rep_na[c].final_residual <= 1e-6
            hn, hr = hist_na.cpu().numpy(), hist_ref.cpu().numpy()
            for c in range(ch):
                k = min(rep_na[c].iterations, rep_ref[c].iterations)
                assert np.allclose(hn[c * max_it: c * max_it + k], hr[c * max_it: c * max_it + k],
                                   rtol=1e-3, atol=1e-9)
            # the target survives bit for bit outside the mask
            from oracle import oracle as O
            keep = np.repeat(O.classify_cells(mask, W, H) == 0, ch)
            assert np.array_equal(a[keep].view(np.uint32), tgt[keep].view(np.uint32))
    finally:
        ctx.close()


@pytest.mark.gpu
def test_noalloc_rejects_problems_beyond_the_array(cuda_lib):
    import torch
    from paintop_b200 import _lib

    dev = torch.device("cuda", 0)
    W = H = 2048
    buf = torch.zeros(16, device=dev)  # never read: the size check comes first
    p = _lib.PtProblem(W, H, 4, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 0.0, 2000, 1e-6,
                       1.8, _lib.PT_FLAG_DEVICE_POINTERS, None)
    reps = (_lib.PtReport * 5)()
    assert _lib.lib().pt_poisson_solve_noalloc(C.byref(p), buf.data_ptr(), reps, None,
                                               None) == _lib.PT_OOM


def _problem(**kw):
    from paintop_b200 import _lib
    a = dict(width=64, height=64, channels=3, lam=0.0, max_it=100, tol=1e-6, omega=1.8,
             flags=_lib.PT_FLAG_DEVICE_POINTERS, ptr=0x1000)
    a.update(kw)
    return _lib.PtProblem(a["width"], a["height"], a["channels"], a["ptr"], a["ptr"], a["ptr"],
                          a["lam"], a["max_it"], a["tol"], a["omega"], a["flags"], a["ptr"])


def _rejections():
    from paintop_b200 import _lib
    return [
        ("host pointers", dict(flags=0)),
        ("warm start", dict(flags=_lib.PT_FLAG_DEVICE_POINTERS | _lib.PT_FLAG_WARM_START)),
        ("automatic omega", dict(flags=_lib.PT_FLAG_DEVICE_POINTERS | _lib.PT_FLAG_OMEGA_AUTO)),
        ("nine channels", dict(channels=9)),
        ("omega 0", dict(omega=0.0)),
        ("omega 2", dict(omega=2.0)),
        ("omega nan", dict(omega=float("nan"))),
        ("negative lambda", dict(lam=-1.0)),
        ("tolerance 0", dict(tol=0.0)),
        ("zero width", dict(width=0)),
        ("null buffers", dict(ptr=0)),
        ("width 2^32-1", dict(width=0xFFFFFFFF, height=1)),
        ("width 2^31", dict(width=1 << 31, height=1)),
        ("2^31+ pixels", dict(width=1 << 16, height=(1 << 15) + 1)),
        ("cap above 10^6", dict(max_it=1000001)),
    ]


@pytest.mark.parametrize("case", range(15))
def test_noalloc_rejects_bad_arguments_before_the_gpu(cuda_lib, case):
    from paintop_b200 import _lib
    cases = _rejections()
    assert len(cases) == 15
    name, kw = cases[case]
    p = _problem(**kw)
    reps = (_lib.PtReport * 10)()
    st = cuda_lib.pt_poisson_solve_noalloc(C.byref(p), 0x1000 if kw.get("ptr", 1) else None,
                                           reps, None, None)
    assert st == _lib.PT_INVALID_ARG, (name, st)


def test_noalloc_rejects_null_problem_or_reports(cuda_lib):
    from paintop_b200 import _lib
    p = _problem()
    assert cuda_lib.pt_poisson_solve_noalloc(None, 0x1000, (_lib.PtReport * 4)(), None,
                                             None) == _lib.PT_INVALID_ARG
    assert cuda_lib.pt_poisson_solve_noalloc(C.byref(p), 0x1000, None, None,
                                             None) == _lib.PT_INVALID_ARG


def test_noalloc_size_limit_is_checked_before_the_gpu(cuda_lib):
    # 2048 x 2048 RGBA needs far more than the fixed array: PT_OOM with no CUDA call
    from paintop_b200 import _lib
    p = _problem(width=2048, height=2048, channels=4, max_it=2000)
    assert cuda_lib.pt_poisson_solve_noalloc(C.byref(p), 0x1000, (_lib.PtReport * 5)(), None,
                                             None) == _lib.PT_OOM


@pytest.mark.parametrize("fault,status", [("host-oom", "PT_OOM"), ("host-exception", "PT_INTERNAL")])
def test_noalloc_host_exception_becomes_a_status(cuda_lib, monkeypatch, fault, status):
    """A C++ exception thrown inside the entry point (here by the test hook,
    after the argument checks and before any device work) is returned as a
    status: host allocation failure as PT_OOM, anything else as PT_INTERNAL.
    Nothing unwinds through the C ABI."""
    from paintop_b200 import _lib
    monkeypatch.setenv("PAINTOP_CUDA_FAULT", fault)
    p = _problem()
    st = cuda_lib.pt_poisson_solve_noalloc(C.byref(p), 0x1000, (_lib.PtReport * 4)(), None, None)
    assert st == getattr(_lib, status)
