"""pt_poisson_solve_noalloc: the solve for callers that may not allocate.

Hosts whose device memory belongs to another allocator (a plugin inside a
framework's caching pool) or that run on latency-critical threads cannot call
cudaMalloc/cudaFree; this entry point works from a fixed device array inside the
library instead. The test drives it through the C ABI twice in a row (the array
keeps the first call's contents, so the second call shows that everything that
must start at zero is cleared) and compares each result with pt_poisson_solve on
the same device buffers. This file sorts last so that a stop-at-first-failure run
has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_ABS = 1e-6  # the agreement the other GPU parity tests require between solvers


def _inputs(seed, size, channels):
    from paintop_b200 import synth
    inst = synth.screened_2048(seed, size=size)
    src = inst.source[:, :, :channels].reshape(-1).copy()
    tgt = inst.target[:, :, :channels].reshape(-1).copy()
    return src, tgt, inst.mask.reshape(-1).copy()


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
