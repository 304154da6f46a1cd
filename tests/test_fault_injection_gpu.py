"""Failure paths on the GPU, made without a GPU fault.

* Host-injected failures (PAINTOP_CUDA_FAULT=oom | launch): the solve returns
  PT_OOM / PT_LAUNCH_FAILED before any device work, the op layer maps them to
  its execution error, and the same context then solves normally. With
  host-oom | host-exception a C++ exception is thrown inside the call and the
  entry point's guard returns PT_OOM / PT_INTERNAL instead of unwinding
  through the C ABI. The
  reference's analogue is the typed GPU-unavailable error
  (crates/paintop-wgpu/src/gpu/error.rs:17, probe.rs:223).
* A bounded device wait that runs out (PAINTOP_CUDA_FAULT=unet-stall): the
  U-Net's first convolution waits on a barrier phase nothing completes, under a
  0.1 s limit; the kernel takes its abort path (drains its copies, frees its
  tensor memory), the call returns PT_TIMEOUT, and the next call on the same
  network gives the result of a network that never timed out.
"""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class injected:
    """PAINTOP_CUDA_FAULT set for the duration of a with-block (the library
    reads it on each call)."""

    def __init__(self, what):
        self.what = what

    def __enter__(self):
        self.old = os.environ.get("PAINTOP_CUDA_FAULT")
        os.environ["PAINTOP_CUDA_FAULT"] = self.what

    def __exit__(self, *exc):
        if self.old is None:
            os.environ.pop("PAINTOP_CUDA_FAULT", None)
        else:
            os.environ["PAINTOP_CUDA_FAULT"] = self.old


def _problem():
    from paintop_b200 import synth
    inst = synth.screened_2048(2, size=96)
    return (inst.source.reshape(-1), inst.target.reshape(-1), inst.mask.reshape(-1),
            inst.width, inst.height, inst.channels)


@pytest.mark.parametrize("fault,status", [("oom", "PT_OOM"), ("launch", "PT_LAUNCH_FAILED")])
def test_injected_host_failure_returns_its_status_and_the_context_survives(ctx, fault, status):
    from paintop_b200 import _lib
    src, tgt, mask, W, H, Ch = _problem()
    want, per, _ = ctx.solve(src, tgt, mask, W, H, Ch, lam=0.01)
    with injected(fault):
        with pytest.raises(_lib.CudaError) as e:
            ctx.solve(src, tgt, mask, W, H, Ch, lam=0.01)
    assert e.value.status == getattr(_lib, status)
    assert "injected" in ctx.last_error()
    got, per2, _ = ctx.solve(src, tgt, mask, W, H, Ch, lam=0.01)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert [r["iterations"] for r in per2] == [r["iterations"] for r in per]


@pytest.mark.parametrize("fault,status,msg", [("host-oom", "PT_OOM", "host memory allocation failed"),
                                              ("host-exception", "PT_INTERNAL", "unexpected host-side exception")])
def test_host_exception_in_a_solve_returns_a_status_and_the_context_survives(ctx, fault, status, msg):
    """A C++ exception inside pt_poisson_solve (thrown by the test hook after
    the argument checks) comes back as a status with the message on the
    context; the context's lock is released and the next solve is unchanged."""
    from paintop_b200 import _lib
    src, tgt, mask, W, H, Ch = _problem()
    want, per, _ = ctx.solve(src, tgt, mask, W, H, Ch, lam=0.01)
    with injected(fault):
        with pytest.raises(_lib.CudaError) as e:
            ctx.solve(src, tgt, mask, W, H, Ch, lam=0.01)
    assert e.value.status == getattr(_lib, status)
    assert msg in ctx.last_error()
    got, per2, _ = ctx.solve(src, tgt, mask, W, H, Ch, lam=0.01)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert [r["iterations"] for r in per2] == [r["iterations"] for r in per]


@pytest.mark.parametrize("fault", ["oom", "launch"])
def test_injected_failure_through_the_op_is_an_execution_error(cuda_lib, fault):
    from paintop_b200 import ops
    src, tgt, mask, W, H, Ch = _problem()
    inputs = {"source": ops.image_value(W, H, Ch, src), "target": ops.image_value(W, H, Ch, tgt),
              "mask": ops.mask_value(W, H, mask)}
    with injected(fault):
        with pytest.raises(ops.PaintopError) as e:
            ops.PoissonBlend().compute(inputs, {})
    assert e.value.error_class == "execution" and e.value.code == "E_CUDA_EXECUTION"
    out = ops.PoissonBlend().compute(inputs, {})
    assert out["report"].as_report().solver.converged


def test_unet_wait_runs_out_returns_timeout_and_the_network_stays_usable(ctx):
    import torch
    from paintop_b200 import _lib, warmstart
    net = warmstart.UNet(ctx, seed=11)
    try:
        g, a, m = warmstart.make_instances(2, 64, seed=12)
        feats = net.features(g, a, m)
        want = net.forward(feats)
        B, H, W, _ = feats.shape
        pred = torch.empty((B, H, W), device=feats.device, dtype=torch.float32)
        torch.cuda.synchronize()
        with injected("unet-stall"):
            st = _lib.lib().pt_unet_forward(net.h, feats.data_ptr(), B, H, W, pred.data_ptr())
        assert st == _lib.PT_TIMEOUT
        assert "wait gave up" in ctx.last_error()
        # the same network and context, same inputs: the result of a network
        # that never timed out, bit for bit
        got = net.forward(feats)
        assert torch.equal(got, want)
        # and a training step still runs and is finite
        target = torch.zeros_like(g)
        loss = net.train_step(feats, target, warmstart.interior_mask(m))
        assert np.isfinite(loss)
    finally:
        net.close()
