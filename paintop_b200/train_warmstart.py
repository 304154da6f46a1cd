"""Train and evaluate the learned warm start on the GPU.

  python -m paintop_b200.train_warmstart train --instances 20000 --epochs 8 --out DIR
  python -m paintop_b200.train_warmstart eval256 --params FILE --instances 256
  python -m paintop_b200.train_warmstart multi4096 --params FILE --scale 8
  python -m paintop_b200.train_warmstart steps --batch 64 --steps 10

``train`` generates the seeded 256x256 single-channel instances on the device,
solves each with the library's own red-black SOR + FP64 refinement to a
relative residual of 1e-7 (the training targets are solves of the plain
method), trains the U-Net with Adam (lr 1e-3, batch 64, masked L2 over interior
pixels) through ``pt_unet_train_step``, writes the parameters, a resumable
checkpoint and a JSON report (dataset, throughput in TFLOP/s of the
convolutions, loss curve, held-out evaluation).

Under torchrun (``python -m torch.distributed.run --nproc-per-node N -m
paintop_b200.train_warmstart train ...``) ``train`` is data-parallel: the
dataset's solves are split over the ranks and broadcast, every rank trains a
replica on its part of each batch of 64, and the gradient records are
all-gathered over NCCL and summed in rank order (DataParallelTrainer), so the
replicas stay identical; rank 0 writes the outputs.

``eval256`` and ``multi4096`` compare the learned warm start with the plain
solve on the same inputs: both stop at the same absolute bar, tolerance x
||r(anchor)|| in FP64, and the plain solve is the fallback (a guess whose
residual is not below the anchor's is replaced by the anchor on the device).
Errors are measured against a tight solve of the same problem (FP64 refinement
to a relative residual of 1e-10).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np

from . import _lib, synth
from . import warmstart as ws


def _log(*a):
    print(*a, file=sys.stderr, flush=True)


def solve_image_device(ctx, g, a, m, *, tol, guess=None, max_iterations=100000):
    """pt_poisson_solve on one interleaved (H, W, C) problem held in device tensors."""
    torch = ws._torch()
    H, W, Ch = g.shape
    out = torch.empty_like(g)
    reps = (_lib.PtReport * (Ch + 1))()
    flags = _lib.PT_FLAG_DEVICE_POINTERS | _lib.PT_FLAG_OMEGA_AUTO
    if guess is not None:
        flags |= _lib.PT_FLAG_WARM_START
    p = _lib.PtProblem(W, H, Ch, g.data_ptr(), a.data_ptr(), m.data_ptr(), 0.0, max_iterations, tol, 1.8,
                       flags, guess.data_ptr() if guess is not None else None)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = _lib.lib().pt_poisson_solve(ctx.h, C.byref(p), out.data_ptr(), reps, None)
    dt = time.perf_counter() - t0
    if st != _lib.PT_OK:
        raise _lib.CudaError(st, ctx.last_error())
    kernel_ms, call_ms, launches = ctx.last_timing()
    return out, [reps[c].as_dict() for c in range(Ch)], dict(wall_s=dt, kernel_ms=kernel_ms, call_ms=call_ms)


def evaluate_256(ctx, net, n=256, seed=424242, tol=1e-6):
    """Held-out 256x256 instances: plain vs learned warm start, one batch each."""
    torch = ws._torch()
    g, a, m = ws.make_instances(n, 256, seed)
    ref, _ = ws.solve_batch_device(ctx, g, a, m, tol=1e-10)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    up, rp = ws.solve_batch_device(ctx, g, a, m, tol=tol)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    ws.predict_guess(net, g, a, m)  # warm-up: sizes the network's buffers for this batch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    guess = ws.predict_guess(net, g, a, m)
    torch.cuda.synchronize()
    t_guess = time.perf_counter() - t0
    t0 = time.perf_counter()
    uw, rw = ws.solve_batch_device(ctx, g, a, m, tol=tol, guess=guess)
    torch.cuda.synchronize()
    t_warm = time.perf_counter() - t0
    lm = ws.interior_mask(m)
    nin = float(lm.sum())

    def err(x):
        d = (x - ref) * lm
        return dict(max=float(d.abs().max()), rms=float(((d ** 2).sum() / nin).sqrt()))

    ip = np.array([r["iterations"] for r in rp])
    iw = np.array([r["iterations"] for r in rw])
    return dict(
        instances=n, tolerance=tol,
        plain=dict(sweeps_mean=float(ip.mean()), sweeps_max=int(ip.max()), solve_s=t_plain,
                   solves_per_s=n / t_plain, converged=all(r["converged"] for r in rp), error=err(up)),
        learned=dict(sweeps_mean=float(iw.mean()), sweeps_max=int(iw.max()), guess_s=t_guess, solve_s=t_warm,
                     solves_per_s=n / (t_guess + t_warm), converged=all(r["converged"] for r in rw),
                     error=err(uw), guess_used=int(sum(r["warm_start"] for r in rw)),
                     fewer_sweeps=int((iw < ip).sum()), more_sweeps=int((iw > ip).sum())),
        sweep_ratio=float(iw.mean() / ip.mean()),
        guess_error=err(guess), anchor_error=err(a))


def evaluate_multi4096(ctx, net, seed=1, scale=8, size=4096, tol=1e-6):
    """4096x4096 RGB with 8 polygons: plain vs learned warm start."""
    torch = ws._torch()
    inst = synth.multi_4096(seed, size)
    g = torch.as_tensor(inst.source, device="cuda").contiguous()
    a = torch.as_tensor(inst.target, device="cuda").contiguous()
    m = torch.as_tensor(inst.mask, device="cuda").contiguous()
    ref, rref, _ = solve_image_device(ctx, g, a, m, tol=1e-10)
    up, rp, tp = solve_image_device(ctx, g, a, m, tol=tol)
    ws.guess_image(net, g, a, m, scale)  # warm-up: sizes the network's buffers for the pooled images
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    guess = ws.guess_image(net, g, a, m, scale)
    torch.cuda.synchronize()
    t_guess = time.perf_counter() - t0
    uw, rw, tw = solve_image_device(ctx, g, a, m, tol=tol, guess=guess)
    inter = ws.interior_mask(m[None])[0][..., None].expand_as(g)
    nin = float(inter.sum())

    def err(x):
        d = (x - ref) * inter
        return dict(max=float(d.abs().max()), rms=float(((d ** 2).sum() / nin).sqrt()))

    return dict(
        size=size, channels=3, scale=scale, tolerance=tol, interior_px=int(nin // 3),
        reference=dict(tolerance=1e-10, sweeps=[r["iterations"] for r in rref]),
        plain=dict(sweeps=[r["iterations"] for r in rp], omega=[r["omega_used"] for r in rp],
                   converged=all(r["converged"] for r in rp), solve_s=tp["wall_s"], kernel_ms=tp["kernel_ms"],
                   solves_per_s=1.0 / tp["wall_s"], error=err(up)),
        learned=dict(sweeps=[r["iterations"] for r in rw], converged=all(r["converged"] for r in rw),
                     guess_used=[r["warm_start"] for r in rw], guess_s=t_guess, solve_s=tw["wall_s"],
                     kernel_ms=tw["kernel_ms"], solves_per_s=1.0 / (t_guess + tw["wall_s"]), error=err(uw)),
        guess_error=err(guess), anchor_error=err(a))


def _init_ranks():
    """Under torchrun (WORLD_SIZE > 1): one NCCL rank per GPU; returns (rank, world, device)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world == 1:
        return 0, 1, 0
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    return dist.get_rank(), world, local


def cmd_train(args):
    torch = ws._torch()
    rank, world, dev = _init_ranks()
    os.makedirs(args.out, exist_ok=True)
    ctx = _lib.Context(dev)
    report = dict(config=dict(instances=args.instances, size=256, tol=1e-7, epochs=args.epochs, batch=64,
                              lr=1e-3, seed=args.seed, ranks=world))
    t0 = time.perf_counter()
    if world > 1:
        data = ws.build_dataset_sharded(ctx, n=args.instances, size=256, seed=args.seed, tol=1e-7)
    else:
        data = ws.build_dataset(ctx, n=args.instances, size=256, seed=args.seed, tol=1e-7)
    report["dataset"] = dict(gen_s=data.gen_s, solve_s=data.solve_s, wall_s=time.perf_counter() - t0,
                             solves_per_s=args.instances / world / max(data.solve_s, 1e-9),
                             sweeps_mean=float(data.sweeps.mean()), sweeps_max=int(data.sweeps.max()))
    if rank == 0:
        _log("dataset", report["dataset"])
    net = ws.UNet(ctx, seed=args.seed)
    if world > 1:
        tr = ws.DataParallelTrainer(net, data, batch=64, lr=1e-3, seed=args.seed)
    else:
        tr = ws.Trainer(net, data, batch=64, lr=1e-3, seed=args.seed)
    ckpt = os.path.join(args.out, "checkpoint.bin")
    if args.resume and os.path.exists(ckpt):
        tr.load(ckpt)
    total = args.epochs * (args.instances // 64)
    losses = []
    t0 = time.perf_counter()
    while tr.steps < total:
        losses.append(tr.step())
        if rank == 0 and tr.steps % 100 == 0:
            _log(f"epoch {tr.epoch} step {tr.steps} loss {np.mean(losses[-100:]):.4e}")
        if args.checkpoint_every and tr.steps % args.checkpoint_every == 0:
            tr.save(ckpt)
    wall = time.perf_counter() - t0
    tr.save(ckpt)
    if rank != 0:
        import torch.distributed as dist
        dist.barrier()  # rank 0 evaluates and writes the report
        dist.destroy_process_group()
        ctx.close()
        return
    ws.save_params(net, os.path.join(args.out, "warmstart_unet.params"))
    flops = ws.train_flops_per_pixel() * 64 * 256 * 256
    report["train"] = dict(
        steps=len(losses), wall_s=wall, step_ms=1e3 * tr.step_s / max(1, len(losses)),
        tflops=flops * len(losses) / tr.step_s / 1e12, flops_per_step=flops,
        samples_per_s=64 * len(losses) / tr.step_s,
        loss_first=float(losses[0]) if losses else None,
        loss_last100=float(np.mean(losses[-100:])) if losses else None,
        loss_curve=[float(np.mean(losses[k:k + 100])) for k in range(0, len(losses), 100)])
    _log("train", {k: v for k, v in report["train"].items() if k != "loss_curve"})
    report["eval256"] = evaluate_256(ctx, net)
    _log("eval256", report["eval256"])
    with open(os.path.join(args.out, "report.json"), "w") as f:
        json.dump(report, f, indent=1)
    del data
    torch.cuda.empty_cache()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()


def _net_from(ctx, path):
    net = ws.UNet(ctx, seed=0)
    ws.load_params(net, path)
    return net


def cmd_eval256(args):
    ctx = _lib.Context(0)
    out = evaluate_256(ctx, _net_from(ctx, args.params), n=args.instances)
    print(json.dumps(out))
    ctx.close()


def cmd_multi4096(args):
    ctx = _lib.Context(0)
    out = evaluate_multi4096(ctx, _net_from(ctx, args.params), seed=args.seed, scale=args.scale)
    print(json.dumps(out))
    ctx.close()


def cmd_steps(args):
    """Training steps on seeded instances without solving them (the target is
    the anchor's correction): a fixed workload for timing and profiling."""
    torch = ws._torch()
    ctx = _lib.Context(0)
    net = ws.UNet(ctx, seed=0)
    g, a, m = ws.make_instances(args.batch, args.size, seed=3)
    f = net.features(g, a, m)
    lm = ws.interior_mask(m)
    t = (a - g).contiguous()
    for _ in range(args.warmup):
        net.train_step(f, t, lm, 1e-3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        net.train_step(f, t, lm, 1e-3)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    flops = ws.train_flops_per_pixel() * args.batch * args.size * args.size
    print(json.dumps(dict(batch=args.batch, size=args.size, steps=args.steps, step_ms=dt * 1e3,
                          tflops=flops / dt / 1e12)))
    ctx.close()


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m paintop_b200.train_warmstart")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--instances", type=int, default=20000)
    t.add_argument("--epochs", type=int, default=8)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--out", required=True)
    t.add_argument("--checkpoint-every", type=int, default=0)
    t.add_argument("--resume", action="store_true")
    e = sub.add_parser("eval256")
    e.add_argument("--params", required=True)
    e.add_argument("--instances", type=int, default=256)
    c = sub.add_parser("multi4096")
    c.add_argument("--params", required=True)
    c.add_argument("--scale", type=int, default=8)
    c.add_argument("--seed", type=int, default=1)
    p = sub.add_parser("steps")
    p.add_argument("--batch", type=int, default=64)
    p.add_argument("--size", type=int, default=256)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args(argv)
    {"train": cmd_train, "eval256": cmd_eval256, "multi4096": cmd_multi4096, "steps": cmd_steps}[args.cmd](args)


if __name__ == "__main__":
    main()
