#!/usr/bin/env python
"""Benchmark: Poisson solves/s at relative residual 1e-6 on the screened 2048^2 workload,
plus the learned warm start against the plain solve on 4096^2 RGB inputs.

Workload (one "step" = one solve): 2048x2048 RGBA f32 screened-Poisson,
lambda = 0.01, a random 12-vertex star mask covering 30% (+-2%), relative
residual 1e-6, at most 2000 sweeps per channel, omega 1.8 (the op's fixed SOR
factor). Inputs come from the seeded generator in paintop_b200/synth.py.

Arms:
  default            the cuda backend. `value`: solves/s with inputs resident in
                     HBM (device pointers); `e2e`: solves/s through the C ABI with
                     pinned host buffers, host<->device copies inside the timed
                     region.
  multigrid          (N=1) the same inputs through multigrid-preconditioned CG
                     (PT_FLAG_MULTIGRID, ``multigrid_leg``).
  learned_warm_start (N=1) solves/s of U-Net guess + SOR vs plain SOR on the
                     same 4096x4096 RGB, 8-polygon inputs, and of multigrid
                     with and without the guess (``learned_leg``).
  --workload masks   the 4096x4096 workload's 8 polygon masks (``mask_arm``).
  --workload multigrid  the 4096x4096 RGB, 8-polygon solve by multigrid-CG
                     (``multigrid_arm``).
  --workload train    the learned warm start's U-Net training step, batch 64 of
                     256x256 (``train_arm``).
  --workload clone_512  the reference's CPU-runnable 512x512 RGB clone, seeds
                     1-5, beside the restated op on one core (``clone_arm``).
  batch_uneven       (N=1) the 256-instance uneven RGB batch, red-black SOR in one
                     persistent launch and multigrid-CG with every instance in each
                     launch (``batch_leg``), tile configuration from the table.
  train              (N=1) one U-Net training step, batch 64 of 256x256
                     (``train_leg``).
  clone_512          (N=1) the reference's CPU-runnable 512x512 RGB clone,
                     seeds 1-5, SOR and multigrid (``clone_leg``).
  parity             (N=1, CPU baseline leg) max |err| and RMS of the GPU results
                     against the FP64 tight oracle and the restated reference op.
  mask_raster        (N=1) the workloads' polygon masks rasterised on the device
                     (mask.polygon@1 semantics, ``mask_leg``) beside the
                     oracle's single-core rasteriser.
  --impl reference   the reference op's CPU algorithm (the oracle restatement of
                     crates/paintop-cpu/src/poisson.rs) on the host cores, one
                     channel solve per step as a bounded sample.

Multi-GPU (torchrun, one rank per GPU): every rank solves its own instance
(weak scaling, no data-path collective); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(name="screened_2048", width=2048, height=2048, channels=4, lam=0.01,
                tolerance=1e-6, max_iterations=2000, omega=1.8)
METRIC = "Poisson solves/s @ rel-res 1e-6 (screened 2048x2048 RGBA, lambda 0.01, star 30%)"
UNIT = "solves/s"

# algorithmic bytes per interior unknown per channel: one red+black sweep reads
# u, b' and the cell flag and writes u (13 B); one FP64 residual evaluation
# reads u, b' and the cell flag (9 B)
BYTES_PER_SWEEP = 13
BYTES_PER_RESIDUAL = 9


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_traffic():
    """DRAM bytes per k_solve launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "k_solve_screened_2048.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region. NVML is
    polled from a thread every 2 ms (reads only; nothing is set), so even a
    timed region of tens of milliseconds gets a few dozen samples; without
    NVML, nvidia-smi is sampled every 50 ms."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.nvml = None
        self.samples = []   # (sm MHz, max MHz, set of reasons)
        self.lines = []

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self.nvml = (pynvml, h, bits, mx)
            self._stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        # wait for the first sample, then count only samples taken from here on
        t0 = time.time()
        while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.mark = len(self.lines)

    def _poll(self):
        pynvml, h, bits, mx = self.nvml
        while not self._stop.is_set():
            try:
                sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), {n for n, b in bits.items() if rs & b}))
            except Exception:
                pass
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self._stop.set()
            self.thread.join(timeout=2)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
            samples, source = self.samples, "nvml, 2 ms"
        elif self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)
            samples, source = [], "nvidia-smi, 50 ms"
            for ln in self.lines[getattr(self, "mark", 0):] or self.lines[-1:]:
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    samples.append((float(parts[1]), float(parts[2]),
                                    {n for n, v in zip(self.NAMES, parts[5:9]) if v.lower() == "active"}))
                except ValueError:
                    continue
        else:
            return None
        if not samples:
            return None
        reasons = set().union(*(r for _, _, r in samples))
        return {"sm_mhz": statistics.median(x for x, _, _ in samples), "sm_max_mhz": samples[-1][1],
                "reasons": sorted(reasons), "samples": len(samples), "source": source}


def make_instance(seed: int):
    from paintop_b200 import synth
    return synth.screened_2048(seed)


def workload_config(inst, n_gpus: int) -> dict:
    """The workload's `config`, the same dict on both arms."""
    return {"workload": WORKLOAD["name"], "width": inst.width, "height": inst.height,
            "channels": inst.channels, "lambda": WORKLOAD["lam"], "tolerance": WORKLOAD["tolerance"],
            "max_iterations": WORKLOAD["max_iterations"], "omega": WORKLOAD["omega"],
            "interior_px": int((inst.mask[1:-1, 1:-1] > 0.5).sum()),
            "l2": "inputs larger than L2 (151 MB/solve)",
            "parallelism": f"instances sharded over {n_gpus} GPU(s)"}


def reference_arm(args):
    """CPU arm: the oracle restatement of the reference op, single thread (the
    reference solves channels one after another, poisson_blend.rs:168-236, and
    its FullDomain op is not tiled). One step is one channel solve of the
    workload (channels rotate); a solve costs the sum of its channel solves, so
    solves/s = 1 / (channels x mean step time)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.build()
    inst = make_instance(1)
    W, H, C = inst.width, inst.height, inst.channels
    src = inst.source.reshape(-1)
    tgt = inst.target.reshape(-1)
    mask = inst.mask.reshape(-1)
    chans = [np.ascontiguousarray(x.reshape(H, W, C)[:, :, k]).reshape(-1)
             for x in (src, tgt) for k in range(C)]
    srcs, tgts = chans[:C], chans[C:]
    sweeps, converged = {}, {}

    def step(k):
        c = k % C
        t0 = time.perf_counter()
        _, worst, per = O.blend_channels(srcs[c], tgts[c], mask, 1, W, H, WORKLOAD["max_iterations"],
                                         WORKLOAD["tolerance"], WORKLOAD["lam"], WORKLOAD["omega"])
        dt = time.perf_counter() - t0
        sweeps[c], converged[c] = int(per[0].iterations), bool(worst.converged)
        return dt

    for k in range(args.warmup):
        step(k)
    times = [step(args.warmup + k) for k in range(args.steps)]
    per_channel = float(np.mean(times))
    value = 1.0 / (C * per_channel)
    sample = (f"one channel of the {W}x{H}x{C} solve per step (channels rotate); "
              f"solves/s = 1 / ({C} x mean step time)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_channel * 1e3,
        "step": f"one channel solve; one {UNIT[:-2]} = {C} channel solves",
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded sinusoid-plus-noise images, star polygon mask)",
        "config": workload_config(inst, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "solver": {"sweeps_per_channel": [sweeps.get(c) for c in range(C)],
                   "channels_solved": sorted(converged), "converged": all(converged.values())},
    }
    print(json.dumps(line), flush=True)
    return 0


# the reference's bounded tier (crates/paintop-testkit/src/differential.rs:58-62)
BOUNDED_MAX_ABS, BOUNDED_RMS = 1e-4, 1e-5


def error_stats(got, want) -> dict:
    """max |got - want| and the RMS over all samples (the reference's ErrorMap)."""
    d = np.asarray(got, dtype=np.float64).reshape(-1) - np.asarray(want, dtype=np.float64).reshape(-1)
    mx, rms = float(np.abs(d).max()), float(np.sqrt(np.mean(d * d)))
    return {"max_abs": mx, "rms": rms, "within_bounded_tier": mx <= BOUNDED_MAX_ABS and rms <= BOUNDED_RMS}


def tight_oracle(inst, lam: float):
    """The FP64 tight oracle on the host cores: multigrid-preconditioned CG to
    relative residual 1e-12 (oracle/mgcg_ref.c, all threads OpenMP gives it)."""
    from oracle import oracle as O
    O.build()
    t0 = time.perf_counter()
    tight, ach, its = O.mgcg_blend_channels(inst.source.reshape(-1), inst.target.reshape(-1),
                                            inst.mask.reshape(-1), inst.channels, inst.width,
                                            inst.height, lam=lam, rel_tol=1e-12)
    return tight, {"method": "FP64 multigrid-preconditioned CG", "rel_res": [float(x) for x in ach],
                   "iterations": [int(x) for x in its], "seconds": time.perf_counter() - t0,
                   "threads": os.cpu_count()}


def cpu_baseline_sample(inst, gpu_out=None, gpu_outs=None):
    """CPU baseline leg: time one full solve (all channels) of the restated
    reference op on one host core. With the GPU's output of the same inputs it
    also states the GPU's error against that CPU output and against the FP64
    tight oracle, and the CPU op's own error against the oracle.
    gpu_outs: further GPU outputs of the same inputs, by name."""
    from oracle import oracle as O
    O.build()
    W, H, C = inst.width, inst.height, inst.channels
    t0 = time.perf_counter()
    ref, worst, per = O.blend_channels(inst.source.reshape(-1), inst.target.reshape(-1),
                                       inst.mask.reshape(-1), C, W, H, WORKLOAD["max_iterations"],
                                       WORKLOAD["tolerance"], WORKLOAD["lam"], WORKLOAD["omega"])
    dt = time.perf_counter() - t0
    cpu = {"value": 1.0 / dt, "unit": UNIT, "cores": 1, "kind": "port",
           "sample": f"one full {W}x{H}x{C} solve ({dt:.1f} s) of the restated reference op",
           "converged": bool(worst.converged), "sweeps": [int(r.iterations) for r in per]}
    if gpu_out is None:
        return cpu, None
    tight, info = tight_oracle(inst, WORKLOAD["lam"])
    parity = {"bounded_tier": {"max_abs": BOUNDED_MAX_ABS, "rms": BOUNDED_RMS,
                               "source": "crates/paintop-testkit/src/differential.rs:58-62"},
              "oracle": info,
              "cpu_op_vs_oracle": error_stats(ref, tight),
              "sor_vs_oracle": error_stats(gpu_out, tight),
              "sor_vs_cpu_op": error_stats(gpu_out, ref)}
    for name, out in (gpu_outs or {}).items():
        parity[f"{name}_vs_oracle"] = error_stats(out, tight)
        parity[f"{name}_vs_cpu_op"] = error_stats(out, ref)
    return cpu, parity


def mask_leg(ctx, dev, peak_gbs, reps: int = 20):
    """Device rasterisation (pt_mask_polygon, device pointers) of the workloads'
    masks: the 12-vertex star of the 2048x2048 screened solve and the 8 polygons
    of the 4096x4096 learned-warm-start workload (one launch per polygon into
    its own plane). CUDA events over `reps` repetitions after 3 warm-ups; the
    output planes (16.8 MB / 537 MB) are written anew each repetition."""
    import torch
    from paintop_b200 import masks, synth
    st = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    out = {}
    for name, inst in (("star_2048", synth.screened_2048(1)), ("polygons8_4096", synth.multi_4096(1))):
        W, H = inst.width, inst.height
        planes = torch.empty((len(inst.polygons), H, W), dtype=torch.float32, device=dev)

        def run():
            for k, pts in enumerate(inst.polygons):
                masks.polygon(ctx, W, H, pts, out=planes[k])
        for _ in range(3):
            run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            run()
        e1.record(st)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        px = len(inst.polygons) * W * H
        gbs = 4.0 * px / t / 1e9
        # the union of the planes is the workload's mask up to the generator's
        # own (non-fused) crossing arithmetic: report the share of pixels that agree
        union = planes.amax(0).cpu().numpy()
        out[name] = {"extent": [W, H], "polygons": len(inst.polygons),
                     "vertices": [len(p) for p in inst.polygons], "us_per_mask": t * 1e6,
                     "mpx_per_s": px / t / 1e6, "write_gbs": gbs, "write_frac_of_hbm": gbs / peak_gbs,
                     "agree_with_workload_mask": float((union == inst.mask).mean())}
        del planes
    return out


def mask_arm(args):
    """Mask workload: the 8 polygon masks of the 4096x4096 learned-warm-start
    workload rasterised with mask.polygon@1 semantics, one pt_mask_polygon call
    per polygon into its own 4096x4096 plane (537 MB per step, larger than L2).
    A step = the 8 masks. `value`: pixels/s with the planes in HBM (device
    pointers); `e2e`: the same calls writing pinned host buffers. Every rank
    rasterises its own 8 (weak scaling)."""
    import ctypes as Ct
    import torch
    from paintop_b200 import _lib, synth
    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", local if ws > 1 else 0)
    L = _lib.lib()
    ctx = _lib.Context(dev.index)
    inst = synth.multi_4096(1)
    W, H, P = inst.width, inst.height, len(inst.polygons)
    pts = [np.ascontiguousarray(np.asarray(p, dtype=np.float64)) for p in inst.polygons]
    planes = torch.empty((P, H, W), dtype=torch.float32, device=dev)
    host = torch.empty((P, H, W), dtype=torch.float32).pin_memory()
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    def step(device_out):
        kms = 0.0
        for k in range(P):
            dst = planes[k] if device_out else host[k]
            st = L.pt_mask_polygon(ctx.h, W, H, pts[k].ctypes.data_as(Ct.c_void_p), pts[k].shape[0],
                                   _lib.PT_FILL_NONZERO, dst.data_ptr(),
                                   _lib.PT_FLAG_DEVICE_POINTERS if device_out else 0)
            if st != _lib.PT_OK:
                raise _lib.CudaError(st, ctx.last_error())
            kms += ctx.last_timing()[0]
        return kms

    def timed(device_out):
        for _ in range(args.warmup):
            step(device_out)
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        kms = []
        a.record(stream)
        for _ in range(args.steps):
            kms.append(step(device_out))
        b.record(stream)
        b.synchronize()
        el = a.elapsed_time(b) / 1e3
        if ws > 1:
            import torch.distributed as dist
            t = torch.tensor([el], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        return el, kms

    sampler = ClockSampler(dev.index)
    sampler.start()
    elapsed, kms = timed(True)
    clocks = sampler.stop()
    e2e_elapsed, _ = timed(False)
    px = P * W * H
    peak, peak_kind = _peaks()
    kernel_s = float(np.mean(kms)) / 1e3 / P        # one launch = one 4096x4096 plane
    achieved = 4.0 * W * H / kernel_s / 1e9
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            from oracle import oracle as O
            t0 = time.perf_counter()
            O.mask_polygon(W, H, inst.polygons[0])
            dt = time.perf_counter() - t0
            cpu = {"value": W * H / dt, "unit": "px/s", "cores": 1, "kind": "port",
                   "sample": f"polygon 0 of 8 on its 4096x4096 plane ({dt:.1f} s), the oracle's rasterize()"}
        line = {
            "metric": "mask.polygon px/s (8 polygons of 8-13 vertices, 4096x4096 planes)",
            "value": ws * px * args.steps / elapsed, "unit": "px/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded polygons)",
            "config": {"workload": "polygons8_4096", "width": W, "height": H, "polygons": P,
                       "vertices": [len(p) for p in inst.polygons], "subsamples": 16,
                       "l2": "output planes larger than L2 (537 MB per step)"},
            "e2e": {"value": ws * px * args.steps / e2e_elapsed, "unit": "px/s", "h2d_bytes_per_step":
                    int(sum(p.nbytes for p in pts)), "d2h_bytes_per_step": 4 * px},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "kernel": "k_mask_polygon",
                         "peak_kind": peak_kind, "kernel_us_mean": kernel_s * 1e6,
                         "algorithmic_bytes_per_launch": 4 * W * H},
            "cpu_baseline": cpu, "gpu_launches": P * args.steps, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def multigrid_arm(args):
    """Multigrid workload: the 4096x4096 RGB, 8-polygon problem (tolerance 1e-6,
    lambda 0) solved by multigrid-preconditioned CG (PT_FLAG_MULTIGRID). A step =
    one solve. `value`: solves/s with inputs in HBM; `e2e`: through the C ABI
    with pinned host buffers. Every rank solves its own copy (weak scaling)."""
    import ctypes as Ct
    import torch
    from paintop_b200 import _lib, synth
    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", local if ws > 1 else 0)
    L = _lib.lib()
    ctx = _lib.Context(dev.index)
    inst = synth.multi_4096(1)
    W, H, C = inst.width, inst.height, inst.channels
    hs = torch.from_numpy(inst.source.reshape(-1)).pin_memory()
    ht = torch.from_numpy(inst.target.reshape(-1)).pin_memory()
    hm = torch.from_numpy(inst.mask.reshape(-1)).pin_memory()
    ho = torch.empty_like(hs).pin_memory()
    g, a, m = hs.to(dev), ht.to(dev), hm.to(dev)
    out = torch.empty_like(g)
    reps = (_lib.PtReport * (C + 1))()
    flags = _lib.PT_FLAG_MULTIGRID
    p_dev = _lib.PtProblem(W, H, C, g.data_ptr(), a.data_ptr(), m.data_ptr(), 0.0, 100000, 1e-6, 1.8,
                           flags | _lib.PT_FLAG_DEVICE_POINTERS, None)
    p_host = _lib.PtProblem(W, H, C, hs.data_ptr(), ht.data_ptr(), hm.data_ptr(), 0.0, 100000, 1e-6, 1.8, flags,
                            None)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    def solve(device):
        st = L.pt_poisson_solve(ctx.h, Ct.byref(p_dev if device else p_host),
                                (out if device else ho).data_ptr(), reps, None)
        if st != _lib.PT_OK:
            raise _lib.CudaError(st, ctx.last_error())
        return ctx.last_timing()

    def timed(device):
        for _ in range(args.warmup):
            solve(device)
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        info = []
        e0.record(stream)
        for _ in range(args.steps):
            info.append(solve(device))
        e1.record(stream)
        e1.synchronize()
        el = e0.elapsed_time(e1) / 1e3
        if ws > 1:
            import torch.distributed as dist
            t = torch.tensor([el], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        return el, info

    sampler = ClockSampler(dev.index)
    sampler.start()
    elapsed, info = timed(True)
    clocks = sampler.stop()
    e2e_elapsed, _ = timed(False)
    its = [int(reps[c].iterations) for c in range(C)]
    interior = int((inst.mask[1:-1, 1:-1] > 0.5).sum())
    # Modelled bytes of one CG iteration per level-0 cell and channel, as the
    # kernels move them: 8 red-black half-sweeps (rhs 2 B, e 4 + 2 B, mask 1 B
    # each), residual 13, restriction 4, prolongation 9, zeroing 4, r.z 8,
    # direction 12, operator 9, update 24 -> 155 B; coarser levels add a third.
    cells = W * H * C
    bytes_per_iter = 155.0 * cells * 4.0 / 3.0
    solve_s = float(np.mean([t[0] for t in info])) / 1e3  # the iterative part (CUDA events)
    achieved = bytes_per_iter * float(np.mean(its)) / solve_s / 1e9
    peak, peak_kind = _peaks()
    if rank == 0:
        line = {
            "metric": "multigrid-CG solves/s @ rel-res 1e-6 (4096x4096 RGB, 8 polygons)",
            "value": ws * args.steps / elapsed, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 residual and refinement)",
            "data": "synthetic (seeded sinusoid-plus-noise images, 8 random polygons)",
            "config": {"workload": "multi_4096_multigrid", "width": W, "height": H, "channels": C, "lambda": 0.0,
                       "tolerance": 1e-6, "interior_px": interior,
                       "l2": "inputs larger than L2 (201 MB per solve)"},
            "e2e": {"value": ws * args.steps / e2e_elapsed, "unit": "solves/s",
                    "h2d_bytes_per_step": 4 * (2 * W * H * C + W * H),
                    "d2h_bytes_per_step": 4 * W * H * C + 64 * (C + 1)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "kernel": "multigrid-CG iteration (all kernels)",
                         "peak_kind": peak_kind, "modelled_bytes_per_iteration": bytes_per_iter,
                         "iterative_part_ms": solve_s * 1e3},
            "cpu_baseline": None, "gpu_launches": int(sum(t[2] for t in info)), "clocks": clocks,
            "solver": {"cg_iterations": its, "refinements": [int(reps[c].refinements) for c in range(C)],
                       "converged": all(reps[c].converged for c in range(C)),
                       "worst_final_residual": max(reps[c].final_residual for c in range(C))},
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def clone_arm(args):
    """Seamless clone, the reference's CPU-runnable configuration: 512x512 RGB,
    ellipse 150 x 110, SOR omega 1.9, relative residual 1e-5, at most 5000
    sweeps, seeds 1-5 (one per step, cycling). Inputs (7 MB) fit in L2, so a
    256 MB buffer is written between steps and each solve is timed alone with
    CUDA events. `e2e` goes through the C ABI with pinned host buffers. The
    CPU baseline is the restated reference op on one core at omega 1.9 (the
    configuration) and at the op's fixed 1.8, on every seed."""
    import ctypes as Ct
    import torch
    from paintop_b200 import _lib, synth
    ws, rank, local = _dist()
    if rank != 0:
        return 0
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    L = _lib.lib()
    ctx = _lib.Context(0)
    seeds = [1, 2, 3, 4, 5]
    insts = [synth.clone_512(sd) for sd in seeds]
    W, H, C = 512, 512, 3
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    bufs = []
    for inst in insts:
        hs = [torch.from_numpy(x.reshape(-1)).pin_memory() for x in (inst.source, inst.target, inst.mask)]
        ds = [h.to(dev) for h in hs]
        bufs.append((hs, ds, torch.empty(W * H * C, device=dev), torch.empty(W * H * C).pin_memory()))
    reps = (_lib.PtReport * (C + 1))()

    def solve(k, device):
        hs, ds, od, oh = bufs[k % len(bufs)]
        src = ds if device else hs
        p = _lib.PtProblem(W, H, C, src[0].data_ptr(), src[1].data_ptr(), src[2].data_ptr(), 0.0, 5000, 1e-5, 1.9,
                           _lib.PT_FLAG_DEVICE_POINTERS if device else 0, None)
        st = L.pt_poisson_solve(ctx.h, Ct.byref(p), (od if device else oh).data_ptr(), reps, None)
        if st != _lib.PT_OK:
            raise _lib.CudaError(st, ctx.last_error())
        return [int(reps[c].iterations) for c in range(C)], all(reps[c].converged for c in range(C))

    def timed(device):
        for k in range(args.warmup):
            solve(k, device)
        total, its = 0.0, []
        for k in range(args.steps):
            flush.fill_(float(k))  # evict the previous step's data from L2
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            its.append(solve(k, device))
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1) / 1e3
        return total, its

    sampler = ClockSampler(0)
    sampler.start()
    elapsed, its = timed(True)
    clocks = sampler.stop()
    e2e_elapsed, _ = timed(False)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        t19, t18, it19 = [], [], []
        for inst in insts:
            for omega, acc in ((1.9, t19), (1.8, t18)):
                t0 = time.perf_counter()
                _, worst, _ = O.blend_channels(inst.source.reshape(-1), inst.target.reshape(-1),
                                               inst.mask.reshape(-1), C, W, H, 5000, 1e-5, 0.0, omega)
                acc.append(time.perf_counter() - t0)
                if omega == 1.9:
                    it19.append(int(worst.iterations))
        cpu = {"value": 1.0 / float(np.mean(t19)), "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": f"full solves of seeds 1-5 at omega 1.9 (mean {np.mean(t19):.2f} s, worst-channel sweeps "
                         f"{it19}); the op's omega 1.8: {1.0 / float(np.mean(t18)):.3f} solves/s"}
    line = {
        "metric": "Poisson solves/s @ rel-res 1e-5 (clone 512x512 RGB, ellipse 150x110, omega 1.9)",
        "value": args.steps / elapsed, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded sinusoid-plus-noise images, ellipse mask)",
        "config": {"workload": "clone_512", "width": W, "height": H, "channels": C, "lambda": 0.0, "tolerance": 1e-5,
                   "max_iterations": 5000, "omega": 1.9, "seeds": seeds,
                   "l2": "inputs fit in L2: 256 MB written between steps, each solve timed alone"},
        "e2e": {"value": args.steps / e2e_elapsed, "unit": "solves/s", "h2d_bytes_per_step": 4 * (2 * W * H * C + W * H),
                "d2h_bytes_per_step": 4 * W * H * C + 64 * (C + 1)},
        "roofline": None, "cpu_baseline": cpu, "gpu_launches": int(ctx.last_timing()[2]) * args.steps,
        "clocks": clocks, "solver": {"sweeps_per_channel": its[-1][0], "converged": all(c for _, c in its)},
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def train_arm(args):
    """U-Net training step of the learned warm start: batch 64 of 256x256
    single-channel instances (seeded, device-generated; the target is the
    anchor's correction), forward + backward + Adam through pt_unet_train_step.
    A step = one training step. `value`: samples/s; the roofline is the bf16
    tensor peak against the convolutions' algorithmic FLOPs. Every rank trains
    its own replica on its own batch (weak scaling; the data-parallel
    exchange is timed by the trainer, not here)."""
    import ctypes as Ct
    import torch
    from paintop_b200 import _lib, warmstart as wsm
    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", local if ws > 1 else 0)
    ctx = _lib.Context(dev.index)
    B, S = 64, 256
    net = wsm.UNet(ctx, seed=rank)
    g, a, m = wsm.make_instances(B, S, seed=3 + rank)
    f = net.features(g, a, m)
    lm = wsm.interior_mask(m)
    t = (a - g).contiguous()
    L = _lib.lib()
    loss = Ct.c_double()

    def step():
        st = L.pt_unet_train_step(net.h, f.data_ptr(), t.data_ptr(), lm.data_ptr(), B, S, S, Ct.c_float(1e-3),
                                  Ct.byref(loss))
        if st != _lib.PT_OK:
            raise _lib.CudaError(st, ctx.last_error())

    for _ in range(args.warmup):
        step()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize(dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    sampler = ClockSampler(dev.index)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    clocks = sampler.stop()
    el = e0.elapsed_time(e1) / 1e3
    if ws > 1:
        import torch.distributed as dist
        tt = torch.tensor([el], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        el = float(tt.item())
    flops = wsm.train_flops_per_pixel() * B * S * S
    step_s = el / args.steps
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        with open(pk_path) as fh:
            pk = json.load(fh)
        peak = float(pk.get("bf16_tflops_sustained", pk.get("bf16_tflops")))
        peak_kind = "measured (sustained: a step loop lasts seconds)"
    else:
        peak, peak_kind = 1400.0, "fallback (sustained bf16 figure of earlier measurements on this hardware)"
    achieved = flops / step_s / 1e12
    if rank == 0:
        line = {
            "metric": "U-Net training samples/s (batch 64, 256x256, bf16 weights, fp32 accumulate, Adam)",
            "value": ws * B * args.steps / el, "unit": "samples/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16", "data": "synthetic (seeded sinusoid-plus-noise instances)",
            "config": {"workload": "unet_train_b64_256", "batch": B, "size": S,
                       "model": "U-Net 16-32-64-128, 3x3 convs, 14 layers", "flops_per_step": flops,
                       "l2": "one 16-channel level-0 activation is 134 MB, larger than L2"},
            "e2e": None,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None, "kernel": "whole training step",
                         "peak_kind": peak_kind},
            "cpu_baseline": None, "gpu_launches": None, "clocks": clocks, "loss_last": loss.value,
        }
        print(json.dumps(line), flush=True)
    net.close()
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def mask_cpu_baseline():
    """The oracle's mask.polygon (the reference's rasterize(), one host core) on
    the 2048x2048 star."""
    from oracle import oracle as O
    from paintop_b200 import synth
    inst = synth.screened_2048(1)
    t0 = time.perf_counter()
    O.mask_polygon(inst.width, inst.height, inst.polygons[0])
    dt = time.perf_counter() - t0
    return {"mpx_per_s": inst.width * inst.height / dt / 1e6, "cores": 1, "kind": "port",
            "sample": f"one 2048x2048 star mask ({dt:.2f} s)"}


def gpu_arm(args):
    import torch
    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", local if ws > 1 else 0)
    from paintop_b200 import _lib
    ctx = _lib.Context(dev.index)
    if args.tile_config >= 0:
        ctx.set_config(args.tile_config)

    inst = make_instance(1 + rank)
    W, H, C = inst.width, inst.height, inst.channels
    n_img, n_mask = W * H * C, W * H
    src_h = torch.from_numpy(inst.source.reshape(-1)).pin_memory()
    tgt_h = torch.from_numpy(inst.target.reshape(-1)).pin_memory()
    mask_h = torch.from_numpy(inst.mask.reshape(-1)).pin_memory()
    out_h = torch.empty(n_img, dtype=torch.float32).pin_memory()
    src_d, tgt_d, mask_d = src_h.to(dev), tgt_h.to(dev), mask_h.to(dev)
    out_d = torch.empty(n_img, dtype=torch.float32, device=dev)
    hist_cap = WORKLOAD["max_iterations"]
    hist_d = torch.empty(C * hist_cap, dtype=torch.float64, device=dev)
    hist_h = torch.empty(C * hist_cap, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    interior = int((inst.mask[1:-1, 1:-1] > 0.5).sum())

    import ctypes as Ct
    L = _lib.lib()
    reps = (_lib.PtReport * (C + 1))()

    def problem(device_ptrs: bool):
        s, t, m = (src_d, tgt_d, mask_d) if device_ptrs else (src_h, tgt_h, mask_h)
        return _lib.PtProblem(W, H, C, s.data_ptr(), t.data_ptr(), m.data_ptr(),
                              WORKLOAD["lam"], WORKLOAD["max_iterations"], WORKLOAD["tolerance"],
                              WORKLOAD["omega"],
                              _lib.PT_FLAG_DEVICE_POINTERS if device_ptrs else 0, None)

    p_dev, p_host = problem(True), problem(False)

    def solve(device_ptrs: bool):
        if device_ptrs:
            st = L.pt_poisson_solve(ctx.h, Ct.byref(p_dev), out_d.data_ptr(), reps,
                                    hist_d.data_ptr())
        else:
            st = L.pt_poisson_solve(ctx.h, Ct.byref(p_host), out_h.data_ptr(), reps,
                                    hist_h.data_ptr())
        if st != _lib.PT_OK:
            raise _lib.CudaError(st, ctx.last_error())

    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident arm -------------------------------------------------
    for _ in range(args.warmup):
        solve(True)
    barrier()
    sampler = ClockSampler(dev.index)
    sampler.start()
    kernel_ms, iters, refines, launches = [], [], [], 0
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        solve(True)
        k, _, nl = ctx.last_timing()
        kernel_ms.append(k)
        launches += nl
        iters.append([reps[c].iterations for c in range(C)])
        refines.append([reps[c].refinements for c in range(C)])
    ev1.record(stream)
    ev1.synchronize()
    barrier()
    elapsed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    clocks = sampler.stop()
    converged = all(reps[c].converged for c in range(C))
    worst_res = max(reps[c].final_residual for c in range(C))
    head_cfg = ctx.last_config()  # the timed solves' tile configuration (later legs change it)
    sor_out = out_d.cpu().numpy()  # the last timed solve's result, for the parity statement

    # ---- end-to-end arm (pinned host buffers through the C ABI) --------------
    e2e_elapsed = float("nan")
    moved = None
    if not args.device_only:
        for _ in range(max(1, args.warmup)):
            solve(False)
        barrier()
        ev2 = torch.cuda.Event(enable_timing=True)
        ev3 = torch.cuda.Event(enable_timing=True)
        ev2.record(stream)
        for _ in range(args.steps):
            solve(False)
            launches += ctx.last_timing()[2]
        ev3.record(stream)
        ev3.synchronize()
        barrier()
        e2e_elapsed = max_over_ranks(ev2.elapsed_time(ev3) / 1e3)
        moved = ctx.last_transfer()  # the same every step: the bands depend on the mask only

    value = ws * args.steps / elapsed
    e2e_value = ws * args.steps / e2e_elapsed
    # bytes each step moves over PCIe, as the library counts them: masks, then
    # source and target only in the row bands the solve reads; the output's
    # bands with interior tiles, reports and history come back
    h2d, d2h = moved if moved else (4 * (2 * n_img + n_mask), 4 * n_img + 8 * C * hist_cap + 64 * (C + 1))

    # roofline for the persistent solve kernel
    it = np.array(iters, dtype=np.float64)       # steps x C sweeps
    rf = np.array(refines, dtype=np.float64)
    alg_bytes = interior * (BYTES_PER_SWEEP * it.sum(axis=1) +
                            BYTES_PER_RESIDUAL * (it.sum(axis=1) + rf.sum(axis=1)))
    kms = np.array(kernel_ms)
    achieved = float(np.mean(alg_bytes / (kms / 1e3)) / 1e9)
    peak, peak_kind = _peaks()
    traffic = _profile_traffic()

    learned = None
    if ws == 1 and not args.no_learned and not args.device_only:
        learned = learned_leg(ctx, dev, with_cpu=not args.no_cpu_baseline)  # reported apart, outside the timed region
    multigrid, mg_out = None, None
    if ws == 1 and not args.device_only:
        multigrid = multigrid_leg(ctx, dev, inst)
        mg_out = multigrid.pop("_out")
    mask_raster = None
    if ws == 1 and not args.device_only:
        mask_raster = mask_leg(ctx, dev, peak)
        if not args.no_cpu_baseline:
            mask_raster["cpu_baseline"] = mask_cpu_baseline()
    batch_uneven, train, clone = None, None, None
    if ws == 1 and not args.device_only:
        batch_uneven = batch_leg(ctx, dev)
        train = train_leg(ctx, dev)
        clone = clone_leg(ctx, dev, with_cpu=not args.no_cpu_baseline)

    line = None
    if rank == 0:
        cpu, parity = None, None
        if ws == 1 and not args.no_cpu_baseline and not args.device_only:
            cpu, parity = cpu_baseline_sample(
                inst, sor_out, {"multigrid": mg_out} if mg_out is not None else None)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded sinusoid-plus-noise images, star polygon mask)",
            "config": workload_config(inst, ws),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "inputs_bytes_per_step": 4 * (2 * n_img + n_mask),
                    "note": "pinned host buffers through pt_poisson_solve; the library uploads the masks, then "
                            "source and target only in the tile row bands holding interior cells, each band as "
                            "one rectangle (its span of interior tile columns, one pixel and one row either "
                            "side), and downloads only the bands' spans of the output; the rest of the output "
                            "is the target, copied on the host inside the call"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "dram_frac": (traffic / (float(kms.mean()) / 1e3) / 1e9 / peak) if traffic else None,
                         "frac_note": "frac: algorithmic bytes (temporal blocking reuses tiles in shared "
                                      "memory, so it can exceed 1); dram_frac: ncu DRAM bytes of the "
                                      "committed capture over this run's kernel time",
                         "kernel": "ptk::k_solve", "peak_kind": peak_kind,
                         "kernel_ms_mean": float(kms.mean()),
                         "algorithmic_bytes_per_launch": float(alg_bytes.mean())},
            "cpu_baseline": cpu,
            "parity": parity,
            "gpu_launches": launches,
            "clocks": clocks,
            "solver": {"iterations_per_channel": iters[-1], "refinements": refines[-1],
                       "converged": converged, "worst_final_residual": worst_res,
                       "tile_config": tile_config_label(head_cfg),
                       "tuned_entry": tuned_entry([dict(width=W, height=H, channels=C,
                                                        lam=WORKLOAD["lam"])])},
            "multigrid": multigrid,
            "learned_warm_start": learned,
            "mask_raster": mask_raster,
            "batch_uneven": batch_uneven,
            "train": train,
            "clone_512": clone,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def measure_batch(ctx, dev, insts, interior, steps: int, warmup: int, multigrid: bool,
                  sync=None, max_over_ranks=None, with_e2e: bool = True) -> dict:
    """Solve a batch of instances in one pt_poisson_solve_batch call per step:
    device-resident (`elapsed`) and through pinned host buffers (`e2e_elapsed`),
    CUDA events on the context stream. Returns the timings, reports and bytes."""
    import ctypes as Ct
    import torch
    from paintop_b200 import _lib
    n = len(insts)
    L = _lib.lib()
    keep = []
    probs_d = (_lib.PtProblem * n)()
    probs_h = (_lib.PtProblem * n)()
    outs_d = (Ct.c_void_p * n)()
    outs_h = (Ct.c_void_p * n)()
    rep_arr = [(_lib.PtReport * (i.channels + 1))() for i in insts]
    rep_ptrs = (Ct.POINTER(_lib.PtReport) * n)(*[Ct.cast(r, Ct.POINTER(_lib.PtReport)) for r in rep_arr])
    flags = _lib.PT_FLAG_MULTIGRID if multigrid else _lib.PT_FLAG_OMEGA_AUTO
    h2d = d2h = 0
    for k, inst in enumerate(insts):
        sh = torch.from_numpy(inst.source.reshape(-1)).pin_memory()
        th = torch.from_numpy(inst.target.reshape(-1)).pin_memory()
        mh = torch.from_numpy(inst.mask.reshape(-1)).pin_memory()
        oh = torch.empty_like(sh).pin_memory()
        sd, td, md = sh.to(dev), th.to(dev), mh.to(dev)
        od = torch.empty_like(sd)
        keep += [sh, th, mh, oh, sd, td, md, od]
        probs_d[k] = _lib.PtProblem(inst.width, inst.height, inst.channels, sd.data_ptr(),
                                    td.data_ptr(), md.data_ptr(), 0.0, 100000, 1e-6, 1.8,
                                    flags | _lib.PT_FLAG_DEVICE_POINTERS, None)
        probs_h[k] = _lib.PtProblem(inst.width, inst.height, inst.channels, sh.data_ptr(),
                                    th.data_ptr(), mh.data_ptr(), 0.0, 100000, 1e-6, 1.8, flags,
                                    None)
        outs_d[k], outs_h[k] = od.data_ptr(), oh.data_ptr()
        h2d += 4 * (sh.numel() + th.numel() + mh.numel())
        d2h += 4 * oh.numel() + 64 * (inst.channels + 1)
    torch.cuda.synchronize()

    def solve(device_ptrs):
        st = L.pt_poisson_solve_batch(ctx.h, probs_d if device_ptrs else probs_h, n,
                                      outs_d if device_ptrs else outs_h, rep_ptrs, None)
        if st != _lib.PT_OK:
            raise _lib.CudaError(st, ctx.last_error())

    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    def timed(device_ptrs):
        for _ in range(warmup):
            solve(device_ptrs)
        if sync:
            sync()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        kms, launches = [], 0
        a.record(stream)
        for _ in range(steps):
            solve(device_ptrs)
            kms.append(ctx.last_timing()[0])
            launches += ctx.last_timing()[2]
        b.record(stream)
        b.synchronize()
        el = a.elapsed_time(b) / 1e3
        return (max_over_ranks(el) if max_over_ranks else el), kms, launches

    sampler = ClockSampler(dev.index)
    sampler.start()
    elapsed, kms, launches = timed(True)
    clocks = sampler.stop()
    e2e_elapsed = timed(False)[0] if with_e2e else float("nan")
    iters = [[r[c].iterations for c in range(i.channels)] for r, i in zip(rep_arr, insts)]
    conv = all(r[c].converged for r, i in zip(rep_arr, insts) for c in range(i.channels))
    if multigrid:
        # the multigrid model: 155 B per level-0 cell and channel per CG
        # iteration, a third more for the coarser levels (multigrid_arm)
        alg = sum(155.0 * 4.0 / 3.0 * i.width * i.height * sum(it) for it, i in zip(iters, insts))
    else:
        alg = sum(n_int * (BYTES_PER_SWEEP * sum(it) + BYTES_PER_RESIDUAL * (
            sum(it) + sum(r[c].refinements for c in range(i.channels))))
            for n_int, it, r, i in zip(interior, iters, rep_arr, insts))
    return dict(elapsed=elapsed, e2e_elapsed=e2e_elapsed, kms=kms, launches=launches, clocks=clocks,
                iters=iters, conv=conv, alg=alg, h2d=h2d, d2h=d2h, reps=rep_arr,
                omegas=[float(r[0].omega_used) for r in rep_arr], config=ctx.last_config())


def tile_config_label(cfg: int):
    if cfg is None or cfg < 0:
        return None
    import ctypes as Ct
    from paintop_b200 import _lib
    s, w, h = Ct.c_int32(), Ct.c_int32(), Ct.c_int32()
    _lib.lib().pt_tile_config_info(cfg, Ct.byref(s), Ct.byref(w), Ct.byref(h))
    return {"index": cfg, "sweeps_per_step": s.value, "tile_w": w.value, "tile_h": h.value}


def tuned_entry(problems) -> dict:
    """The compiled-in B200 table's entry for these problems' shape key, if any
    (paintop_b200/csrc/tune_table_b200.inc, written by paintop_b200.tune)."""
    import re
    from paintop_b200 import tune
    key = tune.shape_key(problems)
    text = open(tune.INC).read()
    for k, v in re.findall(r"\{0x([0-9a-f]{8})u, (\d+)\}", text):
        if int(k, 16) == key:
            return {"key": f"0x{key:08x}", "config": int(v), "source": "compiled-in B200 table"}
    return {"key": f"0x{key:08x}", "config": None, "source": "built-in rule (no tuned entry)"}


def batch_cpu_sample(insts, rep_arr, multigrid: bool) -> dict:
    """CPU baseline leg of the batch: the restated reference op on one host core
    over 8 instances spread across the size range."""
    from oracle import oracle as O
    O.build()
    n = len(insts)
    order = sorted(range(n), key=lambda k: insts[k].width * insts[k].height)
    sample = order[::max(1, n // 8)][:8]
    t0 = time.perf_counter()
    for k in sample:
        i = insts[k]
        om = 1.8 if multigrid else float(rep_arr[k][0].omega_used)
        O.blend_channels(i.source.reshape(-1), i.target.reshape(-1), i.mask.reshape(-1),
                         i.channels, i.width, i.height, 100000, 1e-6, 0.0, om)
    dt = time.perf_counter() - t0
    return {"value": len(sample) / dt, "unit": "instances/s", "cores": 1, "kind": "port",
            "sample": f"{len(sample)} instances spread over the size range ({dt:.1f} s), "
                      + ("row-major SOR at the op's omega 1.8" if multigrid else
                         "row-major SOR at the omega the GPU chose")}


def batch_leg(ctx, dev, steps: int = 3, warmup: int = 1) -> dict:
    """The 256-instance uneven RGB batch in the default run (N=1): red-black
    SOR in one persistent launch per batch, and multigrid-CG with every instance
    in each launch, device-resident, CUDA events; tile configuration from the
    table."""
    from paintop_b200 import synth
    insts = synth.batch_uneven(1, 256)
    interior = [int((i.mask[1:-1, 1:-1] > 0.5).sum()) for i in insts]
    peak, peak_kind = _peaks()
    out = {"workload": "batch_uneven: 256 RGB instances, side log-uniform in [64, 1024], aspect [0.5, 2], "
                       "ellipse masks 20-60%, rel-res 1e-6", "steps": steps}
    probs = [dict(width=i.width, height=i.height, channels=i.channels, lam=0.0) for i in insts]
    for mg in (False, True):
        r = measure_batch(ctx, dev, insts, interior, steps, warmup, mg, with_e2e=False)
        kmean = float(np.mean(r["kms"]))
        out["multigrid" if mg else "sor"] = {
            "instances_per_s": len(insts) * steps / r["elapsed"], "ms_per_batch": r["elapsed"] / steps * 1e3,
            "converged": r["conv"], "max_iterations": int(max(max(x) for x in r["iters"])),
            "roofline": {"bound": "hbm", "achieved": r["alg"] / (kmean / 1e3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": r["alg"] / (kmean / 1e3) / 1e9 / peak,
                         "peak_kind": peak_kind,
                         "kernel": "multigrid-CG iteration (modelled bytes)" if mg else "ptk::k_solve"},
            "gpu_launches_per_batch": r["launches"] // max(1, steps), "clocks": r["clocks"],
            **({} if mg else {"tile_config": tile_config_label(r["config"]),
                              "tuned_entry": tuned_entry(probs)}),
        }
    out["speedup_multigrid"] = out["multigrid"]["instances_per_s"] / out["sor"]["instances_per_s"]
    return out


def clone_leg(ctx, dev, with_cpu: bool = True) -> dict:
    """The reference's CPU-runnable configuration in the default run (N=1):
    512x512 RGB seamless clone, ellipse 150 x 110, omega 1.9, rel-res 1e-5, at
    most 5000 sweeps, seeds 1-5, device buffers. The inputs fit in L2, so a
    256 MB buffer is written before each solve and each solve is timed alone
    (CUDA events on the context stream). Red-black SOR and multigrid-CG; the
    CPU baseline leg times the restated reference op on seed 1 at omega 1.9 and
    states each GPU result's error against the FP64 oracle and that CPU output."""
    import ctypes as Ct
    import torch
    from paintop_b200 import _lib, synth
    L = _lib.lib()
    W, H, C = 512, 512, 3
    insts = [synth.clone_512(sd) for sd in (1, 2, 3, 4, 5)]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    reps = (_lib.PtReport * (C + 1))()
    out = {"workload": "clone_512: 512x512 RGB, ellipse 150x110, omega 1.9, rel-res 1e-5, seeds 1-5",
           "l2": "inputs fit in L2: 256 MB written before each solve, each solve timed alone"}
    first = {}
    for name, flags in (("sor", 0), ("multigrid", _lib.PT_FLAG_MULTIGRID)):
        times, sweeps = [], []
        for k, inst in enumerate(insts):
            ds = [torch.as_tensor(x.reshape(-1), device=dev) for x in (inst.source, inst.target, inst.mask)]
            od = torch.empty(W * H * C, device=dev)
            p = _lib.PtProblem(W, H, C, ds[0].data_ptr(), ds[1].data_ptr(), ds[2].data_ptr(), 0.0, 5000, 1e-5, 1.9,
                               _lib.PT_FLAG_DEVICE_POINTERS | flags, None)
            for rep in range(2):  # the first solve of a seed warms up
                flush.fill_(float(rep))
                torch.cuda.synchronize(dev)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                st = L.pt_poisson_solve(ctx.h, Ct.byref(p), od.data_ptr(), reps, None)
                e1.record(stream)
                e1.synchronize()
                if st != _lib.PT_OK:
                    raise _lib.CudaError(st, ctx.last_error())
            times.append(e0.elapsed_time(e1))
            sweeps.append(max(int(reps[c].iterations) for c in range(C)))
            if k == 0:
                first[name] = od.cpu().numpy()
        out[name] = {"solves_per_s": 1e3 / float(np.mean(times)), "ms_per_solve": float(np.mean(times)),
                     "worst_channel_iterations": sweeps}
    if with_cpu:
        # CPU baseline leg: the restated reference op on one core, seed 1
        from oracle import oracle as O
        O.build()
        i0 = insts[0]
        t0 = time.perf_counter()
        ref, worst, _ = O.blend_channels(i0.source.reshape(-1), i0.target.reshape(-1), i0.mask.reshape(-1), C, W, H,
                                         5000, 1e-5, 0.0, 1.9)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "solves/s", "cores": 1, "kind": "port",
                               "sample": f"seed 1, omega 1.9 ({dt:.2f} s, worst-channel sweeps {worst.iterations})"}
        tight, info = tight_oracle(i0, 0.0)
        cpu_err = error_stats(ref, tight)
        gpu_err = {n: error_stats(v, tight) for n, v in first.items()}
        out["parity"] = {
            "oracle": info,
            "bar": "max error against the FP64 oracle at most twice the CPU op's own (tests/test_gpu_parity.py, "
                   "test_clone_512_against_oracles): at rel-res 1e-5 on pure Poisson the error is set by the "
                   "slowest mode for every method, the reference op's included, so the bounded tier is not the bar",
            "cpu_op_vs_oracle": cpu_err,
            **{f"{n}_vs_oracle": e for n, e in gpu_err.items()},
            **{f"{n}_vs_cpu_op": error_stats(v, ref) for n, v in first.items()},
            "within_bar": {n: e["max_abs"] <= 2.0 * cpu_err["max_abs"] for n, e in gpu_err.items()}}
    return out


def train_leg(ctx, dev, steps: int = 10, warmup: int = 3) -> dict:
    """One U-Net training step (batch 64 of 256x256, forward + backward + Adam)
    in the default run (N=1), CUDA events on the context stream."""
    import ctypes as Ct
    import torch
    from paintop_b200 import _lib, warmstart as wsm
    B, S = 64, 256
    net = wsm.UNet(ctx, seed=0)
    try:
        g, a, m = wsm.make_instances(B, S, seed=3)
        f = net.features(g, a, m)
        lm = wsm.interior_mask(m)
        t = (a - g).contiguous()
        loss = Ct.c_double()
        L = _lib.lib()

        def step():
            st = L.pt_unet_train_step(net.h, f.data_ptr(), t.data_ptr(), lm.data_ptr(), B, S, S,
                                      Ct.c_float(1e-3), Ct.byref(loss))
            if st != _lib.PT_OK:
                raise _lib.CudaError(st, ctx.last_error())

        for _ in range(warmup):
            step()
        torch.cuda.synchronize(dev)
        stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
        sampler = ClockSampler(dev.index)
        sampler.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        e1.synchronize()
        clocks = sampler.stop()
    finally:
        net.close()
    step_s = e0.elapsed_time(e1) / 1e3 / steps
    flops = wsm.train_flops_per_pixel() * B * S * S
    peak, peak_kind = _bf16_peak()
    return {"workload": "unet_train_b64_256: batch 64 of 256x256, bf16 weights, fp32 accumulate, Adam",
            "steps": steps, "samples_per_s": B / step_s, "ms_per_step": step_s * 1e3,
            "roofline": {"bound": "tensor", "achieved": flops / step_s / 1e12, "peak": peak,
                         "unit": "TFLOP/s", "frac": flops / step_s / 1e12 / peak, "peak_kind": peak_kind,
                         "kernel": "whole training step"},
            "loss_last": loss.value, "clocks": clocks}


def _bf16_peak():
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        with open(pk_path) as fh:
            pk = json.load(fh)
        return (float(pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))),
                "measured (sustained: a step loop lasts seconds)")
    return 1400.0, "fallback (sustained bf16 figure of earlier measurements on this hardware)"


def batch_arm(args):
    """Batched uneven workload: 256 RGB instances, side log-uniform in [64, 1024],
    aspect in [0.5, 2], ellipse masks covering 20-60%, tol 1e-6, automatic omega,
    solved in one persistent launch per batch (graph-replayed). A step = the batch.
    With --multigrid the same batch goes through multigrid-preconditioned CG
    (PT_FLAG_MULTIGRID), every instance in each launch."""
    import torch
    from paintop_b200 import _lib, synth
    from paintop_b200.shard import estimate_cost, partition
    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", local if ws > 1 else 0)
    allinst = synth.batch_uneven(1, args.batch)
    interior_all = [int((i.mask[1:-1, 1:-1] > 0.5).sum()) for i in allinst]
    if args.multigrid:  # about as many CG iterations for every size: pixels x channels
        costs = [estimate_cost(i.width, i.height, i.channels) for i in allinst]
    else:  # SOR sweeps grow with the region's extent
        costs = [estimate_cost(i.width, i.height, i.channels, n, n ** 0.5) for i, n in zip(allinst, interior_all)]
    share = partition(costs, ws)[rank]
    insts = [allinst[k] for k in share]
    ctx = _lib.Context(dev.index)

    def sync():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(el):
        if ws == 1:
            return el
        import torch.distributed as dist
        t = torch.tensor([el], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    r = measure_batch(ctx, dev, insts, [interior_all[k] for k in share], args.steps, args.warmup,
                      args.multigrid, sync=sync, max_over_ranks=max_over_ranks)
    elapsed, e2e_elapsed, kms, iters, conv, alg = (r["elapsed"], r["e2e_elapsed"], r["kms"], r["iters"],
                                                   r["conv"], r["alg"])
    total = len(allinst)
    line = None
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            cpu = batch_cpu_sample(insts, r["reps"], args.multigrid)
        peak, peak_kind = _peaks()
        kmean = float(np.mean(kms))
        line = {
            "metric": ("Poisson instances/s @ rel-res 1e-6 (256 uneven RGB instances, multigrid-CG, one call)"
                       if args.multigrid else
                       "Poisson instances/s @ rel-res 1e-6 (256 uneven RGB instances, one launch)"),
            "value": total * args.steps / elapsed, "unit": "instances/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded sinusoid-plus-noise images, ellipse masks)",
            "config": {"workload": "batch_uneven", "instances": total, "tolerance": 1e-6,
                       "omega": "smoother 1.25" if args.multigrid else "automatic (device, per channel)",
                       "solver": "multigrid-CG" if args.multigrid else "red-black SOR",
                       "l2": "inputs larger than L2"},
            "e2e": {"value": total * args.steps / e2e_elapsed, "unit": "instances/s",
                    "h2d_bytes_per_step": r["h2d"] * ws, "d2h_bytes_per_step": r["d2h"] * ws},
            "roofline": {"bound": "hbm", "achieved": alg / (kmean / 1e3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": alg / (kmean / 1e3) / 1e9 / peak, "traffic": None,
                         "kernel": "multigrid-CG iteration (all kernels, modelled bytes)" if args.multigrid
                         else "ptk::k_solve", "peak_kind": peak_kind, "kernel_ms_mean": kmean},
            "cpu_baseline": cpu, "gpu_launches": int(r["launches"]),
            "clocks": r["clocks"],
            "solver": {"converged": conv, "max_iterations": int(max(max(x) for x in iters)),
                       "sum_iterations": int(sum(sum(x) for x in iters)),
                       "tile_config": None if args.multigrid else tile_config_label(r["config"])},
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


LEARNED_PARAMS = os.path.join(ROOT, "paintop_b200", "weights", "warmstart_unet_256.params")


def learned_leg(ctx, dev, steps: int = 2, warmup: int = 1, scale: int = 8, with_cpu: bool = True):
    """Learned warm start vs plain SOR on the same inputs: 4096x4096 RGB, 8
    polygons (3-10% of the area each), relative residual 1e-6, automatic omega
    for both, inputs resident in HBM. The network (trained by
    paintop_b200.train_warmstart on 20,000 256x256 solves) runs on the inputs
    pooled by `scale`; its upsampled correction plus the guidance seeds the
    solve. Time per solve = guess + solve (CUDA events on the context stream)."""
    import ctypes as Ct
    import torch
    from paintop_b200 import _lib, synth, warmstart
    if not os.path.exists(LEARNED_PARAMS):
        return {"unavailable": "no trained parameters at paintop_b200/weights"}
    inst = synth.multi_4096(1)
    W, H, C = inst.width, inst.height, inst.channels
    g = torch.as_tensor(inst.source, device=dev).contiguous()
    a = torch.as_tensor(inst.target, device=dev).contiguous()
    m = torch.as_tensor(inst.mask, device=dev).contiguous()
    out = torch.empty_like(g)
    guess = torch.empty_like(g)
    net = warmstart.UNet(ctx, seed=0)
    warmstart.load_params(net, LEARNED_PARAMS)
    L = _lib.lib()
    reps = (_lib.PtReport * (C + 1))()
    flags = _lib.PT_FLAG_DEVICE_POINTERS | _lib.PT_FLAG_OMEGA_AUTO
    p_plain = _lib.PtProblem(W, H, C, g.data_ptr(), a.data_ptr(), m.data_ptr(), 0.0, 100000, 1e-6, 1.8,
                             flags, None)
    p_warm = _lib.PtProblem(W, H, C, g.data_ptr(), a.data_ptr(), m.data_ptr(), 0.0, 100000, 1e-6, 1.8,
                            flags | _lib.PT_FLAG_WARM_START, guess.data_ptr())
    mgf = _lib.PT_FLAG_DEVICE_POINTERS | _lib.PT_FLAG_MULTIGRID
    p_mg = _lib.PtProblem(W, H, C, g.data_ptr(), a.data_ptr(), m.data_ptr(), 0.0, 100000, 1e-6, 1.8, mgf, None)
    p_mg_warm = _lib.PtProblem(W, H, C, g.data_ptr(), a.data_ptr(), m.data_ptr(), 0.0, 100000, 1e-6, 1.8,
                               mgf | _lib.PT_FLAG_WARM_START, guess.data_ptr())
    problems = {"plain": p_plain, "learned": p_warm, "multigrid": p_mg, "learned_multigrid": p_mg_warm}
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    torch.cuda.synchronize(dev)

    def run(mode: str):
        learned = mode.startswith("learned")
        if learned:
            st = L.pt_unet_guess(net.h, g.data_ptr(), a.data_ptr(), m.data_ptr(), W, H, C, scale, guess.data_ptr())
            if st != _lib.PT_OK:
                raise _lib.CudaError(st, ctx.last_error())
        st = L.pt_poisson_solve(ctx.h, Ct.byref(problems[mode]), out.data_ptr(), reps, None)
        if st != _lib.PT_OK:
            raise _lib.CudaError(st, ctx.last_error())
        return [int(reps[c].iterations) for c in range(C)], all(reps[c].converged for c in range(C)), \
            [bool(reps[c].warm_start) for c in range(C)]

    res, outs = {}, {}
    for mode in problems:
        for _ in range(warmup):
            run(mode)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            its, conv, used = run(mode)
        e1.record(stream)
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3 / steps
        outs[mode] = out.cpu().numpy()
        key = "sweeps" if mode in ("plain", "learned") else "cg_iterations"
        res[mode] = dict(solves_per_s=1.0 / sec, ms_per_solve=sec * 1e3, **{key: its}, converged=conv,
                         **({"guess_used": used} if mode.startswith("learned") else {}))
    net.close()
    # the cost gate's choice per method (warmstart.GuessGate: a fixed table of
    # measured times), and the best gated path against the best plain one
    gate = warmstart.GuessGate()
    gated = {}
    for method, plain_mode in (("sor", "plain"), ("multigrid", "multigrid")):
        use, entry = gate.decide(W, H, C, 1, method)
        mode = ("learned" if method == "sor" else "learned_multigrid") if use else plain_mode
        gated[method] = {"use_guess": use, "table_entry": entry, "ms_per_solve": res[mode]["ms_per_solve"]}
    best_plain = min(res["plain"]["ms_per_solve"], res["multigrid"]["ms_per_solve"])
    best_gated = min(v["ms_per_solve"] for v in gated.values())
    gated["speedup_best_gated_vs_best_plain"] = best_plain / best_gated
    cpu, parity = None, None
    if with_cpu:
        # the restated reference op on one core: 20 sweeps of one channel give its
        # rate; a full solve (three channels, over a thousand sweeps each) is far
        # beyond a 60 s budget
        from oracle import oracle as O
        O.build()
        c0 = [np.ascontiguousarray(x[:, :, 0]).reshape(-1) for x in (inst.source, inst.target)]
        t0 = time.perf_counter()
        O.blend_channels(c0[0], c0[1], inst.mask.reshape(-1), 1, W, H, 20, 1e-6, 0.0, 1.8)
        per_sweep = (time.perf_counter() - t0) / 20
        cpu = {"seconds_per_sweep_per_channel": per_sweep, "budget_s": 60.0,
               "status": "> budget" if per_sweep * 1000 * C > 60.0 else "within budget",
               "lower_bound_s_per_solve": per_sweep * 1000 * C, "cores": 1, "kind": "port",
               "sample": "20 sweeps (each with its FP64 residual) of channel 0; bound assumes 1000 sweeps per channel"}
        # every timed path's result against the FP64 tight oracle (the CPU op's
        # full solve is beyond the budget above, so it is not a comparison here)
        tight, info = tight_oracle(inst, 0.0)
        parity = {"bounded_tier": {"max_abs": BOUNDED_MAX_ABS, "rms": BOUNDED_RMS,
                                          "source": "crates/paintop-testkit/src/differential.rs:58-62"},
                         "oracle": info,
                         **{f"{mode}_vs_oracle": error_stats(o, tight) for mode, o in outs.items()}}
    return {"workload": "multi_4096: 4096x4096 RGB, 8 polygons 3-10% each, rel-res 1e-6, automatic omega for SOR",
            "model": "U-Net 16-32-64-128, bf16, trained on 20,000 256x256 solves; inference pooled x%d" % scale,
            "steps": steps, **res,
            "speedup": res["learned"]["solves_per_s"] / res["plain"]["solves_per_s"],
            "speedup_multigrid": res["multigrid"]["solves_per_s"] / res["plain"]["solves_per_s"],
            "speedup_learned_multigrid": res["learned_multigrid"]["solves_per_s"] / res["multigrid"]["solves_per_s"],
            "gate": gated, "cpu_baseline": cpu, "parity": parity}


def multigrid_leg(ctx, dev, inst, steps: int = 3, warmup: int = 1):
    """The headline workload (same inputs, device pointers) solved by
    multigrid-preconditioned CG instead of red-black SOR: solves/s (CUDA events
    on the context stream) and CG iterations per channel."""
    import ctypes as Ct
    import torch
    from paintop_b200 import _lib
    W, H, C = inst.width, inst.height, inst.channels
    g = torch.as_tensor(inst.source, device=dev).contiguous()
    a = torch.as_tensor(inst.target, device=dev).contiguous()
    m = torch.as_tensor(inst.mask, device=dev).contiguous()
    out = torch.empty_like(g)
    reps = (_lib.PtReport * (C + 1))()
    p = _lib.PtProblem(W, H, C, g.data_ptr(), a.data_ptr(), m.data_ptr(), WORKLOAD["lam"], WORKLOAD["max_iterations"],
                       WORKLOAD["tolerance"], WORKLOAD["omega"],
                       _lib.PT_FLAG_DEVICE_POINTERS | _lib.PT_FLAG_MULTIGRID, None)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    torch.cuda.synchronize(dev)

    def run():
        st = _lib.lib().pt_poisson_solve(ctx.h, Ct.byref(p), out.data_ptr(), reps, None)
        if st != _lib.PT_OK:
            raise _lib.CudaError(st, ctx.last_error())
    for _ in range(warmup):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        run()
    e1.record(stream)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3 / steps
    return {"solves_per_s": 1.0 / sec, "ms_per_solve": sec * 1e3,
            "cg_iterations": [int(reps[c].iterations) for c in range(C)],
            "refinements": [int(reps[c].refinements) for c in range(C)],
            "converged": all(reps[c].converged for c in range(C)),
            "worst_final_residual": max(reps[c].final_residual for c in range(C)),
            "launches_per_solve": ctx.last_timing()[2], "_out": out.cpu().numpy()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--device-only", action="store_true",
                    help="time only the device-resident arm (for profiler runs)")
    ap.add_argument("--workload", default="screened_2048",
                    choices=["screened_2048", "batch_uneven", "masks", "multigrid", "clone_512", "train"])
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--multigrid", action="store_true",
                    help="batch_uneven: solve by multigrid-preconditioned CG instead of red-black SOR")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-warm-start leg (4096x4096 RGB, learned vs plain)")
    ap.add_argument("--tile-config", type=int, default=-1,
                    help="force this tile configuration of the SOR solve (default: the tuned table)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "cuda":
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batch_uneven":
        return batch_arm(args)
    if args.workload == "masks":
        return mask_arm(args)
    if args.workload == "multigrid":
        return multigrid_arm(args)
    if args.workload == "clone_512":
        return clone_arm(args)
    if args.workload == "train":
        return train_arm(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
