"""Learned warm start for the Poisson solve: a small U-Net behind ``pt_unet_*``.

The network (``csrc/unet``) runs and trains on the GPU through the library's
own tensor-core kernels; PyTorch only holds device buffers and generates the
seeded synthetic training images on the device (the same distributions as
:mod:`paintop_b200.synth`). Training data are solves of the plain method
itself: each 256x256 instance is solved by the library's red-black SOR to a
relative residual of 1e-7 and the network learns to predict the correction
u - g (solution minus guidance) from four per-pixel features
(``pt_unet_features``). For Poisson blending that correction is harmonic in
the interior with boundary values anchor - g, so it is smooth where g is not.

At inference the guess seeds ``pt_poisson_solve`` through PT_FLAG_WARM_START;
SOR with FP64 refinement then drives the solve to the same tolerance, measured
against the same anchor-based normalisation as the plain solve. For images
larger than the training size the problem is pooled by an integer factor, the
network predicts the coarse correction, and the guess is the fine guidance plus
the upsampled correction, so the fine detail of g is kept and only the smooth
part comes from the network.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import time
from dataclasses import dataclass

import numpy as np

from . import _lib

PT_OK = 0


def _torch():
    import torch  # device buffers only
    return torch


def _dptr(t) -> int:
    assert t.is_cuda and t.is_contiguous() and t.dtype == _torch().float32, (t.device, t.dtype)
    return t.data_ptr()


class UNet:
    """A network on one library context. Buffers are float32 CUDA tensors."""

    def __init__(self, ctx: "_lib.Context", seed: int = 0):
        self.ctx = ctx
        h = C.c_void_p()
        st = _lib.lib().pt_unet_create(ctx.h, C.c_uint64(seed), C.byref(h))
        if st != PT_OK:
            raise _lib.CudaError(st, ctx.last_error())
        self.h = h
        ctx.adopt(self)

    def close(self):
        """Free the network; the context closes its networks before itself."""
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            _lib.lib().pt_unet_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != PT_OK:
            raise _lib.CudaError(st, f"{what}: {self.ctx.last_error()}")

    @property
    def param_count(self) -> int:
        return int(_lib.lib().pt_unet_param_count(self.h))

    def get_params(self) -> np.ndarray:
        out = np.empty(self.param_count, dtype=np.float32)
        self._check(_lib.lib().pt_unet_get_params(self.h, out.ctypes.data), "get_params")
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.param_count
        self._check(_lib.lib().pt_unet_set_params(self.h, p.ctypes.data), "set_params")

    def save(self, path: str) -> None:
        self._check(_lib.lib().pt_unet_save(self.h, os.fsencode(path)), "save")

    def load(self, path: str) -> None:
        self._check(_lib.lib().pt_unet_load(self.h, os.fsencode(path)), "load")

    def features(self, guidance, anchor, mask):
        """(B, H, W) float32 CUDA tensors -> (B, H, W, 4) features."""
        torch = _torch()
        B, H, W = guidance.shape
        f = torch.empty((B, H, W, 4), device=guidance.device, dtype=torch.float32)
        torch.cuda.synchronize()
        self._check(_lib.lib().pt_unet_features(self.h, _dptr(guidance), _dptr(anchor), _dptr(mask),
                                                B, H, W, _dptr(f)), "features")
        return f

    def forward(self, feats):
        torch = _torch()
        B, H, W, _ = feats.shape
        pred = torch.empty((B, H, W), device=feats.device, dtype=torch.float32)
        torch.cuda.synchronize()
        self._check(_lib.lib().pt_unet_forward(self.h, _dptr(feats), B, H, W, _dptr(pred)), "forward")
        return pred

    def loss_grad(self, feats, target, loss_mask, want_grad=True):
        B, H, W, _ = feats.shape
        loss = C.c_double()
        g = np.empty(self.param_count, dtype=np.float32) if want_grad else None
        _torch().cuda.synchronize()
        self._check(_lib.lib().pt_unet_loss_grad(self.h, _dptr(feats), _dptr(target), _dptr(loss_mask),
                                                 B, H, W, C.byref(loss),
                                                 g.ctypes.data if g is not None else None), "loss_grad")
        return loss.value, g

    def train_step(self, feats, target, loss_mask, lr: float = 1e-3) -> float:
        B, H, W, _ = feats.shape
        loss = C.c_double()
        _torch().cuda.synchronize()
        self._check(_lib.lib().pt_unet_train_step(self.h, _dptr(feats), _dptr(target), _dptr(loss_mask),
                                                  B, H, W, C.c_float(lr), C.byref(loss)), "train_step")
        return loss.value

    def grad_record(self, feats, target, loss_mask, out=None):
        """This replica's gradient record (device float32 tensor of param_count + 1:
        the gradient of the mean loss over its batch, then its interior count)
        and its loss; the parameters do not change."""
        torch = _torch()
        B, H, W, _ = feats.shape
        if out is None:
            out = torch.empty(self.param_count + 1, dtype=torch.float32, device=feats.device)
        loss = C.c_double()
        torch.cuda.synchronize()
        self._check(_lib.lib().pt_unet_grad_record(self.h, _dptr(feats), _dptr(target), _dptr(loss_mask),
                                                   B, H, W, C.byref(loss), _dptr(out)), "grad_record")
        return loss.value, out

    def apply_records(self, records, lr: float = 1e-3) -> None:
        """One Adam step on gradient records stacked replica-major (R x (param_count + 1),
        device float32), combined in replica order."""
        torch = _torch()
        if records.dim() != 2 or records.shape[1] != self.param_count + 1 or not records.is_contiguous():
            raise ValueError("records must be a contiguous (replicas, param_count + 1) tensor")
        torch.cuda.synchronize()
        self._check(_lib.lib().pt_unet_apply_records(self.h, _dptr(records), records.shape[0], C.c_float(lr)),
                    "apply_records")


# ---------------------------------------------------------------------------
# seeded synthetic training instances on the device
# ---------------------------------------------------------------------------
def _sinusoids(gen, rng: np.random.Generator, B: int, size: int, device):
    """B single-channel images of 8 random sinusoids + 0.5 + N(0, 0.02^2), clamped."""
    torch = _torch()
    f = rng.uniform(1.0, 16.0, (B, 8))
    th = rng.uniform(0.0, 2 * math.pi, (B, 8))
    ph = rng.uniform(0.0, 2 * math.pi, (B, 8))
    a = rng.uniform(0.05, 0.2, (B, 8))
    kx = torch.tensor(2 * math.pi * f * np.cos(th), device=device, dtype=torch.float32)
    ky = torch.tensor(2 * math.pi * f * np.sin(th), device=device, dtype=torch.float32)
    ph = torch.tensor(ph, device=device, dtype=torch.float32)
    a = torch.tensor(a, device=device, dtype=torch.float32)
    c = (torch.arange(size, device=device, dtype=torch.float32) + 0.5) / size
    x = c.view(1, 1, 1, size)
    y = c.view(1, 1, size, 1)
    arg = kx.view(B, 8, 1, 1) * x + ky.view(B, 8, 1, 1) * y + ph.view(B, 8, 1, 1)
    img = 0.5 + (a.view(B, 8, 1, 1) * torch.sin(arg)).sum(1)
    img = img + 0.02 * torch.randn((B, size, size), generator=gen, device=device)
    return img.clamp_(0.0, 1.0).contiguous()


def _masks(rng: np.random.Generator, B: int, size: int, device):
    """Random ellipse (pixel-centre test) or blob polygon (4x4 supersampled,
    nonzero rule) masks, as in synth.train_instance."""
    torch = _torch()
    out = torch.empty((B, size, size), device=device, dtype=torch.float32)
    c = torch.arange(size, device=device, dtype=torch.float64) + 0.5
    S = 4
    sub = (torch.arange(size * S, device=device, dtype=torch.float64) + 0.5) / S
    for b in range(B):
        if rng.uniform() < 0.5:
            rx, ry = rng.uniform(0.15, 0.4) * size, rng.uniform(0.15, 0.4) * size
            cx = size / 2 + rng.uniform(-0.08, 0.08) * size
            cy = size / 2 + rng.uniform(-0.08, 0.08) * size
            ang = rng.uniform(0, math.pi)
            X = c.view(1, -1) - cx
            Y = c.view(-1, 1) - cy
            u = X * math.cos(ang) + Y * math.sin(ang)
            v = -X * math.sin(ang) + Y * math.cos(ang)
            out[b] = ((u / rx) ** 2 + (v / ry) ** 2 <= 1.0).float()
        else:
            nv = int(rng.integers(5, 13))
            mean_r = rng.uniform(0.2, 0.38) * size
            angles = np.sort(rng.uniform(0, 2 * math.pi, nv))
            radii = mean_r * (1.0 + rng.uniform(-0.25, 0.25, nv))
            px = size / 2 + radii * np.cos(angles)
            py = size / 2 + radii * np.sin(angles)
            X = sub.view(1, -1)
            Y = sub.view(-1, 1)
            wind = torch.zeros((size * S, size * S), device=device, dtype=torch.int32)
            for k in range(nv):
                ax, ay, bx, by = px[k], py[k], px[(k + 1) % nv], py[(k + 1) % nv]
                straddle = (ay <= Y) != (by <= Y)
                if ay == by:
                    continue
                xc = ax + (Y - ay) * (bx - ax) / (by - ay)
                d = 1 if by > ay else -1
                wind += (straddle & (xc > X)).int() * d
            cov = (wind != 0).float().view(size, S, size, S).sum((1, 3)) / (S * S)
            out[b] = cov
    return out


def make_instances(n: int, size: int = 256, seed: int = 0, device="cuda"):
    """n seeded training instances: (guidance, anchor, mask), each (n, size, size)."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    g = _sinusoids(gen, rng, n, size, device)
    a = _sinusoids(gen, rng, n, size, device)
    m = _masks(rng, n, size, device)
    return g, a, m


def solve_batch_device(ctx, guidance, anchor, mask, *, tol=1e-7, max_iterations=100000,
                       omega_auto=True, omega=1.8, guess=None):
    """Solve B single-channel Poisson-blend problems held in device tensors with
    one pt_poisson_solve_batch call. Returns (out (B, H, W), reports)."""
    torch = _torch()
    B, H, W = guidance.shape
    out = torch.empty_like(guidance)
    arr = (_lib.PtProblem * B)()
    outs = (C.c_void_p * B)()
    reps = [(_lib.PtReport * 2)() for _ in range(B)]
    rep_ptrs = (C.POINTER(_lib.PtReport) * B)()
    flags = _lib.PT_FLAG_DEVICE_POINTERS | (_lib.PT_FLAG_OMEGA_AUTO if omega_auto else 0)
    img = H * W * 4
    for i in range(B):
        arr[i] = _lib.PtProblem(W, H, 1, guidance.data_ptr() + i * img, anchor.data_ptr() + i * img,
                                mask.data_ptr() + i * img, 0.0, max_iterations, tol, omega,
                                flags | (_lib.PT_FLAG_WARM_START if guess is not None else 0),
                                (guess.data_ptr() + i * img) if guess is not None else None)
        outs[i] = out.data_ptr() + i * img
        rep_ptrs[i] = C.cast(reps[i], C.POINTER(_lib.PtReport))
    torch.cuda.synchronize()
    st = _lib.lib().pt_poisson_solve_batch(ctx.h, arr, B, outs, rep_ptrs, None)
    if st != PT_OK:
        raise _lib.CudaError(st, ctx.last_error())
    return out, [r[1].as_dict() for r in reps]


def interior_mask(mask):
    """mask > 0.5 away from the image border (the solver's interior rule)."""
    m = (mask > 0.5).float()
    m[:, 0, :] = 0
    m[:, -1, :] = 0
    m[:, :, 0] = 0
    m[:, :, -1] = 0
    return m.contiguous()


@dataclass
class Dataset:
    guidance: object
    anchor: object
    mask: object
    solution: object
    sweeps: np.ndarray
    gen_s: float
    solve_s: float


def build_dataset(ctx, n: int = 20000, size: int = 256, seed: int = 0, chunk: int = 512,
                  tol: float = 1e-7, _seed_base=None) -> Dataset:
    """Generate and solve n training instances on the device (solves by the plain
    method). Chunk c0 (instances c0 .. c0 + chunk - 1) comes from the seed
    seed * 1000003 + c0."""
    torch = _torch()
    gs, an, ms, us, sw = [], [], [], [], []
    t_gen = t_solve = 0.0
    base = seed * 1000003 if _seed_base is None else _seed_base
    for c0 in range(0, n, chunk):
        k = min(chunk, n - c0)
        t0 = time.perf_counter()
        g, a, m = make_instances(k, size, base + c0)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        u, reps = solve_batch_device(ctx, g, a, m, tol=tol)
        t2 = time.perf_counter()
        t_gen += t1 - t0
        t_solve += t2 - t1
        gs.append(g); an.append(a); ms.append(m); us.append(u)
        sw += [r["iterations"] for r in reps]
        bad = [r for r in reps if not r["converged"]]
        if bad:
            raise RuntimeError(f"{len(bad)} training solves did not converge: {bad[0]}")
    return Dataset(torch.cat(gs), torch.cat(an), torch.cat(ms), torch.cat(us), np.asarray(sw),
                   t_gen, t_solve)


class Trainer:
    """Adam on the masked L2 loss over interior pixels, one shuffled pass per epoch.

    The state that decides every later step is the network (parameters, Adam
    moments, step count: ``pt_unet_save``) plus the epoch, the position in the
    current permutation, that permutation and the shuffling generator's state;
    :meth:`save` and :meth:`load` carry all of it, so a resumed run repeats an
    uninterrupted one bit for bit."""

    def __init__(self, net: UNet, data: Dataset, *, batch: int = 64, lr: float = 1e-3, seed: int = 0):
        self.net, self.data, self.batch, self.lr = net, data, batch, lr
        self.n = data.guidance.shape[0]
        if self.n < batch:
            raise ValueError("the dataset is smaller than one batch")
        self.rng = np.random.default_rng(seed)
        self.epoch, self.pos, self.steps = 0, 0, 0
        self.order = self.rng.permutation(self.n)
        self.step_s = 0.0

    def _next_indices(self):
        if self.pos + self.batch > self.n:
            self.epoch += 1
            self.pos = 0
            self.order = self.rng.permutation(self.n)
        idx = self.order[self.pos:self.pos + self.batch]
        self.pos += self.batch
        return idx

    def step(self) -> float:
        torch = _torch()
        d = self.data
        idx = torch.as_tensor(self._next_indices(), device=d.guidance.device)
        g = d.guidance[idx].contiguous()
        a = d.anchor[idx].contiguous()
        m = d.mask[idx].contiguous()
        target = (d.solution[idx] - g).contiguous()  # the correction u - g
        f = self.net.features(g, a, m)
        lm = interior_mask(m)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss = self.net.train_step(f, target, lm, self.lr)
        torch.cuda.synchronize()
        self.step_s += time.perf_counter() - t0
        self.steps += 1
        return loss

    def save(self, path: str) -> None:
        self.net.save(path)
        state = dict(epoch=self.epoch, pos=self.pos, steps=self.steps, batch=self.batch, lr=self.lr,
                     n=self.n, rng=self.rng.bit_generator.state)
        np.savez(path + ".trainer.npz", order=self.order, state=json.dumps(state))

    def load(self, path: str) -> None:
        self.net.load(path)
        z = np.load(path + ".trainer.npz")
        state = json.loads(str(z["state"]))
        if state["n"] != self.n or state["batch"] != self.batch:
            raise ValueError("checkpoint was written for another dataset size or batch")
        self.epoch, self.pos, self.steps = state["epoch"], state["pos"], state["steps"]
        self.lr = state["lr"]
        self.rng.bit_generator.state = state["rng"]
        self.order = z["order"]


class DataParallelTrainer(Trainer):
    """Data-parallel :class:`Trainer`: one replica per rank of a process group
    (NCCL between GPUs), every rank holding the whole dataset and the same
    network state.

    Every rank draws the same global batch from the same shuffled order and
    takes its contiguous part (rank r of R: positions r*b//R .. (r+1)*b//R).
    A step computes the rank's gradient record (``pt_unet_grad_record``),
    all-gathers the records in rank order and applies them with
    ``pt_unet_apply_records``, which sums them in that fixed order; so all
    ranks take the same step bit for bit, a rerun repeats it bit for bit, and
    the step is the whole batch's gradient up to fp64 summation order. With
    one rank it is :class:`Trainer` exactly.

    `net` needs ``features``, ``param_count``, ``grad_record`` and
    ``apply_records`` (a :class:`UNet`); :meth:`save` writes from rank 0 only."""

    def __init__(self, net, data: Dataset, *, group=None, batch: int = 64, lr: float = 1e-3, seed: int = 0):
        import torch.distributed as dist
        super().__init__(net, data, batch=batch, lr=lr, seed=seed)
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if self.world > batch:
            raise ValueError("more ranks than samples in a batch")
        torch = _torch()
        dev = data.guidance.device
        self._rec = torch.empty(net.param_count + 1, dtype=torch.float32, device=dev)
        # flat gather targets (gloo wants them flat), viewed rank-major
        self._records = torch.empty(self.world * (net.param_count + 1), dtype=torch.float32, device=dev)
        self._loss = torch.zeros(2, dtype=torch.float64, device=dev)
        self._losses = torch.empty(self.world * 2, dtype=torch.float64, device=dev)

    def local_slice(self):
        """Positions of this rank's samples within a global batch."""
        return self.rank * self.batch // self.world, (self.rank + 1) * self.batch // self.world

    def step(self) -> float:
        """One data-parallel step; returns the whole batch's loss (the interior-weighted
        mean of the ranks' losses)."""
        import torch.distributed as dist
        torch = _torch()
        d = self.data
        lo, hi = self.local_slice()
        idx = torch.as_tensor(self._next_indices()[lo:hi], device=d.guidance.device)
        g = d.guidance[idx].contiguous()
        a = d.anchor[idx].contiguous()
        m = d.mask[idx].contiguous()
        target = (d.solution[idx] - g).contiguous()
        f = self.net.features(g, a, m)
        lm = interior_mask(m)
        cuda = g.is_cuda
        if cuda:
            torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss, rec = self.net.grad_record(f, target, lm, out=self._rec)
        dist.all_gather_into_tensor(self._records, rec, group=self.group)
        self.net.apply_records(self._records.view(self.world, -1), self.lr)
        if cuda:
            torch.cuda.synchronize()
        self.step_s += time.perf_counter() - t0
        self.steps += 1
        # whole-batch loss from the ranks' losses and interior counts, in rank order
        self._loss[0] = loss
        self._loss[1] = float(rec[-1])
        dist.all_gather_into_tensor(self._losses, self._loss, group=self.group)
        lc = self._losses.view(self.world, 2).cpu().numpy()
        num = 0.0
        for r in range(self.world):
            num += lc[r, 0] * lc[r, 1]
        return num / max(1.0, float(lc[:, 1].sum()))

    def save(self, path: str) -> None:
        if self.rank == 0:
            super().save(path)


def build_dataset_sharded(ctx, n: int = 20000, size: int = 256, seed: int = 0, chunk: int = 512,
                          tol: float = 1e-7, group=None) -> Dataset:
    """:func:`build_dataset` with its chunks solved round-robin over the ranks of
    `group` and broadcast from their owners in chunk order: every rank ends with
    the single-process dataset (the chunks are seeded by position, and each
    solve depends only on its own instance)."""
    import torch.distributed as dist
    torch = _torch()
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device())
    starts = list(range(0, n, chunk))
    mine = {c0: build_dataset(ctx, n=min(chunk, n - c0), size=size, seed=0, chunk=chunk, tol=tol,
                              _seed_base=seed * 1000003 + c0)
            for j, c0 in enumerate(starts) if j % world == rank}
    gs, an, ms, us = [], [], [], []
    sweeps = np.zeros(n, dtype=np.int64)
    gen_s = solve_s = 0.0
    for j, c0 in enumerate(starts):
        k = min(chunk, n - c0)
        if c0 in mine:
            part = mine[c0]
            tens = [part.guidance, part.anchor, part.mask, part.solution]
            sw = torch.as_tensor(part.sweeps, device=dev)
            gen_s += part.gen_s
            solve_s += part.solve_s
        else:
            tens = [torch.empty((k, size, size), dtype=torch.float32, device=dev) for _ in range(4)]
            sw = torch.empty(k, dtype=torch.int64, device=dev)
        src = dist.get_global_rank(group, j % world) if group is not None else j % world
        for t in tens + [sw]:
            dist.broadcast(t, src=src, group=group)
        gs.append(tens[0]); an.append(tens[1]); ms.append(tens[2]); us.append(tens[3])
        sweeps[c0:c0 + k] = sw.cpu().numpy()
    return Dataset(torch.cat(gs), torch.cat(an), torch.cat(ms), torch.cat(us), sweeps, gen_s, solve_s)


def train(net: UNet, data: Dataset, *, epochs: int = 4, batch: int = 64, lr: float = 1e-3,
          seed: int = 0, log=None, max_steps=None):
    """Run `epochs` passes (or `max_steps` steps); returns the per-step losses and
    the host-timed duration of the training steps."""
    tr = Trainer(net, data, batch=batch, lr=lr, seed=seed)
    total = epochs * (tr.n // batch)
    if max_steps:
        total = min(total, max_steps)
    losses = []
    for k in range(total):
        losses.append(tr.step())
        if log and (k + 1) % 50 == 0:
            log(f"epoch {tr.epoch} step {k + 1} loss {np.mean(losses[-50:]):.3e}")
    return np.asarray(losses), tr.step_s


def train_flops_per_pixel() -> float:
    """Algorithmic FLOPs of one training step per input pixel: forward, backward-data
    and backward-weights of every 3x3 convolution (2 FLOPs per multiply-add, padded
    channel counts as executed; the first layer has no backward-data)."""
    from_level = [0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0]
    layers = [(16, 16), (16, 16), (32, 16), (32, 32), (64, 32), (64, 64), (128, 64), (128, 128),
              (64, 192), (64, 64), (32, 96), (32, 32), (16, 48), (16, 16)]
    total = 0.0
    for l, ((co, ci), lev) in enumerate(zip(layers, from_level)):
        mac = 9.0 * co * ci / (4 ** lev)
        total += 2 * mac * (3 if l > 0 else 2)
    return total


def predict_guess(net: UNet, guidance, anchor, mask, scale: int = 1):
    """Warm-start guess for single-channel problems (B, H, W) through
    ``pt_unet_guess``: guidance + the predicted correction, the network run on
    the problem pooled by `scale` and its correction upsampled bilinearly."""
    torch = _torch()
    B, H, W = guidance.shape
    out = torch.empty_like(guidance)
    torch.cuda.synchronize()
    img = H * W * 4
    for b in range(B) if scale > 1 else []:
        net._check(_lib.lib().pt_unet_guess(net.h, guidance.data_ptr() + b * img, anchor.data_ptr() + b * img,
                                            mask.data_ptr() + b * img, W, H, 1, scale,
                                            out.data_ptr() + b * img), "guess")
    if scale == 1:
        # the batch as channels of one image would share one mask: run the
        # network on the batch directly instead
        out = (guidance + net.forward(net.features(guidance, anchor, mask))).contiguous()
    return out


def guess_image(net: UNet, guidance, anchor, mask, scale: int):
    """pt_unet_guess on one interleaved (H, W, C) problem held in device tensors."""
    torch = _torch()
    H, W, Ch = guidance.shape
    out = torch.empty_like(guidance)
    torch.cuda.synchronize()
    net._check(_lib.lib().pt_unet_guess(net.h, _dptr(guidance), _dptr(anchor), _dptr(mask), W, H, Ch, scale,
                                        _dptr(out)), "guess")
    return out


def save_params(net: UNet, path: str) -> None:
    """The network's fp32 parameters (no optimiser state) as a small file."""
    p = net.get_params()
    with open(path, "wb") as f:
        f.write(b"PTUNETP1")
        f.write(np.array([p.size], dtype="<u8").tobytes())
        f.write(p.astype("<f4").tobytes())


def load_params(net: UNet, path: str) -> None:
    with open(path, "rb") as f:
        if f.read(8) != b"PTUNETP1":
            raise ValueError(f"{path}: not a parameter file")
        n = int(np.frombuffer(f.read(8), dtype="<u8")[0])
        if n != net.param_count:
            raise ValueError(f"{path}: {n} parameters, the network has {net.param_count}")
        net.set_params(np.frombuffer(f.read(4 * n), dtype="<f4"))


# ---------------------------------------------------------------------------
# cost gate: run the network only where its guess pays for its inference
# ---------------------------------------------------------------------------
GATE_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "warmstart_gate_b200.json")
METHODS = ("sor", "multigrid")


def gate_key(width: int, height: int, channels: int, batch: int, method: str) -> str:
    """Entries are keyed like the tile-configuration table: floor(log2) of the
    pixels over all channels and images, floor(log2) of one image's pixels,
    whether the call holds a batch, and the iteration (SOR or multigrid)."""
    if method not in METHODS:
        raise ValueError(f"method must be one of {METHODS}")
    px = float(width) * height
    lt = max(0, math.floor(math.log2(max(px * channels * batch, 1.0))))
    ll = max(0, math.floor(math.log2(max(px, 1.0))))
    return f"{lt}:{ll}:{int(batch > 1)}:{method}"


class GuessGate:
    """A fixed table of measured end-to-end times per shape key and method:
    the time of a plain solve and of network inference plus the warm-started
    solve, both to the same bar. The network runs only where the second was
    measured faster; a shape the table does not hold gets the plain solve (the
    guess is never used blind). The decision depends on nothing but the
    problem's shape and the method, so it is the same on every call."""

    def __init__(self, path: str = GATE_TABLE):
        self.path = path
        self.entries = {}
        if os.path.exists(path):
            with open(path) as f:
                for e in json.load(f)["entries"]:
                    self.entries[e["key"]] = e

    def decide(self, width: int, height: int, channels: int, batch: int = 1, method: str = "sor"):
        """-> (use the guess?, the entry that decided, or None)."""
        e = self.entries.get(gate_key(width, height, channels, batch, method))
        if e is None:
            return False, None
        return bool(e["learned_ms"] < e["plain_ms"]), e
