"""Data-parallel training of the warm-start network on CPU (gloo): the batch
split, the rank-ordered exchange of gradient records and their combination.
The replicas are the numpy oracle network with an Adam of the same update
rule, so no GPU is involved; the device kernels behind ``grad_record`` and
``apply_records`` are checked against single-process training in
tests/test_unet_gpu.py."""
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

from oracle import unet_ref as R

B, SIZE, STEPS, LR = 4, 32, 3, 1e-3


class OracleReplica:
    """The grad_record / apply_records contract of the device network, on the oracle:
    a record is the gradient of the replica's mean loss (float32) and its interior
    count; records combine as sum_r c_r g_r / max(1, sum_r c_r) in fp64, in order."""

    def __init__(self, seed, emulate_bf16):
        self.p = R.init_params(seed).astype(np.float32)
        self.m = np.zeros_like(self.p)
        self.v = np.zeros_like(self.p)
        self.step = 0
        self.emulate_bf16 = emulate_bf16
        self.applied = []  # the combined gradient of every step

    @property
    def param_count(self):
        return self.p.size

    def features(self, g, a, m):
        return torch.from_numpy(R.features(g.numpy(), a.numpy(), m.numpy()))

    def grad_record(self, f, target, lm, out):
        loss, g = R.Net(self.p.astype(np.float64), self.emulate_bf16).loss_grad(f.numpy().astype(np.float64), target.numpy(),
                                                              lm.numpy())
        out[:-1] = torch.from_numpy(g.astype(np.float32))
        out[-1] = float((lm.numpy() > 0.5).sum())
        return loss, out

    def apply_records(self, records, lr):
        rec = records.numpy().astype(np.float64)
        c = rec[:, -1]
        acc = np.zeros(self.p.size)
        for r in range(rec.shape[0]):
            acc += c[r] * rec[r, :-1]
        g = (acc / max(1.0, c.sum())).astype(np.float32)
        self.applied.append(g)
        self.step += 1
        b1, b2, eps = np.float32(0.9), np.float32(0.999), np.float32(1e-8)
        self.m = b1 * self.m + (1 - b1) * g
        self.v = b2 * self.v + (1 - b2) * g * g
        bc1, bc2 = 1 - b1 ** self.step, 1 - b2 ** self.step
        self.p = (self.p - np.float32(lr) * (self.m / bc1) / (np.sqrt(self.v / bc2) + eps)).astype(np.float32)


def _dataset():
    from paintop_b200 import warmstart as ws
    g, a, m = ws.make_instances(2 * B, SIZE, seed=21, device="cpu")
    # any target exercises the exchange; the anchor keeps it smooth
    return ws.Dataset(g, a, m, a.clone(), np.zeros(2 * B, dtype=np.int64), 0.0, 0.0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q, emulate_bf16, steps):
    import torch.distributed as dist
    from datetime import timedelta
    from paintop_b200 import warmstart as ws
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        net = OracleReplica(seed=5, emulate_bf16=emulate_bf16)
        tr = ws.DataParallelTrainer(net, _dataset(), batch=B, lr=LR, seed=3)
        losses = [tr.step() for _ in range(steps)]
        q.put((rank, tr.local_slice(), losses, net.p.tobytes(), np.stack(net.applied)))
    except Exception as e:  # report instead of leaving the parent waiting
        q.put((rank, "error", repr(e), b"", None))
        raise
    finally:
        dist.destroy_process_group()


def _run(world, emulate_bf16, steps=STEPS):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, emulate_bf16, steps))
             for r in range(world)]
    for p in procs:
        p.start()
    got = sorted((q.get(timeout=300) for _ in range(world)), key=lambda g: g[0])
    assert all(g[1] != "error" for g in got), got
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return got


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_data_parallel_step_matches_the_whole_batch():
    """In exact arithmetic (the fp64 network) the combined records are the whole
    batch's gradient: every step's applied gradient and loss agree with one rank's
    to float32 rounding, and both ranks hold the same parameters bit for bit."""
    two = _run(2, emulate_bf16=False)
    one = _run(1, emulate_bf16=False)
    # contiguous halves of every global batch
    assert [g[1] for g in two] == [(0, 2), (2, 4)]
    # both replicas take the same steps bit for bit and report the same loss
    assert two[0][3] == two[1][3] and two[0][2] == two[1][2]
    assert np.array_equal(two[0][4], two[1][4])
    for k in range(STEPS):
        assert _rel(two[0][4][k], one[0][4][k]) < 1e-5, k
    np.testing.assert_allclose(two[0][2], one[0][2], rtol=1e-6)
    p0 = R.init_params(5).astype(np.float32)
    assert not np.array_equal(np.frombuffer(one[0][3], dtype=np.float32), p0)


def test_data_parallel_gradient_with_bf16_activations():
    """With the device's bf16 activations each replica's backward rounds at its own
    scale (dpred = 2 d / its count), so the first step's gradient matches the whole
    batch's to the bf16 tolerance of the device parity tests, layer by layer."""
    two = _run(2, emulate_bf16=True, steps=1)
    one = _run(1, emulate_bf16=True, steps=1)
    assert two[0][3] == two[1][3]
    assert two[0][2][0] == one[0][2][0]  # the first loss is per-sample arithmetic
    g2, g1 = two[0][4][0].astype(np.float64), one[0][4][0].astype(np.float64)
    layout, head_w, _ = R.param_layout()
    for l, (w, b, co, ci) in enumerate(layout):
        assert _rel(g2[w:b], g1[w:b]) < 3e-2, l
    assert _rel(g2[head_w:], g1[head_w:]) < 3e-2
