"""Multi-rank host logic on CPU (gloo, world size 2): the deterministic
partition, the sharded solve gathered on rank 0 (solves run on the oracle, so
no GPU is involved), and failure detection when a rank leaves between steps."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from paintop_b200.shard import estimate_cost, partition


def test_partition_is_deterministic_and_balanced():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1, 100, 257).tolist()
    a = partition(costs, 4)
    b = partition(costs, 4)
    assert a == b
    assert sorted(i for s in a for i in s) == list(range(257))
    loads = [sum(costs[i] for i in s) for s in a]
    assert max(loads) - min(loads) <= max(costs)
    assert partition([5.0], 3) == [[0], [], []]
    assert estimate_cost(10, 10, 3) == 300.0
    with pytest.raises(ValueError):
        partition([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problems():
    out = []
    for k, (w, h, c) in enumerate([(12, 9, 1), (20, 14, 3), (9, 9, 2), (17, 11, 1), (30, 6, 1)]):
        rng = np.random.default_rng(50 + k)
        out.append((w, h, c, rng.random(w * h * c).astype(np.float32),
                    rng.random(w * h * c).astype(np.float32),
                    (rng.random(w * h) < 0.7).astype(np.float32)))
    return out


def _solve(p):
    from oracle import oracle as O
    w, h, c, s, t, m = p
    out, worst, _ = O.blend_channels(s, t, m, c, w, h, 300, 1e-8, 0.1, 1.8)
    return out, worst.iterations


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    from paintop_b200.shard import run_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    probs = _problems()
    costs = [estimate_cost(p[0], p[1], p[2]) for p in probs]
    res = run_sharded(probs, costs, _solve, rank, world)
    if rank == 0:
        q.put([(r[0].tobytes(), r[1]) for r in res])
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_solve_matches_single_process(oracle):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    want = [_solve(p) for p in _problems()]
    assert [g[1] for g in got] == [w[1] for w in want]
    assert all(g[0] == w[0].tobytes() for g, w in zip(got, want))


def _leaving_worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    if rank == 1:
        # leaves between steps, with nothing in flight
        os._exit(0)
    try:
        dist.barrier()
        q.put("no error")
    except Exception as e:  # the survivor learns of it through the short timeout
        q.put(type(e).__name__)


def test_rank_leaving_is_detected_by_the_survivor():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_leaving_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outcome = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert outcome != "no error"
