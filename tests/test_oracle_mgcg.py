"""The FP64 multigrid-preconditioned CG oracle (oracle/mgcg_ref.c), used as the
tight oracle at the benchmark workloads' full sizes, checked against the plain
FP64 CG oracle (oracle/cg_ref.c) on the same systems, against the reference's
analytic known answers, and for independence of the thread count."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("lam", [0.0, 0.01, 1.0])
@pytest.mark.parametrize("size", [64, 200])
def test_mgcg_agrees_with_plain_cg(oracle, lam, size):
    from paintop_b200 import synth
    inst = synth.screened_2048(7, size=size)
    W, H, C = inst.width, inst.height, inst.channels
    s, t, m = inst.source.reshape(-1), inst.target.reshape(-1), inst.mask.reshape(-1)
    u, ach, its = oracle.mgcg_blend_channels(s, t, m, C, W, H, lam=lam, rel_tol=1e-12)
    v, ach2 = oracle.cg_blend_channels(s, t, m, C, W, H, lam=lam, rel_tol=1e-12)
    assert (ach <= 1e-12).all() and (ach2 <= 1e-12).all()
    assert (its < 60).all()
    assert np.abs(u - v).max() <= 1e-9
    # boundary cells hold the anchor exactly
    keep = np.repeat(oracle.classify_cells(m, W, H) == 0, C)
    assert np.array_equal(u[keep], t[keep].astype(np.float64))


def test_mgcg_ragged_mask_and_several_regions(oracle):
    rng = np.random.default_rng(3)
    W, H = 181, 97
    m = (rng.random((H, W)) < 0.7).astype(np.float32)
    m[:, 90] = 0.0  # two regions
    s = rng.random(W * H).astype(np.float32)
    t = rng.random(W * H).astype(np.float32)
    u, ach, _ = oracle.mgcg_blend_channels(s, t, m.reshape(-1), 1, W, H, lam=0.0, rel_tol=1e-12)
    v, _ = oracle.cg_blend_channels(s, t, m.reshape(-1), 1, W, H, lam=0.0, rel_tol=1e-12)
    assert ach[0] <= 1e-12 and np.abs(u - v).max() <= 1e-9


def test_mgcg_known_answers(oracle):
    """poisson/tests.rs: a constant source over a constant target reproduces the
    target; a linear ramp in source and target is reproduced exactly."""
    W, H = 40, 30
    m = np.zeros((H, W), np.float32)
    m[5:25, 5:35] = 1.0
    const = np.full(W * H, 0.25, np.float32)
    u, ach, its = oracle.mgcg_blend_channels(const, const, m.reshape(-1), 1, W, H)
    assert its[0] == 0 and np.abs(u - 0.25).max() == 0.0
    x = np.tile(np.arange(W, dtype=np.float32) / W, H)
    u, ach, _ = oracle.mgcg_blend_channels(x, x, m.reshape(-1), 1, W, H, rel_tol=1e-12)
    assert np.abs(u - x).max() <= 1e-10


def test_mgcg_degenerate_and_empty(oracle):
    one = np.ones(4, np.float32)
    u, ach, its = oracle.mgcg_blend_channels(one, one * 2, one, 1, 2, 2)
    assert its[0] == 0 and (u == 2.0).all()
    z = np.zeros(100, np.float32)
    u, ach, its = oracle.mgcg_blend_channels(z + 1, z + 3, z, 1, 10, 10)
    assert its[0] == 0 and (u == 3.0).all()


def test_mgcg_does_not_depend_on_thread_count(oracle, tmp_path):
    code = ("import sys, numpy as np; sys.path.insert(0, %r)\n"
            "from oracle import oracle as O\n"
            "from paintop_b200 import synth\n"
            "i = synth.screened_2048(9, size=160)\n"
            "u, a, it = O.mgcg_blend_channels(i.source.reshape(-1), i.target.reshape(-1),"
            " i.mask.reshape(-1), i.channels, i.width, i.height, lam=0.01)\n"
            "np.save(sys.argv[1], u)\n") % ROOT
    outs = []
    for n in ("1", "5"):
        path = str(tmp_path / f"u{n}.npy")
        env = dict(os.environ, OMP_NUM_THREADS=n)
        subprocess.run([sys.executable, "-c", code, path], check=True, env=env, cwd=ROOT)
        outs.append(np.load(path))
    assert np.array_equal(outs[0].view(np.uint64), outs[1].view(np.uint64))
