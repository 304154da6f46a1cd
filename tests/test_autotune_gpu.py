"""The tile-configuration autotuner (pt_autotune, paintop_b200/tune.py) on the
GPU: the tuned choice is written to the table file and read back by later
solves of the same shape; re-tuning the same shapes keeps the table unless a
configuration beats the incumbent by the stated margin; solves under the table
are byte-identical across reruns; the tuned configuration's result agrees with
the built-in default's within the solver-agreement bound of the other parity
tests. The compiled-in B200 entries parse and name valid configurations."""
import ctypes as C
import os
import re

import numpy as np
import pytest

TOL_ABS = 1e-6  # agreement between two solves of the same system to rel-res 1e-9
MARGIN = 0.05   # autotune.cpp, kReplaceMargin
NCFG = 5        # tile configurations (pt_tile_config_count)


def _problems():
    # a shape no other test uses (1000x900 RGB, lambda 0.01): the entry this
    # test adds to the process's table touches no other test
    from paintop_b200 import synth
    inst = synth.screened_2048(5, size=1000)
    src = inst.source[:900, :, :3].copy()
    tgt = inst.target[:900, :, :3].copy()
    mask = inst.mask[:900].copy()
    return [dict(width=1000, height=900, channels=3, source=src, target=tgt, mask=mask, lam=0.01,
                 max_iterations=2000, tolerance=1e-9, omega=1.8, flags=0)]


def _table(path):
    out = {}
    if os.path.exists(path):
        for line in open(path):
            k, v = line.split()
            out[int(k, 16)] = int(v)
    return out


@pytest.mark.gpu
def test_autotune_writes_reads_back_and_is_stable(ctx, tmp_path):
    from paintop_b200 import tune
    path = str(tmp_path / "tune_table.txt")
    old = os.environ.get("PAINTOP_CUDA_TUNE_TABLE")
    os.environ["PAINTOP_CUDA_TUNE_TABLE"] = path
    try:
        probs = _problems()
        key = tune.shape_key(probs)
        cfg1, ms1, conv, _ = tune.autotune(ctx, probs, repeats=2)
        assert conv and len(ms1) == NCFG and all(t > 0 for t in ms1)
        assert _table(path)[key] == cfg1
        # re-tuning keeps the entry unless another configuration now beats it
        # by more than the margin
        cfg2, ms2, _, _ = tune.autotune(ctx, probs, repeats=2)
        assert cfg2 == cfg1 or min(ms2) < (1.0 - MARGIN) * ms2[cfg1]
        assert _table(path)[key] == cfg2
        # a plain solve of the same shape reads the entry, and reruns are byte-identical
        p = probs[0]
        outs = []
        for _ in range(2):
            out, per, _ = ctx.solve(p["source"], p["target"], p["mask"], 1000, 900, 3, lam=0.01,
                                    max_iterations=2000, tolerance=1e-9)
            assert ctx.last_config() == cfg2
            assert all(r["converged"] for r in per)
            outs.append(out)
        assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
        # the tuned configuration agrees with every other one on the same system
        for cfg in range(NCFG):
            ctx.set_config(cfg)
            try:
                other, per, _ = ctx.solve(p["source"], p["target"], p["mask"], 1000, 900, 3, lam=0.01,
                                          max_iterations=2000, tolerance=1e-9)
            finally:
                ctx.set_config(-1)
            assert np.abs(other.astype(np.float64) - outs[0]).max() <= TOL_ABS
    finally:
        if old is None:
            os.environ.pop("PAINTOP_CUDA_TUNE_TABLE", None)
        else:
            os.environ["PAINTOP_CUDA_TUNE_TABLE"] = old


def test_compiled_in_table_entries_are_valid(cuda_lib):
    from paintop_b200 import tune
    text = open(tune.INC).read()
    entries = re.findall(r"\{0x([0-9a-f]{8})u, (\d+)\}", text)
    n = int(cuda_lib.pt_tile_config_count())
    for k, v in entries:
        assert 0 <= int(v) < n
    keys = [int(k, 16) for k, _ in entries]
    assert len(keys) == len(set(keys))
