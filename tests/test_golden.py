"""The committed golden fixtures (tests/golden/, made by make_golden.py from the
pinned oracle): the oracle must reproduce them bit for bit, and the cuda
backend must match their converged outputs within the stated tolerance."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import CASES

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "poisson_cases.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("case", [c[0] for c in CASES])
def test_oracle_reproduces_golden(oracle, golden, case):
    w, h, c, lam, omega, max_it, tol = golden[f"{case}/controls"]
    w, h, c, max_it = int(w), int(h), int(c), int(max_it)
    out, worst, per = oracle.blend_channels(golden[f"{case}/source"], golden[f"{case}/target"],
                                            golden[f"{case}/mask"], c, w, h, max_it, tol, lam,
                                            omega)
    assert np.array_equal(out.view(np.uint32), golden[f"{case}/out"].view(np.uint32))
    assert [p.iterations for p in per] == golden[f"{case}/iterations"].tolist()
    for i, p in enumerate(per):
        hist = golden[f"{case}/history"][i, :p.iterations]
        assert np.array_equal(np.array(p.residual_history), hist)


@pytest.mark.gpu
@pytest.mark.parametrize("case", [c[0] for c in CASES])
def test_cuda_matches_golden(ctx, golden, case):
    w, h, c, lam, omega, max_it, tol = golden[f"{case}/controls"]
    w, h, c, max_it = int(w), int(h), int(c), int(max_it)
    src, tgt, mask = golden[f"{case}/source"], golden[f"{case}/target"], golden[f"{case}/mask"]
    out, per, worst = ctx.solve(src, tgt, mask, w, h, c, lam=lam, max_iterations=max_it,
                                tolerance=tol, omega=omega)
    ref = golden[f"{case}/out"]
    stops = golden[f"{case}/stop"].tolist()
    for k, r in enumerate(per):
        assert len(r["residual_history"]) == r["iterations"]
        if stops[k] == 1:  # the reference hit the cap: the cuda backend hits it too
            assert r["iterations"] == max_it and r["stop_reason"] == "max-iterations"
    if all(s == 0 for s in stops) and tol <= 1e-8:
        # both converged tightly: same fixed point
        assert np.abs(out - ref).max() <= 1e-5
    from oracle import oracle as O
    keep = np.repeat(O.classify_cells(mask, w, h) == 0, c)
    assert np.array_equal(out[keep].view(np.uint32), tgt[keep].view(np.uint32))
