"""Pin the C oracle: it must agree bit for bit with the independent pure-Python
restatement (exactly-rounded fma) of crates/paintop-cpu/src/poisson.rs and
poisson_blend.rs on small grids, including the edge cases the reference code
has (W or H < 3, empty masks, masks touching the border, lambda > 0, stalls).
"""
import numpy as np
import pytest

from oracle import pyref


def _case(rng, w, h, c, density, lam, omega, max_it, tol):
    src = rng.random(w * h * c).astype(np.float32)
    tgt = rng.random(w * h * c).astype(np.float32)
    mask = (rng.random(w * h) < density).astype(np.float32)
    return src, tgt, mask


CASES = [
    # w, h, c, mask density, lambda, omega, max_iterations, tolerance
    (9, 7, 2, 0.7, 0.3, 1.7, 40, 1e-9),
    (8, 8, 1, 1.0, 0.0, 1.9, 60, 1e-6),
    (5, 6, 3, 0.5, 2.0, 1.0, 25, 1e-12),
    (2, 9, 1, 1.0, 0.0, 1.8, 10, 1e-6),     # W < 3: all boundary
    (9, 2, 1, 1.0, 0.0, 1.8, 10, 1e-6),     # H < 3: all boundary
    (7, 7, 1, 0.0, 0.0, 1.8, 10, 1e-6),     # empty mask
    (11, 5, 1, 0.9, 1e6, 1.8, 30, 1e-9),    # huge lambda
    (6, 6, 2, 0.8, 0.0, 1.5, 0, 1e-6),      # zero iterations allowed at solver level
]


@pytest.mark.parametrize("case", CASES)
def test_c_oracle_matches_pure_python_bit_for_bit(oracle, case):
    w, h, c, dens, lam, omega, max_it, tol = case
    rng = np.random.default_rng(hash(case) & 0xFFFF)
    src, tgt, mask = _case(rng, w, h, c, dens, lam, omega, max_it, tol)
    out, worst, per = oracle.blend_channels(src, tgt, mask, c, w, h, max_it, tol, lam, omega)
    pout, pworst = pyref.blend_channels(src.tolist(), tgt.tolist(), mask.tolist(), c, w, h,
                                        max_it, tol, lam, omega)
    assert np.array_equal(out.view(np.uint32), np.array(pout, dtype=np.float32).view(np.uint32))
    assert worst.iterations == pworst["iterations"]
    assert worst.stop_reason == pworst["stop_reason"]
    assert worst.converged == pworst["converged"]
    assert worst.residual_history == pworst["residual_history"]
    assert worst.final_residual == pworst["final_residual"] or (
        np.isnan(worst.final_residual) and np.isnan(pworst["final_residual"]))


def test_stall_rule_is_pinned(oracle):
    # A system whose residual cannot fall below the f64 floor: tolerance far
    # below it must end by the stall rule (poisson.rs:219-228), identically in
    # both restatements.
    w, h = 6, 5
    rng = np.random.default_rng(7)
    src = rng.random(w * h).astype(np.float32)
    tgt = rng.random(w * h).astype(np.float32)
    mask = np.ones(w * h, dtype=np.float32)
    out, worst, _ = oracle.blend_channels(src, tgt, mask, 1, w, h, 3000, 1e-300, 0.0, 1.0)
    pout, pworst = pyref.blend_channels(src.tolist(), tgt.tolist(), mask.tolist(), 1, w, h, 3000,
                                        1e-300, 0.0, 1.0)
    assert worst.stop_reason == "stalled" == pworst["stop_reason"]
    assert worst.iterations == pworst["iterations"]
    assert worst.residual_history == pworst["residual_history"]
    assert np.array_equal(out, np.array(pout, dtype=np.float32))


def test_worst_channel_rule(oracle):
    # worse_of: more iterations, then the larger final residual (poisson_blend.rs:240-246)
    w, h, c = 10, 9, 3
    rng = np.random.default_rng(3)
    src = rng.random(w * h * c).astype(np.float32)
    tgt = rng.random(w * h * c).astype(np.float32)
    src[1::3] = 0.5  # channel 1: flat source, converges differently
    mask = np.ones(w * h, dtype=np.float32)
    _, worst, per = oracle.blend_channels(src, tgt, mask, c, w, h, 500, 1e-8, 0.0, 1.8)
    key = [(p.iterations, p.final_residual) for p in per]
    best = 0
    for k in range(1, c):
        if key[k] > key[best]:
            best = k
    assert (worst.iterations, worst.final_residual) == key[best]
