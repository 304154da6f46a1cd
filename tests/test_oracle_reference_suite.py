"""The reference's own known-answer suites, run against the C oracle.

Ports of crates/paintop-cpu/src/poisson/tests.rs:54-242,
poisson/characterization.rs:139-284, poisson_blend/tests.rs:101-277 and
screened_poisson/tests.rs:125-293 (the numerical assertions; manifest and
registry checks have no counterpart here). The reference publishes no golden
arrays for this path, so these analytic answers plus the bit-for-bit agreement
with the pure-Python restatement are what pin the oracle.
"""
import numpy as np

DEFAULT_MAX_ITERATIONS = 2000   # poisson_blend.rs:68
DEFAULT_TOLERANCE = 1e-6        # poisson_blend.rs:74
OMEGA = 1.8                     # poisson_blend.rs:78


def controls():
    # poisson/tests.rs:27-33
    return dict(max_iterations=5000, tolerance=1e-10, omega=1.9)


def laplace_system(w, h, anchor, lam):
    # poisson/tests.rs:38-52
    cells = np.zeros(w * h, dtype=np.uint8)
    for row in range(1, max(h - 1, 1)):
        for col in range(1, max(w - 1, 1)):
            cells[row * w + col] = 1
    return cells, np.zeros(w * h), np.asarray(anchor, dtype=np.float64), lam


def solve(oracle, w, h, cells, rhs, anchor, lam, c):
    return oracle.solve(w, h, cells, rhs, anchor, lam, c["max_iterations"], c["tolerance"],
                        c["omega"])


# ---- poisson/tests.rs ---------------------------------------------------------------

def test_constant_boundary_converges_to_constant(oracle):
    w, h = 7, 5
    cells, rhs, anchor, lam = laplace_system(w, h, np.full(w * h, 3.5), 0.0)
    field, rep = solve(oracle, w, h, cells, rhs, anchor, lam, controls())
    assert rep.converged and rep.stop_reason == "converged"
    assert np.all(np.abs(field[cells == 1] - 3.5) < 1e-6)


def test_linear_ramp_boundary_recovers_linear_solution(oracle):
    w, h = 9, 9
    yy, xx = np.mgrid[0:h, 0:w]
    anchor = (2.0 * xx + 3.0 * yy).reshape(-1).astype(np.float64)
    cells, rhs, anchor, lam = laplace_system(w, h, anchor, 0.0)
    field, rep = solve(oracle, w, h, cells, rhs, anchor, lam, controls())
    assert rep.converged
    assert np.all(np.abs(field - anchor)[cells == 1] < 1e-5)


def test_residual_history_decreases_and_records_metrics(oracle):
    w, h = 11, 11
    anchor = np.zeros(w * h)
    anchor[:w] = 10.0
    cells, rhs, anchor, lam = laplace_system(w, h, anchor, 0.0)
    _, rep = solve(oracle, w, h, cells, rhs, anchor, lam, controls())
    assert rep.iterations >= 1
    assert len(rep.residual_history) == rep.iterations
    assert all(np.isfinite(r) and r >= 0 for r in rep.residual_history)
    assert rep.final_residual < rep.residual_history[0]
    assert rep.converged and rep.final_residual <= rep.tolerance


def test_reruns_are_bit_identical(oracle):
    w, h = 13, 8
    anchor = np.sin(np.arange(w * h, dtype=np.float64))
    cells, rhs, anchor, lam = laplace_system(w, h, anchor, 0.0)
    a, ra = solve(oracle, w, h, cells, rhs, anchor, lam, controls())
    b, rb = solve(oracle, w, h, cells, rhs, anchor, lam, controls())
    assert np.array_equal(a, b)
    assert ra.iterations == rb.iterations and ra.residual_history == rb.residual_history


def test_max_iterations_stop_reason(oracle):
    w, h = 15, 15
    anchor = np.zeros(w * h)
    anchor[:w] = 100.0
    cells, rhs, anchor, lam = laplace_system(w, h, anchor, 0.0)
    _, rep = solve(oracle, w, h, cells, rhs, anchor, lam,
                   dict(max_iterations=2, tolerance=1e-12, omega=1.0))
    assert not rep.converged and rep.stop_reason == "max-iterations" and rep.iterations == 2


def test_large_lambda_snaps_to_anchor(oracle):
    w, h = 9, 9
    yy, xx = np.mgrid[0:h, 0:w]
    anchor = (xx + yy).reshape(-1).astype(np.float64)
    cells, rhs, anchor, _ = laplace_system(w, h, anchor, 1e6)
    field, _ = solve(oracle, w, h, cells, rhs, anchor, 1e6, controls())
    assert np.all(np.abs(field - anchor)[cells == 1] < 1e-2)


# ---- poisson/characterization.rs ----------------------------------------------------

def build_system(oracle, edge):
    # characterization.rs:58-91
    lo, hi = edge // 4, edge - edge // 4
    mask = np.zeros((edge, edge), dtype=np.float32)
    mask[lo:hi, lo:hi] = 1.0
    cells = oracle.classify_cells(mask, edge, edge)
    yy, xx = np.mgrid[0:edge, 0:edge].astype(np.float64)
    source = 0.001 * (xx * xx + yy * yy)  # x.mul_add(x, y*y) is exact here
    from oracle import pyref
    src = source.reshape(-1).tolist()
    rhs = np.zeros(edge * edge)
    for idx in np.flatnonzero(cells == 1):
        rhs[idx] = pyref.guidance_laplacian(src, idx % edge, idx // edge, edge, edge)
    return cells, rhs, np.full(edge * edge, 0.25)


def test_characterization_reruns_bit_identical_and_bounded(oracle):
    for edge in (32, 64, 128):
        cells, rhs, anchor = build_system(oracle, edge)
        c = dict(max_iterations=5000, tolerance=1e-6, omega=1.8)
        a, ra = solve(oracle, edge, edge, cells, rhs, anchor, 0.0, c)
        b, rb = solve(oracle, edge, edge, cells, rhs, anchor, 0.0, c)
        assert np.array_equal(a, b)
        assert np.isfinite(ra.final_residual) and ra.final_residual >= 0
        assert ra.iterations <= 5000


def test_runaway_iterations_stop_at_the_cap(oracle):
    cells, rhs, anchor = build_system(oracle, 64)
    _, rep = solve(oracle, 64, 64, cells, rhs, anchor, 0.0,
                   dict(max_iterations=7, tolerance=1e-30, omega=1.0))
    assert rep.iterations == 7 and rep.stop_reason == "max-iterations" and not rep.converged


def test_no_interior_region_stops_immediately(oracle):
    edge = 32
    cells = np.zeros(edge * edge, dtype=np.uint8)
    anchor = np.full(edge * edge, 0.5)
    field, rep = solve(oracle, edge, edge, cells, np.zeros(edge * edge), anchor, 0.0,
                       dict(max_iterations=1000, tolerance=1e-8, omega=1.5))
    assert rep.iterations == 0 and rep.stop_reason == "converged" and rep.converged
    assert rep.residual_history == []
    assert np.array_equal(field, anchor)


# ---- poisson_blend/tests.rs (op level: defaults, omega 1.8) -------------------------

def square_mask(w, h, lo, hi):
    m = np.zeros((h, w), dtype=np.float32)
    m[lo:hi, lo:hi] = 1.0
    return m.reshape(-1)


def blend(oracle, w, h, src, tgt, mask, params, lam=0.0):
    return oracle.blend_channels(np.asarray(src, np.float32), np.asarray(tgt, np.float32), mask, 1,
                                 w, h, params.get("max_iterations", DEFAULT_MAX_ITERATIONS),
                                 params.get("tolerance", DEFAULT_TOLERANCE),
                                 params.get("lambda", lam), OMEGA)


def test_blend_boundary_pixels_keep_the_target(oracle):
    w = h = 16
    tgt = np.full(w * h, 0.1, np.float32)
    mask = square_mask(w, h, 5, 11)
    out, _, _ = blend(oracle, w, h, np.full(w * h, 0.9), tgt, mask, {})
    assert np.array_equal(out[mask <= 0.5], tgt[mask <= 0.5])


def test_blend_uniform_source_over_uniform_target(oracle):
    w = h = 20
    mask = square_mask(w, h, 6, 14)
    out, rep, _ = blend(oracle, w, h, np.full(w * h, 0.7), np.full(w * h, 0.25), mask,
                        {"tolerance": 1e-8, "max_iterations": 5000})
    assert np.all(np.abs(out[mask > 0.5] - 0.25) < 1e-3)
    assert rep.converged


def test_blend_linear_gradient_reproduced(oracle):
    w = h = 24
    src = np.tile(np.arange(w, dtype=np.float32), h)
    mask = square_mask(w, h, 6, 18)
    out, _, _ = blend(oracle, w, h, src, src.copy(), mask, {"tolerance": 1e-9, "max_iterations": 8000})
    o = out.reshape(h, w)
    m = mask.reshape(h, w)
    for row in range(7, 17):
        for col in range(7, 17):
            if m[row, col] > 0.5:
                assert abs((o[row, col] - o[row, col - 1]) - 1.0) < 5e-2


def test_blend_reruns_bit_identical(oracle):
    w, h = 18, 14
    src = (((np.arange(w * h) * 7) % 13) / 13.0).astype(np.float32)
    tgt = np.full(w * h, 0.3, np.float32)
    mask = square_mask(w, h, 4, 12)
    a, _, _ = blend(oracle, w, h, src, tgt, mask, {"max_iterations": 200})
    b, _, _ = blend(oracle, w, h, src, tgt, mask, {"max_iterations": 200})
    assert np.array_equal(a, b)


def test_blend_report_carries_iterative_metrics(oracle):
    w = h = 16
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    src = (np.float32(0.01) * (xx * xx + yy * yy)).reshape(-1)
    mask = square_mask(w, h, 4, 12)
    _, rep, _ = blend(oracle, w, h, src, np.full(w * h, 0.2), mask,
                      {"max_iterations": 3, "tolerance": 1e-12})
    assert rep.iterations == 3 and rep.stop_reason == "max-iterations" and not rep.converged
    assert len(rep.residual_history) == 3 and np.isfinite(rep.final_residual)


# ---- screened_poisson/tests.rs -------------------------------------------------------

def ramp(w, h):
    return np.tile(np.arange(w, dtype=np.float32), h)


def bump(w, h):
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    return (np.float32(0.02) * (xx * xx + yy * yy)).reshape(-1)


def test_screened_lambda_zero_recovers_guidance_gradient(oracle):
    w = h = 24
    g = ramp(w, h)
    mask = square_mask(w, h, 6, 18)
    out, _, _ = blend(oracle, w, h, g, g.copy(), mask,
                      {"lambda": 0.0, "tolerance": 1e-9, "max_iterations": 8000})
    o = out.reshape(h, w)
    for row in range(7, 17):
        for col in range(7, 17):
            assert abs((o[row, col] - o[row, col - 1]) - 1.0) < 5e-2


def test_screened_large_lambda_snaps_to_anchor(oracle):
    w = h = 20
    mask = square_mask(w, h, 6, 14)
    out, _, _ = blend(oracle, w, h, bump(w, h), np.full(w * h, 0.4), mask,
                      {"lambda": 1e6, "tolerance": 1e-9, "max_iterations": 8000})
    assert np.all(np.abs(out[mask > 0.5] - 0.4) < 1e-2)


def test_screened_larger_lambda_moves_closer_to_anchor(oracle):
    w = h = 20
    mask = square_mask(w, h, 6, 14)
    centre = (h // 2) * w + (w // 2)

    def dist(lam):
        out, _, _ = blend(oracle, w, h, bump(w, h), np.full(w * h, 0.5), mask,
                          {"lambda": lam, "tolerance": 1e-8, "max_iterations": 8000})
        return abs(out[centre] - 0.5)

    assert dist(10.0) < dist(0.01)


def test_screened_boundary_pixels_keep_the_anchor(oracle):
    w = h = 16
    anchor = np.full(w * h, 0.3, np.float32)
    mask = square_mask(w, h, 5, 11)
    out, _, _ = blend(oracle, w, h, ramp(w, h), anchor, mask, {"lambda": 5.0})
    assert np.array_equal(out[mask <= 0.5], anchor[mask <= 0.5])


def test_screened_report_carries_metrics(oracle):
    w = h = 16
    mask = square_mask(w, h, 4, 12)
    _, rep, _ = blend(oracle, w, h, bump(w, h), np.full(w * h, 0.2), mask,
                      {"lambda": 1.0, "max_iterations": 3, "tolerance": 1e-12})
    assert rep.iterations == 3 and len(rep.residual_history) == 3 and rep.tolerance > 0
