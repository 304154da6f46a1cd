"""The multigrid-preconditioned CG path (PT_FLAG_MULTIGRID) against the FP64 CG
oracle and the contract the red-black SOR path keeps: the same FP64 bar,
non-interior pixels equal to the anchor bit for bit, the report's history and
stop reasons, the iteration cap, warm starts with the anchor as fallback, and
byte-identical reruns.

Tolerance: at relative residual t the distance to the exact discrete solution
is at most ||r|| / lambda_min(A); the comparisons below use tight tolerances
where that bound is far below the 1e-6 asserted."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L(cuda_lib):
    from paintop_b200 import _lib
    return _lib


def random_problem(seed, w, h, c, density=0.6):
    rng = np.random.default_rng(seed)
    src = rng.random(w * h * c).astype(np.float32)
    tgt = rng.random(w * h * c).astype(np.float32)
    yy, xx = np.mgrid[0:h, 0:w]
    mask = (((xx - w / 2) / (0.4 * w)) ** 2 + ((yy - h / 2) / (0.4 * h)) ** 2 <= 1.0)
    mask = (mask & (rng.random((h, w)) < density + 0.4)).astype(np.float32).reshape(-1)
    return src, tgt, mask


@pytest.mark.parametrize("w,h,c,lam", [(150, 90, 2, 0.05), (257, 129, 3, 0.0), (64, 300, 1, 0.01)])
def test_multigrid_matches_the_cg_oracle(ctx, oracle, L, w, h, c, lam):
    src, tgt, mask = random_problem(7, w, h, c)
    out, per, worst = ctx.solve(src, tgt, mask, w, h, c, lam=lam, max_iterations=500, tolerance=1e-9,
                                flags=L.PT_FLAG_MULTIGRID)
    cg, ach = oracle.cg_blend_channels(src, tgt, mask, c, w, h, lam=lam, rel_tol=1e-13)
    assert np.abs(out.astype(np.float64) - cg).max() <= 1e-6
    for r in per:
        assert r["converged"] and r["stop_reason"] == "converged" and r["final_residual"] <= 1e-9
        assert r["iterations"] < 80, r["iterations"]
        assert len(r["residual_history"]) == r["iterations"]
        assert r["final_residual"] == r["residual_history"][-1]
        assert r["omega_used"] == 1.25
    # non-interior pixels are the target, bit for bit
    inter = np.zeros((h, w), bool)
    inter[1:-1, 1:-1] = mask.reshape(h, w)[1:-1, 1:-1] > 0.5
    keep = np.repeat(~inter.reshape(-1), c)
    assert np.array_equal(out.view(np.uint32)[keep], tgt.view(np.uint32)[keep])


def test_multigrid_reruns_are_byte_identical(ctx, L):
    src, tgt, mask = random_problem(3, 200, 160, 3)
    a = ctx.solve(src, tgt, mask, 200, 160, 3, lam=0.0, max_iterations=400, tolerance=1e-7, flags=L.PT_FLAG_MULTIGRID)
    b = ctx.solve(src, tgt, mask, 200, 160, 3, lam=0.0, max_iterations=400, tolerance=1e-7, flags=L.PT_FLAG_MULTIGRID)
    assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32))
    assert [r["residual_history"] for r in a[1]] == [r["residual_history"] for r in b[1]]


def test_multigrid_agrees_with_sor_at_the_same_bar(ctx, L):
    src, tgt, mask = random_problem(5, 180, 140, 2)
    mg, pm, _ = ctx.solve(src, tgt, mask, 180, 140, 2, lam=0.02, max_iterations=20000, tolerance=1e-8,
                          flags=L.PT_FLAG_MULTIGRID)
    sor, ps, _ = ctx.solve(src, tgt, mask, 180, 140, 2, lam=0.02, max_iterations=20000, tolerance=1e-8, omega=1.9)
    assert all(r["converged"] for r in pm + ps)
    assert np.abs(mg.astype(np.float64) - sor).max() <= 1e-5
    assert all(m["iterations"] * 10 < s["iterations"] for m, s in zip(pm, ps))


@pytest.mark.parametrize("cap", [1, 2, 5])
def test_multigrid_stops_at_the_cap(ctx, L, cap):
    src, tgt, mask = random_problem(cap, 120, 100, 2)
    _, per, worst = ctx.solve(src, tgt, mask, 120, 100, 2, lam=0.0, max_iterations=cap, tolerance=1e-12,
                              flags=L.PT_FLAG_MULTIGRID)
    for r in per:
        assert r["iterations"] == cap and r["stop_reason"] == "max-iterations" and not r["converged"]
        assert len(r["residual_history"]) == cap
        assert r["final_residual"] == r["residual_history"][-1]


def test_multigrid_degenerate_and_satisfied_systems(ctx, L):
    # no interior (W < 3): nothing to solve, zero iterations, output = target
    src, tgt, mask = random_problem(1, 2, 40, 1)
    out, per, _ = ctx.solve(src, tgt, np.ones(80, np.float32), 2, 40, 1, flags=L.PT_FLAG_MULTIGRID)
    assert per[0]["iterations"] == 0 and per[0]["converged"]
    assert np.array_equal(out.view(np.uint32), tgt.view(np.uint32))
    # an already satisfied system (source = target = constant): r0 = 0
    w = h = 16
    flat = np.full(w * h, 0.5, np.float32)
    out, per, _ = ctx.solve(flat, flat.copy(), np.ones(w * h, np.float32), w, h, 1, flags=L.PT_FLAG_MULTIGRID)
    assert per[0]["iterations"] == 0 and per[0]["converged"] and per[0]["final_residual"] == 0.0


def test_multigrid_warm_start(ctx, oracle, L):
    w, h, c = 160, 120, 2
    src, tgt, mask = random_problem(11, w, h, c)
    plain, pp, _ = ctx.solve(src, tgt, mask, w, h, c, lam=0.1, max_iterations=500, tolerance=1e-9,
                             flags=L.PT_FLAG_MULTIGRID)
    # a guess equal to the anchor is not better: the anchor start is used, bit for bit
    same, ps, _ = ctx.solve(src, tgt, mask, w, h, c, lam=0.1, max_iterations=500, tolerance=1e-9,
                            flags=L.PT_FLAG_MULTIGRID | L.PT_FLAG_WARM_START, initial_guess=tgt.copy())
    assert np.array_equal(plain.view(np.uint32), same.view(np.uint32))
    assert all(r["warm_start"] == 0 for r in ps)
    # the exact solution as the guess converges in fewer iterations, same absolute bar
    cg, _ = oracle.cg_blend_channels(src, tgt, mask, c, w, h, lam=0.1, rel_tol=1e-13)
    good, pg, _ = ctx.solve(src, tgt, mask, w, h, c, lam=0.1, max_iterations=500, tolerance=1e-9,
                            flags=L.PT_FLAG_MULTIGRID | L.PT_FLAG_WARM_START, initial_guess=cg.astype(np.float32))
    assert all(g["warm_start"] == 1 and g["iterations"] < p["iterations"] for g, p in zip(pg, pp))
    assert np.abs(good.astype(np.float64) - cg).max() <= 1e-6


def test_multigrid_batch_and_flag_agreement(ctx, L):
    probs = []
    for k, (w, h) in enumerate([(90, 70), (130, 60), (40, 40)]):
        s, t, m = random_problem(20 + k, w, h, 2)
        probs.append(dict(source=s, target=t, mask=m, width=w, height=h, channels=2, lam=0.0,
                          max_iterations=300, tolerance=1e-8, flags=L.PT_FLAG_MULTIGRID))
    res = ctx.solve_batch(probs)
    for pr, (o, per, _) in zip(probs, res):
        assert all(r["converged"] for r in per)
        one, _, _ = ctx.solve(pr["source"], pr["target"], pr["mask"], pr["width"], pr["height"], 2,
                              max_iterations=300, tolerance=1e-8, flags=L.PT_FLAG_MULTIGRID)
        assert np.array_equal(np.asarray(o).view(np.uint32), one.view(np.uint32))
    probs[1]["flags"] = 0
    with pytest.raises(L.CudaError) as e:
        ctx.solve_batch(probs)
    assert e.value.status == L.PT_INVALID_ARG


def test_multigrid_device_pointers_and_large_regions(ctx, L):
    """4096 x 4096 RGB with 8 polygons (the learned-warm-start workload) from
    device buffers: converged at 1e-6 in tens of iterations where red-black SOR
    takes over two thousand sweeps."""
    import torch
    from paintop_b200 import synth
    inst = synth.multi_4096(1)
    W, H, C = inst.width, inst.height, inst.channels
    g = torch.as_tensor(inst.source, device="cuda").contiguous()
    a = torch.as_tensor(inst.target, device="cuda").contiguous()
    m = torch.as_tensor(inst.mask, device="cuda").contiguous()
    out = torch.empty_like(g)
    p = L.PtProblem(W, H, C, g.data_ptr(), a.data_ptr(), m.data_ptr(), 0.0, 2000, 1e-6, 1.8,
                    L.PT_FLAG_DEVICE_POINTERS | L.PT_FLAG_MULTIGRID, None)
    reps = (L.PtReport * (C + 1))()
    import ctypes as Ct
    torch.cuda.synchronize()
    st = L.lib().pt_poisson_solve(ctx.h, Ct.byref(p), out.data_ptr(), reps, None)
    assert st == L.PT_OK, ctx.last_error()
    for c in range(C):
        assert reps[c].converged and reps[c].final_residual <= 1e-6
        assert reps[c].iterations < 100, reps[c].iterations


@pytest.mark.parametrize("case", ["nan_source_interior", "inf_target_boundary"])
def test_multigrid_non_finite_residual_stalls(ctx, L, case):
    """A NaN residual cannot improve: the multigrid path stops at once as
    stalled with a NaN final residual and non-finite interior pixels (the
    reference's outcome for a poisoned system), while non-interior pixels stay
    the target's."""
    w = h = 16
    rng = np.random.default_rng(1)
    src = rng.random(w * h).astype(np.float32)
    tgt = rng.random(w * h).astype(np.float32)
    mask = np.zeros((h, w), np.float32)
    mask[4:12, 4:12] = 1
    mask = mask.reshape(-1)
    if case == "nan_source_interior":
        src[8 * w + 8] = np.nan
    else:
        tgt[3 * w + 8] = np.inf
    out, per, worst = ctx.solve(src, tgt, mask, w, h, 1, max_iterations=2000, tolerance=1e-6,
                                flags=L.PT_FLAG_MULTIGRID)
    assert worst["stop_reason"] == "stalled" and not worst["converged"] and np.isnan(worst["final_residual"])
    inter = mask.reshape(h, w) > 0.5
    assert not np.isfinite(out.reshape(h, w)[inter]).any()
    assert np.array_equal(out.reshape(h, w)[~inter].view(np.uint32), tgt.reshape(h, w)[~inter].view(np.uint32))


def test_multigrid_mixed_batch_equals_solving_alone(ctx, oracle, L):
    """A batch of unlike problems shares every launch -- one to three channels,
    lambda, tolerance and iteration cap per problem, an image no larger than
    the coarsest level (8 x 8), no interior (2 x 40), no channels, a warm start
    and a NaN -- and each problem's output, reports and residual history are
    bit for bit those of solving it alone."""
    specs = [  # seed, w, h, c, lambda, tolerance, cap, kind
        (31, 150, 90, 3, 0.0, 1e-8, 300, None),
        (32, 8, 8, 1, 0.0, 1e-9, 300, None),
        (33, 2, 40, 2, 0.0, 1e-6, 300, None),
        (34, 257, 129, 2, 0.05, 1e-7, 300, None),
        (35, 60, 30, 1, 0.0, 1e-12, 3, None),
        (36, 40, 50, 0, 0.0, 1e-6, 300, None),
        (37, 120, 100, 2, 0.1, 1e-9, 300, "warm"),
        (38, 16, 16, 1, 0.0, 1e-6, 300, "nan"),
        (39, 33, 500, 3, 0.01, 1e-6, 300, None),
    ]
    probs = []
    for seed, w, h, c, lam, tol, cap, kind in specs:
        if c == 0:
            s = t = np.zeros(0, np.float32)
            m = np.ones(w * h, np.float32)
        else:
            s, t, m = random_problem(seed, w, h, c)
        pr = dict(source=s, target=t, mask=m, width=w, height=h, channels=c, lam=lam, max_iterations=cap,
                  tolerance=tol, flags=L.PT_FLAG_MULTIGRID)
        if kind == "warm":
            cg, _ = oracle.cg_blend_channels(s, t, m, c, w, h, lam=lam, rel_tol=1e-13)
            pr["initial_guess"] = cg.astype(np.float32)
        if kind == "nan":
            s[8 * w + 8] = np.nan
        probs.append(pr)
    res = ctx.solve_batch(probs, want_history=True)
    for pr, (out, per, worst), spec in zip(probs, res, specs):
        c = pr["channels"]
        if c == 0:
            assert worst["converged"] and worst["iterations"] == 0
            continue
        one, per1, worst1 = ctx.solve(pr["source"], pr["target"], pr["mask"], pr["width"], pr["height"], c,
                                      lam=pr["lam"], max_iterations=pr["max_iterations"], tolerance=pr["tolerance"],
                                      flags=pr["flags"], initial_guess=pr.get("initial_guess"))
        assert np.array_equal(np.asarray(out).view(np.uint32), one.view(np.uint32)), spec
        for a, b in zip(per, per1):
            for key in ("iterations", "stop_reason", "converged", "refinements", "warm_start"):
                assert a[key] == b[key], (spec, key)
            assert np.array_equal(np.float64(a["final_residual"]), np.float64(b["final_residual"]), equal_nan=True)
            assert np.array_equal(np.asarray(a["residual_history"]), np.asarray(b["residual_history"]),
                                  equal_nan=True), spec
    by_kind = {sp[7]: r for sp, r in zip(specs, res)}
    assert all(r["warm_start"] == 1 and r["converged"] for r in by_kind["warm"][1])
    assert by_kind["nan"][2]["stop_reason"] == "stalled"
    assert res[4][2]["stop_reason"] == "max-iterations" and res[4][2]["iterations"] == 3
    assert all(r["converged"] for k in (0, 1, 2, 3, 8) for r in res[k][1])


@pytest.mark.parametrize("op_name,lam", [("PoissonBlend", 0.0), ("ScreenedPoisson", 0.05)])
def test_multigrid_implementation_through_the_op(ctx, L, op_name, lam):
    """cuda.multigrid@1: the two Poisson ops through the op layer with
    PT_FLAG_MULTIGRID (pt_op_compute_ex) return the flagged solve's candidate
    bit for bit and SolverData from its worst channel, with steps counting CG
    iterations -- far fewer than the default implementation's sweeps for the
    same bar."""
    from paintop_b200 import ops
    cls = getattr(ops, op_name)
    w, h, c = 120, 90, 3
    src, tgt, mask = random_problem(41, w, h, c)
    op = cls(multigrid=True)
    assert op.implementation_id == "cuda.multigrid@1" and cls().implementation_id == "cuda.poisson@1"
    names = cls.PORTS
    inputs = {names[0]: ops.image_value(w, h, c, src), names[1]: ops.image_value(w, h, c, tgt),
              names[2]: ops.mask_value(w, h, mask)}
    params = {"tolerance": 1e-7, "max_iterations": 5000}
    if lam:
        params["lambda"] = lam
    out = op.compute(inputs, params)
    one, per, worst = ctx.solve(src, tgt, mask, w, h, c, lam=lam, max_iterations=5000, tolerance=1e-7,
                                flags=L.PT_FLAG_MULTIGRID)
    cand = np.asarray(out["candidate"].samples, np.float32)
    assert np.array_equal(cand.view(np.uint32), one.view(np.uint32))
    sd = out["report"].report.solver
    assert sd.steps == sd.iterations == worst["iterations"] and sd.converged
    assert sd.stop_reason == "converged" and sd.final_residual == worst["final_residual"] <= 1e-7
    assert sd.residual_history == worst["residual_history"]
    assert sd.kind == ("poisson" if lam == 0 else "screened-poisson")
    sor = cls().compute(inputs, params)
    assert sor["report"].report.solver.converged and sor["report"].report.solver.steps > 5 * sd.steps
    assert np.abs(cand.astype(np.float64) - np.asarray(sor["candidate"].samples, np.float64)).max() <= 1e-4
