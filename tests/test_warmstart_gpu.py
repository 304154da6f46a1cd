"""The learned warm start end to end on the GPU: the guess path (pooling,
network, upsampled correction), the device-side fallback to the plain start,
bit-identical resume of training, and the measured gain of a trained network
over the plain solve on held-out instances."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def ws(ctx, torch_cuda):
    from paintop_b200 import warmstart
    return warmstart


def oracle_solutions(oracle, g, a, m):
    """The FP64 tight oracle (multigrid-preconditioned CG to rel-res 1e-12) of
    each single-channel instance of a batch held in device tensors -> (B, H, W)
    float64 numpy array."""
    B, H, W = g.shape
    gs, as_, ms = (t.cpu().numpy() for t in (g, a, m))
    out = np.empty((B, H, W))
    for i in range(B):
        u, ach, _ = oracle.mgcg_blend_channels(gs[i].reshape(-1), as_[i].reshape(-1), ms[i].reshape(-1),
                                               1, W, H, lam=0.0, rel_tol=1e-12)
        assert ach[0] <= 1e-12
        out[i] = u.reshape(H, W)
    return out


def test_fallback_to_plain_start_is_exact(ctx, ws, torch_cuda):
    """A guess worse than the anchor is rejected on the device: the solve then
    matches the plain solve bit for bit and reports warm_start = False."""
    torch = torch_cuda
    g, a, m = ws.make_instances(4, 128, seed=21)
    up, rp = ws.solve_batch_device(ctx, g, a, m, tol=1e-6)
    bad = (a + 50.0).contiguous()
    uw, rw = ws.solve_batch_device(ctx, g, a, m, tol=1e-6, guess=bad)
    assert not any(r["warm_start"] for r in rw)
    assert [r["iterations"] for r in rw] == [r["iterations"] for r in rp]
    assert torch.equal(uw, up)
    nan = torch.full_like(a, float("nan"))
    un, rn = ws.solve_batch_device(ctx, g, a, m, tol=1e-6, guess=nan)
    assert not any(r["warm_start"] for r in rn) and torch.equal(un, up)


def test_exact_guess_is_used_and_same_bar(ctx, ws, torch_cuda, oracle):
    """The FP64 oracle's solution as the guess: it is used, the solve stops at
    the same absolute bar as the plain solve, in a fraction of its sweeps, and
    stays at the oracle's solution."""
    torch = torch_cuda
    g, a, m = ws.make_instances(4, 128, seed=22)
    tight = oracle_solutions(oracle, g, a, m)
    ref = torch.as_tensor(tight, dtype=torch.float32, device="cuda").contiguous()
    up, rp = ws.solve_batch_device(ctx, g, a, m, tol=1e-6)
    uw, rw = ws.solve_batch_device(ctx, g, a, m, tol=1e-6, guess=ref)
    assert all(r["warm_start"] and r["converged"] for r in rw)
    for p, w in zip(rp, rw):
        # the same absolute bar: both normalise by ||r(anchor)||
        assert w["initial_residual"] == p["initial_residual"]
        assert w["iterations"] < p["iterations"] // 4
    lm = ws.interior_mask(m).cpu().numpy()
    assert float(np.abs((uw.cpu().numpy() - tight) * lm).max()) < 1e-4


def test_guess_full_resolution_matches_forward(ctx, ws, torch_cuda):
    torch = torch_cuda
    net = ws.UNet(ctx, seed=31)
    g, a, m = ws.make_instances(1, 64, seed=23)
    want = (g + net.forward(net.features(g, a, m)))[0]
    got = ws.guess_image(net, g[0, :, :, None].contiguous(), a[0, :, :, None].contiguous(), m[0].contiguous(),
                         scale=1)[..., 0]
    assert torch.equal(got, want)


def test_guess_pooled_matches_host_emulation(ctx, ws, torch_cuda):
    """scale 4 on 96x112 RGB (pooled 24x28, padded to 24x32): pooled inputs
    are area averages, the guess is guidance + bilinear(correction)."""
    torch = torch_cuda
    net = ws.UNet(ctx, seed=32)
    H, W, Ch, s = 96, 112, 3, 4
    gg, aa, mm = ws.make_instances(Ch, 128, seed=24)
    g = gg[:, :H, :W].permute(1, 2, 0).contiguous()
    a = aa[:, :H, :W].permute(1, 2, 0).contiguous()
    m = mm[0, :H, :W].contiguous()
    got = ws.guess_image(net, g, a, m, scale=s).cpu().numpy()
    # host emulation: float32 block sums in row order, times 1/count
    Hc, Wc = 24, 32
    hv, wv = H // s, W // s

    def pool(img):
        out = np.zeros((Hc, Wc), np.float32)
        acc = np.zeros((hv, wv), np.float32)
        for dy in range(s):
            for dx in range(s):
                acc = acc + img[dy::s, dx::s]
        out[:hv, :wv] = acc * np.float32(1.0 / (s * s))
        return out

    gn, an, mn = g.cpu().numpy(), a.cpu().numpy(), m.cpu().numpy()
    cg = np.stack([pool(gn[..., c]) for c in range(Ch)])
    ca = np.stack([pool(an[..., c]) for c in range(Ch)])
    cm = np.stack([pool(mn) for _ in range(Ch)])
    T = lambda x: torch.as_tensor(x, device="cuda").contiguous()
    corr = net.forward(net.features(T(cg), T(ca), T(cm))).cpu().numpy().astype(np.float64)
    ys = np.clip((np.arange(H) + 0.5) / s - 0.5, 0, hv - 1)
    xs = np.clip((np.arange(W) + 0.5) / s - 0.5, 0, wv - 1)
    iy, ix = np.floor(ys).astype(int), np.floor(xs).astype(int)
    jy, jx = np.minimum(iy + 1, hv - 1), np.minimum(ix + 1, wv - 1)
    wy, wx = (ys - iy)[:, None], (xs - ix)[None, :]
    want = np.empty((H, W, Ch))
    for c in range(Ch):
        k = corr[c]
        top = k[iy][:, ix] + wx * (k[iy][:, jx] - k[iy][:, ix])
        bot = k[jy][:, ix] + wx * (k[jy][:, jx] - k[jy][:, ix])
        want[..., c] = gn[..., c] + top + wy * (bot - top)
    assert np.abs(got - want).max() < 1e-5


def test_guess_at_a_large_coarse_size(ctx, ws, torch_cuda):
    """A 1024x1024 RGB problem pooled by 2: the network runs on 512x512
    images, where the deeper layers meet other widths than in training."""
    torch = torch_cuda
    net = ws.UNet(ctx, seed=33)
    gg, aa, mm = ws.make_instances(3, 1024, seed=25)
    g = gg.permute(1, 2, 0).contiguous()
    a = aa.permute(1, 2, 0).contiguous()
    m = mm[0].contiguous()
    got = ws.guess_image(net, g, a, m, scale=2)
    assert got.shape == g.shape and bool(torch.isfinite(got).all())


def test_trainer_resume_is_bit_identical(ctx, ws, torch_cuda, tmp_path):
    data = ws.build_dataset(ctx, n=256, size=64, seed=5, chunk=256)
    straight = ws.Trainer(ws.UNet(ctx, seed=7), data, batch=64, seed=3)
    l_straight = [straight.step() for _ in range(10)]  # crosses two epoch boundaries
    first = ws.Trainer(ws.UNet(ctx, seed=7), data, batch=64, seed=3)
    l_first = [first.step() for _ in range(6)]
    path = str(tmp_path / "ckpt.bin")
    first.save(path)
    resumed = ws.Trainer(ws.UNet(ctx, seed=99), data, batch=64, seed=12345)
    resumed.load(path)
    l_rest = [resumed.step() for _ in range(4)]
    assert l_first + l_rest == l_straight
    assert resumed.epoch == straight.epoch and resumed.steps == straight.steps == 10
    assert np.array_equal(resumed.net.get_params().view(np.uint32), straight.net.get_params().view(np.uint32))


def test_trained_network_gain_over_plain(ctx, ws, torch_cuda, capsys, oracle):
    """Train briefly on solves of the plain method, then solve held-out
    instances both ways to the same absolute bar. Shows the gain: fewer sweeps
    on average, every solve converged, and errors against the FP64 oracle
    within the same bound as the plain solve's."""
    torch = torch_cuda
    data = ws.build_dataset(ctx, n=2048, size=256, seed=41, tol=1e-7)
    net = ws.UNet(ctx, seed=41)
    losses, _ = ws.train(net, data, epochs=20, batch=64, lr=1e-3, seed=41, max_steps=400)
    assert np.mean(losses[-20:]) < 0.2 * losses[0]
    g, a, m = ws.make_instances(64, 256, seed=4242)
    ref = torch.as_tensor(oracle_solutions(oracle, g, a, m), dtype=torch.float64, device="cuda")
    up, rp = ws.solve_batch_device(ctx, g, a, m, tol=1e-6)
    guess = ws.predict_guess(net, g, a, m)
    uw, rw = ws.solve_batch_device(ctx, g, a, m, tol=1e-6, guess=guess)
    assert all(r["converged"] for r in rp) and all(r["converged"] for r in rw)
    assert [r["initial_residual"] for r in rw] == [r["initial_residual"] for r in rp]
    lm = ws.interior_mask(m).double()
    e_plain = float(((up.double() - ref) * lm).abs().max())
    e_warm = float(((uw.double() - ref) * lm).abs().max())
    assert e_warm < 2e-5 and e_plain < 2e-5
    ip = np.array([r["iterations"] for r in rp])
    iw = np.array([r["iterations"] for r in rw])
    g_err = float((((guess.double() - ref) * lm) ** 2).sum() / lm.sum()) ** 0.5
    a_err = float((((a.double() - ref) * lm) ** 2).sum() / lm.sum()) ** 0.5
    with capsys.disabled():
        print(f"\nwarm start after 400 steps: mean sweeps {iw.mean():.1f} vs plain {ip.mean():.1f} "
              f"(ratio {iw.mean() / ip.mean():.3f}), guess RMS error {g_err:.4f} vs anchor {a_err:.4f}, "
              f"guess used {sum(r['warm_start'] for r in rw)}/64")
    assert g_err < 0.5 * a_err
    assert iw.mean() < ip.mean()
