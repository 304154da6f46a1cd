"""The numpy network oracle pinned on the CPU: its analytic gradient against
central finite differences (float64, no bf16 rounding), its bf16 rounding, its
feature extraction, and the training-FLOP count."""
import numpy as np
import pytest

from oracle import unet_ref as R


def _problem(B=1, H=16, W=16, seed=3):
    rng = np.random.default_rng(seed)
    feats = np.zeros((B, H, W, 4))
    feats[..., 0] = rng.normal(0, 0.1, (B, H, W))
    feats[..., 1] = rng.uniform(0, 1, (B, H, W))
    feats[..., 2] = rng.uniform(0, 1, (B, H, W)) > 0.4
    feats[..., 3] = rng.uniform(0, 1, (B, H, W))
    target = rng.uniform(0, 1, (B, H, W))
    mask = (rng.uniform(0, 1, (B, H, W)) > 0.3).astype(np.float64)
    return feats, target, mask


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -2.5, 0.0, 2.0 ** -133])
    got = R.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0)
    assert got[0] == 1.0 and got[1] == 1.0
    assert got[2] == 1.0 + 2 ** -7          # above the tie: rounds up
    assert got[3] == 1.0                     # below the tie
    assert got[4] == -2.5 and got[5] == 0.0
    assert got[6] == 2.0 ** -133              # the smallest bf16 subnormal survives


def test_param_layout_matches_library_count():
    _, head_w, total = R.param_layout()
    convs = sum(co * 9 * ci + co for co, ci in R.LAYERS)
    assert head_w == convs and total == convs + 17


def test_gradient_matches_finite_differences():
    feats, target, mask = _problem()
    p = R.init_params(7)
    net = R.Net(p, emulate_bf16=False)
    loss, g = net.loss_grad(feats, target, mask)
    layout, head_w, total = R.param_layout()
    rng = np.random.default_rng(11)
    picks = [head_w + k for k in (0, 5, 16)]
    for (w, b, co, ci) in layout:
        picks += list(rng.integers(w, b, 3)) + [int(rng.integers(b, b + co))]
    eps = 1e-6
    for i in picks:
        if g[i] == 0.0 and i < layout[0][1] and (i - layout[0][0]) % layout[0][3] >= R.IN_REAL:
            continue  # padded input channel: exactly zero both ways
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        lp, _ = R.Net(pp, emulate_bf16=False).loss_grad(feats, target, mask)
        lm, _ = R.Net(pm, emulate_bf16=False).loss_grad(feats, target, mask)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_features_rule():
    rng = np.random.default_rng(2)
    B, H, W = 2, 40, 48
    g = rng.uniform(0, 1, (B, H, W)).astype(np.float32)
    a = rng.uniform(0, 1, (B, H, W)).astype(np.float32)
    m = np.zeros((B, H, W), np.float32)
    m[:, 5:35, 4:44] = 1.0
    f = R.features(g, a, m)
    # interior cell (20, 20): Laplacian of g, distance to the region's edge
    y, x = 20, 20
    lap = (g[0, y, x - 1] + g[0, y, x + 1] + g[0, y - 1, x] + g[0, y + 1, x]) - 4 * g[0, y, x]
    assert f[0, y, x, 0] == np.float32(lap)
    assert f[0, y, x, 1] == 0 and f[0, y, x, 2] == 1
    # nearest non-interior along the row/column: x = 3 is 17 away, y = 35 is 15 away
    assert f[0, y, x, 3] == np.float32(15 / 32)
    # outside: the correction's boundary value anchor - guidance, no divergence
    assert f[1, 2, 2, 1] == a[1, 2, 2] - g[1, 2, 2] and f[1, 2, 2, 0] == 0 and f[1, 2, 2, 2] == 0
    # the image border is never interior
    m2 = np.ones((1, 8, 8), np.float32)
    f2 = R.features(g[:1, :8, :8], a[:1, :8, :8], m2)
    assert f2[0, 0, 3, 2] == 0 and f2[0, 3, 3, 2] == 1


def test_train_flops_count():
    from paintop_b200.warmstart import train_flops_per_pixel
    # forward MACs per input pixel of the 16-32-64-128 network (padded first layer)
    fwd = 0.0
    lev = [0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0]
    for (co, ci), l in zip(R.LAYERS, lev):
        fwd += 9 * co * ci / 4 ** l
    assert train_flops_per_pixel() == pytest.approx(2 * (3 * fwd - 9 * 16 * 16))
