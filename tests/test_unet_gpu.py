"""GPU parity of the learned warm start's network: the tensor-core forward pass,
loss and every parameter gradient against the numpy oracle (bf16 rounding
emulated at the points where the GPU stores bf16), feature extraction bit for
bit, deterministic training steps, and the C ABI's argument checks.

Tolerances: the GPU accumulates in fp32 in its own order and the oracle in
fp64, so a bf16 rounding can land one ulp (2^-8 relative) apart and carry
forward. Forward predictions agree to 1e-2 relative L2, each layer's gradient
to 3e-2 relative L2 (measured well below both)."""
import numpy as np
import pytest

from oracle import unet_ref as R

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


def _realistic(ws, torch, B, H, W, seed):
    g, a, m = ws.make_instances(B, max(H, W), seed)
    g, a, m = g[:, :H, :W].contiguous(), a[:, :H, :W].contiguous(), m[:, :H, :W].contiguous()
    return g, a, m


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_features_bit_exact(ctx, ws, torch_cuda):
    torch = torch_cuda
    net = ws.UNet(ctx, seed=1)
    g, a, m = _realistic(ws, torch, 3, 64, 72, seed=5)
    f = net.features(g, a, m).cpu().numpy()
    ref = R.features(g.cpu().numpy(), a.cpu().numpy(), m.cpu().numpy())
    assert f.shape == ref.shape
    assert np.array_equal(f.view(np.uint32), ref.view(np.uint32))


# 128-pixel segments (W >= 128, the last one partial for 200), whole-row
# segments rounded up to 16 pixels (40, 24, 5 at the deepest level), and the
# first layer's one-chunk K beside the 192-channel decoder layer's three
SHAPES = [(2, 32, 32), (1, 24, 40), (2, 64, 64), (1, 64, 256), (2, 40, 128), (1, 16, 200)]


@pytest.mark.parametrize("B,H,W", SHAPES)
def test_forward_matches_oracle(ctx, ws, torch_cuda, B, H, W):
    torch = torch_cuda
    net = ws.UNet(ctx, seed=2)
    p = R.init_params(4).astype(np.float32)
    net.set_params(p)
    g, a, m = _realistic(ws, torch, B, H, W, seed=6)
    f = net.features(g, a, m)
    pred = net.forward(f).cpu().numpy()
    ref = R.Net(p.astype(np.float64)).forward(f.cpu().numpy().astype(np.float64))
    assert np.isfinite(pred).all()
    assert _rel(pred, ref) < 1e-2


@pytest.mark.parametrize("B,H,W", SHAPES)
def test_gradients_match_oracle(ctx, ws, torch_cuda, B, H, W):
    torch = torch_cuda
    net = ws.UNet(ctx, seed=3)
    p = R.init_params(8).astype(np.float32)
    net.set_params(p)
    g, a, m = _realistic(ws, torch, B, H, W, seed=7)
    f = net.features(g, a, m)
    u = a.clone()  # any target works for a gradient check
    lm = ws.interior_mask(m)
    loss, grad = net.loss_grad(f, u, lm)
    rl, rg = R.Net(p.astype(np.float64)).loss_grad(f.cpu().numpy().astype(np.float64),
                                                     u.cpu().numpy(), lm.cpu().numpy())
    assert abs(loss - rl) <= 1e-2 * abs(rl)
    layout, head_w, total = R.param_layout()
    assert grad.size == total
    errs = {}
    for l, (w, b, co, ci) in enumerate(layout):
        errs[f"W{l}"] = _rel(grad[w:b], rg[w:b])
        errs[f"b{l}"] = _rel(grad[b:b + co], rg[b:b + co])
    errs["head"] = _rel(grad[head_w:], rg[head_w:])
    worst = max(errs, key=errs.get)
    assert errs[worst] < 3e-2, (worst, errs[worst], errs)
    # padded input channels of the first layer get exactly zero gradient
    w0, b0, co0, ci0 = layout[0]
    assert not grad[w0:b0].reshape(co0, 9, ci0)[:, :, R.IN_REAL:].any()


def test_loss_grad_is_deterministic(ctx, ws, torch_cuda):
    net = ws.UNet(ctx, seed=4)
    g, a, m = _realistic(ws, torch_cuda, 2, 64, 256, seed=8)
    f = net.features(g, a, m)
    lm = ws.interior_mask(m)
    l1, g1 = net.loss_grad(f, a, lm)
    l2, g2 = net.loss_grad(f, a, lm)
    assert l1 == l2 and np.array_equal(g1.view(np.uint32), g2.view(np.uint32))


def test_training_is_deterministic_and_learns(ctx, ws, torch_cuda):
    g, a, m = _realistic(ws, torch_cuda, 8, 64, 64, seed=9)
    u, reps = ws.solve_batch_device(ctx, g, a, m, tol=1e-7)
    assert all(r["converged"] for r in reps)
    lm = ws.interior_mask(m)
    runs = []
    for _ in range(2):
        net = ws.UNet(ctx, seed=10)
        f = net.features(g, a, m)
        losses = [net.train_step(f, u, lm, 1e-3) for _ in range(60)]
        runs.append((losses, net.get_params()))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1].view(np.uint32), runs[1][1].view(np.uint32))
    losses = runs[0][0]
    assert np.isfinite(losses).all()
    assert np.mean(losses[-5:]) < 0.5 * losses[0], (losses[0], losses[-5:])


def test_save_load_roundtrip(ctx, ws, torch_cuda, tmp_path):
    net = ws.UNet(ctx, seed=11)
    g, a, m = _realistic(ws, torch_cuda, 2, 32, 32, seed=12)
    f = net.features(g, a, m)
    lm = ws.interior_mask(m)
    net.train_step(f, a, lm, 1e-3)
    path = str(tmp_path / "net.bin")
    net.save(path)
    other = ws.UNet(ctx, seed=99)
    other.load(path)
    assert np.array_equal(net.get_params(), other.get_params())
    # the Adam state travels too: one more identical step on both
    la = net.train_step(f, a, lm, 1e-3)
    lb = other.train_step(f, a, lm, 1e-3)
    assert la == lb and np.array_equal(net.get_params(), other.get_params())


def test_shape_checks(ctx, ws, torch_cuda):
    from paintop_b200 import _lib
    torch = torch_cuda
    net = ws.UNet(ctx, seed=13)
    f = torch.zeros((1, 20, 32, 4), device="cuda")
    with pytest.raises(_lib.CudaError) as e:
        net.forward(f)  # 20 is not a multiple of 8
    assert e.value.status == _lib.PT_INVALID_ARG


def test_one_gradient_record_is_a_training_step(ctx, ws, torch_cuda):
    """grad_record then apply_records with one record repeats train_step bit for bit."""
    g, a, m = _realistic(ws, torch_cuda, 4, 64, 64, seed=14)
    lm = ws.interior_mask(m)
    nets = [ws.UNet(ctx, seed=15) for _ in range(2)]
    f = nets[0].features(g, a, m)
    for _ in range(3):
        la = nets[0].train_step(f, a, lm, 1e-3)
        lb, rec = nets[1].grad_record(f, a, lm)
        nets[1].apply_records(rec.view(1, -1), 1e-3)
        assert la == lb
    assert np.array_equal(nets[0].get_params().view(np.uint32), nets[1].get_params().view(np.uint32))


def test_gradient_records_combine_in_replica_order(ctx, ws, torch_cuda):
    """Two replicas' records (halves of a batch with different interior counts)
    combine to c0 g0 + c1 g1 over c0 + c1 summed in fp64 in replica order, which
    is the whole batch's gradient up to the bf16 rounding of each half's backward."""
    torch = torch_cuda
    g, a, m = _realistic(ws, torch, 4, 64, 64, seed=16)
    m[2:, 20:40, 10:50] = 0.0  # uneven interior counts
    lm = ws.interior_mask(m)
    net = ws.UNet(ctx, seed=17)
    f = net.features(g, a, m)
    P = net.param_count
    recs = torch.empty((2, P + 1), dtype=torch.float32, device="cuda")
    net.grad_record(f[:2].contiguous(), a[:2].contiguous(), lm[:2].contiguous(), out=recs[0])
    net.grad_record(f[2:].contiguous(), a[2:].contiguous(), lm[2:].contiguous(), out=recs[1])
    _, full = net.grad_record(f, a, lm)
    r = recs.cpu().numpy().astype(np.float64)
    c = r[:, -1]
    assert c[0] != c[1] and c[0] + c[1] == float(full[-1])
    acc = np.zeros(P)
    for k in range(2):
        acc = acc + c[k] * r[k, :-1]
    comb = (acc / (c[0] + c[1])).astype(np.float32)
    layout, head_w, _ = R.param_layout()
    fg = full[:-1].cpu().numpy()
    for l, (w, b, co, ci) in enumerate(layout):
        assert _rel(comb[w:b], fg[w:b]) < 3e-2, l
    # the device combination is that fp64 sum bit for bit: the same step as one
    # record that already holds it
    one = torch.from_numpy(np.append(comb, np.float32(c[0] + c[1]))).cuda().view(1, -1)
    other = ws.UNet(ctx, seed=17)
    net.apply_records(recs, 1e-3)
    other.apply_records(one, 1e-3)
    assert np.array_equal(net.get_params().view(np.uint32), other.get_params().view(np.uint32))


def test_data_parallel_trainer_over_nccl(ctx, ws, torch_cuda):
    """DataParallelTrainer over a one-rank NCCL group is Trainer bit for bit."""
    import torch.distributed as dist
    torch = torch_cuda
    data = ws.build_dataset(ctx, n=16, size=64, seed=3, chunk=16)
    dist.init_process_group("nccl", store=dist.HashStore(), rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        a, b = ws.UNet(ctx, seed=18), ws.UNet(ctx, seed=18)
        ta = ws.Trainer(a, data, batch=8, lr=1e-3, seed=4)
        tb = ws.DataParallelTrainer(b, data, batch=8, lr=1e-3, seed=4)
        la = [ta.step() for _ in range(3)]
        lb = [tb.step() for _ in range(3)]
    finally:
        dist.destroy_process_group()
    assert lb == pytest.approx(la, rel=1e-12)  # the count-weighted mean of one loss
    assert np.array_equal(a.get_params().view(np.uint32), b.get_params().view(np.uint32))
