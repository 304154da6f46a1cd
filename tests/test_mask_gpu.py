"""GPU parity of the device mask generators against the oracle
(oracle/mask_ref.c, the reference's rasterize() restated): polygons bit for
bit, ellipses within the op's declared tolerance, through the C ABI with
device and host buffers and through the op-level compute()."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M(ctx):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from paintop_b200 import masks
    return masks


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _star(cx, cy, r_out, r_in, n=12, rot=0.0):
    return [(cx + (r_out if k % 2 == 0 else r_in) * math.cos(rot + 2 * math.pi * k / n),
             cy + (r_out if k % 2 == 0 else r_in) * math.sin(rot + 2 * math.pi * k / n)) for k in range(n)]


def _pentagram(c, r):
    return [(r * math.cos(k * 4 * math.pi / 5 - math.pi / 2) + c, r * math.sin(k * 4 * math.pi / 5 - math.pi / 2) + c)
            for k in range(5)]


def _blob(rng, cx, cy, r, n):
    a = np.sort(rng.uniform(0, 2 * math.pi, n))
    rr = r * (1 + rng.uniform(-0.3, 0.3, n))
    return np.stack([cx + rr * np.cos(a), cy + rr * np.sin(a)], 1)


POLYGONS = [
    ("square", 6, 6, [[1, 1], [4, 1], [4, 4], [1, 4]]),
    ("triangle", 64, 64, [[8, 8], [56, 16], [24, 56]]),
    ("pentagram", 40, 40, _pentagram(20.0, 15.0)),
    ("repeated_vertex", 8, 8, [[1, 1], [1, 1], [5, 1], [5, 5], [1, 5]]),
    ("bowtie", 8, 8, [[0, 0], [6, 6], [6, 0], [0, 6]]),
    ("spike", 8, 8, [[1, 1], [5, 1], [3, 1], [3, 5]]),
    ("two_points", 6, 6, [[1, 1], [4, 4]]),
    # vertices on subsample positions and horizontal edges
    ("on_subsamples", 33, 17, [[1.125, 2.375], [30.875, 2.375], [30.875, 14.625], [16.5, 8.125], [1.125, 14.625]]),
    # partly outside the image, negative coordinates
    ("clipped", 50, 30, [[-20, -5], [70, 10], [25, 45]]),
    ("star_512", 512, 512, _star(256.3, 250.7, 200, 90)),
    # more edges than one 256-edge chunk, rows of many crossings
    ("blob_700", 300, 260, _blob(np.random.default_rng(3), 150, 130, 100, 700)),
    ("zigzag", 257, 64, [(x * 0.5 + 1, 2 + 60 * (x % 2)) for x in range(500)] + [(250.5, 63.0), (1.0, 63.0)]),
]


@pytest.mark.parametrize("name,w,h,pts", POLYGONS, ids=[p[0] for p in POLYGONS])
@pytest.mark.parametrize("rule", ["nonzero", "even-odd"])
def test_polygon_bit_exact(ctx, M, oracle, name, w, h, pts, rule):
    got = M.polygon(ctx, w, h, pts, rule).cpu().numpy()
    want = oracle.mask_polygon(w, h, pts, rule)
    assert np.array_equal(_bits(got), _bits(want)), (name, int((got != want).sum()))


def test_polygon_star_2048_bit_exact(ctx, M, oracle):
    # the 2048 x 2048 screened-Poisson workload's 12-vertex star, ~30% coverage
    pts = _star(1024.0, 1024.0, 860.0, 430.0, rot=0.3)
    got = M.polygon(ctx, 2048, 2048, pts).cpu().numpy()
    want = oracle.mask_polygon(2048, 2048, pts)
    assert np.array_equal(_bits(got), _bits(want))
    assert 0.2 < float(got.mean()) < 0.5


def test_polygon_tall_extent_beyond_one_grid_row_span(ctx, M, oracle):
    # 70,000 rows: more than the 65,535 blocks of one grid column
    pts = [[0.3, 2.0], [2.7, 100.0], [0.9, 69990.5]]
    got = M.polygon(ctx, 3, 70000, pts).cpu().numpy()
    want = oracle.mask_polygon(3, 70000, pts)
    assert np.array_equal(_bits(got), _bits(want))


def test_polygon_host_buffer_path(ctx, M, oracle):
    pts = _pentagram(30.0, 25.0)
    got = M.polygon_host(ctx, 61, 57, pts, "even-odd")
    assert np.array_equal(_bits(got), _bits(oracle.mask_polygon(61, 57, pts, "even-odd")))


ELLIPSES = [
    ((64, 64), (33.0, 24.0), (18.0, 7.0), 0.6, 3.0),
    ((32, 32), (16.0, 16.0), (9.0, 9.0), math.pi / 2, 2.0),
    ((17, 17), (8.5, 8.5), (4.0, 4.0), 0.0, 0.0),
    ((512, 512), (256.0, 256.0), (150.0, 110.0), 0.0, 0.0),
    ((300, 200), (120.5, 90.25), (80.0, 33.0), 2.2, 5.5),
]


@pytest.mark.parametrize("extent,center,radii,angle,half", ELLIPSES)
def test_ellipse_matches_oracle(ctx, M, oracle, extent, center, radii, angle, half):
    w, h = extent
    got = M.ellipse(ctx, w, h, center, radii, angle, half).cpu().numpy()
    want = oracle.mask_ellipse(w, h, center, radii, angle, half)
    # the device's hypot may differ from libm's in the last bit of the
    # distance; in f32 coverage that is at most a few ulps, never a flipped pixel
    assert np.abs(got.astype(np.float64) - want).max() <= 1e-6
    assert (got != want).mean() < 1e-3
    hard = half == 0.0
    if hard:
        assert np.array_equal(got, want)


def test_ellipse_host_buffer_path(ctx, M, oracle):
    got = M.ellipse_host(ctx, 40, 30, (18.0, 14.0), (12.0, 7.0), 0.4, 2.0)
    want = oracle.mask_ellipse(40, 30, (18.0, 14.0), (12.0, 7.0), 0.4, 2.0)
    assert np.abs(got.astype(np.float64) - want).max() <= 1e-6


def test_mask_ops_through_compute(ctx, M, oracle):
    from paintop_b200 import ops
    src = ops.image_value(48, 40, 3, np.zeros(48 * 40 * 3, np.float32))
    pts = [[2.0, 3.0], [45.5, 5.0], [30.0, 37.25], [5.0, 30.0]]
    out = ops.PolygonMask().compute({"extent_from": src}, {"points": pts, "fill_rule": "even-odd"})["mask"]
    assert (out.kind, out.width, out.height, out.channels) == ("mask", 48, 40, 1)
    assert np.array_equal(_bits(out.samples), _bits(oracle.mask_polygon(48, 40, pts, "even-odd").reshape(-1)))
    e = ops.EllipseMask().compute({"extent_from": src}, {"center_px": [20, 18], "radii_px": [14, 9],
                                                         "angle_rad": 0.25})["mask"]
    want = oracle.mask_ellipse(48, 40, (20.0, 18.0), (14.0, 9.0), 0.25).reshape(-1)
    assert np.array_equal(e.samples, want)
    with pytest.raises(ops.PaintopError) as err:
        ops.EllipseMask().compute({"extent_from": src}, {"center_px": [1, 1], "radii_px": [0, 1]})
    assert err.value.code == "E_ELLIPSE_PARAM"


def test_device_mask_feeds_a_solve(ctx, M, oracle):
    """A solve whose mask came from the device rasteriser equals the same solve
    fed the oracle's mask, byte for byte."""
    import torch
    from paintop_b200 import synth, warmstart as ws
    inst = synth.clone_512(seed=2)
    pts = _star(256.0, 256.0, 200.0, 100.0)
    W = H = 512
    dm = M.polygon(ctx, W, H, pts)
    hm = oracle.mask_polygon(W, H, pts)
    # one channel of the clone instance as the guidance / anchor
    g = torch.from_numpy(np.ascontiguousarray(inst.source[:, :, 0])).cuda()[None]
    a = torch.from_numpy(np.ascontiguousarray(inst.target[:, :, 0])).cuda()[None]
    u1, r1 = ws.solve_batch_device(ctx, g, a, dm[None].contiguous(), tol=1e-6, omega_auto=False)
    u2, r2 = ws.solve_batch_device(ctx, g, a, torch.from_numpy(hm).cuda()[None], tol=1e-6, omega_auto=False)
    assert r1[0]["converged"] and r1[0]["iterations"] == r2[0]["iterations"]
    assert torch.equal(u1, u2)
