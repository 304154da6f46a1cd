"""The automatic SOR factor with several interior regions: the GPU labels the
connected regions of the mask and bounds the Jacobi spectral radius by the
smaller of the union's bounding-box bound and the largest region's area
(Faber-Krahn) bound. Checked against the same formula evaluated on the host
with scipy's labelling, and for convergence."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PI_J0_SQ = math.pi * 2.404825557695773 ** 2


def expected_omega(mask, lam=0.0):
    from scipy import ndimage
    H, W = mask.shape
    inter = mask > 0.5
    inter[0, :] = inter[-1, :] = False
    inter[:, 0] = inter[:, -1] = False
    ys, xs = np.nonzero(inter)
    a = xs.max() - xs.min() + 2
    b = ys.max() - ys.min() + 2
    rho = (2 * math.cos(math.pi / a) + 2 * math.cos(math.pi / b)) / (4 + lam)
    lab, n = ndimage.label(inter)
    nmax = np.bincount(lab.ravel())[1:].max()
    area = (math.sqrt(nmax) + 1) ** 2
    rho = min(rho, (4 - PI_J0_SQ / area) / (4 + lam))
    return 2 / (1 + math.sqrt(1 - rho * rho)), int(nmax), n


def _solve(ctx, mask, seed=3):
    from paintop_b200 import _lib, synth
    rng = np.random.default_rng(seed)
    H, W = mask.shape
    src = synth.sinusoid_image(rng, W, H, 1)
    tgt = synth.sinusoid_image(rng, W, H, 1)
    out, per, worst = ctx.solve(src, tgt, mask, W, H, 1, tolerance=1e-6, max_iterations=100000,
                                flags=_lib.PT_FLAG_OMEGA_AUTO, want_history=False)
    return per[0]


@pytest.mark.parametrize("shape", ["two_squares", "disk", "eight_blobs", "single_square"])
def test_omega_matches_region_bound(ctx, shape):
    from paintop_b200 import synth
    if shape == "two_squares":
        mask = np.zeros((256, 1024), np.float32)
        mask[60:160, 20:120] = 1
        mask[100:130, 900:960] = 1
    elif shape == "disk":
        mask = synth.ellipse_mask(384, 384, 192, 192, 150, 150)
    elif shape == "single_square":
        mask = np.zeros((200, 200), np.float32)
        mask[50:150, 50:150] = 1
    else:
        rng = np.random.default_rng(9)
        mask = np.zeros((512, 1024), np.float32)
        for k in range(8):
            cx, cy = (k % 4 + 0.5) * 256, (k // 4 + 0.5) * 256
            pts = synth.random_blob_polygon(rng, cx, cy, 90, 9, 0.2)
            mask = np.maximum(mask, synth.polygon_mask(1024, 512, pts))
    want, nmax, nreg = expected_omega(mask.copy())
    rep = _solve(ctx, mask)
    assert rep["converged"]
    assert rep["omega_used"] == pytest.approx(want, rel=0, abs=1e-12), (shape, nmax, nreg)


def test_several_regions_converge_faster_than_union_box(ctx):
    """Eight separate blobs: the region bound gives a smaller omega than the
    union's box would and fewer sweeps than that box's omega."""
    from paintop_b200 import synth
    rng = np.random.default_rng(11)
    mask = np.zeros((512, 1024), np.float32)
    for k in range(8):
        cx, cy = (k % 4 + 0.5) * 256, (k // 4 + 0.5) * 256
        mask = np.maximum(mask, synth.polygon_mask(1024, 512, synth.random_blob_polygon(rng, cx, cy, 100, 10, 0.2)))
    rep_auto = _solve(ctx, mask)
    inter = mask > 0.5
    ys, xs = np.nonzero(inter[1:-1, 1:-1])
    a, b = xs.max() - xs.min() + 2, ys.max() - ys.min() + 2
    rho_box = (math.cos(math.pi / a) + math.cos(math.pi / b)) / 2
    om_box = 2 / (1 + math.sqrt(1 - rho_box ** 2))
    assert rep_auto["omega_used"] < om_box
    from paintop_b200 import _lib
    rng2 = np.random.default_rng(3)
    src = synth.sinusoid_image(rng2, 1024, 512, 1)
    tgt = synth.sinusoid_image(rng2, 1024, 512, 1)
    _, per, _ = ctx.solve(src, tgt, mask, 1024, 512, 1, tolerance=1e-6, max_iterations=100000, omega=om_box,
                          want_history=False)
    assert per[0]["converged"] and rep_auto["converged"]
    assert rep_auto["iterations"] < per[0]["iterations"]
