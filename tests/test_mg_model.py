"""The multigrid-CG preconditioner's properties on its CPU model
(oracle/mg_model.py, the V-cycle of paintop_b200/csrc/mg_solver.cu in numpy):
CG needs a symmetric positive-definite preconditioner, and the V-cycle is one
only because the post-smoothing runs the colours in the reverse order of the
pre-smoothing and restriction is the transpose of prolongation (/ 4). The
GPU path itself is checked against the FP64 CG oracle in
tests/test_multigrid_gpu.py."""
import math

import numpy as np
import pytest

from oracle import mg_model as M


def irregular_mask(w, h, seed):
    """An interior region with ragged edges and holes, off the border."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    blob = ((xx - w / 2) / (0.42 * w)) ** 2 + ((yy - h / 2) / (0.4 * h)) ** 2 <= 1.0 + 0.3 * rng.random((h, w))
    act = blob & (rng.random((h, w)) > 0.15)
    act[0, :] = act[-1, :] = False
    act[:, 0] = act[:, -1] = False
    return act


@pytest.mark.parametrize("w,h,lam", [(23, 17, 0.0), (30, 21, 0.05), (19, 26, 0.0)])
def test_vcycle_is_symmetric_positive_definite(w, h, lam):
    act = irregular_mask(w, h, seed=w)
    assert len(M.levels(act, lam)) >= 3  # smoothing, restriction and the coarsest solve all take part
    m = M.operator_matrix(act, lam)
    asym = np.abs(m - m.T).max() / np.abs(m).max()
    assert asym < 1e-12, asym
    eig = np.linalg.eigvalsh(0.5 * (m + m.T))
    assert eig.min() > 0.0, eig.min()


def test_same_colour_order_after_the_correction_breaks_symmetry():
    """The check is sensitive: post-smoothing red then black (the order of the
    pre-smoothing) makes the V-cycle non-symmetric."""
    act = irregular_mask(23, 17, seed=23)
    m = M.operator_matrix(act, 0.0, post_order=(0, 1))
    assert np.abs(m - m.T).max() / np.abs(m).max() > 1e-3


def test_preconditioned_cg_converges_in_a_handful_of_iterations():
    """Eight separate polygons on 128 x 128 (the 4096 x 4096 workload's layout,
    scaled): CG with the V-cycle reaches 1e-6 in about as many iterations as on
    the GPU, and the 3-of-4 coarsening beats 'any child'."""
    from paintop_b200 import synth
    size = 128
    rng = np.random.default_rng(1)
    mask = np.zeros((size, size), bool)
    cw, ch = size // 4, size // 2
    for k in range(8):
        cx, cy = (k % 4 + 0.5) * cw, (k // 4 + 0.5) * ch
        pts = synth.random_blob_polygon(rng, cx, cy, 0.33 * cw, int(rng.integers(7, 14)), 0.2)
        mask |= synth.polygon_mask(size, size, pts) > 0.5
    act = np.zeros_like(mask)
    act[1:-1, 1:-1] = mask[1:-1, 1:-1]
    b = np.random.default_rng(2).standard_normal(act.shape)
    its = M.pcg_iterations(act, 0.0, b)
    assert its <= 10, its
    assert M.pcg_iterations(act, 0.0, b, rule=1) > its
    # unpreconditioned CG needs many more
    lv = M.levels(act, 0.0)
    plain = 0
    x = np.zeros_like(b)
    r = np.where(act, b, 0.0)
    p = r.copy()
    rho = float(np.sum(r * r))
    nb0 = math.sqrt(rho)
    while plain < 1000 and math.sqrt(rho) > 1e-6 * nb0:
        q = M.apply_a(act, p, 1.0, 4.0)
        a = rho / float(np.sum(p * q))
        x += a * p
        r -= a * q
        rho_new = float(np.sum(r * r))
        p = r + (rho_new / rho) * p
        rho = rho_new
        plain += 1
    assert plain > 5 * its, (plain, its)
    assert len(lv) >= 4
