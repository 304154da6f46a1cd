"""CPU model of the multigrid-CG preconditioner (test infrastructure only).

The reference has no multigrid: it iterates row-major SOR
(crates/paintop-cpu/src/poisson.rs:244-265). This file is therefore not a
restatement of reference code. It is the float64 numpy statement of the V-cycle
that ``paintop_b200/csrc/mg_solver.cu`` runs as the preconditioner behind
PT_FLAG_MULTIGRID, kernel for kernel:

- levels (``ptk_solve_mg_batch`` / ``solve_group``): level k halves level k-1
  (ceil) while a level has more than 64 cells; s_k = 4^-k, d_k = 4 s_k + lambda;
- ``k_mg_coarsen``: a coarse cell is active when at least 3 of its 2 x 2
  children are;
- ``k_mg_smooth_first`` / ``k_mg_smooth``: red-black SOR half-sweeps at
  omega 1.25 on A_k e = rhs, e = e + omega ((rhs + s_k nsum(e)) / d_k - e) at
  active cells of one colour ((i + j) & 1), red then black twice before the
  coarse correction and black then red twice after it;
- ``k_mg_resid_restrict``: the residual rhs - A_k e at active fine cells,
  restricted with weights (1/4, 3/4, 3/4, 1/4) per axis and / 4, at active
  coarse cells;
- ``k_mg_prolong``: bilinear (9/16, 3/16, 3/16, 1/16) into active fine cells;
- ``k_mg_coarse``: the coarsest level, 24 Gauss-Seidel sweeps red-black then
  24 black-red, from zero.

The tests use it to show that this V-cycle is a symmetric positive-definite
operator -- what conjugate gradients needs of a preconditioner -- and that CG
with it reaches 1e-6 in a handful of iterations.
"""
from __future__ import annotations

import numpy as np

COARSE_MAX = 64      # cells of the coarsest level (kCoarseMax)
COARSE_RULE = 3      # children that make a coarse cell active (kCoarseRule)
OMEGA = 1.25         # the half-sweeps' relaxation (kSmoothOmega)
COARSE_SWEEPS = 24   # k_mg_coarse's sweeps per half
_W = np.array([0.25, 0.75, 0.75, 0.25])  # restriction weights for a = -1, 0, 1, 2


def nsum(e: np.ndarray) -> np.ndarray:
    """Sum of the four neighbours, zero outside the grid."""
    n = np.zeros_like(e)
    n[:, 1:] += e[:, :-1]
    n[:, :-1] += e[:, 1:]
    n[1:, :] += e[:-1, :]
    n[:-1, :] += e[1:, :]
    return n


def coarsen(act: np.ndarray, rule: int = COARSE_RULE) -> np.ndarray:
    h, w = act.shape
    cnt = np.zeros(((h + 1) // 2, (w + 1) // 2), int)
    for dy in range(2):
        for dx in range(2):
            sub = act[dy::2, dx::2]
            cnt[:sub.shape[0], :sub.shape[1]] += sub
    return cnt >= rule


def levels(act: np.ndarray, lam: float, rule: int = COARSE_RULE):
    """[(active mask, s_k, d_k)] from level 0 to the coarsest."""
    out = [(act, 1.0, 4.0 + lam)]
    k = 0
    while out[-1][0].size > COARSE_MAX:
        k += 1
        s = 0.25 ** k
        out.append((coarsen(out[-1][0], rule), s, 4.0 * s + lam))
    return out


def apply_a(act, e, s, d):
    """A_k e at active cells (the level operator), 0 elsewhere."""
    return np.where(act, d * e - s * nsum(e), 0.0)


def half_sweep(act, rhs, e, s, d, color, omega):
    h, w = act.shape
    jj, ii = np.mgrid[0:h, 0:w]
    sel = act & (((ii + jj) & 1) == color)
    gs = (rhs + s * nsum(e)) / d  # the other colour's values: none of them change in this half-sweep
    e = e.copy()
    e[sel] = e[sel] + omega * (gs[sel] - e[sel])
    return e


def restrict(res, act_c):
    hf, wf = res.shape
    hc, wc = act_c.shape
    pad = np.zeros((2 * hc + 2, 2 * wc + 2))
    pad[1:hf + 1, 1:wf + 1] = res
    out = np.zeros((hc, wc))
    for b in range(4):
        for a in range(4):
            out += _W[b] * _W[a] * pad[b:b + 2 * hc:2, a:a + 2 * wc:2]
    return np.where(act_c, 0.25 * out, 0.0)


def prolong(act_f, e_c):
    hf, wf = act_f.shape
    hc, wc = e_c.shape
    pad = np.zeros((hc + 2, wc + 2))
    pad[1:-1, 1:-1] = e_c
    jj, ii = np.mgrid[0:hf, 0:wf]
    i0, j0 = ii >> 1, jj >> 1
    i1 = np.where(ii & 1, i0 + 1, i0 - 1)
    j1 = np.where(jj & 1, j0 + 1, j0 - 1)
    at = lambda i, j: pad[j + 1, i + 1]
    v = 0.5625 * at(i0, j0) + 0.1875 * (at(i1, j0) + at(i0, j1)) + 0.0625 * at(i1, j1)
    return np.where(act_f, v, 0.0)


def vcycle(lv, rhs, k: int = 0, omega: float = OMEGA, post_order=(1, 0)):
    """z = M rhs at level k. ``post_order`` is the colour order of the
    post-smoothing half-sweeps: (1, 0) (black then red) makes the cycle the
    adjoint-symmetric one the CUDA code runs; (0, 1) is a deliberately
    non-symmetric variant for the tests."""
    act, s, d = lv[k]
    e = np.zeros_like(rhs)
    if k == len(lv) - 1:
        for _ in range(COARSE_SWEEPS):
            e = half_sweep(act, rhs, e, s, d, 0, 1.0)
            e = half_sweep(act, rhs, e, s, d, 1, 1.0)
        for _ in range(COARSE_SWEEPS):
            e = half_sweep(act, rhs, e, s, d, 1, 1.0)
            e = half_sweep(act, rhs, e, s, d, 0, 1.0)
        return e
    for _ in range(2):
        e = half_sweep(act, rhs, e, s, d, 0, omega)
        e = half_sweep(act, rhs, e, s, d, 1, omega)
    res = np.where(act, rhs - apply_a(act, e, s, d), 0.0)
    e = e + prolong(act, vcycle(lv, restrict(res, lv[k + 1][0]), k + 1, omega, post_order))
    for _ in range(2):
        e = half_sweep(act, rhs, e, s, d, post_order[0], omega)
        e = half_sweep(act, rhs, e, s, d, post_order[1], omega)
    return e


def operator_matrix(act: np.ndarray, lam: float, **kw) -> np.ndarray:
    """The V-cycle as a matrix on the active level-0 cells (one column per
    unit right-hand side)."""
    lv = levels(act, lam, kw.pop("rule", COARSE_RULE))
    idx = np.flatnonzero(act)
    m = np.zeros((idx.size, idx.size))
    for col, q in enumerate(idx):
        rhs = np.zeros(act.shape)
        rhs.flat[q] = 1.0
        m[:, col] = vcycle(lv, rhs, **kw).flat[idx]
    return m


def pcg_iterations(act: np.ndarray, lam: float, b: np.ndarray, tol: float = 1e-6, cap: int = 200, **kw) -> int:
    """Preconditioned CG iterations on A_0 x = b until ||r|| <= tol ||b||."""
    lv = levels(act, lam, kw.pop("rule", COARSE_RULE))
    b = np.where(act, b, 0.0)
    x = np.zeros_like(b)
    r = b.copy()
    p = None
    rho = 0.0
    for it in range(cap):
        z = vcycle(lv, r, **kw)
        rho_new = float(np.sum(r * z))
        p = z if p is None else z + (rho_new / rho) * p
        rho = rho_new
        q = apply_a(act, p, 1.0, 4.0 + lam)
        alpha = rho / float(np.sum(p * q))
        x += alpha * p
        r -= alpha * q
        if np.linalg.norm(r) <= tol * np.linalg.norm(b):
            return it + 1
    return cap
