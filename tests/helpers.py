"""Shared problem builders for the tests (seeded, deterministic)."""
import numpy as np

import pgmg_b200 as P


def q1_problem(m, n, o, sigma=1.0, seed=1, width=8.0):
    """Variable-kappa Q1 stencils, boxes and RHS of an m x n x o grid."""
    kap = P.problem_kappa(m, n, o, sigma, seed, width) if sigma is not None else None
    coef, S = P.problem_q1(m, n, o, kap)
    r = P.problem_rhs(m, n, o, seed)
    return coef, S, r


def simple_problem(m, n, o):
    """The reference's problem_simple (problem_simple.hh/.cc) as arrays:
    interior 7-point cell-centre Laplacian box [-1,2)^3, boundary fix rows
    [0,1)^3 with -0.375, point sources +1 at (3,3,3) and -1 at (12,12,12)."""
    st = np.array([0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 1, -6, 1, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0], float)
    N = m * n * o
    coef = np.zeros((N, 27))
    S = np.zeros((N, 6), np.int32)
    r = np.zeros(N)
    k, j, i = np.meshgrid(np.arange(o), np.arange(n), np.arange(m), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    interior = (i > 0) & (i < m - 1) & (j > 0) & (j < n - 1) & (k > 0) & (k < o - 1)
    coef[interior] = st
    coef[~interior, 13] = -0.375
    S[interior] = [-1, 2, -1, 2, -1, 2]
    S[~interior] = [0, 1, 0, 1, 0, 1]
    r[(i == 3) & (j == 3) & (k == 3)] = 1
    r[(i == 12) & (j == 12) & (k == 12)] = -1
    return coef.ravel(), S.ravel(), r


def relerr(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    den = np.abs(b).max()
    return np.abs(a - b).max() / (den if den > 0 else 1.0)


def periodic_problem(m, n, o, prd, seed=0, shift=0.3, spread=0.2):
    """Random 27-point stencils on an m x n x o grid with the axes flagged in
    prd periodic: a 27-point Q1-Laplacian pattern (centre 8/3 + shift, edge
    -1/6, corner -1/12, face 0) with every entry scaled by 1 + U(-spread,
    spread); full [-1,2) boxes on periodic axes, boxes cropped at the
    boundary of non-periodic ones.  Returns (coef27, S6, r)."""
    rng = np.random.default_rng(seed)
    N = m * n * o
    slots = np.arange(27)
    d = np.stack([slots % 3 - 1, (slots // 3) % 3 - 1, slots // 9 - 1], 1)
    nd = np.abs(d).sum(1)
    base = np.select([nd == 0, nd == 1, nd == 2, nd == 3], [8.0 / 3.0 + shift, 0.0, -1.0 / 6.0, -1.0 / 12.0])
    k, j, i = np.meshgrid(np.arange(o), np.arange(n), np.arange(m), indexing="ij")
    idx = [i.reshape(-1), j.reshape(-1), k.reshape(-1)]
    size = [m, n, o]
    S = np.zeros((N, 6), np.int32)
    ok = np.ones((N, 27), bool)
    for a in range(3):
        lo = np.where(prd[a] | (idx[a] > 0), -1, 0)
        hi = np.where(prd[a] | (idx[a] < size[a] - 1), 2, 1)
        S[:, 2 * a], S[:, 2 * a + 1] = lo, hi
        ok &= (d[None, :, a] >= lo[:, None]) & (d[None, :, a] < hi[:, None])
    coef = base[None, :] * (1.0 + spread * rng.uniform(-1, 1, (N, 27)))
    coef[~ok] = 0.0
    r = rng.uniform(-1, 1, N)
    return coef, S, r
