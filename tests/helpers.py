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
