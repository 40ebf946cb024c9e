"""Periodic axes (region.cc:14 coarse sizes, grid_map/igrid_map periodic
branches region.cc:1202-1208, 1233-1242, ghost wrap region.cc:1338-1469):
the CUDA path against the reference itself (oracle/_ref, built with the
periodic ghost exchange of its single-rank MPI shim).

Odd periodic sizes are included, on the finest level and on levels above the
coarsest: their transfers take igrid_map's odd periodic branch, and such a
level is swept lexicographically by the 8-colour smoother too.

The reference adds the contributions that cross a periodic boundary through
its restriction and RAT strips after the local ones, so sums at those points
associate differently here.  Tolerances (relative to the largest entry):
1e-13 for the Galerkin stencils, restriction and interpolation, 1e-12 for a
lexicographic Gauss-Seidel sweep (the reference's stale-ghost order is
reproduced), 1e-10 for lexicographic V-cycle iterates; the 8-colour smoother
and mixed precision reach 1e-10 and agree with the reference's solution
driven to 1e-13 within 1e-9."""
import numpy as np
import pytest

import pgmg_b200 as P
from oracle.pyoracle import Reference, ref_available
from tests.helpers import periodic_problem, relerr

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

CASES = [((16, 12, 18), (True, False, True)), ((16, 16, 16), (True, True, True)),
         ((32, 20, 16), (False, True, True)), ((24, 24, 40), (True, True, False)),
         # odd periodic sizes above the coarsest level (region.cc:1202-1208,
         # 1236-1243): 50 -> 25 -> 13; 30 -> 15 and 18 -> 9; 25 on level 0;
         # 44 -> 22 -> 11 -> 6 on all three axes
         ((50, 16, 16), (True, False, False)), ((30, 18, 18), (True, False, True)),
         ((25, 16, 16), (True, False, False)), ((44, 44, 44), (True, True, True))]


def make(mno, prd, precision=P.FP64, smoother=P.SMOOTH_LEX, coarse=P.COARSE_LU_EXACT, seed=3):
    coef, S, r = periodic_problem(*mno, prd, seed=seed)
    R = Reference(*mno, S, coef, r, prd=prd)
    G = P.Multigrid(*mno, precision=precision, coarse=coarse if R.lu_enabled else P.COARSE_GS,
                    smoother=smoother, prd=prd)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    return G, R


@pytest.mark.parametrize("mno,prd", CASES)
def test_periodic_levels_and_rat(mno, prd):
    G, R = make(mno, prd)
    assert G.nlevels == R.nlevels
    assert G.lu_enabled == R.lu_enabled
    for l in range(G.nlevels):
        assert G.dims(l) == R.dims(l)
        assert relerr(G.get_coef(l), R.get_A27(l)) < 1e-13, l


@pytest.mark.parametrize("mno,prd", CASES)
def test_periodic_transfers(mno, prd):
    G, R = make(mno, prd)
    rng = np.random.default_rng(5)
    for l in range(1, G.nlevels):
        xf = rng.standard_normal(G.npts(l - 1))
        G.set_x(l - 1, xf)
        R.set_x(l - 1, xf)
        G.restriction(l)
        R.restriction(l)
        assert relerr(G.get_r(l), R.get_r(l)) < 1e-13, ("restriction", l)
        xc = rng.standard_normal(G.npts(l))
        G.set_x(l, xc)
        R.set_x(l, xc)
        G.interpolation(l)
        R.interpolation(l)
        assert relerr(G.get_x(l - 1), R.get_x(l - 1)) < 1e-13, ("interpolation", l)


@pytest.mark.parametrize("mno,prd", CASES)
@pytest.mark.parametrize("mode", [0, 1])
def test_periodic_lex_sweeps(mno, prd, mode):
    G, R = make(mno, prd)
    x0 = np.random.default_rng(7).standard_normal(G.npts(0))
    G.set_x(0, x0)
    R.set_x(0, x0)
    for _ in range(3):
        G.gauss_seidel(mode, 0, P.SMOOTH_LEX)
        R.gauss_seidel(mode, 0)
        assert relerr(G.get_x(0), R.get_x(0)) < 1e-12


@pytest.mark.parametrize("mno,prd", CASES)
def test_periodic_lex_vcycles(mno, prd):
    G, R = make(mno, prd)
    for c in range(4):
        G.v_cycle(0, P.SMOOTH_LEX)
        R.v_cycle(0)
        assert relerr(G.get_x(0), R.get_x(0)) < 1e-10, c


def reference_solution(R, tol=1e-13):
    rhs = R.rhs_l2norm()
    for _ in range(200):
        if np.sqrt(R.l2_error_all() / rhs) < tol:
            break
        R.v_cycle(0)
    return R.get_x(0)


@pytest.mark.parametrize("mno,prd", CASES)
@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_periodic_mc8_solve(mno, prd, precision):
    G, R = make(mno, prd, precision=precision, smoother=P.SMOOTH_MC8, coarse=P.COARSE_LU)
    cyc, rr = G.solve(1e-10, 100, 0)
    assert rr < 1e-10 and cyc < 40
    xr = reference_solution(R)
    assert relerr(G.get_x(0), xr) < 1e-9


@pytest.mark.parametrize("mno,prd", CASES[:2])
def test_periodic_mc8_contraction(mno, prd):
    """Per-cycle residual reduction of the 8-colour V-cycle no worse than 1.05x
    the reference's lexicographic one."""
    G, R = make(mno, prd, smoother=P.SMOOTH_MC8)
    rhs = R.rhs_l2norm()
    rg, rref = [], []
    for _ in range(4):
        G.v_cycle(0, P.SMOOTH_MC8)
        R.v_cycle(0)
        rg.append(np.sqrt(G.l2_error_all() / G.rhs_l2norm()))
        rref.append(np.sqrt(R.l2_error_all() / rhs))
    fg = (rg[-1] / rg[0]) ** (1 / 3)
    fr = (rref[-1] / rref[0]) ** (1 / 3)
    assert fg <= 1.05 * fr


def test_periodic_odd_levels_planned():
    """A periodic axis that turns odd on a smoothed level is planned as the
    reference plans it (coarse size (m+1)>>1, region.cc:14)."""
    G = P.Multigrid(44, 44, 44, prd=(True, True, True))
    assert [G.dims(l) for l in range(G.nlevels)] == [(44, 44, 44), (22, 22, 22), (11, 11, 11), (6, 6, 6)]
