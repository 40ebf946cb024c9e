"""Parity at the benchmark configurations, against the reference itself
(oracle/_ref, compiled from its own sources):

* 257^3, sigma = 1 (the benchmark problem): coarse boxes and Galerkin
  stencils bit for bit on all six levels, and one lexicographic V-cycle bit
  for bit (with the reference's own coarse solver: its LU order, or its
  24-sweep fallback when its LU was disabled);
* 129^3, sigma = 2.3 (the contrast of the 513^3 configuration): the 8-colour
  V-cycle's per-cycle residual reduction (geometric mean over cycles 2-6) no
  worse than 1.05x the reference's lexicographic one, and the FP64 and mixed
  FP32/FP64 solutions to 1e-10 within 1e-9 (max norm, relative to the
  largest entry) of the reference's solution driven to 1e-13.

The inputs come from the oracle library's generator, which is pinned bit for
bit to the library's own (tests/test_oracle_inputs.py)."""
import numpy as np
import pytest

import pgmg_b200 as P
from oracle.pyoracle import Reference, benchmark_problem, ref_available
from tests.helpers import relerr

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]


def test_257_galerkin_hierarchy_and_lex_vcycle_bitwise():
    m = 257
    coef, S, r = benchmark_problem(m, m, m, 1.0, 1)
    R = Reference(m, m, m, S, coef, r)
    coarse = P.COARSE_LU_EXACT if R.lu_enabled else P.COARSE_GS
    G = P.Multigrid(m, m, m, coarse=coarse, smoother=P.SMOOTH_LEX)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    del coef, S
    assert G.nlevels == R.nlevels == 6
    assert G.lu_enabled == R.lu_enabled
    for l in range(G.nlevels):
        assert G.dims(l) == R.dims(l)
        assert np.array_equal(G.get_boxes(l), R.get_S(l)), f"boxes, level {l}"
        assert np.array_equal(G.get_coef(l), R.get_A27(l)), f"Galerkin stencils, level {l}"
    G.v_cycle(0)
    R.v_cycle(0)
    assert np.array_equal(G.get_x(0), R.get_x(0))
    R.close()
    G.close()


def _contraction(res):
    """Geometric mean of the per-cycle residual reduction over cycles 2-6."""
    q = np.array(res[2:7]) / np.array(res[1:6])
    return float(np.exp(np.mean(np.log(q))))


@pytest.fixture(scope="module")
def contrast129():
    m = 129
    coef, S, r = benchmark_problem(m, m, m, 2.3, 3)
    R = Reference(m, m, m, S, coef, r)
    res = [np.sqrt(R.l2_error_all())]
    for _ in range(6):
        R.v_cycle(0)
        res.append(np.sqrt(R.l2_error_all()))
    rho_ref = _contraction(res)
    # The reference's solution driven to 1e-13 (relative residual).
    rhs = np.sqrt(R.rhs_l2norm())
    n = 6
    while np.sqrt(R.l2_error_all()) / rhs >= 1e-13 and n < 400:
        R.v_cycle(0)
        n += 1
    assert np.sqrt(R.l2_error_all()) / rhs < 1e-13
    x_ref = R.get_x(0)
    lu = R.lu_enabled
    R.close()
    return (coef, S, r), rho_ref, x_ref, lu


def test_129_sigma23_mc8_contraction_within_5pct(contrast129):
    (coef, S, r), rho_ref, _, _ = contrast129
    m = 129
    G = P.Multigrid(m, m, m, smoother=P.SMOOTH_MC8)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    res = [np.sqrt(G.norms()[0])]
    for _ in range(6):
        G.v_cycle(0)
        res.append(np.sqrt(G.norms()[0]))
    rho = _contraction(res)
    assert rho <= 1.05 * rho_ref, (rho, rho_ref)
    G.close()


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_129_sigma23_solution_matches_reference(contrast129, precision):
    (coef, S, r), _, x_ref, _ = contrast129
    m = 129
    G = P.Multigrid(m, m, m, precision=precision)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    cyc, rr = G.solve(1e-10, 200, 0)
    assert rr < 1e-10
    assert relerr(G.get_x(0), x_ref) < 1e-9
    G.close()
