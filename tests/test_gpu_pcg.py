"""The PCG helpers of the reference's single-process path (region.cc:
1848-1940, region.hh:226-236, multigrid.hh:222-251) on the device, through
the C ABI, against the reference's own helpers (oracle/_ref):

* bit for bit: compute_residual, Ax / unpadded_Ax (periodic axes wrap),
  l0_error_all (a maximum), copy_rhs_to_soln;
* 1e-12 relative: source_soln_dot and soln_diff (the same terms summed in
  another order)."""
import numpy as np
import pytest

import pgmg_b200 as P
from oracle.pyoracle import Reference, ref_available
from tests.helpers import periodic_problem, q1_problem

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]


def rel(a, b):
    return abs(a - b) / abs(b)


@pytest.mark.parametrize("mno", [(33, 33, 33), (16, 17, 18), (20, 33, 9)])
def test_pcg_helpers_match_reference(mno):
    m, n, o = mno
    coef, S, r = q1_problem(m, n, o, sigma=1.0, seed=sum(mno) + 1)
    R = Reference(m, n, o, S, coef, r)
    G = P.Multigrid(m, n, o)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    rng = np.random.default_rng(4)
    x = rng.standard_normal(m * n * o)
    G.set_x(0, x)
    R.set_x(0, x)
    assert np.array_equal(G.get_field(0, P.FIELD_RES), R.compute_residual())
    v = rng.standard_normal(m * n * o)
    av = G.apply(0, v)
    assert np.array_equal(av, R.Ax(v))
    assert np.array_equal(av, R.Ax(v, unpadded=True))
    assert G.l0_error() == R.l0_error_all()
    assert rel(G.source_soln_dot(), R.source_soln_dot()) < 1e-12
    ext = x + 1e-3 * rng.standard_normal(m * n * o)
    assert rel(G.soln_diff(ext), R.soln_diff(ext)) < 1e-12
    G.copy_rhs_to_soln()
    R.copy_rhs_to_soln()
    assert np.array_equal(G.get_x(0), R.get_x(0))
    assert np.array_equal(G.get_x(0), r)
    # A few V-cycles later the helpers still agree (lexicographic smoother,
    # the reference's coarse solver: the iterates are equal bit for bit).
    L = P.Multigrid(m, n, o, coarse=P.COARSE_LU_EXACT if R.lu_enabled else P.COARSE_GS, smoother=P.SMOOTH_LEX)
    L.setup_matrices(coef, S)
    L.setup_fields(r)
    R.set_x(0, np.zeros(m * n * o))
    for _ in range(2):
        L.v_cycle(0)
        R.v_cycle(0)
    assert L.l0_error() == R.l0_error_all()
    assert rel(L.source_soln_dot(), R.source_soln_dot()) < 1e-12


@pytest.mark.parametrize("mno,prd", [((16, 12, 18), (True, False, True)), ((16, 16, 16), (True, True, True))])
def test_pcg_helpers_periodic(mno, prd):
    coef, S, r = periodic_problem(*mno, prd, seed=9)
    R = Reference(*mno, S, coef, r, prd=prd)
    G = P.Multigrid(*mno, prd=prd)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    N = mno[0] * mno[1] * mno[2]
    rng = np.random.default_rng(8)
    v = rng.standard_normal(N)
    assert np.array_equal(G.apply(0, v), R.Ax(v, unpadded=True))
    x = rng.standard_normal(N)
    G.set_x(0, x)
    R.set_x(0, x)
    assert rel(G.source_soln_dot(), R.source_soln_dot()) < 1e-12
    G.copy_rhs_to_soln()
    R.copy_rhs_to_soln()
    assert np.array_equal(G.get_x(0), R.get_x(0))
