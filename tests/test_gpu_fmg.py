"""The full multigrid cycle (multigrid::fmg_cycle, multigrid.cc:109-134)
through the C ABI, lexicographic smoother, bit for bit against the reference
itself (oracle/_ref) on the parity grids, from x = 0 and from a random x."""
import numpy as np
import pytest

import pgmg_b200 as P
from oracle.pyoracle import Reference, ref_available
from tests.helpers import q1_problem

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]


@pytest.mark.parametrize("mno", [(17, 17, 17), (33, 33, 33), (16, 17, 18), (20, 33, 9), (41, 41, 41)])
def test_fmg_cycle_lex_bitwise_vs_reference(mno):
    m, n, o = mno
    coef, S, r = q1_problem(m, n, o, sigma=1.0, seed=sum(mno) + 5)
    R = Reference(m, n, o, S, coef, r)
    G = P.Multigrid(m, n, o, coarse=P.COARSE_LU_EXACT if R.lu_enabled else P.COARSE_GS, smoother=P.SMOOTH_LEX)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    G.fmg_cycle(P.SMOOTH_LEX)
    R.fmg_cycle()
    for l in range(G.nlevels):
        assert np.array_equal(G.get_x(l), R.get_x(l)), f"level {l} after one FMG cycle"
    x0 = np.random.default_rng(2).standard_normal(m * n * o)
    G.set_x(0, x0)
    R.set_x(0, x0)
    G.fmg_cycle(P.SMOOTH_LEX)
    R.fmg_cycle()
    assert np.array_equal(G.get_x(0), R.get_x(0))
    # A V-cycle after the FMG cycle stays in step.
    G.v_cycle(0)
    R.v_cycle(0)
    assert np.array_equal(G.get_x(0), R.get_x(0))
