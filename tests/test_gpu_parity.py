"""GPU parity: the CUDA path (through the C ABI) against the oracle, which is
itself pinned bit for bit to the reference (tests/test_oracle_pin.py), and
against the reference directly where oracle/_ref is present.

Tolerances: bit-exact (array_equal) for the Galerkin stencils, boxes,
restriction, interpolation and both Gauss-Seidel smoothers and the
lexicographic V-cycle with reference-order coarse solves; 1e-12 relative
(max-norm, relative to the largest entry) for the explicit-inverse coarse
solve and the norms (parallel reduction order).
"""
import numpy as np
import pytest

import pgmg_b200 as P
from oracle.pyoracle import Oracle, Reference, ref_available
from tests.helpers import q1_problem, relerr, simple_problem

pytestmark = pytest.mark.gpu

SIZES = [(17, 17, 17), (16, 17, 18), (20, 33, 9), (33, 33, 33), (34, 18, 10), (41, 41, 41)]


def make(mno, coarse=P.COARSE_LU_EXACT, precision=P.FP64, sigma=1.0, seed=None, smoother=P.SMOOTH_MC8):
    m, n, o = mno
    coef, S, r = q1_problem(m, n, o, sigma=sigma, seed=sum(mno) if seed is None else seed)
    G = P.Multigrid(m, n, o, precision=precision, coarse=coarse, smoother=smoother)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    return G, (coef, S, r)


def oracle_for(mno, prob, lu):
    m, n, o = mno
    coef, S, r = prob
    return Oracle(m, n, o, S, coef, r, coarse=lu)


@pytest.mark.parametrize("mno", SIZES)
def test_rat_and_boxes_bitwise(mno):
    G, prob = make(mno)
    O = oracle_for(mno, prob, G.lu_enabled)
    assert G.nlevels == O.nlevels
    for l in range(G.nlevels):
        assert G.dims(l) == O.dims(l)
        assert np.array_equal(G.get_boxes(l), O.get_S(l))
        assert np.array_equal(G.get_coef(l), O.get_A27(l))


@pytest.mark.parametrize("mno", SIZES)
def test_transfers_bitwise(mno):
    G, prob = make(mno)
    O = oracle_for(mno, prob, G.lu_enabled)
    rng = np.random.default_rng(11)
    for l in range(1, G.nlevels):
        xf = rng.standard_normal(G.npts(l - 1))
        G.set_x(l - 1, xf)
        O.set_x(l - 1, xf)
        G.restriction(l)
        O.restriction(l)
        assert np.array_equal(G.get_r(l), O.get_r(l))
        assert not np.any(G.get_x(l))
        xc = rng.standard_normal(G.npts(l))
        for h in (G, O):
            h.set_x(l, xc)
            h.set_x(l - 1, xf)
            h.interpolation(l)
        assert np.array_equal(G.get_x(l - 1), O.get_x(l - 1))


@pytest.mark.parametrize("mno", SIZES)
@pytest.mark.parametrize("mode", [0, 1])
def test_gauss_seidel_bitwise(mno, mode):
    G, prob = make(mno)
    O = oracle_for(mno, prob, G.lu_enabled)
    rng = np.random.default_rng(3)
    for l in range(G.nlevels):
        x0 = rng.standard_normal(G.npts(l))
        rr = rng.standard_normal(G.npts(l))
        for h in (G, O):
            h.set_x(l, x0)
            h.set_r(l, rr)
        G.gauss_seidel(mode, l, P.SMOOTH_LEX)
        O.gauss_seidel(mode, l)
        assert np.array_equal(G.get_x(l), O.get_x(l)), f"lex level {l}"
        for h in (G, O):
            h.set_x(l, x0)
        G.gauss_seidel(mode, l, P.SMOOTH_MC8)
        O.gauss_seidel_mc8(mode, l)
        assert np.array_equal(G.get_x(l), O.get_x(l)), f"mc8 level {l}"


@pytest.mark.parametrize("mno", [(17, 17, 17), (16, 17, 18), (33, 33, 33), (41, 41, 41)])
@pytest.mark.parametrize("coarse", [P.COARSE_LU_EXACT, P.COARSE_GS])
def test_lex_vcycle_bitwise(mno, coarse):
    G, prob = make(mno, coarse=coarse, smoother=P.SMOOTH_LEX)
    O = oracle_for(mno, prob, G.lu_enabled)
    if coarse == P.COARSE_LU_EXACT:
        assert G.lu_enabled == O.lu_enabled == True  # noqa: E712
    for it in range(4):
        G.v_cycle(0)
        O.v_cycle(0)
        assert np.array_equal(G.get_x(0), O.get_x(0)), f"cycle {it}"
    G.v_cycle(1)
    O.v_cycle(1)
    assert np.array_equal(G.get_x(0), O.get_x(0))
    res_g, rhs_g = G.norms()
    assert relerr(res_g, O.l2_error_all()) < 1e-12
    assert relerr(rhs_g, O.rhs_l2norm()) < 1e-12


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("mno", [(33, 33, 33), (16, 17, 18)])
def test_lex_vcycle_matches_reference_directly(mno):
    m, n, o = mno
    coef, S, r = q1_problem(m, n, o, sigma=1.0, seed=sum(mno))
    R = Reference(m, n, o, S, coef, r)
    coarse = P.COARSE_LU_EXACT if R.lu_enabled else P.COARSE_GS
    G = P.Multigrid(m, n, o, coarse=coarse, smoother=P.SMOOTH_LEX)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    assert G.lu_enabled == R.lu_enabled
    for it in range(3):
        G.v_cycle(0)
        R.v_cycle(0)
        assert np.array_equal(G.get_x(0), R.get_x(0))


@pytest.mark.parametrize("mno", [(33, 33, 33), (20, 33, 9)])
def test_inverse_coarse_solve_close_to_lu(mno):
    G, prob = make(mno, coarse=P.COARSE_LU, smoother=P.SMOOTH_LEX)
    O = oracle_for(mno, prob, True)
    assert G.lu_enabled and O.lu_enabled
    lb = G.nlevels - 1
    rr = np.random.default_rng(5).standard_normal(G.npts(lb))
    G.set_r(lb, rr)
    O.set_r(lb, rr)
    G.solve_exact()
    O.solve_exact(lb)
    assert relerr(G.get_x(lb), O.get_x(lb)) < 1e-12
    G.setup_fields(prob[2])
    O.set_x(0, np.zeros(G.npts(0)))
    for it in range(4):
        G.v_cycle(0)
        O.v_cycle(0)
        assert relerr(G.get_x(0), O.get_x(0)) < 1e-12


def test_small_grids_and_single_level():
    for mno in [(2, 2, 2), (3, 3, 3), (5, 4, 3), (11, 10, 9)]:
        G, prob = make(mno, smoother=P.SMOOTH_LEX)
        O = oracle_for(mno, prob, G.lu_enabled)
        assert G.nlevels == O.nlevels == 1
        for it in range(2):
            G.v_cycle(0)
            O.v_cycle(0)
        assert np.array_equal(G.get_x(0), O.get_x(0))


def test_interpolation_of_linear_field_is_exact():
    coef, S, r = simple_problem(65, 65, 65)
    G = P.Multigrid(65, 65, 65)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    G.clear_x(2)
    G.setup_test(1, True, 3)
    G.interpolation(3)
    m, n, o = G.dims(2)
    j = np.broadcast_to(np.arange(n)[None, :, None], (o, n, m)).ravel()
    np.testing.assert_array_equal(G.get_x(2), j / 2.0)


def test_solve_v_cycles_matches_oracle():
    mno = (33, 33, 33)
    G, prob = make(mno, coarse=P.COARSE_LU_EXACT, smoother=P.SMOOTH_LEX)
    O = oracle_for(mno, prob, True)
    ps = 8.0 / 3 / 32
    for rep in range(2):
        G.clear_x(0)
        O.set_x(0, np.zeros(G.npts(0)))
        st_g, res_g, cyc = G.solve_v_cycles(ps)
        st_o, res_o, sweeps = O.solve_v_cycles(ps)
        assert st_g == st_o == 0
        assert relerr(res_g, res_o) < 1e-10
        assert np.array_equal(G.get_x(0), O.get_x(0))


@pytest.mark.parametrize("mno", [(33, 33, 33), (65, 65, 65)])
def test_mc8_contraction_within_5pct_of_reference(mno):
    """Per-V-cycle residual reduction of the 8-colour smoother vs the
    reference's lexicographic smoother (geometric mean over cycles 2-6):
    the 8-colour factor must be no worse than 1.05x the reference's.  (It is
    smaller -- faster convergence -- on these Q1 problems.)"""
    Gl, prob = make(mno, coarse=P.COARSE_LU, smoother=P.SMOOTH_LEX)
    Gm, _ = make(mno, coarse=P.COARSE_LU, smoother=P.SMOOTH_MC8)

    def factors(G):
        r = [G.l2_error_all()]
        for it in range(6):
            G.v_cycle(0)
            r.append(G.l2_error_all())
        f = np.sqrt(np.array(r[1:]) / np.array(r[:-1]))
        return np.exp(np.log(f[1:]).mean())

    fl, fm = factors(Gl), factors(Gm)
    assert fm <= 1.05 * fl, (fm, fl)


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_solve_relres_against_fp64_oracle(precision):
    mno = (33, 33, 33)
    G, prob = make(mno, precision=precision, coarse=P.COARSE_LU, sigma=2.3)
    cyc, rr = G.solve(1e-10, 60, 1)
    assert rr < 1e-10, (cyc, rr)
    # FP64 oracle solve driven to 1e-13 relative residual.
    O = oracle_for(mno, prob, True)
    rhs2 = O.rhs_l2norm()
    for it in range(100):
        if np.sqrt(O.l2_error_all() / rhs2) < 1e-13:
            break
        O.v_cycle(0)
    xo = O.get_x(0)
    assert relerr(G.get_x(0), xo) < 1e-9


def test_errors_are_statuses():
    G = P.Multigrid(9, 9, 9)
    with pytest.raises(P.PgmgError) as e:
        G.v_cycle()
    assert e.value.status == 6
    coef, S, r = q1_problem(9, 9, 9)
    bad = S.reshape(-1, 6).copy()
    bad[0] = [-1, 2, -1, 2, -1, 2]  # corner box leaves the grid
    with pytest.raises(P.PgmgError) as e:
        G.setup_matrices(coef, bad.ravel())
    assert e.value.status == 7
    with pytest.raises(P.PgmgError):
        G.gauss_seidel(0, 5)


@pytest.mark.parametrize("mno", [(33, 33, 33), (65, 65, 65), (41, 41, 41), (16, 17, 18), (20, 33, 9)])
def test_mc8_vcycle_bitwise(mno):
    """The 8-colour V-cycle (grid kernels on fine levels, the one-cluster
    kernel on coarse ones, 24 coarse sweeps) equals the oracle's 8-colour
    V-cycle bit for bit."""
    G, prob = make(mno, coarse=P.COARSE_GS, smoother=P.SMOOTH_MC8)
    O = oracle_for(mno, prob, False)
    O.set_smoother(True)
    for it in range(3):
        G.v_cycle(0)
        O.v_cycle(0)
        assert np.array_equal(G.get_x(0), O.get_x(0)), f"cycle {it}"
    G.v_cycle(1)
    O.v_cycle(1)
    assert np.array_equal(G.get_x(0), O.get_x(0))


@pytest.mark.parametrize("mno", [(33, 33, 33), (65, 65, 65)])
def test_mc8_vcycle_with_lu_close(mno):
    G, prob = make(mno, coarse=P.COARSE_LU, smoother=P.SMOOTH_MC8)
    O = oracle_for(mno, prob, True)
    O.set_smoother(True)
    for it in range(3):
        G.v_cycle(0)
        O.v_cycle(0)
        assert relerr(G.get_x(0), O.get_x(0)) < 1e-12, f"cycle {it}"


@pytest.mark.parametrize("mno,budget", [((33, 33, 33), 100_000), ((65, 65, 65), 400_000), ((41, 41, 41), 150_000)])
def test_mc8_slab_order_bitwise(mno, budget):
    """Slab-blocked 8-colour sweeps (forced by a small slab budget) on the
    grid, single-block and cluster paths equal the oracle's slab order."""
    G, prob = make(mno, coarse=P.COARSE_GS, smoother=P.SMOOTH_MC8)
    G.set_option(P.OPT_SLAB_BUDGET, budget)
    O = oracle_for(mno, prob, False)
    O.set_smoother(True)
    O.set_slab_budget(budget)
    for it in range(2):
        G.v_cycle(0)
        O.v_cycle(0)
        assert np.array_equal(G.get_x(0), O.get_x(0)), f"cycle {it}"
    G.v_cycle(1)
    O.v_cycle(1)
    assert np.array_equal(G.get_x(0), O.get_x(0))


def test_apply_matches_oracle_residual():
    mno = (20, 17, 18)
    G, prob = make(mno)
    O = oracle_for(mno, prob, True)
    v = np.random.default_rng(9).standard_normal(G.npts(0))
    av = G.apply(0, v)
    O.set_x(0, v)
    O.set_r(0, np.zeros(G.npts(0)))
    # oracle residual with r = 0 is -A v, accumulated in the same order
    O.set_r(0, np.zeros(G.npts(0)))
    A = O.get_A27(0)
    m, n, o = mno
    ref = np.zeros(m * n * o)
    x3 = np.pad(v.reshape(o, n, m), 1)
    for q in range(27):
        di, dj, dk = q % 3 - 1, (q // 3) % 3 - 1, q // 9 - 1
        ref += A[:, q] * x3[1 + dk:1 + dk + o, 1 + dj:1 + dj + n, 1 + di:1 + di + m].ravel()
    assert relerr(av, ref) < 1e-14


def test_sweep_count_options():
    mno = (33, 33, 33)
    G, prob = make(mno, coarse=P.COARSE_GS, smoother=P.SMOOTH_MC8)
    assert (G.get_option(P.OPT_V_DOWN), G.get_option(P.OPT_V_UP), G.get_option(P.OPT_V_BOTTOM)) == (2, 2, 20)
    G.set_option(P.OPT_V_DOWN, 3)
    G.set_option(P.OPT_V_UP, 1)
    r0 = G.l2_error_all()
    G.v_cycle(0)
    r1 = G.l2_error_all()
    assert r1 < 1e-2 * r0
    G2, _ = make(mno, coarse=P.COARSE_GS, smoother=P.SMOOTH_MC8)
    G2.v_cycle(0)
    assert not np.array_equal(G.get_x(0), G2.get_x(0))


@pytest.mark.parametrize("mno", [(65, 65, 65), (81, 40, 66), (66, 58, 49), (97, 33, 70)])
@pytest.mark.parametrize("rat_tile", [0, 1])
def test_rat_large_levels_bitwise(mno, rat_tile):
    """Coarse levels of more than 20,000 points, built one thread per coarse
    point (default) or by the tiled kernel (one thread per coarse point and
    stencil slot): boxes and stencils bit for bit the oracle's, on odd, even
    and mixed sizes whose tiles are cut at every edge."""
    m, n, o = mno
    coef, S, r = q1_problem(m, n, o, sigma=1.0, seed=sum(mno))
    G = P.Multigrid(m, n, o, coarse=P.COARSE_LU_EXACT)
    G.set_option(P.OPT_RAT_TILE, rat_tile)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    O = oracle_for(mno, (coef, S, r), G.lu_enabled)
    assert G.nlevels == O.nlevels
    assert G.dims(1)[0] * G.dims(1)[1] * G.dims(1)[2] > 20000
    for l in range(G.nlevels):
        assert np.array_equal(G.get_boxes(l), O.get_S(l)), l
        assert np.array_equal(G.get_coef(l), O.get_A27(l)), l
