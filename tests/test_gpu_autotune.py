"""The autotuner (pgmg_dev_autotune) and the options it chooses among: every
candidate must leave the iterates bit for bit unchanged, the chosen options
must be valid, and a second handle of the same shape takes the remembered
choice."""
import numpy as np
import pytest

import pgmg_b200 as P
from tests.helpers import q1_problem

pytestmark = pytest.mark.gpu


def make(mno, precision):
    coef, S, r = q1_problem(*mno, sigma=1.0, seed=sum(mno))
    G = P.Multigrid(*mno, precision=precision)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    return G


@pytest.mark.parametrize("mno", [(65, 65, 65), (33, 40, 17)])
@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_autotune_changes_no_result(mno, precision):
    A = make(mno, precision)
    A.solve(1e-10, 100, 1)
    xa = A.get_x(0)
    B = make(mno, precision)
    t = B.autotune()
    assert t["gs_block"] in (128, 256, 512) and t["pdl"] in (0, 1) and t["vcycle_ms"] > 0
    assert 0 <= t["cluster_first"] <= B.nlevels and t["cluster_size"] in (1, 2, 4, 8, 16)
    B.clear_x(0)
    B.solve(1e-10, 100, 1)
    assert np.array_equal(B.get_x(0), xa)
    # The same shape again: the remembered choice, without timing.
    C = make(mno, precision)
    t2 = C.autotune()
    assert {k: t2[k] for k in ("gs_block", "cluster_first", "cluster_size", "pdl")} == \
           {k: t[k] for k in ("gs_block", "cluster_first", "cluster_size", "pdl")}


@pytest.mark.parametrize("block", [128, 256, 512])
def test_gs_block_bitwise(block):
    mno = (41, 41, 41)
    A = make(mno, P.FP64)
    B = make(mno, P.FP64)
    B.set_option(P.OPT_GS_BLOCK, block)
    for _ in range(2):
        A.v_cycle(0)
        B.v_cycle(0)
    assert np.array_equal(A.get_x(0), B.get_x(0))


def test_grid_sweeps_bitwise_and_bounded_wait():
    """The persistent whole-GPU sweeps give the per-pass launches' iterates bit
    for bit; a grid barrier whose wait runs out (it waits for one block more
    than the launch has) ends with PGMG_ERR_TIMEOUT and the device stays
    usable."""
    mno = (129, 97, 65)
    A = make(mno, P.FP64)
    B = make(mno, P.FP64)
    B.set_option(P.OPT_GRID_MAX, 10 ** 8)  # every level above the cluster levels
    for _ in range(2):
        A.v_cycle(0)
        B.v_cycle(0)
    assert np.array_equal(A.get_x(0), B.get_x(0))
    assert P.lib().pgmg_dev_grid_check(B.handle, 1, 0) == 0
    assert P.lib().pgmg_dev_grid_check(B.handle, 1, 1) == 9
    assert P.lib().pgmg_dev_grid_check(B.handle, 1, 0) == 0
    B.clear_x(0)
    A.clear_x(0)
    A.solve(1e-10, 100, 1)
    B.solve(1e-10, 100, 1)
    assert np.array_equal(A.get_x(0), B.get_x(0))


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_grid_sweeps_solve_bitwise(precision):
    mno = (97, 97, 97)
    A = make(mno, precision)
    B = make(mno, precision)
    B.set_option(P.OPT_GRID_MAX, 10 ** 8)
    A.solve(1e-10, 100, 0)
    B.solve(1e-10, 100, 0)
    assert np.array_equal(A.get_x(0), B.get_x(0))


@pytest.mark.parametrize("mno", [(41, 41, 41), (33, 40, 17), (65, 20, 9)])
@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
@pytest.mark.parametrize("vec", [1, 2])
def test_gs_vector_bitwise(mno, precision, vec):
    """The vector-load colour sweeps (16-byte loads: 2 or 4 points per
    thread; or 2 points per thread) give the one-point-per-thread sweep's
    iterates bit for bit, odd sizes included."""
    A = make(mno, precision)
    B = make(mno, precision)
    B.set_option(P.OPT_GS_VECTOR, vec)
    assert B.get_option(P.OPT_GS_VECTOR) == vec
    for _ in range(2):
        A.v_cycle(0)
        B.v_cycle(0)
    assert np.array_equal(A.get_x(0), B.get_x(0))


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_gs_alternate_bitwise(precision):
    """Colour passes alternating their traversal direction give the same
    iterates as passes that all run bottom up."""
    mno = (65, 49, 33)
    A = make(mno, precision)
    B = make(mno, precision)
    A.set_option(P.OPT_GS_ALTERNATE, 0)
    B.set_option(P.OPT_GS_ALTERNATE, 1)
    for _ in range(2):
        A.v_cycle(0)
        B.v_cycle(0)
    assert np.array_equal(A.get_x(0), B.get_x(0))


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
@pytest.mark.parametrize("pdl", [0, 1])
def test_gs_prefetch_bitwise(precision, pdl):
    """Colour passes that load their stencil before the launch dependency
    give the same iterates as the default passes, with and without
    programmatic dependent launches."""
    mno = (97, 65, 49)
    A = make(mno, precision)
    B = make(mno, precision)
    for G in (A, B):
        G.set_option(P.OPT_PDL, pdl)
    A.set_option(P.OPT_GS_PREFETCH, 0)
    B.set_option(P.OPT_GS_PREFETCH, 1 << 30)
    for _ in range(2):
        A.v_cycle(0)
        B.v_cycle(0)
    assert np.array_equal(A.get_x(0), B.get_x(0))


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
@pytest.mark.parametrize("mno,first", [((65, 65, 65), 2), ((97, 81, 49), 2), ((129, 129, 129), 3),
                                       ((65, 65, 65), 1), ((129, 129, 129), 2), ((66, 60, 50), 1)])
def test_coarse_shared_bitwise(precision, mno, first):
    """The cluster coarse cycle sweeping from a shared-memory copy of each
    level's x -- or, for a 33^3-sized level whose copy does not fit, from
    per-CTA windows of z planes -- gives the same iterates as sweeping from
    global memory."""
    A = make(mno, precision)
    B = make(mno, precision)
    for G in (A, B):
        G.set_option(P.OPT_CLUSTER_FIRST, first)
    A.set_option(P.OPT_COARSE_SHARED, 0)
    B.set_option(P.OPT_COARSE_SHARED, 1)
    for _ in range(3):
        A.v_cycle(0)
        B.v_cycle(0)
    assert np.array_equal(A.get_x(0), B.get_x(0))
    for G in (A, B):
        c, rr = G.solve(1e-10, 60, 0)
    assert np.array_equal(A.get_x(0), B.get_x(0))


def test_autotune_cache_file(tmp_path):
    """A shape in the tuning cache gets the stored options without timing."""
    cache = str(tmp_path / "tune.json")
    A = make((65, 49, 33), P.FP64)
    t = A.autotune(cache=cache)
    assert "cached" not in t
    B = make((65, 49, 33), P.FP64)
    B.set_option(P.OPT_GS_BLOCK, 512 if t["gs_block"] != 512 else 128)
    t2 = B.autotune(cache=cache)
    assert t2["cached"] is True
    for name, opt in P.Multigrid.TUNED_OPTIONS.items():
        assert B.get_option(opt) == t[name]
    # Another precision is a different entry.
    C = make((65, 49, 33), P.MIXED)
    assert "cached" not in C.autotune(cache=cache)


@pytest.mark.parametrize("mno", [(65, 65, 65), (41, 33, 18), (66, 34, 20), (129, 97, 65), (20, 33, 9)])
@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_fused_restriction_bitwise(mno, precision):
    """The restriction that computes its residuals in shared memory gives the
    coarse sources of the residual pass plus restriction bit for bit, on odd,
    even and anisotropic grids (tiles cut at every edge), and the same
    solves."""
    A = make(mno, precision)
    A.set_option(P.OPT_FUSED_RESTRICT, 0)
    rng = np.random.default_rng(6)
    xs = [rng.standard_normal(A.npts(l - 1)) for l in range(1, A.nlevels)]
    ref = []
    for l in range(1, A.nlevels):
        A.set_x(l - 1, xs[l - 1])
        A.restriction(l)
        ref.append(A.get_r(l))
    A.clear_x(0)
    A.solve(1e-10, 100, 1)
    xa = A.get_x(0)
    for variant in (1,):
        B = make(mno, precision)
        B.set_option(P.OPT_FUSED_RESTRICT, variant)
        for l in range(1, B.nlevels):
            B.set_x(l - 1, xs[l - 1])
            B.restriction(l)
            assert np.array_equal(B.get_r(l), ref[l - 1]), (variant, l)
            assert not np.any(B.get_x(l))
        B.clear_x(0)
        B.solve(1e-10, 100, 1)
        assert np.array_equal(B.get_x(0), xa), variant


@pytest.mark.parametrize("mno", [(33, 33, 33), (65, 65, 65), (20, 33, 9), (41, 41, 41), (16, 17, 18)])
@pytest.mark.parametrize("coarse", [P.COARSE_LU_EXACT, P.COARSE_LU])
def test_lu_window_same_factors(mno, coarse):
    """The coarse LU factorised in a shared-memory band window gives the
    one-block device-memory factorisation's factors and pivots bit for bit:
    the reference-order coarse solve and the explicit inverse (and so the
    V-cycles that use them) agree exactly."""
    coef, S, r = q1_problem(*mno, sigma=1.0, seed=sum(mno) + 3)
    hs = []
    for win in (0, 1):
        G = P.Multigrid(*mno, coarse=coarse, smoother=P.SMOOTH_LEX)
        G.set_option(P.OPT_LU_WINDOW, win)
        G.setup_matrices(coef, S)
        G.setup_fields(r)
        assert G.lu_enabled
        hs.append(G)
    for _ in range(3):
        for G in hs:
            G.v_cycle(0)
        assert np.array_equal(hs[0].get_x(0), hs[1].get_x(0))


@pytest.mark.parametrize("mno", [(65, 65, 65), (41, 33, 18), (66, 34, 20), (129, 97, 65)])
@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
@pytest.mark.parametrize("block", [128, 256])
def test_gs_tma_bitwise(mno, precision, block):
    """The colour pass whose stencils and sources arrive by bulk copies into
    shared memory gives the iterates of the usual pass bit for bit (odd and
    even sizes: the last CTA's copies are rounded up inside the plane
    padding)."""
    A = make(mno, precision)
    B = make(mno, precision)
    for G in (A, B):
        G.set_option(P.OPT_GS_BLOCK, block)
    B.set_option(P.OPT_GS_TMA, 10 ** 9)  # every level the grid kernels sweep
    for _ in range(2):
        A.v_cycle(0)
        B.v_cycle(0)
    assert np.array_equal(A.get_x(0), B.get_x(0))
    A.clear_x(0)
    B.clear_x(0)
    A.solve(1e-10, 100, 0)
    B.solve(1e-10, 100, 0)
    assert np.array_equal(A.get_x(0), B.get_x(0))


def test_tma_bounded_wait():
    """A TMA pass whose mbarrier expects more bytes than arrive waits about a
    second in all, reports PGMG_ERR_TIMEOUT, and leaves the device usable."""
    mno = (65, 49, 33)
    A = make(mno, P.FP64)
    assert P.lib().pgmg_dev_tma_check(A.handle, 1, 0) == 0
    assert P.lib().pgmg_dev_tma_check(A.handle, 1, 1) == 9
    assert P.lib().pgmg_dev_tma_check(A.handle, 1, 0) == 0
    A.clear_x(0)
    cyc, rr = A.solve(1e-10, 100, 0)
    assert rr < 1e-10


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_gs_l2_prefetch_bitwise(precision):
    """Prefetching the next colour pass's stencils into L2 changes no
    iterate (sweeps in both directions: symmetric mode too)."""
    mno = (97, 81, 65)
    A = make(mno, precision)
    B = make(mno, precision)
    B.set_option(P.OPT_GS_L2_PREFETCH, 10 ** 9)
    for mode in (0, 1, 0):
        A.v_cycle(mode)
        B.v_cycle(mode)
    assert np.array_equal(A.get_x(0), B.get_x(0))
    A.clear_x(0)
    B.clear_x(0)
    A.solve(1e-10, 100, 0)
    B.solve(1e-10, 100, 0)
    assert np.array_equal(A.get_x(0), B.get_x(0))


def _pivoting_problem(m, n, o, seed):
    """Random 27-point stencils (boxes cropped at the grid's faces) whose
    diagonal is small against the rest, so that partial pivoting interchanges
    rows at most steps of the coarse LU."""
    rng = np.random.default_rng(seed)
    N = m * n * o
    k, j, i = np.meshgrid(np.arange(o), np.arange(n), np.arange(m), indexing="ij")
    idx, size = [i.reshape(-1), j.reshape(-1), k.reshape(-1)], [m, n, o]
    slots = np.arange(27)
    d = np.stack([slots % 3 - 1, (slots // 3) % 3 - 1, slots // 9 - 1], 1)
    S = np.zeros((N, 6), np.int32)
    ok = np.ones((N, 27), bool)
    for a in range(3):
        lo = np.where(idx[a] > 0, -1, 0)
        hi = np.where(idx[a] < size[a] - 1, 2, 1)
        S[:, 2 * a], S[:, 2 * a + 1] = lo, hi
        ok &= (d[None, :, a] >= lo[:, None]) & (d[None, :, a] < hi[:, None])
    coef = rng.uniform(-1, 1, (N, 27))
    coef[:, 13] *= 0.05
    coef[~ok] = 0.0
    return coef, S, rng.uniform(-1, 1, N)


@pytest.mark.parametrize("mno", [(9, 9, 9), (10, 9, 8), (6, 7, 5)])
def test_lu_window_pivoting(mno):
    """Both coarse LU kernels on single-level problems whose factorisation
    interchanges rows: the reference-order solve gives the same x bit for bit
    (the window kernel applies the interchanges to the multipliers it has
    already written at the end), and x solves the system."""
    coef, S, r = _pivoting_problem(*mno, seed=sum(mno))
    xs = []
    for win in (0, 1):
        G = P.Multigrid(*mno, coarse=P.COARSE_LU_EXACT, smoother=P.SMOOTH_LEX)
        G.set_option(P.OPT_LU_WINDOW, win)
        G.setup_matrices(coef, S)
        G.setup_fields(r)
        assert G.nlevels == 1 and G.lu_enabled
        G.solve_exact()
        xs.append(G.get_x(0))
        G.close()
    assert np.array_equal(xs[0], xs[1])
    m, n, o = mno
    N = m * n * o
    A = np.zeros((N, N))
    for p in range(N):
        i, j, k = p % m, (p // m) % n, p // (m * n)
        for s in range(27):
            if coef[p, s] != 0.0:
                A[p, (i + s % 3 - 1) + m * ((j + (s // 3) % 3 - 1) + n * (k + s // 9 - 1))] = coef[p, s]
    assert np.abs(A @ xs[0] - r).max() < 1e-9 * np.abs(r).max() * max(1.0, np.abs(xs[0]).max())


def _weak_rows_problem(m, n, o, seed, nweak=8):
    """Diagonally dominant random stencils with a few rows whose diagonal is
    tiny: the LU interchanges rows at some two dozen steps, and the factors
    stay within a band of about 100 (small grids)."""
    rng = np.random.default_rng(seed)
    coef, S, _ = _pivoting_problem(m, n, o, seed)
    ok = coef != 0.0
    ok[:, 13] = True
    coef = rng.uniform(-1, 1, coef.shape) * 0.1
    coef[:, 13] = 4.0
    coef[rng.choice(coef.shape[0], nweak, replace=False), 13] = 1e-3
    coef[~ok] = 0.0
    return coef, S, rng.uniform(-1, 1, coef.shape[0])


@pytest.mark.parametrize("case", ["q1_33", "q1_65", "q1_20x33x9", "weak_4x5x6", "weak_5", "weak_6x5x4",
                                  "weak_8x6x7", "weak_7x6x5", "pivot_9"])
def test_lu_inverse_band_same_inverse(case):
    """The explicit coarse inverse computed one warp per column over the
    factors' band equals the one-block-per-column dense computation bit for
    bit: the coarse solves, and so the V-cycles, agree exactly (Q1 problems;
    single-level problems whose LU interchanges rows at a few steps, with the
    factors still banded; and one with interchanges at most steps, whose
    factors are not banded, where both take the dense kernel)."""
    if case.startswith("q1"):
        mno = {"q1_33": (33, 33, 33), "q1_65": (65, 65, 65), "q1_20x33x9": (20, 33, 9)}[case]
        coef, S, r = q1_problem(*mno, sigma=1.5, seed=7)
    elif case.startswith("weak"):
        # band below the diagonal 87, 81, 74 (4 rows per lane); 161, 140 (8)
        mno = {"weak_4x5x6": (4, 5, 6), "weak_5": (5, 5, 5), "weak_6x5x4": (6, 5, 4), "weak_8x6x7": (8, 6, 7),
               "weak_7x6x5": (7, 6, 5)}[case]
        coef, S, r = _weak_rows_problem(*mno, seed=5)
    else:
        coef, S, r = _pivoting_problem(9, 9, 9, seed=28)
        mno = (9, 9, 9)
    hs = []
    for band in (0, 1):
        G = P.Multigrid(*mno, coarse=P.COARSE_LU, smoother=P.SMOOTH_LEX)
        G.set_option(P.OPT_LU_INVERSE_BAND, band)
        G.setup_matrices(coef, S)
        G.setup_fields(r)
        assert G.lu_enabled
        hs.append(G)
    for _ in range(3):
        for G in hs:
            G.v_cycle(0)
        assert np.array_equal(hs[0].get_x(0), hs[1].get_x(0))
    for G in hs:
        G.close()


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
@pytest.mark.parametrize("pattern", [0b110110, 0b011011, 0b111001])
def test_gs_block_levels_bitwise(precision, pattern):
    """Per-level block sizes of the colour sweep (2 bits per level) give the
    default sweep's iterates bit for bit; the option round-trips."""
    mno = (129, 97, 65)
    A = make(mno, precision)
    B = make(mno, precision)
    B.set_option(P.OPT_CLUSTER_FIRST, B.nlevels)  # every level swept by launches
    A.set_option(P.OPT_CLUSTER_FIRST, A.nlevels)
    B.set_option(P.OPT_GS_BLOCK_LEVELS, pattern)
    assert B.get_option(P.OPT_GS_BLOCK_LEVELS) == pattern
    for _ in range(2):
        A.v_cycle(0)
        B.v_cycle(0)
        assert np.array_equal(A.get_x(0), B.get_x(0))
    A.clear_x(0)
    B.clear_x(0)
    assert A.solve(1e-10, 100, 0) == B.solve(1e-10, 100, 0)
    assert np.array_equal(A.get_x(0), B.get_x(0))
