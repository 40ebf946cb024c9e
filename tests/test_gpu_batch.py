"""Batched solves: uneven problems in one launch per level and colour give,
problem by problem, exactly the iterates of the same problem solved alone
(pgmg_dev_solve_relres with a residual check every cycle)."""
import numpy as np
import pytest

import pgmg_b200 as P
from tests.helpers import q1_problem

pytestmark = pytest.mark.gpu

SHAPES = [(33, 33, 33), (65, 33, 17), (17, 65, 33), (33, 17, 65), (65, 65, 33), (41, 33, 25), (17, 17, 17),
          (9, 9, 9)]


def build(mno, precision, seed):
    m, n, o = mno
    coef, S, r = q1_problem(m, n, o, sigma=0.5 + 0.25 * (seed % 7), seed=seed)
    G = P.Multigrid(m, n, o, precision=precision)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    return G


@pytest.mark.parametrize("precision", [P.MIXED, P.FP64])
def test_batch_equals_alone(precision):
    probs = [build(s, precision, 10 + i) for i, s in enumerate(SHAPES)]
    B = P.Batch(16, precision)
    slots = [0, 3, 4, 5, 8, 9, 12, 15]
    for s, G in zip(slots, probs):
        B.attach(s, G)
    cyc, rr = B.solve(1e-10, 60)
    xb = [G.get_x(0) for G in probs]
    for s, G, x in zip(slots, probs, xb):
        assert rr[s] < 1e-10 and cyc[s] > 0
        G.clear_x(0)
        c1, r1 = G.solve(1e-10, 60, 1)
        assert c1 == cyc[s] and r1 == rr[s]
        assert np.array_equal(G.get_x(0), x)
    # The same problem in a smaller mix (detach others): same result again.
    for s in slots[1:]:
        B.detach(s)
    cyc2, rr2 = B.solve(1e-10, 60)
    assert cyc2[slots[0]] == cyc[slots[0]]
    assert np.array_equal(probs[0].get_x(0), xb[0])
    B.close()


def test_batch_rejects_unsupported():
    B = P.Batch(4, P.MIXED)
    G = build((17, 17, 17), P.FP64, 1)
    with pytest.raises(P.PgmgError):
        B.attach(0, G)  # precision differs
    G2 = P.Multigrid(17, 17, 17, precision=P.MIXED, smoother=P.SMOOTH_LEX)
    coef, S, r = q1_problem(17, 17, 17)
    G2.setup_matrices(coef, S)
    with pytest.raises(P.PgmgError):
        B.attach(0, G2)  # lexicographic smoother
    B.close()


@pytest.mark.parametrize("precision", [P.MIXED, P.FP64])
def test_batch_adaptive_schedule(precision):
    """Adaptive residual checks, per problem on the device: every problem
    converges, fewer checks than cycles are paid, and a problem's result is
    the same in the mix and in a batch of its own."""
    probs = [build(s, precision, 30 + i) for i, s in enumerate(SHAPES)]
    B = P.Batch(8, precision)
    B.set_option(P.OPT_CHECK_EVERY, 0)
    for s, G in enumerate(probs):
        B.attach(s, G)
    cyc, rr = B.solve(1e-10, 60)
    xb = [G.get_x(0) for G in probs]
    for s, G in enumerate(probs):
        assert rr[s] < 1e-10 and cyc[s] > 0
        # Close to the problem's own FP64-checked solve.
        H = build(SHAPES[s], precision, 30 + s)
        H.solve(1e-12, 80, 1)
        xh = H.get_x(0)
        assert np.abs(xb[s] - xh).max() / np.abs(xh).max() < 1e-8
    B.close()
    # The same problems, fresh (same starting state), each in a batch of its
    # own: the same result as in the mix.
    for s in (0, 3, 7):
        G = build(SHAPES[s], precision, 30 + s)
        C = P.Batch(2, precision)
        C.set_option(P.OPT_CHECK_EVERY, 0)
        C.attach(1, G)
        c1, r1 = C.solve(1e-10, 60)
        assert c1[1] == cyc[s] and r1[1] == rr[s]
        assert np.array_equal(G.get_x(0), xb[s])
        C.close()


def test_batch_cluster_size_changes_no_result():
    """The coarse-tail cluster size of a batch (default 4 CTAs per problem)
    changes no iterate: 1, 4 and 16 CTAs, and the handles' own size, give the
    same cycles and solutions bit for bit."""
    out = []
    for cs in (1, 4, 16, 0):
        probs = [build(s, P.MIXED, 50 + i) for i, s in enumerate(SHAPES[:5])]
        B = P.Batch(8, P.MIXED)
        B.set_option(P.OPT_CLUSTER_SIZE, cs)
        for s, G in enumerate(probs):
            B.attach(s, G)
        cyc, rr = B.solve(1e-10, 60)
        out.append((cyc[:5].copy(), rr[:5].copy(), [G.get_x(0) for G in probs]))
        B.close()
        for G in probs:
            G.close()
    for cyc, rr, xs in out[1:]:
        assert np.array_equal(cyc, out[0][0]) and np.array_equal(rr, out[0][1])
        for a, b in zip(xs, out[0][2]):
            assert np.array_equal(a, b)
