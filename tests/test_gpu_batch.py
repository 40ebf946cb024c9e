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
