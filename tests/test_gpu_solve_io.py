"""pgmg_dev_solve_io (source in, solution out, in one call, with the
solution's copy overlapping the final residual check) against the same solve
through the separate entry points: identical iterates, cycle counts and
relative residuals, bit for bit, in both precisions, with host pinned and
pageable buffers; and the FP64 solve's first V-cycle, which is enqueued
before the source norm is read, undone when the source is zero."""
import numpy as np
import pytest

import pgmg_b200 as P
from tests.helpers import periodic_problem, q1_problem

pytestmark = pytest.mark.gpu


def _pair(mno, precision, prd=(False, False, False)):
    if any(prd):
        coef, S, r = periodic_problem(*mno, prd, seed=4)
    else:
        coef, S, r = q1_problem(*mno, sigma=1.0, seed=9)
    hs = []
    for _ in range(2):
        G = P.Multigrid(*mno, precision=precision, prd=prd)
        G.setup_matrices(coef, S)
        hs.append(G)
    return hs, r


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
@pytest.mark.parametrize("mno,prd", [((65, 65, 65), (False, False, False)), ((33, 40, 29), (False, False, False)),
                                     ((24, 20, 16), (True, False, True))])
@pytest.mark.parametrize("check_every", [0, 1])
def test_solve_io_equals_separate_calls(precision, mno, prd, check_every):
    import torch
    (A, B), r = _pair(mno, precision, prd)
    # Three solves each way: from the second on, a solve starts from the
    # reduction factor the handle remembered from the one before.
    ref = []
    for _ in range(3):
        A.setup_fields(r)
        c, rr = A.solve(1e-10, 100, check_every)
        ref.append((c, rr, A.get_x(0)))
    hr = torch.from_numpy(np.ascontiguousarray(r)).pin_memory()
    for k in range(3):
        if k < 2:  # pinned host buffers
            hx = torch.full((r.size,), np.nan, dtype=torch.float64).pin_memory()
            c, rr = B.solve_io(hr.data_ptr(), hx.data_ptr(), 1e-10, 100, check_every)
            x = hx.numpy()
        else:  # pageable
            x = np.full(r.size, np.nan)
            c, rr = B.solve_io(r, x, 1e-10, 100, check_every)
        assert (c, rr) == ref[k][:2], k
        assert np.array_equal(x, ref[k][2]), k
    A.close()
    B.close()


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_zero_source_gives_zero_solution(precision):
    (A, B), r = _pair((33, 33, 33), precision)
    z = np.zeros(r.size)
    x = np.full(r.size, np.nan)
    c, rr = B.solve_io(z, x, 1e-10, 100, 0)
    assert c == 0 and rr == 0.0 and not np.any(x)
    A.setup_fields(z)
    c, rr = A.solve(1e-10, 100, 0)
    assert c == 0 and not np.any(A.get_x(0))
    A.close()
    B.close()
