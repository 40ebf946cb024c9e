"""Device-side input synthesis and caller-owned handle memory."""
import numpy as np
import pytest

import pgmg_b200 as P
from tests.helpers import q1_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mno", [(17, 17, 17), (33, 20, 17), (9, 12, 10)])
def test_device_assembly_equals_host(mno):
    m, n, o = mno
    kap = P.problem_kappa(m, n, o, 1.3, 4)
    coef, S = P.problem_q1(m, n, o, kap)
    r = P.problem_rhs(m, n, o, 4)
    H = P.Multigrid(m, n, o)
    H.setup_matrices(coef, S)
    D = P.Multigrid(m, n, o)
    D.assemble_q1(kap)
    D.rhs_uniform(4)
    assert np.array_equal(D.get_coef(0), H.get_coef(0).reshape(-1, 27))
    assert np.array_equal(D.get_boxes(0), S.reshape(-1, 6))
    assert np.array_equal(D.get_r(0), r)
    for l in range(1, H.nlevels):
        assert np.array_equal(D.get_coef(l), H.get_coef(l))
    # constant kappa
    c1, S1 = P.problem_q1(m, n, o)
    D.assemble_q1(None)
    assert np.array_equal(D.get_coef(0), c1.reshape(-1, 27))
    # kappa = exp(sigma * g) on the device: the host exp and the device exp
    # may differ in the last bit, so compare to 1e-14.
    g = P.problem_gauss(m, n, o, 4)
    D.assemble_q1(g, from_log=True, sigma=1.3)
    assert np.abs(D.get_coef(0) - coef.reshape(-1, 27)).max() <= 1e-14 * np.abs(coef).max()


def test_handle_in_caller_memory_matches():
    import torch
    m = n = o = 33
    coef, S, r = q1_problem(m, n, o)
    nbytes = P.plan_bytes(m, n, o, P.MIXED)
    buf = torch.empty(nbytes + 256, dtype=torch.uint8, device="cuda")
    base = (buf.data_ptr() + 255) // 256 * 256
    A = P.Multigrid(m, n, o, precision=P.MIXED, mem=(base, nbytes))
    B = P.Multigrid(m, n, o, precision=P.MIXED)
    for G in (A, B):
        G.setup_matrices(coef, S)
        G.setup_fields(r)
        G.solve(1e-10, 50, 1)
    assert np.array_equal(A.get_x(0), B.get_x(0))
    with pytest.raises(P.PgmgError):
        P.Multigrid(m, n, o, precision=P.MIXED, mem=(base, nbytes // 2))
    A.close()
    del buf
