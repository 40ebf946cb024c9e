"""The allocation-free residual-norm entry point, for callers that cannot
allocate device memory (their framework owns the card's memory, or their
loop must not stall in an allocation).  Compared through the C ABI with the
library's regular norms on the same problem, on two calls in a row; sizes
beyond its fixed scratch are rejected.  Collected last on purpose."""
import numpy as np
import pytest

import pgmg_b200 as P
from tests.helpers import q1_problem, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mno", [(33, 33, 33), (65, 40, 33)])
def test_noalloc_norms_match_regular_norms(mno):
    import torch
    m, n, o = mno
    coef, S, r = q1_problem(m, n, o, sigma=1.0, seed=12)
    G = P.Multigrid(m, n, o)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    dc = torch.from_numpy(coef).cuda()
    dr = torch.from_numpy(r).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(5)
    for call in range(2):
        x = rng.standard_normal(m * n * o) if call == 0 else G.get_x(0)
        G.set_x(0, x)
        res2, rhs2 = G.norms(0)
        dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        P.residual_norms_noalloc(m, n, o, dc.data_ptr(), dx.data_ptr(), dr.data_ptr(), out.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert relerr(got[0], res2) < 1e-12
        assert relerr(got[1], rhs2) < 1e-12
        G.v_cycle(0)  # a different x for the second call


def test_noalloc_rejects_oversize_and_host_pointers():
    import torch
    small = torch.zeros(27, dtype=torch.float64, device="cuda")
    with pytest.raises(P.PgmgError) as e:
        P.residual_norms_noalloc(257, 257, 257, small.data_ptr(), small.data_ptr(), small.data_ptr(),
                                 small.data_ptr())
    assert e.value.status == 7
    host = np.zeros(27)
    with pytest.raises(P.PgmgError):
        P.residual_norms_noalloc(1, 1, 1, host.ctypes.data, small.data_ptr(), small.data_ptr(), small.data_ptr())
