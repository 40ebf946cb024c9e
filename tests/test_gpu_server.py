"""Continuous-batching server: every request's result equals the same problem
solved alone (bit for bit), under staggered arrivals, RHS-only reuse of
resident hierarchies, and eviction under a small memory cap."""
import numpy as np
import pytest

import pgmg_b200 as P
from pgmg_b200.server import FieldPool, SolveServer, poisson_requests

pytestmark = pytest.mark.gpu


def alone(req, fields):
    m, n, o = req.shape
    G = P.Multigrid(m, n, o, precision=P.MIXED)
    G.assemble_q1(fields.get(req.shape, req.field).data_ptr(), from_log=True, sigma=req.sigma)
    G.rhs_uniform(req.rhs_seed)
    G.clear_x(0)
    cyc, rr = G.solve(1e-10, 100, 1)
    x = G.get_x(0)
    G.close()
    return cyc, rr, x


@pytest.mark.parametrize("cap_mb", [2000, 40])
def test_server_results_equal_alone(cap_mb):
    reqs = poisson_requests(rate=120.0, duration=0.25, seed=3, reuse=0.3, sizes=(17, 33), sigma=(0.5, 2.0))
    assert len(reqs) >= 10
    fields = FieldPool(0)
    srv = SolveServer(cap_mb * 1e6, max_slots=8, precision=P.MIXED, keep_solutions=True, fields=fields,
                      check_every=1)
    done = srv.run(reqs)
    assert len(done) == len(reqs)
    assert any(r.reused for r in done)
    for r in done:
        assert r.relres < 1e-10 and r.finished >= r.arrival
        cyc, rr, x = alone(r, fields)
        assert cyc == r.cycles and rr == r.relres
        assert np.array_equal(x, r.x), r.rid
    srv.close()


def test_server_adaptive_alone_equals_mix():
    """With the adaptive residual-check schedule (evaluated per problem on
    the device), each request's result in the mix equals the same request
    served alone, bit for bit (requests that built their hierarchy: a re-used
    one starts from the reduction factor its earlier solve learned)."""
    reqs = poisson_requests(rate=150.0, duration=0.15, seed=5, reuse=0.3, sizes=(17, 33), sigma=(0.5, 2.0))
    assert len(reqs) >= 8
    fields = FieldPool(0)
    srv = SolveServer(2e9, max_slots=8, precision=P.MIXED, keep_solutions=True, fields=fields)
    done = {r.rid: r for r in srv.run(reqs)}
    srv.close()
    fresh = [r for r in reqs if not done[r.rid].reused][:6]
    assert len(fresh) >= 4
    for r in fresh:
        solo = SolveServer(2e9, max_slots=2, precision=P.MIXED, keep_solutions=True, fields=fields)
        one = solo.run([type(r)(rid=r.rid, arrival=0.0, shape=r.shape, field=r.field, sigma=r.sigma,
                                rhs_seed=r.rhs_seed, problem=r.problem)])[0]
        solo.close()
        d = done[r.rid]
        assert d.relres < 1e-10
        assert one.cycles == d.cycles and one.relres == d.relres
        assert np.array_equal(one.x, d.x), r.rid
