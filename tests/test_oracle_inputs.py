"""The oracle's input generator (oracle/inputs.c) gives the same arrays as
the library's host generators, bit for bit, so that the reference arm of the
benchmark can build the benchmark problem without loading the product
library."""
import numpy as np
import pytest

import pgmg_b200 as P
from oracle import pyoracle as O


@pytest.mark.parametrize("mno,sigma,seed,width", [((9, 10, 11), 1.0, 3, 8.0), ((33, 17, 25), 2.3, 7, 8.0),
                                                  ((65, 65, 65), 1.0, 1, 8.0), ((20, 12, 10), 0.5, 11, 2.0),
                                                  ((5, 3, 2), 1.7, 0, 0.0)])
def test_inputs_match_product_generators(mno, sigma, seed, width):
    m, n, o = mno
    assert np.array_equal(O.input_gauss(m, n, o, seed, width), P.problem_gauss(m, n, o, seed, width))
    kap_o = O.input_kappa(m, n, o, sigma, seed, width)
    kap_p = P.problem_kappa(m, n, o, sigma, seed, width)
    assert np.array_equal(kap_o, kap_p)
    c_o, S_o = O.input_q1(m, n, o, kap_o)
    c_p, S_p = P.problem_q1(m, n, o, kap_p)
    assert np.array_equal(c_o, c_p.reshape(-1))
    assert np.array_equal(S_o, S_p.reshape(-1))
    assert np.array_equal(O.input_rhs(m, n, o, seed), P.problem_rhs(m, n, o, seed))


def test_constant_q1_matches():
    c_o, S_o = O.input_q1(17, 9, 13)
    c_p, S_p = P.problem_q1(17, 9, 13)
    assert np.array_equal(c_o, c_p.reshape(-1)) and np.array_equal(S_o, S_p.reshape(-1))


def test_benchmark_problem_helper():
    coef, S, r = O.benchmark_problem(17, 17, 17, 1.0, 5)
    kap = P.problem_kappa(17, 17, 17, 1.0, 5, 8.0)
    c_p, S_p = P.problem_q1(17, 17, 17, kap)
    assert np.array_equal(coef, c_p.reshape(-1)) and np.array_equal(S, S_p.reshape(-1))
    assert np.array_equal(r, P.problem_rhs(17, 17, 17, 5))
