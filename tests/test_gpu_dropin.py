"""The C++ drop-in headers (include/pgmg/) used the way the reference's own
drivers use the reference: compiled with g++ against libpgmg_b200.so, run
on the GPU, checked against the oracle (lexicographic smoother and the
reference-order LU solve, so the V-cycle iterates agree bit for bit)."""
import os
import struct
import subprocess

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.conftest import ROOT
from tests.helpers import q1_problem

pytestmark = pytest.mark.gpu


def build_driver(tmp):
    exe = os.path.join(tmp, "dropin_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include", "pgmg"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_driver.cc"), "-o", exe,
           "-L", os.path.join(ROOT, "pgmg_b200"), "-lpgmg_b200", "-Wl,-rpath," + os.path.join(ROOT, "pgmg_b200")]
    subprocess.run(cmd, check=True)
    return exe


def write_problem(fn, m, n, o, S, coef, r):
    with open(fn, "wb") as f:
        f.write(struct.pack("3i", m, n, o))
        f.write(np.ascontiguousarray(S, np.int32).tobytes())
        f.write(np.ascontiguousarray(coef, np.float64).tobytes())
        f.write(np.ascontiguousarray(r, np.float64).tobytes())


@pytest.mark.parametrize("mno", [(33, 33, 33), (20, 17, 18)])
def test_dropin_driver_matches_oracle(tmp_path, mno):
    m, n, o = mno
    coef, S, r = q1_problem(m, n, o, sigma=1.0, seed=3)
    write_problem(str(tmp_path / "p.bin"), m, n, o, S, coef, r)
    exe = build_driver(str(tmp_path))
    env = dict(os.environ, PGMG_SMOOTHER="lex", PGMG_COARSE="lu_exact")
    out = subprocess.run([exe, str(tmp_path / "p.bin"), str(tmp_path)], check=True, capture_output=True,
                         text=True, env=env).stdout
    lines = [l.split() for l in out.splitlines()]
    O = Oracle(m, n, o, S, coef, r, coarse=True)
    assert int(lines[0][1]) == O.nlevels
    for it in range(3):
        O.v_cycle(0)
        rec = [l for l in lines if l[0] == "vcycle" and int(l[1]) == it][0]
        assert abs(float(rec[2]) - O.l2_error_all()) <= 1e-12 * O.l2_error_all()
    assert abs(float([l for l in lines if l[0] == "rhs"][0][1]) - O.rhs_l2norm()) <= 1e-12 * O.rhs_l2norm()
    # Slice file: reference binary-matrix layout of x after three V-cycles.
    raw = np.fromfile(str(tmp_path / "x.slice"), np.float32).reshape(n + 1, m + 1)
    assert raw[0, 0] == m and np.array_equal(raw[0, 1:], np.arange(m))
    assert np.array_equal(raw[1:, 0], np.arange(n))
    x = O.get_x(0).reshape(o, n, m)[o // 2].astype(np.float32)
    assert np.array_equal(raw[1:, 1:], x)
    assert float([l for l in lines if l[0] == "ax_check"][0][1]) < 1e-12
    # solve_v_cycles: same status and guide state as the oracle.
    ps = 8.0 / 3.0 / (m - 1)
    for rep in range(2):
        O.set_x(0, np.zeros(m * n * o))
        st, res, _ = O.solve_v_cycles(ps)
        rec = [l for l in lines if l[0] == "solve" and int(l[1]) == rep][0]
        assert int(rec[2]) == st == 0
        assert abs(float(rec[3]) - res) <= 1e-10 * res
        assert int(rec[4]) == O.guide_pred_iters()
    # Standalone region sweeps.
    O2 = Oracle(m, n, o, S, coef, r, coarse=True)
    g = [l for l in lines if l[0] == "gs"]
    assert abs(float(g[0][2]) - O2.l2_error_all()) <= 1e-12 * O2.l2_error_all()
    for s in range(1, 4):
        O2.gauss_seidel(0, 0)
        assert abs(float(g[s][2]) - O2.l2_error_all()) <= 1e-12 * O2.l2_error_all()
