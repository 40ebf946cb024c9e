"""C-ABI library: loads on a machine without a GPU, exports every symbol
include/pgmg_dev.h declares, host generators are deterministic, and the
device entry points fail with a status (not a crash) without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import pgmg_b200 as P
from tests.conftest import ROOT, gpu_available


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "pgmg_dev.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pgmg_(?:dev|problem)_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(P.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    bound = {name for name, _, _ in P.SIGNATURES}
    assert set(syms) <= bound, set(syms) - bound


def test_generators_deterministic():
    a = P.problem_kappa(9, 10, 11, 1.0, 3)
    b = P.problem_kappa(9, 10, 11, 1.0, 3)
    c = P.problem_kappa(9, 10, 11, 1.0, 4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    g = np.log(a)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1.0) < 1e-12
    r1 = P.problem_rhs(9, 10, 11, 3)
    assert np.array_equal(r1, P.problem_rhs(9, 10, 11, 3))
    r3 = r1.reshape(11, 10, 9)
    assert np.all(r3[0] == 0) and np.all(r3[:, 0] == 0) and np.all(r3[:, :, -1] == 0)
    inner = r3[1:-1, 1:-1, 1:-1]
    assert inner.min() >= -1 and inner.max() <= 1 and inner.std() > 0.4


def test_q1_constant_stencil():
    m = 9
    coef, S = P.problem_q1(m, m, m)
    h = 1.0 / (m - 1)
    c = coef.reshape(-1, 27)
    st = c[4 + 9 * (4 + 9 * 4)].reshape(3, 3, 3)
    ndiff = np.add.outer(np.add.outer([1, 0, 1], [1, 0, 1]), [1, 0, 1])  # differing coordinates
    expect = np.choose(ndiff, [8 / 3, 0.0, -1 / 6, -1 / 12]) * h
    np.testing.assert_allclose(st, expect, rtol=1e-15, atol=1e-17)
    assert abs(st.sum()) < 1e-15
    # Boundary rows: one positive fix entry, box [0,1)^3.
    assert np.count_nonzero(c[0]) == 1 and c[0, 13] == pytest.approx(8 / 3 * h)
    assert list(S.reshape(-1, 6)[0]) == [0, 1, 0, 1, 0, 1]


def test_plan_bytes_and_levels():
    b65 = P.plan_bytes(65, 65, 65)
    b257 = P.plan_bytes(257, 257, 257)
    bm = P.plan_bytes(257, 257, 257, P.MIXED)
    assert 0 < b65 < b257 < bm
    # 27 FP64 stencils per point dominate.
    assert b257 > 27 * 8 * 257 ** 3


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU path")
def test_create_without_gpu_raises():
    with pytest.raises(P.PgmgError) as e:
        P.Multigrid(9, 9, 9)
    assert e.value.status == 12


def test_create_rejects_bad_args():
    d = P.Dims(1, 9, 9, 0, 0, 0, 0, 0, 0, -1)
    h = C.c_void_p()
    assert P.lib().pgmg_dev_create(C.byref(d), C.byref(h)) == 7
    # Periodic axes pass argument checks (without a GPU: no device).
    d = P.Dims(8, 9, 9, 1, 0, 0, 0, 0, 0, -1)
    rc = P.lib().pgmg_dev_create(C.byref(d), C.byref(h))
    assert rc in (0, 12)
    if rc == 0:
        P.lib().pgmg_dev_destroy(h)


def test_q1_variable_kappa_stencil_symmetric():
    """The interior block of the assembled operator is symmetric, rows sum to
    zero, and the element couplings use the kappa of the shared cells."""
    m = 9
    kap = P.problem_kappa(m, m, m, 1.0, 1, 2.0)
    coef, S = P.problem_q1(m, m, m, kap)
    C = coef.reshape(m, m, m, 27)
    inner = C[1:-1, 1:-1, 1:-1]
    assert np.abs(inner.sum(-1)).max() < 1e-14
    for q in range(27):
        di, dj, dk = q % 3 - 1, (q // 3) % 3 - 1, q // 9 - 1
        a = C[2:-2, 2:-2, 2:-2, q]
        b = C[2 + dk:m - 2 + dk, 2 + dj:m - 2 + dj, 2 + di:m - 2 + di, 26 - q]
        assert np.abs(a - b).max() < 1e-15
    # Corner coupling (+1,+1,+1) of node (1,1,1) comes only from cell (1,1,1).
    K = kap.reshape(m - 1, m - 1, m - 1)
    h = 1.0 / (m - 1)
    assert C[1, 1, 1, 26] == pytest.approx(-h * K[1, 1, 1] / 12, rel=1e-14)


def test_dropin_headers_compile_and_link(tmp_path):
    """The drop-in C++ headers compile with a driver written against the
    reference's interface and link against libpgmg_b200.so (no GPU needed)."""
    import subprocess
    exe = tmp_path / "dropin_driver"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include", "pgmg"), "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "dropin_driver.cc"), "-o",
                    str(exe), "-L", os.path.join(ROOT, "pgmg_b200"), "-lpgmg_b200"], check=True)
    assert exe.exists()


@pytest.mark.parametrize("mno", [(257, 257, 257), (1 << 21, 1 << 21, 1 << 21), (2**31 - 1, 2**31 - 1, 2**31 - 1),
                                 (2**31 - 1, 1, 1), (1, 1, 2**31 - 1), (4097, 4097, 1)])
def test_noalloc_rejects_oversize_before_any_launch(mno):
    """Grids beyond the allocation-free entry point's fixed scratch are
    rejected by the argument check, before any pointer is looked at or any
    kernel launched, including sizes whose point count would overflow a
    64-bit product.  (The pointers passed are not valid memory.)"""
    m, n, o = mno
    fake = C.c_void_p(0x1000)
    assert P.lib().pgmg_residual_norms_noalloc(m, n, o, fake, fake, fake, fake, None) == 7
