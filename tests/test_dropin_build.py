"""The C++ drop-in headers (include/pgmg/) compile and link against
libpgmg_b200.so with g++ and strict warnings, as a reference driver would be
built -- no GPU needed.  Running the driver is covered by the GPU tests."""
import os
import subprocess

import pytest

from tests.conftest import ROOT

LIB = os.path.join(ROOT, "pgmg_b200", "libpgmg_b200.so")


@pytest.mark.skipif(not os.path.exists(LIB), reason="libpgmg_b200.so not built")
def test_dropin_driver_builds_with_strict_warnings(tmp_path):
    exe = str(tmp_path / "dropin_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include", "pgmg"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_driver.cc"), "-o", exe,
           "-L", os.path.join(ROOT, "pgmg_b200"), "-lpgmg_b200", "-Wl,-rpath," + os.path.join(ROOT, "pgmg_b200")]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-3000:]
    assert os.path.exists(exe)


def test_c_header_compiles_as_c(tmp_path):
    """include/pgmg_dev.h is plain C: a C translation unit including it
    compiles with -std=c99 and strict warnings."""
    src = tmp_path / "t.c"
    src.write_text('#include "pgmg_dev.h"\nint main(void) { pgmg_handle *h = 0; (void)h; return PGMG_OK; }\n')
    out = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I",
                          os.path.join(ROOT, "include"), "-c", str(src), "-o", str(tmp_path / "t.o")],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-3000:]
