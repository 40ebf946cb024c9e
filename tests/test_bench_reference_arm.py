"""bench.py --impl reference on the CPU: the reference's own multigrid
solving a small case of the benchmark problem prints one JSON line with the
benchmark's metric and the keys the reference arm carries.  Skipped when the
compiled reference is absent."""
import json
import os
import subprocess
import sys

import pytest

from oracle.pyoracle import ref_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--size", "33", "--steps", "2",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    # the reference's own printf output (grid hierarchy) goes to stderr
    assert len(lines) == 1 and lines[0].startswith("{"), out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "s/solve" and d["higher_is_better"] is False
    assert d["steps"] == 2 and d["warmup"] == 1 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert 1 <= d["config"]["cycles"] < 100


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_reference_arm_loads_no_product_library():
    """The reference arm builds its inputs with the oracle library's generator:
    the product library is never mapped into its process."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--size', '17', '--steps', '1', "
            "'--warmup', '1']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT_MAPPED', 'libpgmg_b200' in maps, 'REF_MAPPED', 'libpgmg_ref' in maps)")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "PRODUCT_MAPPED False REF_MAPPED True" in out.stdout, out.stdout[-2000:]


def test_reference_arm_other_ranks_print_nothing():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--size", "17", "--steps", "1",
                          "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
