"""The CPU baseline of the batch and serving benchmarks: the reference solving
a sample of problems in a spawn-started pool of host processes.  Runs on the
CPU (tiny problems); skipped when the compiled reference is absent."""
import pytest

import bench
from oracle.pyoracle import ref_available


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_pool_baseline_solves_every_job():
    jobs = [((17, 17, 9), 1.0, 101, [0], 1e-10), ((9, 17, 17), 0.7, 102, [1, 2], 1e-10)]
    out = bench.cpu_pool_baseline(jobs, True, "two tiny problems")
    assert out["kind"] == "reference" and out["unit"] == "solves/s"
    assert out["cores"] >= 1 and out["value"] > 0
    assert "3 solves" in out["sample"]
    lo, hi = out["cycles_min_max"]
    assert 1 <= lo <= hi < 100


def test_pool_baseline_empty_sample():
    assert bench.cpu_pool_baseline([], False, "nothing") is None
