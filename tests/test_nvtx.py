"""NVTX ranges of the library (pgmg_b200/csrc/trace.cuh): a small NVTX tool
(tests/cpp/nvtx_record.c), injected through NVTX_INJECTION64_PATH, records
every range push and pop with the thread's stack of open ranges; the tests
check the ranges a set-up and a solve open, their nesting and their counts."""
import json
import os
import subprocess
import sys
import textwrap
from collections import Counter

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOOL_SRC = os.path.join(ROOT, "tests", "cpp", "nvtx_record.c")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


def _build_tool(tmp_path):
    lib = tmp_path / "libnvtx_record.so"
    subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-o", str(lib), TOOL_SRC, "-lpthread"], check=True)
    return lib


def _read_log(path):
    """(thread, event, path) triples of the recorded pushes and pops."""
    out = []
    for line in open(path):
        tid, ev, *rest = line.rstrip("\n").split(" ", 2)
        out.append((tid, ev, rest[0] if rest else ""))
    return out


def _balanced(events):
    depth = Counter()
    for tid, ev, path in events:
        assert ev in ("push", "pop"), (tid, ev, path)
        depth[tid] += 1 if ev == "push" else -1
        assert depth[tid] >= 0
    return all(d == 0 for d in depth.values())


@pytest.mark.skipif(not os.path.isdir(os.path.join(CUDA_INC, "nvtx3")), reason="no NVTX v3 headers")
def test_recording_tool(tmp_path):
    """The recording tool itself, on the CPU: a program that pushes two
    nested ranges through the NVTX v3 headers."""
    lib = _build_tool(tmp_path)
    src = tmp_path / "probe.c"
    src.write_text(textwrap.dedent("""\
        #include <nvtx3/nvToolsExt.h>
        int main(void) {
            nvtxRangePushA("outer");
            nvtxRangePushA("inner");
            nvtxRangePop();
            nvtxRangePop();
            return 0;
        }
        """))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-O2", "-I" + CUDA_INC, "-o", str(exe), str(src), "-ldl"], check=True)
    log = tmp_path / "nvtx.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(lib), PGMG_NVTX_LOG=str(log))
    subprocess.run([str(exe)], env=env, check=True, timeout=60)
    ev = _read_log(log)
    assert [(e, p) for _, e, p in ev] == [("push", "outer"), ("push", "outer/inner"), ("pop", "outer/inner"),
                                          ("pop", "outer")]


_CHILD = textwrap.dedent("""\
    import json, sys
    import pgmg_b200 as P
    m = 33
    kap = P.problem_kappa(m, m, m, 1.0, 3, 8.0)
    coef, S = P.problem_q1(m, m, m, kap)
    r = P.problem_rhs(m, m, m, 3)
    res = {}
    for name, prec in (("fp64", P.FP64), ("mixed", P.MIXED)):
        G = P.Multigrid(m, m, m, precision=prec, coarse=P.COARSE_LU, smoother=P.SMOOTH_MC8, device=0)
        G.setup_matrices(coef, S)
        G.setup_fields(r)
        res[name] = G.solve(1e-10, 100, 0)
        G.close()
    print(json.dumps(res))
    """)


@pytest.mark.gpu
def test_library_ranges(tmp_path):
    lib = _build_tool(tmp_path)
    log = tmp_path / "nvtx.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(lib), PGMG_NVTX_LOG=str(log))
    out = subprocess.run([sys.executable, "-c", _CHILD], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    c64, c32 = res["fp64"][0], res["mixed"][0]
    assert res["fp64"][1] < 1e-10 and res["mixed"][1] < 1e-10

    ev = [e for e in _read_log(log) if e[2].startswith("pgmg")]
    assert ev and _balanced(ev)
    pushes = Counter(p for _, e, p in ev if e == "push")
    # Set-up of each handle: the stencil upload, then the Galerkin hierarchy
    # with the coarse LU inside it.
    assert pushes["pgmg upload_level0"] == 2
    assert pushes["pgmg build_rat"] == 2 and pushes["pgmg build_rat/pgmg coarse LU"] == 2
    assert pushes["pgmg solve"] == 2
    # FP64: every V-cycle of the solve inside it (the first one enqueued
    # during the source-norm check), and at least two checks.
    v64 = sum(n for p, n in pushes.items() if p.startswith("pgmg solve") and p.endswith("pgmg V-cycle fp64"))
    assert v64 == c64
    assert pushes["pgmg solve/pgmg check/pgmg V-cycle fp64"] == 1
    assert pushes["pgmg solve/pgmg check"] >= 2
    # Mixed: FP32 V-cycles in refinement steps (or enqueued during a check
    # that was expected to continue the solve: at most one beyond the count).
    v32 = sum(n for p, n in pushes.items() if p.endswith("pgmg V-cycle fp32"))
    assert c32 <= v32 <= c32 + 1
    assert pushes["pgmg solve/pgmg refinement step"] >= 1
    assert all(p.startswith(("pgmg solve/pgmg refinement step/", "pgmg solve/pgmg check/"))
               for p in pushes if p.endswith("pgmg V-cycle fp32"))
    assert not any("fp64" in p for p in pushes if "refinement step" in p)
