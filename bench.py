#!/usr/bin/env python
"""Benchmark: seconds to a 1e-10 relative residual on a 257^3
variable-coefficient 27-point Q1 problem (kappa = exp(sigma*g), sigma = 1.0,
Gaussian-smoothed seeded field of width 8 cells), FP64 on one B200.

One step = one solve from x = 0: V-cycles (2+l pre/post sweeps on level l,
8-colour Gauss-Seidel, FP64 LU on the coarsest level) until
sqrt(sum r^2 / sum b^2) < 1e-10, with residual checks where the observed
reduction factor predicts convergence (the mixed-precision solve runs its
FP32 V-cycles between FP64 residual checks the same way).

  python bench.py [--gpus N --steps K --warmup W]          this library
  python bench.py --impl reference [--steps K --warmup W]  the reference's own
                                                           CPU multigrid

Prints one JSON line (rank 0).  ``value`` is the device-timed s/solve with
the operator and source resident in device memory (inputs > L2, so no flush
is needed); ``e2e`` times the same solve through the C ABI from pinned host
buffers (source up, solution down, pgmg_dev_solve_io) every step.  Under
torchrun every rank solves its own replica (independent problems; no
collective on the data path) and the line reports the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to 1e-10 rel residual @257^3 (FP64 GPU; mixed FP32/FP64 alongside)"
UNIT = "s/solve"
BYTES_GS_PER_POINT = {8: (27 + 3) * 8, 4: (27 + 3) * 4}  # algorithmic bytes per point-sweep


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=257)
    ap.add_argument("--sigma", type=float, default=1.0)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--tune-cache", default=None,
                    help="JSON file of autotuner choices: a shape found there is not re-tuned (so that the same "
                         "command run under a profiler uses the options a plain run chose)")
    ap.add_argument("--workload", default="solve257",
                    choices=["solve257", "small65", "large513", "batch96", "serve", "entrypoints"],
                    help="solve257 is the benchmark line; small65 .. serve measure the other configurations; "
                         "entrypoints times every drop-in entry point on its own at --size")
    ap.add_argument("--profile-mixed", action="store_true",
                    help="only the mixed-precision solves of the benchmark problem (for profiler launch lists)")
    ap.add_argument("--smoother", default="mc8", choices=["mc8", "lex"],
                    help="lex: the reference-order wavefront smoother instead of 8 colours")
    ap.add_argument("--device-setup", action="store_true",
                    help="assemble the stencils and the source on the GPU (same values as the host generators)")
    ap.add_argument("--batch-problems", type=int, default=96, help="problems in the batch96 workload")
    ap.add_argument("--set-option", action="append", default=[], metavar="NAME=VALUE",
                    help="an execution option (as named in Multigrid.TUNED_OPTIONS) applied after autotuning, "
                         "e.g. to profile a kernel variant the tuner did not choose; repeatable")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-seq-seconds", type=float, default=60.0,
                    help="time budget of the one-request-at-a-time comparison")
    ap.add_argument("--serve-sustained-seconds", type=float, default=30.0,
                    help="length of the second serving run, at a fraction of the saturated throughput (0 = skip)")
    ap.add_argument("--serve-sustained-fraction", type=float, default=0.7,
                    help="arrival rate of the second serving run as a fraction of the saturated throughput")
    return ap.parse_args()


# ----------------------------------------------------------------- helpers

class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.f = None

    def _lines(self):
        try:
            with open(self.f.name) as fh:
                return sum(1 for _ in fh)
        except Exception:
            return 0

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
            # The timed region starts once the sampler is producing samples.
            t0 = time.time()
            while self._lines() < 1 and time.time() - t0 < 10 and self.proc.poll() is None:
                time.sleep(0.02)
            self.skip = self._lines()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            # Keep it until it has logged the samples taken during the region.
            t0 = time.time()
            while self._lines() < self.skip + 2 and time.time() - t0 < 2 and self.proc.poll() is None:
                time.sleep(0.02)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for q, line in enumerate(fh):
                p = [x.strip() for x in line.split(",")]
                if q >= getattr(self, "skip", 0) and len(p) >= 9 and p[1].replace(".", "").isdigit():
                    rows.append(p)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3] not in ("", "[N/A]"))}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(name: str):
    """Per-launch DRAM bytes of a kernel, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except Exception:
        pass
    return None


def apply_set_options(G, a):
    """--set-option NAME=VALUE pairs onto a handle (after its autotuning)."""
    import pgmg_b200 as P
    for kv in a.set_option:
        name, val = kv.split("=", 1)
        G.set_option(P.Multigrid.TUNED_OPTIONS[name], int(val))


def build_problem(m, sigma, seed):
    import pgmg_b200 as P
    kap = P.problem_kappa(m, m, m, sigma, seed, 8.0)
    coef, S = P.problem_q1(m, m, m, kap)
    del kap
    r = P.problem_rhs(m, m, m, seed)
    return coef, S, r


# ----------------------------------------------------------------- reference

def reference_cycles(R, tol, max_cycles=100):
    """The reference's own multigrid (oracle/_ref): V-cycles with a residual
    check after each, to the relative tolerance.  Returns (cycles, relres)."""
    rhs2 = R.rhs_l2norm()
    n = 0
    while True:
        rr = np.sqrt(R.l2_error_all() / rhs2)
        if rr < tol or n >= max_cycles or not np.isfinite(rr):
            return n, rr
        R.v_cycle(0)
        n += 1


def reference_solve(R, tol, predicted, max_cycles=100):
    """One solve from the current x the way the reference's own
    solve_v_cycles works (multigrid.hh:182-219): the predicted number of
    V-cycles before the first residual check, then one more cycle per check
    until the relative residual is below tol.  Returns (cycles, relres)."""
    rhs2 = R.rhs_l2norm()
    n = 0
    for _ in range(predicted):
        R.v_cycle(0)
        n += 1
    while True:
        rr = np.sqrt(R.l2_error_all() / rhs2)
        if rr < tol or n >= max_cycles or not np.isfinite(rr):
            return n, rr
        R.v_cycle(0)
        n += 1


def reference_discovery(R, tol, max_cycles=100):
    """A solve from x = 0 with a residual check after every V-cycle, to find
    the cycle count.  Also returns the time the reference's own solve would
    take with that count predicted: the source norm, the V-cycles and one
    final residual check, each measured here (the earlier checks only find
    the count and are not counted)."""
    t0 = time.perf_counter()
    rhs2 = R.rhs_l2norm()
    t_norm = time.perf_counter() - t0
    t_cycles = 0.0
    n = 0
    while True:
        t0 = time.perf_counter()
        rr = np.sqrt(R.l2_error_all() / rhs2)
        t_check = time.perf_counter() - t0
        if rr < tol or n >= max_cycles or not np.isfinite(rr):
            return n, rr, t_norm + t_cycles + t_check
        t0 = time.perf_counter()
        R.v_cycle(0)
        t_cycles += time.perf_counter() - t0
        n += 1


def run_reference(a):
    """--impl reference: the reference's own CPU multigrid (compiled from its
    sources into oracle/_ref with a single-rank MPI shim) on the same 257^3
    problem, whose seeded inputs come from the oracle library's generator
    (the product library is never loaded).  An untimed solve from x = 0 finds
    the reference's cycle count; each warm-up step is one V-cycle; each timed
    step is a full solve from x = 0 with that count predicted, as the
    reference's solve_v_cycles runs it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.pyoracle import Reference, benchmark_problem, ref_available
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpgmg_ref.so not built"}))
        return
    m = a.size
    tg = time.perf_counter()
    coef, S, r = benchmark_problem(m, m, m, a.sigma, a.seed)
    gen_s = time.perf_counter() - tg
    t0 = time.perf_counter()
    R = Reference(m, m, m, S, coef, r)
    setup_s = time.perf_counter() - t0
    del coef, S
    zero = np.zeros(m * m * m)
    R.set_x(0, zero)
    t0 = time.perf_counter()
    cycles, rr, _ = reference_discovery(R, a.tol)
    discovery_s = time.perf_counter() - t0
    for _ in range(a.warmup):
        R.v_cycle(0)
    times = []
    for _ in range(a.steps):
        R.set_x(0, zero)
        t0 = time.perf_counter()
        c, rr = reference_solve(R, a.tol, cycles)
        times.append(time.perf_counter() - t0)
    v = float(np.mean(times))
    sample = (f"{a.steps} full solves from x = 0, each {cycles} V-cycles (the count an untimed solve with a check "
              f"after every cycle found, {discovery_s:.1f} s) then a residual check, as the reference's own "
              f"solve_v_cycles runs a predicted count")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded kappa field and RHS)",
        "config": {"workload": f"{m}^3 Q1 variable-kappa sigma={a.sigma}, solve to {a.tol} rel residual",
                   "cycles": c, "final_relres": rr, "lu_enabled": R.lu_enabled, "setup_s": setup_s,
                   "input_generation_s": gen_s, "inputs": "oracle library generator (bit for bit the library's)",
                   "warmup_step": "one V-cycle", "step_s_min_max": [min(times), max(times)]},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": sample + "; one core: the reference has no threading and no MPI here"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- ours

def run_ours(a):
    import torch

    import pgmg_b200 as P
    from pgmg_b200.replicas import Replicas
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    world, rank = rep.world, rep.rank
    barrier, max_over_ranks = rep.barrier, rep.max

    m = a.size
    npts = m ** 3
    smoother = P.SMOOTH_LEX if a.smoother == "lex" else P.SMOOTH_MC8
    tg = time.perf_counter()
    if a.device_setup:
        gfield = P.problem_gauss(m, m, m, rep.seed(a.seed), 8.0)
        coef = S = None
    else:
        coef, S, r = build_problem(m, a.sigma, rep.seed(a.seed))
    gen_s = time.perf_counter() - tg

    stream = torch.cuda.Stream(device=torch.device("cuda", local))
    G = P.Multigrid(m, m, m, precision=P.FP64, coarse=P.COARSE_LU, smoother=smoother, device=local)
    G.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()

    def setup(H):
        if a.device_setup:
            H.assemble_q1(gfield, from_log=True, sigma=a.sigma)
            H.rhs_uniform(rep.seed(a.seed))
        else:
            H.setup_matrices(coef, S)
            H.setup_fields(r)

    t0 = time.perf_counter()
    setup(G)
    G.sync()
    setup_s = time.perf_counter() - t0
    if a.device_setup:
        r = G.get_field(0, P.FIELD_R)
    # Result-neutral execution options chosen by the library's autotuner
    # (before any timed region).
    tuning = G.autotune(cache=a.tune_cache)
    apply_set_options(G, a)

    def solve_once(H):
        H.clear_x(0)
        return H.solve(a.tol, 100, 0)

    # --- device-resident solves -------------------------------------------
    for _ in range(a.warmup):
        cyc, rr = solve_once(G)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = G.launches
    with Clocks(local) as clk:
        ev0.record(stream)
        cyc_list = []
        for _ in range(a.steps):
            cyc, rr = solve_once(G)
            cyc_list.append(cyc)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1) / a.steps
    launches_total = G.launches - launches0
    launches = launches_total // a.steps
    clocks = clk.summary()
    ms = max_over_ranks(ms)
    final_relres = rr

    # --- end to end through the C ABI with pinned host buffers -------------
    hr = torch.from_numpy(r).pin_memory()
    hx = torch.empty(npts, dtype=torch.float64).pin_memory()
    # pgmg_dev_solve_io: the source copied in, the solve, the solution copied
    # out (its copy overlapping the final residual check), in one call.
    for _ in range(1):
        G.solve_io(hr.data_ptr(), hx.data_ptr(), a.tol, 100, 0)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        G.solve_io(hr.data_ptr(), hx.data_ptr(), a.tol, 100, 0)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / a.steps)

    # --- roofline of the dominant kernel: level-0 8-colour sweep ----------
    nsw = 8
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    G.clear_x(0)
    G.gauss_seidel(0, 0, smoother)
    torch.cuda.synchronize()
    k0.record(stream)
    for _ in range(nsw):
        G.gauss_seidel(0, 0, smoother)
    k1.record(stream)
    torch.cuda.synchronize()
    launch_ms = k0.elapsed_time(k1) / (8 * nsw)
    alg_bytes = BYTES_GS_PER_POINT[8] * npts / 8  # one colour = N/8 point updates
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    # DRAM bytes per level-0 pass: the warm-cache capture of the 257^3
    # passes (as in a live solve); other sizes scale the cold 193^3 capture.
    if m == 257:
        traffic = profiled_traffic("gs_colour_fp64_257_warm.md")
    else:
        traffic = profiled_traffic("gs_colour_fp64_193.md")
        if traffic:
            traffic *= (m ** 3) / 257 ** 3

    # --- mixed precision alongside ----------------------------------------
    mixed = None
    if not a.no_mixed:
        Gm = P.Multigrid(m, m, m, precision=P.MIXED, coarse=P.COARSE_LU, smoother=smoother, device=local)
        Gm.set_stream(stream.cuda_stream)
        setup(Gm)
        mixed_tuning = Gm.autotune(cache=a.tune_cache)
        apply_set_options(Gm, a)
        for _ in range(a.warmup):
            mc, mr = solve_once(Gm)
        torch.cuda.synchronize()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        for _ in range(a.steps):
            mc, mr = solve_once(Gm)
        m1.record(stream)
        torch.cuda.synchronize()
        mms = max_over_ranks(m0.elapsed_time(m1) / a.steps)
        xm = Gm.get_x(0)
        xd = hx.numpy()  # FP64 solution of the last end-to-end step
        mixed = {"value": mms / 1e3, "unit": UNIT, "cycles": mc, "relres": mr, "tuning": mixed_tuning,
                 "speedup_vs_fp64": ms / mms,
                 "max_rel_diff_vs_fp64_solution": float(np.abs(xm - xd).max() / np.abs(xd).max())}
        Gm.close()

    # --- CPU baseline: the reference itself, bounded sample ---------------
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        if coef is None:
            coef, S = P.problem_q1(m, m, m, P.problem_kappa(m, m, m, a.sigma, rep.seed(a.seed), 8.0))
        cpu = cpu_baseline(a, coef, S, r)

    if rank == 0:
        line = {
            "metric": METRIC, "value": rep.per_solve(ms) / 1e3, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded kappa field and RHS)",
            "config": {"workload": f"{m}^3 Q1 variable-kappa sigma={a.sigma} FP64, solve to {a.tol} rel residual",
                       "levels": G.nlevels, "cycles": cyc_list[-1], "final_relres": final_relres,
                       "smoother": ("lexicographic (wavefront) Gauss-Seidel" if a.smoother == "lex"
                                    else "8-colour Gauss-Seidel"), "coarse": "FP64 LU (explicit inverse)",
                       "l2": f"inputs larger than L2 ({216 * m ** 3 / 1e9:.2f} GB of level-0 stencils)",
                       "setup_s": setup_s,
                       "host_generation_s": gen_s, "parallelism": f"replicas x{world}", "tuning": tuning,
                       "per_rank_s_per_solve": ms / 1e3},
            "e2e": {"value": rep.per_solve(e2e_ms) / 1e3, "unit": UNIT, "h2d_bytes_per_step": npts * 8,
                    "d2h_bytes_per_step": npts * 8},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic if a.smoother == "mc8" else None,
                         "kernel": ("k_gs_colour<double> level 0" if a.smoother == "mc8"
                                    else "k_gs_plane<double> level 0 (per colour-sized share of a sweep)"),
                         "peak_source": peak_kind, "launch_ms": launch_ms},
            "gpu_launches": launches_total, "gpu_launches_per_step": launches,
            "clocks": clocks,
            "mixed": mixed,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    G.close()
    rep.close()


def cpu_baseline(a, coef, S, r):
    """The reference (oracle/_ref) on one host core: its set-up (untimed) and
    one full solve from x = 0 with a residual check after every V-cycle.  The
    value is that solve as the reference's own solve_v_cycles would run it
    with the count predicted: the source norm, the V-cycles and the final
    check, all measured in this solve."""
    from oracle.pyoracle import Reference, ref_available
    if not ref_available():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": "oracle/_ref not built"}
    m = a.size
    t0 = time.perf_counter()
    R = Reference(m, m, m, S, coef, r)
    setup_s = time.perf_counter() - t0
    R.set_x(0, np.zeros(m * m * m))
    n_ref, rr, solve_s = reference_discovery(R, a.tol)
    lu = R.lu_enabled
    R.close()
    return {"value": solve_s, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"one full solve from x = 0: {n_ref} V-cycles to {rr:.2e} (lu_enabled={lu}); timed: the "
                      f"source norm, the V-cycles and the final residual check (set-up {setup_s:.1f} s untimed)"}


# ----------------------------------------------------------------- other configurations

def vcycle_bytes(dims, s, v_down=2, v_up=2):
    """Algorithmic bytes of one V-cycle (2+l / 1+l+... sweeps as the cycle runs)
    with s-byte scalars: sweeps (27+3)s per point, residual+restriction
    (27+2)s per fine point + s per coarse point, interpolation 2s per fine point
    + s per coarse point, coarse solve n^2 * 8."""
    npts = [m * n * o for (m, n, o) in dims]
    b = 0.0
    L = len(dims)
    for l in range(L - 1):
        b += (v_down + l) * 30 * s * npts[l] + (v_up + l) * 30 * s * npts[l]
        b += 29 * s * npts[l] + s * npts[l + 1]
        b += 2 * s * npts[l] + s * npts[l + 1]
    b += npts[-1] ** 2 * 8
    return b


def level_dims(m, n, o):
    dims = [(m, n, o)]
    while m * n * o > 1024:
        m, n, o = (m + 2) >> 1, (n + 2) >> 1, (o + 2) >> 1
        dims.append((m, n, o))
    return dims


def ir_step_bytes(m, n, o):
    """One mixed-precision refinement step: FP64 residual (27+2)*8 + FP32 source
    write 4, FP32 V-cycle, FP32 clear 4 and FP64 update 8+4+8 per fine point."""
    N = m * n * o
    return vcycle_bytes(level_dims(m, n, o), 4) + (29 * 8 + 4 + 4 + 20) * N


def timed(stream, fn, reps):
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    out = None
    for _ in range(reps):
        out = fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps / 1e3, out


def run_small65(a):
    """Config 1: 65^3 constant-coefficient Q1, Dirichlet, FP64, to 1e-10;
    this library on the GPU and the reference on one host core."""
    import torch

    import pgmg_b200 as P
    from oracle.pyoracle import Reference, ref_available
    m = 65
    coef, S = P.problem_q1(m, m, m)
    r = P.problem_rhs(m, m, m, a.seed)
    st = torch.cuda.Stream()
    G = P.Multigrid(m, m, m)
    G.set_stream(st.cuda_stream)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    tuning = G.autotune(cache=a.tune_cache)  # result-neutral options, before the timed region

    def solve():
        G.clear_x(0)
        return G.solve(a.tol, 100, 0)
    for _ in range(a.warmup):
        solve()
    t, (cyc, rr) = timed(st, solve, a.steps)
    ref = None
    if ref_available():
        R = Reference(m, m, m, S, coef, r)
        ts = []
        for _ in range(3):
            R.set_x(0, np.zeros(m ** 3))
            t0 = time.perf_counter()
            n_ref, rr_ref = reference_cycles(R, a.tol)
            ts.append(time.perf_counter() - t0)
        ref = {"value": float(np.median(ts)), "unit": UNIT, "cores": 1, "kind": "reference", "cycles": n_ref,
               "lu_enabled": R.lu_enabled, "sample": "3 full solves, median"}
    print(json.dumps({"workload": "65^3 constant-kappa Q1 FP64 to 1e-10 (config 1)", "value": t, "unit": UNIT,
                      "cycles": cyc, "relres": rr, "steps": a.steps, "warmup": a.warmup, "tuning": tuning,
                      "cpu_baseline": ref}))


def _ref_sample_worker(job):
    """The reference's set-up and two V-cycles (each followed by its residual
    check) of a seeded variable-kappa problem, in a host process of its own,
    with inputs from the oracle library's generator.  Returns (set-up s, s
    per V-cycle with its check, relative residual after the two cycles,
    lu_enabled)."""
    m, sigma, seed, tol = job
    from oracle.pyoracle import Reference, benchmark_problem
    coef, S, r = benchmark_problem(m, m, m, sigma, seed)
    t0 = time.perf_counter()
    R = Reference(m, m, m, S, coef, r)
    setup = time.perf_counter() - t0
    del coef, S
    rhs2 = R.rhs_l2norm()
    t0 = time.perf_counter()
    for _ in range(2):
        R.v_cycle(0)
        rr = float(np.sqrt(R.l2_error_all() / rhs2))
    per_cycle = (time.perf_counter() - t0) / 2
    lu = R.lu_enabled
    R.close()
    return setup, per_cycle, rr, lu


def large_cpu_baseline(a, m, sigma, seed, m_sample=257):
    """The reference on one host core for an m^3 solve.  The unmodified
    reference cannot be set up at 513^3 in one process: it counts the level's
    stencil entries in an int (region.hh:61, 494-510), and 27 x 513^3 = 3.6e9
    overflows it (std::bad_array_new_length).  So its set-up and two V-cycles
    run at m_sample^3 with the same sigma (a spawn-started host process), the
    time per V-cycle is scaled by the point ratio (a V-cycle's work is linear
    in the points), and the solve by the reference's cycle count at m^3 --
    the count of this library's lexicographic mode, which runs the
    reference's algorithm in its order (its iterates are the reference's bit
    for bit where the reference runs)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    import torch

    import pgmg_b200 as P
    from oracle.pyoracle import ref_available
    if not ref_available():
        return None
    with ProcessPoolExecutor(1, mp_context=mp.get_context("spawn")) as pool:
        setup, per_cycle, rr2, lu = pool.submit(_ref_sample_worker, (m_sample, sigma, seed, a.tol)).result()
    scale = (m / m_sample) ** 3
    L = P.Multigrid(m, m, m, coarse=P.COARSE_LU_EXACT if lu else P.COARSE_GS, smoother=P.SMOOTH_LEX)
    L.assemble_q1(P.problem_gauss(m, m, m, seed, 8.0), from_log=True, sigma=sigma)
    L.rhs_uniform(seed)
    n_ref, rr = L.solve(a.tol, 300, 1)
    L.close()
    torch.cuda.empty_cache()
    return {"value": per_cycle * scale * n_ref, "unit": UNIT, "cores": 1, "kind": "reference",
            "estimate": True,
            "sample": f"the reference cannot be set up at {m}^3 in one process (int stencil-entry count, "
                      f"region.hh:61,494-510); set-up ({setup:.1f} s, untimed) and 2 V-cycles with residual checks "
                      f"at {m_sample}^3, sigma {sigma} ({per_cycle:.2f} s per cycle, relres {rr2:.2e} after 2), "
                      f"scaled by the point ratio {scale:.2f} and by {n_ref} cycles to {a.tol}, the reference "
                      f"algorithm's count at {m}^3 (lexicographic GPU mode, lu_enabled={lu})"}


def run_large513(a):
    """Config 3: 513^3, sigma 2.3: FP64 and mixed solves to 1e-10, and the
    error of each against the library's FP64 solve driven to 1e-13 (that FP64
    path agrees with the reference's own solution driven to 1e-13 within 1e-9
    at 129^3 and sigma 2.3, tests/test_gpu_benchscale.py); the reference on
    one host core beside it."""
    import torch

    import pgmg_b200 as P
    m = 513
    sigma = 2.3
    t0 = time.perf_counter()
    g = P.problem_gauss(m, m, m, a.seed, 8.0)
    gen_s = time.perf_counter() - t0
    st = torch.cuda.Stream()
    out = {"workload": "513^3 Q1 variable-kappa sigma=2.3 to 1e-10 (config 3)", "unit": UNIT,
           "host_generation_s": gen_s}
    xs = {}
    for name, prec in (("fp64", P.FP64), ("mixed", P.MIXED)):
        G = P.Multigrid(m, m, m, precision=prec)
        G.set_stream(st.cuda_stream)
        t0 = time.perf_counter()
        G.assemble_q1(g, from_log=True, sigma=sigma)
        G.sync()
        setup = time.perf_counter() - t0
        G.rhs_uniform(a.seed)

        def solve():
            G.clear_x(0)
            return G.solve(a.tol, 200, 0)
        for _ in range(max(1, a.warmup - 1)):
            solve()
        t, (cyc, rr) = timed(st, solve, max(1, a.steps // 2))
        xs[name] = G.get_x(0)
        out[name] = {"value": t, "cycles": cyc, "relres": rr, "setup_s": setup, "memory_gb": G.memory_bytes / 1e9}
        if prec == P.FP64:
            # reference solution: continue the FP64 iteration to 1e-13
            cyc2, rr2 = G.solve(1e-13, 300, 1)
            xs["ref"] = G.get_x(0)
            out["reference_solution"] = {"relres": rr2, "extra_cycles": cyc2}
        G.close()
        torch.cuda.empty_cache()
    nrm = np.abs(xs["ref"]).max()
    out["fp64"]["max_err_vs_1e-13"] = float(np.abs(xs["fp64"] - xs["ref"]).max() / nrm)
    out["mixed"]["max_err_vs_1e-13"] = float(np.abs(xs["mixed"] - xs["ref"]).max() / nrm)
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["value"] / out["mixed"]["value"]
    dims = level_dims(m, m, m)
    out["fp64"]["vcycle_roofline_ms"] = vcycle_bytes(dims, 8) / measured_peak_hbm()[0] / 1e6
    out["reference_solution"]["what"] = ("this library's FP64 solve continued to 1e-13 (its FP64 path is pinned "
                                         "to the reference's own solution at 129^3, sigma 2.3)")
    if not a.no_cpu_baseline:
        out["cpu_baseline"] = large_cpu_baseline(a, m, sigma, a.seed)
    print(json.dumps(out))


def _ref_problem_worker(job):
    """One problem of the batch or serving CPU baseline, in a host process of
    its own: the problem built with the oracle library's generator (the same
    arrays the library's host and device generators give), the reference's set-up, then its V-cycles to tol
    for each right-hand side.  Returns (set-up s, [solve s per RHS], cycles)."""
    (m, n, o), sigma, field_seed, rhs_seeds, tol = job
    from oracle.pyoracle import Reference, input_kappa, input_q1, input_rhs
    kap = input_kappa(m, n, o, sigma, field_seed, 8.0)
    coef, S = input_q1(m, n, o, kap)
    del kap
    t0 = time.perf_counter()
    R = Reference(m, n, o, S, coef, input_rhs(m, n, o, rhs_seeds[0]))
    setup = time.perf_counter() - t0
    solves, cycles = [], []
    for k, rs in enumerate(rhs_seeds):
        if k:
            R.set_r(0, input_rhs(m, n, o, rs))
        R.set_x(0, np.zeros(m * n * o))
        t0 = time.perf_counter()
        c, _ = reference_cycles(R, tol)
        solves.append(time.perf_counter() - t0)
        cycles.append(c)
    return setup, solves, cycles


def cpu_pool_baseline(jobs, with_setup, sample):
    """The reference on the host cores: independent single-process solves,
    one per core at a time (a spawn-started pool: no process forks after the
    GPU is in use), throughput summed over the wall time of the sample."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    from oracle.pyoracle import ref_available
    if not ref_available() or not jobs:
        return None
    cores = max(1, min(os.cpu_count() or 1, len(jobs), 16))
    t0 = time.perf_counter()
    # (A worker that dies breaks the pool and raises here, instead of being
    # re-spawned.)
    with ProcessPoolExecutor(cores, mp_context=mp.get_context("spawn")) as pool:
        res = list(pool.map(_ref_problem_worker, jobs))
    wall = time.perf_counter() - t0
    nsol = sum(len(j[3]) for j in jobs)
    busy = sum((st if with_setup else 0.0) + sum(sv) for st, sv, _ in res)
    # Throughput of `cores` processes working through the sample: the work
    # each would do back to back, summed, over the busy time per core.
    return {"value": nsol / (busy / cores), "unit": "solves/s", "cores": cores, "kind": "reference",
            "sample": sample + f"; {nsol} solves, {busy:.1f} s of reference time "
                      f"({'set-up and ' if with_setup else ''}solves), {wall:.1f} s wall on {cores} processes",
            "cycles_min_max": [min(min(c) for _, _, c in res), max(max(c) for _, _, c in res)]}


def run_batch96(a):
    """Config 4: 96 independent problems, dims per axis from {33,65,129},
    sigma uniform in [0.5,2], mixed precision to 1e-10, one launch per level
    and colour across all problems, graph-captured steps."""
    import torch

    import pgmg_b200 as P
    rng = np.random.default_rng(a.seed)
    nprob = a.batch_problems
    shapes = [tuple(int(v) for v in rng.choice([33, 65, 129], 3)) for _ in range(nprob)]
    sigmas = rng.uniform(0.5, 2.0, nprob)
    hs = []
    gen_s = setup_s = 0.0
    for p, (shape, sg) in enumerate(zip(shapes, sigmas)):
        t0 = time.perf_counter()
        g = P.problem_gauss(*shape, seed=a.seed * 1000 + p, width=8.0)  # the cell field, on the host
        t1 = time.perf_counter()
        G = P.Multigrid(*shape, precision=P.MIXED)
        G.assemble_q1(g, from_log=True, sigma=float(sg))
        G.rhs_uniform(p)
        G.sync()
        gen_s += t1 - t0
        setup_s += time.perf_counter() - t1
        hs.append(G)
    B = P.Batch(nprob, P.MIXED)
    B.set_option(P.OPT_CHECK_EVERY, 0)  # the adaptive schedule, per problem
    for p, G in enumerate(hs):
        B.attach(p, G)
    for _ in range(a.warmup):
        cyc, rr = B.solve(a.tol, 100)
    l0 = B.launches
    t_b, (cyc, rr) = timed(B_stream := torch.cuda.current_stream(), lambda: B.solve(a.tol, 100), a.steps)
    launches = (B.launches - l0) // a.steps
    # wall clock agrees with the device here (the batch syncs each step); use it as well
    t0 = time.perf_counter()
    B.solve(a.tol, 100)
    wall = time.perf_counter() - t0
    t_batch = max(t_b, wall)
    # sequential: each problem alone, one after the other
    st = torch.cuda.Stream()
    for G in hs:
        G.set_stream(st.cuda_stream)

    def seq():
        for G in hs:
            G.clear_x(0)
            G.solve(a.tol, 100, 0)
    seq()
    t_seq, _ = timed(st, seq, 1)
    alg = sum(int(c) * ir_step_bytes(*s) for c, s in zip(cyc[:nprob], shapes))
    peak, kind = measured_peak_hbm()
    cpu = None
    if not a.no_cpu_baseline:
        # A bounded sample: the first problems of the batch up to about 3
        # million points per host process.
        budget, jobs, pts = 3e6 * max(1, min(os.cpu_count() or 1, 16)), [], 0
        for p, (shape, sg) in enumerate(zip(shapes, sigmas)):
            npt = shape[0] * shape[1] * shape[2]
            if jobs and pts + npt > budget:
                break
            jobs.append((shape, float(sg), a.seed * 1000 + p, [p], a.tol))
            pts += npt
        cpu = cpu_pool_baseline(jobs, False, f"the first {len(jobs)} of the {nprob} problems, solves only "
                                             "(set-up untimed, as in the batch)")
    print(json.dumps({
        "workload": f"{nprob} problems, dims per axis in {{33,65,129}}, mixed FP32/FP64 to 1e-10 (config 4)",
        "metric": "solves/s", "value": nprob / t_batch, "unit": "solves/s", "ms_per_batch": t_batch * 1e3,
        "sequential": {"value": nprob / t_seq, "unit": "solves/s", "ms": t_seq * 1e3},
        "speedup_vs_sequential": t_seq / t_batch, "max_relres": float(rr[:nprob].max()),
        "cycles_min_max": [int(cyc[:nprob].min()), int(cyc[:nprob].max())], "gpu_launches_per_batch": launches,
        "points_total": int(sum(x * y * z for x, y, z in shapes)), "setup_s_all": setup_s, "host_generation_s_all": gen_s,
        "roofline": {"bound": "hbm", "achieved": alg / t_batch / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / t_batch / 1e9 / peak, "peak_source": kind},
        "cpu_baseline": cpu,
    }))


def run_serve(a):
    """Config 5: open-loop Poisson arrivals, dims per axis 65..257 rounded to
    {65,129,257}, sigma in [0.5,2.3], 20% RHS-only reuse, 150 GB cap; solves/s
    and latency percentiles, next to the same requests served one at a time."""
    import torch

    import pgmg_b200 as P
    from pgmg_b200.server import FieldPool, SolveServer, poisson_requests
    reqs = poisson_requests(a.serve_rate, a.serve_seconds, seed=a.seed, reuse=0.2, sizes=(65, 129, 257),
                            sigma=(0.5, 2.3))
    fields = FieldPool(0)
    for r in reqs:  # the field pool is the requests' payload: generate it before the clock starts
        fields.get(r.shape, r.field)
    srv = SolveServer(150e9, max_slots=64, precision=P.MIXED, fields=fields)
    t0 = time.perf_counter()
    done = srv.run(reqs)
    wall = time.perf_counter() - t0
    lat = np.array([r.latency for r in done])
    span = max(r.finished for r in done) - min(r.arrival for r in done)
    out = {"workload": f"serving: Poisson {a.serve_rate:g} req/s for {a.serve_seconds:g} s, dims per axis "
                       "65..257 -> {65,129,257}, 20% RHS-only reuse, 150 GB cap, mixed to 1e-10 (config 5)",
           "metric": "solves/s", "value": len(done) / span, "unit": "solves/s", "requests": len(done),
           "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
           "reused": int(sum(r.reused for r in done)), "max_relres": float(max(r.relres for r in done)),
           "steps": srv.steps, "wall_s": wall}
    srv.close()
    del srv
    torch.cuda.empty_cache()
    # Latency at a load the server sustains: a second open-loop stream at a
    # fraction (default 70 %) of the saturated throughput just measured.
    # Sustained means the late requests wait no longer than the early ones
    # (the queue does not grow).
    if a.serve_sustained_seconds > 0:
        rate2 = a.serve_sustained_fraction * out["value"]
        reqs2 = poisson_requests(rate2, a.serve_sustained_seconds, seed=a.seed + 1, reuse=0.2, sizes=(65, 129, 257),
                                 sigma=(0.5, 2.3))
        for r in reqs2:
            fields.get(r.shape, r.field)
        srv = SolveServer(150e9, max_slots=64, precision=P.MIXED, fields=fields)
        done2 = sorted(srv.run(reqs2), key=lambda r: r.arrival)
        srv.close()
        del srv
        torch.cuda.empty_cache()
        lat2 = np.array([r.latency for r in done2])
        half = len(lat2) // 2
        span2 = max(r.finished for r in done2) - min(r.arrival for r in done2)
        out["sustained"] = {"rate_req_s": rate2, "requests": len(done2), "value": len(done2) / span2,
                            "unit": "solves/s", "p50_latency_s": float(np.percentile(lat2, 50)),
                            "p99_latency_s": float(np.percentile(lat2, 99)),
                            "p50_first_half_s": float(np.percentile(lat2[:half], 50)) if half else None,
                            "p50_second_half_s": float(np.percentile(lat2[half:], 50)) if half else None,
                            "max_relres": float(max(r.relres for r in done2))}
    # The same requests one at a time (set-up when not resident, then a
    # solve), in arrival order, for at most --serve-seq-seconds.
    cache = {}
    t0 = time.perf_counter()
    nseq = 0
    for r in reqs:
        if time.perf_counter() - t0 > a.serve_seq_seconds:
            break
        nseq += 1
        G = cache.get(r.problem)
        if G is None:
            G = P.Multigrid(*r.shape, precision=P.MIXED)
            G.assemble_q1(fields.get(r.shape, r.field).data_ptr(), from_log=True, sigma=r.sigma)
            cache[r.problem] = G
            total = sum(x.memory_bytes for x in cache.values())
            while total > 150e9 and len(cache) > 1:
                k = next(iter(cache))
                cache.pop(k).close()
                total = sum(x.memory_bytes for x in cache.values())
        G.rhs_uniform(r.rhs_seed)
        G.clear_x(0)
        G.solve(1e-10, 100, 0)
    seq = time.perf_counter() - t0
    out["sequential"] = {"value": nseq / seq, "unit": "solves/s", "s": seq,
                         "sample": f"the first {nseq} of the {len(reqs)} requests"}
    out["speedup_vs_sequential"] = out["value"] / out["sequential"]["value"]
    if not a.no_cpu_baseline:
        # A bounded sample of the requests in arrival order (about 4 million
        # points per host process); a problem's requests go to one process,
        # which sets it up once and solves each right-hand side.
        budget, groups, pts = 4e6 * max(1, min(os.cpu_count() or 1, 16)), {}, 0
        nreq = 0
        for r in reqs:
            npt = r.shape[0] * r.shape[1] * r.shape[2]
            if groups and pts + npt > budget:
                break
            m, n, o = r.shape
            fseed = 1000 + 7919 * r.field + 31 * m + 17 * n + o  # FieldPool's seed of that field
            groups.setdefault(r.problem, [r.shape, r.sigma, fseed, [], 1e-10])[3].append(r.rhs_seed)
            pts += npt
            nreq += 1
        out["cpu_baseline"] = cpu_pool_baseline([tuple(g) for g in groups.values()], True,
                                                f"the first {nreq} of the {len(reqs)} requests, set-up and solves")
    print(json.dumps(out))


def run_entrypoints(a):
    """Every drop-in entry point timed on its own (CUDA events, after one
    untimed call): on an FP64 problem of --size^3 with the cluster tail off,
    so that the per-level kernels down to the explicit-inverse coarse solve
    run; the field, stencil and PCG-helper accessors; the mixed set-up; a
    periodic 64^3 problem; a batch of four 33^3 problems; the no-alloc norms.
    Each kernel of the library is launched here at least once (for per-kernel
    profiles of those the benchmark solve does not launch)."""
    import torch

    import pgmg_b200 as P
    m, reps = a.size, max(1, a.steps)
    N = m ** 3
    st = torch.cuda.Stream()
    out = {}

    def t(name, fn, nbytes=None):
        fn()
        dt, _ = timed(st, fn, reps)
        out[name] = {"ms": round(dt * 1e3, 4)}
        if nbytes:
            out[name]["alg_GBs"] = round(nbytes / dt / 1e9, 1)

    g = P.problem_gauss(m, m, m, a.seed, 8.0)
    G = P.Multigrid(m, m, m)
    G.set_stream(st.cuda_stream)
    t0 = time.perf_counter()
    G.assemble_q1(g, from_log=True, sigma=a.sigma)
    G.sync()
    out["assemble_q1+build_rat (host clock, first call)"] = {"ms": round((time.perf_counter() - t0) * 1e3, 2)}
    G.rhs_uniform(a.seed)
    G.set_option(P.OPT_CLUSTER_SIZE, 0)
    dev = torch.randn(N, dtype=torch.float64, device="cuda")
    dev2 = torch.empty_like(dev)
    h = G.handle
    L = P.lib()
    t("set_field x (natural -> halo'd)", lambda: G.set_field(0, P.FIELD_X, dev.data_ptr()), 16 * N)
    t("get_field x", lambda: G.get_field(0, P.FIELD_X, dev2.data_ptr()), 16 * N)
    t("set_field r (natural -> colour-major)", lambda: G.set_field(0, P.FIELD_R, dev.data_ptr()), 16 * N)
    t("get_field r", lambda: G.get_field(0, P.FIELD_R, dev2.data_ptr()), 16 * N)
    t("apply (A x, device pointers)", lambda: L.pgmg_dev_apply(h, 0, dev.data_ptr(), dev2.data_ptr()), 240 * N)
    t("clear_x", lambda: G.clear_x(0), 8 * N)
    t("setup_test", lambda: G.setup_test(1, True, 0), 16 * N)
    t("copy_rhs_to_soln", lambda: G.copy_rhs_to_soln(0), 16 * N)
    t("l0_error", lambda: G.l0_error(0), 232 * N)
    t("source_soln_dot", lambda: G.source_soln_dot(0), 16 * N)
    t("norms", lambda: G.norms(0), 232 * N)
    t("gauss_seidel mc8 level 0 (one sweep)", lambda: G.gauss_seidel(0, 0, P.SMOOTH_MC8), 240 * N)
    t("gauss_seidel lex level 0 (one sweep)", lambda: G.gauss_seidel(0, 0, P.SMOOTH_LEX))
    t("restriction 0 -> 1", lambda: G.restriction(1))
    t("interpolation 1 -> 0", lambda: G.interpolation(1))
    t("solve_exact (explicit inverse)", lambda: G.solve_exact())
    t("v_cycle mc8, per-level kernels", lambda: G.v_cycle(0, P.SMOOTH_MC8))
    t("fmg_cycle mc8", lambda: G.fmg_cycle(P.SMOOTH_MC8))
    G.close()
    del g

    # Stencils uploaded from and read back to the host (natural 27-slot rows).
    ms = min(m, 65)
    coef, S = P.problem_q1(ms, ms, ms)
    H = P.Multigrid(ms, ms, ms)
    H.set_stream(st.cuda_stream)
    t(f"setup_matrices {ms}^3 (upload + build_rat)", lambda: H.setup_matrices(coef, S))
    t(f"get_coef level 0 {ms}^3", lambda: H.get_coef(0))
    H.close()

    # Mixed precision: FP32 copies of the stencils at set-up.
    gm = P.problem_gauss(m, m, m, a.seed, 8.0)
    Hm = P.Multigrid(m, m, m, precision=P.MIXED)
    Hm.set_stream(st.cuda_stream)
    t("assemble_q1+build_rat, mixed", lambda: Hm.assemble_q1(gm, from_log=True, sigma=a.sigma))
    Hm.close()
    del gm

    # Periodic 64^3: halo images and the periodic transfers.
    mp = 64
    Np = mp ** 3
    base = np.zeros(27)
    for s in range(27):
        nd = abs(s % 3 - 1) + abs((s // 3) % 3 - 1) + abs(s // 9 - 1)
        base[s] = (8.0 / 3.0 + 0.3, 0.0, -1.0 / 6.0, -1.0 / 12.0)[nd]
    Sp = np.tile(np.array([-1, 2, -1, 2, -1, 2], np.int32), (Np, 1))
    rp = np.random.default_rng(a.seed).uniform(-1, 1, Np)
    Hp = P.Multigrid(mp, mp, mp, prd=(True, True, True))
    Hp.set_stream(st.cuda_stream)
    Hp.setup_matrices(np.tile(base, (Np, 1)), Sp)
    Hp.setup_fields(rp)
    t("v_cycle periodic 64^3", lambda: Hp.v_cycle(0))
    Hp.close()

    # A batch of four 33^3 problems, mixed precision.
    hs = []
    for p in range(4):
        Gb = P.Multigrid(33, 33, 33, precision=P.MIXED)
        Gb.assemble_q1(P.problem_gauss(33, 33, 33, a.seed + p, 8.0), from_log=True, sigma=1.0)
        Gb.rhs_uniform(p)
        hs.append(Gb)
    B = P.Batch(4, P.MIXED)
    for p, Gb in enumerate(hs):
        B.attach(p, Gb)
    t("batch of 4 x 33^3, mixed, to 1e-10", lambda: B.solve(a.tol, 100))

    def stepwise():
        for p in range(4):
            B.begin(p)
        while B.step(a.tol, 100) > 0:
            pass
    t("the same batch by begin + step (continuous batching)", stepwise)
    B.close()
    for Gb in hs:
        Gb.close()

    # No-alloc norms on caller-owned arrays (65^3).
    mn = 65
    cn, _ = P.problem_q1(mn, mn, mn)
    dc = torch.from_numpy(np.ascontiguousarray(cn)).cuda()
    dx = torch.randn(mn ** 3, dtype=torch.float64, device="cuda")
    dr = torch.randn(mn ** 3, dtype=torch.float64, device="cuda")
    o2 = torch.zeros(2, dtype=torch.float64, device="cuda")
    t(f"residual_norms_noalloc {mn}^3",
      lambda: P.residual_norms_noalloc(mn, mn, mn, dc.data_ptr(), dx.data_ptr(), dr.data_ptr(), o2.data_ptr(),
                                       st.cuda_stream), 232 * mn ** 3)
    print(json.dumps({"workload": f"drop-in entry points one by one, {m}^3 FP64 (others as named)",
                      "unit": "ms per call", "reps": reps, "entry_points": out}))


def run_profile_mixed(a):
    import torch

    import pgmg_b200 as P
    m = a.size
    coef, S, r = build_problem(m, a.sigma, a.seed)
    st = torch.cuda.Stream()
    G = P.Multigrid(m, m, m, precision=P.MIXED)
    G.set_stream(st.cuda_stream)
    G.setup_matrices(coef, S)
    G.setup_fields(r)
    del coef, S
    G.autotune(cache=a.tune_cache)  # the options the benchmark's mixed leg runs with

    def solve():
        G.clear_x(0)
        return G.solve(a.tol, 100, 0)
    for _ in range(a.warmup):
        solve()
    t, (cyc, rr) = timed(st, solve, a.steps)
    print(json.dumps({"workload": "mixed only", "value": t, "cycles": cyc, "relres": rr}))


def results_only_on_stdout():
    """Keep the process's standard output for the JSON result lines: file
    descriptor 1 is pointed at standard error, so that what native code
    prints with printf (the reference prints its grid hierarchy and its LU
    fallback notice) goes there, and Python's sys.stdout writes to the
    original standard output."""
    sys.stdout.flush()
    keep = os.dup(1)
    os.dup2(2, 1)
    sys.stdout = os.fdopen(keep, "w", buffering=1)


def main():
    a = parse()
    results_only_on_stdout()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "small65":
        run_small65(a)
    elif a.workload == "large513":
        run_large513(a)
    elif a.workload == "batch96":
        run_batch96(a)
    elif a.workload == "serve":
        run_serve(a)
    elif a.workload == "entrypoints":
        run_entrypoints(a)
    elif a.profile_mixed:
        run_profile_mixed(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
