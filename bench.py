#!/usr/bin/env python
"""Benchmark: seconds to a 1e-10 relative residual on a 257^3
variable-coefficient 27-point Q1 problem (kappa = exp(sigma*g), sigma = 1.0,
Gaussian-smoothed seeded field of width 8 cells), FP64 on one B200.

One step = one solve from x = 0: V-cycles (2+l pre/post sweeps on level l,
8-colour Gauss-Seidel, FP64 LU on the coarsest level) with a residual check
after every cycle, until sqrt(sum r^2 / sum b^2) < 1e-10.

  python bench.py [--gpus N --steps K --warmup W]          this library
  python bench.py --impl reference [--steps K --warmup W]  the reference's own
                                                           CPU multigrid

Prints one JSON line (rank 0).  ``value`` is the device-timed s/solve with
the operator and source resident in device memory (inputs > L2, so no flush
is needed); ``e2e`` times the same solve through the C ABI from pinned host
buffers (source up, solution down) every step.  Under torchrun every rank
solves its own replica (independent problems; no collective on the data
path) and the line reports the max over ranks.
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

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
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
            for line in fh:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9 and p[1].replace(".", "").isdigit():
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


def run_reference(a):
    """--impl reference: the reference's own CPU multigrid (compiled from its
    sources into oracle/_ref with a single-rank MPI shim), each step a full
    solve from x = 0 on the same 257^3 problem."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.pyoracle import Reference, ref_available
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpgmg_ref.so not built"}))
        return
    m = a.size
    coef, S, r = build_problem(m, a.sigma, a.seed)
    t0 = time.perf_counter()
    R = Reference(m, m, m, S, coef, r)
    setup_s = time.perf_counter() - t0
    del coef, S
    times, cycles = [], None
    for it in range(a.warmup + a.steps):
        R.set_x(0, np.zeros(m * m * m))
        t0 = time.perf_counter()
        n, rr = reference_cycles(R, a.tol)
        dt = time.perf_counter() - t0
        if it >= a.warmup:
            times.append(dt)
        cycles = n
    v = float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded kappa field and RHS)",
        "config": {"workload": f"{m}^3 Q1 variable-kappa sigma={a.sigma}, solve to {a.tol} rel residual",
                   "cycles": cycles, "lu_enabled": R.lu_enabled, "setup_s": setup_s},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"{a.steps} full solves (V-cycles + residual check per cycle) on one core; "
                                   "the reference has no threading and no MPI here"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- ours

def run_ours(a):
    import torch
    import torch.distributed as dist

    import pgmg_b200 as P

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    m = a.size
    npts = m ** 3
    tg = time.perf_counter()
    coef, S, r = build_problem(m, a.sigma, a.seed + rank)
    gen_s = time.perf_counter() - tg

    stream = torch.cuda.Stream(device=dev)
    G = P.Multigrid(m, m, m, precision=P.FP64, coarse=P.COARSE_LU, smoother=P.SMOOTH_MC8, device=local)
    G.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    G.setup_matrices(coef, S)
    G.sync()
    setup_s = time.perf_counter() - t0
    G.setup_fields(r)

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
    launches = (G.launches - launches0) // a.steps
    clocks = clk.summary()
    ms = max_over_ranks(ms)
    final_relres = rr

    # --- end to end through the C ABI with pinned host buffers -------------
    hr = torch.from_numpy(r).pin_memory()
    hx = torch.empty(npts, dtype=torch.float64).pin_memory()
    for _ in range(1):
        G.set_field(0, P.FIELD_R, hr.data_ptr())
        solve_once(G)
        G.get_field(0, P.FIELD_X, hx.data_ptr())
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        G.set_field(0, P.FIELD_R, hr.data_ptr())
        G.clear_x(0)
        G.solve(a.tol, 100, 0)
        G.get_field(0, P.FIELD_X, hx.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / a.steps)

    # --- roofline of the dominant kernel: level-0 8-colour sweep ----------
    nsw = 8
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    G.clear_x(0)
    G.gauss_seidel(0, 0, P.SMOOTH_MC8)
    torch.cuda.synchronize()
    k0.record(stream)
    for _ in range(nsw):
        G.gauss_seidel(0, 0, P.SMOOTH_MC8)
    k1.record(stream)
    torch.cuda.synchronize()
    launch_ms = k0.elapsed_time(k1) / (8 * nsw)
    alg_bytes = BYTES_GS_PER_POINT[8] * npts / 8  # one colour = N/8 point updates
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic = profiled_traffic("gs_colour_fp64_257.md")

    # --- mixed precision alongside ----------------------------------------
    mixed = None
    if not a.no_mixed:
        Gm = P.Multigrid(m, m, m, precision=P.MIXED, coarse=P.COARSE_LU, smoother=P.SMOOTH_MC8, device=local)
        Gm.set_stream(stream.cuda_stream)
        Gm.setup_matrices(coef, S)
        Gm.setup_fields(r)
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
        mixed = {"value": mms / 1e3, "unit": UNIT, "cycles": mc, "relres": mr,
                 "speedup_vs_fp64": ms / mms,
                 "max_rel_diff_vs_fp64_solution": float(np.abs(xm - xd).max() / np.abs(xd).max())}
        Gm.close()

    # --- CPU baseline: the reference itself, bounded sample ---------------
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a, coef, S, r, G)

    if rank == 0:
        line = {
            "metric": METRIC, "value": ms / 1e3, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded kappa field and RHS)",
            "config": {"workload": f"{m}^3 Q1 variable-kappa sigma={a.sigma} FP64, solve to {a.tol} rel residual",
                       "levels": G.nlevels, "cycles": cyc_list[-1], "final_relres": final_relres,
                       "smoother": "8-colour Gauss-Seidel", "coarse": "FP64 LU (explicit inverse)",
                       "l2": "inputs larger than L2 (3.7 GB stencils)", "setup_s": setup_s,
                       "host_generation_s": gen_s, "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_ms / 1e3, "unit": UNIT, "h2d_bytes_per_step": npts * 8,
                    "d2h_bytes_per_step": npts * 8},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": "k_gs_colour<double> level 0",
                         "peak_source": peak_kind, "launch_ms": launch_ms},
            "gpu_launches": launches,
            "clocks": clocks,
            "mixed": mixed,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    G.close()
    if world > 1:
        dist.destroy_process_group()


def cpu_baseline(a, coef, S, r, G):
    """The reference (oracle/_ref) on one host core: its set-up and two
    V-cycles at the full size, scaled to a solve by the reference's own cycle
    count (which the GPU's lexicographic mode reproduces bit for bit)."""
    from oracle.pyoracle import Reference, ref_available
    if not ref_available():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": "oracle/_ref not built"}
    import pgmg_b200 as P
    m = a.size
    t0 = time.perf_counter()
    R = Reference(m, m, m, S, coef, r)
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    R.l2_error_all()
    R.v_cycle(0)
    R.v_cycle(0)
    R.l2_error_all()
    per_cycle = (time.perf_counter() - t0) / 2
    # The reference's cycle count: the GPU lexicographic mode with the same
    # coarse solver reproduces the reference's iterates exactly.
    lu = R.lu_enabled
    R.close()
    L = P.Multigrid(m, m, m, coarse=P.COARSE_LU_EXACT if lu else P.COARSE_GS, smoother=P.SMOOTH_LEX)
    L.setup_matrices(coef, S)
    L.setup_fields(r)
    n_ref, rr = L.solve(a.tol, 100, 1)
    L.close()
    return {"value": per_cycle * n_ref, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"reference set-up ({setup_s:.1f} s, untimed) + 2 V-cycles with residual checks "
                      f"({per_cycle:.2f} s/cycle) x {n_ref} cycles to {a.tol} (the reference's count, "
                      f"lu_enabled={lu})"}


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
