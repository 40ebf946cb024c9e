"""Continuous-batching solve server on one GPU.

Requests (grid size, coefficient field, right-hand side) arrive over time.
The server:

* admits a request when a batch slot is free and its hierarchy fits the
  device-memory cap (one pool allocation, first-fit sub-allocation; idle
  resident hierarchies are evicted least recently used first);
* builds a fresh problem on a set-up thread, on the problem's own CUDA
  stream: Q1 stencils assembled on the device from the request's cell field,
  Galerkin hierarchy, coarse LU, source;
* keeps every hierarchy resident after its solve, so that a later request for
  the same problem with a new source skips the set-up;
* steps all running problems together with ``Batch.step`` -- one refinement
  step (FP64 residual and convergence check, FP32 V-cycle, FP64 update in
  mixed precision) per problem per step, every launch covering every running
  problem -- and lets problems join and leave between steps.

A problem's iterates do not depend on what else runs with it (the batched
kernels share the single-problem device code), so each result is the same
alone and in the mix.

Synthetic requests name their coefficient field as (shape, field id, sigma):
kappa = exp(sigma * g) with g a smoothed Gaussian field from a pool that is
generated once on the host and kept on the device, and their source by a seed
(generated on the device).
"""
from __future__ import annotations

import collections
import dataclasses
import queue
import threading
import time

import numpy as np

from . import (MIXED, OPT_CHECK_EVERY, Batch, Multigrid, PgmgError, plan_bytes, problem_gauss)


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float                 # seconds after the start of the run
    shape: tuple                   # (m, n, o)
    field: int                     # id of the g field of this shape
    sigma: float
    rhs_seed: int
    problem: int                   # problem id; equal ids = same operator (RHS-only reuse)
    # filled by the server
    admitted: float = -1.0
    started: float = -1.0
    finished: float = -1.0
    cycles: int = -1
    relres: float = float("nan")
    reused: bool = False
    x: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class DevicePool:
    """One device allocation, first-fit sub-allocation (256-byte aligned)."""

    def __init__(self, nbytes: int, device: int):
        import torch
        self.buf = torch.empty(nbytes + 256, dtype=torch.uint8, device=f"cuda:{device}")
        self.base = (self.buf.data_ptr() + 255) // 256 * 256
        self.size = nbytes
        self.free = [(0, nbytes)]  # sorted (offset, length)

    def alloc(self, n: int):
        n = (n + 255) // 256 * 256
        for i, (off, ln) in enumerate(self.free):
            if ln >= n:
                if ln == n:
                    self.free.pop(i)
                else:
                    self.free[i] = (off + n, ln - n)
                return off, n
        return None

    def release(self, off: int, n: int):
        self.free.append((off, n))
        self.free.sort()
        merged = []
        for o, ln in self.free:
            if merged and merged[-1][0] + merged[-1][1] == o:
                merged[-1] = (merged[-1][0], merged[-1][1] + ln)
            else:
                merged.append((o, ln))
        self.free = merged

    @property
    def free_bytes(self) -> int:
        return sum(ln for _, ln in self.free)


class FieldPool:
    """Smoothed Gaussian cell fields g per (shape, id), generated on the host
    once and kept on the device."""

    def __init__(self, device: int, width: float = 8.0):
        self.device = device
        self.width = width
        self.fields = {}
        self.lock = threading.Lock()
        self.stream = None

    def get(self, shape, fid: int):
        key = (tuple(shape), fid)
        with self.lock:
            if key not in self.fields:
                import torch
                m, n, o = shape
                g = problem_gauss(m, n, o, 1000 + 7919 * fid + 31 * m + 17 * n + o, self.width)
                # Uploaded on a stream of its own and waited for on that
                # stream only: a device-wide synchronisation from this thread
                # would break a CUDA-graph capture the serving loop may have
                # in progress on another stream.
                if self.stream is None:
                    self.stream = torch.cuda.Stream(self.device)
                with torch.cuda.stream(self.stream):
                    t = torch.from_numpy(g).to(f"cuda:{self.device}")
                self.stream.synchronize()
                self.fields[key] = t
            return self.fields[key]


class _Resident:
    def __init__(self, pid, mg, off, nbytes):
        self.pid = pid
        self.mg = mg
        self.off = off
        self.nbytes = nbytes
        self.busy = True  # built for a request that is about to start
        self.slot = -1
        self.last_used = 0.0


class SolveServer:
    def __init__(self, cap_bytes: float, max_slots: int = 64, precision: int = MIXED, tol: float = 1e-10,
                 max_cycles: int = 100, device: int = 0, keep_solutions: bool = False, fields: FieldPool | None = None,
                 setup_threads: int = 4, check_every: int = 0):
        self.cap = int(cap_bytes)
        self.max_slots = max_slots
        self.precision = precision
        self.tol = tol
        self.max_cycles = max_cycles
        self.device = device
        self.keep = keep_solutions
        # Set-up threads: each builds one problem at a time on that problem's
        # own stream, so the set-up kernels of several problems (the coarse LU
        # is one thread block) overlap each other and the batch steps.
        self.setup_threads = max(1, int(setup_threads))
        self.pool = DevicePool(self.cap, device)
        self.fields = fields or FieldPool(device)
        self.batch = Batch(max_slots, precision, device)
        # Residual checks per problem: 0 = the adaptive schedule (several
        # FP32 V-cycles per refinement step), 1 = every cycle.
        self.batch.set_option(OPT_CHECK_EVERY, check_every)
        self.resident = collections.OrderedDict()  # pid -> _Resident (LRU order)
        self.free_slots = list(range(max_slots))
        self.running = {}  # slot -> (request, resident)
        self.steps = 0
        self.lock = threading.Lock()  # pool and resident table (set-up thread + loop)
        # Where the time goes: seconds in set-up (set-up thread), in batch
        # steps and polls (loop), and the number of set-ups and evictions.
        self.stats = {"setup_s": 0.0, "setups": 0, "step_s": 0.0, "poll_s": 0.0, "start_s": 0.0,
                      "evictions": 0, "idle_s": 0.0}

    # -- resident hierarchies --------------------------------------------------
    def _evict_for(self, nbytes: int):
        with self.lock:
            return self._evict_locked(nbytes)

    def _evict_locked(self, nbytes: int):
        while True:
            got = self.pool.alloc(nbytes)
            if got is not None:
                return got
            victim = None
            for pid, r in self.resident.items():
                if not r.busy:
                    victim = pid
                    break
            if victim is None:
                return None
            r = self.resident.pop(victim)
            r.mg.close()
            self.pool.release(r.off, r.nbytes)
            self.stats["evictions"] += 1

    def _build(self, req: Request, now: float):
        m, n, o = req.shape
        nbytes = plan_bytes(m, n, o, self.precision)
        if nbytes > self.cap:
            raise PgmgError(10, "admission", f"problem of {nbytes} bytes exceeds the {self.cap}-byte cap")
        got = self._evict_for(nbytes)
        if got is None:
            return None
        off, nb = got
        mg = Multigrid(m, n, o, precision=self.precision, device=self.device, mem=(self.pool.base + off, nb))
        g = self.fields.get(req.shape, req.field)
        mg.assemble_q1(g.data_ptr(), from_log=True, sigma=req.sigma, build=True)
        r = _Resident(req.problem, mg, off, nb)
        return r

    # -- the loop ---------------------------------------------------------------
    def run(self, requests):
        """Serves `requests` (sorted by arrival) in real time, open loop.
        Returns the list with admission/finish times and results filled."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()       # arrived, not admitted
        ready = queue.Queue()               # (req, resident) built by the set-up thread
        todo = queue.Queue()                # requests for the set-up thread
        building = set()                    # pids being built
        done = []
        stop = threading.Event()
        t0 = time.perf_counter()
        err = []

        def setup_worker():
            while not stop.is_set():
                try:
                    req = todo.get(timeout=0.01)
                except queue.Empty:
                    continue
                try:
                    ts = time.perf_counter()
                    r = self._build(req, ts - t0)
                    with self.lock:
                        self.stats["setup_s"] += time.perf_counter() - ts
                        self.stats["setups"] += 1
                    ready.put((req, r))
                except Exception as e:  # noqa: BLE001 -- reported to the caller
                    err.append(e)
                    ready.put((req, None))

        workers = [threading.Thread(target=setup_worker, daemon=True) for _ in range(self.setup_threads)]
        for w in workers:
            w.start()
        max_in_setup = 2 * self.setup_threads
        in_setup = 0
        total = len(pending)
        try:
            while len(done) < total:
                now = time.perf_counter() - t0
                while pending and pending[0].arrival <= now:
                    waiting.append(pending.popleft())
                # Admission: reuse a resident idle hierarchy, or hand a fresh
                # one to the set-up thread.
                keep = collections.deque()
                while waiting:
                    req = waiting.popleft()
                    with self.lock:
                        # Claim an idle resident hierarchy before a set-up
                        # thread can pick it for eviction.
                        res = self.resident.get(req.problem)
                        reuse = res is not None and not res.busy and bool(self.free_slots)
                        if reuse:
                            res.busy = True
                    if reuse:
                        self._start(req, res, reused=True, now=now)
                    elif res is None and req.problem not in building and in_setup < max_in_setup and \
                            len(self.free_slots) > in_setup:
                        building.add(req.problem)
                        in_setup += 1
                        req.admitted = now
                        todo.put(req)
                    else:
                        keep.append(req)
                waiting = keep
                while True:
                    try:
                        req, res = ready.get_nowait()
                    except queue.Empty:
                        break
                    in_setup -= 1
                    building.discard(req.problem)
                    if err:
                        raise err[0]
                    if res is None:  # no memory now: retry later
                        req.admitted = -1.0
                        waiting.appendleft(req)
                        continue
                    with self.lock:
                        self.resident[res.pid] = res
                    self._start(req, res, reused=False, now=time.perf_counter() - t0)
                if self.running:
                    ts = time.perf_counter()
                    self.batch.step(self.tol, self.max_cycles)
                    self.steps += 1
                    tp = time.perf_counter()
                    act, cyc, rr = self.batch.poll()
                    now = time.perf_counter() - t0
                    self.stats["step_s"] += tp - ts
                    self.stats["poll_s"] += now + t0 - tp
                    for slot in [s for s in self.running if not act[s]]:
                        req, res = self.running.pop(slot)
                        req.finished = now
                        req.cycles = int(cyc[slot])
                        req.relres = float(rr[slot])
                        if self.keep:
                            req.x = res.mg.get_x(0)
                        self.batch.detach(slot)
                        self.free_slots.append(slot)
                        with self.lock:
                            res.busy = False
                            res.slot = -1
                            res.last_used = now
                            self.resident.move_to_end(res.pid)
                        done.append(req)
                else:
                    nxt = pending[0].arrival - (time.perf_counter() - t0) if pending else 0.0
                    ts = time.perf_counter()
                    time.sleep(min(max(nxt, 0.0), 0.002))
                    self.stats["idle_s"] += time.perf_counter() - ts
        finally:
            stop.set()
            for w in workers:
                w.join(timeout=5)
        return done

    def _start(self, req: Request, res: _Resident, reused: bool, now: float):
        ts = time.perf_counter()
        slot = self.free_slots.pop()
        with self.lock:
            res.busy = True
        res.slot = slot
        req.reused = reused
        if req.admitted < 0:
            req.admitted = now
        req.started = now
        res.mg.rhs_uniform(req.rhs_seed)
        self.batch.attach(slot, res.mg)
        self.batch.begin(slot)
        self.running[slot] = (req, res)
        self.stats["start_s"] += time.perf_counter() - ts

    def close(self):
        for r in self.resident.values():
            r.mg.close()
        self.resident.clear()
        self.batch.close()


def poisson_requests(rate: float, duration: float, seed: int = 0, reuse: float = 0.2, sizes=(65, 129, 257),
                     sigma=(0.5, 2.3), fields_per_shape: int = 2):
    """Open-loop Poisson arrivals; dims per axis drawn uniformly from
    [sizes[0], sizes[-1]] and rounded to the nearest listed size; a fraction
    `reuse` of requests re-solve an earlier problem with a new source."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    problems = []  # (shape, field, sigma)
    lo, hi = sizes[0], sizes[-1]
    arr = np.asarray(sizes)
    rid = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        if problems and rng.random() < reuse:
            pid = int(rng.integers(len(problems)))
            shape, field, sg = problems[pid]
        else:
            dims = rng.uniform(lo, hi, 3)
            shape = tuple(int(arr[np.abs(arr - d).argmin()]) for d in dims)
            field = int(rng.integers(fields_per_shape))
            sg = float(rng.uniform(*sigma))
            problems.append((shape, field, sg))
            pid = len(problems) - 1
        out.append(Request(rid=rid, arrival=t, shape=shape, field=field, sigma=sg,
                           rhs_seed=int(rng.integers(1 << 62)), problem=pid))
        rid += 1
    return out
