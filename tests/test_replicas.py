"""Multi-process plumbing of multi-GPU runs (pgmg_b200.replicas), on CPU with
the gloo backend and two ranks: one independent problem per rank, barriers,
the max over ranks of a timing, and the job's aggregate time per solve."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from pgmg_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    rep.barrier()
    t = 1.0 + rank  # a rank's device time
    tmax = rep.max(t)
    out.put((rank, rep.seed(7), tmax, rep.per_solve(tmax), rep.is_root))
    rep.barrier()
    rep.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_replicas_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    world = 2
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [7, 8]            # one problem per rank
    assert all(r[2] == 2.0 for r in res)             # max over ranks, on every rank
    assert all(r[3] == 1.0 for r in res)             # 2 solves within the max time
    assert [r[4] for r in res] == [True, False]      # rank 0 reports


def test_single_process_needs_no_launcher(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from pgmg_b200.replicas import Replicas
    rep = Replicas("gloo")
    assert rep.world == 1 and rep.max(3.5) == 3.5 and rep.per_solve(2.0) == 2.0 and rep.seed(4) == 4
    rep.barrier()
    rep.close()
