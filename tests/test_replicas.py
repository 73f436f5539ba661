"""The multi-rank path of bench.py (one replica per rank, no data exchange):
rank discovery, barrier and max-over-ranks timing, exercised with two CPU
ranks over gloo."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from dedisp_tests_b200.replicas import Replicas
    r = Replicas.from_env("gloo", timeout_s=60)
    r.barrier()
    t = r.max_over_ranks(1.5 + rank)          # each replica's own time
    units = 1000 * r.world                    # whole-job units: every rank's work
    q.put((r.rank, r.world, t, units / t))
    r.close()


def test_two_replicas_take_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(i, world, port, q)) for i in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == 2 and r[2] == 2.5 for r in res)  # max over ranks
    assert all(abs(r[3] - 2000 / 2.5) < 1e-9 for r in res)


def test_single_process_defaults(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from dedisp_tests_b200.replicas import Replicas
    r = Replicas.from_env("gloo")
    assert (r.world, r.rank, r.local) == (1, 0, 0)
    r.barrier()
    assert r.max_over_ranks(3.0) == 3.0
    r.close()
