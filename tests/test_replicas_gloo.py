"""Replica mode over two ranks on the CPU (gloo): the process group, barrier,
max over ranks and whole-job rate that bench.py uses for --gpus N (one
independent grid per GPU, no data-path collective), and a rank that never
joins turning into an error on the other instead of a hang."""
import os
import socket
import time

import pytest
import torch.multiprocessing as mp

from gpluto_dev_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))


def _replica(rank, world, port, q):
    _env(rank, world, port)
    r = replicas.init("gloo", timeout_s=60)
    t_ms = 10.0 + 5.0 * rank              # this rank's timed region
    r.barrier()
    tmax = r.max_over_ranks(t_ms)
    q.put((rank, tmax, replicas.replica_seed(1, r.rank), replicas.replica_seed(0, r.rank, 512),
           replicas.whole_job_rate(r.world, 1000, 4, tmax)))
    r.close()


def _lonely(rank, world, port, q):
    _env(rank, world, port)
    if rank == 1:                          # never joins, never crashes
        time.sleep(8)
        return
    t0 = time.time()
    try:
        replicas.init("gloo", timeout_s=3)
        q.put(("joined", time.time() - t0))
    except Exception as e:                 # the short timeout ends the wait
        q.put(("error", time.time() - t0, type(e).__name__))


def _run(target, world=2, timeout=120):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    return ps, q


def test_two_replicas_are_timed_by_the_slowest_rank():
    ps, q = _run(_replica)
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]                 # max over ranks
    assert res[0][2] != res[1][2] and res[0][3] != res[1][3]    # different grids
    assert res[0][4] == pytest.approx(2 * 1000 * 4 / 15e-3 / 1e6)


def test_a_rank_that_never_joins_times_out_instead_of_hanging():
    ps, q = _run(_lonely)
    out = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert out[0] == "error", out
    assert out[1] < 8.0


def test_one_rank_needs_no_process_group(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "1")
    monkeypatch.setenv("RANK", "0")
    r = replicas.init("gloo")
    assert r.dist is None and r.max_over_ranks(3.5) == 3.5
    r.barrier()
    r.close()
