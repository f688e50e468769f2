"""Replica timing over two gloo ranks on the CPU: the max over ranks and the
whole-job rate that bench.py reports for --gpus N (no GPU needed)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, ws, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    from yafel_b200.replicas import Replicas
    r = Replicas("gloo", timeout_s=60)
    r.barrier()
    step = 0.5 + rank  # rank 1 is the slow one
    m = r.max(step)
    q.put((rank, r.ws, m, r.job_rate(1000, m)))
    r.close()


def test_two_gloo_ranks_take_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ws, m, rate in res:
        assert ws == 2 and m == 1.5
        assert rate == pytest.approx(2 * 1000 / 1.5)


def test_single_process_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from yafel_b200.replicas import Replicas
    r = Replicas("gloo")
    assert r.ws == 1 and r.max(2.5) == 2.5 and r.job_rate(10, 2.0) == 5.0
    r.close()
