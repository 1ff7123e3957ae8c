"""The multi-process (replica) path of bench.py on CPU: two gloo ranks, as torchrun starts them.

Each rank reports a different device time; both must see the maximum, and the whole-job
throughput is world size × solves per rank / that maximum.
"""

from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from bwpm_b200 import replicas

    dist, r, ws, local = replicas.init("gloo", timeout_s=60)
    try:
        replicas.barrier(dist)
        m = replicas.max_over_ranks(dist, 100.0 + 50.0 * r)  # rank 1 is the slower one
        out.put((r, ws, local, m, replicas.throughput(ws, 256, m)))
        replicas.barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time_and_throughput():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    for r, ws, local, m, thr in got:
        assert ws == 2 and local == r
        assert m == 150.0
        assert thr == pytest.approx(2 * 256 / 0.150)


def test_one_process_needs_no_group():
    from bwpm_b200 import replicas

    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK") if k in os.environ}
    try:
        dist, rank, ws, local = replicas.init("gloo")
        assert dist is None and (rank, ws, local) == (0, 1, 0)
        assert replicas.max_over_ranks(None, 3.5) == 3.5
        assert replicas.throughput(1, 10, 1000.0) == pytest.approx(10.0)
    finally:
        os.environ.update(env)
