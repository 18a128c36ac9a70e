"""Replica helpers across 2 processes (gloo, CPU): the max over ranks, the
barrier, and round-robin sharding of independent scans -- what bench.py --gpus N
uses (one process per GPU, no data-path collective)."""

from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp

from aprict_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    replicas.init("gloo", timeout_s=60)
    replicas.barrier()
    m = replicas.max_over_ranks(1.5 + rank)
    mine = replicas.shard(list(range(7)))
    replicas.barrier()
    replicas.finish()
    out.put((rank, m, mine))


def test_two_gloo_ranks() -> None:
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.5, 2.5]
    assert res[0][2] == [0, 2, 4, 6] and res[1][2] == [1, 3, 5]


def test_single_process_is_a_no_op() -> None:
    assert replicas.max_over_ranks(3.0) == 3.0
    replicas.barrier()
    assert replicas.shard([1, 2, 3], rank=0, world=1) == [1, 2, 3]
