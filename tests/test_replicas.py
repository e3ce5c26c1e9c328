"""Replica harness on CPU: two gloo ranks, as torchrun would start them.

The multi-GPU path is replicas only (independent systems, batch matrices or
requests per rank, nothing exchanged on the data path); these tests run its
host side -- process group, barrier, max-over-ranks timing, sharding of
independent units -- with world size 2 on the gloo backend.
"""
import os
import socket

import pytest

from snusolver_b200 import replicas


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    w, r, _ = replicas.init(backend="gloo", timeout_s=60)
    replicas.barrier(w)
    # each rank reports its own step time; the job's time is the slowest
    t = replicas.max_over_ranks(w, 0.25 + 0.5 * r)
    mine = replicas.shard(list(range(10)), w, r)
    replicas.barrier(w)
    replicas.finish(w)
    out.put((r, w, t, mine))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[1] for x in res] == [2, 2]
    assert all(x[2] == pytest.approx(0.75) for x in res)
    a, b = res[0][3], res[1][3]
    assert sorted(a + b) == list(range(10)) and not set(a) & set(b)


def test_single_rank_needs_no_group():
    ws, rank, _ = replicas.init(backend="gloo")
    assert (ws, rank) == (1, 0)
    assert replicas.max_over_ranks(ws, 1.5) == 1.5
    assert replicas.shard([1, 2, 3], 1, 0) == [1, 2, 3]
