"""Separator-tree distribution (snusolver_b200.dist) on CPU ranks.

World-size 2 and 4 gloo process groups run the distributed driver with the
host restatement of the front numerics (tests/host_engine.py) in place of
the CUDA engine: the partition into subtrees and shared fronts, the
exchanges (the shared fronts after phase 1, their solve work vectors, X)
and the phases are the product's.  Checks: the shared fronts summed over
the ranks equal the single-process assembly of the same fronts (the
reference's reduced Schur complements, kernel_sparse.cu:54-90), and every
rank's solution equals the C restatement of the reference's numerics.
"""
import os
import socket

import multiprocessing as mp
import numpy as np
import pytest

from snusolver_b200 import generators
from snusolver_b200.dist import subtree_owner


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _matrix():
    rng = np.random.default_rng(17)
    nx, ny = 26, 23
    rp, ci, v = generators.laplace2d_perturbed(nx, ny, seed=5)
    n = nx * ny
    rows = list(np.repeat(np.arange(n), np.diff(rp)))
    cols, vals = list(ci), list(v)
    seen = set(zip(rows, cols))
    for _ in range(60):  # structurally unsymmetric extras
        r = int(rng.integers(n))
        c = int(min(n - 1, r + int(rng.integers(2, 4))))
        if (r, c) not in seen:
            seen.add((r, c))
            rows.append(r), cols.append(c), vals.append(0.3 * float(rng.normal()))
    rows, cols, vals = np.array(rows), np.array(cols), np.array(vals)
    o = np.lexsort((cols, rows))
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, rows + 1, 1)
    b = rng.uniform(-1, 1, (n, 3))
    return (np.cumsum(rowptr).astype(np.int32), cols[o].astype(np.int32),
            vals[o], b)


def _rank_main(rank, world, nleaves, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import torch.distributed as dist
    from host_engine import HostEngine
    from snusolver_b200.dist import DistSolver
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world)
        rp, ci, v, b = _matrix()
        eng = HostEngine(rank, world, nleaves=nleaves)
        ds = DistSolver(rank, world, nleaves=nleaves, engine=eng)
        ds.construct(rp, ci, v)
        # factorize, keeping the summed shared fronts for the check
        eng.factor_phase(1)
        buf = eng.buffer(0)
        eng.copy(0, 0, 0, buf)
        ds._allreduce(buf)
        summed = buf.copy()
        eng.copy(0, 1, 0, buf)
        eng.factor_phase(2)
        x = ds.solve(b)
        q.put((rank, summed, x, ds.stats, int(eng.own.sum()), None))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        q.put((rank, None, None, None, 0, repr(e)))


@pytest.mark.parametrize("world,nleaves", [(2, 4), (4, 8)])
def test_distributed_factor_and_solve(world, nleaves):
    from host_engine import HostEngine
    from util import oracle_solve, free_blocks
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, nleaves, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    res.sort(key=lambda t: t[0])
    for r in res:
        assert r[5] is None, r[5]
    rp, ci, v, b = _matrix()
    # every front belongs to exactly one rank or to the shared top
    ref = HostEngine(None, world, nleaves=nleaves)
    ref.construct(rp, ci, v)
    owners = [subtree_owner(int(blk), world) for blk in ref.fp["block"]]
    counts = [sum(1 for o in owners if o == r) for r in range(world)]
    assert counts == [r[4] for r in res]
    assert sum(counts) + sum(1 for o in owners if o < 0) == len(owners)
    assert any(o < 0 for o in owners)
    # the shared fronts summed over the ranks = the single-process assembly
    # of the same fronts after every subtree's updates
    ref.factor_phase(1)
    want = ref.buffer(0)
    ref.copy(0, 0, 0, want)
    for r in res:
        err = np.abs(r[1] - want).max() / np.abs(want).max()
        assert err <= 1e-12, f"rank {r[0]}: shared fronts differ by {err:.3e}"
    # every rank's X = the reference numerics (C restatement)
    import snusolver_b200 as snu
    order, sizes = snu.Solver(nleaves=nleaves).analyze(rp, ci).ordering()
    for c in range(b.shape[1]):
        xo, lus, blocks, lib = oracle_solve(rp, ci, v, b[:, c], nleaves,
                                            order, sizes)
        free_blocks(lib, blocks)
        for r in res:
            err = np.abs(r[2][:, c] - xo).max() / np.abs(xo).max()
            assert err <= 1e-10, f"rank {r[0]} column {c}: {err:.3e}"
    for r in res:
        assert r[3]["backward_error"] <= 1e-12


def _gpu_rank_main(rank, world, nleaves, precision, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    from snusolver_b200.dist import DistSolver
    try:
        torch.cuda.set_device(0)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        rp, ci, v = generators.convdiff3d(22)
        b = generators.rhs(len(rp) - 1, 3, seed=19)
        ds = DistSolver(rank, world, nleaves=nleaves, precision=precision,
                        device=0)
        ds.construct(rp, ci, v).factorize()
        x = ds.solve(b)
        q.put((rank, x, ds.stats, None))
        dist.barrier()
        ds.close()
        dist.destroy_process_group()
    except Exception as e:
        q.put((rank, None, None, repr(e)))


@pytest.mark.gpu
@pytest.mark.parametrize("world,nleaves,precision", [(2, 8, 0), (4, 8, 1)])
def test_distributed_on_the_gpu(gpu, world, nleaves, precision):
    # the CUDA engine's distributed phases, every rank a process on the one
    # GPU of this machine (their kernels never wait on one another; the
    # exchanges are host-side gloo collectives), against the reference
    # numerics (C restatement): FP64 x within 1e-10; FP32 factors refined
    # in FP64 to a backward error of 1e-10
    import snusolver_b200 as snu
    from util import oracle_solve, free_blocks
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_rank_main,
                         args=(r, world, nleaves, precision, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=600) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
    for r in res:
        assert r[3] is None, r[3]
    rp, ci, v = generators.convdiff3d(22)
    b = generators.rhs(len(rp) - 1, 3, seed=19)
    order, sizes = snu.Solver(nleaves=nleaves).analyze(rp, ci).ordering()
    for c in range(3):
        xo, lus, blocks, lib = oracle_solve(rp, ci, v, b[:, c], nleaves,
                                            order, sizes)
        free_blocks(lib, blocks)
        for r in res:
            err = np.abs(r[1][:, c] - xo).max() / np.abs(xo).max()
            assert err <= (1e-10 if precision == 0 else 1e-8), (r[0], c, err)
    for r in res:
        assert r[2]["backward_error"] <= (1e-12 if precision == 0 else 1e-10)
