"""One process per GPU: replicas of the factorize-and-solve path.

The path shards only by independent units -- whole systems (one replica per
GPU), the matrices of a batch, or the requests of a serving stream -- so the
ranks exchange nothing on the data path.  The process group (NCCL on GPUs,
gloo on CPU) carries only the start/stop barriers and the max-over-ranks
timing.  Launch under torchrun (RANK / WORLD_SIZE / LOCAL_RANK / MASTER_*).
"""
from __future__ import annotations

import datetime
import os

__all__ = ["init", "barrier", "max_over_ranks", "shard", "finish"]


def init(backend=None, timeout_s=600):
    """(world size, rank, local rank); joins the process group when the world
    has more than one rank.  backend None: NCCL with a GPU, else gloo."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    use_gpu = torch.cuda.is_available() and backend in (None, "nccl")
    if use_gpu:
        torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        be = backend or ("nccl" if use_gpu else "gloo")
        kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if be == "nccl":
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(be, **kw)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, x):
    """Max of a float over all ranks (the job's time is its slowest rank)."""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(units, ws, rank):
    """The independent units (matrices of a batch, requests of a stream)
    this rank owns: round robin, so every unit has exactly one owner."""
    return [u for i, u in enumerate(units) if i % ws == rank]


def finish(ws):
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
