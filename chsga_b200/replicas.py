"""Multi-GPU replicas: one process per GPU, each holding the whole graph and
hierarchy, reads dealt round-robin, results gathered.

Reads are independent and the graph is read-only, so the alignment shards by
read with no data-path collective. torch.distributed is only plumbing here:
the gather of per-read scores at the end and the max over ranks of device
times for reporting.
"""
from __future__ import annotations

from typing import Callable, List, Sequence

import numpy as np


def shard_indices(n: int, world: int, rank: int) -> np.ndarray:
    """Read indices of `rank`: round-robin, so each rank gets the same mix of
    lengths when reads arrive in length order."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return np.arange(rank, n, world, dtype=np.int64)


def collective_device(group=None, device=None):
    """Where this rank's collective buffers live: `device` when given, else
    the current CUDA device for an NCCL group (NCCL moves device memory
    only) and the host for any other backend."""
    import torch
    import torch.distributed as dist
    if device is not None:
        return torch.device(device)
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def align_sharded(reads: Sequence[bytes], align: Callable[[List[bytes]], np.ndarray],
                  world: int, rank: int, group=None, device=None) -> np.ndarray:
    """Aligns this rank's share with `align` and all-gathers the int32 scores
    back into read order on every rank (through `collective_device`)."""
    import torch
    import torch.distributed as dist
    idx = shard_indices(len(reads), world, rank)
    local = np.asarray(align([reads[i] for i in idx]), dtype=np.int32)
    if world == 1:
        return local
    dev = collective_device(group, device)
    per = (len(reads) + world - 1) // world
    buf = torch.full((per,), -1, dtype=torch.int32)
    buf[: len(local)] = torch.from_numpy(local)
    buf = buf.to(dev)
    out = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    scores = np.empty(len(reads), dtype=np.int32)
    for r in range(world):
        ri = shard_indices(len(reads), world, r)
        scores[ri] = out[r].cpu().numpy()[: len(ri)]
    return scores


def max_over_ranks(x: float, world: int, group=None, device=None) -> float:
    """Largest value of x over all ranks (device times are reported as the
    slowest rank's)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=collective_device(group, device))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
