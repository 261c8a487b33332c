"""Replica sharding over torch.distributed, world size 2 on the gloo backend
(CPU): every read is aligned exactly once, scores come back in read order
on every rank, and the reported time is the slowest rank's. The per-rank
aligner here is the CPU oracle, standing in for a GPU context."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, files, reads, want, q):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist
    import oracle as orc
    from chsga_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        o = orc.Oracle(files, threads=1)
        seen = []

        def align(batch):
            seen.extend(batch)
            return o.scores(batch)

        got = replicas.align_sharded(reads, align, world, rank)
        slowest = replicas.max_over_ranks(float(rank + 1), world)
        q.put((rank, got.tolist(), len(seen), slowest))
    finally:
        dist.destroy_process_group()


def test_world2_round_robin_and_gather(small_graph, oracle_small):
    g, files, reads = small_graph
    reads = reads[:9]
    want = oracle_small.scores(reads).tolist()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, files, reads, want, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == want and res[1][1] == want
    assert res[0][2] + res[1][2] == len(reads)  # each read aligned once
    assert res[0][2] == 5 and res[1][2] == 4  # round-robin
    assert res[0][3] == res[1][3] == 2.0


def test_shard_indices_cover_everything():
    from chsga_b200 import replicas
    for n in (0, 1, 7, 64):
        for w in (1, 2, 3, 8):
            parts = [replicas.shard_indices(n, w, r) for r in range(w)]
            allv = np.sort(np.concatenate(parts)) if parts else np.array([])
            assert allv.tolist() == list(range(n))


def _nccl_worker(port, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from chsga_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        dev = replicas.collective_device()
        buf = torch.arange(4, dtype=torch.int32, device=dev)
        out = [torch.empty_like(buf)]
        dist.all_gather(out, buf)
        t = torch.tensor([3.5], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((dev.type, out[0].cpu().tolist(), float(t.item())))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_nccl_group_gathers_on_the_device():
    """Under NCCL the gather and max buffers go to the current CUDA device
    (one rank: this run has one GPU)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_worker, args=(_free_port(), q))
    p.start()
    res = q.get(timeout=180)
    p.join(timeout=60)
    assert p.exitcode == 0
    assert res == ("cuda", [0, 1, 2, 3], 3.5)
