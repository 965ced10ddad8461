"""Host logic of the multi-GPU benchmark paths on CPU (no GPU): the
largest-first sharding of the batched cases, and a world-size-2 gloo run of
the rank protocol (shards disjoint and complete, max-over-ranks timing,
reference arm on rank 0 only)."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_lpt_shard_partitions_cases():
    sizes = [50_000 + (i * 7919) % 750_000 for i in range(64)]
    for ws in range(1, 9):
        shards = [bench.lpt_shard(sizes, ws, r) for r in range(ws)]
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in s) for s in shards]
        # greedy largest-first: no rank exceeds the mean by more than one case
        assert max(loads) <= sum(sizes) / ws + max(sizes)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    sizes = [50_000 + (i * 7919) % 750_000 for i in range(64)]
    mine = bench.lpt_shard(sizes, ws, rank)
    got = [None] * ws
    dist.all_gather_object(got, mine)
    t = torch.tensor([1.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    # the reference arm: rank 0 prints its line, the others exit 0 without work
    out = io.StringIO()
    rc = 0
    if rank != 0:
        class A:
            gpus, steps, warmup, n = ws, 1, 3, 64
        with redirect_stdout(out):
            rc = bench.reference_arm(A())
    q.put((rank, got, float(t.item()), rc, out.getvalue()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_follow_the_rank_protocol():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res.sort()
    shards = res[0][1]
    assert res[1][1] == shards
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(64)) and not (set(shards[0]) & set(shards[1]))
    assert res[0][2] == res[1][2] == 2.0
    assert res[1][3] == 0 and res[1][4] == ""
