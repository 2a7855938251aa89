"""Scene sharding for the multi-GPU batched form, on CPU: the partition
covers every scene once and balances the work, and two gloo ranks compute
the same partition and reduce timings as the GPU ranks do over NCCL."""
import os
import socket

import pytest

from nexus_b200.sharding import shard_scenes


def test_partition_covers_and_balances():
    work = [4096 * (1 + (7 * i) % 31) for i in range(256)]
    for world in (1, 2, 3, 8):
        shards = shard_scenes(work, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(work)))
        loads = [sum(work[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(work)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from nexus_b200.sharding import all_max, all_sum
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        work = [1000 + 37 * i for i in range(50)]
        mine = shard_scenes(work, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = all_max(float(10 + rank), world, device="cpu")
        n = all_sum(float(sum(work[i] for i in mine)), world, device="cpu")
        out.put((rank, gathered, t, n, sum(work)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_shards_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (_, g0, t0, n0, total), (_, g1, t1, n1, _) = res
    assert g0 == g1 and sorted(g0[0] + g0[1]) == list(range(50)) and not set(g0[0]) & set(g0[1])
    assert t0 == t1 == 11.0
    assert n0 == n1 == total
