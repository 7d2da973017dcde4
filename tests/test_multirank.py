"""The N > 1 path on the CPU: two gloo ranks shard the batched mix and agree on
the max-over-ranks time, as bench.py does with NCCL on GPUs."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from graph_render_b200 import batch


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    total = 64
    costs = [batch.graph_cost(4, i) for i in range(total)]
    mine = batch.shard(costs, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    load = torch.tensor([sum(costs[i] for i in mine)], dtype=torch.float64)
    loads = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(loads, load)
    q.put((rank, got, float(t.item()), [float(x.item()) for x in loads], max(costs)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_partition_the_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=90) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, got, tmax, loads, cmax in out:
        flat = sorted(i for shard in got for i in shard)
        assert flat == list(range(64))                    # every graph once
        assert not set(got[0]) & set(got[1])              # disjoint
        assert tmax == 2.0                                # max over ranks
        assert abs(loads[0] - loads[1]) <= cmax           # LPT balance bound


def test_shard_is_a_partition_for_any_world():
    costs = [batch.graph_cost(4, i) for i in range(100)]
    for world in (1, 2, 3, 8):
        bins = batch.shard(costs, world)
        assert sorted(i for b in bins for i in b) == list(range(100))
