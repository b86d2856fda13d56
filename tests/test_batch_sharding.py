"""Sharding of the batched workload over ranks (bench.shard_instances), run
as two gloo ranks on the CPU: every instance lands on exactly one rank and
the node counts are balanced to within the largest instance."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from pardiso2_b200 import model as M


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = [n ** 3 for n, _, _ in M.batch_specs(64, 4)]
    mine = bench.shard_instances(sizes, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, (mine, sum(sizes[i] for i in mine)))
    if rank == 0:
        q.put(got)
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2])
def test_shards_cover_every_instance_once(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sizes = [n ** 3 for n, _, _ in M.batch_specs(64, 4)]
    allidx = sorted(i for part, _ in got for i in part)
    assert allidx == list(range(64))
    loads = [load for _, load in got]
    assert max(loads) - min(loads) <= max(sizes)
    assert bench.shard_instances(sizes, 1) == [list(range(64))]
