"""Host logic of the multi-GPU ensemble: members are split across ranks with
no exchange. Two gloo ranks on the CPU check that every rank computes the same
partition, that it covers every member exactly once, and that the node counts
are balanced."""
import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from lbm_solver_3d_b200.ensemble import shard_members
from lbm_solver_3d_b200.workloads import ensemble_members


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ps = ensemble_members(256)
    mine = shard_members(ps, rank, world)
    got = [None] * world
    dist.all_gather_object(got, mine)
    out[rank] = got
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_a_balanced_partition():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, 29517, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        views = [out[r] for r in range(world)]
    assert views[0] == views[1]
    shards = views[0]
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(256))
    ps = ensemble_members(256)
    loads = [sum(ps[i].ncells for i in s) for s in shards]
    assert max(loads) / min(loads) < 1.01


@pytest.mark.parametrize("world", [1, 3, 8])
def test_partition_is_complete_and_balanced(world):
    ps = ensemble_members(256)
    shards = [shard_members(ps, r, world) for r in range(world)]
    assert sorted(i for s in shards for i in s) == list(range(256))
    loads = [sum(ps[i].ncells for i in s) for s in shards]
    assert max(loads) / min(loads) < 1.03
    with pytest.raises(ValueError):
        shard_members(ps, world, world)
