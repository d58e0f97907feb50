"""Sharding a batch of independent scenes across ranks (k3dom_b200/shard.py): the partition is
deterministic, complete and disjoint, balanced within the longest-processing-time bound, and
every rank of a gloo process group (world size 2, CPU) computes the same partition."""
import os
import socket

import numpy as np
import pytest

from k3dom_b200 import scene, shard


def costs16():
    cfgs = scene.config3(seed=0)
    return [shard.scene_cost(c.params, c.n_points) for c in cfgs]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_complete_disjoint_balanced(world):
    c = costs16()
    parts = shard.partition(c, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(c)))
    loads = [sum(c[i] for i in p) for p in parts]
    # LPT bound: max load <= mean load + largest job
    assert max(loads) <= sum(c) / world + max(c) + 1e-6
    assert parts == shard.partition(c, world)  # deterministic


def test_partition_edge_cases():
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5.0], 2) == [[0], []]
    assert shard.partition([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.partition([1.0], 0)


def test_cost_grows_with_work():
    base = dict(resolution=0.1, size=12.8, size_z=3.2, particle_count=1 << 18, new_born_particle_count=1 << 16,
                ls=0.3)
    big = dict(base, particle_count=1 << 22)
    assert shard.scene_cost(big, 30000) > shard.scene_cost(base, 30000)
    assert shard.scene_cost(base, 200000) > shard.scene_cost(base, 10000)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        c = costs16()
        mine = shard.my_scenes(c, rank, world)
        # every rank's view of the whole partition, gathered
        t = torch.full((len(c),), -1, dtype=torch.int64)
        for i in mine:
            t[i] = rank
        gathered = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(gathered, t)
        owner = torch.stack(gathered).max(dim=0).values
        # each scene owned by exactly one rank, and it matches the locally computed partition
        claims = (torch.stack(gathered) >= 0).sum(dim=0)
        ok = bool((claims == 1).all()) and all(
            int(owner[i]) == r for r, p in enumerate(shard.partition(c, world)) for i in p)
        out.put((rank, ok, mine))
    finally:
        dist.destroy_process_group()


def test_ranks_agree_on_partition_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok, _ in res)
    mine = {r: m for r, _, m in res}
    assert sorted(mine[0] + mine[1]) == list(range(16))
