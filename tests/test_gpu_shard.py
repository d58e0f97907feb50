"""A batch sharded across two ranks (k3dom_b200/shard.py): each rank of a gloo process group
updates its own share of the scenes in a BatchDOM, the per-scene results are gathered on rank 0,
and each equals, bit for bit, the same scene updated in one single-rank batch of all scenes.

Both ranks use the one GPU of the test box. Their kernels never wait on each other (the scenes
are independent and nothing on the data path is shared): only the gloo gather on the host
connects them, as on a multi-GPU node where each rank would own a GPU.
"""
import datetime
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_FRAMES = 3
FIELDS = ("free_mass", "static_mass", "dynamic_mass", "pers_mass", "born_mass", "mean_x_vel", "del_free")


def specs():
    return [dict(seed=30 + k, G=G, Gz=Gz, P=P, n=n, ego=e) for k, (G, Gz, P, n, e) in enumerate([
        (32, 8, 8192, 1500, 0.0), (24, 6, 4096, 900, 2.5), (40, 10, 16384, 2600, 1.2), (28, 8, 6144, 1200, 0.6),
        (36, 8, 12288, 2000, 3.0)])]


def configs():
    from k3dom_b200 import scene
    out = []
    for k, s in enumerate(specs()):
        cfg = scene.small(seed=s["seed"], G=s["G"], Gz=s["Gz"], res=0.2, P=s["P"], B=s["P"] // 4, n_points=s["n"],
                          ego=s["ego"])
        cfg.params["seed"] = 500 + k
        out.append(cfg)
    return out


def run_batch(cfgs):
    """N_FRAMES frames of the scenes in one BatchDOM; per scene a dict of cell fields and particles."""
    import k3dom_b200 as K
    params = [K.make_params("k3dom", **c.params) for c in cfgs]
    b = K.BatchDOM(params, "k3dom")
    try:
        for f in range(N_FRAMES):
            t = 0.1 + 0.1 * f
            pts = []
            for s, c in enumerate(cfgs):
                pose, p = c.scene.scan(f, t, c.n_points)
                b.updatePose(s, *pose)
                pts.append(p)
            b.update([t] * len(cfgs), pts)
        out = []
        for s in range(len(cfgs)):
            d = b.scene(s)
            r = {k: d.get_cell_field(k) for k in FIELDS}
            r["pos"] = d.get_particles("persistent")["pos"]
            out.append(r)
        return out
    finally:
        b.close()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist

    from k3dom_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        cfgs = configs()
        mine = shard.my_scenes([shard.scene_cost(c.params, c.n_points) for c in cfgs], rank, world)
        res = run_batch([cfgs[i] for i in mine]) if mine else []
        gathered = [None] * world
        dist.all_gather_object(gathered, (mine, res))
        verdict = None
        if rank == 0:
            whole = run_batch(cfgs)
            bad = []
            seen = set()
            for owned, results in gathered:
                for i, r in zip(owned, results):
                    seen.add(i)
                    for k, v in r.items():
                        if not np.array_equal(v, whole[i][k], equal_nan=True):
                            bad.append((i, k))
            verdict = (sorted(seen) == list(range(len(cfgs))), bad, [o for o, _ in gathered])
        dist.barrier()
        q.put((rank, verdict))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_batch_equals_single_batch():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    complete, bad, owned = res[0]
    assert complete, owned
    assert all(len(o) > 0 for o in owned), owned  # both ranks had work
    assert not bad, bad
