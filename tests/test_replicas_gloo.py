"""Several-GPU host logic on CPU: two gloo ranks (127.0.0.1) run the replica
helpers the bench uses — seeds, shards of independent scenes or requests,
the max of the ranks' times and the sum of their work."""
from __future__ import annotations

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_package


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        load_package()
        from pfs_b200 import replicas
        items = list(range(11))
        mine = replicas.shard(items, rank, world)
        ms = 10.0 + 5.0 * rank                      # rank 1 is the slower one
        q.put({"rank": rank, "seed": replicas.replica_seed(1, rank), "shard": mine,
               "max": replicas.max_over_ranks(ms, dist),
               "sum": replicas.sum_over_ranks(len(mine), dist),
               "tput": replicas.job_throughput(1000.0, world, replicas.max_over_ranks(ms, dist))})
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r["seed"] for r in res] == [1, 2]
    assert sorted(res[0]["shard"] + res[1]["shard"]) == list(range(11))
    assert not set(res[0]["shard"]) & set(res[1]["shard"])
    assert all(r["max"] == 15.0 for r in res)
    assert all(r["sum"] == 11.0 for r in res)
    assert all(r["tput"] == pytest.approx(2000.0 / 0.015) for r in res)


def test_shard_rejects_bad_rank():
    load_package()
    from pfs_b200 import replicas
    with pytest.raises(ValueError):
        replicas.shard([1, 2], 2, 2)
    assert replicas.max_over_ranks(3.0) == 3.0


def _scenes_small():
    """Seven small dam-break scenes with their own parameters (sizes 64 to
    1,000), as the batched workload draws them."""
    load_package()
    from pfs_b200 import scenes
    return scenes.scene_batch(count=7, seed=11, lo=64, hi=1000)


def _step_scene(ora, sc, steps):
    pos, vel, dens, _ = ora.step(sc.params, sc.pos, sc.vel, steps)
    return pos, vel, dens


def _shard_rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from conftest import load_oracle
        ora = load_oracle()
        load_package()
        from pfs_b200 import replicas
        all_scenes = _scenes_small()
        mine = replicas.shard(list(range(len(all_scenes))), rank, world)
        local = {i: _step_scene(ora, all_scenes[i], 3) for i in mine}
        work = replicas.sum_over_ranks(sum(all_scenes[i].n for i in mine), dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
        if rank == 0:
            union = {}
            for part in gathered:
                union.update(part)
            q.put({"union": union, "work": work})
        else:
            q.put(None)
    except Exception as exc:  # reported to the parent instead of a silent timeout
        q.put({"error": f"rank {rank}: {exc!r}"})
        raise
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_step_their_shares_of_a_batch():
    """Each rank steps its share of seven independent scenes (3 steps of 3
    substeps) through the oracle; the union of the shares equals stepping
    every scene in one process, bit for bit, and the summed work is the
    batch's particle count."""
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    errors = [g["error"] for g in got if g is not None and "error" in g]
    assert not errors, errors
    res = next(g for g in got if g is not None)
    from conftest import load_oracle
    ora = load_oracle()
    all_scenes = _scenes_small()
    assert sorted(res["union"]) == list(range(len(all_scenes)))
    assert res["work"] == float(sum(s.n for s in all_scenes))
    import numpy as np
    for i, sc in enumerate(all_scenes):
        want = _step_scene(ora, sc, 3)
        for a, b in zip(res["union"][i], want):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), i
