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
