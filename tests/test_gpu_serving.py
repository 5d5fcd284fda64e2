"""Serving form: continuous batching under a device-memory budget.

A request admitted into a batch with other requests — some already running
when it arrives, some arriving and retiring while it runs, in both precisions
— must give the same result as when it is served alone, and the same as a
World stepping it alone.  A scene's slice of a batch is bit-identical to its
own world, so the bar is bit equality (both precisions).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _req(serving, rid, scene, steps):
    return serving.ServeRequest(rid, 0.0, steps, scene.params.precision,
                                lambda s=scene: (s.params, s.pos, s.vel))


def test_capacity_for_budget_is_tight():
    pfs = load_package()
    from pfs_b200 import serving
    for prec in (pfs.PFS_FP32, pfs.PFS_FP16_CELL):
        for budget in (1 << 26, 3 << 28, 150 * (1 << 30)):
            cap = serving.capacity_for_budget(budget, 512, prec)
            assert cap > 0
            assert pfs.Batch.bytes_for(cap, 512, prec) <= budget
            if cap < (1 << 24):
                assert pfs.Batch.bytes_for(cap + 1, 512, prec) > budget


def _serve(serving, reqs_by_tick, ticks, budget=1 << 30):
    with serving.Server(budget, max_scenes=16, substeps=3) as srv:
        for t in range(ticks):
            for r in reqs_by_tick.get(t, []):
                srv.submit(r)
            srv.tick(float(t))
        assert srv.pending() == 0
        return {r.rid: r for r in srv.finished}


@pytest.mark.gpu
def test_same_result_alone_and_in_mix(cuda_device):
    pfs = load_package()
    from pfs_b200 import scenes, serving
    a = scenes.dam_break(n=6000, seed=11, h=0.03)
    b = scenes.dam_break(n=9000, seed=12, h=0.035, target_density=900.0)
    c = scenes.dam_break(n=4097, seed=13, h=0.025, precision=pfs.PFS_FP16_CELL)
    d = scenes.dam_break(n=3000, seed=14, h=0.02, viscosity=0.08)
    e = scenes.dam_break(n=5000, seed=15, h=0.03, precision=pfs.PFS_FP16_CELL)
    steps = {1: 5, 2: 3, 3: 6, 4: 2, 5: 4}
    alone = {}
    for rid, sc in ((1, a), (3, c)):
        alone[rid] = _serve(serving, {0: [_req(serving, rid, sc, steps[rid])]}, steps[rid])[rid]
    # b runs before a arrives and retires while a runs; d and e arrive and
    # leave in the middle of a's steps
    mix = _serve(serving, {0: [_req(serving, 2, b, steps[2])],
                           1: [_req(serving, 1, a, steps[1]), _req(serving, 3, c, steps[3])],
                           2: [_req(serving, 4, d, steps[4])],
                           3: [_req(serving, 5, e, steps[5])]}, 12)
    assert sorted(mix) == [1, 2, 3, 4, 5]
    for rid in (1, 3):
        for k in ("pos", "vel", "density"):
            assert np.array_equal(_bits(mix[rid].result[k]), _bits(alone[rid].result[k])), (rid, k)
    for rid, sc in ((1, a), (2, b), (4, d)):
        with pfs.World(sc.params, sc.pos, sc.vel) as w:
            w.step(steps[rid])
            want = w.read(pos=True, vel=True)
        assert np.array_equal(_bits(mix[rid].result["pos"]), _bits(want["pos"])), rid
        assert np.array_equal(_bits(mix[rid].result["vel"]), _bits(want["vel"])), rid


@pytest.mark.gpu
def test_oversize_request_rejected(cuda_device):
    pfs = load_package()
    from pfs_b200 import scenes, serving
    big = scenes.dam_break(n=40000, seed=1)
    small = scenes.dam_break(n=2000, seed=2)
    budget = pfs.Batch.bytes_for(30000, 4, pfs.PFS_FP32) * 2 + (1 << 20)
    with serving.Server(budget, max_scenes=4, substeps=3) as srv:
        srv.submit(_req(serving, 1, big, 2))
        srv.submit(_req(serving, 2, small, 2))
        for t in range(3):
            srv.tick(float(t))
        assert [r.rid for r in srv.rejected] == [1]
        assert [r.rid for r in srv.finished] == [2]
