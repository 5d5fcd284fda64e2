"""Batched scenes (pfs_batch_*) against single-scene worlds, through the C ABI.

Bar: bit-exact.  A scene in a batch owns its own slots of the shared table
and keys, so one shared sort leaves it in exactly the order its own world
gives and every kernel computes the same floats; adding and removing other
scenes between steps must not change any scene's results.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _scenes(pfs, precision):
    from pfs_b200 import scenes
    out = [
        scenes.dam_break(n=3000, seed=1, precision=precision),
        scenes.dam_break(n=16384, seed=2, h=0.03, target_density=900.0, pressure_multiplier=150.0,
                         viscosity=0.08, precision=precision),
        scenes.dam_break(n=2048, seed=3, h=0.04, precision=precision),
        scenes.dam_break(n=7777, seed=4, h=0.02, target_density=1100.0, precision=precision),
    ]
    return out


def _world_run(pfs, sc, steps):
    with pfs.World(sc.params, sc.pos, sc.vel) as w:
        w.step(steps)
        return w.read(pos=True, vel=True, density=True)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp32", "fp16cell"])
def test_batch_matches_worlds(cuda_device, precision):
    pfs = load_package()
    scs = _scenes(pfs, precision)
    total = sum(s.n for s in scs)
    with pfs.Batch(total + 100, 8, precision=precision, substeps=3) as b:
        ids = [b.add(s.params, s.pos, s.vel) for s in scs]
        b.step(3)
        b.sync()
        for sid, sc in zip(ids, scs):
            got = b.read(sid, density=True)
            want = _world_run(pfs, sc, 3)
            for k in ("pos", "vel", "density"):
                assert np.array_equal(_bits(got[k]), _bits(want[k])), (sc.n, k)


def test_batch_add_remove_between_steps(cuda_device):
    pfs = load_package()
    from pfs_b200 import scenes
    a, bsc, c = _scenes(pfs, 0)[:3]
    d = scenes.dam_break(n=5000, seed=9, h=0.025)
    with pfs.Batch(60000, 8, substeps=3) as b:
        ia, ib, ic = b.add(a.params, a.pos, a.vel), b.add(bsc.params, bsc.pos, bsc.vel), \
            b.add(c.params, c.pos, c.vel)
        b.step(2)
        before = b.read(ic, density=True)
        b.remove(ib)           # middle scene leaves: c moves down
        moved = b.read(ic, density=True)
        for k in ("pos", "vel", "density"):
            assert np.array_equal(_bits(moved[k]), _bits(before[k])), k
        idd = b.add(d.params, d.pos, d.vel)
        b.step(2)
        b.sync()
        for sid, sc, steps in ((ia, a, 4), (ic, c, 4), (idd, d, 2)):
            got = b.read(sid)
            want = _world_run(pfs, sc, steps)
            assert np.array_equal(_bits(got["pos"]), _bits(want["pos"])), sc.n
            assert np.array_equal(_bits(got["vel"]), _bits(want["vel"])), sc.n
        info = b.info()
        assert info["scenes"] == 3 and info["particles"] == a.n + c.n + d.n


def test_batch_feed_mode_reruns_inputs(cuda_device):
    pfs = load_package()
    scs = _scenes(pfs, 0)[:2]
    with pfs.Batch(40000, 4, substeps=3) as b:
        ids = [b.add(s.params, s.pos, s.vel) for s in scs]
        b.set_feed(True)
        b.step(5)              # five times the first step
        b.sync()
        for sid, sc in zip(ids, scs):
            got = b.read(sid)
            want = _world_run(pfs, sc, 1)
            assert np.array_equal(_bits(got["pos"]), _bits(want["pos"]))


def test_batch_capacity_refusals(cuda_device):
    pfs = load_package()
    sc = _scenes(pfs, 0)[0]
    with pfs.Batch(sc.n + 10, 1, substeps=3) as b:
        b.add(sc.params, sc.pos, sc.vel)
        with pytest.raises(pfs.PfsError) as ei:
            b.add(sc.params, sc.pos, sc.vel)
        assert ei.value.status == pfs.PFS_EBUDGET
        q = sc.params.copy()
        q.substeps = 1
        with pytest.raises(pfs.PfsError):
            b.remove(12345)


def test_batch_flat_shape_matches_worlds(cuda_device):
    """The flat shape in a batch (scenes with both searches): every scene
    bit-identical to its own world."""
    pfs = load_package()
    scs = _scenes(pfs, 0)
    total = sum(s.n for s in scs)
    with pfs.Batch(total + 100, 8, substeps=3) as b:
        b.set_shape(pfs.PFS_SHAPE_FLAT, pfs.PFS_SEARCH_AUTO)
        ids = [b.add(s.params, s.pos, s.vel) for s in scs]
        b.step(3)
        b.sync()
        for sid, sc in zip(ids, scs):
            got = b.read(sid, density=True)
            want = _world_run(pfs, sc, 3)
            for k in ("pos", "vel", "density"):
                assert np.array_equal(_bits(got[k]), _bits(want[k])), (sc.n, k)
