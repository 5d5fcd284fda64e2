"""Autotuner and explicit kernel shapes: every shape and neighbour search
gives the same bits, and tuning leaves the state as it found it."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _run(pfs, sc, steps, shape=None, search=-1, tune=False):
    with pfs.World(sc.params, sc.pos, sc.vel) as w:
        w.step(1)
        res = None
        if tune:
            before = w.read(pos=True, vel=True, keys=True, perm=True)
            res = w.autotune(2)
            after = w.read(pos=True, vel=True, keys=True, perm=True)
            for k in before:
                assert np.array_equal(_bits(before[k]), _bits(after[k])), k
        elif shape is not None:
            if shape == pfs.PFS_SHAPE_STAGED and not w.staged_available():
                return None, None
            w.set_shape(shape, search)
        w.step(steps)
        out = w.read(pos=True, vel=True, density=True)
        assert w.device_error() == 0
    return out, res


@pytest.mark.parametrize("n", [4096, 12289])
def test_every_shape_same_bits(cuda_device, n):
    pfs = load_package()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=n, seed=7)
    ref, _ = _run(pfs, sc, 3, pfs.PFS_SHAPE_LIST, pfs.PFS_SEARCH_TABLE)
    for shape in (pfs.PFS_SHAPE_SIMPLE, pfs.PFS_SHAPE_SLAB, pfs.PFS_SHAPE_LIST, pfs.PFS_SHAPE_FLAT,
                  pfs.PFS_SHAPE_STAGED):
        for search in (pfs.PFS_SEARCH_TABLE, pfs.PFS_SEARCH_GRID):
            if shape == pfs.PFS_SHAPE_STAGED and search == pfs.PFS_SEARCH_GRID:
                continue  # the staged shape scans table ranges only
            got, _ = _run(pfs, sc, 3, shape, search)
            if got is None:
                continue  # staged stage too small for this table (refused)
            for k in ("pos", "vel", "density"):
                assert np.array_equal(_bits(got[k]), _bits(ref[k])), (shape, search, k)


def test_world_autotune_keeps_results(cuda_device):
    pfs = load_package()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=12289, seed=8)
    plain, _ = _run(pfs, sc, 4)
    tuned, res = _run(pfs, sc, 4, tune=True)
    # four shapes x two searches, and the staged shape where its stage fits
    staged = any(t["shape"] == "staged" for t in res["trials"])
    assert len(res["trials"]) == (9 if staged else 8) and res["chosen"] is not None
    assert all(t["ms_per_step"] > 0 for t in res["trials"])
    for k in ("pos", "vel", "density"):
        assert np.array_equal(_bits(tuned[k]), _bits(plain[k])), k


def test_batch_autotune_keeps_results(cuda_device):
    pfs = load_package()
    from pfs_b200 import scenes
    scs = [scenes.dam_break(n=n, seed=i) for i, n in enumerate((4097, 3000, 8192))]
    outs = []
    for tune in (False, True):
        with pfs.Batch(sum(s.n for s in scs), 4, substeps=3) as b:
            ids = [b.add(s.params, s.pos, s.vel) for s in scs]
            b.step(1)
            if tune:
                res = b.autotune(2)
                assert len(res["trials"]) == 8 and res["chosen"] is not None
            b.step(2)
            outs.append([b.read(i, density=True) for i in ids])
    for a, t in zip(outs[0], outs[1]):
        for k in ("pos", "vel", "density"):
            assert np.array_equal(_bits(a[k]), _bits(t[k])), k
