"""Density map (the reference's updateDensityMap.comp) on the GPU, through the
C ABI, against the oracle (itself pinned to the reference shader by
tests/golden/glsl_density_map.npz).  Bar: bit-exact, every voxel."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_oracle, load_package

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
@pytest.mark.parametrize("factor", [1.0, 0.7, 1.6])
def test_density_map_matches_oracle(cuda_device, precision, factor):
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    prec = pfs.PFS_FP32 if precision == "fp32" else pfs.PFS_FP16_CELL
    sc = scenes.dam_break(n=16384, seed=3, precision=prec)
    cs = float(np.float32(np.float32(sc.params.h) * np.float32(factor)))
    with pfs.World(sc.params, sc.pos, sc.vel) as w:
        w.step(2)
        st = w.read(pos=True, keys=True)
        got = w.density_map(cs)
        assert w.device_error() == 0
    want = ora.density_map(sc.params, st["pos"], st["keys"], cs)
    assert got.shape == want.shape == tuple(reversed(ora.density_map_dims(sc.params, cs)))
    assert np.count_nonzero(want) > 0
    assert np.array_equal(_bits(got), _bits(want))


def test_density_map_large_and_device_output(cuda_device):
    """The 1M-particle slab at cell size h (101^3 voxels), written straight
    into device memory, equals the host copy and the oracle."""
    import torch
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    sc = scenes.slab_1m()
    cs = sc.params.h
    with pfs.World(sc.params, sc.pos, sc.vel) as w:
        w.step(1)
        st = w.read(pos=True, keys=True)
        host = w.density_map(cs)
        dev = torch.empty(host.shape, dtype=torch.float32, device="cuda")
        w.density_map_ptr(cs, dev.data_ptr())
        torch.cuda.synchronize()
        assert w.device_error() == 0
    assert np.array_equal(_bits(dev.cpu().numpy()), _bits(host))
    want = ora.density_map(sc.params, st["pos"], st["keys"], cs)
    assert np.array_equal(_bits(host), _bits(want))


def test_density_map_needs_a_step_and_a_cell_size(cuda_device):
    pfs = load_package()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=2048, seed=1)
    with pfs.World(sc.params, sc.pos, sc.vel) as w:
        with pytest.raises(pfs.PfsError):
            w.density_map(sc.params.h)       # no sort yet
        w.step(1)
        with pytest.raises(pfs.PfsError):
            w.density_map(0.0)
        with pytest.raises(pfs.PfsError):
            w.density_map(1e-5)              # 10^15 voxels
        w.write(sc.pos, sc.vel)
        with pytest.raises(pfs.PfsError):
            w.density_map(sc.params.h)       # state rewritten, no sort since
