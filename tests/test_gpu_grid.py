"""Grid search of the neighbour passes against the table scan and the oracle.

The cell table has 2^popcount(n - 1) slots, so sizes such as 4097 (two
slots) or 12289 (four) put thousands of particles of distant cells into each
slot range.  The grid search finds the in-range candidates through the
spatial grid of x* instead and replays them in table order; the bar is the
same as for the table scan: bit-exact with the oracle in FP32, and
bit-identical to the table scan in the FP16-cell form.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_oracle, load_package
from test_gpu_parity import _assert_bits_equal, _check_substep, _uniform_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["table", "grid"])
def search(request, monkeypatch):
    monkeypatch.setenv("PFS_NEIGHBOR_SEARCH", request.param)
    return request.param


@pytest.mark.parametrize("n", [1, 3, 1000, 3001, 4097, 12289])
def test_substep_stages(cuda_device, search, n):
    pfs, ora = load_package(), load_oracle()
    p, pos, vel = _uniform_scene(pfs, n, seed=100 + n)
    _check_substep(pfs, ora, p, pos, vel)


def test_dense_overflow_falls_back(cuda_device, search):
    """Neighbourhoods larger than the warp buffers fall back to walking the
    table ranges for those particles; mixed with ordinary ones in one pass."""
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=20000, seed=5, h=0.09)
    _check_substep(pfs, ora, sc.params, sc.pos, sc.vel)


def test_walls_and_outside(cuda_device, search):
    """Particles outside the box (edge cells of the grid after clamping) and
    piled against the walls."""
    pfs, ora = load_package(), load_oracle()
    rng = np.random.default_rng(9)
    n = 6145
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-0.2, 1.2, (n, 3))
    pos[: n // 4, 0] = 0.0
    pos[n // 4: n // 2, 1] = 1.0
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0.0, 3.0, (n, 3))
    p = pfs.make_params(0.06, 1000.0, 250.0, 0.03, dt=1.0 / 240.0)
    _check_substep(pfs, ora, p, pos, vel)


def _rollout(pfs, params, pos, vel, steps):
    with pfs.World(params, pos, vel) as w:
        w.step(steps)
        out = w.read(pos=True, vel=True, density=True)
        assert w.device_error() == 0
    return out


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_rollout_grid_equals_table(cuda_device, monkeypatch, precision):
    pfs = load_package()
    from pfs_b200 import scenes
    prec = pfs.PFS_FP32 if precision == "fp32" else pfs.PFS_FP16_CELL
    sc = scenes.dam_break(n=24577, seed=2, precision=prec)
    got = {}
    for mode in ("table", "grid"):
        monkeypatch.setenv("PFS_NEIGHBOR_SEARCH", mode)
        got[mode] = _rollout(pfs, sc.params, sc.pos, sc.vel, 12)
    for k in ("pos", "vel", "density"):
        _assert_bits_equal(k, got["grid"][k], got["table"][k])


def test_rollout_grid_matches_oracle(cuda_device, monkeypatch):
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    monkeypatch.setenv("PFS_NEIGHBOR_SEARCH", "grid")
    sc = scenes.dam_break(n=3001, seed=4)
    got = _rollout(pfs, sc.params, sc.pos, sc.vel, 10)
    opos, ovel = ora.step(sc.params, sc.pos, sc.vel, 10)[:2]
    _assert_bits_equal("pos", got["pos"], opos)
    _assert_bits_equal("vel", got["vel"], ovel)


def test_batch_mixed_modes(cuda_device, monkeypatch):
    """Scenes choosing different searches (by their own size) share one
    batch; each matches its standalone world bit for bit."""
    monkeypatch.delenv("PFS_NEIGHBOR_SEARCH", raising=False)
    pfs = load_package()
    from pfs_b200 import scenes
    scs = [scenes.dam_break(n=n, seed=i, h=h) for i, (n, h) in
           enumerate([(4097, 0.03), (4096, 0.035), (12289, 0.04), (3000, 0.02), (20481, 0.05)])]
    with pfs.Batch(sum(s.pos.shape[0] for s in scs), len(scs), substeps=3) as b:
        ids = [b.add(s.params, s.pos, s.vel) for s in scs]
        b.step(4)
        res = [b.read(i) for i in ids]
    for s, r in zip(scs, res):
        want = _rollout(pfs, s.params, s.pos, s.vel, 4)
        _assert_bits_equal("pos", r["pos"], want["pos"])
        _assert_bits_equal("vel", r["vel"], want["vel"])
