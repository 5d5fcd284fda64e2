"""The seeded synthetic inputs (particle-fluid-simulation_b200/scenes.py)
follow the five workload descriptions: particle counts, boxes, initial
distributions, parameters, seeds and the request stream's statistics."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_package


@pytest.fixture(scope="module")
def sc():
    load_package()
    from pfs_b200 import scenes
    return scenes


def _params(p):
    return {"h": p.h, "rho0": p.target_density, "k": p.pressure_multiplier, "visc": p.viscosity,
            "g": tuple(p.gravity), "dt": p.dt, "substeps": p.substeps, "lo": tuple(p.box_min),
            "hi": tuple(p.box_max), "rest": tuple(p.restitution), "mass": p.particle_mass,
            "margins": (p.margin_predict, p.margin_integrate)}


def test_dam_break(sc):
    s = sc.dam_break()
    q = _params(s.params)
    assert s.n == 16384 and s.steps == 200
    assert q["h"] == pytest.approx(0.035) and q["rho0"] == 1000 and q["k"] == 200
    assert q["visc"] == pytest.approx(0.05) and q["g"] == pytest.approx((0, -9.81, 0))
    assert q["substeps"] == 3 and q["dt"] == np.float32(np.float32(1 / 120) / np.float32(3))
    assert q["lo"] == (0, 0, 0) and q["hi"] == (1, 1, 1)
    assert q["rest"] == pytest.approx((0.5,) * 6) and q["mass"] == 1 and q["margins"] == (0, 0)
    p = s.pos[:, :3].astype(np.float64)
    assert (p >= 0).all() and (p <= [0.4, 0.8, 1.0]).all()
    assert not s.vel.any()
    # the lattice fills the block: its extent reaches the block's far faces
    assert (p.max(axis=0) > [0.38, 0.76, 0.95]).all()
    again = sc.dam_break()
    assert np.array_equal(again.pos, s.pos)  # seeded


def test_lattice_jitter_bound(sc):
    rng = np.random.default_rng(0)
    n, lo, hi = 1000, (0.0, 0.0, 0.0), (1.0, 2.0, 0.5)
    pts = sc.lattice_fill(n, lo, hi, rng)[:, :3].astype(np.float64)
    ext = np.array(hi) - np.array(lo)
    s = (np.prod(ext) / n) ** (1 / 3)
    while np.prod(np.floor(ext / s)) < n:
        s *= 0.995
    frac = pts / s - 0.5
    dev = np.abs(frac - np.round(frac))
    assert dev.max() <= 0.1 + 1e-5


def test_slab_1m(sc):
    s = sc.slab_1m()
    q = _params(s.params)
    assert s.n == 1 << 20 and s.steps == 1000
    assert q["h"] == pytest.approx(0.02) and q["rho0"] == 1000 and q["k"] == 250
    assert q["visc"] == pytest.approx(0.03) and q["substeps"] == 1
    assert q["dt"] == np.float32(1 / 240) and q["hi"] == (2, 2, 2)
    p = s.pos[:, :3]
    assert (p >= 0).all() and (p <= [0.8, 1.6, 2.0]).all()
    # uniform: the means sit at the slab centre
    assert np.allclose(p.mean(axis=0), [0.4, 0.8, 1.0], atol=2e-3)
    v = s.vel[:, :3].astype(np.float64)
    assert abs(v.mean()) < 1e-3 and v.std() == pytest.approx(0.05, rel=1e-2)


def test_colliding_blocks(sc):
    s = sc.colliding_blocks()
    assert s.n == 1 << 22 and s.params.h == pytest.approx(0.015)
    assert tuple(s.params.box_max) == (4, 4, 4)
    a, b = s.pos[: 1 << 21, :3], s.pos[1 << 21:, :3]
    assert (a[:, 0] >= 0.5).all() and (a[:, 0] <= 1.9).all()
    assert (b[:, 0] >= 2.1).all() and (b[:, 0] <= 3.5).all()
    for blk in (a, b):
        assert (blk[:, 1:] >= 1).all() and (blk[:, 1:] <= 3).all()
    assert (s.vel[: 1 << 21, 0] == 1.5).all() and (s.vel[1 << 21:, 0] == -1.5).all()
    assert not s.vel[:, 1:].any()


def test_scene_batch(sc):
    scs = sc.scene_batch(256)
    sizes = np.array([s.n for s in scs])
    assert len(scs) == 256 and sizes.min() >= 2048 and sizes.max() <= 262144
    # log-uniform: about half below the geometric mean of the bounds
    gm = math.sqrt(2048 * 262144)
    assert 0.4 < (sizes < gm).mean() < 0.6
    for s in scs:
        q = _params(s.params)
        assert 0.015 <= q["h"] <= 0.04 and 800 <= q["rho0"] <= 1200
        assert 100 <= q["k"] <= 300 and 0.01 <= q["visc"] <= 0.1
        assert q["substeps"] == 3 and q["hi"] == (1, 1, 1)
    assert len({round(s.params.h, 6) for s in scs}) > 200  # drawn per scene


def test_request_stream(sc):
    reqs = sc.request_stream()
    t = np.array([r.arrival_s for r in reqs])
    # Poisson at 200/s for 60 s: 12,000 expected, sd about 110
    assert abs(len(reqs) - 12000) < 500
    assert (np.diff(t) > 0).all() and t[-1] < 60
    gaps = np.diff(t)
    assert gaps.mean() == pytest.approx(1 / 200, rel=0.05)
    assert gaps.std() == pytest.approx(1 / 200, rel=0.1)  # exponential gaps
    n = np.array([r.n for r in reqs])
    steps = np.array([r.steps for r in reqs])
    assert n.min() >= 1024 and n.max() <= 524288
    assert steps.min() >= 10 and steps.max() <= 1000
    fp16 = np.mean([r.precision == sc.PFS_FP16_CELL for r in reqs])
    assert abs(fp16 - 0.5) < 0.03
    assert 0.45 < (n < math.sqrt(1024 * 524288)).mean() < 0.55
    one = reqs[0].make_scene()
    assert one.n == reqs[0].n and one.params.h == pytest.approx(reqs[0].h)
