"""Seeded synthetic scenes for the five workloads this library is measured on.

No public dataset is involved: every initial state is generated here from a
seed (numpy PCG64).  The reference initialises its one scene with rand() in a
centred sub-box and v = (0, 0, -100) (src/renderer/renderer.c:569-642); the
scenes below follow the workload descriptions instead:

  dam_break        16,384 particles, jittered cubic lattice in
                   [0,0.4]x[0,0.8]x[0,1] of the unit box, v = 0, seed 0
  slab_1m          1,048,576 particles uniform in [0,0.8]x[0,1.6]x[0,2] of the
                   [0,2]^3 box, v ~ N(0, 0.05^2), seed 1
  colliding_blocks 4,194,304 particles, two blocks of 2^21 in the [0,4]^3 box
                   (x in [0.5,1.9] and [2.1,3.5], y and z in [1,3]),
                   v = +-(1.5, 0, 0), seed 2
  scene_batch      256 dam-break scenes, sizes log-uniform in [2048, 262144],
                   per-scene h, target density, pressure multiplier and
                   viscosity drawn uniformly, seed 3
  request_stream   Poisson arrivals at 200 requests/s for 60 s, sizes
                   log-uniform in [1024, 524288], FP32 or FP16-cell 50/50,
                   step counts log-uniform in [10, 1000], seed 4
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import PFS_FP16_CELL, PFS_FP32, Params, make_params


def lattice_fill(n: int, lo, hi, rng: np.random.Generator, jitter: float = 0.1) -> np.ndarray:
    """n points on a cubic lattice filling the box [lo, hi] in z-major order,
    spacing chosen as the largest one that fits n points, jittered uniformly by
    +-jitter * spacing per axis.  Returns (n, 4) float32 with w = 0."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    ext = hi - lo
    s = (np.prod(ext) / n) ** (1.0 / 3.0)
    while True:
        dims = np.floor(ext / s).astype(np.int64)
        if int(np.prod(dims)) >= n:
            break
        s *= 0.995
    nx, ny, nz = (int(d) for d in dims)
    idx = np.arange(n, dtype=np.int64)
    ix = idx % nx
    iy = (idx // nx) % ny
    iz = idx // (nx * ny)
    base = np.stack([ix, iy, iz], axis=1).astype(np.float64) + 0.5
    pos = lo + base * s
    pos += rng.uniform(-jitter * s, jitter * s, size=pos.shape)
    out = np.zeros((n, 4), np.float32)
    out[:, :3] = pos.astype(np.float32)
    return out


@dataclass
class Scene:
    name: str
    params: Params
    pos: np.ndarray
    vel: np.ndarray
    steps: int

    @property
    def n(self) -> int:
        return self.pos.shape[0]


def dam_break(n: int = 16384, seed: int = 0, h: float = 0.035, target_density: float = 1000.0,
              pressure_multiplier: float = 200.0, viscosity: float = 0.05,
              precision: int = PFS_FP32, flags: int = 0) -> Scene:
    rng = np.random.default_rng(seed)
    pos = lattice_fill(n, (0.0, 0.0, 0.0), (0.4, 0.8, 1.0), rng)
    vel = np.zeros((n, 4), np.float32)
    p = make_params(h, target_density, pressure_multiplier, viscosity, gravity=(0.0, -9.81, 0.0),
                    dt=1.0 / 120.0, substeps=3, box_min=(0, 0, 0), box_max=(1, 1, 1), damping=0.5,
                    precision=precision, flags=flags)
    return Scene("dam_break", p, pos, vel, 200)


def slab_1m(n: int = 1 << 20, seed: int = 1, precision: int = PFS_FP32, flags: int = 0) -> Scene:
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = rng.uniform(0.0, 0.8, n)
    pos[:, 1] = rng.uniform(0.0, 1.6, n)
    pos[:, 2] = rng.uniform(0.0, 2.0, n)
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0.0, 0.05, (n, 3))
    p = make_params(0.02, 1000.0, 250.0, 0.03, gravity=(0.0, -9.81, 0.0), dt=1.0 / 240.0,
                    substeps=1, box_min=(0, 0, 0), box_max=(2, 2, 2), damping=0.5,
                    precision=precision, flags=flags)
    return Scene("slab_1m", p, pos, vel, 1000)


def colliding_blocks(n: int = 1 << 22, seed: int = 2, precision: int = PFS_FP32,
                     flags: int = 0) -> Scene:
    rng = np.random.default_rng(seed)
    half = n // 2
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    for b, (x0, x1, vx) in enumerate(((0.5, 1.9, 1.5), (2.1, 3.5, -1.5))):
        sl = slice(b * half, (b + 1) * half if b == 0 else n)
        m = sl.stop - sl.start
        pos[sl, 0] = rng.uniform(x0, x1, m)
        pos[sl, 1] = rng.uniform(1.0, 3.0, m)
        pos[sl, 2] = rng.uniform(1.0, 3.0, m)
        vel[sl, 0] = vx
    p = make_params(0.015, 1000.0, 250.0, 0.03, gravity=(0.0, -9.81, 0.0), dt=1.0 / 240.0,
                    substeps=1, box_min=(0, 0, 0), box_max=(4, 4, 4), damping=0.5,
                    precision=precision, flags=flags)
    return Scene("colliding_blocks", p, pos, vel, 100)


def _log_uniform_int(rng: np.random.Generator, lo: int, hi: int, size=None):
    return np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi + 1), size))).astype(np.int64)


def scene_batch(count: int = 256, seed: int = 3, lo: int = 2048, hi: int = 262144,
                precision: int = PFS_FP32) -> List[Scene]:
    rng = np.random.default_rng(seed)
    sizes = np.clip(_log_uniform_int(rng, lo, hi, count), lo, hi)
    out = []
    for i, n in enumerate(sizes):
        h = float(rng.uniform(0.015, 0.04))
        rho0 = float(rng.uniform(800.0, 1200.0))
        k = float(rng.uniform(100.0, 300.0))
        visc = float(rng.uniform(0.01, 0.1))
        s = dam_break(int(n), seed=int(rng.integers(0, 2**31 - 1)), h=h, target_density=rho0,
                      pressure_multiplier=k, viscosity=visc, precision=precision)
        s.name = f"scene{i}"
        out.append(s)
    return out


@dataclass
class RequestSpec:
    """One serving request; its scene is built on demand (make_scene)."""
    rid: int
    arrival_s: float
    n: int
    steps: int
    precision: int
    h: float
    target_density: float
    pressure_multiplier: float
    viscosity: float
    scene_seed: int

    def make_scene(self) -> Scene:
        sc = dam_break(self.n, seed=self.scene_seed, h=self.h, target_density=self.target_density,
                       pressure_multiplier=self.pressure_multiplier, viscosity=self.viscosity,
                       precision=self.precision)
        sc.name = f"req{self.rid}"
        return sc


def request_stream(rate: float = 200.0, duration_s: float = 60.0, seed: int = 4,
                   lo: int = 1024, hi: int = 524288, steps_lo: int = 10, steps_hi: int = 1000,
                   max_requests: int = 0) -> List[RequestSpec]:
    """Poisson arrivals at `rate` per second for `duration_s`; sizes
    log-uniform in [lo, hi], FP32 or FP16-cell 50/50, step counts log-uniform
    in [steps_lo, steps_hi], scene parameters drawn as for scene_batch, dam-break
    lattice initial states (built lazily: a 60 s stream holds ~10^9 particles)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out: List[RequestSpec] = []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration_s:
            break
        n = int(np.clip(_log_uniform_int(rng, lo, hi), lo, hi))
        prec = PFS_FP16_CELL if rng.uniform() < 0.5 else PFS_FP32
        steps = int(np.clip(_log_uniform_int(rng, steps_lo, steps_hi), steps_lo, steps_hi))
        out.append(RequestSpec(len(out), t, n, steps, prec, float(rng.uniform(0.015, 0.04)),
                               float(rng.uniform(800.0, 1200.0)), float(rng.uniform(100.0, 300.0)),
                               float(rng.uniform(0.01, 0.1)), int(rng.integers(0, 2**31 - 1))))
        if max_requests and len(out) >= max_requests:
            break
    return out
