"""Known-answer and property tests of the oracle that need no fixtures:
hand-derived two-particle values, sort stability, table invariants, walls."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_oracle, load_package


def _hash_py(x, y, z):
    m = 0xFFFFFFFF
    h = ((x * 73856093) & m) ^ ((y * 19349663) & m) ^ ((z * 83492791) & m)
    h ^= h >> 16
    h = (h * 0x7FEB352D) & m
    h ^= h >> 15
    h = (h * 0x846CA68B) & m
    h ^= h >> 16
    return h


def test_hash_matches_python_restatement():
    ora = load_oracle()
    rng = np.random.default_rng(0)
    for x, y, z in rng.integers(0, 2**32, (200, 3), dtype=np.uint64):
        assert ora.cell_hash(int(x), int(y), int(z)) == _hash_py(int(x), int(y), int(z))


def test_stable_sort_and_table_invariants():
    ora = load_oracle()
    rng = np.random.default_rng(1)
    n = 5000
    keys = rng.integers(0, 300, n).astype(np.uint32)
    sk, perm = ora.sort(keys)
    assert np.array_equal(perm, np.argsort(keys, kind="stable"))
    assert np.all(np.diff(sk.astype(np.int64)) >= 0)
    start, end = ora.table(sk)
    for k in range(n):
        if start[k] == -1:
            assert k not in set(keys[:0])  # untouched slot
            assert not np.any(sk == k)
        else:
            s, e = start[k], end[k]
            assert np.all(sk[s:e] == k)
            assert s == 0 or sk[s - 1] != k
            assert e == n or sk[e] != k


def _key_py(p, n, xyz):
    c = [int(math.floor(np.float32(np.float32(xyz[a]) - np.float32(p.box_min[a])) /
                        np.float32(p.h))) for a in range(3)]
    return _hash_py(c[0] & 0xFFFFFFFF, c[1] & 0xFFFFFFFF, c[2] & 0xFFFFFFFF) & (n - 1), c


@pytest.mark.parametrize("n,kn", [(2, 0.0), (3, 2.0), (8, 1.5)])
def test_few_particle_density_and_force_analytic(n, kn):
    """Density and force of a few particles from the reference formulas in
    float64, including the reference's counting of a neighbour once per
    sample point / cell offset whose key lands on the neighbour's slot (keys
    are not de-duplicated; with n slots, distinct cells collide often)."""
    pfs, ora = load_package(), load_oracle()
    h, m, rho0, k = 1.0, 0.7, 0.5, 10.0
    p = pfs.make_params(h, rho0, k, 1.0, gravity=(0.0, 0.0, 0.0), dt=0.01, box_min=(0, 0, 0),
                        box_max=(10, 10, 10), damping=1.0, near_pressure_multiplier=kn,
                        particle_mass=m)
    rng = np.random.default_rng(n)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = (5.0 + rng.uniform(-0.6, 0.6, (n, 3))).astype(np.float32)
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0, 1, (n, 3)).astype(np.float32)
    _, _, _, tr, _, _ = ora.substep(p, pos, vel, trace=True)
    xp = tr["xp"][:, :3].astype(np.float64)
    vs = vel[tr["perm"], :3].astype(np.float64)
    slot = tr["keys"]                     # key slot each sorted particle is listed under
    V = 2 * math.pi * h**5 / 15
    rho = np.zeros(n)
    rhon = np.zeros(n)
    for i in range(n):
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    s = [np.float32(np.float32(tr["xp"][i, a]) + np.float32(h * o))
                         for a, o in enumerate((dx, dy, dz))]
                    if any(s[a] < p.box_min[a] or s[a] > p.box_max[a] for a in range(3)):
                        continue
                    key, _ = _key_py(p, n, s)
                    for j in range(n):
                        if slot[j] == key:
                            dist = np.linalg.norm(xp[j] - xp[i])
                            if dist < h:
                                rho[i] += m * (h - dist) ** 2
                                rhon[i] += m * (h - dist) ** 3
    rho = np.maximum(rho / V, 0.01)
    rhon = np.maximum(rhon * 15 / (math.pi * h**6), 0.01)
    assert np.allclose(tr["density"], rho, rtol=1e-5)
    assert np.allclose(tr["near_density"], rhon, rtol=1e-5)
    rho_f, rhon_f = tr["density"].astype(np.float64), tr["near_density"].astype(np.float64)
    for i in range(n):
        _, ci = _key_py(p, n, tr["xp"][i, :3])
        f = np.zeros(3)
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    cc = [(ci[0] + dx) & 0xFFFFFFFF, (ci[1] + dy) & 0xFFFFFFFF,
                          (ci[2] + dz) & 0xFFFFFFFF]
                    key = _hash_py(*cc) & (n - 1)
                    for j in range(n):
                        if j == i or slot[j] != key:
                            continue
                        d = xp[j] - xp[i]
                        dist = np.linalg.norm(d)
                        if dist >= h or dist < 1e-7:
                            continue
                        shared = ((rho_f[j] - rho0) * k + (rho_f[i] - rho0) * k) / 2
                        f += shared * (dist - h) * 15 / (math.pi * h**5) * m / rho_f[j] * d / dist
                        f += m * (h - dist) ** 2 / rho_f[j] * (vs[j] - tr["vp"][i, :3])
                        snp = (kn * rhon_f[i] + kn * rhon_f[j]) / 2
                        f += snp * (h - dist) ** 2 * (-45 / (math.pi * h**6)) * m / rhon_f[j] * d / dist
        want = vs[i] + f / rho_f[i] * p.dt
        assert np.allclose(tr["vel_force"][i, :3], want, rtol=1e-5, atol=1e-6), (i, want)


def test_walls_clamp_and_reflect():
    pfs, ora = load_package(), load_oracle()
    p = pfs.make_params(0.5, 1.0, 1.0, 1.0, gravity=(0.0, 0.0, 0.0), dt=0.1, box_min=(0, 0, 0),
                        box_max=(1, 1, 1), damping=0.5)
    pos = np.array([[0.05, 0.5, 0.5, 0.0]], np.float32)
    vel = np.array([[-1.0, 0.0, 0.0, 0.0]], np.float32)
    opos, ovel, _, tr, _, _ = ora.substep(p, pos, vel, trace=True)
    # predict: x* = 0.05 - 0.1 < 0 -> clamped to 0, v* = +0.5
    assert tr["xp"][0, 0] == 0.0 and tr["vp"][0, 0] == np.float32(0.5)
    # integrate from x = 0.05 with v = -1 (single particle: no force) -> same
    assert opos[0, 0] == 0.0 and ovel[0, 0] == np.float32(0.5)


def test_reference_defaults():
    pfs = load_package()
    p = pfs.reference_default()
    assert p.h == 2.5 and p.gravity[2] == -100.0 and p.substeps == 1
    assert p.particle_mass == 1.0 and p.pressure_multiplier == 15000.0
    assert p.target_density == 1.0 and p.near_pressure_multiplier == 0.0
    assert list(p.box_min) == [-140.0, -40.0, -40.0] and list(p.box_max) == [140.0, 40.0, 40.0]
    assert p.margin_predict == np.float32(0.3)
    assert p.margin_integrate == np.float32(np.float32(0.3) + np.float32(0.5))
    assert list(p.restitution) == [1.0, 1.0, 1.0, 1.0, np.float32(0.95), 1.0]
    assert p.dt == np.float32(0.01)


def test_rollout_deterministic_and_finite_small():
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=2048)
    a = ora.step(sc.params, sc.pos, sc.vel, 5)
    b = ora.step(sc.params, sc.pos, sc.vel, 5)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.all(np.isfinite(a[0]))
