"""Oracle density map (updateDensityMap.comp:93-147, image sized as
renderer.c:774-781) against a direct float32 restatement of the shader's
loop, on small cases (CPU)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_oracle, load_package

f32 = np.float32


def _hash(cx, cy, cz):
    h = (cx * 73856093 ^ cy * 19349663 ^ cz * 83492791) & 0xFFFFFFFF
    h ^= h >> 16
    h = (h * 0x7FEB352D) & 0xFFFFFFFF
    h ^= h >> 15
    h = (h * 0x846CA68B) & 0xFFFFFFFF
    h ^= h >> 16
    return h


def _shader_map(p, pos, sk, cs):
    """The shader's main() per voxel, every operation in float32."""
    n = pos.shape[0]
    lo = [f32(p.box_min[a]) for a in range(3)]
    hi = [f32(p.box_max[a]) for a in range(3)]
    h, cs = f32(p.h), f32(cs)
    m = [int(np.ceil(f32(hi[a] - lo[a]) / cs)) for a in range(3)]       # shader bound
    img = [int(np.ceil(np.float64(f32(f32(hi[a] - lo[a]) * f32(f32(1.0) / cs))))) for a in range(3)]
    vol = f32(2.0 * np.pi * float(p.h) ** 5 / 15.0) if p.volume <= 0 else f32(p.volume)
    start = {}
    end = {}
    for s in range(n):
        k = int(sk[s])
        start.setdefault(k, s)
        end[k] = s + 1

    def oob(v):
        return any(c < 0 for c in v) or any(v[a] > m[a] for a in range(3)) or all(v[a] == m[a] for a in range(3))

    out = np.zeros((img[2], img[1], img[0]), np.float32)
    for vz in range(img[2]):
        for vy in range(img[1]):
            for vx in range(img[0]):
                v = (vx, vy, vz)
                if oob(v):
                    continue
                ctr = [f32(lo[a] + f32(f32(f32(v[a]) + f32(0.5)) * cs)) for a in range(3)]
                if any(ctr[a] < lo[a] or ctr[a] > hi[a] for a in range(3)):
                    vc = (-1, -1, -1)
                else:
                    vc = tuple(int(np.floor(f32(f32(ctr[a] - lo[a]) / h))) for a in range(3))
                dens = f32(0.0)
                for dz in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dx in (-1, 0, 1):
                            c = (vc[0] + dx, vc[1] + dy, vc[2] + dz)
                            if oob(c):
                                continue
                            key = _hash(*c) & (n - 1)
                            if key not in start:
                                continue
                            for i in range(start[key], end[key]):
                                d = [f32(ctr[a] - pos[i, a]) for a in range(3)]
                                d2 = f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2]))
                                if d2 < f32(h * h):
                                    dist = np.sqrt(d2, dtype=np.float32)
                                    k = f32(0.0) if dist >= h else f32(f32(h - dist) * f32(h - dist))
                                    dens = f32(dens + f32(f32(p.particle_mass) * k))
                out[vz, vy, vx] = f32(dens / vol)
    return out


@pytest.mark.parametrize("n,cs_over_h", [(64, 1.0), (128, 0.7), (64, 1.6), (1, 1.0)])
def test_density_map_matches_shader_loop(n, cs_over_h):
    pfs, ora = load_package(), load_oracle()
    rng = np.random.default_rng(n)
    p = pfs.make_params(0.25, 1000.0, 200.0, 0.05, dt=1 / 120)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0.0, 1.0, (n, 3))
    k = ora.keys(p, pos)
    sk, perm = ora.sort(k)
    sp = pos[perm]
    cs = float(np.float32(0.25 * cs_over_h))
    got = ora.density_map(p, sp, sk, cs)
    want = _shader_map(p, sp, sk, cs)
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert got.shape == tuple(reversed(ora.density_map_dims(p, cs)))


def test_single_particle_value():
    """One particle at a voxel centre, n = 4 (distinct keys nearby): the
    centre voxel holds m h^2 / volume times the number of sampled cells whose
    key is the particle's."""
    pfs, ora = load_package(), load_oracle()
    p = pfs.make_params(0.1, 1000.0, 200.0, 0.05, dt=1 / 120)
    pos = np.zeros((4, 4), np.float32)
    pos[:, :3] = [[0.15, 0.25, 0.35], [0.95, 0.95, 0.95], [0.95, 0.05, 0.95], [0.05, 0.95, 0.05]]
    sk, perm = ora.sort(ora.keys(p, pos))
    got = ora.density_map(p, pos[perm], sk, 0.1)
    want = _shader_map(p, pos[perm], sk, 0.1)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert got[3, 2, 1] > 0.0


def test_density_map_matches_reference_shader():
    """Against the reference's own updateDensityMap.comp, executed on the CPU
    by oracle/glsl_ref.py (golden_map) on the state after one reference
    substep: bit-exact, every voxel, three cell sizes per case."""
    import os
    pfs, ora = load_package(), load_oracle()
    path = os.path.join(os.path.dirname(__file__), "golden", "glsl_density_map.npz")
    g = np.load(path)
    names = [str(x) for x in g["names"]]
    assert len(names) >= 3
    checked = 0
    for nm in names:
        h, mass, vol, *box = (float(x) for x in g[f"{nm}__scalars"])
        p = pfs.make_params(h, 1000.0, 200.0, 0.05)
        p.particle_mass = mass
        p.volume = vol
        for a in range(3):
            p.box_min[a] = box[a]
            p.box_max[a] = box[3 + a]
        pos, keys = g[f"{nm}__pos"], g[f"{nm}__keys"]
        for f in (1.0, 0.7, 1.6):
            cs = float(g[f"{nm}__cs{f}"][0])
            want = g[f"{nm}__map{f}"]
            got = ora.density_map(p, pos, keys, cs)
            assert got.shape == want.shape, (nm, f)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (nm, f)
            checked += 1
    assert checked == 3 * len(names)
