"""Oracle volumetric rendering (calculateLightVolume.comp, volumetricFluid.comp):
known answers of its sampler, light march and view march (CPU)."""
from __future__ import annotations

import ctypes

import numpy as np

from conftest import load_oracle, load_package

f32 = np.float32


def _params(pfs, box=(8.0, 4.0, 4.0), h=1.0):
    p = pfs.make_params(h, 1000.0, 200.0, 0.05)
    for a in range(3):
        p.box_min[a] = 0.0
        p.box_max[a] = box[a]
    return p


def test_texture_linear_field_and_clamp():
    ora = load_oracle()
    nx, ny, nz = 6, 5, 4
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    img = (x + 10 * y + 100 * z).astype(np.float32)
    dims = np.array([nx, ny, nz], np.int32)
    L = ora.lib()
    for uvw, want in ([(0.5 / nx, 0.5 / ny, 0.5 / nz), 0.0],          # texel centre (0,0,0)
                      [(2.5 / nx, 1.5 / ny, 3.5 / nz), 2 + 10 + 300],  # texel centre (2,1,3)
                      [(3.0 / nx, 1.5 / ny, 0.5 / nz), 2.5 + 10],      # halfway in x
                      [(-1.0, -1.0, -1.0), 0.0],                       # clamp to edge below
                      [(2.0, 2.0, 2.0), 5 + 40 + 300]):                # and above
        u = np.array(uvw, np.float32)
        got = L.pfso_texture3d(img.ctypes.data, dims.ctypes.data, u.ctypes.data)
        assert abs(got - want) < 1e-4, (uvw, got, want)


def test_light_volume_constant_density():
    """A constant density map c: each light voxel sums c * step over its march."""
    pfs, ora = load_package(), load_oracle()
    p = _params(pfs)
    dmap = np.full((8, 8, 16), 2.0, np.float32)
    sun = np.array([1.0, 0.0, 0.0], np.float32)
    lv = ora.light_volume(p, dmap, 1.0, sun)
    assert lv.shape == (4, 4, 8)
    # voxel x = 0: centre 0.5, box exit at 8 -> tFar + 1 = 8.5; t from 0 to 8 in steps of 1
    assert lv[0, 0, 0] == f32(2.0) * 9
    assert lv[0, 0, 7] == f32(2.0) * 2   # centre 7.5: t = 0, 1
    assert np.all(lv > 0)


def test_volumetric_empty_map_is_black():
    pfs, ora = load_package(), load_oracle()
    p = _params(pfs)
    dmap = np.zeros((8, 8, 16), np.float32)
    lv = np.zeros((4, 4, 8), np.float32)
    cam = np.array([4.0, -10.0, 2.0, 0, 1, 0, 1, 0, 0, 0, 0, 1], np.float32)
    img = ora.volumetric(p, dmap, lv, cam, 0.7, 0.1, (0.01, 0.01, 0.005), 16, 12)
    assert np.all(img[..., :3] == 0.0) and np.all(img[..., 3] == 1.0)


def test_volumetric_fog_brightens_centre_rays():
    pfs, ora = load_package(), load_oracle()
    p = _params(pfs)
    dmap = np.full((8, 8, 16), 50.0, np.float32)
    lv = np.zeros((4, 4, 8), np.float32)
    cam = np.array([4.0, -10.0, 2.0, 0, 1, 0, 1, 0, 0, 0, 0, 1], np.float32)
    tanf = ctypes.CDLL("libm.so.6").tanf
    tanf.restype, tanf.argtypes = ctypes.c_float, [ctypes.c_float]
    img = ora.volumetric(p, dmap, lv, cam, tanf(f32(0.5) * f32(0.9 * np.pi / 2)), 0.1,
                         (0.01, 0.01, 0.005), 32, 24)
    centre, corner = img[12, 16, :3], img[0, 0, :3]
    assert np.all(centre > 0.05) and np.all(corner == 0.0)   # the corner ray misses the box
