"""The oracle's render modes against fixtures from the reference's own
shaders: calculateLightVolume.comp, volumetricFluid.comp and properFluid.comp
translated to C++ by oracle/glsl_ref.py and dispatched as commands.c:437-467
does, on the density maps updateDensityMap.comp produced for the step cases
(tests/golden/glsl_render.npz, glsl_density_map.npz).

Both sides run on the host with the same libm, so light volumes and images
must agree bit for bit; tan(FOV / 2), which the shaders compute per pixel and
the oracle takes from its caller, comes from the same libm tanf.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import GOLDEN, load_oracle, load_package
from test_oracle_golden import _cases, _params_for

_REND = np.load(f"{GOLDEN}/glsl_render.npz")
_MAPS = np.load(f"{GOLDEN}/glsl_density_map.npz")
NAMES = [str(n) for n in _REND["names"]]


_LIBM = ctypes.CDLL("libm.so.6")
_LIBM.tanf.restype = ctypes.c_float
_LIBM.tanf.argtypes = [ctypes.c_float]


def _half_height(fov):
    return float(_LIBM.tanf(float(np.float32(np.float32(0.5) * np.float32(fov)))))


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name", NAMES)
def test_light_volume_and_image_match_reference_shaders(name):
    pfs, ora = load_package(), load_oracle()
    case = {c["name"]: c for c in _cases()}[name]
    p = _params_for(pfs, case)
    dmap = _MAPS[f"{name}__map1.0"]
    view = _REND[f"{name}__view"]
    cam, fov, step, light_step = view[:12], view[12], view[13], view[14]
    ext, sun = view[15:18], view[18:21]
    ref_lv = _REND[f"{name}__lvol"]
    ref_img = _REND[f"{name}__rgba"]

    lv = ora.light_volume(p, dmap, float(light_step), sun)
    assert lv.shape == ref_lv.shape
    assert np.array_equal(_bits(lv), _bits(ref_lv))

    half_height = _half_height(fov)
    h, w = ref_img.shape[:2]
    img = ora.volumetric(p, dmap, ref_lv, cam, half_height, float(step), ext, w, h)
    assert np.array_equal(_bits(img), _bits(ref_img))
    assert (ref_img[..., :3] > 0).any(-1).sum() > 50   # the fixture sees the fluid


@pytest.mark.parametrize("name", NAMES)
def test_refractive_image_matches_reference_shader(name):
    pfs, ora = load_package(), load_oracle()
    case = {c["name"]: c for c in _cases()}[name]
    p = _params_for(pfs, case)
    dmap = _MAPS[f"{name}__map1.0"]
    view = _REND[f"{name}__view"]
    cam, fov, step, light_step, ext = view[:12], view[12], view[13], view[14], view[15:18]
    thr, ior, nrefr = _REND[f"{name}__refr_args"]
    ref = _REND[f"{name}__refr"]
    h, w = ref.shape[:2]
    img = ora.refractive(p, dmap, cam, _half_height(fov), float(step), float(light_step), ext,
                         int(nrefr), float(thr), float(ior), w, h)
    assert np.array_equal(_bits(img), _bits(ref))
    assert len(np.unique(ref[..., 0])) > 50   # surfaces found, rays refracted and reflected


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("which", ["rgba", "refr"])
def test_fxaa_matches_reference_fragment_shader(name, which):
    """raymarchShader.frag run once per pixel (outNDC at the pixel centre) on
    the volumetric and refractive fixture images."""
    ora = load_oracle()
    src = _REND[f"{name}__{which}"]
    want = _REND[f"{name}__fxaa_{which}"]
    got = ora.fxaa(src)
    assert np.array_equal(_bits(got), _bits(want))
