"""The oracle's volumetric render mode against fixtures from the reference's
own shaders: calculateLightVolume.comp and volumetricFluid.comp translated to
C++ by oracle/glsl_ref.py and dispatched as commands.c:437-453 does, on the
density maps updateDensityMap.comp produced for the step cases
(tests/golden/glsl_render.npz, glsl_density_map.npz).

Both sides run on the host with the same libm, so the light volume and the
image must agree bit for bit, tan(FOV / 2) included.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN, load_oracle, load_package
from test_oracle_golden import _cases, _params_for

_REND = np.load(f"{GOLDEN}/glsl_render.npz")
_MAPS = np.load(f"{GOLDEN}/glsl_density_map.npz")
NAMES = [str(n) for n in _REND["names"]]


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

    half_height = float(np.float32(math.tan(np.float32(np.float32(0.5) * fov))))
    h, w = ref_img.shape[:2]
    img = ora.volumetric(p, dmap, ref_lv, cam, half_height, float(step), ext, w, h)
    assert np.array_equal(_bits(img), _bits(ref_img))
    assert (ref_img[..., :3] > 0).any(-1).sum() > 50   # the fixture sees the fluid
