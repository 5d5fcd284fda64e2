"""ctypes binding of the CPU oracle (oracle/libpfs_oracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
legs use this module as the checker / CPU baseline.  The product library does
not import it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfs_oracle.so")

_lib = None


class Consts(ctypes.Structure):
    _fields_ = [
        ("volume", ctypes.c_float),
        ("near_inv", ctypes.c_float),
        ("slope_scale", ctypes.c_float),
        ("near_slope_scale", ctypes.c_float),
        ("r2", ctypes.c_float),
        ("skip_d2", ctypes.c_float),
        ("margin_i", ctypes.c_float),
        ("mask", ctypes.c_uint32),
    ]


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib(params_type=None) -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    u32 = ctypes.c_uint32
    sig = {
        "pfso_derive": (None, [vp, u32, ctypes.POINTER(Consts)]),
        "pfso_cell_hash": (u32, [u32, u32, u32]),
        "pfso_cell_coord": (ctypes.c_int32, [ctypes.c_float, ctypes.c_float, ctypes.c_float]),
        "pfso_keys": (None, [vp, u32, vp, vp]),
        "pfso_sort": (None, [u32, vp, vp, vp]),
        "pfso_table": (None, [u32, vp, vp, vp]),
        "pfso_predict": (None, [vp, u32, vp, vp, vp, vp]),
        "pfso_density": (None, [vp, u32, vp, vp, vp, vp, vp]),
        "pfso_force": (None, [vp, u32, vp, vp, vp, vp, vp, vp, vp, vp]),
        "pfso_integrate": (None, [vp, u32, vp, vp, vp]),
        "pfso_color": (None, [vp, vp]),
        "pfso_substep": (ctypes.c_int, [vp, u32, vp, vp, vp, vp, vp, vp]),
        "pfso_step": (ctypes.c_int, [vp, u32, vp, vp, u32, vp, vp]),
        "pfso_subset_f64": (None, [vp, u32, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp]),
        "pfso_density_map_extent": (None, [vp, ctypes.c_float, vp, vp]),
        "pfso_density_map": (None, [vp, u32, vp, vp, vp, ctypes.c_float, vp]),
        "pfso_texture3d": (ctypes.c_float, [vp, vp, vp]),
        "pfso_light_volume": (None, [vp, vp, vp, ctypes.c_float, vp, vp, vp]),
        "pfso_volumetric": (None, [vp, vp, vp, vp, vp, vp, ctypes.c_float, ctypes.c_float, vp, u32,
                                   u32, vp]),
        "pfso_refractive": (None, [vp, vp, vp, vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, vp,
                                   ctypes.c_int32, ctypes.c_float, ctypes.c_float, u32, u32, vp]),
        "pfso_fxaa": (None, [vp, u32, u32, vp]),
        "pfso_splat_camera": (None, [vp, vp, vp, vp, vp, vp]),
        "pfso_splats": (None, [u32, vp, vp, vp, vp, vp, ctypes.c_float, u32, u32, vp, vp]),
        "pfso_splat_clip": (None, [vp, vp, vp, vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, vp]),
        "pfso_splat_shade": (None, [vp, ctypes.c_float, ctypes.c_float, vp]),
        "pfso_set_threads": (None, [ctypes.c_int]),
        "pfso_max_threads": (ctypes.c_int, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _pp(params) -> ctypes.c_void_p:
    return ctypes.cast(ctypes.pointer(params), ctypes.c_void_p)


def derive(params, n: int) -> Consts:
    c = Consts()
    lib().pfso_derive(_pp(params), n, ctypes.byref(c))
    return c


def cell_hash(cx: int, cy: int, cz: int) -> int:
    return int(lib().pfso_cell_hash(cx & 0xFFFFFFFF, cy & 0xFFFFFFFF, cz & 0xFFFFFFFF))


def keys(params, pos4: np.ndarray) -> np.ndarray:
    pos4 = np.ascontiguousarray(pos4, np.float32)
    out = np.empty(pos4.shape[0], np.uint32)
    lib().pfso_keys(_pp(params), pos4.shape[0], _p(pos4), _p(out))
    return out


def sort(k: np.ndarray):
    k = np.ascontiguousarray(k, np.uint32)
    n = k.shape[0]
    sk = np.empty(n, np.uint32)
    perm = np.empty(n, np.uint32)
    lib().pfso_sort(n, _p(k), _p(sk), _p(perm))
    return sk, perm


def table(sk: np.ndarray):
    sk = np.ascontiguousarray(sk, np.uint32)
    n = sk.shape[0]
    start = np.empty(n, np.int32)
    end = np.empty(n, np.int32)
    lib().pfso_table(n, _p(sk), _p(start), _p(end))
    return start, end


def density_map_dims(params, cell_size: float):
    """(nx, ny, nz) voxels of the density map: the reference's image extent."""
    img = np.empty(3, np.int32)
    bound = np.empty(3, np.int32)
    lib().pfso_density_map_extent(_pp(params), ctypes.c_float(cell_size), _p(img), _p(bound))
    return tuple(int(e) for e in img)


def density_map(params, pos4: np.ndarray, sorted_keys: np.ndarray, cell_size: float) -> np.ndarray:
    """Density map (updateDensityMap.comp) of positions stored in the order
    of the sort that produced sorted_keys; returns (nz, ny, nx) float32."""
    pos4 = np.ascontiguousarray(pos4, np.float32)
    n = pos4.shape[0]
    start, end = table(sorted_keys)
    nx, ny, nz = density_map_dims(params, cell_size)
    out = np.empty((nz, ny, nx), np.float32)
    lib().pfso_density_map(_pp(params), n, _p(pos4), _p(start), _p(end), ctypes.c_float(cell_size),
                           _p(out))
    return out


def light_volume_dims(params, light_step: float):
    """The light volume the reference allocates (renderer.c:812-819)."""
    f32 = np.float32
    inv = f32(f32(1.0) / f32(light_step))
    return tuple(int(np.ceil(np.float64(f32(f32(f32(params.box_max[a]) - f32(params.box_min[a])) * inv))))
                 for a in range(3))


def light_volume(params, dmap: np.ndarray, light_step: float, sun) -> np.ndarray:
    """calculateLightVolume over a density map (nz, ny, nx); returns (nz, ny, nx)."""
    dmap = np.ascontiguousarray(dmap, np.float32)
    dd = np.array(dmap.shape[::-1], np.int32)
    nx, ny, nz = light_volume_dims(params, light_step)
    ld = np.array([nx, ny, nz], np.int32)
    out = np.empty((nz, ny, nx), np.float32)
    sun = np.ascontiguousarray(sun, np.float32)
    lib().pfso_light_volume(_pp(params), _p(dmap), _p(dd), ctypes.c_float(light_step), _p(sun), _p(ld),
                            _p(out))
    return out


def refractive(params, dmap: np.ndarray, cam: np.ndarray, half_height: float, step: float,
               light_step: float, extinction, num_refractions: int, threshold: float, ior: float,
               width: int, height: int) -> np.ndarray:
    """properFluid image (height, width, 4) over a density map (nz, ny, nx)."""
    dmap = np.ascontiguousarray(dmap, np.float32)
    dd = np.array(dmap.shape[::-1], np.int32)
    cam = np.ascontiguousarray(cam, np.float32)
    ext = np.ascontiguousarray(extinction, np.float32)
    out = np.empty((height, width, 4), np.float32)
    lib().pfso_refractive(_pp(params), _p(dmap), _p(dd), _p(cam), ctypes.c_float(half_height),
                          ctypes.c_float(step), ctypes.c_float(light_step), _p(ext),
                          ctypes.c_int32(num_refractions), ctypes.c_float(threshold),
                          ctypes.c_float(ior), ctypes.c_uint32(width), ctypes.c_uint32(height),
                          _p(out))
    return out


def fxaa(img: np.ndarray) -> np.ndarray:
    """raymarchShader.frag's FXAA of a (height, width, 4) float32 image."""
    img = np.ascontiguousarray(img, np.float32)
    h, w = img.shape[:2]
    out = np.empty_like(img)
    lib().pfso_fxaa(_p(img), w, h, _p(out))
    return out


def splat_camera(model: np.ndarray, view: np.ndarray, proj: np.ndarray):
    """(mvp, right, up) from column-major 4x4 matrices (16 floats each)."""
    m = [np.ascontiguousarray(a, np.float32).reshape(16) for a in (model, view, proj)]
    mvp = np.empty(16, np.float32)
    right = np.empty(3, np.float32)
    up = np.empty(3, np.float32)
    lib().pfso_splat_camera(_p(m[0]), _p(m[1]), _p(m[2]), _p(mvp), _p(right), _p(up))
    return mvp, right, up


def splats(pos4: np.ndarray, color4: np.ndarray, model, view, proj, radius: float, width: int,
           height: int):
    """Point-splat raster (shader.vert / shader.frag) of particles in slot
    order: (rgba (height, width, 4), depth (height, width))."""
    pos4 = np.ascontiguousarray(pos4, np.float32)
    color4 = np.ascontiguousarray(color4, np.float32)
    mvp, right, up = splat_camera(model, view, proj)
    rgba = np.empty((height, width, 4), np.float32)
    depth = np.empty((height, width), np.float32)
    lib().pfso_splats(pos4.shape[0], _p(pos4), _p(color4), _p(mvp), _p(right), _p(up),
                      ctypes.c_float(radius), width, height, _p(rgba), _p(depth))
    return rgba, depth


def volumetric(params, dmap: np.ndarray, lvol: np.ndarray, cam: np.ndarray, half_height: float,
               step: float, extinction, width: int, height: int) -> np.ndarray:
    """volumetricFluid image (height, width, 4); cam = position, forward,
    right, up (12 floats); half_height = tan(FOV / 2) as the caller computes it."""
    dmap = np.ascontiguousarray(dmap, np.float32)
    lvol = np.ascontiguousarray(lvol, np.float32)
    dd = np.array(dmap.shape[::-1], np.int32)
    ld = np.array(lvol.shape[::-1], np.int32)
    cam = np.ascontiguousarray(cam, np.float32)
    ext = np.ascontiguousarray(extinction, np.float32)
    out = np.empty((height, width, 4), np.float32)
    lib().pfso_volumetric(_pp(params), _p(dmap), _p(dd), _p(lvol), _p(ld), _p(cam),
                          ctypes.c_float(half_height), ctypes.c_float(step), _p(ext), width, height,
                          _p(out))
    return out


def substep(params, pos4: np.ndarray, vel4: np.ndarray, trace: bool = False, ids=None,
            colors: bool = False):
    """One substep in place on copies; returns (pos, vel, density, trace|None, ids, rgba)."""
    from importlib import import_module  # noqa: F401
    pos = np.ascontiguousarray(pos4, np.float32).copy()
    vel = np.ascontiguousarray(vel4, np.float32).copy()
    n = pos.shape[0]
    dens = np.empty(n, np.float32)
    tr = None
    trp = None
    if trace:
        tr = {
            "keys_in": np.empty(n, np.uint32), "keys": np.empty(n, np.uint32),
            "perm": np.empty(n, np.uint32), "start": np.empty(n, np.int32),
            "end": np.empty(n, np.int32), "xp": np.empty((n, 4), np.float32),
            "vp": np.empty((n, 4), np.float32), "density": np.empty(n, np.float32),
            "near_density": np.empty(n, np.float32), "vel_force": np.empty((n, 4), np.float32),
        }
        trp = (ctypes.c_void_p * 10)(*[tr[k].ctypes.data for k in (
            "keys_in", "keys", "perm", "start", "end", "xp", "vp", "density", "near_density",
            "vel_force")])
    idsa = None if ids is None else np.ascontiguousarray(ids, np.uint32).copy()
    rgba = np.empty((n, 4), np.float32) if colors else None
    rc = lib().pfso_substep(_pp(params), n, _p(pos), _p(vel),
                            None if trp is None else ctypes.cast(trp, ctypes.c_void_p),
                            _p(dens), _p(idsa), _p(rgba))
    if rc != 0:
        raise RuntimeError(f"pfso_substep failed: {rc}")
    return pos, vel, dens, tr, idsa, rgba


def step(params, pos4: np.ndarray, vel4: np.ndarray, nsteps: int, ids=None):
    pos = np.ascontiguousarray(pos4, np.float32).copy()
    vel = np.ascontiguousarray(vel4, np.float32).copy()
    n = pos.shape[0]
    dens = np.empty(n, np.float32)
    idsa = None if ids is None else np.ascontiguousarray(ids, np.uint32).copy()
    rc = lib().pfso_step(_pp(params), n, _p(pos), _p(vel), nsteps, _p(dens), _p(idsa))
    if rc != 0:
        raise RuntimeError(f"pfso_step failed: {rc}")
    return pos, vel, dens, idsa


def subset_f64(params, xp4, vp4, vel4, start, end, subset):
    n = xp4.shape[0]
    subset = np.ascontiguousarray(subset, np.uint32)
    m = subset.shape[0]
    d = np.empty(m, np.float64)
    nd = np.empty(m, np.float64)
    v3 = np.empty((m, 3), np.float64)
    lib().pfso_subset_f64(_pp(params), n, _p(np.ascontiguousarray(xp4, np.float32)),
                          _p(np.ascontiguousarray(vp4, np.float32)),
                          _p(np.ascontiguousarray(vel4, np.float32)),
                          _p(np.ascontiguousarray(start, np.int32)),
                          _p(np.ascontiguousarray(end, np.int32)), m, _p(subset), _p(d), _p(nd),
                          _p(v3))
    return d, nd, v3


def set_threads(t: int) -> None:
    lib().pfso_set_threads(t)


def max_threads() -> int:
    return int(lib().pfso_max_threads())
