"""Python mirror of the pfs C ABI (include/pfs.h) over ctypes.

The product is libpfs.so (CUDA, sm_100a) beside this file; this module only
binds it.  There is no CPU fallback: if the library is missing or no GPU is
present, the calls fail loudly with PfsError.

The reference (mojofill/particle-fluid-simulation) exposes no library API;
its world step is the substep block of recordCommands()
(src/renderer/commands.c:193-402).  ``World`` mirrors the C entry points that
replace it: ``World(params, pos4, vel4)`` / ``step`` / ``sync`` / ``read`` /
``write`` / ``close``.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfs.so")

PFS_OK = 0
PFS_EINVAL = -1
PFS_ENOMEM = -2
PFS_ECUDA = -3
PFS_ETIMEDOUT = -4
PFS_ENODEV = -5
PFS_EDEVICE = -6
PFS_ERANGE = -7
PFS_EBUDGET = -8
PFS_ENOTFOUND = -9

PFS_MAX_PARTICLES = 1 << 24
PFS_FP32 = 0
PFS_FP16_CELL = 1
PFS_FP32_FAST = 2
PFS_FLAG_COLORS = 1
PFS_FLAG_IDS = 2

STAGES = ("sort", "reorder", "density", "force", "integrate")


class PfsError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {status_name(status)} ({status})")


class Params(ctypes.Structure):
    """pfs_params (include/pfs.h)."""

    _fields_ = [
        ("h", ctypes.c_float),
        ("target_density", ctypes.c_float),
        ("pressure_multiplier", ctypes.c_float),
        ("near_pressure_multiplier", ctypes.c_float),
        ("viscosity", ctypes.c_float),
        ("particle_mass", ctypes.c_float),
        ("gravity", ctypes.c_float * 3),
        ("dt", ctypes.c_float),
        ("box_min", ctypes.c_float * 3),
        ("box_max", ctypes.c_float * 3),
        ("margin_predict", ctypes.c_float),
        ("margin_integrate", ctypes.c_float),
        ("restitution", ctypes.c_float * 6),
        ("volume", ctypes.c_float),
        ("substeps", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]

    def copy(self) -> "Params":
        out = Params()
        ctypes.memmove(ctypes.byref(out), ctypes.byref(self), ctypes.sizeof(Params))
        return out

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d


class StageTimes(ctypes.Structure):
    _fields_ = [
        ("ms_total", ctypes.c_double * 5),
        ("launches", ctypes.c_uint64 * 5),
        ("substeps", ctypes.c_uint64),
    ]


class DebugSubstep(ctypes.Structure):
    _fields_ = [
        ("keys_in", ctypes.c_void_p),
        ("keys", ctypes.c_void_p),
        ("perm", ctypes.c_void_p),
        ("start", ctypes.c_void_p),
        ("end", ctypes.c_void_p),
        ("xp", ctypes.c_void_p),
        ("vp", ctypes.c_void_p),
        ("density", ctypes.c_void_p),
        ("near_density", ctypes.c_void_p),
        ("vel_force", ctypes.c_void_p),
    ]


PFS_SHAPE_SIMPLE, PFS_SHAPE_SLAB, PFS_SHAPE_LIST, PFS_SHAPE_FLAT, PFS_SHAPE_STAGED = 0, 1, 2, 3, 4
PFS_SEARCH_AUTO, PFS_SEARCH_TABLE, PFS_SEARCH_GRID = -1, 0, 1
SHAPE_NAMES = {0: "simple", 1: "slab", 2: "list", 3: "flat", 4: "staged"}
SEARCH_NAMES = {-1: "auto", 0: "table", 1: "grid"}


class VolumeView(ctypes.Structure):
    """pfs_volume_view: camera and the reference's volumetric render constants."""
    _fields_ = [
        ("position", ctypes.c_float * 3), ("forward", ctypes.c_float * 3),
        ("right", ctypes.c_float * 3), ("up", ctypes.c_float * 3),
        ("fov", ctypes.c_float), ("density_cell_size", ctypes.c_float),
        ("step_size", ctypes.c_float), ("light_step_size", ctypes.c_float),
        ("extinction", ctypes.c_float * 3), ("dir_to_sun", ctypes.c_float * 3),
    ]


def volume_view(position, forward, right, up, fov=0.9 * np.pi / 2, density_cell_size=0.5,
                step_size=0.01, light_step_size=1.0, extinction=(0.01, 0.01, 0.005),
                dir_to_sun=(0.75, -0.25, 0.5)) -> VolumeView:
    """A view with the reference's defaults (main.c:14,23-25,389-394); the
    sun direction is normalised here as glm_normalize does there."""
    v = VolumeView()
    for name, val in (("position", position), ("forward", forward), ("right", right), ("up", up),
                      ("extinction", extinction)):
        arr = getattr(v, name)
        for a in range(3):
            arr[a] = float(val[a])
    s = np.asarray(dir_to_sun, np.float32)
    s = s / np.float32(np.sqrt(np.float32(np.dot(s, s))))
    for a in range(3):
        v.dir_to_sun[a] = float(s[a])
    v.fov, v.density_cell_size = float(np.float32(fov)), float(density_cell_size)
    v.step_size, v.light_step_size = float(step_size), float(light_step_size)
    return v


class Refraction(ctypes.Structure):
    _fields_ = [
        ("num_refractions", ctypes.c_int32),
        ("surface_density_threshold", ctypes.c_float),
        ("index_of_refraction", ctypes.c_float),
        ("reserved", ctypes.c_float),
    ]


def refraction(num_refractions=3, surface_density_threshold=0.75, index_of_refraction=1.333) -> Refraction:
    """Refractive-mode settings; defaults are the reference's (main.c:27-29)."""
    r = Refraction()
    r.num_refractions = int(num_refractions)
    r.surface_density_threshold = float(surface_density_threshold)
    r.index_of_refraction = float(index_of_refraction)
    return r


class SplatView(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_float * 16),
        ("view", ctypes.c_float * 16),
        ("proj", ctypes.c_float * 16),
        ("particle_radius", ctypes.c_float),
        ("reserved", ctypes.c_float * 3),
    ]


def look_at(eye, center, up=(0.0, 0.0, 1.0)) -> np.ndarray:
    """Right-handed view matrix, column-major 16 floats (the published
    lookAt formula cglm's glm_lookat implements; main.c:45)."""
    f32 = np.float32
    eye, center, up = (np.asarray(a, f32) for a in (eye, center, up))
    f = center - eye
    f = f / f32(np.sqrt(f32(np.dot(f, f))))
    s = np.cross(f, up).astype(f32)
    s = s / f32(np.sqrt(f32(np.dot(s, s))))
    u = np.cross(s, f).astype(f32)
    m = np.zeros((4, 4), f32)              # m[column][row]
    m[0, :3] = (s[0], u[0], -f[0])
    m[1, :3] = (s[1], u[1], -f[1])
    m[2, :3] = (s[2], u[2], -f[2])
    m[3, :3] = (-f32(np.dot(s, eye)), -f32(np.dot(u, eye)), f32(np.dot(f, eye)))
    m[3, 3] = 1.0
    return m.reshape(16)


def perspective(fovy: float, aspect: float, near: float = 0.1, far: float = 10000.0,
                flip_y: bool = True) -> np.ndarray:
    """Right-handed perspective with clip z in [-w, w] (glm_perspective's
    published formula), y flipped as main.c:51 does for Vulkan."""
    f32 = np.float32
    f = f32(1.0) / f32(np.tan(f32(fovy) * f32(0.5)))
    fn = f32(1.0) / f32(f32(near) - f32(far))
    m = np.zeros((4, 4), f32)
    m[0, 0] = f / f32(aspect)
    m[1, 1] = -f if flip_y else f
    m[2, 2] = f32(f32(near) + f32(far)) * fn
    m[2, 3] = -1.0
    m[3, 2] = f32(f32(2.0) * f32(near)) * f32(far) * fn
    return m.reshape(16)


def splat_view(position, forward, width: int, height: int, particle_radius: float,
               fov: float = 0.9 * np.pi / 2, up=(0.0, 0.0, 1.0), near: float = 0.1,
               far: float = 10000.0) -> SplatView:
    """The UBO matrices updateUniforms (main.c:37-51) builds for a camera:
    model identity, lookat(position, position + forward, up), perspective."""
    v = SplatView()
    model = np.eye(4, dtype=np.float32).reshape(16)
    view = look_at(position, np.asarray(position, np.float32) + np.asarray(forward, np.float32), up)
    proj = perspective(fov, width / float(height), near, far)
    for k in range(16):
        v.model[k], v.view[k], v.proj[k] = float(model[k]), float(view[k]), float(proj[k])
    v.particle_radius = float(particle_radius)
    return v


class TuneResult(ctypes.Structure):
    _fields_ = [
        ("candidates", ctypes.c_int32),
        ("chosen", ctypes.c_int32),
        ("shape", ctypes.c_int32 * 12),
        ("search", ctypes.c_int32 * 12),
        ("ms_per_step", ctypes.c_float * 12),
    ]

    def as_dict(self) -> dict:
        trials = [{"shape": SHAPE_NAMES[self.shape[k]], "search": SEARCH_NAMES[self.search[k]],
                   "ms_per_step": float(self.ms_per_step[k])} for k in range(self.candidates)]
        return {"trials": trials, "chosen": trials[self.chosen] if self.chosen >= 0 else None}


class BatchInfo(ctypes.Structure):
    _fields_ = [
        ("particles", ctypes.c_uint32),
        ("scenes", ctypes.c_uint32),
        ("max_particles", ctypes.c_uint32),
        ("max_scenes", ctypes.c_uint32),
        ("device_bytes", ctypes.c_uint64),
        ("launches_per_substep", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libpfs.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PfsError(PFS_ENODEV, f"libpfs.so not built at {LIB_PATH} (run __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    u32 = ctypes.c_uint32
    sig = {
        "pfs_params_reference_default": (None, [P(Params)]),
        "pfs_params_validate": (ctypes.c_int, [P(Params)]),
        "pfs_strerror": (ctypes.c_char_p, [ctypes.c_int]),
        "pfs_version": (ctypes.c_int, []),
        "pfs_world_create": (ctypes.c_int, [P(Params), u32, vp, vp, P(vp)]),
        "pfs_world_set_params": (ctypes.c_int, [vp, P(Params)]),
        "pfs_world_step": (ctypes.c_int, [vp, u32]),
        "pfs_world_sync": (ctypes.c_int, [vp, ctypes.c_uint64]),
        "pfs_world_read": (ctypes.c_int, [vp, vp, vp, vp, vp, vp]),
        "pfs_world_write": (ctypes.c_int, [vp, vp, vp]),
        "pfs_world_destroy": (ctypes.c_int, [vp]),
        "pfs_world_read_colors": (ctypes.c_int, [vp, vp]),
        "pfs_world_read_ids": (ctypes.c_int, [vp, vp]),
        "pfs_world_size": (u32, [vp]),
        "pfs_world_stream": (vp, [vp]),
        "pfs_world_device_state": (ctypes.c_int, [vp, P(vp), P(vp)]),
        "pfs_world_profile": (ctypes.c_int, [vp, ctypes.c_int]),
        "pfs_world_stage_times": (ctypes.c_int, [vp, P(StageTimes)]),
        "pfs_world_launches_per_substep": (ctypes.c_int, [vp]),
        "pfs_world_debug_substep": (ctypes.c_int, [vp, P(DebugSubstep)]),
        "pfs_world_device_error": (ctypes.c_int, [vp, P(u32)]),
        "pfs_sort_keys_static": (ctypes.c_int, [vp, u32, u32, vp, vp, vp]),
        "pfs_sort_static_status": (ctypes.c_int, [vp]),
        "pfs_world_density_map_dims": (ctypes.c_int, [vp, ctypes.c_float, vp]),
        "pfs_world_set_shape": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32]),
        "pfs_world_shape_available": (ctypes.c_int, [vp, ctypes.c_int32]),
        "pfs_world_light_volume_dims": (ctypes.c_int, [vp, ctypes.c_float, vp]),
        "pfs_world_render_volumetric": (ctypes.c_int, [vp, P(VolumeView), u32, u32, vp, vp]),
        "pfs_world_render_refractive": (ctypes.c_int, [vp, P(VolumeView), P(Refraction), u32, u32, vp]),
        "pfs_world_render_splats": (ctypes.c_int, [vp, P(SplatView), u32, u32, vp, vp]),
        "pfs_world_run_pipelined": (ctypes.c_int, [vp, u32, vp, vp, vp, vp, u32]),
        "pfs_world_fxaa": (ctypes.c_int, [vp, vp, u32, u32, vp]),
        "pfs_world_autotune": (ctypes.c_int, [vp, u32, P(TuneResult)]),
        "pfs_batch_set_shape": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32]),
        "pfs_batch_autotune": (ctypes.c_int, [vp, u32, P(TuneResult)]),
        "pfs_world_density_map": (ctypes.c_int, [vp, ctypes.c_float, vp]),
        "pfs_batch_create": (ctypes.c_int, [u32, u32, ctypes.c_int32, ctypes.c_int32, P(vp)]),
        "pfs_batch_bytes": (ctypes.c_uint64, [u32, u32, ctypes.c_int32]),
        "pfs_batch_add_scene": (ctypes.c_int, [vp, P(Params), u32, vp, vp, P(ctypes.c_int32)]),
        "pfs_batch_remove_scene": (ctypes.c_int, [vp, ctypes.c_int32]),
        "pfs_batch_step": (ctypes.c_int, [vp, u32]),
        "pfs_batch_sync": (ctypes.c_int, [vp, ctypes.c_uint64]),
        "pfs_batch_read_scene": (ctypes.c_int, [vp, ctypes.c_int32, vp, vp, vp]),
        "pfs_batch_write_scene": (ctypes.c_int, [vp, ctypes.c_int32, vp, vp]),
        "pfs_batch_info_get": (ctypes.c_int, [vp, P(BatchInfo)]),
        "pfs_batch_set_feed": (ctypes.c_int, [vp, ctypes.c_int]),
        "pfs_batch_stream": (vp, [vp]),
        "pfs_batch_destroy": (ctypes.c_int, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def status_name(status: int) -> str:
    names = {
        0: "PFS_OK", -1: "PFS_EINVAL", -2: "PFS_ENOMEM", -3: "PFS_ECUDA", -4: "PFS_ETIMEDOUT",
        -5: "PFS_ENODEV", -6: "PFS_EDEVICE", -7: "PFS_ERANGE", -8: "PFS_EBUDGET",
        -9: "PFS_ENOTFOUND",
    }
    return names.get(status, "unknown")


def check(status: int, what: str) -> None:
    if status != PFS_OK:
        raise PfsError(status, what)


def reference_default() -> Params:
    """The reference's compile-time parameters (src/main.c:11-30)."""
    p = Params()
    lib().pfs_params_reference_default(ctypes.byref(p))
    return p


def make_params(h: float, target_density: float, pressure_multiplier: float, viscosity: float,
                gravity=(0.0, -9.81, 0.0), dt: float = 1.0 / 120.0, substeps: int = 1,
                box_min=(0.0, 0.0, 0.0), box_max=(1.0, 1.0, 1.0), damping: float = 0.5,
                particle_mass: float = 1.0, near_pressure_multiplier: float = 0.0,
                margin_predict: float = 0.0, margin_integrate: float = 0.0,
                precision: int = PFS_FP32, flags: int = 0) -> Params:
    """Parameter set in the vocabulary of the reference's world step.

    dt is the per-step dt; the per-substep dt is dt / substeps, as
    updateUniforms() computes it (src/main.c:57).  damping is the velocity
    factor after every wall hit (restitution on all six walls)."""
    p = Params()
    p.h = h
    p.target_density = target_density
    p.pressure_multiplier = pressure_multiplier
    p.near_pressure_multiplier = near_pressure_multiplier
    p.viscosity = viscosity
    p.particle_mass = particle_mass
    for a in range(3):
        p.gravity[a] = gravity[a]
        p.box_min[a] = box_min[a]
        p.box_max[a] = box_max[a]
    p.dt = np.float32(np.float32(dt) / np.float32(substeps))
    p.margin_predict = margin_predict
    p.margin_integrate = margin_integrate
    for i in range(6):
        p.restitution[i] = damping
    p.volume = 0.0
    p.substeps = substeps
    p.precision = precision
    p.flags = flags
    return p


def _f4(a: Optional[np.ndarray], n: Optional[int] = None) -> Optional[np.ndarray]:
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] != 4:
        raise ValueError("expected an (n, 4) float32 array")
    if n is not None and a.shape[0] != n:
        raise ValueError(f"expected {n} rows, got {a.shape[0]}")
    return a


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class World:
    """One simulated scene: device state owned by libpfs, one CUDA stream."""

    def __init__(self, params: Params, pos4: np.ndarray, vel4: Optional[np.ndarray] = None):
        pos4 = _f4(pos4)
        n = pos4.shape[0]
        vel4 = _f4(vel4, n)
        self.n = n
        self.params = params.copy()
        h = ctypes.c_void_p()
        check(lib().pfs_world_create(ctypes.byref(self.params), n, _ptr(pos4), _ptr(vel4),
                                     ctypes.byref(h)), "pfs_world_create")
        self._h = h

    @property
    def handle(self) -> ctypes.c_void_p:
        if self._h is None:
            raise PfsError(PFS_EINVAL, "world closed")
        return self._h

    def set_params(self, params: Params) -> None:
        check(lib().pfs_world_set_params(self.handle, ctypes.byref(params)), "pfs_world_set_params")
        self.params = params.copy()

    def step(self, nsteps: int = 1) -> None:
        check(lib().pfs_world_step(self.handle, nsteps), "pfs_world_step")

    def sync(self, timeout_ns: int = 0) -> None:
        check(lib().pfs_world_sync(self.handle, timeout_ns), "pfs_world_sync")

    def read(self, pos=True, vel=True, density=False, keys=False, perm=False) -> dict:
        n = self.n
        out = {}
        if pos:
            out["pos"] = np.empty((n, 4), np.float32)
        if vel:
            out["vel"] = np.empty((n, 4), np.float32)
        if density:
            out["density"] = np.empty(n, np.float32)
        if keys:
            out["keys"] = np.empty(n, np.uint32)
        if perm:
            out["perm"] = np.empty(n, np.uint32)
        check(lib().pfs_world_read(self.handle, _ptr(out.get("pos")), _ptr(out.get("vel")),
                                   _ptr(out.get("density")), _ptr(out.get("keys")),
                                   _ptr(out.get("perm"))), "pfs_world_read")
        return out

    def read_into(self, pos4: Optional[np.ndarray], vel4: Optional[np.ndarray]) -> None:
        check(lib().pfs_world_read(self.handle, _ptr(pos4), _ptr(vel4), None, None, None),
              "pfs_world_read")

    def set_shape(self, shape: int, search: int = PFS_SEARCH_AUTO) -> None:
        """Kernel shape (PFS_SHAPE_*) and neighbour search (PFS_SEARCH_*); all
        combinations give the same results."""
        check(lib().pfs_world_set_shape(self.handle, shape, search), "pfs_world_set_shape")

    def staged_available(self) -> bool:
        """Whether the staged shape can run on this world."""
        return bool(lib().pfs_world_shape_available(self.handle, PFS_SHAPE_STAGED))

    def autotune(self, trial_steps: int = 2) -> dict:
        """Time every shape and search over trial_steps single steps, each
        from this world's state (the fastest counts), keep the fastest
        candidate, restore the state (results are unchanged)."""
        r = TuneResult()
        check(lib().pfs_world_autotune(self.handle, trial_steps, ctypes.byref(r)),
              "pfs_world_autotune")
        return r.as_dict()

    def density_map(self, cell_size: float, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Density map of the current state (the reference's
        updateDensityMap.comp): float32 array (nz, ny, nx)."""
        dims = np.empty(3, np.uint32)
        check(lib().pfs_world_density_map_dims(self.handle, ctypes.c_float(cell_size), _ptr(dims)),
              "pfs_world_density_map_dims")
        nx, ny, nz = (int(d) for d in dims)
        if out is None:
            out = np.empty((nz, ny, nx), np.float32)
        check(lib().pfs_world_density_map(self.handle, ctypes.c_float(cell_size), _ptr(out)),
              "pfs_world_density_map")
        return out

    def render_volumetric(self, view: VolumeView, width: int, height: int,
                          with_light_volume: bool = False):
        """The reference's volumetric render mode, headless: (height, width, 4)
        float32 RGBA, and the light volume (nz, ny, nx) when asked."""
        rgba = np.empty((height, width, 4), np.float32)
        lv = None
        if with_light_volume:
            dims = np.empty(3, np.uint32)
            check(lib().pfs_world_light_volume_dims(self.handle, ctypes.c_float(view.light_step_size),
                                                    _ptr(dims)), "pfs_world_light_volume_dims")
            lv = np.empty((int(dims[2]), int(dims[1]), int(dims[0])), np.float32)
        check(lib().pfs_world_render_volumetric(self.handle, ctypes.byref(view), width, height,
                                                _ptr(rgba), _ptr(lv)), "pfs_world_render_volumetric")
        return (rgba, lv) if with_light_volume else rgba

    def render_refractive(self, view: VolumeView, refr: "Refraction", width: int, height: int):
        """The reference's refractive render mode, headless: (height, width, 4)
        float32 RGBA."""
        rgba = np.empty((height, width, 4), np.float32)
        check(lib().pfs_world_render_refractive(self.handle, ctypes.byref(view), ctypes.byref(refr),
                                                width, height, _ptr(rgba)), "pfs_world_render_refractive")
        return rgba

    def render_refractive_ptr(self, view: VolumeView, refr: "Refraction", width: int, height: int,
                              ptr: int) -> None:
        check(lib().pfs_world_render_refractive(self.handle, ctypes.byref(view), ctypes.byref(refr),
                                                width, height, ctypes.c_void_p(ptr)),
              "pfs_world_render_refractive")

    def run_pipelined_ptrs(self, pos_in, vel_in, pos_out, vel_out, steps_each: int = 1) -> None:
        """pfs_world_run_pipelined over lists of buffer addresses (host or
        device; vel lists may be None, entries 0)."""
        count = len(pos_in)
        if len(pos_out) != count or (vel_in is not None and len(vel_in) != count) or \
                (vel_out is not None and len(vel_out) != count):
            raise ValueError("input and output lists differ in length")
        arr = lambda xs: (ctypes.c_void_p * count)(*[ctypes.c_void_p(int(x)) if x else None for x in xs])
        check(lib().pfs_world_run_pipelined(self.handle, count, arr(pos_in),
                                            arr(vel_in) if vel_in is not None else None, arr(pos_out),
                                            arr(vel_out) if vel_out is not None else None, steps_each),
              "pfs_world_run_pipelined")

    def run_pipelined(self, inputs, steps_each: int = 1, velocities: bool = True):
        """For each (pos4, vel4) in inputs: write, step steps_each, read back;
        copies overlap the steps.  Returns [(pos4, vel4 or None)]."""
        ins = [(_f4(p, self.n), _f4(v, self.n) if v is not None else None) for p, v in inputs]
        outs = [(np.empty((self.n, 4), np.float32), np.empty((self.n, 4), np.float32) if velocities else None)
                for _ in ins]
        self.run_pipelined_ptrs([p.ctypes.data for p, _ in ins],
                                [v.ctypes.data if v is not None else 0 for _, v in ins],
                                [p.ctypes.data for p, _ in outs],
                                [v.ctypes.data for _, v in outs] if velocities else None, steps_each)
        return outs

    def render_splats(self, view: SplatView, width: int, height: int, with_depth: bool = False):
        """The reference's rasterised point splats, headless: (height, width, 4)
        float32 RGBA (and the depth buffer when asked)."""
        rgba = np.empty((height, width, 4), np.float32)
        depth = np.empty((height, width), np.float32) if with_depth else None
        check(lib().pfs_world_render_splats(self.handle, ctypes.byref(view), width, height, _ptr(rgba),
                                            _ptr(depth)), "pfs_world_render_splats")
        return (rgba, depth) if with_depth else rgba

    def render_splats_ptr(self, view: SplatView, width: int, height: int, rgba_ptr: int,
                          depth_ptr: int = 0) -> None:
        check(lib().pfs_world_render_splats(self.handle, ctypes.byref(view), width, height,
                                            ctypes.c_void_p(rgba_ptr),
                                            ctypes.c_void_p(depth_ptr) if depth_ptr else None),
              "pfs_world_render_splats")

    def fxaa(self, rgba: np.ndarray) -> np.ndarray:
        """raymarchShader.frag's FXAA of a (height, width, 4) float32 image."""
        rgba = np.ascontiguousarray(rgba, np.float32)
        h, w = rgba.shape[:2]
        out = np.empty_like(rgba)
        check(lib().pfs_world_fxaa(self.handle, _ptr(rgba), w, h, _ptr(out)), "pfs_world_fxaa")
        return out

    def fxaa_ptr(self, in_ptr: int, width: int, height: int, out_ptr: int) -> None:
        check(lib().pfs_world_fxaa(self.handle, ctypes.c_void_p(in_ptr), width, height,
                                   ctypes.c_void_p(out_ptr)), "pfs_world_fxaa")

    def render_volumetric_ptr(self, view: VolumeView, width: int, height: int, ptr: int) -> None:
        check(lib().pfs_world_render_volumetric(self.handle, ctypes.byref(view), width, height,
                                                ctypes.c_void_p(ptr), None),
              "pfs_world_render_volumetric")

    def density_map_ptr(self, cell_size: float, ptr: int) -> None:
        """Density map into caller-owned memory (host or device pointer)."""
        check(lib().pfs_world_density_map(self.handle, ctypes.c_float(cell_size),
                                          ctypes.c_void_p(ptr)), "pfs_world_density_map")

    def read_colors(self) -> np.ndarray:
        out = np.empty((self.n, 4), np.float32)
        check(lib().pfs_world_read_colors(self.handle, _ptr(out)), "pfs_world_read_colors")
        return out

    def read_ids(self) -> np.ndarray:
        out = np.empty(self.n, np.uint32)
        check(lib().pfs_world_read_ids(self.handle, _ptr(out)), "pfs_world_read_ids")
        return out

    def write(self, pos4: np.ndarray, vel4: Optional[np.ndarray] = None) -> None:
        pos4 = _f4(pos4, self.n)
        vel4 = _f4(vel4, self.n)
        check(lib().pfs_world_write(self.handle, _ptr(pos4), _ptr(vel4)), "pfs_world_write")

    def write_ptr(self, pos_ptr: int, vel_ptr: int) -> None:
        """Write from raw host pointers (pinned buffers owned by the caller)."""
        check(lib().pfs_world_write(self.handle, ctypes.c_void_p(pos_ptr), ctypes.c_void_p(vel_ptr)),
              "pfs_world_write")

    def read_ptr(self, pos_ptr: int, vel_ptr: int) -> None:
        check(lib().pfs_world_read(self.handle, ctypes.c_void_p(pos_ptr), ctypes.c_void_p(vel_ptr),
                                   None, None, None), "pfs_world_read")

    @property
    def stream(self) -> int:
        return lib().pfs_world_stream(self.handle) or 0

    def device_state(self):
        p, v = ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().pfs_world_device_state(self.handle, ctypes.byref(p), ctypes.byref(v)),
              "pfs_world_device_state")
        return p.value, v.value

    def profile(self, enable: bool) -> None:
        check(lib().pfs_world_profile(self.handle, int(enable)), "pfs_world_profile")

    def stage_times(self) -> dict:
        t = StageTimes()
        check(lib().pfs_world_stage_times(self.handle, ctypes.byref(t)), "pfs_world_stage_times")
        return {
            "substeps": int(t.substeps),
            "ms_total": {s: float(t.ms_total[i]) for i, s in enumerate(STAGES)},
            "launches": {s: int(t.launches[i]) for i, s in enumerate(STAGES)},
        }

    def launches_per_substep(self) -> int:
        return int(lib().pfs_world_launches_per_substep(self.handle))

    def debug_substep(self) -> dict:
        n = self.n
        out = {
            "keys_in": np.empty(n, np.uint32), "keys": np.empty(n, np.uint32),
            "perm": np.empty(n, np.uint32), "start": np.empty(n, np.int32),
            "end": np.empty(n, np.int32), "xp": np.empty((n, 4), np.float32),
            "vp": np.empty((n, 4), np.float32), "density": np.empty(n, np.float32),
            "near_density": np.empty(n, np.float32), "vel_force": np.empty((n, 4), np.float32),
        }
        d = DebugSubstep(**{k: v.ctypes.data for k, v in out.items()})
        check(lib().pfs_world_debug_substep(self.handle, ctypes.byref(d)), "pfs_world_debug_substep")
        return out

    def device_error(self) -> int:
        w = ctypes.c_uint32()
        check(lib().pfs_world_device_error(self.handle, ctypes.byref(w)), "pfs_world_device_error")
        return int(w.value)

    def close(self) -> None:
        if self._h is not None:
            lib().pfs_world_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent scenes stepped together (pfs_batch_* in include/pfs.h).

    Each scene's results are bit-identical to a World holding it alone; the
    batch shares one sort and one launch per stage across all scenes."""

    def __init__(self, max_particles: int, max_scenes: int, precision: int = PFS_FP32,
                 substeps: int = 1):
        h = ctypes.c_void_p()
        check(lib().pfs_batch_create(max_particles, max_scenes, precision, substeps,
                                     ctypes.byref(h)), "pfs_batch_create")
        self._h = h
        self.sizes = {}

    @staticmethod
    def bytes_for(max_particles: int, max_scenes: int, precision: int = PFS_FP32) -> int:
        return int(lib().pfs_batch_bytes(max_particles, max_scenes, precision))

    @property
    def handle(self):
        if self._h is None:
            raise PfsError(PFS_EINVAL, "batch closed")
        return self._h

    def add(self, params: Params, pos4: np.ndarray, vel4: Optional[np.ndarray] = None) -> int:
        pos4 = _f4(pos4)
        vel4 = _f4(vel4, pos4.shape[0])
        sid = ctypes.c_int32()
        p = params.copy()
        check(lib().pfs_batch_add_scene(self.handle, ctypes.byref(p), pos4.shape[0], _ptr(pos4),
                                        _ptr(vel4), ctypes.byref(sid)), "pfs_batch_add_scene")
        self.sizes[sid.value] = pos4.shape[0]
        return sid.value

    def add_ptr(self, params: Params, n: int, pos_ptr: int, vel_ptr: int) -> int:
        sid = ctypes.c_int32()
        p = params.copy()
        check(lib().pfs_batch_add_scene(self.handle, ctypes.byref(p), n, ctypes.c_void_p(pos_ptr),
                                        ctypes.c_void_p(vel_ptr), ctypes.byref(sid)),
              "pfs_batch_add_scene")
        self.sizes[sid.value] = n
        return sid.value

    def remove(self, sid: int) -> None:
        check(lib().pfs_batch_remove_scene(self.handle, sid), "pfs_batch_remove_scene")
        self.sizes.pop(sid, None)

    def step(self, nsteps: int = 1) -> None:
        check(lib().pfs_batch_step(self.handle, nsteps), "pfs_batch_step")

    def sync(self, timeout_ns: int = 0) -> None:
        check(lib().pfs_batch_sync(self.handle, timeout_ns), "pfs_batch_sync")

    def set_shape(self, shape: int, search: int = PFS_SEARCH_AUTO) -> None:
        check(lib().pfs_batch_set_shape(self.handle, shape, search), "pfs_batch_set_shape")

    def autotune(self, trial_steps: int = 2) -> dict:
        """Time each shape with each scene's own search and with the table scan
        everywhere, keep the fastest, restore the scenes' states."""
        r = TuneResult()
        check(lib().pfs_batch_autotune(self.handle, trial_steps, ctypes.byref(r)),
              "pfs_batch_autotune")
        return r.as_dict()

    def set_feed(self, enable: bool) -> None:
        check(lib().pfs_batch_set_feed(self.handle, int(enable)), "pfs_batch_set_feed")

    def read(self, sid: int, density: bool = False) -> dict:
        n = self.sizes[sid]
        out = {"pos": np.empty((n, 4), np.float32), "vel": np.empty((n, 4), np.float32)}
        if density:
            out["density"] = np.empty(n, np.float32)
        check(lib().pfs_batch_read_scene(self.handle, sid, _ptr(out["pos"]), _ptr(out["vel"]),
                                         _ptr(out.get("density"))), "pfs_batch_read_scene")
        return out

    def read_ptr(self, sid: int, pos_ptr: int, vel_ptr: int) -> None:
        check(lib().pfs_batch_read_scene(self.handle, sid, ctypes.c_void_p(pos_ptr),
                                         ctypes.c_void_p(vel_ptr), None), "pfs_batch_read_scene")

    def write(self, sid: int, pos4: np.ndarray, vel4: Optional[np.ndarray] = None) -> None:
        n = self.sizes[sid]
        pos4 = _f4(pos4, n)
        vel4 = _f4(vel4, n)
        check(lib().pfs_batch_write_scene(self.handle, sid, _ptr(pos4), _ptr(vel4)),
              "pfs_batch_write_scene")

    def info(self) -> dict:
        i = BatchInfo()
        check(lib().pfs_batch_info_get(self.handle, ctypes.byref(i)), "pfs_batch_info_get")
        return {k: getattr(i, k) for k, _ in BatchInfo._fields_ if k != "reserved"}

    @property
    def stream(self) -> int:
        return lib().pfs_batch_stream(self.handle) or 0

    def close(self) -> None:
        if self._h is not None:
            lib().pfs_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
