#!/usr/bin/env python3
"""Benchmark of the SPH world step (particle-steps/s).

Default workload: the 1,048,576-particle FP32 drop-in scene (uniform slab in
[0,0.8]x[0,1.6]x[0,2] of the [0,2]^3 box, v ~ N(0, 0.05^2), seed 1, h = 0.02,
target density 1000, pressure multiplier 250, viscosity 0.03, gravity -9.81 y,
dt = 1/240, one substep).  A "step" is one world step over that batch of
particles: every timed step first feeds the batch into the world
(pfs_world_write from a resident device copy, keys recomputed) and then runs
the full step (sort, reorder+predict, table, density, force, integrate).
Feeding the same batch keeps every timed step on the workload's inputs; a
1,000-step rollout of this parameter set pushes particles into the box
corners, which is a different (degenerate) workload.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pfs|reference]
                  [--workload slab_1m|dam_break|colliding_blocks] [--precision fp32|fp16]
                  [--no-extra] [--batched-steps S] [--serving-seconds T] [--serving-wall T]

Beside the headline, a one-GPU run also reports (keys of the same JSON line):
fp16_cell (the same workload in the FP16-cell form), colliding_blocks (the
4,194,304-particle precision workload in every form: throughput, and errors
against the host FP64 oracle on an 8,192-particle subset after substeps 1 and
100), batched (256 scenes in
one batch vs per-scene plain worlds, per-step p50/p99) and serving (continuous
batching of the Poisson request stream under a 150 GB budget: request latency
p50/p99 and aggregate particle-steps/s).

Under torchrun every rank simulates its own replica (independent scene, seed
offset by rank): no data-path collective, "scaling": "weak"; the timed
region is bracketed by barriers and the max over ranks is reported.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "particle-fluid-simulation_b200")
FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes per particle-substep per stage (FP32 form): one read and
# one write of each array a stage must touch, neighbour data assumed reused
# from L2.  P = number of 8-bit radix passes for keys < n.
STAGE_BYTES = {
    # R x,v gathered 32 + R perm 4 + W xs,vs,xp,vp 64, and the cell table it
    # builds in the same kernel: R sorted keys 4 + W start,end 8
    "reorder": 112,
    "density": 32,     # R x* 16 + table 8 + W rho,rho_near 8
    "force": 80,       # R x*,v*,v 48 + rho 8 + table 8 + W v 16
    "integrate": 68,   # R x,v 32 + W x,v 32 + W key 4
}


def sort_bytes(n: int) -> int:
    bits = 0 if n <= 1 else int(n - 1).bit_length()
    passes = (bits + 7) // 8
    return 0 if passes == 0 else 12 + 16 * (passes - 1) + 4


def step_bytes(n: int) -> int:
    return sum(STAGE_BYTES.values()) + sort_bytes(n)


def issue_roofline(workload, precision, kernel, shape, launch_ms, sm_mhz, sms):
    """The instruction-issue bound of the dominant kernel beside its HBM
    roofline: the warp instructions one launch executes (ncu,
    smsp__inst_executed.sum, from the capture summarised in profiles/) over
    the issue rate of one warp instruction per clock per SM sub-partition
    (4 per SM) at the SM clock sampled during the timed region, against the
    launch's measured time."""
    path = os.path.join(ROOT, "profiles", "instructions.json")
    try:
        with open(path) as f:
            table = json.load(f)
    except Exception:
        return None
    w = table.get(f"{workload}:{precision}:{kernel}:{shape}",
                  table.get(f"{workload}:{precision}:{kernel}"))
    if not w or not sm_mhz or not launch_ms:
        return None
    rate = sms * 4 * sm_mhz * 1e6
    return {"warp_instructions": w, "peak_warp_inst_per_s": rate,
            "achieved_warp_inst_per_s": w / (launch_ms / 1e3),
            "frac": (w / rate) / (launch_ms / 1e3)}


def load_package():
    if "pfs_b200" in sys.modules:
        return sys.modules["pfs_b200"]
    spec = importlib.util.spec_from_file_location(
        "pfs_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pfs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def make_scene(name: str, precision: str, rank: int):
    pkg = load_package()
    from pfs_b200 import replicas, scenes
    prec = {"fp16": pkg.PFS_FP16_CELL, "fp32": pkg.PFS_FP32, "fp32_fast": pkg.PFS_FP32_FAST}[precision]
    if name == "slab_1m":
        return scenes.slab_1m(seed=replicas.replica_seed(1, rank), precision=prec)
    if name == "dam_break":
        return scenes.dam_break(seed=replicas.replica_seed(0, rank), precision=prec)
    if name == "colliding_blocks":
        return scenes.colliding_blocks(seed=replicas.replica_seed(2, rank), precision=prec)
    raise SystemExit(f"unknown workload {name}")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, name in enumerate(names):
                    if r[5 + k].lower() == "active":
                        reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def cpu_baseline(scene, budget_s: float, threads: int = 0):
    """Oracle (the restated reference step) on the host cores: bounded sample
    of the same workload (each step from the fed batch), particle-steps/s."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as ora
    if threads:
        ora.set_threads(threads)
    cores = ora.max_threads()
    n = scene.n
    steps = 0
    t0 = time.perf_counter()
    while True:
        ora.step(scene.params, scene.pos, scene.vel, 1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or steps >= 1000:
            break
    return {"value": n * steps / el, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "sample": f"{steps} step(s) of the {n}-particle workload ({el:.1f} s, each step from "
                      f"the fed batch, oracle/pfs_oracle.c with OpenMP)"}


def time_fed_world(pkg, torch, scene, steps, warmup, dev):
    """Device time of `steps` fed world steps (CUDA events on the world's stream)."""
    world = pkg.World(scene.params, scene.pos, scene.vel)
    world.autotune(5)
    stream = torch.cuda.ExternalStream(world.stream)
    fp = torch.from_numpy(scene.pos).to(dev)
    fv = torch.from_numpy(scene.vel).to(dev)
    torch.cuda.synchronize()
    for _ in range(warmup):
        world.write_ptr(fp.data_ptr(), fv.data_ptr())
        world.step(1)
    world.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(steps):
            world.write_ptr(fp.data_ptr(), fv.data_ptr())
            world.step(1)
        e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    assert world.device_error() == 0
    world.close()
    return ms


def measure_form(pkg, torch, precision, steps, warmup, dev, head_value):
    """The headline workload (slab_1m, fed steps) in another FP32 form."""
    from pfs_b200 import scenes
    prec = pkg.PFS_FP32 if precision == "fp32" else pkg.PFS_FP32_FAST
    sc = scenes.slab_1m(precision=prec)
    ms = time_fed_world(pkg, torch, sc, steps, warmup, dev)
    value = sc.n * steps / (ms / 1000.0)
    return {"value": value, "unit": "particle-steps/s", "ms_per_step": ms / steps,
            "vs_headline": value / head_value,
            "form": "the reference's IEEE operation sequence, bit-exact with the oracle"
                    if precision == "fp32" else
                    "fused multiply-adds and hardware reciprocals in the neighbour sums"}


def measure_fp16(pkg, torch, steps, warmup, dev, fp32_value):
    from pfs_b200 import scenes
    sc = scenes.slab_1m(precision=pkg.PFS_FP16_CELL)
    ms = time_fed_world(pkg, torch, sc, steps, warmup, dev)
    value = sc.n * steps / (ms / 1000.0)
    return {"value": value, "unit": "particle-steps/s", "ms_per_step": ms / steps,
            "vs_fp32": value / fp32_value,
            "workload": "slab_1m in the FP16-cell form (16-byte cell-relative records, "
                        "FP32 accumulation)",
            # bytes a neighbour pass reads per candidate (mostly from L2): the
            # record against the FP32 form's float4 arrays
            "candidate_bytes": {"density": 16, "force": 16 + 8},
            "candidate_bytes_fp32": {"density": 16, "force": 16 + 16 + 8}}


def _subset_errors(ora, params, got, vel_in, subset):
    """Errors of one substep's densities and post-force velocities against the
    host FP64 evaluation of the same neighbour sums on `subset`: max relative
    density error, and max velocity error over the subset's largest FP64
    speed."""
    vs = vel_in[got["perm"]]
    d64, _, v64 = ora.subset_f64(params, got["xp"], got["vp"], vs, got["start"], got["end"], subset)
    dens = got["density"][subset].astype(np.float64)
    vel = got["vel_force"][subset, :3].astype(np.float64)
    de = float(np.max(np.abs(dens - d64) / d64))
    ve = float(np.max(np.linalg.norm(vel - v64, axis=1)) / np.max(np.linalg.norm(v64, axis=1)))
    return {"density": de, "velocity": ve}


def measure_colliding_blocks(pkg, torch, steps, warmup, dev):
    """The precision workload: 4,194,304 particles in two colliding blocks,
    each form's fed-step throughput, and each form's errors against the host
    FP64 oracle on a fixed 8,192-particle subset for substep 1 and for
    substep 100 of the form's own rollout."""
    from pfs_b200 import scenes
    sys.path.insert(0, ROOT)
    from oracle import oracle as ora
    forms = [("fp32", pkg.PFS_FP32), ("fp16_cell", pkg.PFS_FP16_CELL)]
    if hasattr(pkg, "PFS_FP32_FAST"):
        forms.insert(1, ("fp32_fast", pkg.PFS_FP32_FAST))
    out = {"workload": "colliding_blocks (4194304 particles, 1 substep/step), each step fed "
                       "the workload's batch", "subset": 8192}
    subset = None
    for name, prec in forms:
        sc = scenes.colliding_blocks(precision=prec)
        if subset is None:
            rng = np.random.default_rng(8192)
            subset = np.sort(rng.choice(sc.n, 8192, replace=False)).astype(np.uint32)
        ms = time_fed_world(pkg, torch, sc, steps, warmup, dev)
        entry = {"value": sc.n * steps / (ms / 1000.0), "unit": "particle-steps/s",
                 "ms_per_step": ms / steps, "errors_vs_fp64": {}}
        with pkg.World(sc.params, sc.pos, sc.vel) as w:
            done = 0
            for at in (1, 100):
                if at - 1 > done:
                    w.step(at - 1 - done)
                    done = at - 1
                st = w.read(pos=False, vel=True)
                got = w.debug_substep()
                done += 1
                entry["errors_vs_fp64"][f"step{at}"] = _subset_errors(ora, sc.params, got,
                                                                       st["vel"], subset)
            assert w.device_error() == 0
        out[name] = entry
    base = out["fp32"]["value"]
    for name, _ in forms:
        out[name]["vs_fp32"] = out[name]["value"] / base
    return out


def measure_density_map(pkg, torch, dev, calls=10, with_cpu=False):
    """Density map (the reference's updateDensityMap.comp) of the slab_1m state
    after one step at cell size h (101^3 voxels) through the C ABI into device
    memory; CUDA events on the world's stream around `calls` calls."""
    from pfs_b200 import scenes
    sc = scenes.slab_1m()
    cs = sc.params.h
    w = pkg.World(sc.params, sc.pos, sc.vel)
    w.step(1)
    shape = w.density_map(cs).shape
    out = torch.empty(shape, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(w.stream)
    for _ in range(2):
        w.density_map_ptr(cs, out.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(calls):
        w.density_map_ptr(cs, out.data_ptr())
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / calls
    assert w.device_error() == 0
    st = w.read(pos=True, keys=True) if with_cpu else None
    w.close()
    voxels = int(np.prod(shape))
    out = {"voxels": voxels, "dims": list(reversed(shape)), "cell_size": cs,
           "ms_per_map": ms, "voxels_per_s": voxels / (ms / 1e3),
           "workload": "slab_1m state after one step, cell size h, output in device memory"}
    if with_cpu:
        sys.path.insert(0, ROOT)
        from oracle import oracle as ora
        t0 = time.perf_counter()
        ora.density_map(sc.params, st["pos"], st["keys"], cs)
        cpu_ms = (time.perf_counter() - t0) * 1e3
        out["cpu_baseline"] = {"ms_per_map": cpu_ms, "cores": ora.max_threads(), "kind": "port",
                               "sample": "one map of the same state (oracle/pfs_oracle.c, OpenMP)"}
    return out


def measure_volumetric(pkg, torch, dev, width=1280, height=720, calls=5, with_cpu=False):
    """The reference's volumetric render mode (updateDensityMap.comp,
    calculateLightVolume.comp, volumetricFluid.comp) of the slab_1m state after
    one step, headless into device memory: density map at cell size h, light
    volume at 2h, ray-march step h / 2, camera in front of the box looking
    along +y.  One call runs all three kernels; CUDA events on the world's
    stream around `calls` calls."""
    from pfs_b200 import scenes
    sc = scenes.slab_1m()
    h = float(sc.params.h)
    lo = np.array(sc.params.box_min[:3], np.float64)
    hi = np.array(sc.params.box_max[:3], np.float64)
    c = (lo + hi) / 2
    view = pkg.volume_view(position=(c[0], lo[1] - 1.2 * (hi[1] - lo[1]), c[2]), forward=(0, 1, 0),
                           right=(1, 0, 0), up=(0, 0, 1), density_cell_size=h, step_size=h / 2,
                           light_step_size=2 * h)
    w = pkg.World(sc.params, sc.pos, sc.vel)
    w.step(1)
    out = torch.empty((height, width, 4), dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(w.stream)
    for _ in range(2):
        w.render_volumetric_ptr(view, width, height, out.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(calls):
        w.render_volumetric_ptr(view, width, height, out.data_ptr())
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / calls
    assert w.device_error() == 0
    lit = int((out[..., :3] > 0).any(-1).sum().item())
    st = w.read(pos=True, keys=True) if with_cpu else None
    ldims = w.render_volumetric(view, 8, 8, with_light_volume=True)[1].shape
    w.close()
    res = {"width": width, "height": height, "pixels_lit": lit, "ms_per_frame": ms,
           "frames_per_s": 1e3 / ms, "light_volume_dims": list(reversed(ldims)),
           "workload": "slab_1m state after one step; density map (cell h) + light volume "
                       "(2h) + ray march (step h/2) per frame, output in device memory"}
    if with_cpu:
        sys.path.insert(0, ROOT)
        from oracle import oracle as ora
        t0 = time.perf_counter()
        dmap = ora.density_map(sc.params, st["pos"], st["keys"], h)
        lv = ora.light_volume(sc.params, dmap, view.light_step_size, np.array(view.dir_to_sun[:3]))
        cam = np.array(list(view.position) + list(view.forward) + list(view.right) + list(view.up),
                       np.float32)
        half = float(np.float32(np.tan(np.float32(0.5) * np.float32(view.fov))))
        ora.volumetric(sc.params, dmap, lv, cam, half, view.step_size, np.array(view.extinction[:3]),
                       width, height)
        cpu_ms = (time.perf_counter() - t0) * 1e3
        res["cpu_baseline"] = {"ms_per_frame": cpu_ms, "cores": ora.max_threads(), "kind": "port",
                               "sample": "one frame of the same state and view "
                                         "(oracle/pfs_oracle.c, OpenMP)"}
    return res


def measure_refractive(pkg, torch, dev, width=1280, height=720, calls=3, with_cpu=False):
    """The reference's refractive render mode (updateDensityMap.comp +
    properFluid.comp) of the slab_1m state after one step, headless into
    device memory: density map at cell size h, surface threshold rho0 / 2,
    3 refractions, IOR 1.333, step h / 2, light step 2h, same camera as the
    volumetric measurement."""
    from pfs_b200 import scenes
    sc = scenes.slab_1m()
    h = float(sc.params.h)
    lo = np.array(sc.params.box_min[:3], np.float64)
    hi = np.array(sc.params.box_max[:3], np.float64)
    c = (lo + hi) / 2
    view = pkg.volume_view(position=(c[0], lo[1] - 1.2 * (hi[1] - lo[1]), c[2]), forward=(0, 1, 0),
                           right=(1, 0, 0), up=(0, 0, 1), density_cell_size=h, step_size=h / 2,
                           light_step_size=2 * h, extinction=(0.4, 0.4, 0.2))
    refr = pkg.refraction(surface_density_threshold=0.5 * float(sc.params.target_density))
    w = pkg.World(sc.params, sc.pos, sc.vel)
    w.step(1)
    out = torch.empty((height, width, 4), dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(w.stream)
    for _ in range(2):
        w.render_refractive_ptr(view, refr, width, height, out.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(calls):
        w.render_refractive_ptr(view, refr, width, height, out.data_ptr())
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / calls
    assert w.device_error() == 0
    distinct = int(torch.unique(out[..., 0]).numel())
    st = w.read(pos=True, keys=True) if with_cpu else None
    w.close()
    res = {"width": width, "height": height, "distinct_values": distinct, "ms_per_frame": ms,
           "frames_per_s": 1e3 / ms,
           "workload": "slab_1m state after one step; density map (cell h) + refractive march "
                       "(step h/2, light step 2h, threshold rho0/2, 3 refractions) per frame, "
                       "output in device memory"}
    if with_cpu:
        sys.path.insert(0, ROOT)
        from oracle import oracle as ora
        t0 = time.perf_counter()
        dmap = ora.density_map(sc.params, st["pos"], st["keys"], h)
        map_ms = (time.perf_counter() - t0) * 1e3
        cam = np.array(list(view.position) + list(view.forward) + list(view.right) + list(view.up),
                       np.float32)
        half = float(np.float32(np.tan(np.float32(0.5) * np.float32(view.fov))))
        # the same view at a quarter of the resolution in each direction,
        # scaled by the pixel count
        sw, sh = width // 4, height // 4
        t0 = time.perf_counter()
        ora.refractive(sc.params, dmap, cam, half, view.step_size, view.light_step_size,
                       np.array(view.extinction[:3]), refr.num_refractions,
                       refr.surface_density_threshold, refr.index_of_refraction, sw, sh)
        march_ms = (time.perf_counter() - t0) * 1e3
        res["cpu_baseline"] = {"ms_per_frame_est": map_ms + march_ms * (width * height) / (sw * sh),
                               "ms_map": map_ms, "ms_march_sample": march_ms,
                               "cores": ora.max_threads(), "kind": "port",
                               "sample": f"density map + the same view at {sw}x{sh} "
                                         "(oracle/pfs_oracle.c, OpenMP); the march is scaled by "
                                         "the pixel count"}
    return res


def measure_splats(pkg, torch, dev, width=1280, height=720, calls=5, with_cpu=False):
    """The reference's default render (shader.vert / shader.frag point splats,
    depth test LESS) of the slab_1m state after one step, radius h / 2,
    headless into device memory, followed by the FXAA presentation pass
    (raymarchShader.frag) timed on its own."""
    from pfs_b200 import scenes
    sc = scenes.slab_1m()
    p = sc.params
    p.flags |= pkg.PFS_FLAG_COLORS
    h = float(p.h)
    lo = np.array(p.box_min[:3], np.float64)
    hi = np.array(p.box_max[:3], np.float64)
    c = (lo + hi) / 2
    view = pkg.splat_view((c[0], lo[1] - 1.2 * (hi[1] - lo[1]), c[2]), (0, 1, 0), width, height, h / 2)
    w = pkg.World(p, sc.pos, sc.vel)
    w.step(1)
    out = torch.empty((height, width, 4), dtype=torch.float32, device=dev)
    dep = torch.empty((height, width), dtype=torch.float32, device=dev)
    fx = torch.empty_like(out)
    stream = torch.cuda.ExternalStream(w.stream)
    for _ in range(2):
        w.render_splats_ptr(view, width, height, out.data_ptr(), dep.data_ptr())
        w.fxaa_ptr(out.data_ptr(), width, height, fx.data_ptr())
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    for _ in range(calls):
        w.render_splats_ptr(view, width, height, out.data_ptr(), dep.data_ptr())
    e1.record(stream)
    for _ in range(calls):
        w.fxaa_ptr(out.data_ptr(), width, height, fx.data_ptr())
    e2.record(stream)
    e2.synchronize()
    ms = e0.elapsed_time(e1) / calls
    ms_fx = e1.elapsed_time(e2) / calls
    assert w.device_error() == 0
    covered = int((dep < 1).sum().item())
    st = w.read(pos=True) if with_cpu else None
    col = w.read_colors() if with_cpu else None
    w.close()
    res = {"width": width, "height": height, "particles": sc.n, "pixels_covered": covered,
           "ms_per_frame": ms, "frames_per_s": 1e3 / ms, "fxaa_ms_per_frame": ms_fx,
           "workload": "slab_1m state after one step, 1,048,576 discs of radius h/2, depth test "
                       "LESS, output and depth in device memory; FXAA of the result timed apart"}
    if with_cpu:
        sys.path.insert(0, ROOT)
        from oracle import oracle as ora
        mats = [np.array(m[:], np.float32) for m in (view.model, view.view, view.proj)]
        t0 = time.perf_counter()
        img, _ = ora.splats(st["pos"], col, *mats, view.particle_radius, width, height)
        splat_ms = (time.perf_counter() - t0) * 1e3
        t0 = time.perf_counter()
        ora.fxaa(img)
        fxaa_ms = (time.perf_counter() - t0) * 1e3
        res["cpu_baseline"] = {"ms_per_frame": splat_ms, "fxaa_ms_per_frame": fxaa_ms,
                               "cores": 1, "fxaa_cores": ora.max_threads(), "kind": "port",
                               "sample": "one frame of the same state and camera (oracle/pfs_oracle.c: "
                                         "sequential draw in slot order; FXAA with OpenMP)"}
    return res


def _pct(a, q):
    return float(np.percentile(np.asarray(a), q)) if len(a) else None


def measure_batched(pkg, torch, steps, dev):
    """256 scenes (sizes log-U[2048, 262144], per-scene h, rho0, k, visc; seed
    3): one batch (one sort and one launch per stage for all scenes, a CUDA
    graph per step) against one World per scene stepped by plain per-scene
    launches.  Both feed every step from the scenes' inputs; each step is
    timed by the wall clock around a device-synchronised step, so the host
    cost of launching is included for both paths."""
    from pfs_b200 import scenes
    scs = scenes.scene_batch(256)
    total = sum(s.n for s in scs)
    subs = scs[0].params.substeps
    b = pkg.Batch(total, len(scs), pkg.PFS_FP32, substeps=subs)
    for s in scs:
        b.add(s.params, s.pos, s.vel)
    b.set_feed(True)
    b.step(1)
    tune = b.autotune(1)
    for _ in range(2):
        b.step(1)
    b.sync()
    bt = []
    for _ in range(steps):
        t0 = time.perf_counter()
        b.step(1)
        b.sync()
        bt.append((time.perf_counter() - t0) * 1e3)
    info = b.info()
    b.close()
    feeds = [(torch.from_numpy(s.pos).to(dev), torch.from_numpy(s.vel).to(dev)) for s in scs]

    def plain_run(search, nsteps):
        # worlds take their neighbour search from the environment at creation
        old = os.environ.get("PFS_NEIGHBOR_SEARCH")
        if search:
            os.environ["PFS_NEIGHBOR_SEARCH"] = search
        try:
            worlds = [pkg.World(s.params, s.pos, s.vel) for s in scs]
        finally:
            if search:
                if old is None:
                    del os.environ["PFS_NEIGHBOR_SEARCH"]
                else:
                    os.environ["PFS_NEIGHBOR_SEARCH"] = old
        torch.cuda.synchronize()

        def plain_step():
            for w, (fp, fv) in zip(worlds, feeds):
                w.write_ptr(fp.data_ptr(), fv.data_ptr())
                w.step(1)
            for w in worlds:
                w.sync()

        plain_step()
        times = []
        for _ in range(nsteps):
            t0 = time.perf_counter()
            plain_step()
            times.append((time.perf_counter() - t0) * 1e3)
        launches = sum(w.launches_per_substep() * subs + 1 for w in worlds)
        for w in worlds:
            w.close()
        return times, launches

    pt, plain_launches = plain_run(None, steps)
    tt, _ = plain_run("table", max(1, min(steps, 2)))
    value = total * steps / (sum(bt) / 1000.0)
    plain = total * steps / (sum(pt) / 1000.0)
    plain_table = total * len(tt) / (sum(tt) / 1000.0)
    return {"scenes": len(scs), "particles": total, "steps": steps, "substeps_per_step": subs,
            "value": value, "plain_value": plain, "unit": "particle-steps/s",
            "ratio_vs_plain": value / plain,
            "plain_table_scan_value": plain_table,
            "ratio_vs_plain_table_scan": value / plain_table,
            "plain": "one World per scene on its own stream, graph per step; plain_value with "
                     "the same neighbour search as the batch, plain_table_scan_value with the "
                     "reference's table scan for every scene",
            "step_ms_p50": _pct(bt, 50), "step_ms_p99": _pct(bt, 99),
            "plain_step_ms_p50": _pct(pt, 50), "plain_step_ms_p99": _pct(pt, 99),
            "autotune": tune,
            "launches_per_step": info["launches_per_substep"] * subs + 1,
            "plain_launches_per_step": plain_launches,
            "timing": "wall clock around device-synchronised steps (host launch cost included "
                      "for both paths); every step runs the scenes' input states"}


def measure_serving(pkg, seconds, wall_s):
    """Poisson arrivals at 200 requests/s (seed 4) for `seconds` of the 60 s
    stream, served by continuous batching under a 150 GB budget, until all are
    served or `wall_s` passes."""
    from pfs_b200 import scenes, serving
    specs = scenes.request_stream(duration_s=seconds)
    reqs = serving.requests_from_stream(specs)
    budget = 150 * 10**9
    with serving.Server(budget, max_scenes=1024, substeps=3, feed=True,
                        keep_results=False) as srv:
        stats = serving.run(srv, reqs, wall_limit_s=wall_s)
        stats["capacity_particles"] = {("fp32" if k == pkg.PFS_FP32 else "fp16"): v
                                       for k, v in srv.capacity.items()}
    offered = sum(s.n * s.steps for s in specs)
    stats.update({"arrival_rate_per_s": 200.0, "arrival_seconds": seconds,
                  "wall_cap_s": wall_s,
                  "offered_particle_steps": offered,
                  "offered_particle_steps_per_s": offered / max(seconds, 1e-9),
                  "hbm_budget_gb": budget / 1e9,
                  "feed": "each step runs the request's input state"})
    return stats


def serve_plain(pkg, torch, dev, specs, wall_s):
    """The plain per-request path: each request, in arrival order and one at a
    time, gets its own World and steps it (each step from its input state, as
    the continuous-batching server's feed mode does), until all are served or
    `wall_s` passes.  Requests cut off by the wall limit count the steps they
    made."""
    specs = sorted(specs, key=lambda r: r.arrival_s)
    t0 = time.perf_counter()
    lat, psteps, finished = [], 0, 0
    for spec in specs:
        now = time.perf_counter() - t0
        if now > wall_s:
            break
        if spec.arrival_s > now:
            time.sleep(spec.arrival_s - now)
        sc = spec.make_scene()
        w = pkg.World(sc.params, sc.pos, sc.vel)
        xin = torch.from_numpy(sc.pos).to(dev)
        vin = torch.from_numpy(sc.vel).to(dev)
        done = 0
        for _ in range(spec.steps):
            w.write_ptr(xin.data_ptr(), vin.data_ptr())
            w.step(1)
            done += 1
            if done % 8 == 0:
                w.sync()
                if time.perf_counter() - t0 > wall_s:
                    break
        w.sync()
        w.close()
        psteps += sc.n * done
        if done == spec.steps:
            finished += 1
            lat.append(time.perf_counter() - t0 - spec.arrival_s)
    elapsed = time.perf_counter() - t0
    return {"requests": len(specs), "finished": finished, "elapsed_s": elapsed,
            "particle_steps": psteps, "particle_steps_per_s": psteps / elapsed if elapsed > 0 else 0.0,
            "latency_p50_s": _pct(lat, 50), "latency_p99_s": _pct(lat, 99),
            "path": "one World per request, in arrival order, one request at a time"}


def measure_serving_matched(pkg, torch, dev, count=64, max_steps=30):
    """Equal work for both paths: the stream's first `count` requests (their
    arrival times, sizes, precisions and parameters), step counts capped at
    `max_steps`, served to completion by continuous batching and by the plain
    per-request path; throughput and request latency of each."""
    import dataclasses
    from pfs_b200 import scenes, serving
    specs = [dataclasses.replace(r, steps=min(r.steps, max_steps))
             for r in scenes.request_stream(duration_s=60.0)[:count]]
    with serving.Server(150 * 10**9, max_scenes=1024, substeps=3, feed=True,
                        keep_results=False) as srv:
        batched = serving.run(srv, serving.requests_from_stream(specs), wall_limit_s=600.0)
    plain = serve_plain(pkg, torch, dev, specs, 600.0)
    out = {"requests": count, "max_steps": max_steps,
           "particle_steps": sum(r.n * r.steps for r in specs),
           "batched": {k: batched[k] for k in ("finished", "elapsed_s", "particle_steps_per_s",
                                                "latency_p50_s", "latency_p99_s", "tick_p50_ms",
                                                "tick_p99_ms")},
           "plain_per_request": {k: plain[k] for k in ("finished", "elapsed_s", "particle_steps_per_s",
                                                       "latency_p50_s", "latency_p99_s")}}
    if plain["particle_steps_per_s"] > 0:
        out["vs_plain"] = batched["particle_steps_per_s"] / plain["particle_steps_per_s"]
    return out


def run_batched_workload(args, rank, world_size, local_rank):
    """The batched workload on its own: 256 scenes (every batch_stride-th) in
    one batch, fed from their inputs every step, timed with CUDA events on
    the batch's stream (no per-scene plain comparison; see measure_batched)."""
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world_size > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    pkg = load_package()
    from pfs_b200 import scenes
    from pfs_b200 import replicas
    # each rank steps its own share of the 256 scenes
    scs = replicas.shard(scenes.scene_batch(256)[::max(1, args.batch_stride)], rank, world_size)
    total = sum(s.n for s in scs)
    subs = scs[0].params.substeps
    b = pkg.Batch(total, len(scs), pkg.PFS_FP32, substeps=subs)
    for sc in scs:
        b.add(sc.params, sc.pos, sc.vel)
    b.set_feed(True)
    for _ in range(args.warmup):
        b.step(1)
    b.sync()
    stream = torch.cuda.ExternalStream(b.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            b.step(1)
        e1.record(stream)
        e1.synchronize()
    cdev = torch.device("cuda", local_rank)
    ms_max = replicas.max_over_ranks(e0.elapsed_time(e1), dist, cdev)
    all_particles = replicas.sum_over_ranks(total, dist, cdev)
    info = b.info()
    b.close()
    if rank == 0:
        print(json.dumps({
            "metric": "particle-steps/s",
            "value": all_particles * args.steps / (ms_max / 1e3),
            "unit": "particle-steps/s", "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched_256 ({len(scs)} scenes, {total} particles, "
                                   f"{subs} substeps/step, fp32)", "particles": total,
                       "l2": "no flush: batch arrays exceed 126 MB L2",
                       "feed": "each step runs the scenes' input states"},
            "gpu_launches": args.steps * (info["launches_per_substep"] * subs + 1),
            "parallelism": f"scenes sharded over {world_size} rank(s) (every world_size-th scene)",
            "clocks": clk.summary()}), flush=True)
    if world_size > 1:
        dist.destroy_process_group()
    return 0


def run_reference(args, rank, world_size):
    if rank != 0:
        return 0
    scene = make_scene(args.workload, args.precision, 0)
    for _ in range(args.warmup):
        pass  # the CPU arm needs no warm-up; kept for the flag contract
    # each timed step: one oracle world step over the batch; bounded sample per step
    sys.path.insert(0, ROOT)
    from oracle import oracle as ora
    cores = ora.max_threads()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ora.step(scene.params, scene.pos, scene.vel, 1)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = scene.n * args.steps / total
    subs = scene.params.substeps
    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
        "impl": "reference", "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        # the same workload label as the GPU arm's; the reference's step is FP32
        "config": {"workload": f"{args.workload} ({scene.n} particles, {subs} substep(s)/step, fp32)",
                   "particles": scene.n, "substeps_per_step": subs, "precision": "fp32",
                   "parallelism": f"rank 0 only, {cores} host threads", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores,
                         "kind": "port",
                         "sample": f"{args.steps} oracle step(s) of the {scene.n}-particle "
                                   f"workload, each from the fed batch"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="pfs", choices=["pfs", "reference"])
    ap.add_argument("--workload", default="slab_1m",
                    choices=["slab_1m", "dam_break", "colliding_blocks", "batched_256"])
    ap.add_argument("--batch-stride", type=int, default=1,
                    help="batched_256: keep every k-th of the 256 scenes (smaller profiling case)")
    # fp32_fast: FP32 with fused arithmetic in the neighbour sums, held to
    # the 1e-5 per-step tolerance; fp32: the reference's exact operation
    # sequence (bit-exact with the oracle); fp16: FP16-cell neighbour data
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp32_fast", "fp16"])
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=5)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default kernel shape instead of pfs_world_autotune's pick")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the FP16-cell, batched and serving legs")
    ap.add_argument("--batched-steps", type=int, default=5)
    ap.add_argument("--serving-seconds", type=float, default=60.0,
                    help="seconds of the 60 s request stream to serve (0: skip)")
    ap.add_argument("--serving-wall", type=float, default=70.0,
                    help="wall-clock cap of the serving leg (arrivals keep coming until "
                         "--serving-seconds)")
    args = ap.parse_args()

    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world_size)
    if args.workload == "batched_256":
        return run_batched_workload(args, rank, world_size, local_rank)

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world_size > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    pkg = load_package()
    scene = make_scene(args.workload, args.precision, rank)
    n = scene.n
    subs = scene.params.substeps
    world = pkg.World(scene.params, scene.pos, scene.vel)
    # every shape gives the same bits; the autotuner keeps the fastest on this
    # workload's state and leaves the state as it was
    tune = None if args.no_autotune else world.autotune(5)
    stream = torch.cuda.ExternalStream(world.stream)
    dev = torch.device("cuda", local_rank)
    feed_pos = torch.from_numpy(scene.pos).to(dev)
    feed_vel = torch.from_numpy(scene.vel).to(dev)
    torch.cuda.synchronize()

    def step():
        world.write_ptr(feed_pos.data_ptr(), feed_vel.data_ptr())
        world.step(1)

    for _ in range(args.warmup):
        step()
    world.sync()

    def barrier():
        if world_size > 1:
            dist.barrier()
        torch.cuda.synchronize()

    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                step()
            end.record(stream)
        end.synchronize()
    barrier()
    from pfs_b200 import replicas
    ms_max = replicas.max_over_ranks(start.elapsed_time(end), dist, dev)
    value = replicas.job_throughput(n * args.steps, world_size, ms_max)
    world.sync()
    assert world.device_error() == 0

    # per-stage device times (separate, event-bracketed run; not the headline)
    world.profile(True)
    for _ in range(args.profile_steps):
        step()
    st = world.stage_times()
    world.profile(False)
    per_launch_ms = {k: st["ms_total"][k] / max(1, st["substeps"]) for k in st["ms_total"]}
    dominant = max(per_launch_ms, key=per_launch_ms.get)
    dom_bytes = (sort_bytes(n) if dominant == "sort" else STAGE_BYTES[dominant]) * n
    peak, peak_kind = peaks()
    achieved = dom_bytes / (per_launch_ms[dominant] / 1000.0) / 1e9
    traffic = None
    # the neighbour shape that ran: the autotuner's pick, else the one the
    # environment forces, else the library's default (the flat shape)
    shape_used = (tune["chosen"]["shape"] if tune and tune.get("chosen")
                  else os.environ.get("PFS_NBR_VARIANT", "flat"))
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                table = json.load(f)
            traffic = table.get(f"{args.workload}:{args.precision}:{dominant}:{shape_used}",
                                table.get(f"{args.workload}:{args.precision}:{dominant}"))
        except Exception:
            traffic = None

    # end to end through the C ABI with pinned host buffers
    pin_in_p = torch.from_numpy(scene.pos).pin_memory()
    pin_in_v = torch.from_numpy(scene.vel).pin_memory()
    pin_out_p = torch.empty_like(pin_in_p).pin_memory()
    pin_out_v = torch.empty_like(pin_in_v).pin_memory()
    # the same step count as the device-timed region: one pipelined call
    # fills and drains its copy pipeline once
    e2e_steps = max(3, args.steps)

    # each step: upload its input (pos, vel) from pinned host memory, one
    # step, read its result (pos, vel) back; pfs_world_run_pipelined overlaps
    # step k's compute with input k + 1's upload and output k - 1's read-back
    def e2e_run(count):
        world.run_pipelined_ptrs([pin_in_p.data_ptr()] * count, [pin_in_v.data_ptr()] * count,
                                 [pin_out_p.data_ptr()] * count, [pin_out_v.data_ptr()] * count, 1)

    e2e_run(2)
    barrier()
    with torch.cuda.stream(stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_run(e2e_steps)
        e1.record(stream)
    e1.synchronize()
    barrier()
    e2e_value = replicas.job_throughput(
        n * e2e_steps, world_size, replicas.max_over_ranks(e0.elapsed_time(e1), dist, dev))

    # PCIe copy rates of one step's inputs alone (pinned host memory), the
    # bound of the end-to-end figure when they exceed the step's device time
    def copy_gbs(dst, src):
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dst.copy_(src, non_blocking=True)
        c0.record()
        for _ in range(3):
            dst.copy_(src, non_blocking=True)
        c1.record()
        c1.synchronize()
        return 3 * src.numel() * src.element_size() / (c0.elapsed_time(c1) / 1e3) / 1e9

    dev_buf = torch.empty_like(feed_pos)
    pcie = {"h2d_gbs": copy_gbs(dev_buf, pin_in_p), "d2h_gbs": copy_gbs(pin_out_p, dev_buf)}
    del dev_buf

    launches = args.steps * (world.launches_per_substep() * subs + 1)
    world.close()

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu:
        cpu = cpu_baseline(scene, args.cpu_budget)

    extras = {}

    def extra(name, fn, *a, **kw):
        # a failing side measurement is reported in its place; the headline
        # line is printed either way
        try:
            extras[name] = fn(*a, **kw)
        except Exception as exc:  # noqa: BLE001
            extras[name] = {"error": f"{type(exc).__name__}: {exc}"}

    if world_size == 1 and not args.no_extra and args.workload == "slab_1m":
        if args.precision in ("fp32", "fp32_fast"):
            extra("fp32_exact" if args.precision == "fp32_fast" else "fp32_fast", measure_form, pkg,
                  torch, "fp32" if args.precision == "fp32_fast" else "fp32_fast", args.steps,
                  args.warmup, dev, value)
            extra("fp16_cell", measure_fp16, pkg, torch, args.steps, args.warmup, dev, value)
            extra("colliding_blocks", measure_colliding_blocks, pkg, torch, args.steps,
                  args.warmup, dev)
            extra("density_map", measure_density_map, pkg, torch, dev, with_cpu=not args.no_cpu)
            extra("volumetric", measure_volumetric, pkg, torch, dev, with_cpu=not args.no_cpu)
            extra("refractive", measure_refractive, pkg, torch, dev, with_cpu=not args.no_cpu)
            extra("splats", measure_splats, pkg, torch, dev, with_cpu=not args.no_cpu)
        if args.batched_steps > 0:
            extra("batched", measure_batched, pkg, torch, args.batched_steps, dev)
        if args.serving_seconds > 0:
            extra("serving", measure_serving, pkg, args.serving_seconds, args.serving_wall)
            extra("serving_matched", measure_serving_matched, pkg, torch, dev)
    if rank == 0:
        clocks = clk.summary()
        issue = issue_roofline(args.workload, args.precision, dominant,
                               shape_used, per_launch_ms[dominant], clocks.get("sm_mhz"),
                               torch.cuda.get_device_properties(dev).multi_processor_count)
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f16-cell/f32" if args.precision == "fp16" else "f32",
            "data": "synthetic",
            "config": {
                # both FP32 forms are the FP32 workload; "form" names which
                "workload": f"{args.workload} ({n} particles, {subs} substep(s)/step, "
                            f"{'fp16' if args.precision == 'fp16' else 'fp32'})",
                "form": {"fp32_fast": "fp32 with fused multiply-adds and hardware reciprocals in "
                                      "the neighbour sums (1e-5 per-step tolerance)",
                         "fp32": "fp32, the reference's IEEE operation sequence (bit-exact)",
                         "fp16": "fp16-cell neighbour data, fp32 accumulation"}[args.precision],
                "particles": n, "substeps_per_step": subs, "precision": args.precision,
                "parallelism": f"replicas x{world_size}",
                "l2": "no flush: per-step working set "
                      f"{(step_bytes(n) * n) / 1e6:.0f} MB of algorithmic traffic, resident "
                      f"arrays {(n * 150) / 1e6:.0f} MB > 126 MB L2",
                "feed": "each step writes the workload's batch (x, v) into the world first",
                "kernel_shape": tune["chosen"] if tune else
                f"default ({os.environ.get('PFS_NBR_VARIANT', 'flat')}, "
                f"{os.environ.get('PFS_NEIGHBOR_SEARCH', 'automatic')} search)",
            },
            "autotune": tune,
            "particle_substeps_per_s": value * subs,
            "step_roofline": {
                "bytes_per_particle_substep": step_bytes(n),
                "achieved_gbs": step_bytes(n) * value * subs / 1e9,
                "frac": step_bytes(n) * value * subs / 1e9 / peak,
            },
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": dom_bytes,
                         "launch_ms": per_launch_ms[dominant], "issue": issue},
            "stage_ms_per_substep": per_launch_ms,
            "e2e": {"value": e2e_value, "unit": "particle-steps/s",
                    "h2d_bytes_per_step": 2 * n * 16, "d2h_bytes_per_step": 2 * n * 16,
                    "steps": e2e_steps, "pcie": pcie},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world_size > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
