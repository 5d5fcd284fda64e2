#!/usr/bin/env python3
"""Execute the reference's own step shaders on the CPU (TEST INFRASTRUCTURE).

The reference ships its SPH step only as GLSL compute shaders
(src/shaders/*.comp) driven from C (src/renderer/commands.c:193-402); there
is no Vulkan device, loader or glslc on this machine or the GPU box.  This
script pins the oracle against those sources anyway:

  build   translate each step shader mechanically into a C++ struct (uniform
          and buffer blocks become members, 'out' parameters references,
          float literals float, shared arrays views of a per-workgroup arena)
          into oracle/_ref/gen/, and compile them with glsl_emu.hpp,
          glsl_dispatch.hpp and glsl_driver.cpp into oracle/_ref/libglsl_ref.so
          (g++ -O2 -ffp-contract=off).  The generated sources and the library
          stay out of version control.
  golden  run that library on seeded inputs and write the fixtures in
          tests/golden/ that the CPU tests check the oracle against.
  golden_map
          the same for the density map (updateDensityMap.comp):
          tests/golden/glsl_density_map.npz.
  golden_render
          light volume and image of the volumetric render mode
          (calculateLightVolume.comp, volumetricFluid.comp), the image of the
          refractive mode (properFluid.comp) on those maps, and both images
          after the presentation pass (raymarchShader.frag, one fragment per
          pixel): tests/golden/glsl_render.npz.
  golden_raster
          vertex outputs (shader.vert) of seeded particles' quad corners and
          fragment outputs (shader.frag) over a grid of fragQuadPos values:
          tests/golden/glsl_raster.npz.

The reference sources are read from the directory named by PFS_REFERENCE_ROOT
(the reference checkout; /root/reference when unset), read-only; nothing here
runs on the GPU box.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_ROOT = os.environ.get("PFS_REFERENCE_ROOT", "/root/reference")
REF_SHADERS = os.path.join(REF_ROOT, "src", "shaders")
OUT = os.path.join(HERE, "_ref")
GEN = os.path.join(OUT, "gen")
LIB = os.path.join(OUT, "libglsl_ref.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")

SHADERS = [
    "predictPositions", "updateCellEntries", "multiRadixSortHistograms", "multiRadixSort",
    "scatterPass", "clearStartIndices", "updateStartIndices", "calculateDensities",
    "applyPressureAndViscosityForce", "updateVelocities", "updateDensityMap",
    "calculateLightVolume", "volumetricFluid", "properFluid", "raymarchShader", "shader_vert",
    "shader_frag",
]
# shaders with images or samplers, dispatched with ref_dispatch_rt_<name>
RENDER_SHADERS = {"updateDensityMap", "calculateLightVolume", "volumetricFluid", "properFluid"}
# fragment shaders, run once per pixel by the generated ref_fragment_<name>
FRAG_SHADERS = {"raymarchShader"}
# shaders whose unreachable code (functions main never calls, statements
# after a function's top-level return, constants only those use) is dropped
# before translation: properFluid.comp keeps a floor/sky environment behind
# `return vec3(1);` that uses vector types the emulator does not provide
PRUNE_SHADERS = {"properFluid", "shader_frag"}
# the rasterisation pipeline's stages (src/shaders/shader.vert / shader.frag),
# run one vertex or one fragment at a time by glsl_driver.cpp
STAGE_SHADERS = {"shader_vert", "shader_frag"}


def shader_file(name: str) -> str:
    if name.endswith("_vert"):
        return name[:-5] + ".vert"
    if name.endswith("_frag"):
        return name[:-5] + ".frag"
    return name + (".frag" if name in FRAG_SHADERS else ".comp")
WORKGROUP_THREADS = {"multiRadixSortHistograms", "multiRadixSort"}
LOCAL_SIZE = {"multiRadixSortHistograms": 256, "multiRadixSort": 256}


def strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")


def construct_structs(src: str) -> str:
    """GLSL struct constructors Name(a, b, ...) -> C++ aggregate Name{a, b, ...}
    for the structs the shader defines."""
    names = re.findall(r"\bstruct\s+(\w+)\s*\{", src)
    for nm in names:
        out, i = [], 0
        pat = re.compile(r"\b" + nm + r"\s*\(")
        while True:
            m = pat.search(src, i)
            if not m:
                out.append(src[i:])
                break
            # a declaration "Name name(" (a function returning the struct) is not a call
            before = src[:m.start()].rstrip()
            prev = re.search(r"(\w+)$", before)
            if prev and prev.group(1) not in ("return",) and not before.endswith(("=", ",", "(")):
                out.append(src[i:m.end()])
                i = m.end()
                continue
            depth, j = 1, m.end()
            while depth:
                c = src[j]
                depth += c == "("
                depth -= c == ")"
                j += 1
            out.append(src[i:m.start()] + nm + "{" + src[m.end():j - 1] + "}")
            i = j
        src = "".join(out)
    return src


def _block_end(src: str, open_brace: int) -> int:
    """Index just past the brace that closes the one at open_brace."""
    depth, j = 0, open_brace
    while True:
        depth += src[j] == "{"
        depth -= src[j] == "}"
        j += 1
        if depth == 0:
            return j


def _functions(src: str) -> dict:
    """Top-level function definitions: name -> (start, end, body start)."""
    header = re.compile(r"^(\w+)\s+(\w+)\s*\(([^;{}]*)\)\s*\{", re.M)
    funcs = {}
    for m in header.finditer(src):
        if src[:m.start()].count("{") != src[:m.start()].count("}"):
            continue  # not at top level
        funcs[m.group(2)] = (m.start(), _block_end(src, m.end() - 1), m.end())
    return funcs


def prune_unreachable(src: str) -> str:
    """Drop what main cannot reach: statements after a function's top-level
    return, then top-level functions main never calls (transitively), then
    top-level constants no remaining code names."""
    out, i = [], 0
    for name, (a, b, body) in sorted(_functions(src).items(), key=lambda kv: kv[1][0]):
        out.append(src[i:a])
        text = src[a:b]
        k, depth, cut = body - a, 1, None
        while k < len(text) - 1:
            c = text[k]
            depth += c == "{"
            depth -= c == "}"
            # a return that is a statement of the body itself, not the
            # unbraced branch of an if / else / loop
            if (depth == 1 and re.match(r"return\b", text[k:]) and not re.match(r"\w", text[k - 1])
                    and text[:k].rstrip()[-1:] in (";", "{", "}")):
                cut = text.index(";", k) + 1
                break
            k += 1
        out.append(text[:cut] + "\n}" if cut else text)
        i = b
    out.append(src[i:])
    src = "".join(out)
    funcs = _functions(src)
    keep, todo = set(), ["main"]
    while todo:
        f = todo.pop()
        if f in keep or f not in funcs:
            continue
        keep.add(f)
        a, b, _ = funcs[f]
        todo += [c for c in re.findall(r"\b(\w+)\s*\(", src[a:b]) if c in funcs]
    for name, (a, b, _) in sorted(funcs.items(), key=lambda kv: -kv[1][0]):
        if name not in keep:
            src = src[:a] + src[b:]
    for m in list(re.finditer(r"^\s*const\s+\w+\s+(\w+)\s*=[^;]*;[ \t]*\n", src, re.M)):
        if len(re.findall(r"\b" + m.group(1) + r"\b", src)) == 1:
            src = src.replace(m.group(0), "\n", 1)
    return src


def scope_for_init(src: str) -> str:
    """GLSL scopes a for-init declaration from after its initializer, so
    `for (float t = t; ...)` starts from the enclosing t; C++ would read the
    new, uninitialised t.  Rename the loop variable within the loop."""
    pat = re.compile(r"for\s*\(\s*(\w+)\s+(\w+)\s*=\s*\2\s*;")
    while True:
        m = pat.search(src)
        if not m:
            return src
        ty, var = m.group(1), m.group(2)
        new = var + "_loop"
        hdr_end = src.index(")", m.end())
        body_open = src.index("{", hdr_end)
        end = _block_end(src, body_open)
        loop = src[m.end():end]
        loop = re.sub(r"\b" + var + r"\b", new, loop)
        src = src[:m.start()] + f"for ({ty} {new} = {var};" + loop + src[end:]


def translate(name: str, src: str) -> str:
    src = strip_comments(src)
    if name in PRUNE_SHADERS:
        src = prune_unreachable(src)
    src = scope_for_init(src)
    src = re.sub(r"^\s*#(version|extension)[^\n]*\n", "", src, flags=re.M)
    src = src.replace("#define WORKGROUP_SIZE gl_WorkGroupSize.x", "#define WORKGROUP_SIZE 256u")
    src = re.sub(r"layout\s*\([^)]*\)\s*in\s*;", "", src)
    src = re.sub(r"layout\s*\(\s*constant_id\s*=\s*\d+\s*\)\s*const\s+(\w+)\s+(\w+)\s*=\s*([^;]+);",
                 r"static constexpr \1 \2 = \3;", src)
    images = re.findall(r"layout\s*\([^)]*\)\s*uniform\s+writeonly\s+image3D\s+(\w+)\s*;", src)
    images2 = re.findall(r"layout\s*\([^)]*\)\s*uniform\s+writeonly\s+image2D\s+(\w+)\s*;", src)
    samplers = re.findall(r"layout\s*\(\s*binding\s*=\s*(\d+)\s*\)\s*uniform\s+sampler3D\s+(\w+)\s*;", src)
    src = re.sub(r"layout\s*\(\s*binding\s*=\s*(\d+)\s*\)\s*uniform\s+sampler3D\s+(\w+)\s*;",
                 r"Sampler3D \2;", src)
    # fragment-stage interface: inputs and outputs become members, samplers
    # of 2-D images Sampler2D
    src = re.sub(r"layout\s*\(\s*location\s*=\s*\d+\s*\)\s*(?:flat\s+)?(?:in|out)\s+(\w+)\s+(\w+)\s*;",
                 r"\1 \2 = {};", src)
    src = re.sub(r"layout\s*\(\s*binding\s*=\s*(\d+)\s*\)\s*uniform\s+sampler2D\s+(\w+)\s*;",
                 r"Sampler2D \2;", src)
    if name in RENDER_SHADERS:
        src = re.sub(r"layout\s*\([^)]*\)\s*uniform\s+writeonly\s+image2D\s+(\w+)\s*;", r"Image2D \1;", src)
    else:
        images2 = []
    images_ro = re.findall(r"layout\s*\([^)]*\)\s*uniform\s+readonly\s+image3D\s+(\w+)\s*;", src)
    src = re.sub(r"layout\s*\([^)]*\)\s*uniform\s+(?:writeonly|readonly)\s+image3D\s+(\w+)\s*;",
                 r"Image3D \1;", src)
    src = re.sub(r"layout\s*\([^)]*\)\s*uniform\s+writeonly\s+image\w+\s+\w+\s*;", "", src)
    # uniform / push-constant blocks -> plain members
    src = re.sub(r"layout\s*\([^)]*\)\s*uniform\s+\w+\s*\{(.*?)\}\s*;", r"\1", src, flags=re.S)
    src = re.sub(r"\bdiscard\s*;", "{ discarded = true; return; }", src)
    # single-array buffer blocks -> pointers, remember their bindings
    bindings = []

    def buf(m):
        args, ty, var = m.group(1), m.group(2), m.group(3)
        b = int(re.search(r"binding\s*=\s*(\d+)", args).group(1))
        bindings.append((b, ty, var))
        return f"{ty}* {var} = nullptr;"

    src = re.sub(r"layout\s*\(([^)]*)\)\s*(?:readonly\s+|writeonly\s+)?buffer\s+\w+\s*\{\s*(\w+)\s+(\w+)\s*\[\s*\]\s*;\s*\}\s*;",
                 buf, src)
    shared = []

    def sh(m):
        ty, count, var = m.group(1), m.group(2), m.group(3)
        shared.append((ty, count, var))
        return f"{ty}* {var} = nullptr;"

    src = re.sub(r"shared\s+(\w+)\s*\[([^\]]+)\]\s*(\w+)\s*;", sh, src)
    src = re.sub(r"\b(?:out|inout)\s+(\w+)\s+(\w+)\s*(?=[,)])", r"\1& \2", src)
    src = FLOAT_LIT.sub(lambda m: m.group(1) + "f", src)
    src = re.sub(r"\.xyz\b", ".xyz()", src)
    src = re.sub(r"\.xy\b", ".xy()", src)
    src = re.sub(r"\.rgb\b", ".xyz()", src)
    src = re.sub(r"\.r\b", ".x", src)
    src = re.sub(r"\.g\b", ".y", src)
    src = re.sub(r"\.b\b", ".z", src)
    src = construct_structs(src)
    if "layout" in src or re.search(r"\bbuffer\b", src):
        raise SystemExit(f"{name}: untranslated declaration left")
    bind_cases = "\n".join(
        f"            case {b}: {var} = static_cast<{ty}*>(p); break;" for b, ty, var in bindings)
    shared_lines = "\n".join(
        f"        {var} = reinterpret_cast<{ty}*>(s + o); o += sizeof({ty}) * ({count}); "
        f"o = (o + 15) & ~size_t(15);" for ty, count, var in shared)
    local = LOCAL_SIZE.get(name, 128)
    threads = "true" if name in WORKGROUP_THREADS else "false"
    extra = ""
    image_bind = f"{images[0]} = im;" if images else "(void)im;"
    rt_lines = []
    if images:
        rt_lines.append(f"{images[0]} = rb.img3;")
    if images2:
        rt_lines.append(f"{images2[0]} = rb.img2;")
    for nm in images_ro:
        rt_lines.append(f"{nm} = rb.img3;")
    for b, nm in samplers:
        rt_lines.append(f"{nm} = rb.tex[{b}];")
    rt_bind = " ".join(rt_lines) if rt_lines else "(void)rb;"
    if name in RENDER_SHADERS:
        extra += f"""
extern "C" void ref_dispatch_rt_{name}(const glsl::RefUbo* u, void* const* bindings, glsl::uint nx,
                                       glsl::uint ny, glsl::uint nz, const glsl::RtBind* rb) {{
    glsl::dispatch_rt<glsl::ref_{name}::Shader>(*u, bindings, nx, ny, nz, *rb);
}}
"""
    if name == "shader_vert":
        extra += f"""
// one vertex: quad corner quadPos of instance `instance` at particlePos
extern "C" void ref_vertex_{name}(const glsl::RefUbo* u, float qx, float qy, const float pos[3], int instance,
                                  float clip[4]) {{
    glsl::ref_{name}::Shader s;
    glsl::set_uniforms(s, *u);
    s.quadPos = glsl::vec2(qx, qy);
    s.particlePos = glsl::vec3(pos[0], pos[1], pos[2]);
    s.gl_InstanceIndex = instance;
    s.main();
    clip[0] = s.gl_Position.x; clip[1] = s.gl_Position.y; clip[2] = s.gl_Position.z; clip[3] = s.gl_Position.w;
}}
"""
    if name == "shader_frag":
        extra += f"""
// one fragment of particle `index` at fragQuadPos; returns 1 if discarded
extern "C" int ref_fragment_{name}(const glsl::RefUbo* u, void* const* bindings, int index, float qx, float qy,
                                   float out[4]) {{
    glsl::ref_{name}::Shader s;
    glsl::set_uniforms(s, *u);
    for (int b = 0; b < 32; b++)
        if (bindings[b]) s.bind(b, bindings[b]);
    s.particleIndex = index;
    s.fragQuadPos = glsl::vec2(qx, qy);
    s.shouldDiscard = 0;
    s.main();
    out[0] = s.outColor.x; out[1] = s.outColor.y; out[2] = s.outColor.z; out[3] = s.outColor.w;
    return s.discarded ? 1 : 0;
}}
"""
    if name in FRAG_SHADERS:
        extra += f"""
// one fragment per pixel of a width x height target: outNDC at the pixel
// centre, ((x + 0.5) / width * 2 - 1, (y + 0.5) / height * 2 - 1)
extern "C" void ref_fragment_{name}(const float* img, int w, int h, float* out) {{
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {{
            glsl::ref_{name}::Shader s;
            s.outputImage.data = img; s.outputImage.nx = w; s.outputImage.ny = h;
            s.outNDC = glsl::vec2(((float)x + 0.5f) / (float)w * 2.0f - 1.0f,
                                  ((float)y + 0.5f) / (float)h * 2.0f - 1.0f);
            s.main();
            float* q = out + 4 * ((size_t)y * w + x);
            q[0] = s.outColor.x; q[1] = s.outColor.y; q[2] = s.outColor.z; q[3] = s.outColor.w;
        }}
}}
"""
    if images:
        extra += f"""
extern "C" void ref_dispatch3_{name}(const glsl::RefUbo* u, void* const* bindings, glsl::uint nx,
                                     glsl::uint ny, glsl::uint nz, float* img, int ix, int iy, int iz) {{
    glsl::Image3D im;
    im.data = img; im.nx = ix; im.ny = iy; im.nz = iz;
    glsl::dispatch3<glsl::ref_{name}::Shader>(*u, bindings, nx, ny, nz, im);
}}
"""
    if "cellCoordToHash" in src and name not in RENDER_SHADERS:
        extra += f"""
extern "C" glsl::uint ref_hash_{name}(glsl::uint x, glsl::uint y, glsl::uint z) {{
    glsl::ref_{name}::Shader s;
    return s.cellCoordToHash(glsl::uvec3(x, y, z));
}}
"""
    return f"""// GENERATED by oracle/glsl_ref.py from the reference's src/shaders/{name}.comp.
// Not committed; rebuilt by __graft_entry__.build() where the sources exist.
#include <cstddef>
#include "glsl_dispatch.hpp"

namespace glsl {{
namespace ref_{name} {{
struct Shader : Invocation {{
{src}
    void bind(int binding, void* p) {{
        switch (binding) {{
{bind_cases}
            default: break;
        }}
    }}
    void bind_image(Image3D im) {{
        {image_bind}
    }}
    void bind_rt(const RtBind& rb) {{
        {rt_bind}
    }}
    void bind_shared(char* s) {{
        size_t o = 0;
        (void)s; (void)o;
{shared_lines}
    }}
}};
}}  // namespace ref_{name}
}}  // namespace glsl

extern "C" void ref_dispatch_{name}(const glsl::RefUbo* u, void* const* bindings, glsl::uint groups,
                                    glsl::InvocationHook hook, void* ctx) {{
    glsl::dispatch<glsl::ref_{name}::Shader>(*u, bindings, groups, {local}u, {threads}, hook, ctx);
}}
{extra}"""


def build() -> str:
    os.makedirs(GEN, exist_ok=True)
    srcs = []
    for name in SHADERS:
        with open(os.path.join(REF_SHADERS, shader_file(name))) as f:
            code = translate(name, f.read())
        path = os.path.join(GEN, name + ".cpp")
        with open(path, "w") as f:
            f.write(code)
        srcs.append(path)
    cmd = ["g++", "-O2", "-std=c++20", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-pthread", "-w", "-I", HERE, "-o", LIB, os.path.join(HERE, "glsl_driver.cpp")] + srcs
    subprocess.run(cmd, check=True)
    return LIB


class RefParams(ctypes.Structure):
    _fields_ = [
        ("particleRadius", ctypes.c_float), ("smoothingRadius", ctypes.c_float),
        ("g", ctypes.c_float), ("minXYZ", ctypes.c_float * 3), ("dt", ctypes.c_float),
        ("maxXYZ", ctypes.c_float * 3), ("particleMass", ctypes.c_float),
        ("pressureMultiplier", ctypes.c_float), ("targetDensity", ctypes.c_float),
        ("viscosityStrength", ctypes.c_float), ("volume", ctypes.c_float),
        ("nearPressureMultiplier", ctypes.c_float), ("numBlocksPerWorkGroup", ctypes.c_uint32),
    ]


TRACE_KEYS = ("keys_in", "keys", "perm", "start", "end", "xp", "vp", "density", "near_density",
              "vel_force", "colors")


def load():
    if not os.path.exists(LIB):
        build()
    L = ctypes.CDLL(LIB)
    L.ref_substep.restype = ctypes.c_int
    L.ref_substep.argtypes = [ctypes.POINTER(RefParams), ctypes.c_uint32, ctypes.c_void_p,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    return L


def ref_params_from(case: dict) -> RefParams:
    import math
    p = RefParams()
    p.particleRadius = case["radius"]
    p.smoothingRadius = case["h"]
    p.g = case["g"]
    for a in range(3):
        p.minXYZ[a] = case["box_min"][a]
        p.maxXYZ[a] = case["box_max"][a]
    p.dt = case["dt"]
    p.particleMass = case["mass"]
    p.pressureMultiplier = case["k"]
    p.targetDensity = case["rho0"]
    p.viscosityStrength = 0.0
    # main.c:349 in double precision, stored as float
    import numpy as np
    p.volume = float(np.float32(2.0 * math.pi * math.pow(float(np.float32(case["h"])), 5) / 15.0))
    p.nearPressureMultiplier = case["kn"]
    p.numBlocksPerWorkGroup = 128
    return p


def run_case(L, case: dict, pos, vel):
    import numpy as np
    n = pos.shape[0]
    pos = np.ascontiguousarray(pos, np.float32).copy()
    vel = np.ascontiguousarray(vel, np.float32).copy()
    tr = {
        "keys_in": np.empty(n, np.uint32), "keys": np.empty(n, np.uint32),
        "perm": np.empty(n, np.uint32), "start": np.empty(n, np.int32), "end": np.empty(n, np.int32),
        "xp": np.empty((n, 4), np.float32), "vp": np.empty((n, 4), np.float32),
        "density": np.empty(n, np.float32), "near_density": np.empty(n, np.float32),
        "vel_force": np.empty((n, 4), np.float32), "colors": np.empty((n, 4), np.float32),
    }
    ptrs = (ctypes.c_void_p * len(TRACE_KEYS))(*[tr[k].ctypes.data for k in TRACE_KEYS])
    p = ref_params_from(case)
    rc = L.ref_substep(ctypes.byref(p), n, pos.ctypes.data, vel.ctypes.data,
                       ctypes.cast(ptrs, ctypes.c_void_p), 1)
    if rc != 0:
        raise RuntimeError("ref_substep failed")
    tr["pos"] = pos
    tr["vel"] = vel
    return tr


def golden_cases():
    """Seeded inputs in the reference's parameter form (gravity along -z,
    wall margins r and r + 0.5, z-min restitution 0.95, unscaled viscosity)."""
    import numpy as np
    cases = []
    # 1. the reference's own scene parameters (main.c:11-30) on a small slab
    #    in a box shrunk so the slab has neighbours
    cases.append(dict(name="ref_default_small", n=3000, seed=10, h=2.5, g=100.0, dt=0.01,
                      mass=1.0, k=15000.0, rho0=1.0, kn=0.0, radius=0.3,
                      box_min=(-14.0, -8.0, -8.0), box_max=(14.0, 8.0, 8.0),
                      init=("slab", (-6.0, -4.0, -6.0), (2.0, 4.0, 2.0)), v=(0.0, 0.0, -100.0)))
    # 2. near pressure on, different h, particles close to every wall
    cases.append(dict(name="near_walls", n=2500, seed=11, h=0.9, g=9.81, dt=0.005,
                      mass=0.6, k=400.0, rho0=2.0, kn=30.0, radius=0.1,
                      box_min=(0.0, 0.0, 0.0), box_max=(8.0, 6.0, 5.0),
                      init=("box", (0.0, 0.0, 0.0), (8.0, 6.0, 5.0)), v=None))
    # 3. non-power-of-two particle count (the key mask is then sparse) and
    #    two workgroups' worth of sort blocks (> 16384 elements)
    cases.append(dict(name="npot_two_groups", n=20001, seed=12, h=1.5, g=50.0, dt=0.008,
                      mass=1.0, k=2000.0, rho0=1.5, kn=5.0, radius=0.3,
                      box_min=(-20.0, -10.0, -10.0), box_max=(20.0, 10.0, 10.0),
                      init=("slab", (-15.0, -8.0, -9.0), (5.0, 8.0, 3.0)), v=(3.0, -2.0, -20.0)))
    # 4. tiny counts: the sort's ballot ranks and the table edge cases
    cases.append(dict(name="tiny_n2", n=2, seed=13, h=1.0, g=10.0, dt=0.01, mass=1.0, k=100.0,
                      rho0=1.0, kn=1.0, radius=0.0, box_min=(0.0, 0.0, 0.0),
                      box_max=(4.0, 4.0, 4.0), init=("box", (1.0, 1.0, 1.0), (1.6, 1.6, 1.6)),
                      v=None))
    cases.append(dict(name="small_n64", n=64, seed=14, h=1.0, g=10.0, dt=0.01, mass=1.0,
                      k=100.0, rho0=1.0, kn=1.0, radius=0.0, box_min=(0.0, 0.0, 0.0),
                      box_max=(4.0, 4.0, 4.0), init=("box", (0.5, 0.5, 0.5), (3.0, 3.0, 3.0)),
                      v=None))
    # 5. NaN velocities in a dense cluster: their predicted positions are NaN,
    #    so every neighbour meets a NaN distance; the shaders' tests do not
    #    skip it, and the NaN reaches the neighbours' sums
    cases.append(dict(name="nan_neighbours", n=512, seed=15, h=1.0, g=10.0, dt=0.01, mass=1.0,
                      k=100.0, rho0=1.0, kn=1.0, radius=0.0, box_min=(0.0, 0.0, 0.0),
                      box_max=(4.0, 4.0, 4.0), init=("box", (0.5, 0.5, 0.5), (2.5, 2.5, 2.5)),
                      v=None, nan_rows=[3, 100, 511]))
    out = []
    for c in cases:
        rng = np.random.default_rng(c["seed"])
        n = c["n"]
        pos = np.zeros((n, 4), np.float32)
        lo, hi = np.array(c["init"][1]), np.array(c["init"][2])
        pos[:, :3] = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
        vel = np.zeros((n, 4), np.float32)
        if c["v"] is None:
            vel[:, :3] = rng.normal(0.0, 3.0, (n, 3)).astype(np.float32)
        else:
            vel[:, :3] = np.array(c["v"], np.float32)
        for r in c.get("nan_rows", ()):
            vel[r, :3] = np.float32("nan")
        out.append((c, pos, vel))
    return out


def _digest(a) -> str:
    import hashlib
    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


HASH_COORDS = [
    (0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 2, 3), (3, 2, 1), (12, 34, 56),
    (111, 0, 7), (1023, 1023, 1023), (0xFFFFFFFF, 0, 5), (0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF),
    (0xFFFFFFFE, 1, 0), (0x80000000, 0x7FFFFFFF, 3), (65536, 65535, 4096),
    (0xDEADBEEF, 0x12345678, 0x0BADF00D),
]


def golden() -> None:
    """Fixtures from the reference shaders: full arrays for cases up to 4096
    particles, sha256 digests of every stage output for all cases, spatial
    hash vectors and radix-sort known answers."""
    import json
    import numpy as np
    L = load()
    os.makedirs(GOLDEN, exist_ok=True)
    index = []
    for case, pos, vel in golden_cases():
        tr = run_case(L, case, pos, vel)
        meta = {k: v for k, v in case.items() if k != "init"}
        meta["init"] = [case["init"][0], list(case["init"][1]), list(case["init"][2])]
        meta["digest_in"] = {"pos": _digest(pos), "vel": _digest(vel)}
        meta["digest"] = {k: _digest(v) for k, v in tr.items()}
        if case["n"] <= 4096:
            path = os.path.join(GOLDEN, f"glsl_{case['name']}.npz")
            np.savez_compressed(path, pos_in=pos, vel_in=vel, **tr)
            meta["arrays"] = os.path.basename(path)
        index.append(meta)
    with open(os.path.join(GOLDEN, "glsl_cases.json"), "w") as f:
        json.dump(index, f, indent=1)

    # cellCoordToHash from every shader that carries a copy of it
    copies = [n for n in SHADERS if hasattr(L, f"ref_hash_{n}")]
    vec = []
    for (x, y, z) in HASH_COORDS:
        vals = set()
        for n in copies:
            fn = getattr(L, f"ref_hash_{n}")
            fn.restype = ctypes.c_uint32
            fn.argtypes = [ctypes.c_uint32] * 3
            vals.add(int(fn(x, y, z)))
        if len(vals) != 1:
            raise SystemExit(f"shader copies of cellCoordToHash disagree at {(x, y, z)}")
        vec.append({"cell": [x, y, z], "hash": vals.pop()})
    with open(os.path.join(GOLDEN, "glsl_hash.json"), "w") as f:
        json.dump({"copies": copies, "vectors": vec}, f, indent=1)

    # radix sort known answers (testSort, main.c:274-338, made assertive)
    L.ref_sort.restype = ctypes.c_int
    L.ref_sort.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                           ctypes.c_void_p]
    rng = np.random.default_rng(99)
    sort_cases = {
        "shuffled_perm_20000": rng.permutation(20000).astype(np.uint32),
        "dup_16_5000": rng.integers(0, 16, 5000).astype(np.uint32),
        "all_equal_3000": np.full(3000, 7, np.uint32),
        "full_range_4000": rng.integers(0, 2**32, 4000, dtype=np.uint64).astype(np.uint32),
        "small_7": np.array([5, 3, 5, 0, 3, 3, 1], np.uint32),
    }
    out = {}
    summary = {}
    for name, keys in sort_cases.items():
        ok = np.empty_like(keys)
        ov = np.empty_like(keys)
        L.ref_sort(keys.size, keys.ctypes.data, 128, ok.ctypes.data, ov.ctypes.data)
        summary[name] = {"n": int(keys.size), "keys": _digest(keys), "sorted": _digest(ok),
                         "perm": _digest(ov)}
        if keys.size <= 5000:
            out[name + "_keys"] = keys
            out[name + "_sorted"] = ok
            out[name + "_perm"] = ov
    np.savez_compressed(os.path.join(GOLDEN, "glsl_sort.npz"), **out)
    with open(os.path.join(GOLDEN, "glsl_sort.json"), "w") as f:
        json.dump(summary, f, indent=1)
    print(f"wrote {len(index)} step cases, {len(vec)} hash vectors, {len(summary)} sort cases "
          f"to {GOLDEN}")


MAP_CELL_FACTORS = (1.0, 0.7, 1.6)


def map_image_dims(box_min, box_max, cell_size):
    """The image renderer.c:774-781 allocates: (int)ceil((max - min) * (1 / cs))
    per axis in float."""
    import numpy as np
    cs = np.float32(cell_size)
    inv = np.float32(np.float32(1.0) / cs)
    return tuple(int(np.ceil(np.float64(np.float32(np.float32(np.float32(box_max[a]) -
                                                              np.float32(box_min[a])) * inv))))
                 for a in range(3))


def golden_map() -> None:
    """Density maps (updateDensityMap.comp) from the reference shader, on the
    state after one reference substep of each step case whose image is small,
    at cell sizes h x MAP_CELL_FACTORS: tests/golden/glsl_density_map.npz."""
    import numpy as np
    L = load()
    L.ref_density_map.restype = ctypes.c_int
    L.ref_density_map.argtypes = [ctypes.POINTER(RefParams), ctypes.c_uint32, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    out = {}
    names = []
    for case, pos, vel in golden_cases():
        if case["n"] > 4096:
            continue
        tr = run_case(L, case, pos, vel)
        p = ref_params_from(case)
        n = case["n"]
        spos = np.ascontiguousarray(tr["pos"], np.float32)
        start = np.ascontiguousarray(tr["start"], np.int32)
        end = np.ascontiguousarray(tr["end"], np.int32)
        nm = case["name"]
        names.append(nm)
        out[f"{nm}__pos"] = spos
        out[f"{nm}__keys"] = np.ascontiguousarray(tr["keys"], np.uint32)
        out[f"{nm}__scalars"] = np.array([case["h"], case["mass"], p.volume, *case["box_min"],
                                          *case["box_max"]], np.float32)
        for f in MAP_CELL_FACTORS:
            cs = float(np.float32(np.float32(case["h"]) * np.float32(f)))
            ix, iy, iz = map_image_dims(case["box_min"], case["box_max"], cs)
            img = np.zeros((iz, iy, ix), np.float32)
            L.ref_density_map(ctypes.byref(p), n, spos.ctypes.data, start.ctypes.data,
                              end.ctypes.data, cs, ix, iy, iz, img.ctypes.data)
            out[f"{nm}__map{f}"] = img
            out[f"{nm}__cs{f}"] = np.array([cs], np.float32)
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(GOLDEN, "glsl_density_map.npz"), **out)
    print(f"wrote density maps of {len(names)} cases x {len(MAP_CELL_FACTORS)} cell sizes")


def golden_render() -> None:
    """Volumetric render mode from the reference shaders (calculateLightVolume,
    volumetricFluid) and refractive mode (properFluid) on the reference-computed
    density maps of golden_map's cases at cell size h:
    tests/golden/glsl_render.npz."""
    import math
    import numpy as np
    L = load()
    f32 = np.float32
    dm = np.load(os.path.join(GOLDEN, "glsl_density_map.npz"))
    vp, fl, i32 = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
    L.ref_light_volume.restype = i32
    L.ref_light_volume.argtypes = [ctypes.POINTER(RefParams), vp, vp, fl, vp, vp, vp]
    L.ref_volumetric.restype = i32
    L.ref_volumetric.argtypes = [ctypes.POINTER(RefParams), vp, vp, vp, vp, vp, fl, fl, vp, i32, i32, vp]
    L.ref_fragment_raymarchShader.restype = None
    L.ref_fragment_raymarchShader.argtypes = [vp, i32, i32, vp]
    L.ref_refractive.restype = i32
    L.ref_refractive.argtypes = [ctypes.POINTER(RefParams), vp, vp, vp, fl, fl, fl, vp, i32, fl, fl, i32,
                                 i32, vp]
    out = {}
    names = []
    for case, pos, vel in golden_cases():
        nm = case["name"]
        if f"{nm}__map1.0" not in dm.files:
            continue
        p = ref_params_from(case)
        dmap = np.ascontiguousarray(dm[f"{nm}__map1.0"], np.float32)
        ddims = np.array(dmap.shape[::-1], np.int32)
        lo, hi = np.array(case["box_min"], np.float32), np.array(case["box_max"], np.float32)
        size = hi - lo
        light_step = 1.0
        ldims = np.array(map_image_dims(case["box_min"], case["box_max"], light_step), np.int32)
        sun = np.array([0.75, -0.25, 0.5], np.float32)
        sun = sun / f32(np.sqrt(f32(np.dot(sun, sun))))
        lvol = np.zeros(ldims[::-1], np.float32)
        L.ref_light_volume(ctypes.byref(p), dmap.ctypes.data, ddims.ctypes.data, ctypes.c_float(light_step),
                           sun.ctypes.data, ldims.ctypes.data, lvol.ctypes.data)
        centre = (lo + hi) * f32(0.5)
        cam = np.array([centre[0], lo[1] - f32(0.75) * size[1], centre[2], 0, 1, 0, 1, 0, 0, 0, 0, 1],
                       np.float32)
        fov = f32(0.9 * math.pi / 2)
        step = f32(float(min(size)) / 40.0)
        ext = np.array([0.02, 0.02, 0.01], np.float32)
        W, H = 32, 24
        rgba = np.zeros((H, W, 4), np.float32)
        L.ref_volumetric(ctypes.byref(p), dmap.ctypes.data, ddims.ctypes.data, lvol.ctypes.data,
                         ldims.ctypes.data, cam.ctypes.data, ctypes.c_float(fov), ctypes.c_float(step),
                         ext.ctypes.data, W, H, rgba.ctypes.data)
        names.append(nm)
        out[f"{nm}__lvol"] = lvol
        out[f"{nm}__rgba"] = rgba
        out[f"{nm}__view"] = np.concatenate([cam, [fov, step, light_step], ext, sun]).astype(np.float32)
        # refractive mode (properFluid.comp) with the same camera, surface
        # threshold at the map's 40th percentile of non-zero voxels
        nz = dmap[dmap > 0]
        thr = f32(np.percentile(nz, 40)) if nz.size else f32(0.5)
        refr = np.zeros((H, W, 4), np.float32)
        L.ref_refractive(ctypes.byref(p), dmap.ctypes.data, ddims.ctypes.data, cam.ctypes.data,
                         ctypes.c_float(fov), ctypes.c_float(step), ctypes.c_float(light_step),
                         ext.ctypes.data, 3, ctypes.c_float(thr), ctypes.c_float(1.333), W, H,
                         refr.ctypes.data)
        out[f"{nm}__refr"] = refr
        out[f"{nm}__refr_args"] = np.array([thr, 1.333, 3], np.float32)
        # the presentation pass (raymarchShader.frag's FXAA) of both images
        for key, src in (("rgba", rgba), ("refr", refr)):
            fx = np.zeros_like(src)
            L.ref_fragment_raymarchShader(np.ascontiguousarray(src).ctypes.data, W, H, fx.ctypes.data)
            out[f"{nm}__fxaa_{key}"] = fx
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(GOLDEN, "glsl_render.npz"), **out)
    print(f"wrote light volumes and images of {len(names)} cases")


def golden_raster() -> None:
    """The rasterisation pipeline's programmable stages from the reference's
    shader.vert / shader.frag on seeded particles and a camera the way
    updateUniforms (main.c:37-51) builds the UBO: clip positions of each
    particle's quad corners (and centre), and fragment outputs at a grid of
    fragQuadPos values (discards included): tests/golden/glsl_raster.npz."""
    import math
    import numpy as np
    sys.path.insert(0, ROOT)
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "pfs_pkg", os.path.join(ROOT, "particle-fluid-simulation_b200", "__init__.py"),
        submodule_search_locations=[os.path.join(ROOT, "particle-fluid-simulation_b200")])
    pkg = importlib.util.module_from_spec(spec)
    sys.modules["pfs_pkg"] = pkg
    spec.loader.exec_module(pkg)
    L = load()
    vp, fl, i32 = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
    L.ref_splat_vertex.restype = None
    L.ref_splat_vertex.argtypes = [vp, vp, vp, fl, fl, fl, vp, i32, vp]
    L.ref_splat_fragment.restype = i32
    L.ref_splat_fragment.argtypes = [vp, i32, fl, fl, vp]
    rng = np.random.default_rng(31)
    n = 64
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-30.0, 30.0, (n, 3)).astype(np.float32)
    col = np.ones((n, 4), np.float32)
    col[:, :3] = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    W, H = 1280, 720
    view = pkg.splat_view((3.0, -100.0, 10.0), (0.1, 1.0, -0.05), W, H, 0.3)
    mats = [np.ascontiguousarray(np.array(m[:], np.float32)) for m in (view.model, view.view, view.proj)]
    corners = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1], [0, 0]], np.float32)
    clip = np.zeros((n, len(corners), 4), np.float32)
    for i in range(n):
        p3 = np.ascontiguousarray(pos[i, :3])
        for c, (qx, qy) in enumerate(corners):
            out = np.zeros(4, np.float32)
            L.ref_splat_vertex(mats[0].ctypes.data, mats[1].ctypes.data, mats[2].ctypes.data, 0.3, float(qx),
                               float(qy), p3.ctypes.data, i, out.ctypes.data)
            clip[i, c] = out
    g = np.linspace(-1.1, 1.1, 23).astype(np.float32)
    qs = np.array([(a, b) for a in g for b in g], np.float32)
    frag = np.zeros((8, len(qs), 4), np.float32)
    disc = np.zeros((8, len(qs)), np.int32)
    for i in range(8):
        for k, (qx, qy) in enumerate(qs):
            out = np.zeros(4, np.float32)
            disc[i, k] = L.ref_splat_fragment(col.ctypes.data, i, float(qx), float(qy), out.ctypes.data)
            frag[i, k] = out
    np.savez_compressed(os.path.join(GOLDEN, "glsl_raster.npz"), pos=pos, col=col,
                        model=mats[0], view=mats[1], proj=mats[2], radius=np.float32(0.3), corners=corners,
                        clip=clip, qs=qs, frag=frag, discarded=disc)
    print(f"wrote vertex outputs of {n} particles and {8 * len(qs)} fragments")


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "build"
    if what == "build":
        print(build())
    elif what == "golden":
        golden()
    elif what == "golden_map":
        golden_map()
    elif what == "golden_render":
        golden_render()
    elif what == "golden_raster":
        golden_raster()
    else:
        raise SystemExit("usage: glsl_ref.py build|golden|golden_map|golden_render|golden_raster")
