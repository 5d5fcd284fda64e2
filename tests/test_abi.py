"""The C-ABI library loads on any machine and exports every entry point that
include/pfs.h declares; host-side validation works without a GPU."""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available, load_oracle, load_package

HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def _declared():
    names = []
    for h in HEADERS:
        with open(h) as f:
            src = f.read()
        names += re.findall(r"^PFS_API\s+[\w\s\*]+?\b(pfs_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = _declared()
    for must in ("pfs_world_create", "pfs_world_step", "pfs_world_sync", "pfs_world_read",
                 "pfs_world_write", "pfs_world_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol():
    pfs = load_package()
    path = pfs.LIB_PATH
    assert os.path.exists(path), "libpfs.so not built"
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\s[TW]\s+(pfs_\w+)$", out, flags=re.M))
    missing = [n for n in _declared() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    lib = ctypes.CDLL(path)
    for n in _declared():
        assert getattr(lib, n) is not None


def test_params_struct_layout():
    pfs = load_package()
    # 25 floats then substeps, precision, flags, reserved (include/pfs.h)
    assert ctypes.sizeof(pfs.Params) == 4 * 29
    assert pfs.Params.substeps.offset == 4 * 25


def test_validation_without_gpu():
    pfs = load_package()
    L = pfs.lib()
    p = pfs.reference_default()
    assert L.pfs_params_validate(ctypes.byref(p)) == pfs.PFS_OK
    for field, bad in (("h", 0.0), ("h", float("nan")), ("dt", -1.0), ("substeps", 0),
                       ("precision", 7), ("flags", 1 << 20)):
        q = p.copy()
        setattr(q, field, bad)
        assert L.pfs_params_validate(ctypes.byref(q)) == pfs.PFS_EINVAL, field
    q = p.copy()
    q.box_min[0] = q.box_max[0]
    assert L.pfs_params_validate(ctypes.byref(q)) == pfs.PFS_EINVAL
    # the FP16-cell form packs cells into 10-bit fields: huge boxes are refused
    q = p.copy()
    q.precision = pfs.PFS_FP16_CELL
    assert L.pfs_params_validate(ctypes.byref(q)) == pfs.PFS_OK  # 112 cells along x
    q.h = 0.1
    assert L.pfs_params_validate(ctypes.byref(q)) == pfs.PFS_EINVAL
    assert L.pfs_strerror(pfs.PFS_ETIMEDOUT) == b"timed out"


def test_create_rejects_bad_sizes_before_touching_the_device():
    pfs = load_package()
    L = pfs.lib()
    p = pfs.reference_default()
    h = ctypes.c_void_p()
    pos = np.zeros((4, 4), np.float32)
    assert L.pfs_world_create(ctypes.byref(p), 0, pos.ctypes.data, None, ctypes.byref(h)) == pfs.PFS_EINVAL
    assert L.pfs_world_create(ctypes.byref(p), pfs.PFS_MAX_PARTICLES + 1, pos.ctypes.data, None,
                              ctypes.byref(h)) == pfs.PFS_ERANGE
    assert L.pfs_world_create(ctypes.byref(p), 4, None, None, ctypes.byref(h)) == pfs.PFS_EINVAL


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    pfs = load_package()
    p = pfs.reference_default()
    with pytest.raises(pfs.PfsError) as ei:
        pfs.World(p, np.zeros((8, 4), np.float32))
    assert ei.value.status == pfs.PFS_ENODEV


def test_c_host_builds_and_runs(tmp_path):
    """A C99 host (tests/c/host_stub.c) compiles against the header, links
    against the library and runs: on a machine without a GPU every call
    reports a status (PFS_ENODEV) and the process exits normally."""
    pfs = load_package()
    exe = str(tmp_path / "host_stub")
    libdir = os.path.dirname(pfs.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", "host_stub.c"),
                    "-L", libdir, "-lpfs", "-Wl,-rpath," + libdir, "-o", exe], check=True)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    m = re.match(r"status (-?\d+): ", p.stdout)
    assert m, p.stdout
    if not gpu_available():
        assert int(m.group(1)) == pfs.PFS_ENODEV, p.stdout


def test_batch_bytes_without_gpu():
    """pfs_batch_bytes is host arithmetic: monotone in particles and scenes,
    about 2.3 KB per particle (512 neighbour-list rows of 4 bytes dominate)."""
    pfs = load_package()
    f = pfs.Batch.bytes_for
    for prec in (pfs.PFS_FP32, pfs.PFS_FP16_CELL):
        a, b = f(1 << 20, 256, prec), f(1 << 21, 256, prec)
        assert b > a and f(1 << 20, 512, prec) > a
        assert 2.1e3 < a / (1 << 20) < 2.5e3
        assert (b - a) / (1 << 20) > 512 * 4  # the list rows alone


@pytest.mark.gpu
def test_c_host_steps_a_world_on_the_gpu(cuda_device, tmp_path):
    """The same C99 host on a GPU: it creates a world, steps it once (3
    substeps), reads the positions back and renders a frame, all with status
    0; the positions it read equal the oracle's step of its own inputs bit for
    bit."""
    pfs, ora = load_package(), load_oracle()
    exe, dump = str(tmp_path / "host_stub"), str(tmp_path / "step.bin")
    libdir = os.path.dirname(pfs.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", "host_stub.c"),
                    "-L", libdir, "-lpfs", "-Wl,-rpath," + libdir, "-o", exe], check=True)
    p = subprocess.run([exe, dump], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.startswith("status 0: "), p.stdout
    raw = open(dump, "rb").read()
    n = int(np.frombuffer(raw[:4], np.uint32)[0])
    ps = ctypes.sizeof(pfs.Params)
    params = pfs.Params.from_buffer_copy(raw[4:4 + ps])
    body = np.frombuffer(raw[4 + ps:], np.float32).reshape(2, n, 4)
    pos_in, pos_out = body[0].copy(), body[1].copy()
    want, _, _, _ = ora.step(params, pos_in, np.zeros_like(pos_in), 1)
    assert np.array_equal(pos_out.view(np.uint32), want.view(np.uint32))
