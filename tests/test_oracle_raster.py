"""Oracle point-splat rasteriser (shader.vert / shader.frag restated) and FXAA
(raymarchShader.frag): known answers on the CPU."""
from __future__ import annotations

import numpy as np

from conftest import load_oracle, load_package

f32 = np.float32


def _cam(pfs, W=64, H=48, radius=0.5):
    # camera on -y looking along +y at the origin, z up (the reference's
    # initializeCamera orientation, main.c:237-243)
    return pfs.splat_view((0.0, -20.0, 0.0), (0.0, 1.0, 0.0), W, H, radius)


def _mats(v):
    return (np.array(v.model[:], f32), np.array(v.view[:], f32), np.array(v.proj[:], f32))


def test_single_splat_is_a_centred_shaded_disc():
    pfs, ora = load_package(), load_oracle()
    W, H = 64, 48
    v = _cam(pfs, W, H, radius=2.0)
    pos = np.array([[0.0, 0.0, 0.0, 0.0]], f32)
    col = np.array([[0.2, 0.4, 0.8, 1.0]], f32)
    rgba, depth = ora.splats(pos, col, *_mats(v), v.particle_radius, W, H)
    lit = rgba[..., 3] > 0
    ys, xs = np.nonzero(lit)
    assert lit.sum() > 20
    # centred on the screen, symmetric, round
    assert abs(xs.mean() + 0.5 - W / 2) < 0.6 and abs(ys.mean() + 0.5 - H / 2) < 0.6
    assert abs((xs.max() - xs.min()) - (ys.max() - ys.min())) <= 1
    # untouched pixels keep the clear values
    assert np.all(rgba[~lit] == 0) and np.all(depth[~lit] == 1.0)
    assert np.all((depth[lit] > 0) & (depth[lit] < 1))
    # colour = ramp colour x (0.7 + 0.3 * lighting) <= ramp colour; brighter
    # toward the light (-x, +z in view: up-left on screen... lightDir -0.5,-0.5,1)
    assert np.all(rgba[lit][:, :3] <= col[0, :3] + 1e-7)
    assert np.all(rgba[lit][:, :3] >= 0.7 * col[0, :3] - 1e-7)


def test_nearer_splat_wins_and_ties_keep_the_first():
    pfs, ora = load_package(), load_oracle()
    W, H = 64, 48
    v = _cam(pfs, W, H, radius=2.0)
    col = np.array([[1, 0, 0, 1], [0, 1, 0, 1], [0, 0, 1, 1]], f32)
    # particle 1 nearer the camera (smaller y) than 0; particle 2 at 0's place
    pos = np.array([[0, 0, 0, 0], [0, -5, 0, 0], [0, 0, 0, 0]], f32)
    rgba, depth = ora.splats(pos, col, *_mats(v), v.particle_radius, W, H)
    c = rgba[H // 2, W // 2]
    assert c[1] > 0 and c[0] == 0 and c[2] == 0       # the nearer (green) one
    rgba2, _ = ora.splats(pos[[0, 2]], col[[0, 2]], *_mats(v), v.particle_radius, W, H)
    c2 = rgba2[H // 2, W // 2]
    assert c2[0] > 0 and c2[2] == 0                  # equal depth: the first drawn


def test_fxaa_keeps_flat_images_and_softens_edges():
    ora = load_oracle()
    flat = np.full((24, 32, 4), 0.25, f32)
    out = ora.fxaa(flat)
    assert np.allclose(out[..., :3], 0.25, atol=1e-6) and np.all(out[..., 3] == 1)
    # a vertical edge: FXAA samples along it (dir is vertical), nothing blurs
    step = np.zeros((24, 32, 4), f32)
    step[:, 16:, :3] = 1.0
    assert np.array_equal(ora.fxaa(step)[..., :3], step[..., :3])
    # a diagonal edge is softened on the edge, kept away from it
    yy, xx = np.mgrid[0:24, 0:32]
    diag = np.zeros((24, 32, 4), f32)
    diag[..., :3] = (2 * xx > 3 * yy)[..., None]
    out = ora.fxaa(diag)
    far = np.abs(2 * xx - 3 * yy) > 8
    assert np.array_equal(out[far][:, :3], diag[far][:, :3])
    mid = (out[..., 0] > 0) & (out[..., 0] < 1)
    assert mid.sum() > 10


def test_stages_match_reference_shaders():
    """The oracle's vertex arithmetic (pfso_splat_clip with pfso_splat_camera's
    mvp) and fragment arithmetic (discard rule, pfso_splat_shade) against
    shader.vert / shader.frag run through the CPU harness
    (tests/golden/glsl_raster.npz, written by oracle/glsl_ref.py
    golden_raster): bit for bit."""
    import ctypes
    from conftest import GOLDEN
    ora = load_oracle()
    g = np.load(f"{GOLDEN}/glsl_raster.npz")
    mvp, right, up = ora.splat_camera(g["model"], g["view"], g["proj"])
    L = ora.lib()
    r = float(g["radius"])
    for i in range(g["pos"].shape[0]):
        p3 = np.ascontiguousarray(g["pos"][i, :3])
        for c, (qx, qy) in enumerate(g["corners"]):
            out = np.zeros(4, f32)
            L.pfso_splat_clip(mvp.ctypes.data, p3.ctypes.data, right.ctypes.data, up.ctypes.data,
                              ctypes.c_float(r), ctypes.c_float(qx), ctypes.c_float(qy), out.ctypes.data)
            assert np.array_equal(out.view(np.uint32), g["clip"][i, c].view(np.uint32)), (i, c)
    col = g["col"]
    for i in range(g["frag"].shape[0]):
        for k, (qx, qy) in enumerate(g["qs"]):
            discarded = f32(qx) * f32(qx) + f32(qy) * f32(qy) > f32(1.0)
            assert bool(g["discarded"][i, k]) == discarded, (i, qx, qy)
            if discarded:
                continue
            out = np.zeros(4, f32)
            L.pfso_splat_shade(np.ascontiguousarray(col[i]).ctypes.data, ctypes.c_float(qx),
                               ctypes.c_float(qy), out.ctypes.data)
            assert np.array_equal(out.view(np.uint32), g["frag"][i, k].view(np.uint32)), (i, qx, qy)
    assert g["discarded"].sum() > 0 and (g["discarded"] == 0).sum() > 100
