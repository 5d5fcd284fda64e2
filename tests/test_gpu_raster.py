"""Point-splat rasteriser and FXAA on the GPU through the C ABI against the
oracle.  Only +, -, *, / and sqrt are involved, each one IEEE operation in
the oracle's order, and the depth test keeps the first particle of the
smallest depth exactly as sequential drawing does: images and depth buffers
must match bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_oracle, load_package

pytestmark = pytest.mark.gpu
f32 = np.float32


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _mats(v):
    return (np.array(v.model[:], f32), np.array(v.view[:], f32), np.array(v.proj[:], f32))


@pytest.mark.parametrize("n,W,H,radius", [(1, 64, 48, 0.2), (4096, 160, 120, 0.05), (20000, 320, 200, 0.02)])
def test_splats_match_oracle(cuda_device, n, W, H, radius):
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=n, seed=5)
    p = sc.params
    p.flags |= pfs.PFS_FLAG_COLORS
    lo, hi = np.array(p.box_min[:3]), np.array(p.box_max[:3])
    c = (lo + hi) / 2
    v = pfs.splat_view((c[0] + 0.3 * (hi[0] - lo[0]), lo[1] - 1.5 * (hi[1] - lo[1]), c[2] + 0.4),
                       (-0.25, 1.0, -0.2), W, H, radius)
    with pfs.World(p, sc.pos, sc.vel) as w:
        w.step(2)
        st = w.read(pos=True)
        col = w.read_colors()
        rgba, depth = w.render_splats(v, W, H, with_depth=True)
        assert w.device_error() == 0
    want, want_d = ora.splats(st["pos"], col, *_mats(v), radius, W, H)
    assert np.array_equal(_bits(depth), _bits(want_d))
    assert np.array_equal(_bits(rgba), _bits(want))
    assert (want[..., 3] > 0).sum() > (10 if n == 1 else 200)


def test_splats_device_buffers_and_errors(cuda_device):
    import torch
    pfs = load_package()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=2048, seed=2)
    v = pfs.splat_view((0.5, -2.0, 0.5), (0, 1, 0), 64, 48, 0.05)
    with pfs.World(sc.params, sc.pos, sc.vel) as w:          # no colour ramp
        with pytest.raises(pfs.PfsError):
            w.render_splats(v, 64, 48)
    p = sc.params
    p.flags |= pfs.PFS_FLAG_COLORS
    with pfs.World(p, sc.pos, sc.vel) as w:
        w.step(1)
        host, hd = w.render_splats(v, 64, 48, with_depth=True)
        dev = torch.empty((48, 64, 4), dtype=torch.float32, device="cuda")
        dd = torch.empty((48, 64), dtype=torch.float32, device="cuda")
        w.render_splats_ptr(v, 64, 48, dev.data_ptr(), dd.data_ptr())
        assert np.array_equal(dev.cpu().numpy(), host) and np.array_equal(dd.cpu().numpy(), hd)
        assert w.device_error() == 0


def test_fxaa_matches_oracle(cuda_device):
    import torch
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=1024, seed=1)
    rng = np.random.default_rng(4)
    img = rng.random((90, 160, 4)).astype(f32)
    yy, xx = np.mgrid[0:90, 0:160]
    img[..., :3] *= (2 * xx > 3 * yy)[..., None]
    with pfs.World(sc.params, sc.pos, sc.vel) as w:
        got = w.fxaa(img)
        src = torch.from_numpy(img).cuda()
        dst = torch.empty_like(src)
        w.fxaa_ptr(src.data_ptr(), 160, 90, dst.data_ptr())
        assert np.array_equal(dst.cpu().numpy(), got)
    assert np.array_equal(_bits(got), _bits(ora.fxaa(img)))
