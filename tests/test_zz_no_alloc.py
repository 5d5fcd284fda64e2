"""pfs_sort_keys_static: the cell-key sort for hosts that cannot allocate.

Engines and renderers that own the whole device heap (every buffer comes from
their own pools) or run a frame loop with a fixed memory plan cannot let a
library call cudaMalloc: it may fail against their budget or stall the device
while it synchronises.  This entry point sorts with scratch that lives in the
library's static device memory instead.  Checked here, through the C ABI,
against the sort the world step itself runs (pfs_world_debug_substep's keys
and permutation): integers, so bit-exact, on two calls in a row of different
sizes (the second at the size limit), plus the size limit itself; full 32-bit
keys (four passes) and tiny inputs (one pass) against numpy's stable sort;
overlapping arrays refused; the device status of each call read back.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


def _world_sort(pfs, scene):
    with pfs.World(scene.params, scene.pos, scene.vel) as w:
        got = w.debug_substep()
    return got["keys_in"], got["keys"], got["perm"]


def test_static_sort_matches_world_sort(cuda_device):
    import torch

    pfs = load_package()
    from pfs_b200 import scenes

    fn = pfs.lib().pfs_sort_keys_static
    limit = 1 << 20  # PFS_STATIC_SORT_MAX_KEYS
    cases = [scenes.dam_break(n=16384, seed=0), scenes.slab_1m(n=limit, seed=1)]
    stream = torch.cuda.current_stream().cuda_stream
    for scene in cases:
        keys_in, want_keys, want_perm = _world_sort(pfs, scene)
        n = keys_in.size
        keys = torch.from_numpy(keys_in.view(np.int32).copy()).cuda()
        out_k = torch.full_like(keys, -1)
        out_p = torch.full_like(keys, -1)
        torch.cuda.synchronize()
        rc = fn(keys.data_ptr(), n, 0, out_k.data_ptr(), out_p.data_ptr(), stream)
        assert rc == pfs.PFS_OK, pfs.status_name(rc)
        assert pfs.lib().pfs_sort_static_status(stream) == pfs.PFS_OK
        torch.cuda.synchronize()
        got_k = out_k.cpu().numpy().view(np.uint32)
        got_p = out_p.cpu().numpy().view(np.uint32)
        assert np.array_equal(got_k, want_keys), f"n={n}: sorted keys differ"
        assert np.array_equal(got_p, want_perm), f"n={n}: permutation differs"


def test_static_sort_refuses_more_than_its_scratch(cuda_device):
    import torch

    pfs = load_package()
    fn = pfs.lib().pfs_sort_keys_static
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    too_many = (1 << 20) + 1
    rc = fn(buf.data_ptr(), too_many, 0, buf.data_ptr(), buf.data_ptr(), None)
    assert rc == pfs.PFS_ERANGE
    assert fn(buf.data_ptr(), 16, 33, buf.data_ptr(), buf.data_ptr(), None) == pfs.PFS_EINVAL


@pytest.mark.parametrize("n,key_bits", [(1, 32), (200, 0), (256, 8), (1000, 32), (1 << 20, 32),
                                        (777_777, 24)])
def test_static_sort_explicit_key_bits_vs_numpy(cuda_device, n, key_bits):
    """Random keys of key_bits bits (0: keys < n), sorted stably: the
    permutation is numpy's stable argsort, the keys are its sorted keys."""
    import torch

    pfs = load_package()
    fn = pfs.lib().pfs_sort_keys_static
    rng = np.random.default_rng(n + key_bits)
    hi = (1 << key_bits) if key_bits else n
    keys_np = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
    keys_np[: n // 3] = keys_np[n // 3: 2 * (n // 3)]  # plenty of ties
    keys = torch.from_numpy(keys_np.view(np.int32).copy()).cuda()
    out_k = torch.full_like(keys, -1)
    out_p = torch.full_like(keys, -1)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    assert fn(keys.data_ptr(), n, key_bits, out_k.data_ptr(), out_p.data_ptr(), stream) == pfs.PFS_OK
    assert pfs.lib().pfs_sort_static_status(stream) == pfs.PFS_OK
    want_p = np.argsort(keys_np, kind="stable").astype(np.uint32)
    assert np.array_equal(out_p.cpu().numpy().view(np.uint32), want_p)
    assert np.array_equal(out_k.cpu().numpy().view(np.uint32), keys_np[want_p])


def test_static_sort_refuses_overlapping_arrays(cuda_device):
    import torch

    pfs = load_package()
    fn = pfs.lib().pfs_sort_keys_static
    buf = torch.zeros(3 * 64, dtype=torch.int32, device="cuda")
    a, b, c = (buf.data_ptr() + 4 * 64 * i for i in range(3))
    assert fn(a, 64, 0, a, c, None) == pfs.PFS_EINVAL          # in place
    assert fn(a, 64, 0, b, a + 4 * 10, None) == pfs.PFS_EINVAL  # perm inside the keys
    assert fn(a, 64, 0, b, b + 4 * 32, None) == pfs.PFS_EINVAL  # outputs share memory
    assert fn(a, 64, 0, b, c, None) == pfs.PFS_OK
    torch.cuda.synchronize()
