"""pfs_sort_keys_static: the cell-key sort for hosts that cannot allocate.

Engines and renderers that own the whole device heap (every buffer comes from
their own pools) or run a frame loop with a fixed memory plan cannot let a
library call cudaMalloc: it may fail against their budget or stall the device
while it synchronises.  This entry point sorts with scratch that lives in the
library's static device memory instead.  Checked here, through the C ABI,
against the sort the world step itself runs (pfs_world_debug_substep's keys
and permutation): integers, so bit-exact, on two calls in a row of different
sizes (the second at the size limit), plus the size limit itself.

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
