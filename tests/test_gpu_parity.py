"""GPU parity of the FP32 step against the oracle, through the C ABI.

Bar: bit-exact.  Keys, permutation and cell table are integer work; the FP32
form evaluates every float expression in the reference shaders' order with
one IEEE round-to-nearest operation each (no FMA contraction) and sums
neighbours in the reference's order, so densities, predicted state and
velocities match the oracle bit for bit as well (tolerance 0 ulp).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_oracle, load_package

pytestmark = pytest.mark.gpu

STAGES = ("keys_in", "keys", "perm", "start", "end", "xp", "vp", "density", "near_density",
          "vel_force")


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _assert_bits_equal(name, got, want):
    g, w = _bits(got), _bits(want)
    if not np.array_equal(g, w):
        bad = np.flatnonzero(g.ravel() != w.ravel())
        raise AssertionError(
            f"{name}: {bad.size} of {g.size} words differ; first at {bad[:5]}: "
            f"got {np.ascontiguousarray(got).ravel()[bad[:5]]} want {np.ascontiguousarray(want).ravel()[bad[:5]]}")


def _uniform_scene(pfs, n, seed, h=0.05, box=1.0):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0.0, box, (n, 3))
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0.0, 0.5, (n, 3))
    p = pfs.make_params(h, 1000.0, 250.0, 0.03, dt=1.0 / 240.0, box_max=(box, box, box))
    return p, pos, vel


def _set_shape_or_skip(pfs, w, shape, search):
    """Apply a kernel shape; the staged shape is refused (PFS_EINVAL) where
    its shared-memory stage cannot hold a block's neighbourhood (tables with
    few slots, dense scenes), which is then checked instead."""
    if shape == pfs.PFS_SHAPE_STAGED and w.staged_available() is False:
        with pytest.raises(pfs.PfsError) as ei:
            w.set_shape(shape, search)
        assert ei.value.status == pfs.PFS_EINVAL
        pytest.skip("staged shape unavailable for this scene (refused as documented)")
    w.set_shape(shape, search)


def _check_substep(pfs, ora, params, pos, vel, shape=None):
    with pfs.World(params, pos, vel) as w:
        if shape is not None:
            _set_shape_or_skip(pfs, w, shape, pfs.PFS_SEARCH_AUTO)
        got = w.debug_substep()
        state = w.read(pos=True, vel=True, density=True, keys=True, perm=True)
        assert w.device_error() == 0
    opos, ovel, odens, tr, _, _ = ora.substep(params, pos, vel, trace=True)
    for k in STAGES:
        _assert_bits_equal(k, got[k], tr[k])
    _assert_bits_equal("pos", state["pos"], opos)
    _assert_bits_equal("vel", state["vel"], ovel)
    _assert_bits_equal("density", state["density"], odens)
    _assert_bits_equal("read keys", state["keys"], tr["keys"])
    _assert_bits_equal("read perm", state["perm"], tr["perm"])


@pytest.mark.parametrize("n", [1, 2, 3, 64, 1000, 2048, 4097, 16384])
def test_substep_stages_uniform(cuda_device, n):
    pfs, ora = load_package(), load_oracle()
    p, pos, vel = _uniform_scene(pfs, n, seed=n)
    _check_substep(pfs, ora, p, pos, vel)


@pytest.mark.parametrize("n", [2048, 16384])
def test_substep_stages_dam_break(cuda_device, n):
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=n, seed=0)
    _check_substep(pfs, ora, sc.params, sc.pos, sc.vel)


@pytest.mark.parametrize("shape", ["SIMPLE", "SLAB", "LIST", "FLAT", "STAGED"])
@pytest.mark.parametrize("scene", ["uniform", "dam_break"])
def test_substep_every_shape_vs_oracle(cuda_device, shape, scene):
    """Each kernel shape of the neighbour passes against the oracle directly."""
    pfs, ora = load_package(), load_oracle()
    if scene == "uniform":
        p, pos, vel = _uniform_scene(pfs, 16384, seed=5)
    else:
        from pfs_b200 import scenes
        sc = scenes.dam_break(n=16384, seed=3)
        p, pos, vel = sc.params, sc.pos, sc.vel
    _check_substep(pfs, ora, p, pos, vel, shape=getattr(pfs, "PFS_SHAPE_" + shape))


@pytest.mark.parametrize("shape", ["SIMPLE", "SLAB", "LIST", "FLAT", "STAGED"])
@pytest.mark.parametrize("n", [4096, 4097, 12000])
def test_lattice_on_the_cut_radius(cuda_device, shape, n):
    """A lattice of spacing exactly h (a power of two) puts many pairs at
    d2 == h*h, on the cut itself, and particles on cell faces; n = 4097 and
    12000 give tables whose slots join several cells (hash collisions), so
    runs hold particles of distant cells."""
    pfs, ora = load_package(), load_oracle()
    h = 0.0625
    side = int(np.ceil(n ** (1.0 / 3.0)))
    ax = np.arange(side, dtype=np.float32) * np.float32(h) + np.float32(0.25)
    grid = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)[:n]
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = grid
    rng = np.random.default_rng(n)
    # a third of the particles jittered off the lattice, the rest exact
    jit = rng.random(n) < 1.0 / 3.0
    pos[jit, :3] += rng.uniform(-0.3 * h, 0.3 * h, (int(jit.sum()), 3)).astype(np.float32)
    vel = np.zeros((n, 4), np.float32)
    box = float(ax[-1]) + 0.5
    p = pfs.make_params(h, 1000.0, 250.0, 0.03, dt=1.0 / 240.0, box_max=(box, box, box))
    _check_substep(pfs, ora, p, pos, vel, shape=getattr(pfs, "PFS_SHAPE_" + shape))


@pytest.mark.parametrize("shape", ["LIST", "FLAT"])
def test_long_table_runs(cuda_device, shape):
    """Clumps of 2,500 and 300 particles inside single cells among a sparse
    uniform background: table runs far longer than one packed range word of
    the flat walk (127 candidates), particles whose ranges need more words
    than the walk stages (they walk the table from global memory), and lists
    past their rows (the force pass's scan queue)."""
    pfs, ora = load_package(), load_oracle()
    h = 0.05
    rng = np.random.default_rng(2500)
    n = 6000
    pos = np.zeros((n, 4), np.float32)
    pos[:2500, :3] = rng.uniform(0.505, 0.545, (2500, 3))
    pos[2500:2800, :3] = rng.uniform(0.555, 0.595, (300, 3))
    pos[2800:, :3] = rng.uniform(0.0, 1.0, (n - 2800, 3))
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0.0, 0.1, (n, 3))
    p = pfs.make_params(h, 1000.0, 250.0, 0.03, dt=1.0 / 240.0, box_max=(1.0, 1.0, 1.0))
    _check_substep(pfs, ora, p, pos, vel, shape=getattr(pfs, "PFS_SHAPE_" + shape))


def test_reference_default_params(cuda_device):
    """The reference's own parameter set (main.c:11-30), its box and wall
    margins, on a small slab with the reference's initial velocity."""
    pfs, ora = load_package(), load_oracle()
    p = pfs.reference_default()
    n = 8192
    rng = np.random.default_rng(7)
    pos = np.zeros((n, 4), np.float32)
    lo = np.array(p.box_min[:]) * 0.3
    hi = np.array(p.box_max[:]) * 0.3
    pos[:, :3] = rng.uniform(lo, hi, (n, 3))
    vel = np.zeros((n, 4), np.float32)
    vel[:, 2] = -100.0
    _check_substep(pfs, ora, p, pos, vel)


def test_slab_1m_substep(cuda_device):
    """Full 1,048,576-particle drop-in workload: one substep, every stage
    bit-exact (keys, permutation and table included)."""
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    sc = scenes.slab_1m()
    _check_substep(pfs, ora, sc.params, sc.pos, sc.vel)
    _check_substep(pfs, ora, sc.params, sc.pos, sc.vel, shape=pfs.PFS_SHAPE_FLAT)
    _check_substep(pfs, ora, sc.params, sc.pos, sc.vel, shape=pfs.PFS_SHAPE_STAGED)


def test_dam_break_rollout_bit_exact(cuda_device):
    """30 steps (90 substeps) of the 16,384-particle dam break through the
    graph-captured step: state identical to the oracle after every 10 steps."""
    pfs, ora = load_package(), load_oracle()
    from pfs_b200 import scenes
    sc = scenes.dam_break()
    opos, ovel = sc.pos, sc.vel
    with pfs.World(sc.params, sc.pos, sc.vel) as w:
        for _ in range(3):
            w.step(10)
            w.sync()
            st = w.read(pos=True, vel=True, density=True)
            opos, ovel, odens, _ = ora.step(sc.params, opos, ovel, 10)
            _assert_bits_equal("pos", st["pos"], opos)
            _assert_bits_equal("vel", st["vel"], ovel)
            _assert_bits_equal("density", st["density"], odens)


def test_ids_and_colors(cuda_device):
    pfs, ora = load_package(), load_oracle()
    p, pos, vel = _uniform_scene(pfs, 5000, seed=11)
    p.flags = pfs.PFS_FLAG_COLORS | pfs.PFS_FLAG_IDS
    ids0 = np.arange(5000, dtype=np.uint32)
    with pfs.World(p, pos, vel) as w:
        w.step(2)
        st = w.read(pos=True, vel=True)
        ids = w.read_ids()
        rgba = w.read_colors()
    q = p.copy()
    q.flags = 0
    opos, ovel, _, _, oids, _ = ora.substep(q, pos, vel, ids=ids0)
    opos, ovel, _, _, oids, orgba = ora.substep(q, opos, ovel, ids=oids, colors=True)
    _assert_bits_equal("pos", st["pos"], opos)
    _assert_bits_equal("ids", ids, oids)
    _assert_bits_equal("rgba", rgba, orgba)
    # ids are a permutation and pos[ids] follows the particles
    assert np.array_equal(np.sort(ids), ids0)


def test_step_equals_repeated_debug_substeps(cuda_device):
    """The graph-captured multi-substep step and the stage-by-stage path run
    the same kernels in the same order."""
    pfs = load_package()
    from pfs_b200 import scenes
    sc = scenes.dam_break(n=4096)
    with pfs.World(sc.params, sc.pos, sc.vel) as a, pfs.World(sc.params, sc.pos, sc.vel) as b:
        a.step(2)
        for _ in range(2 * sc.params.substeps):
            b.debug_substep()
        sa, sb = a.read(), b.read()
    _assert_bits_equal("pos", sa["pos"], sb["pos"])
    _assert_bits_equal("vel", sa["vel"], sb["vel"])


def test_write_resets_state(cuda_device):
    pfs = load_package()
    p, pos, vel = _uniform_scene(pfs, 3000, seed=5)
    with pfs.World(p, pos, vel) as w:
        w.step(3)
        first = w.read()
        w.write(pos, vel)
        w.step(3)
        second = w.read()
    _assert_bits_equal("pos", first["pos"], second["pos"])
    _assert_bits_equal("vel", first["vel"], second["vel"])


def test_sync_timeout_and_errors(cuda_device):
    pfs = load_package()
    p, pos, vel = _uniform_scene(pfs, 1000, seed=3)
    with pfs.World(p, pos, vel) as w:
        w.step(1)
        w.sync(timeout_ns=10_000_000_000)
        with pytest.raises(ValueError):
            w.write(pos[:10])
        with pytest.raises(pfs.PfsError) as ei:
            w.read_colors()  # colours were not requested at create
        assert ei.value.status == pfs.PFS_EINVAL


def test_run_pipelined_equals_write_step_read(cuda_device):
    """pfs_world_run_pipelined gives, input by input, the bits of the plain
    write / step / read sequence (pageable and pinned host buffers)."""
    import torch
    pfs = load_package()
    from pfs_b200 import scenes
    ins = []
    for seed in range(4):
        sc = scenes.dam_break(n=12289, seed=seed)
        ins.append((sc.pos, sc.vel if seed != 2 else None))
    p = scenes.dam_break(n=12289, seed=0).params
    with pfs.World(p, ins[0][0], ins[0][1]) as w:
        want = []
        for pos, vel in ins:
            w.write(pos, vel)
            w.step(2)
            st = w.read(pos=True, vel=True)
            want.append((st["pos"], st["vel"]))
        got = w.run_pipelined(ins, steps_each=2)
        for (gp, gv), (wp, wv) in zip(got, want):
            _assert_bits_equal("pos", gp, wp)
            _assert_bits_equal("vel", gv, wv)
        pin_in = [torch.from_numpy(np.ascontiguousarray(p_)).pin_memory() for p_, _ in ins]
        pin_out = [torch.empty((12289, 4), dtype=torch.float32).pin_memory() for _ in ins]
        w.run_pipelined_ptrs([t.data_ptr() for t in pin_in], None, [t.data_ptr() for t in pin_out], None, 2)
        w.write(ins[3][0], None)
        w.step(2)
        last = w.read(pos=True)["pos"]
        _assert_bits_equal("pinned, zero velocities", pin_out[3].numpy(), last)
        assert w.device_error() == 0


def _assert_equal_nan_aware(name, got, want):
    """Bit-equal where finite; NaN exactly where the oracle has NaN (a NaN's
    payload is the hardware's own: the GPU and the host CPU write different
    ones)."""
    g, w = np.ascontiguousarray(got), np.ascontiguousarray(want)
    gn, wn = np.isnan(g), np.isnan(w)
    assert np.array_equal(gn, wn), f"{name}: NaN in {int(gn.sum())} entries, oracle {int(wn.sum())}"
    z = np.float32(0)
    _assert_bits_equal(name, np.where(gn, z, g).astype(g.dtype), np.where(wn, z, w).astype(w.dtype))


@pytest.mark.parametrize("shape", ["SIMPLE", "SLAB", "LIST", "FLAT", "STAGED"])
def test_nan_neighbours_like_the_reference(cuda_device, shape):
    """Three particles with NaN velocities in a dense cluster (the golden case
    the reference's own shaders produced, tests/golden/glsl_nan_neighbours):
    their neighbours meet NaN distances, which the shaders do not skip, so
    the NaN reaches the same densities and velocities as in the oracle (the
    oracle matches the shaders' fixture bit for bit)."""
    pfs, ora = load_package(), load_oracle()
    from test_oracle_golden import _cases, _inputs, _params_for
    case = next(c for c in _cases() if c["name"] == "nan_neighbours")
    p = _params_for(pfs, case)
    pos, vel = _inputs(case)
    with pfs.World(p, pos, vel) as w:
        _set_shape_or_skip(pfs, w, getattr(pfs, "PFS_SHAPE_" + shape), pfs.PFS_SEARCH_TABLE)
        got = w.debug_substep()
        state = w.read(pos=True, vel=True)
    opos, ovel, _, tr, _, _ = ora.substep(p, pos, vel, trace=True)
    assert np.isnan(tr["vel_force"]).any()
    for k in STAGES:
        _assert_equal_nan_aware(k, got[k], tr[k])
    _assert_equal_nan_aware("pos", state["pos"], opos)
    _assert_equal_nan_aware("vel", state["vel"], ovel)
