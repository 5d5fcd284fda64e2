"""Host logic of the serving loop (particle-fluid-simulation_b200/serving.py)
on the CPU, with the device batch replaced by a recording fake: admission
by capacity and scene slots in arrival order, rejection of requests larger
than a batch, retirement after the requested steps, continuous admission as
room frees up, and the latency bookkeeping of run()."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package


class FakeBatch:
    """Stands in for pfs_b200.Batch: records the calls, steps nothing."""
    instances = []
    bytes_per_particle = 100
    bytes_per_scene = 1000

    def __init__(self, max_particles, max_scenes, precision=0, substeps=3):
        self.max_particles, self.max_scenes, self.precision = max_particles, max_scenes, precision
        self.scenes = {}
        self.next_id = 0
        self.steps = 0
        self.feed = False
        self.log = []
        FakeBatch.instances.append(self)

    @staticmethod
    def bytes_for(max_particles, max_scenes, precision=0):
        return FakeBatch.bytes_per_particle * max_particles + FakeBatch.bytes_per_scene * max_scenes

    def set_feed(self, on):
        self.feed = bool(on)

    def add(self, params, pos, vel):
        assert sum(p.shape[0] for p in self.scenes.values()) + pos.shape[0] <= self.max_particles
        assert len(self.scenes) < self.max_scenes
        sid = self.next_id
        self.next_id += 1
        self.scenes[sid] = pos.copy()
        self.log.append(("add", sid, pos.shape[0]))
        return sid

    def remove(self, sid):
        del self.scenes[sid]
        self.log.append(("remove", sid))

    def step(self, n):
        self.steps += n
        self.log.append(("step", len(self.scenes)))

    def sync(self):
        pass

    def read(self, sid, density=False):
        return {"pos": self.scenes[sid]}

    def close(self):
        pass


@pytest.fixture()
def serving(monkeypatch):
    load_package()
    from pfs_b200 import serving as srv
    FakeBatch.instances = []
    monkeypatch.setattr(srv, "Batch", FakeBatch)
    return srv


def _req(srv, rid, n, steps, precision, arrival=0.0):
    def make(n=n, rid=rid):
        pos = np.full((n, 4), float(rid), np.float32)
        return None, pos, np.zeros_like(pos)
    return srv.ServeRequest(rid, arrival, steps, precision, make)


def test_capacity_for_budget_is_the_largest_fitting(serving):
    budget = 100 * 5000 + 1000 * 8 + 99
    cap = serving.capacity_for_budget(budget, 8, serving.PFS_FP32)
    assert cap == 5000
    assert FakeBatch.bytes_for(cap, 8) <= budget < FakeBatch.bytes_for(cap + 1, 8)
    assert serving.capacity_for_budget(100, 8, serving.PFS_FP32) == 0


def test_admission_order_capacity_and_slots(serving):
    # one FP32 batch of 1000 particles, at most 3 scenes
    budget = FakeBatch.bytes_for(1000, 3)
    with serving.Server(budget, max_scenes=3, precisions=(serving.PFS_FP32,)) as s:
        assert s.capacity[serving.PFS_FP32] == 1000
        p = serving.PFS_FP32
        for rid, n in enumerate([400, 500, 200, 50, 50]):
            s.submit(_req(serving, rid, n, steps=2, precision=p))
        s.tick(0.0)
        b = FakeBatch.instances[0]
        # 400 + 500 fit, 200 would exceed 1000: admission stops in arrival order
        assert [e[2] for e in b.log if e[0] == "add"] == [400, 500]
        assert s.used[p] == 900 and len(s.waiting[p]) == 3
        s.tick(0.1)  # both finish their 2 steps here
        assert sorted(r.rid for r in s.finished) == [0, 1]
        assert s.used[p] == 0
        s.tick(0.2)  # the three waiting ones fit now, but only 3 slots
        assert [e[2] for e in b.log if e[0] == "add"][2:] == [200, 50, 50]
        s.tick(0.3)
        assert sorted(r.rid for r in s.finished) == [0, 1, 2, 3, 4]
        assert s.pending() == 0
        # every finished request stepped exactly its step count, and its
        # result is its own scene's state
        for r in s.finished:
            assert r.n == [400, 500, 200, 50, 50][r.rid]
            assert np.all(r.result["pos"] == float(r.rid))


def test_oversize_request_is_rejected_not_blocking(serving):
    budget = FakeBatch.bytes_for(100, 4)
    with serving.Server(budget, max_scenes=4, precisions=(serving.PFS_FP32,)) as s:
        p = serving.PFS_FP32
        s.submit(_req(serving, 0, 500, steps=1, precision=p))
        s.submit(_req(serving, 1, 60, steps=1, precision=p))
        s.tick(0.0)
        assert [r.rid for r in s.rejected] == [0]
        assert [r.rid for r in s.finished] == [1]


def test_precisions_have_separate_batches(serving):
    budget = 2 * FakeBatch.bytes_for(300, 2)
    with serving.Server(budget, max_scenes=2) as s:
        assert set(s.batches) == {serving.PFS_FP32, serving.PFS_FP16_CELL}
        s.submit(_req(serving, 0, 200, steps=3, precision=serving.PFS_FP32))
        s.submit(_req(serving, 1, 250, steps=1, precision=serving.PFS_FP16_CELL))
        s.tick(0.0)
        by_prec = {b.precision: b for b in FakeBatch.instances}
        assert by_prec[serving.PFS_FP32].steps == 1 and by_prec[serving.PFS_FP16_CELL].steps == 1
        assert [r.rid for r in s.finished] == [1]
        s.tick(0.1)
        s.tick(0.2)
        # the FP16 batch is empty after its request retired: it is not stepped
        assert by_prec[serving.PFS_FP16_CELL].steps == 1
        assert by_prec[serving.PFS_FP32].steps == 3
        assert [r.rid for r in s.finished] == [1, 0]


def test_run_admits_arrivals_while_others_run(serving):
    """A request that arrives while another is resident joins the running
    batch at the next tick (continuous batching), and latencies are measured
    from arrival."""
    budget = FakeBatch.bytes_for(1000, 4)
    t = [0.0]

    def clock():
        t[0] += 0.01  # every clock read advances 10 ms
        return t[0]

    with serving.Server(budget, max_scenes=4, precisions=(serving.PFS_FP32,)) as s:
        p = serving.PFS_FP32
        reqs = [_req(serving, 0, 100, steps=20, precision=p, arrival=0.0),
                _req(serving, 1, 100, steps=5, precision=p, arrival=0.05)]
        stats = serving.run(s, reqs, wall_limit_s=10.0, clock=clock)
        b = FakeBatch.instances[0]
        assert stats["finished"] == 2 and stats["unfinished"] == 0
        # some step ran with both scenes resident
        assert ("step", 2) in b.log
        r1 = next(r for r in s.finished if r.rid == 1)
        r0 = next(r for r in s.finished if r.rid == 0)
        assert r1.done_s < r0.done_s  # the short late request left first
        assert r1.admitted_s >= r1.arrival_s
        assert stats["latency_p50_s"] > 0 and stats["latency_p99_s"] >= stats["latency_p50_s"]
        assert stats["particle_steps"] == 100 * 20 + 100 * 5
