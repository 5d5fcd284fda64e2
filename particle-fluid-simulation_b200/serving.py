"""Request loop of the serving form: continuous batching of scene requests
under a device-memory budget.

A request is one scene (parameters + initial particle state) and a number of
world steps.  The server keeps one Batch per precision (FP32 and FP16-cell),
each sized so that the batches together fit the budget
(``pfs_batch_bytes``).  Every tick it

  1. admits waiting requests of each precision in arrival order while the
     batch has room for their particles and one more scene (a request larger
     than a whole batch is rejected);
  2. launches one step of every non-empty batch, each on its own stream, and
     only then waits for them, so the batches' work overlaps on the device;
  3. retires the requests whose step count is reached: their state is read
     back (the result) and their scene removed, freeing room for the next
     admissions.

Scene state stays resident on the device between ticks.  Because a scene in a
batch steps exactly as it would alone (bit-identical; see pfs_batch_* in
include/pfs.h), a request's result does not depend on what else is resident.

With ``feed=True`` every step starts again from each request's input state
(the batch's feed mode): the device work per step stays that of the inputs
instead of following a rollout, which is how the benchmark measures the cost
of serving the request mix.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from . import PFS_FP16_CELL, PFS_FP32, Batch, Params


@dataclass
class ServeRequest:
    rid: int
    arrival_s: float
    steps: int
    precision: int
    make: Callable[[], "tuple"]          # -> (params, pos4, vel4), built at admission
    admitted_s: Optional[float] = None
    done_s: Optional[float] = None
    result: Optional[dict] = None
    n: int = 0
    meta: dict = field(default_factory=dict)


def capacity_for_budget(budget_bytes: int, max_scenes: int, precision: int,
                        limit: int = 1 << 24) -> int:
    """Largest particle capacity whose batch fits in budget_bytes (0 if none)."""
    lo, hi = 0, limit
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if Batch.bytes_for(mid, max_scenes, precision) <= budget_bytes:
            lo = mid
        else:
            hi = mid - 1
    return lo


class Server:
    def __init__(self, hbm_budget_bytes: int, max_scenes: int = 512, substeps: int = 3,
                 precisions=(PFS_FP32, PFS_FP16_CELL), feed: bool = False,
                 keep_results: bool = True, max_particles_per_batch: int = 1 << 24):
        self.feed = feed
        self.keep_results = keep_results
        self.budget = int(hbm_budget_bytes)
        share = self.budget // len(precisions)
        self.batches: Dict[int, Batch] = {}
        self.capacity: Dict[int, int] = {}
        for p in precisions:
            cap = min(capacity_for_budget(share, max_scenes, p), max_particles_per_batch)
            if cap <= 0:
                raise ValueError("budget too small for a batch")
            b = Batch(cap, max_scenes, precision=p, substeps=substeps)
            if feed:
                b.set_feed(True)
            self.batches[p] = b
            self.capacity[p] = cap
        self.max_scenes = max_scenes
        self.waiting: Dict[int, collections.deque] = {p: collections.deque() for p in precisions}
        self.active: Dict[int, Dict[int, tuple]] = {p: {} for p in precisions}  # sid -> (req, left)
        self.used: Dict[int, int] = {p: 0 for p in precisions}
        self.finished: List[ServeRequest] = []
        self.rejected: List[ServeRequest] = []
        self.tick_ms: List[float] = []
        self.particle_steps = 0

    def close(self) -> None:
        for b in self.batches.values():
            b.close()
        self.batches = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, req: ServeRequest) -> None:
        self.waiting[req.precision].append(req)

    def pending(self) -> int:
        return sum(len(q) for q in self.waiting.values()) + sum(len(a) for a in self.active.values())

    def _admit(self, now: float) -> None:
        for p, q in self.waiting.items():
            b = self.batches[p]
            while q:
                req = q[0]
                if "scene" not in req.meta:  # built once, kept while it waits
                    req.meta["scene"] = req.make()
                params, pos, vel = req.meta["scene"]
                n = pos.shape[0]
                if n > self.capacity[p]:
                    q.popleft()
                    del req.meta["scene"]
                    req.n = n
                    self.rejected.append(req)
                    continue
                if self.used[p] + n > self.capacity[p] or len(self.active[p]) >= self.max_scenes:
                    break
                q.popleft()
                del req.meta["scene"]
                sid = b.add(params, pos, vel)
                req.n = n
                req.admitted_s = now
                self.active[p][sid] = (req, req.steps)
                self.used[p] += n

    def tick(self, now: float) -> None:
        """Admit, step every resident scene once, retire finished requests."""
        t0 = time.perf_counter()
        self._admit(now)
        stepped = [p for p, a in self.active.items() if a]
        for p in stepped:
            self.batches[p].step(1)
        for p in stepped:
            self.batches[p].sync()
        done_t = now + (time.perf_counter() - t0)
        for p in stepped:
            b = self.batches[p]
            for sid in list(self.active[p]):
                req, left = self.active[p][sid]
                self.particle_steps += req.n
                left -= 1
                if left > 0:
                    self.active[p][sid] = (req, left)
                    continue
                if self.keep_results:
                    req.result = b.read(sid, density=True)
                b.remove(sid)
                del self.active[p][sid]
                self.used[p] -= req.n
                req.done_s = done_t
                self.finished.append(req)
        self.tick_ms.append((time.perf_counter() - t0) * 1e3)


def run(server: Server, requests: List[ServeRequest], wall_limit_s: float = 120.0,
        clock=time.perf_counter) -> dict:
    """Feed requests to the server at their arrival times (seconds from the
    start) and tick until all are served or wall_limit_s passes."""
    reqs = sorted(requests, key=lambda r: r.arrival_s)
    t_start = clock()
    k = 0
    while True:
        now = clock() - t_start
        while k < len(reqs) and reqs[k].arrival_s <= now:
            server.submit(reqs[k])
            k += 1
        if k == len(reqs) and server.pending() == 0:
            break
        if now > wall_limit_s:
            break
        if server.pending() == 0:
            time.sleep(max(0.0, min(0.01, reqs[k].arrival_s - now)))
            continue
        server.tick(now)
    elapsed = clock() - t_start
    # a request is one requested step batch (its scene's N steps): latency is
    # arrival to result, split into the wait for admission and the service
    # from admission to result
    lat = [r.done_s - r.arrival_s for r in server.finished]
    wait = [r.admitted_s - r.arrival_s for r in server.finished]
    service = [r.done_s - r.admitted_s for r in server.finished]
    per_step = [(r.done_s - r.admitted_s) / max(1, r.steps) for r in server.finished]
    pct = (lambda a, q: float(np.percentile(a, q)) if a else None)
    return {
        "requests": len(reqs),
        "arrived": k,
        "finished": len(server.finished),
        "unfinished": len(reqs) - len(server.finished) - len(server.rejected),
        "rejected_over_budget": len(server.rejected),
        "elapsed_s": elapsed,
        "particle_steps": server.particle_steps,
        "particle_steps_per_s": server.particle_steps / elapsed if elapsed > 0 else 0.0,
        "latency_p50_s": pct(lat, 50),
        "latency_p99_s": pct(lat, 99),
        "admission_wait_p50_s": pct(wait, 50),
        "admission_wait_p99_s": pct(wait, 99),
        "service_p50_s": pct(service, 50),
        "service_p99_s": pct(service, 99),
        "service_per_step_p50_ms": None if not per_step else 1e3 * pct(per_step, 50),
        "service_per_step_p99_ms": None if not per_step else 1e3 * pct(per_step, 99),
        "tick_p50_ms": pct(server.tick_ms, 50),
        "tick_p99_ms": pct(server.tick_ms, 99),
        "ticks": len(server.tick_ms),
    }


def requests_from_stream(specs) -> List[ServeRequest]:
    """ServeRequests from scenes.request_stream entries (scenes built lazily)."""
    out = []
    for s in specs:
        def make(s=s):
            sc = s.make_scene()
            return sc.params, sc.pos, sc.vel
        out.append(ServeRequest(s.rid, s.arrival_s, s.steps, s.precision, make))
    return out
