"""Continuous-batching server of scene-simulation requests.

A request is a staged scene (a ``Solver`` built through the reference API,
never stepped) plus a number of steps.  The server keeps every admitted
scene resident on the device inside one ``Batch`` and advances all of them
with one persistent-kernel launch per tick.  Requests that arrive while
others run wait in a FIFO and are admitted as soon as their scene fits in
the free pool space (HBM-budget admission); finished scenes are read back
and retired, and their space is reused by the next admissions.  Scene
results do not depend on what else shares the batch.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from .solver import Batch, Solver


@dataclass
class Request:
    rid: int
    scene: Solver            # staged scene
    steps: int
    arrival: float           # seconds since the server clock started
    admitted: float = -1.0
    finished: float = -1.0
    slot: int = -1
    remaining: int = 0
    dynamic: int = 0         # dynamic bodies (body-iterations per step / iterations)
    status: str = ""
    result: tuple = field(default=None, repr=False)   # (pos, quat) after the last step
    sample: bool = False     # also keep the state after the request's first step (tolerance checks)
    first: tuple = field(default=None, repr=False)    # (pos, quat) after the first step, for samples


# Pool bytes per body of a typical scene (bodies, candidate pairs, contacts,
# incidence) used to turn an HBM budget into pool capacities.
BYTES_PER_BODY_BUDGET = 9000


class Server:
    def __init__(self, budget_bytes: int, max_scenes: int = 8192, iterations: int = 10, dt: float = 1.0 / 60.0,
                 launch: dict | None = None, keep_results: bool = True):
        self.batch = Batch(iterations=iterations, dt=dt)
        if launch:
            from . import autotune
            autotune.apply(self.batch, launch)
        bodies = max(1024, int(budget_bytes // BYTES_PER_BODY_BUDGET))
        self.capacity_bodies = bodies
        self.batch.reserve(bodies, bodies // 4, 2 * bodies, bodies // 4, max_scenes)
        self.pending = collections.deque()
        self.active = {}          # slot -> Request
        self.done = []
        self.keep_results = keep_results
        self.t0 = None
        self.ticks = 0
        self.body_iters = 0
        self.resident_dynamic = 0
        self.iterations = iterations

    def clock(self) -> float:
        return time.perf_counter() - self.t0

    def start(self):
        self.t0 = time.perf_counter()

    def submit(self, req: Request):
        req.dynamic = req.scene.num_dynamic
        self.pending.append(req)

    def _admit(self, now: float):
        while self.pending and self.pending[0].arrival <= now:
            req = self.pending[0]
            slot = self.batch.try_add_scene(req.scene)
            if slot is None:
                break             # no room: admit in arrival order once space frees up
            self.pending.popleft()
            req.slot = slot
            req.admitted = now
            req.remaining = req.steps
            self.active[slot] = req
            self.resident_dynamic += req.dynamic

    def tick(self) -> int:
        """Admits arrived requests, advances every resident scene one step,
        retires finished ones. Returns the number of resident scenes stepped."""
        self._admit(self.clock())
        if not self.active:
            return 0
        n = len(self.active)
        self.batch.step(1)
        self.ticks += 1
        self.body_iters += self.iterations * self.resident_dynamic
        finished = []
        for slot, req in self.active.items():
            req.remaining -= 1
            if req.sample and req.first is None:
                req.first = tuple(a.copy() for a in self.batch.get_state(slot)[:2])
            if req.remaining <= 0:
                finished.append(slot)
        for slot in finished:
            req = self.active.pop(slot)
            self.resident_dynamic -= req.dynamic
            req.status = self.batch.scene_status(slot)
            if self.keep_results or req.sample:
                pos, quat = self.batch.get_state(slot)[:2]
                req.result = (pos, quat)
            self.batch.remove_scene(slot)
            req.finished = self.clock()
            req.scene = None          # release the staged host copy
            self.done.append(req)
        return n

    def run(self, until: float | None = None):
        """Ticks until every submitted request is done (or the clock passes `until`)."""
        while self.pending or self.active:
            if until is not None and self.clock() > until:
                break
            if not self.active and self.pending:
                wait = self.pending[0].arrival - self.clock()
                if wait > 0:
                    time.sleep(min(wait, 0.01))
            self.tick()

    def latency_stats(self, since: float = 0.0):
        lat = np.array([r.finished - r.arrival for r in self.done if r.arrival >= since])
        if lat.size == 0:
            return {"completed": 0}
        return {"completed": int(lat.size), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean())}


def poisson_arrivals(rate: float, duration: float, seed: int = 0x5EED0005):
    """Arrival times of a Poisson process of `rate` requests/s over `duration` s."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        out.append(t)
