"""Continuous-batching server of scene-simulation requests, over the C-ABI
server (``avbd_server_*`` in include/avbd.h).

A request is a staged scene (a ``Solver`` built through the reference API,
never stepped) plus a number of steps.  The server keeps every admitted
scene resident on the device inside one batch and advances all of them with
one persistent-kernel launch per tick.  Requests that arrive while others
run wait in arrival order and are admitted as soon as their scene fits in
the free pool space (HBM-budget admission); finished scenes are read back
and retired, and their space is reused by the next admissions.  A tick
returns while its step runs on the GPU; the next tick stages its newcomers
meanwhile.  Scene results do not depend on what else shares the batch.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from ._lib import AvbdServedRequest, AvbdServerStats, STATUS, check, default_params, load
from .solver import Solver

KEEP_RESULT = 1   # AVBD_SERVE_KEEP_RESULT
KEEP_FIRST = 2    # AVBD_SERVE_KEEP_FIRST


@dataclass
class Request:
    rid: int
    scene: Solver            # staged scene (released once submitted)
    steps: int
    arrival: float           # seconds since the server clock started
    admitted: float = -1.0
    finished: float = -1.0
    dynamic: int = 0         # dynamic bodies (body-iterations per step / iterations)
    status: str = ""
    result: tuple = field(default=None, repr=False)   # (pos, quat) after the last step
    sample: bool = False     # also keep the state after the request's first step (tolerance checks)
    first: tuple = field(default=None, repr=False)    # (pos, quat) after the first step, for samples
    sid: int = -1            # the server's request id


# Pool bytes per body of a typical scene (bodies, candidate pairs, contacts,
# incidence) used to turn an HBM budget into pool capacities.
BYTES_PER_BODY_BUDGET = 9000


class Server:
    def __init__(self, budget_bytes: int, max_scenes: int = 8192, iterations: int = 10, dt: float = 1.0 / 60.0,
                 launch: dict | None = None, keep_results: bool = True, device: int = 0):
        self._lib = load()
        self._p = default_params(num_iterations=int(iterations), step_value=float(dt))
        bodies = max(1024, int(budget_bytes // BYTES_PER_BODY_BUDGET))
        self.capacity_bodies = bodies
        h = C.c_void_p()
        check(self._lib.avbd_server_create(C.byref(self._p), int(device), bodies, int(max_scenes), C.byref(h)),
              "avbd_server_create")
        self._h = h
        if launch:
            from . import autotune
            autotune.apply(_BatchKnobs(self._lib, self._lib.avbd_server_batch(h)), launch)
        self.keep_results = keep_results
        self.iterations = iterations
        self.requests = {}        # server id -> Request
        self.done = []
        self.t0 = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.avbd_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clock(self) -> float:
        return time.perf_counter() - self.t0

    def start(self):
        self.t0 = time.perf_counter()

    def submit(self, req: Request):
        """Hands the request's staged scene to the server (the Solver may be dropped afterwards)."""
        req.dynamic = req.scene.num_dynamic
        flags = (KEEP_RESULT if (self.keep_results or req.sample) else 0) | (KEEP_FIRST if req.sample else 0)
        req.sid = check(self._lib.avbd_server_submit(self._h, req.scene.handle, int(req.steps), float(req.arrival),
                                                     flags), "avbd_server_submit")
        req.scene = None
        self.requests[req.sid] = req

    def _collect(self):
        out = AvbdServedRequest()
        while check(self._lib.avbd_server_poll(self._h, C.byref(out)), "avbd_server_poll") == 1:
            req = self.requests.pop(out.request)
            req.status = STATUS.get(out.status, str(out.status))
            req.admitted = out.admitted_s
            req.finished = out.finished_s
            n = out.bodies
            if self.keep_results or req.sample:
                pos, quat = np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32)
                fp = C.POINTER(C.c_float)
                if req.sample:
                    fpos, fquat = np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32)
                    check(self._lib.avbd_server_result(self._h, out.request, pos.ctypes.data_as(fp),
                                                       quat.ctypes.data_as(fp), fpos.ctypes.data_as(fp),
                                                       fquat.ctypes.data_as(fp)), "avbd_server_result")
                    req.first = (fpos, fquat)
                else:
                    check(self._lib.avbd_server_result(self._h, out.request, pos.ctypes.data_as(fp),
                                                       quat.ctypes.data_as(fp), None, None), "avbd_server_result")
                req.result = (pos, quat)
                self._lib.avbd_server_release(self._h, out.request)
            self.done.append(req)

    def tick(self) -> int:
        """Admits arrived requests, launches one step of every resident scene,
        retires the scenes the previous step finished. Returns the number of
        resident scenes the launched step advances."""
        n = check(self._lib.avbd_server_tick(self._h, self.clock()), "avbd_server_tick")
        self._collect()
        return n

    def drain(self):
        check(self._lib.avbd_server_drain(self._h, self.clock()), "avbd_server_drain")
        self._collect()

    def stats(self) -> dict:
        st = AvbdServerStats()
        check(self._lib.avbd_server_stats(self._h, C.byref(st)), "avbd_server_stats")
        return {k: int(getattr(st, k)) for k, _ in AvbdServerStats._fields_}

    @property
    def ticks(self) -> int:
        return self.stats()["ticks"]

    @property
    def body_iters(self) -> int:
        return self.stats()["body_iterations"]

    def run(self, until: float | None = None):
        """Ticks until every submitted request is done (or the clock passes `until`)."""
        while True:
            st = self.stats()
            if not (st["pending"] or st["active"]):
                break
            if until is not None and self.clock() > until:
                break
            if not st["active"] and st["pending"]:
                nxt = min(r.arrival for r in self.requests.values() if r.admitted < 0)
                wait = nxt - self.clock()
                if wait > 0:
                    time.sleep(min(wait, 0.01))
            self.tick()
        self.drain()

    @property
    def pending(self) -> int:
        return self.stats()["pending"]

    @property
    def active(self) -> int:
        return self.stats()["active"]

    def latency_stats(self, since: float = 0.0, until: float | None = None):
        lat = np.array([r.finished - r.arrival for r in self.done
                        if r.arrival >= since and (until is None or r.arrival < until)])
        if lat.size == 0:
            return {"completed": 0}
        return {"completed": int(lat.size), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean())}


class _BatchKnobs:
    """The launch setters of autotune.apply on the server's batch."""

    def __init__(self, lib, handle):
        self._lib, self._h = lib, handle

    def set_groups(self, rigid_group, fem_group):
        check(self._lib.avbd_batch_set_groups(self._h, int(rigid_group), int(fem_group)), "set_groups")

    def set_kernel(self, variant):
        check(self._lib.avbd_batch_set_kernel(self._h, int(variant)), "set_kernel")

    def set_launch(self, threads, ctas_per_sm):
        check(self._lib.avbd_batch_set_launch(self._h, int(threads), int(ctas_per_sm)), "set_launch")

    def set_team_work(self, units):
        check(self._lib.avbd_batch_set_team_work(self._h, int(units)), "set_team_work")

    def set_fem_team_work(self, units):
        check(self._lib.avbd_batch_set_fem_team_work(self._h, int(units)), "set_fem_team_work")

    def set_cluster(self, cluster_size, min_units):
        check(self._lib.avbd_batch_set_cluster(self._h, int(cluster_size), int(min_units)), "set_cluster")

    def set_queue_weight(self, body_weight):
        check(self._lib.avbd_batch_set_queue_weight(self._h, int(body_weight)), "set_queue_weight")

    def set_grid_broadphase(self, min_bodies):
        check(self._lib.avbd_batch_set_grid_broadphase(self._h, int(min_bodies)), "set_grid_broadphase")


def poisson_arrivals(rate: float, duration: float, seed: int = 0x5EED0005):
    """Arrival times of a Poisson process of `rate` requests/s over `duration` s."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        out.append(t)
