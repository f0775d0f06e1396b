"""Dynamic admission and the continuous-batching server.

Scenes join a running batch as pool space frees up and leave when done; a
scene's result is the same (bit for bit) whether it runs alone or shares the
batch with whatever else is resident, admitted before or after it.
"""
import numpy as np
import pytest

from skyephyx_b200 import scenes

pytestmark = pytest.mark.gpu


def staged(build):
    from skyephyx_b200 import Solver
    s = Solver()
    build(s)
    return s


def alone(build, steps):
    from skyephyx_b200 import Batch
    b = Batch()
    b.add_scene(staged(build))
    b.step(steps)
    return b.get_state(0)[:2]


BUILDS = [
    lambda s: scenes.pyramid_wall(s, rows=6),
    lambda s: scenes.fem_scene(s, 700, scenes.rng_for(4, 11)),
    lambda s: scenes.rigid_pile(s, 60, scenes.rng_for(4, 12), stack=False),
    scenes.level_joint_playground,
    lambda s: scenes.rigid_pile(s, 120, scenes.rng_for(4, 13), stack=True),
]


def same(a, b):
    return all(np.array_equal(x.view(np.uint32), y.view(np.uint32)) for x, y in zip(a, b))


def test_admit_after_start_and_reuse_slots():
    from skyephyx_b200 import Batch
    b = Batch()
    b.reserve(bodies=20000, forces=200, tets=20000, tris=0, scenes=8)
    ids = [b.add_scene(staged(f)) for f in BUILDS[:3]]
    b.step(4)
    b.remove_scene(ids[1])                      # retire the FEM scene mid-run
    late = b.add_scene(staged(BUILDS[3]))       # admitted into the freed space
    late2 = b.add_scene(staged(BUILDS[4]))
    b.step(6)
    assert same(b.get_state(ids[0])[:2], alone(BUILDS[0], 10))
    assert same(b.get_state(ids[2])[:2], alone(BUILDS[2], 10))
    assert same(b.get_state(late)[:2], alone(BUILDS[3], 6))
    assert same(b.get_state(late2)[:2], alone(BUILDS[4], 6))
    assert b.num_scenes == 4


def test_admission_waits_when_pools_are_full():
    from skyephyx_b200 import Batch
    b = Batch()
    b.reserve(bodies=300, forces=0, tets=0, tris=0, scenes=4)
    first = b.try_add_scene(staged(lambda s: scenes.rigid_pile(s, 200, scenes.rng_for(4, 1), stack=True)))
    assert first is not None
    assert b.try_add_scene(staged(lambda s: scenes.rigid_pile(s, 200, scenes.rng_for(4, 2), stack=True))) is None
    b.step(1)
    b.remove_scene(first)
    assert b.try_add_scene(staged(lambda s: scenes.rigid_pile(s, 200, scenes.rng_for(4, 2), stack=True))) is not None


def test_served_results_equal_alone():
    from skyephyx_b200.serve import Request, Server, poisson_arrivals
    arrivals = poisson_arrivals(rate=400.0, duration=0.06, seed=3)
    rng = np.random.default_rng(5)
    srv = Server(budget_bytes=2 << 30, max_scenes=64)
    builds = []
    for i, t in enumerate(arrivals):
        f = BUILDS[i % len(BUILDS)]
        steps = int(rng.integers(3, 12))
        builds.append((f, steps))
        srv.submit(Request(rid=i, scene=staged(f), steps=steps, arrival=t))
    srv.start()
    srv.run()
    assert len(srv.done) == len(arrivals) >= 10
    for req in srv.done:
        f, steps = builds[req.rid]
        assert req.status == "ok"
        assert same(req.result, alone(f, steps)), f"request {req.rid}"
    st = srv.latency_stats()
    assert st["completed"] == len(arrivals) and st["p99_s"] >= st["p50_s"] > 0


def test_server_admits_by_pool_space_and_keeps_samples():
    """A server whose pools hold two of three equal requests: the third waits
    for a retirement, every result equals the scene alone, and a sampled
    request's first-step poses equal one step alone."""
    from skyephyx_b200.serve import Request, Server
    build = lambda s: scenes.rigid_pile(s, 400, scenes.rng_for(4, 21), stack=False)
    srv = Server(budget_bytes=1000 * 9000, max_scenes=8)   # about 1,000 bodies of pool space
    steps = [4, 6, 5]
    for i, n in enumerate(steps):
        srv.submit(Request(rid=i, scene=staged(build), steps=n, arrival=0.0, sample=(i == 2)))
    srv.start()
    srv.run()
    done = {r.rid: r for r in srv.done}
    assert sorted(done) == [0, 1, 2]
    assert done[2].admitted >= min(done[0].finished, done[1].finished)
    for i, n in enumerate(steps):
        assert done[i].status == "ok"
        assert same(done[i].result, alone(build, n)), f"request {i}"
    assert same(done[2].first, alone(build, 1))
    st = srv.stats()
    assert st["completed"] == 3 and st["pending"] == 0 and st["active"] == 0
