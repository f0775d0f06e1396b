"""Batched path: one persistent kernel per step over many scenes.

* a scene's result is bitwise the same alone and inside a mixed batch
  (one CTA runs a whole scene in a fixed per-body order);
* batched results match the oracle like the single-scene path does.
"""
import numpy as np
import pytest

from skyephyx_b200 import scenes

pytestmark = pytest.mark.gpu


def mix_builders():
    rng = scenes.rng_for
    return [
        lambda s: scenes.pyramid_wall(s, rows=8),
        lambda s: scenes.fem_scene(s, 700, rng(4, 1)),
        lambda s: scenes.rigid_pile(s, 40, rng(4, 2), stack=False),
        lambda s: scenes.rigid_pile(s, 100, rng(4, 3), stack=True),
        scenes.level_joint_playground,
        scenes.level_cloth,
        lambda s: scenes.fem_scene(s, 1500, rng(4, 4)),
        scenes.level_mass_springs,
    ]


def staged(build):
    from skyephyx_b200 import Solver
    s = Solver()
    build(s)
    return s


def test_alone_equals_in_mix():
    from skyephyx_b200 import Batch
    builders = mix_builders()
    mix = Batch()
    keep = []
    for b in builders:
        w = staged(b)
        keep.append(w)
        mix.add_scene(w)
    assert mix.step(3) == "ok"
    for i, b in enumerate(builders):
        alone = Batch()
        w = staged(b)
        alone.add_scene(w)
        assert alone.step(3) == "ok"
        pa, qa = alone.get_state(0)[:2]
        pm, qm = mix.get_state(i)[:2]
        assert np.array_equal(pa.view(np.uint32), pm.view(np.uint32)), f"scene {i} positions differ"
        assert np.array_equal(qa.view(np.uint32), qm.view(np.uint32)), f"scene {i} rotations differ"
        assert mix.scene_status(i) == "ok"


def test_batch_matches_oracle(oracle_mod):
    from skyephyx_b200 import Batch
    builders = mix_builders()
    batch = Batch()
    keep = []
    for b in builders:
        w = staged(b)
        keep.append(w)
        batch.add_scene(w)
    assert batch.step(1) == "ok"
    for i, b in enumerate(builders):
        o = oracle_mod.OracleSolver()
        b(o)
        assert o.step_coloured() == 0
        po = o.get_state()[0]
        pb = batch.get_state(i)[0]
        assert np.abs(po - pb).max(initial=0.0) <= 1e-4, f"scene {i}"


def fem_on_ground(s):
    """A free tet block whose bottom particles touch a static ground box
    (particle-box manifolds beside the tet terms)."""
    s.add_body(scenes.CUBE, 1.0, 0.5, scenes.v3(0, -0.5, 0), scenes.v3(10, 1, 10), is_static=True)
    s.make_tet_volume(-0.9, 0.04, -0.45, 7, 3, 4, 0.3, 2e4, 0.3, 1.0, 0.5, False)


FEM_BUILDERS = [
    lambda s: scenes.fem_scene(s, 700, scenes.rng_for(4, 1)),
    lambda s: scenes.fem_scene(s, 1500, scenes.rng_for(4, 4)),
    fem_on_ground,
    scenes.level_soft_beam,
    lambda s: scenes.stvk_block(s),
]


def run_groups(builders, fem_group, steps):
    from skyephyx_b200 import Batch
    b = Batch()
    b.set_groups(1, fem_group)
    keep = [staged(f) for f in builders]
    for w in keep:
        b.add_scene(w)
    assert b.step(steps) == "ok"
    for i in range(len(builders)):
        assert b.scene_status(i) == "ok", f"scene {i}"
    return [b.get_state(i)[:2] for i in range(len(builders))]


def test_flat_sweep_matches_one_lane_per_particle():
    """The term-per-lane sweep sums each particle's terms in incidence order,
    like one lane per particle; the two differ only where the compiler fuses a
    term's last multiply into the sum differently (a few ulp per step)."""
    from skyephyx_b200 import GROUP_FLAT
    one = run_groups(FEM_BUILDERS, 1, 4)
    flat = run_groups(FEM_BUILDERS, GROUP_FLAT, 4)
    for i, ((p1, q1), (pf, qf)) in enumerate(zip(one, flat)):
        assert np.abs(p1 - pf).max(initial=0.0) <= 1e-5, f"scene {i}"
        assert np.abs(q1 - qf).max(initial=0.0) <= 1e-5, f"scene {i}"


def test_flat_sweep_matches_oracle(oracle_mod):
    from skyephyx_b200 import GROUP_FLAT
    flat = run_groups(FEM_BUILDERS, GROUP_FLAT, 1)
    for i, f in enumerate(FEM_BUILDERS):
        o = oracle_mod.OracleSolver()
        f(o)
        assert o.step_coloured() == 0
        assert np.abs(o.get_state()[0] - flat[i][0]).max(initial=0.0) <= 1e-4, f"scene {i}"


def test_team_split_changes_nothing():
    """Small scenes run by half- or quarter-CTA teams give bitwise the results
    of one scene per CTA (no per-body arithmetic depends on the team size)."""
    from skyephyx_b200 import Batch
    builders = mix_builders()
    results = []
    for team_work in (0, 64):
        b = Batch()
        b.set_team_work(team_work)
        keep = [staged(f) for f in builders]
        for w in keep:
            b.add_scene(w)
        assert b.step(3) == "ok"
        results.append([b.get_state(i)[:2] for i in range(len(builders))])
    for i, ((p0, q0), (p1, q1)) in enumerate(zip(*results)):
        assert np.array_equal(p0.view(np.uint32), p1.view(np.uint32)), f"scene {i}"
        assert np.array_equal(q0.view(np.uint32), q1.view(np.uint32)), f"scene {i}"


GRID_BUILDERS = [
    scenes.pyramid_wall,
    lambda s: scenes.rigid_pile(s, 300, scenes.rng_for(4, 21), stack=True),
    lambda s: scenes.rigid_pile(s, 400, scenes.rng_for(4, 22), stack=False),
    lambda s: scenes.fem_scene(s, 700, scenes.rng_for(4, 23)),
]


def test_grid_broadphase_matches_oracle(oracle_mod):
    """Scenes of 128+ bodies take the uniform-grid broadphase in the batch:
    after the first step their contact points and colours equal the oracle's
    (whose broadphase is the reference's all-pairs loop) and poses agree."""
    from skyephyx_b200 import Batch
    b = Batch()
    keep = [staged(f) for f in GRID_BUILDERS]
    for w in keep:
        b.add_scene(w)
    assert b.step(1) == "ok"
    for i, f in enumerate(GRID_BUILDERS):
        o = oracle_mod.OracleSolver()
        f(o)
        assert o.step_coloured() == 0
        info = b.scene_info(i)
        points = sum(len(v[0]) for v in o.contacts().values())
        assert info["status"] == 0 and info["contacts"] == points, f"scene {i}: {info} vs {points}"
        assert info["colours"] == o.colours()[1], f"scene {i}"
        assert np.abs(o.get_state()[0] - b.get_state(i)[0]).max(initial=0.0) <= 1e-4, f"scene {i}"


def test_grid_broadphase_equals_all_pairs_over_time():
    """A collapsing pile and a settling stack, 30 steps: the batch (grid
    broadphase) and the single-scene path (all-pairs broadphase kernels), both
    with one lane per body, agree bit for bit."""
    from skyephyx_b200 import Batch, Solver
    for build in GRID_BUILDERS[1:3]:
        w = Solver()
        w.set_group(1)
        build(w)
        b = Batch()
        b.set_groups(1, 4)
        b.add_scene(staged(build))
        for _ in range(30):
            assert w.step() == "ok"
        assert b.step(30) == "ok" and b.scene_status(0) == "ok"
        pw, qw = w.get_state()[:2]
        pb, qb = b.get_state(0)[:2]
        assert np.array_equal(pw.view(np.uint32), pb.view(np.uint32))
        assert np.array_equal(qw.view(np.uint32), qb.view(np.uint32))


def test_batch_grows_full_tables():
    """A scene whose contacts outgrow its tables (a self-colliding block of
    0.05 m particles) gets larger tables and takes the steps it missed: it
    ends on the same step count, and bitwise on the same poses, as the
    single-scene path, which grows its tables in place.  Its batch neighbour
    is unaffected."""
    from skyephyx_b200 import Batch, Solver
    block = lambda s: scenes.fem_block(s, nx=9, ny=4, nz=4)
    small = lambda s: scenes.pyramid_wall(s, rows=5)
    w = Solver()
    w.set_group(1)
    block(w)
    for _ in range(5):
        assert w.step() == "ok"
    b = Batch()
    b.set_groups(1, 1)
    b.add_scene(staged(block))
    b.add_scene(staged(small))
    assert b.step(1) == "ok"
    nbody = b.get_state(0)[0].shape[0]
    first = b.scene_info(0)
    # more candidates than the scene's first table holds: it did grow
    assert first["steps"] == 1 and first["candidates"] > 16 * nbody + 64, first
    assert b.step(1) == "ok"
    assert b.step(3) == "ok"
    for i in (0, 1):
        info = b.scene_info(i)
        assert info["status"] == 0 and info["steps"] == 5, f"scene {i}: {info}"
    pw, qw = w.get_state()[:2]
    pb, qb = b.get_state(0)[:2]
    assert np.array_equal(pw.view(np.uint32), pb.view(np.uint32))
    assert np.array_equal(qw.view(np.uint32), qb.view(np.uint32))
    assert same(b.get_state(1)[:2], alone_steps(small, 5))


def same(a, b):
    return all(np.array_equal(x.view(np.uint32), y.view(np.uint32)) for x, y in zip(a, b))


def alone_steps(build, steps):
    from skyephyx_b200 import Batch
    b = Batch()
    b.set_groups(1, 1)
    b.add_scene(staged(build))
    assert b.step(steps) == "ok"
    return b.get_state(0)[:2]


def test_prepare_then_step_equals_step():
    """avbd_batch_prepare (pools, launch and page-locked staging ahead of the
    first step) changes nothing in the results."""
    from skyephyx_b200 import Batch
    builders = mix_builders()
    runs = []
    for prep in (False, True):
        b = Batch()
        keep = [staged(f) for f in builders]
        for w in keep:
            b.add_scene(w)
        if prep:
            b.prepare()
            b.prepare()   # a second call is a no-op
        assert b.step(3) == "ok"
        runs.append([b.get_state(i)[:2] for i in range(len(builders))])
    for a, c in zip(*runs):
        assert same(a, c)
