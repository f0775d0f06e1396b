"""Batched path: one persistent kernel per step over many scenes.

* a scene's result is bitwise the same alone and inside a mixed batch
  (one CTA runs a whole scene in a fixed per-body order);
* batched results match the oracle like the single-scene path does.
"""
import numpy as np
import pytest

from skyephyx_b200 import scenes
from conftest import rot_err

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
    """A collapsing pile and a settling stack, 30 steps, one lane per body:
    the batch with its in-CTA grid broadphase, the batch with the all-pairs
    loop, and the single-scene path with its grid-wide grid agree bit for
    bit."""
    from skyephyx_b200 import Batch, Solver
    for build in GRID_BUILDERS[1:3]:
        w = Solver()
        w.set_group(1)
        build(w)
        for _ in range(30):
            assert w.step() == "ok"
        results = [w.get_state()[:2]]
        for grid_min in (128, 0):
            b = Batch()
            b.set_groups(1, 4)
            b.set_grid_broadphase(grid_min)
            b.add_scene(staged(build))
            assert b.step(30) == "ok" and b.scene_status(0) == "ok"
            results.append(b.get_state(0)[:2])
        for other in results[1:]:
            assert same(results[0], other)


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


def test_prepare_then_remove_and_add_admits_the_new_scene():
    """Scenes staged by prepare() reach the device before a remove/add pair
    reuses their space: the newly admitted scene steps as it does alone."""
    from skyephyx_b200 import Batch
    builders = mix_builders()
    b = Batch()
    keep = [staged(f) for f in builders]
    for w in keep:
        b.add_scene(w)
    b.prepare()
    b.remove_scene(2)
    newcomer = lambda s: scenes.rigid_pile(s, 30, scenes.rng_for(4, 77), stack=True)
    slot = b.add_scene(staged(newcomer))
    assert b.scene_status(slot) == "ok"
    assert b.step(3) == "ok"
    ref = Batch()
    ref.add_scene(staged(newcomer))
    assert ref.step(3) == "ok"
    assert same(b.get_state(slot)[:2], ref.get_state(0)[:2])
    # the other scenes are the ones staged before the swap
    alone = Batch()
    alone.add_scene(staged(builders[0]))
    assert alone.step(3) == "ok"
    assert same(b.get_state(0)[:2], alone.get_state(0)[:2])


def moving_boxes(s, seed, n=24):
    """Boxes thrown with linear and angular velocity over a static ground."""
    rng = np.random.default_rng(seed)
    s.add_body(scenes.CUBE, 1.0, 0.5, (0, -0.5, 0), (40, 1, 40), is_static=True)
    for i in range(n):
        s.add_body(scenes.CUBE, 1.0 + 0.1 * i, 0.4, (rng.uniform(-4, 4), rng.uniform(1, 4), rng.uniform(-4, 4)),
                   (rng.uniform(0.4, 1.2), rng.uniform(0.4, 1.2), rng.uniform(0.4, 1.2)),
                   vel=tuple(rng.uniform(-3, 3, 3)), omega=tuple(rng.uniform(-2, 2, 3)))


def test_staged_upload_equals_direct_upload_for_moving_scenes():
    """The first step's upload of staged scenes (one copy per device array;
    zero data left to the freshly zeroed pools; the last and inertial poses
    filled from the pose on the device) gives the device state a scene placed
    in reserved pools gets from its own copies, bit for bit, for scenes that
    start with velocities, at rest, or with tets."""
    from skyephyx_b200 import Batch
    builders = [lambda s: moving_boxes(s, 11), lambda s: scenes.fem_scene(s, 700, scenes.rng_for(4, 1)),
                lambda s: moving_boxes(s, 12, n=40), lambda s: scenes.rigid_pile(s, 40, scenes.rng_for(4, 2))]
    first = Batch()
    for f in builders:
        first.add_scene(staged(f))
    assert first.step(3) == "ok"
    later = Batch()
    later.reserve(4096, 1024, 4096, 256, 8)   # pools in place: each scene is copied on its own
    slots = [later.add_scene(staged(f)) for f in builders]
    assert later.step(3) == "ok"
    for i, slot in enumerate(slots):
        assert same(first.get_state(i)[:4], later.get_state(slot)[:4]), f"scene {i}"


def headline_slice(n_sample=256):
    """A slice of the 4,096-scene batched mix: every 16th scene plus the eight
    largest rigid and the eight largest FEM scenes."""
    specs = scenes.batch_mix_specs()
    rigid = sorted((i for i, sp in enumerate(specs) if sp[0] != "fem"), key=lambda i: -specs[i][1])[:8]
    fem = sorted((i for i, sp in enumerate(specs) if sp[0] == "fem"), key=lambda i: -specs[i][1])[:8]
    picks = sorted(set(range(0, len(specs), len(specs) // n_sample)) | set(rigid) | set(fem))
    return [specs[i] for i in picks]


def test_headline_launch_matches_oracle(oracle_mod):
    """The launch the benchmark runs the 4,096-scene mix with (the autotuned
    kernel build, lanes per body, flat FEM sweep, team split and grid
    threshold for this mix) on a 270-scene slice that holds the mix's largest
    scenes: after one step every scene's positions and rotations are within
    1e-4 of the colour-ordered oracle, and its contact-point and colour
    counts are equal."""
    import os
    from skyephyx_b200 import Batch, autotune
    specs = headline_slice()
    full = scenes.batch_mix_specs()
    nfem = sum(1 for sp in full if sp[0] == "fem")
    # the signature of the full mix (4,096 scenes, 25% FEM, ~512 bodies each)
    cfg = autotune.lookup(autotune.signature(len(full), nfem, 512 * len(full)))
    b = Batch()
    keep = []
    for sp in specs:
        w = staged(lambda s: scenes.build_spec(s, sp))
        keep.append(w)
        b.add_scene(w)
    autotune.apply(b, cfg)
    assert b.step(1) == "ok"
    orcs = []
    for sp in specs:
        o = oracle_mod.OracleSolver()
        scenes.build_spec(o, sp)
        orcs.append(o)
    oracle_mod.step_many(orcs, 1, os.cpu_count() or 8, coloured=True)
    worst_p = worst_r = 0.0
    for i, (sp, o) in enumerate(zip(specs, orcs)):
        info = b.scene_info(i)
        assert info["status"] == 0, f"{sp}: {info}"
        pb, qb = b.get_state(i)[:2]
        po, qo = o.get_state()[:2]
        dp = float(np.abs(pb - po).max(initial=0.0))
        dr = float(rot_err(qb, qo).max(initial=0.0))
        worst_p, worst_r = max(worst_p, dp), max(worst_r, dr)
        assert dp <= 1e-4 and dr <= 1e-4, f"{sp}: |dpos| {dp:.3g} m, |drot| {dr:.3g} rad"
        points = sum(len(v[0]) for v in o.contacts().values())
        assert info["contacts"] == points, f"{sp}: {info['contacts']} contact points vs {points}"
        assert info["colours"] == o.colours()[1], f"{sp}: colours"
    print(f"headline slice: {len(specs)} scenes, max |dpos| {worst_p:.3g} m, max |drot| {worst_r:.3g} rad")


def test_scene_snapshot_restores_elsewhere_and_replays():
    """Pre-emption of scenes inside a batch: after 4 steps each scene is
    snapshotted and removed, a newcomer takes the freed space, the snapshots
    come back (in reverse order, so at other pool offsets) and 5 more steps
    follow.  Every restored scene ends bitwise where it ends running 9 steps
    alone (the flat FEM sweep's tet-term records and the grid broadphase
    included)."""
    from skyephyx_b200 import Batch, GROUP_FLAT
    builders = [
        lambda s: scenes.rigid_pile(s, 300, scenes.rng_for(4, 31), stack=False),
        lambda s: scenes.fem_scene(s, 700, scenes.rng_for(4, 32)),
        scenes.level_joint_playground,
        scenes.level_cloth,
    ]
    b = Batch()
    b.set_groups(1, GROUP_FLAT)
    b.reserve(bodies=20000, forces=2000, tets=20000, tris=2000, scenes=16)
    keep = [staged(f) for f in builders]
    ids = [b.add_scene(w) for w in keep]
    assert b.step(4) == "ok"
    snaps = [b.snapshot_scene(i) for i in ids]
    for i in ids:
        b.remove_scene(i)
    filler = b.add_scene(staged(lambda s: scenes.pyramid_wall(s, rows=7)))
    back = {k: b.restore_scene(snaps[k]) for k in reversed(range(len(builders)))}
    assert b.step(5) == "ok"
    for k, f in enumerate(builders):
        assert b.scene_status(back[k]) == "ok"
        alone = Batch()
        alone.set_groups(1, GROUP_FLAT)
        alone.add_scene(staged(f))
        assert alone.step(9) == "ok"
        assert same(b.get_state(back[k])[:2], alone.get_state(0)[:2]), f"scene {k}"
        assert b.scene_info(back[k])["steps"] == 9
    assert b.scene_status(filler) == "ok"


def test_cluster_runs_change_nothing():
    """Scenes run by a whole thread-block cluster (ranks over 2 or 4 CTAs,
    team scalars and stage in the first CTA's shared memory) end bitwise
    where the plain launch leaves them, large and small, rigid and FEM."""
    from skyephyx_b200 import Batch, GROUP_FLAT
    builders = mix_builders() + [
        lambda s: scenes.rigid_pile(s, 400, scenes.rng_for(4, 41), stack=False),
        lambda s: scenes.rigid_pile(s, 300, scenes.rng_for(4, 42), stack=True),
        lambda s: scenes.fem_scene(s, 2500, scenes.rng_for(4, 43)),
    ]
    runs = []
    for cluster, min_units in ((1, 0), (2, 0), (4, 300)):
        b = Batch()
        b.set_groups(1, GROUP_FLAT)
        b.set_team_work(2)
        b.set_cluster(cluster, min_units)
        keep = [staged(f) for f in builders]
        for w in keep:
            b.add_scene(w)
        assert b.step(3) == "ok"
        runs.append([b.get_state(i)[:2] for i in range(len(builders))])
        for i in range(len(builders)):
            assert b.scene_status(i) == "ok", (cluster, i)
    for run in runs[1:]:
        for i, (a, c) in enumerate(zip(runs[0], run)):
            assert same(a, c), f"scene {i}"


def test_scene_timing_stamps_every_scene_and_changes_nothing():
    """Per-scene device timing: after a step every slot holds its nine stamps
    in order (start, the phase ends, end) within one launch, and the results
    are bitwise those of a batch stepped without timing."""
    from skyephyx_b200 import Batch
    builders = mix_builders()
    runs = []
    for timed in (False, True):
        b = Batch()
        keep = [staged(f) for f in builders]
        for w in keep:
            b.add_scene(w)
        assert b.step(1) == "ok"
        if timed:
            b.set_scene_timing(True)
        assert b.step(2) == "ok"
        runs.append([b.get_state(i)[:2] for i in range(len(builders))])
        if timed:
            t = b.scene_times()
            assert t.shape == (len(builders), b.SCENE_STAMPS)
            assert (t[:, 0] > 0).all() and (np.diff(t, axis=1) >= 0).all() and (t[:, -1] > t[:, 0]).all()
            # the stamps of the last step lie within one launch
            assert t[:, -1].max() - t[:, 0].min() < 5e9
            b.set_scene_timing(False)
            with pytest.raises(Exception):
                b.scene_times()
    for i, (a, c) in enumerate(zip(*runs)):
        assert same(a, c), f"scene {i}"


def test_overlapped_pose_readback_equals_synchronous():
    """avbd_batch_read_poses (device snapshot, copy on a second stream while
    the next step runs) delivers each step's poses exactly as the
    synchronous avbd_batch_get_all_poses read right after that step."""
    import ctypes as C
    from skyephyx_b200 import Batch
    b = Batch()
    keep = [staged(f) for f in mix_builders()[:4]]
    for w in keep:
        b.add_scene(w)
    assert b.step(1) == "ok"
    lib, h = b._lib, b._h
    n = lib.avbd_batch_get_all_poses(h, None, None, 1 << 30)
    fp = C.POINTER(C.c_float)
    sync = []
    for _ in range(3):
        p, q = np.zeros((n, 4), np.float32), np.zeros((n, 4), np.float32)
        assert lib.avbd_batch_get_all_poses(h, p.ctypes.data_as(fp), q.ctypes.data_as(fp), n) == n
        sync.append((p, q))
        assert b.step(1) == "ok"
    # the same three steps again, from the same start, read with overlap
    b2 = Batch()
    keep2 = [staged(f) for f in mix_builders()[:4]]
    for w in keep2:
        b2.add_scene(w)
    assert b2.step(1) == "ok"
    bufs = [(np.zeros((n, 4), np.float32), np.zeros((n, 4), np.float32)) for _ in range(3)]
    for k in range(3):
        p, q = bufs[k]
        assert b2._lib.avbd_batch_read_poses(b2._h, p.ctypes.data_as(fp), q.ctypes.data_as(fp), n) == n
        assert b2.step(1) == "ok"
    assert b2._lib.avbd_batch_read_poses_wait(b2._h) == 0
    for (p, q), (ps, qs) in zip(bufs, sync):
        assert np.array_equal(p.view(np.uint32), ps.view(np.uint32))
        assert np.array_equal(q.view(np.uint32), qs.view(np.uint32))
