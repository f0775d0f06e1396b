"""Failure paths of the step, each against the oracle, with every failure made
on the host (an out-of-bounds launch, a velocity spike or a NaN pose written
through set_state, a force that breaks under its own load); nothing here
faults or stalls a GPU.

* out-of-bounds removal (solver.cpp:521-534) with the forces of the removed
  body dropped (geometry.cpp:11-25);
* explosion / emergencyStop (solver.cpp:182-196, 528-529): the step ends
  before post-stabilisation and later steps are no-ops;
* a NaN pose: reported and frozen (the reference would keep stepping NaNs);
* fracture of a spring and of a joint row with the reset of every manifold
  of their bodies (solver.cpp:473-481);
* in a batch, an exploding and a NaN scene leave every other scene bitwise
  as it is alone.
"""
import numpy as np
import pytest

from skyephyx_b200 import INF, scenes
from conftest import rot_err

pytestmark = pytest.mark.gpu


def oob_scene(s):
    """A small wall plus, created last, a box leaving the +x bound within one
    step (60 m/s, under the 500 m/s explosion limit), tied to a world anchor by
    a soft spring that goes with it."""
    scenes.pyramid_wall(s, rows=4)
    b = s.add_body(scenes.CUBE, 1000.0, 0.5, (49.4, 3.0, 0.0), (0.5, 0.5, 0.5), vel=(60.0, 0.0, 0.0))
    f = s.add_spring(-1, (40.0, 3.0, 0.0), b, (0.0, 0.0, 0.0), 1.0)
    return b, f


def fracture_scene(s):
    """Three boxes on a ground box: a hangs from a breakable spring (fracture
    50 N), c sits on b and hangs from a joint whose y row breaks at 50 N."""
    s.add_body(scenes.CUBE, 1.0, 0.5, (0, -0.5, 0), (20, 1, 20), is_static=True)
    a = s.add_body(scenes.CUBE, 1000.0, 0.5, (0, 0.5, 0), (1, 1, 1))
    s.add_body(scenes.CUBE, 1000.0, 0.5, (3, 0.5, 0), (1, 1, 1))
    c = s.add_body(scenes.CUBE, 1000.0, 0.5, (3, 1.5, 0), (1, 1, 1))
    fs = s.add_spring(-1, (0, 3.0, 0), a, (0, 0.5, 0), 1e4, 1.0, False, 50.0)
    fj = s.add_joint(-1, (3, 2.2, 0), c, (0, 0.5, 0), (INF,) * 6, (INF, 50.0, INF, INF, INF, INF))
    return fs, fj


def explode_scene(s):
    scenes.pyramid_wall(s, rows=3)
    return s.add_body(scenes.CUBE, 1000.0, 0.5, (-10.0, 5.0, 0.0), (1, 1, 1))


def spike(s, body, value):
    """Writes a velocity (value: float) or NaN position (value: None) into one body."""
    p, q, v, w = s.get_state()
    if value is None:
        p = p.copy()
        p[body] = np.nan
        s.set_state(pos=p)
    else:
        v = v.copy()
        v[body] = (value, 0.0, 0.0)
        s.set_state(vel=v)


def both(build, oracle_mod):
    from skyephyx_b200 import Solver
    g, o = Solver(), oracle_mod.OracleSolver()
    return g, o, build(g), build(o)


def test_out_of_bounds_removal_matches_oracle(oracle_mod):
    g, o, (b, f), _ = both(oob_scene, oracle_mod)
    for step in range(3):
        assert g.step() == "ok"
        assert o.step_coloured() == 0
        pg, qg = g.get_state()[:2]
        po, qo = o.get_state()[:2]
        # the removed body reads NaN on both sides, every other body agrees
        assert np.isnan(pg[b]).all() and np.isnan(po[b]).all(), f"step {step}"
        keep = np.ones(len(pg), bool)
        keep[b] = False
        tol = 1e-4 if step == 0 else 1e-3
        assert np.abs(pg[keep] - po[keep]).max() <= tol, f"step {step}"
        assert rot_err(qg[keep], qo[keep]).max() <= tol, f"step {step}"
        assert not g.force_live(f) and not o.force_live(f)
        assert set(g.contacts()) == set(o.contacts()), f"step {step}"
    g.close()


def test_explosion_stops_like_emergency_stop(oracle_mod):
    g, o, b, _ = both(explode_scene, oracle_mod)
    spike(g, b, 2000.0)
    spike(o, b, 2000.0)
    assert g.step() == "exploded"
    assert o.step_coloured() == 1
    assert g.emergency_stop and o.emergency_stop
    pg, qg = g.get_state()[:2]
    po, qo = o.get_state()[:2]
    # the step ended before post-stabilisation on both sides
    assert np.abs(pg - po).max() <= 1e-4
    assert rot_err(qg, qo).max() <= 1e-4
    # later steps are no-ops
    assert g.step() == "exploded"
    assert o.step_coloured() == 1
    assert np.array_equal(g.get_state()[0], pg)
    assert np.array_equal(o.get_state()[0], po)
    g.close()


def test_nan_pose_is_reported_and_frozen(oracle_mod):
    from skyephyx_b200 import Solver
    g = Solver()
    b = explode_scene(g)
    assert g.step() == "ok"
    spike(g, b, None)
    assert g.step() == "nan"
    assert g.emergency_stop
    frozen = g.get_state()[0]
    assert g.step() == "nan"
    assert np.array_equal(g.get_state()[0], frozen, equal_nan=True)
    g.close()


def test_fracture_resets_linked_manifolds_like_oracle(oracle_mod):
    g, o, (fs, fj), _ = both(fracture_scene, oracle_mod)
    for step in range(3):
        assert g.step() == "ok"
        assert o.step_coloured() == 0
        assert not g.force_live(fs) and not o.force_live(fs), f"step {step}"
        assert not g.force_live(fj) and not o.force_live(fj), f"step {step}"
        pg, qg = g.get_state()[:2]
        po, qo = o.get_state()[:2]
        tol = 1e-4 if step == 0 else 1e-3
        assert np.abs(pg - po).max() <= tol, f"step {step}"
        assert rot_err(qg, qo).max() <= tol, f"step {step}"
        cg, co = g.contacts(), o.contacts()
        assert set(cg) == set(co), f"step {step}"
        for pair in co:
            ids_g, dg = cg[pair]
            ids_o, do = co[pair]
            assert ids_g == ids_o, f"step {step} {pair}"
            # penalty and lambda of every row: the reset manifolds start the
            # next iteration from zero on both sides
            np.testing.assert_allclose(dg[:, 10:16], do[:, 10:16], rtol=1e-3, atol=1e-2,
                                       err_msg=f"step {step} {pair}")
    g.close()


def test_failing_scenes_leave_batch_neighbours_unchanged():
    from skyephyx_b200 import Batch, Solver
    rng = scenes.rng_for

    def exploding(s):
        b = explode_scene(s)
        spike(s, b, 2000.0)

    def nan_pose(s):
        b = explode_scene(s)
        spike(s, b, None)

    builders = [
        lambda s: scenes.pyramid_wall(s, rows=6),
        exploding,
        lambda s: scenes.fem_scene(s, 700, rng(4, 1)),
        nan_pose,
        lambda s: scenes.rigid_pile(s, 80, rng(4, 3), stack=False),
    ]
    failing = {1: "exploded", 3: "nan"}
    mix = Batch()
    keep = []
    for build in builders:
        w = Solver()
        build(w)
        keep.append(w)
        mix.add_scene(w)
    assert mix.step(3) == "ok"
    for i, build in enumerate(builders):
        if i in failing:
            assert mix.scene_status(i) == failing[i], f"scene {i}"
            continue
        assert mix.scene_status(i) == "ok"
        alone = Batch()
        w = Solver()
        build(w)
        alone.add_scene(w)
        assert alone.step(3) == "ok"
        pa, qa = alone.get_state(0)[:2]
        pm, qm = mix.get_state(i)[:2]
        assert np.array_equal(pa.view(np.uint32), pm.view(np.uint32)), f"scene {i}"
        assert np.array_equal(qa.view(np.uint32), qm.view(np.uint32)), f"scene {i}"
