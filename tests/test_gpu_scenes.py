"""Scene builders and consumers beyond the step:

* makeTetSphere (geometry.cpp:106-232) and the safety net (levels.h:493-547)
  as batched fixtures against the oracle;
* the headless pose export in the renderer's 128-byte instance layout
  (RenderEngine.hpp:43-49, packed as RenderEngine.cpp:951-1000 packs it)
  against a CPU pack of the same poses.
"""
import numpy as np
import pytest

from skyephyx_b200 import scenes
from conftest import rot_err

pytestmark = pytest.mark.gpu


def staged(build):
    from skyephyx_b200 import Solver
    s = Solver()
    build(s)
    return s


def test_tet_sphere_builds_the_reference_sphere(oracle_mod):
    """The library's makeTetSphere places the reference's particles bit for
    bit (positions from the same float operations)."""
    g = staged(scenes.level_soft_spheres)
    o = oracle_mod.OracleSolver()
    scenes.level_soft_spheres(o)
    assert g.num_bodies == o.num_bodies == 150
    pg, po = g.get_state()[0], o.get_state()[0]
    assert np.array_equal(pg.view(np.uint32), po.view(np.uint32))


BATCH_FIXTURES = {
    "soft_spheres": scenes.level_soft_spheres,
    "safety_net": scenes.level_safety_net,
    "rope_bridge": scenes.level_joint_playground,
    "cloth": scenes.level_cloth,
}


def test_reference_scenes_as_batched_fixtures(oracle_mod):
    """The sphere, the net, the joint playground's rope bridge and the cloth
    in one batch: after one step each matches the colour-ordered oracle (1e-4
    m / rad, equal colour counts); after ten, within 1e-3."""
    from skyephyx_b200 import Batch
    names = list(BATCH_FIXTURES)
    b = Batch()
    keep = [staged(BATCH_FIXTURES[n]) for n in names]
    for w in keep:
        b.add_scene(w)
    orcs = []
    for n in names:
        o = oracle_mod.OracleSolver()
        BATCH_FIXTURES[n](o)
        orcs.append(o)
    for step in range(10):
        assert b.step(1) == "ok"
        for i, (n, o) in enumerate(zip(names, orcs)):
            assert o.step_coloured() == 0
            pb, qb = b.get_state(i)[:2]
            po, qo = o.get_state()[:2]
            tol = 1e-4 if step == 0 else 1e-3
            assert np.abs(pb - po).max() <= tol, f"{n} step {step}"
            assert rot_err(qb, qo).max() <= tol, f"{n} step {step}"
            if step == 0:
                assert b.scene_info(i)["colours"] == o.colours()[1], n


def quat_matrix(q):
    w, x, y, z = [float(v) for v in q]
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def cpu_pack(models, scales, colors, removed, pos, quat):
    """GPUInstanceData records as the renderer packs them: per model type (in
    ModelType order) the bodies in id order; model matrix R diag(s) | p,
    normal matrix its inverse transpose, colour (r, g, b, 1)."""
    out, first, count = [], [], []
    for m in (0, 1, 2):
        first.append(len(out))
        for b in range(len(models)):
            if models[b] != m or removed[b]:
                continue
            M = quat_matrix(quat[b]) * np.asarray(scales[b], np.float64)[None, :]
            N = np.linalg.inv(M).T
            rec = np.zeros(32)
            rec[0:16] = np.vstack([np.hstack([M, np.asarray(pos[b], np.float64)[:, None]]), [0, 0, 0, 1]]).T.ravel()
            for k in range(3):
                rec[16 + 4 * k:16 + 4 * k + 3] = N[:, k]
            rec[28:31] = colors[b]
            rec[31] = 1.0
            out.append(rec)
        count.append(len(out) - first[-1])
    return np.array(out), first, count


def export_scene(s):
    rng = np.random.default_rng(11)
    models, scales, colors = [scenes.CUBE], [(20.0, 1.0, 20.0)], [(1.0, 1.0, 1.0)]
    s.add_body(scenes.CUBE, 1.0, 0.5, (0, -0.5, 0), scales[0], is_static=True)
    for i in range(9):
        m = scenes.SPHERE if i % 3 == 1 else scenes.CUBE
        sc = (1.0, 0.5 + 0.1 * i, 0.8)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        b = s.add_body(m, 1000.0, 0.5, (1.6 * i - 7, 1.5 + 0.4 * i, 0.3 * i), sc, quat=tuple(q))
        col = (i / 9.0, 0.5, 1.0 - i / 9.0)
        s.set_color(b, col)
        models.append(m)
        scales.append(sc)
        colors.append(col)
    return models, scales, colors


def test_instance_export_matches_cpu_pack():
    import torch
    from skyephyx_b200 import Batch, Solver
    s = Solver()
    models, scales, colors = export_scene(s)
    for _ in range(6):
        assert s.step() == "ok"
    s.remove_body(4)
    removed = [False] * len(models)
    removed[4] = True
    out, first, count = s.export_instances()
    p, q = s.get_state()[:2]
    ref, rfirst, rcount = cpu_pack(models, scales, colors, removed, p, q)
    assert first == rfirst and count == rcount and out.shape == ref.shape
    np.testing.assert_allclose(out, ref, rtol=2e-5, atol=2e-6)
    # into device memory a renderer could read in place
    buf = torch.zeros((len(models), 32), dtype=torch.float32, device="cuda")
    k, dfirst, dcount = s.export_instances(buf.data_ptr())
    torch.cuda.synchronize()
    assert k == len(out) and dfirst == first and dcount == count
    assert np.array_equal(buf.cpu().numpy()[:k], out)
    # a scene of a batch exports its own records
    w = Solver()
    export_scene(w)
    bt = Batch()
    bt.set_groups(4, 8)
    bt.add_scene(w)
    assert bt.step(6) == "ok"
    import ctypes as C
    from skyephyx_b200._lib import load
    lib = load()
    rec = np.zeros((len(models), 32), np.float32)
    fm, cm = (C.c_int32 * 3)(), (C.c_int32 * 3)()
    n = lib.avbd_batch_export_instances(bt._h, 0, rec.ctypes.data, len(models), fm, cm)
    assert n == len(models)
    p2, q2 = bt.get_state(0)[:2]
    ref2, _, _ = cpu_pack(models, scales, colors, [False] * len(models), p2, q2)
    np.testing.assert_allclose(rec, ref2, rtol=2e-5, atol=2e-6)
