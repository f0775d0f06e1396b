"""The CPU oracle: Eigen-shim self-tests, the colour-order harness self-check,
and the golden vectors produced by the compiled reference (no GPU)."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def test_shim_ldlt_against_numpy(oracle_mod):
    lib = oracle_mod._lib()
    rng = np.random.default_rng(0)
    worst = 0.0
    for t in range(600):
        J = rng.normal(size=(6, 8))
        A = (J @ J.T + 0.1 * np.eye(6)).astype(np.float32)
        b = rng.normal(size=6).astype(np.float32)
        if t % 3 == 0:   # particle-like system: zero angular block -> pseudo-inverse gives 0 there
            A[3:, :] = 0
            A[:, 3:] = 0
            b[3:] = 0
        x = np.zeros(6, np.float32)
        lib.orc_shim_ldlt6(_fp(np.asfortranarray(A).ravel(order="F").copy()), _fp(b), _fp(x))
        ref = np.linalg.lstsq(A.astype(np.float64), b.astype(np.float64), rcond=None)[0]
        worst = max(worst, np.abs(x - ref).max() / (np.abs(ref).max() + 1e-12))
        if t % 3 == 0:
            assert np.all(x[3:] == 0)
    assert worst < 1e-4


def test_shim_svd_and_eigen(oracle_mod):
    lib = oracle_mod._lib()
    rng = np.random.default_rng(1)
    for _ in range(500):
        F = (np.eye(3) + 0.3 * rng.normal(size=(3, 3))).astype(np.float32)
        U = np.zeros(9, np.float32)
        S = np.zeros(3, np.float32)
        V = np.zeros(9, np.float32)
        lib.orc_shim_svd3(_fp(F.ravel(order="F").copy()), _fp(U), _fp(S), _fp(V))
        U = U.reshape(3, 3, order="F")
        V = V.reshape(3, 3, order="F")
        assert np.abs(U @ np.diag(S) @ V.T - F).max() < 1e-5
        assert np.linalg.det(U) > 0 and np.linalg.det(V) > 0     # rotations (math.cpp:23-32)
        assert abs(S[0]) >= abs(S[1]) >= abs(S[2]) - 1e-6
        A = rng.normal(size=(3, 3)).astype(np.float32)
        A = A + A.T
        w = np.zeros(3, np.float32)
        Q = np.zeros(9, np.float32)
        lib.orc_shim_eig3(_fp(A.ravel(order="F").copy()), _fp(w), _fp(Q))
        Q = Q.reshape(3, 3, order="F")
        assert np.abs(A @ Q - Q @ np.diag(w)).max() < 1e-4
        assert np.all(np.diff(w) >= 0)
        F2 = rng.normal(size=(3, 2)).astype(np.float32)
        U2 = np.zeros(9, np.float32)
        S2 = np.zeros(2, np.float32)
        V2 = np.zeros(4, np.float32)
        lib.orc_shim_svd32(_fp(F2.ravel(order="F").copy()), _fp(U2), _fp(S2), _fp(V2))
        U2 = U2.reshape(3, 3, order="F")
        V2 = V2.reshape(2, 2, order="F")
        assert np.abs(U2[:, :2] @ np.diag(S2) @ V2.T - F2).max() < 1e-5


def test_identity_order_harness_equals_reference_step(oracle_mod):
    """The restated step with one colour per body in index order is Solver::Step() bit for bit."""
    from skyephyx_b200 import scenes
    for build in (scenes.pyramid_wall, scenes.level_joint_playground, scenes.level_cloth,
                  lambda s: scenes.fem_block(s, nx=7, ny=3, nz=3)):
        a = oracle_mod.OracleSolver()
        b = oracle_mod.OracleSolver()
        build(a)
        build(b)
        for _ in range(3):
            a.step()
            b.step_coloured(identity_order=True)
        for x, y in zip(a.get_state(), b.get_state()):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(oracle_mod, path):
    """The oracle reproduces the committed outputs of the reference bit for bit."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import golden_scenes, run
    name = os.path.basename(path)[:-4]
    g = np.load(path)
    build = golden_scenes()[name]
    for mode, coloured in (("seq", False), ("col", True)):
        pos, quat, (p1, i1), (pl, il), colours = run(name, build, coloured)
        assert np.array_equal(pos.view(np.uint32), g[f"{mode}_pos"].view(np.uint32)), mode
        assert np.array_equal(quat.view(np.uint32), g[f"{mode}_quat"].view(np.uint32)), mode
        assert np.array_equal(p1, g[f"{mode}_pairs"]) and np.array_equal(i1, g[f"{mode}_ids"])
        assert np.array_equal(pl, g[f"{mode}_last_pairs"]) and np.array_equal(il, g[f"{mode}_last_ids"])
        if coloured:
            assert np.array_equal(colours, g["col_colours"])


def test_golden_files_present():
    assert len(GOLDEN) >= 10


def test_colouring_is_proper(oracle_mod):
    """CPU twin of the device colouring: no two dynamic bodies sharing a force/energy share a colour."""
    from skyephyx_b200 import scenes
    o = oracle_mod.OracleSolver()
    scenes.fem_block(o, nx=6, ny=4, nz=4)
    o.step_coloured()
    col, k = o.colours()
    assert k > 1
    c = o.contacts()
    for (a, b), _ in c.items():
        if col[a] >= 0 and col[b] >= 0:
            assert col[a] != col[b]


def test_stvk_tet_oracle_is_sane(oracle_mod):
    """The StVK tet restatement (no reference counterpart): at small strain it
    moves a pinned beam like the reference's Neo-Hookean tet; under large
    sag it stays finite and stiffer-in-tension behaviour does not blow up."""
    from skyephyx_b200 import scenes
    nh = oracle_mod.OracleSolver()
    nh.make_tet_volume(-3.0, 0.0, -0.9, 9, 3, 3, 0.9, 8000.0, 0.3, 1.0, 0.5, True)
    sv = oracle_mod.OracleSolver()
    sv.make_stvk_tet_volume(-3.0, 0.0, -0.9, 9, 3, 3, 0.9, 8000.0, 0.3, 1.0, 0.5, True)
    for o in (nh, sv):
        assert o.step_coloured() == 0
    p_nh, p_sv = nh.get_state()[0], sv.get_state()[0]
    assert np.abs(p_nh - p_sv).max() < 1e-4
    big = oracle_mod.OracleSolver()
    scenes.stvk_block(big)
    for _ in range(60):
        big.step_coloured()
    assert np.isfinite(big.get_state()[0]).all()


FP64_SCENES = ["pyramid", "joint_playground", "soft_beam", "cloth", "mixed_300"]


@pytest.mark.parametrize("name", FP64_SCENES)
def test_fp64_oracle_agrees_with_fp32(oracle_mod, name):
    """The FP64 build (the reference's code carried out in double) is the
    FP32 oracle up to rounding: after one colour-ordered step the poses agree
    to 2e-6 and the contact manifolds and colours are the same."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import golden_scenes
    build = golden_scenes()[name]
    a = oracle_mod.OracleSolver()
    b = oracle_mod.OracleSolver(f64=True)
    build(a)
    build(b)
    assert a.step_coloured() == 0 and b.step_coloured() == 0
    pa, qa = a.get_state()[:2]
    pb, qb = b.get_state()[:2]
    assert pb.dtype == np.float64
    assert np.abs(pa - pb).max() <= 2e-6
    assert np.abs(qa - qb).max() <= 2e-6
    assert {k: v[0] for k, v in a.contacts().items()} == {k: v[0] for k, v in b.contacts().items()}
    assert a.colours()[1] == b.colours()[1]


def test_metrics_measure_the_state(oracle_mod):
    """orc_metrics: a resting pyramid has only gravitational energy (m g y)
    and no violation; lifting one box by 1 m adds m g; a joint pulled apart
    reports its positional violation."""
    from skyephyx_b200 import scenes
    o = oracle_mod.OracleSolver()
    scenes.pyramid_wall(o, rows=3)
    m = o.metrics()
    masses = 1000.0  # unit cubes of density 1000
    ys = o.get_state()[0][1:, 1]
    assert m["max_violation"] == 0.0 and m["kinetic_j"] == 0.0 and m["elastic_j"] == 0.0
    assert abs(m["potential_j"] - masses * 9.81 * float(np.sum(ys))) < 1e-3 * m["potential_j"]
    p = o.get_state()[0].copy()
    p[1, 1] += 1.0
    o.set_state(pos=p)
    assert abs(o.metrics()["potential_j"] - m["potential_j"] - masses * 9.81) < 1e-2
    j = oracle_mod.OracleSolver()
    b = j.add_body(scenes.CUBE, 1000.0, 0.5, (0.0, 5.0, 0.0), (1, 1, 1))
    j.add_joint(-1, (0.0, 5.5, 0.0), b, (0.0, 0.5, 0.0))
    assert j.metrics()["max_violation"] < 1e-6
    p = j.get_state()[0].copy()
    p[b, 1] -= 0.25
    j.set_state(pos=p)
    assert abs(j.metrics()["max_violation"] - 0.25) < 1e-5
