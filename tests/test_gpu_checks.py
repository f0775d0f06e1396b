"""The debug build (libavbd_checks.so, AVBD_CHECKS): device index checks at
the incidence, broadphase, colour-list, tet-term record and contact writes
record a violation in a check word instead of trapping.  On valid scenes no
check fails and every result is bitwise the release build's (the checks only
read indices)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RUN = r"""
import json, sys
import numpy as np
sys.path.insert(0, {root!r})
from skyephyx_b200 import Batch, Solver, scenes, GROUP_FLAT
import skyephyx_b200._lib as L
lib = L.load()
import ctypes as C
out = {{}}
w = Solver()
scenes.mixed_large(w, n_boxes=600, n_chains=8, links=4, n_springs=16, seed_scene=3)
for _ in range(3):
    assert w.step() == "ok"
word = (C.c_int32 * 4)()
out["world_checks"] = lib.avbd_check_word(w.handle, word)
out["world_word"] = list(word)
out["world_pos"] = w.get_state()[0].tolist()
b = Batch()
b.set_groups(1, GROUP_FLAT)
b.set_team_work(2)
keep = []
for f in (lambda s: scenes.pyramid_wall(s, rows=8), lambda s: scenes.fem_scene(s, 700, scenes.rng_for(4, 1)),
          lambda s: scenes.rigid_pile(s, 300, scenes.rng_for(4, 2), stack=False), scenes.level_joint_playground):
    s = Solver(); f(s); keep.append(s); b.add_scene(s)
assert b.step(3) == "ok"
out["batch_checks"] = lib.avbd_batch_check_word(b._h, word)
out["batch_word"] = list(word)
out["batch_pos"] = [b.get_state(i)[0].tolist() for i in range(len(keep))]
print(json.dumps(out))
"""


def run(checks):
    env = dict(os.environ)
    env["AVBD_CHECKS"] = "1" if checks else "0"
    r = subprocess.run([sys.executable, "-c", RUN.format(root=ROOT)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_checked_build_flags_nothing_and_matches_release():
    rel, dbg = run(False), run(True)
    assert rel["world_checks"] == 0 and rel["batch_checks"] == 0   # release build: no checks compiled
    assert dbg["world_checks"] == 1 and dbg["batch_checks"] == 1
    assert dbg["world_word"] == [0, 0, 0, 0], dbg["world_word"]
    assert dbg["batch_word"] == [0, 0, 0, 0], dbg["batch_word"]
    assert np.array_equal(np.array(rel["world_pos"], np.float32).view(np.uint32),
                          np.array(dbg["world_pos"], np.float32).view(np.uint32))
    for a, c in zip(rel["batch_pos"], dbg["batch_pos"]):
        assert np.array_equal(np.array(a, np.float32).view(np.uint32), np.array(c, np.float32).view(np.uint32))
