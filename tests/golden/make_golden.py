"""Generates the golden vectors in tests/golden/ by running the reference.

The reference's physics (SkyePhyX src/physics, src/helpers) is compiled
unmodified by oracle/Makefile from a local checkout of the reference
(default /root/reference); this script runs it on the demo scenes of
src/levels.h (re-expressed in skyephyx_b200/scenes.py) and on small instances
of the workload scenes, and stores poses at a few checkpoints over 60 steps,
the contact manifolds after the first and the last step, and the colour
assignment of the colour-ordered step.

    python tests/golden/make_golden.py [--ref /path/to/SkyePhyX]

Regenerate only deliberately: the tests compare the oracle against these.
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

STEPS = 60
CHECKPOINTS = (1, 2, 5, 10, 20, 40, 60)


def golden_scenes():
    from skyephyx_b200 import scenes
    d = dict(scenes.LEVELS)
    d["pyramid_wall_20"] = scenes.pyramid_wall
    d["fem_block_9x4x4"] = lambda s: scenes.fem_block(s, nx=9, ny=4, nz=4)
    d["mixed_300"] = lambda s: scenes.mixed_large(s, n_boxes=300, n_chains=3, links=8, n_springs=40)
    d["fem_scene_600"] = lambda s: scenes.fem_scene(s, 600, scenes.rng_for(4, 3))
    return d


def _contacts(o):
    c = o.contacts()
    keys = sorted(c)
    pairs = np.array(keys, np.int32).reshape(-1, 2)
    ids = np.full((len(keys), 8), 0xFFFFFFFF, np.uint32)
    for i, key in enumerate(keys):
        ids[i, :len(c[key][0])] = c[key][0]
    return pairs, ids


def run(name, build, coloured, steps=STEPS):
    """Steps the reference `steps` times; returns poses at CHECKPOINTS, the
    contacts after step 1 and after the last step, and the step-1 colours."""
    from oracle.oracle import OracleSolver
    o = OracleSolver()
    build(o)
    pos, quat = [], []
    first = last = None
    colours = None
    for k in range(1, steps + 1):
        if coloured:
            o.step_coloured()
        else:
            o.step()
        if k in CHECKPOINTS:
            p, q = o.get_state()[:2]
            pos.append(p)
            quat.append(q)
        if k == 1:
            first = _contacts(o)
            if coloured:
                colours = o.colours()[0]
    last = _contacts(o)
    return np.stack(pos), np.stack(quat), first, last, colours


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="SkyePhyX source tree (default: $SKYEPHYX_REF or the oracle "
                                                 "Makefile's default)")
    args = ap.parse_args()
    from oracle import oracle
    oracle.build(args.ref)
    for name, build in golden_scenes().items():
        out = {}
        for mode, coloured in (("seq", False), ("col", True)):
            pos, quat, (p1, i1), (pl, il), colours = run(name, build, coloured)
            out[f"{mode}_pos"] = pos
            out[f"{mode}_quat"] = quat
            out[f"{mode}_pairs"] = p1
            out[f"{mode}_ids"] = i1
            out[f"{mode}_last_pairs"] = pl
            out[f"{mode}_last_ids"] = il
            if colours is not None:
                out["col_colours"] = colours
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
