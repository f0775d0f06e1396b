"""Launch-shape autotuner of the batched persistent kernel.

Knobs (all exact: they change only which lanes do which work, never the
arithmetic of a scene, so every candidate gives bitwise-identical results
for a given lanes-per-body choice):
  * kernel build: CTA size bound and register budget (156, 128, 80 or 64
    registers per thread at 256 threads; 512- and 1024-thread builds);
  * threads per CTA;
  * lanes sharing one body's primal update, for rigid and for FEM scenes
    (64: the term-per-lane flat sweep of FEM scenes);
  * scene work per lane below which a CTA splits into teams running one
    scene each.

``tune(staged_solvers)`` times every candidate on the given staged scenes
(device time of a few steps after a warm-up) and returns the fastest;
``load_table()``/``save_table()`` keep results as JSON keyed by device name
and a coarse signature of the scene mix.
"""
from __future__ import annotations

import itertools
import json
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "autotune_table.json")

DEFAULT = {"variant": 4, "threads": 256, "rigid_group": 1, "fem_group": 64}

# largest CTA each kernel build serves (avbd_batch_set_kernel)
VARIANT_MAX_THREADS = {1: 256, 2: 256, 3: 256, 4: 256, 5: 512, 6: 512, 7: 1024}

SPACE = {
    "variant": (1, 2, 3, 4, 5, 6, 7),
    "threads": (128, 256, 512, 1024),
    "rigid_group": (1, 2),
    "fem_group": (2, 4, 8, 64),   # 64: term-per-lane flat sweep
    "team_work": (0, 2, 4, 8),    # scene work per lane below which CTAs split into teams
    "grid_min": (0, 128, 512),    # scenes from this many bodies use the grid broadphase
    "fem_team_work": (0, 4, 8, 16),   # the split threshold for scenes with tets
    "queue_body_weight": (1, 2, 3, 4),   # queue key: weight x bodies + tets
}


def signature(n_scenes: int, n_fem: int, n_bodies: int) -> str:
    """Coarse key: scene count, FEM share and bodies per scene, bucketed."""
    fem_pct = int(round(100.0 * n_fem / max(1, n_scenes) / 5.0)) * 5
    bps = 1 << max(0, int(round(__import__("math").log2(max(1, n_bodies / max(1, n_scenes))))))
    return f"scenes{n_scenes}-fem{fem_pct}-bps{bps}"


def device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "cuda"


def load_table() -> dict:
    if os.path.exists(TABLE):
        with open(TABLE) as f:
            return json.load(f)
    return {}


def save_table(table: dict) -> None:
    with open(TABLE, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)


def lookup(sig: str) -> dict:
    t = load_table().get(device_name(), {})
    return dict(t.get(sig, DEFAULT))


def apply(batch, cfg: dict) -> None:
    """Applies a configuration to a Batch that has not been stepped yet."""
    batch.set_groups(cfg["rigid_group"], cfg["fem_group"])
    batch.set_kernel(cfg["variant"])
    batch.set_launch(cfg["threads"], 0)
    batch.set_team_work(cfg.get("team_work", 0))
    batch.set_fem_team_work(cfg.get("fem_team_work", 0))
    batch.set_grid_broadphase(cfg.get("grid_min", 128))
    if cfg.get("cluster", 1) > 1:
        batch.set_cluster(cfg["cluster"], cfg.get("cluster_min", 0))
    if cfg.get("queue_body_weight", 1) != 1:
        batch.set_queue_weight(cfg["queue_body_weight"])


def candidates(space=SPACE):
    """Every combination whose CTA size the kernel build serves."""
    keys = list(space)
    for vals in itertools.product(*(space[k] for k in keys)):
        cfg = dict(zip(keys, vals))
        if cfg["threads"] <= VARIANT_MAX_THREADS.get(cfg["variant"], 256):
            yield cfg


def time_config(staged, cfg, steps=3, warmup=2, iterations=10):
    from .solver import Batch
    b = Batch(iterations=iterations)
    for s in staged:
        b.add_scene(s)
    apply(b, cfg)
    b.step(warmup)
    b.step(steps)
    ms = b.last_ms / steps
    b.close()
    return ms


def tune(staged, space=SPACE, steps=3, warmup=2, log=None, start=None, rounds=2):
    """Coordinate descent from `start` (default DEFAULT): each knob in turn
    takes its fastest value with the others fixed, for up to `rounds` passes
    or until nothing changes.  Returns (best_cfg, best_ms, results)."""
    results = []
    t0 = time.perf_counter()
    cache = {}

    def measure(cfg):
        key = tuple(sorted(cfg.items()))
        if key not in cache:
            if cfg["threads"] > VARIANT_MAX_THREADS.get(cfg["variant"], 256):
                cache[key] = float("inf")
            else:
                cache[key] = time_config(staged, cfg, steps, warmup)
                results.append((dict(cfg), cache[key]))
                if log:
                    log(f"{cfg} {cache[key]:.3f} ms/step")
        return cache[key]

    best = dict(start or DEFAULT)
    best_ms = measure(best)
    for _ in range(rounds):
        changed = False
        for knob, values in space.items():
            for v in values:
                cfg = dict(best, **{knob: v})
                ms = measure(cfg)
                if ms < best_ms:
                    best, best_ms, changed = cfg, ms, True
        if not changed:
            break
    if log:
        log(f"tuned {len(results)} candidates in {time.perf_counter() - t0:.1f} s: {best} {best_ms:.3f} ms")
    return best, best_ms, results


if __name__ == "__main__":
    import argparse
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    ap = argparse.ArgumentParser(description="tune the batched kernel on the bench scene mix")
    ap.add_argument("--scenes", type=int, default=1024)
    ap.add_argument("--save", action="store_true")
    args = ap.parse_args()
    from skyephyx_b200 import Solver, scenes
    specs = scenes.batch_mix_specs(n_scenes=args.scenes)
    staged = []
    nb = 0
    for sp in specs:
        s = Solver()
        scenes.build_spec(s, sp)
        staged.append(s)
        nb += s.num_bodies
    best, best_ms, results = tune(staged, log=print)
    if args.save:
        table = load_table()
        nfem = sum(1 for sp in specs if sp[0] == "fem")
        table.setdefault(device_name(), {})[signature(len(specs), nfem, nb)] = best
        save_table(table)
        print("saved", TABLE)
