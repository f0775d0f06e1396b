"""Builds the in-tree CUDA library ``skyephyx_b200/libavbd.so`` for sm_100a.

    python -m skyephyx_b200.build          # or skyephyx_b200.build.build()
    python -m skyephyx_b200.build --checks # debug build libavbd_checks.so (AVBD_CHECKS)

nvcc compiles device code for ``sm_100a`` only (no PTX for other targets).
Host code is compiled with ``-ffp-contract=off`` so the scene staging rounds
exactly like the reference's constructors.  The translation units (the host
side, and one per build of the batched persistent kernel) compile in
parallel.  The debug build (checks=True, -DAVBD_CHECKS) adds device index
checks that record the first violation in a check word instead of trapping
(avbd_check_word); the loader takes it when AVBD_CHECKS=1 is set.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libavbd.so")
LIB_CHECKS = os.path.join(HERE, "libavbd_checks.so")
# (object name, source, extra flags)
UNITS = [("avbd_api", "avbd_api.cu", []), ("avbd_batch_host", "avbd_batch_host.cu", []),
         ("avbd_server", "avbd_server.cu", []), ("avbd_scene_snapshot", "avbd_scene_snapshot.cu", []),
         ("avbd_host", "avbd_host.cpp", [])] + [
    (f"avbd_batch_v{i}", "avbd_batch_v.cu", [f"-DAVBD_BATCH_ID={i}"]) for i in range(1, 8)]
SOURCES = sorted({u[1] for u in UNITS})
HEADERS = ["avbd_common.cuh", "avbd_narrow.cuh", "avbd_fem.cuh", "avbd_phases.cuh", "avbd_step.cuh", "avbd_host.h",
           "avbd_batch.h", "avbd_pools.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-Xptxas", "-warn-spills", "-Xfatbin=-compress-all",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "avbd.h"))
    deps.append(__file__)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, csrc: str = CSRC, lib: str = None, checks: bool = False) -> str:
    """Compiles libavbd.so (libavbd_checks.so with checks=True) if any source
    is newer than it; returns its path."""
    lib = lib or (LIB_CHECKS if checks else LIB)
    if not force and lib in (LIB, LIB_CHECKS) and not _stale(lib):
        return lib
    flags = ["-DAVBD_CHECKS"] if checks else []
    tag = "_checks" if checks else ""

    def compile_unit(unit):
        name, src, extra = unit
        obj = os.path.join(csrc, name + tag + ".o")
        cmd = [_nvcc(), *NVCC_FLAGS, *flags, *extra, "-c", os.path.join(csrc, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return obj, r

    jobs = max(1, min(len(UNITS), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(compile_unit, UNITS))
    objs = []
    failed = None
    for obj, r in results:
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode and failed is None:
            failed = r
        objs.append(obj)
    if failed is not None:
        for o in objs:
            if os.path.exists(o):
                os.remove(o)
        raise subprocess.CalledProcessError(failed.returncode, failed.args, failed.stdout, failed.stderr)
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", lib, "-lcudart"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checks="--checks" in sys.argv))
