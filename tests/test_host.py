"""Host-side checks that need no GPU: the C-ABI library exports every
declared symbol, the scene generators build the stated workloads, and the
multi-rank timing logic of bench.py (gloo, world size 2)."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "avbd.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(avbd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from skyephyx_b200 import _lib
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), n
    declared_py = {n for n, _, _ in _lib.SIGNATURES}
    assert set(names) <= declared_py | {"avbd_collide_noalloc"}


def test_default_params_match_reference():
    from skyephyx_b200 import _lib
    p = _lib.default_params()
    # solver.hpp:69-84
    assert p.num_iterations == 10 and abs(p.step_value - 1 / 60) < 1e-9
    assert abs(p.alpha - 0.95) < 1e-7 and p.beta == 100000.0 and abs(p.gamma - 0.99) < 1e-7
    assert p.post_stabilization == 1 and p.projection_mode == 1 and p.on_penetration_penalty == 0.0


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from skyephyx_b200 import AvbdError, Solver
    with pytest.raises(AvbdError):
        Solver()


class Recorder:
    """Counts the scene calls a generator makes."""

    def __init__(self):
        self.bodies = []
        self.static = []
        self.joints = self.springs = self.tets = self.tris = 0

    def add_body(self, model, density, friction, pos, scale, vel=(0, 0, 0), quat=(1, 0, 0, 0), omega=(0, 0, 0),
                 is_static=False):
        self.bodies.append(np.asarray(pos, np.float32))
        self.static.append(bool(is_static))
        return len(self.bodies) - 1

    def add_bodies(self, model, density, friction, pos, scale, quat, is_static, vel=None, omega=None):
        first = len(self.bodies)
        for p, st in zip(np.asarray(pos).reshape(-1, 3), np.asarray(is_static).reshape(-1)):
            self.bodies.append(p)
            self.static.append(bool(st))
        return first

    def add_particle(self, mass, friction, pos, vel=(0, 0, 0), is_static=False):
        return self.add_body(0, 1, friction, pos, (0.1, 0.1, 0.1), is_static=is_static)

    def set_static(self, b, s=True):
        self.static[b] = s

    def add_joint(self, *a, **k):
        self.joints += 1
        return self.joints - 1

    def add_spring(self, *a, **k):
        self.springs += 1
        return self.springs - 1

    def add_neohookean_tet(self, v, E, nu):
        self.tets += 1

    def add_stvk_tri(self, v, E, nu):
        self.tris += 1

    def make_tet_volume(self, ox, oy, oz, nx, ny, nz, cell, E, nu, pm=1.0, fr=0.5, pin=False):
        first = len(self.bodies)
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    self.add_particle(pm, fr, (ox + i * cell, oy + j * cell, oz + k * cell), is_static=pin and i == 0)
        self.tets += 5 * (nx - 1) * (ny - 1) * (nz - 1)
        return first


def test_workload_sizes():
    from skyephyx_b200 import scenes
    r = Recorder()
    scenes.pyramid_wall(r)
    assert len(r.bodies) == 211 and sum(r.static) == 1
    r = Recorder()
    scenes.fem_block(r)
    assert len(r.bodies) == 4961 and r.tets == 20000 and sum(r.static) == 121
    r = Recorder()
    scenes.mixed_large(r)
    assert len(r.bodies) == 32768 + 64 * 32 + 5 and r.joints == 2048 and r.springs == 2048
    assert np.abs(np.stack(r.bodies)).max() < 50.0          # inside the reference's +-50 m bounds
    specs = scenes.batch_mix_specs()
    assert len(specs) == 4096
    fem = [s for s in specs if s[0] == "fem"]
    assert 0.2 < len(fem) / 4096 < 0.3
    assert all(500 <= s[1] <= 5000 for s in fem)
    assert all(8 <= s[1] <= 2048 for s in specs if s[0] != "fem")


def test_generators_are_deterministic():
    from skyephyx_b200 import scenes
    a, b = Recorder(), Recorder()
    scenes.build_spec(a, ("pile", 300, 17))
    scenes.build_spec(b, ("pile", 300, 17))
    assert np.array_equal(np.stack(a.bodies), np.stack(b.bodies))


def test_rank_specs_are_disjoint_and_equal_size():
    sys.path.insert(0, ROOT)
    import bench
    s0 = bench.rank_specs(64, 0, 2)
    s1 = bench.rank_specs(64, 1, 2)
    assert len(s0) == len(s1) == 64
    assert not ({x[2] for x in s0} & {x[2] for x in s1})


_WORKER = r"""
import os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank=int(sys.argv[1]), world_size=2)
r = dist.get_rank()
m = bench._max_over_ranks(dist, 10.0 + r)
print("MAX", r, m, flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def test_max_over_ranks_gloo(tmp_path):
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    script = tmp_path / "w.py"
    script.write_text(_WORKER.format(root=ROOT, port=port))
    procs = [subprocess.Popen([sys.executable, str(script), str(r)], stdout=subprocess.PIPE, text=True)
             for r in range(2)]
    outs = [p.communicate(timeout=120)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs)
    vals = [float(line.split()[2]) for o in outs for line in o.splitlines() if line.startswith("MAX")]
    assert vals == [11.0, 11.0]


def test_cpp_facade_compiles_and_links(tmp_path):
    """include/avbd.hpp (the C++ facade with the reference Solver's method
    names) compiles against include/avbd.h and links against the library."""
    import shutil
    import subprocess
    from skyephyx_b200 import build
    lib = build.build()
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = tmp_path / "facade_scene"
    cmd = [gxx, "-std=c++17", "-O1", "-I", os.path.join(root, "include"), os.path.join(root, "tests", "cpp", "facade_scene.cpp"),
           "-L", os.path.dirname(lib), "-lavbd", "-Wl,-rpath," + os.path.dirname(lib), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_staging_sinks(tmp_path):
    """The scene staging sinks on the host: a pose staged once for the three
    arrays that start equal to it (one host buffer plus two device-side
    copies, or one arena copy scattered three times), zero data left to the
    freshly zeroed pools, and writes past a pool array refused."""
    import shutil
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc) and not shutil.which(nvcc):
        pytest.skip("no nvcc")
    out = tmp_path / "staging_sinks"
    cmd = [nvcc, "-std=c++17", "-O1", "-Wno-deprecated-gpu-targets", "-I", os.path.join(ROOT, "skyephyx_b200", "csrc"),
           "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "staging_sinks.cu"), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "OK", r.stdout + r.stderr
