"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the reference's own physics (SkyePhyX src/physics/*.cpp,
src/helpers/{geometry,math}.cpp) compiled unmodified against the Eigen-API shim
in ``oracle/eigen_shim`` and linked with ``oracle/harness.cpp`` (see
``oracle/Makefile``).  ``OracleSolver`` exposes the same scene-building method
names as :class:`skyephyx_b200.Solver`, so one scene generator feeds both.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module.  Parity at the Eigen boundary is unpinned: the
reference publishes no tests or golden vectors, so the shim's LDLT/SVD/eigen
solvers are restated from their documented behaviour.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict = {}

INF = float("inf")


def reference_root(ref_root: str | None = None) -> str | None:
    """The SkyePhyX source tree: the argument, else $SKYEPHYX_REF, else the
    oracle Makefile's default; None when that directory does not exist."""
    ref = ref_root or os.environ.get("SKYEPHYX_REF")
    if not ref:
        out = subprocess.run(["make", "-s", "-C", _HERE, "print-ref"], capture_output=True, text=True)
        ref = out.stdout.strip() if out.returncode == 0 else ""
    return ref if ref and os.path.isdir(ref) else None


def build(ref_root: str | None = None) -> None:
    """Compile oracle/_ref/liboracle{,_fast}.so from the reference sources
    (nothing when the source tree is absent)."""
    ref = reference_root(ref_root)
    if ref is None:
        return
    subprocess.run(["make", "-C", _HERE, f"REF={ref}", "-j2"], check=True, stdout=subprocess.DEVNULL)


def _lib(kind: str = "parity"):
    """The oracle build: "parity" (liboracle.so), "fast" (the timed CPU
    baseline) or "f64" (the parity build carried out in double)."""
    name = {"parity": "liboracle.so", "fast": "liboracle_fast.so", "f64": "liboracle64.so"}[kind]
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(_HERE, "_ref", name)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    real = C.c_double if kind == "f64" else C.c_float   # the build's float
    fp = C.POINTER(real)
    ip = C.POINTER(C.c_int)
    up = C.POINTER(C.c_uint32)
    vp = C.c_void_p
    sig = {
        "orc_create": ([], vp),
        "orc_destroy": ([vp], None),
        "orc_set_params": ([vp, C.c_int, real, real, real, real, real, C.c_int,
                            C.c_int], None),
        "orc_add_box": ([vp, C.c_int, real, real, fp, fp, fp, fp, fp, C.c_int], C.c_int),
        "orc_add_particle": ([vp, real, real, fp, fp, C.c_int], C.c_int),
        "orc_add_bodies": ([vp, C.c_int, C.c_int, fp, fp, fp, fp, fp, fp, fp, ip], C.c_int),
        "orc_set_static": ([vp, C.c_int, C.c_int], C.c_int),
        "orc_add_spring": ([vp, C.c_int, fp, C.c_int, fp, real, real, C.c_int, real], C.c_int),
        "orc_add_joint": ([vp, C.c_int, fp, C.c_int, fp, fp, fp], C.c_int),
        "orc_add_nh_tet": ([vp, ip, real, real], C.c_int),
        "orc_add_stvk_tri": ([vp, ip, real, real], C.c_int),
        "orc_make_tet_volume": ([vp, real, real, real, C.c_int, C.c_int, C.c_int, real,
                                 real, real, real, real, C.c_int], C.c_int),
        "orc_make_stvk_tet_volume": ([vp, real, real, real, C.c_int, C.c_int, C.c_int, real,
                                      real, real, real, real, C.c_int], C.c_int),
        "orc_add_stvk_tet": ([vp, ip, real, real], C.c_int),
        "orc_make_tet_sphere": ([vp, real, real, real, real, real, real, real, real, real], C.c_int),
        "orc_step": ([vp], C.c_int),
        "orc_step_coloured": ([vp, C.c_int], C.c_int),
        "orc_step_many": ([C.POINTER(vp), C.c_int, C.c_int, C.c_int, C.c_int], C.c_double),
        "orc_num_bodies": ([vp], C.c_int),
        "orc_num_dynamic": ([vp], C.c_int),
        "orc_emergency_stop": ([vp], C.c_int),
        "orc_force_live": ([vp, C.c_int], C.c_int),
        "orc_metrics": ([vp, C.POINTER(C.c_double)], None),
        "orc_get_state": ([vp, fp, fp, fp, fp], None),
        "orc_set_state": ([vp, fp, fp, fp, fp], None),
        "orc_get_contacts": ([vp, C.c_int, ip, ip, up, fp], C.c_int),
        "orc_collide": ([vp, C.c_int, C.c_int, up, fp], C.c_int),
        "orc_get_colours": ([vp, ip], C.c_int),
        "orc_get_phase_ms": ([vp, C.POINTER(C.c_double)], None),
        "orc_get_solver_timings": ([vp, fp], None),
    }
    for fn, (args, res) in sig.items():
        f = getattr(lib, fn)
        f.argtypes = args
        f.restype = res
    _LIBS[name] = lib
    return lib


def _f(a, n=None, dtype=np.float32):
    """Scene inputs rounded to float32 (the reference's input type), widened
    for the FP64 build, so both builds start from the same values."""
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1).astype(dtype))
    if n is not None:
        assert arr.size == n, (arr.size, n)
    return arr


def _r(x):
    """A scalar scene input rounded to float32 (widened again by the FP64 build)."""
    return float(np.float32(x))


def _fp(arr):
    ct = C.c_double if arr.dtype == np.float64 else C.c_float
    return arr.ctypes.data_as(C.POINTER(ct))


class OracleSolver:
    """The reference ``Solver`` (solver.hpp:22-94) driven through the harness."""

    def __init__(self, iterations=10, dt=1.0 / 60.0, alpha=0.95, beta=100000.0, gamma=0.99,
                 on_penetration_penalty=0.0, post_stabilization=True, projection_mode=1, fast=False, f64=False):
        """fast: the timed CPU-baseline build; f64: the same code in double
        (state arrays are then float64)."""
        self._kind = "f64" if f64 else ("fast" if fast else "parity")
        self._ft = np.float64 if f64 else np.float32
        self._lib = _lib(self._kind)
        self._h = self._lib.orc_create()
        self._keep = []
        self.set_params(iterations, dt, alpha, beta, gamma, on_penetration_penalty, post_stabilization,
                        projection_mode)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.orc_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def set_params(self, iterations=10, dt=1.0 / 60.0, alpha=0.95, beta=100000.0, gamma=0.99,
                   on_penetration_penalty=0.0, post_stabilization=True, projection_mode=1):
        self._lib.orc_set_params(self._h, int(iterations), _r(dt), _r(alpha), _r(beta), _r(gamma),
                                 _r(on_penetration_penalty), int(bool(post_stabilization)),
                                 int(projection_mode))

    # ---- scene building (same names/semantics as skyephyx_b200.Solver) ----
    def add_body(self, model_type, density, friction, pos, scale, vel=(0, 0, 0), quat=(1, 0, 0, 0),
                 omega=(0, 0, 0), is_static=False):
        ft = self._ft
        p, s, v, q, w = _f(pos, 3, ft), _f(scale, 3, ft), _f(vel, 3, ft), _f(quat, 4, ft), _f(omega, 3, ft)
        return self._lib.orc_add_box(self._h, int(model_type), _r(density), _r(friction), _fp(p), _fp(s),
                                     _fp(v), _fp(q), _fp(w), int(bool(is_static)))

    def add_bodies(self, model_type, density, friction, pos, scale, quat, is_static, vel=None, omega=None):
        def c(a):
            return None if a is None else np.ascontiguousarray(np.asarray(a, np.float32).astype(self._ft).reshape(-1))
        arrs = [c(pos), c(scale), c(quat), c(density), c(friction), c(vel), c(omega)]
        n = arrs[0].size // 3
        st = np.ascontiguousarray(np.asarray(is_static, np.int32).reshape(-1))
        ptr = [None if a is None else _fp(a) for a in arrs]
        return self._lib.orc_add_bodies(self._h, n, int(model_type), ptr[3], ptr[4], ptr[0], ptr[1], ptr[5], ptr[2],
                                        ptr[6], st.ctypes.data_as(C.POINTER(C.c_int)))

    def add_particle(self, mass, friction, pos, vel=(0, 0, 0), is_static=False):
        p, v = _f(pos, 3, self._ft), _f(vel, 3, self._ft)
        return self._lib.orc_add_particle(self._h, _r(mass), _r(friction), _fp(p), _fp(v),
                                          int(bool(is_static)))

    def set_static(self, body, is_static=True):
        return self._lib.orc_set_static(self._h, int(body), int(bool(is_static)))

    def add_spring(self, a, rA, b, rB, stiffness, rest_length=-1.0, is_rope=False, fracture=INF):
        ra, rb = _f(rA, 3, self._ft), _f(rB, 3, self._ft)
        return self._lib.orc_add_spring(self._h, int(a), _fp(ra), int(b), _fp(rb), _r(stiffness),
                                        _r(rest_length), int(bool(is_rope)), _r(fracture))

    def add_joint(self, a, rA, b, rB, stiffness=(INF,) * 6, fracture=(INF,) * 6):
        ft = self._ft
        ra, rb, k, fr = _f(rA, 3, ft), _f(rB, 3, ft), _f(stiffness, 6, ft), _f(fracture, 6, ft)
        return self._lib.orc_add_joint(self._h, int(a), _fp(ra), int(b), _fp(rb), _fp(k), _fp(fr))

    def add_neohookean_tet(self, v, E, nu):
        iv = (C.c_int * 4)(*[int(x) for x in v])
        return self._lib.orc_add_nh_tet(self._h, iv, _r(E), _r(nu))

    def add_stvk_tri(self, v, E, nu):
        iv = (C.c_int * 3)(*[int(x) for x in v])
        return self._lib.orc_add_stvk_tri(self._h, iv, _r(E), _r(nu))

    def add_stvk_tet(self, v, E, nu):
        iv = (C.c_int * 4)(*[int(x) for x in v])
        return self._lib.orc_add_stvk_tet(self._h, iv, _r(E), _r(nu))

    def make_stvk_tet_volume(self, ox, oy, oz, nx, ny, nz, cell, E, nu, particle_mass=1.0, friction=0.5,
                             pin_min_x=False):
        return self._lib.orc_make_stvk_tet_volume(self._h, _r(ox), _r(oy), _r(oz), int(nx), int(ny),
                                                  int(nz), _r(cell), _r(E), _r(nu), _r(particle_mass),
                                                  _r(friction), int(bool(pin_min_x)))

    def make_tet_volume(self, ox, oy, oz, nx, ny, nz, cell, E, nu, particle_mass=1.0, friction=0.5,
                        pin_min_x=False):
        return self._lib.orc_make_tet_volume(self._h, _r(ox), _r(oy), _r(oz), int(nx), int(ny), int(nz),
                                             _r(cell), _r(E), _r(nu), _r(particle_mass),
                                             _r(friction), int(bool(pin_min_x)))

    def make_tet_sphere(self, cx, cy, cz, radius, res, E, nu, particle_mass=1.0, friction=0.5):
        return self._lib.orc_make_tet_sphere(self._h, _r(cx), _r(cy), _r(cz), _r(radius), _r(res), _r(E), _r(nu),
                                             _r(particle_mass), _r(friction))

    # ---- stepping ----
    def step(self):
        """The reference Solver::Step() as written (sequential Gauss-Seidel)."""
        return self._lib.orc_step(self._h)

    def step_coloured(self, identity_order=False):
        """Restated Step() with colour-ordered primal sweeps (the parity oracle)."""
        return self._lib.orc_step_coloured(self._h, int(bool(identity_order)))

    # ---- readback ----
    @property
    def num_bodies(self):
        return self._lib.orc_num_bodies(self._h)

    @property
    def num_dynamic(self):
        return self._lib.orc_num_dynamic(self._h)

    @property
    def emergency_stop(self):
        return bool(self._lib.orc_emergency_stop(self._h))

    def metrics(self) -> dict:
        """Long-horizon measures of the current state (orc_metrics): max |C|
        over hard joint rows, deepest penetration, kinetic, gravitational and
        elastic energy, non-finite dynamic bodies."""
        out = (C.c_double * 6)()
        self._lib.orc_metrics(self._h, out)
        keys = ("max_violation", "max_penetration_m", "kinetic_j", "potential_j", "elastic_j", "nonfinite")
        m = dict(zip(keys, list(out)))
        m["energy_j"] = m["kinetic_j"] + m["potential_j"] + m["elastic_j"]
        return m

    def force_live(self, force):
        """False once a fracture disabled the force or the solver dropped it."""
        return self._lib.orc_force_live(self._h, int(force)) == 1

    def get_state(self):
        n = self.num_bodies
        pos = np.zeros((n, 3), self._ft)
        quat = np.zeros((n, 4), self._ft)
        vel = np.zeros((n, 3), self._ft)
        omega = np.zeros((n, 3), self._ft)
        self._lib.orc_get_state(self._h, _fp(pos), _fp(quat), _fp(vel), _fp(omega))
        return pos, quat, vel, omega

    def set_state(self, pos=None, quat=None, vel=None, omega=None):
        n = self.num_bodies
        arrs = [None if a is None else _f(a, n * k, self._ft) for a, k in ((pos, 3), (quat, 4), (vel, 3), (omega, 3))]
        ptrs = [None if a is None else _fp(a) for a in arrs]
        self._lib.orc_set_state(self._h, *ptrs)

    def contacts(self):
        """Live manifolds: dict (A, B) -> (ids[list], data[n,16])."""
        n = self._lib.orc_get_contacts(self._h, 0, None, None, None, None)
        pairs = np.zeros((max(n, 1), 2), np.int32)
        counts = np.zeros(max(n, 1), np.int32)
        ids = np.zeros((max(n, 1), 8), np.uint32)
        data = np.zeros((max(n, 1), 8, 16), self._ft)
        self._lib.orc_get_contacts(self._h, n, pairs.ctypes.data_as(C.POINTER(C.c_int)),
                                   counts.ctypes.data_as(C.POINTER(C.c_int)),
                                   ids.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(data))
        out = {}
        for m in range(n):
            a, b = int(pairs[m, 0]), int(pairs[m, 1])
            k = int(counts[m])
            out[(a, b)] = ([int(x) for x in ids[m, :k]], data[m, :k].copy())
        return out

    def collide(self, a, b):
        ids = np.zeros(8, np.uint32)
        data = np.zeros((8, 13), self._ft)
        n = self._lib.orc_collide(self._h, int(a), int(b), ids.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(data))
        return [int(x) for x in ids[:n]], data[:n].copy()

    def colours(self):
        n = self.num_bodies
        c = np.zeros(n, np.int32)
        k = self._lib.orc_get_colours(self._h, c.ctypes.data_as(C.POINTER(C.c_int)))
        return c, k

    def phase_ms(self):
        out = (C.c_double * 8)()
        self._lib.orc_get_phase_ms(self._h, out)
        return list(out)

    def solver_timings(self):
        out = np.zeros(7, self._ft)
        self._lib.orc_get_solver_timings(self._h, _fp(out))
        return out


def step_many(solvers, steps, threads, coloured=False, fast=None):
    """Steps independent oracle solvers on `threads` host threads; returns ms.
    The solvers' own build (parity or fast) runs them; `fast` is ignored."""
    if not solvers:
        return 0.0
    lib = solvers[0]._lib
    arr = (C.c_void_p * len(solvers))(*[s.handle for s in solvers])
    return lib.orc_step_many(arr, len(solvers), int(steps), int(threads), int(bool(coloured)))
