"""Python mirror of the reference ``Solver`` API over the CUDA C-ABI.

``Solver`` keeps the method names and argument meaning of SkyePhyX's
``Solver`` (src/physics/solver.hpp:22-94) and of the Force/Energy
constructors it is given (``Spring``, ``Joint``, ``NeoHookeanFEM``,
``STVKFEM``); ``step()`` replaces ``Solver::Step()``.  ``Batch`` advances
many independent scenes per persistent-kernel launch.  Every step runs on
the GPU; without a CUDA device the constructors raise ``AvbdError``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import AvbdError, AvbdParams, AvbdTimings, STATUS, check, default_params, load

INF = float("inf")
GROUP_FLAT = 64   # AVBD_GROUP_FLAT: one lane per (particle, tet) term in FEM scenes


_FLOAT_ARRAYS = {n: C.c_float * n for n in (3, 4, 6)}


class _Floats:
    """A small float32 argument: a ctypes array (tuples) or a numpy buffer."""
    __slots__ = ("buf", "size")

    def __init__(self, buf, size):
        self.buf = buf
        self.size = size


def _f(a, n):
    if isinstance(a, (tuple, list)) and len(a) == n and n in _FLOAT_ARRAYS:
        return _Floats(_FLOAT_ARRAYS[n](*a), n)
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1))
    if arr.size != n:
        raise ValueError(f"expected {n} floats, got {arr.size}")
    return arr


def _bulk(pos, scale, quat, density, friction, vel=None, omega=None):
    """Contiguous float32 buffers for a bulk body insert."""
    c = lambda a: None if a is None else np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1))
    return [c(pos), c(scale), c(quat), c(density), c(friction), c(vel), c(omega)]


def _fp(a):
    if isinstance(a, _Floats):
        return C.cast(a.buf, C.POINTER(C.c_float))
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Solver:
    """One scene (the reference's Solver) stepped on one GPU."""

    def __init__(self, iterations=10, dt=1.0 / 60.0, alpha=0.95, beta=100000.0, gamma=0.99,
                 on_penetration_penalty=0.0, post_stabilization=True, projection_mode=1, device=0):
        self._lib = load()
        self._p = default_params(num_iterations=int(iterations), step_value=float(dt), alpha=float(alpha),
                                 beta=float(beta), gamma=float(gamma),
                                 on_penetration_penalty=float(on_penetration_penalty),
                                 post_stabilization=int(bool(post_stabilization)),
                                 projection_mode=int(projection_mode))
        h = C.c_void_p()
        check(self._lib.avbd_world_create(C.byref(self._p), int(device), C.byref(h)), "avbd_world_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.avbd_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ---- parameters (solver.hpp:69-84) ----
    def set_params(self, **kw):
        for k, v in kw.items():
            setattr(self._p, k, v)
        check(self._lib.avbd_set_params(self._h, C.byref(self._p)), "avbd_set_params")

    @property
    def params(self) -> AvbdParams:
        return self._p

    # ---- scene building ----
    def add_body(self, model_type, density, friction, pos, scale, vel=(0, 0, 0), quat=(1, 0, 0, 0),
                 omega=(0, 0, 0), is_static=False):
        """Solver::AddBody (solver.cpp:50-101); quat is (w, x, y, z). Returns the body id."""
        p, s, v, q, w = _f(pos, 3), _f(scale, 3), _f(vel, 3), _f(quat, 4), _f(omega, 3)
        return check(self._lib.avbd_add_body(self._h, int(model_type), float(density), float(friction), _fp(p),
                                             _fp(s), _fp(v), _fp(q), _fp(w), int(bool(is_static))), "add_body")

    def add_bodies(self, model_type, density, friction, pos, scale, quat, is_static, vel=None, omega=None):
        """n x Solver::AddBody from arrays (pos/scale/vel/omega [n,3], quat [n,4] w x y z,
        density/friction/is_static [n]). Returns the first body id."""
        arrs = _bulk(pos, scale, quat, density, friction, vel, omega)
        n = arrs[0].shape[0] // 3
        st = np.ascontiguousarray(np.asarray(is_static, np.int32).reshape(-1))
        ptr = [None if a is None else _fp(a) for a in arrs]
        return check(self._lib.avbd_add_bodies(self._h, n, int(model_type), ptr[3], ptr[4], ptr[0], ptr[1], ptr[5],
                                               ptr[2], ptr[6], st.ctypes.data_as(C.POINTER(C.c_int32))),
                     "add_bodies")

    def add_particle(self, mass, friction, pos, vel=(0, 0, 0), is_static=False):
        """Solver::AddParticle (solver.cpp:119-131)."""
        p, v = _f(pos, 3), _f(vel, 3)
        return check(self._lib.avbd_add_particle(self._h, float(mass), float(friction), _fp(p), _fp(v),
                                                 int(bool(is_static))), "add_particle")

    def set_static(self, body, is_static=True):
        return check(self._lib.avbd_set_body_static(self._h, int(body), int(bool(is_static))), "set_static")

    def add_spring(self, a, rA, b, rB, stiffness, rest_length=-1.0, is_rope=False, fracture=INF):
        """Spring (force.hpp:95); a = -1 anchors rA in world space. Returns the force id."""
        ra, rb = _f(rA, 3), _f(rB, 3)
        return check(self._lib.avbd_add_spring(self._h, int(a), _fp(ra), int(b), _fp(rb), float(stiffness),
                                               float(rest_length), int(bool(is_rope)), float(fracture)),
                     "add_spring")

    def add_joint(self, a, rA, b, rB, stiffness=(INF,) * 6, fracture=(INF,) * 6):
        """Joint (force.hpp:119-122). Returns the force id."""
        ra, rb, k, fr = _f(rA, 3), _f(rB, 3), _f(stiffness, 6), _f(fracture, 6)
        return check(self._lib.avbd_add_joint(self._h, int(a), _fp(ra), int(b), _fp(rb), _fp(k), _fp(fr)),
                     "add_joint")

    def add_neohookean_tet(self, v, E, nu):
        """NeoHookeanFEM (energy.hpp:50-52). Returns the energy id."""
        iv = (C.c_int32 * 4)(*[int(x) for x in v])
        return check(self._lib.avbd_add_neohookean_tet(self._h, iv, float(E), float(nu)), "add_neohookean_tet")

    def add_stvk_tri(self, v, E, nu):
        """STVKFEM (energy.hpp:90-92). Returns the energy id."""
        iv = (C.c_int32 * 3)(*[int(x) for x in v])
        return check(self._lib.avbd_add_stvk_tri(self._h, iv, float(E), float(nu)), "add_stvk_tri")

    def add_stvk_tet(self, v, E, nu):
        """St. Venant-Kirchhoff tet (no reference counterpart). Returns the tet id."""
        iv = (C.c_int32 * 4)(*[int(x) for x in v])
        return check(self._lib.avbd_add_stvk_tet(self._h, iv, float(E), float(nu)), "add_stvk_tet")

    def make_stvk_tet_volume(self, ox, oy, oz, nx, ny, nz, cell, E, nu, particle_mass=1.0, friction=0.5,
                             pin_min_x=False):
        """makeTetVolume's particles and tets with StVK tets. Returns the first particle id."""
        return check(self._lib.avbd_make_stvk_tet_volume(self._h, float(ox), float(oy), float(oz), int(nx), int(ny),
                                                         int(nz), float(cell), float(E), float(nu),
                                                         float(particle_mass), float(friction), int(bool(pin_min_x))),
                     "make_stvk_tet_volume")

    def make_tet_volume(self, ox, oy, oz, nx, ny, nz, cell, E, nu, particle_mass=1.0, friction=0.5,
                        pin_min_x=False):
        """GeometryHelpers::makeTetVolume (geometry.cpp:30-94). Returns the first particle id."""
        return check(self._lib.avbd_make_tet_volume(self._h, float(ox), float(oy), float(oz), int(nx), int(ny),
                                                    int(nz), float(cell), float(E), float(nu),
                                                    float(particle_mass), float(friction), int(bool(pin_min_x))),
                     "make_tet_volume")

    def set_color(self, body, rgb):
        """Mesh::color of a body (read only by the instance export)."""
        c = _f(rgb, 3)
        check(self._lib.avbd_set_body_color(self._h, int(body), _fp(c)), "set_body_color")

    def export_instances(self, dst=None):
        """Headless pose export in the renderer's 128-byte instance layout
        (RenderEngine.cpp:951-1000).  dst: a device pointer (int) of room for
        num_bodies records, or None for a host array of shape (n, 32) float32
        (model matrix 16, normal matrix 12, colour 4).  Returns (array or
        count, first index per model, count per model)."""
        n = self.num_bodies
        first = (C.c_int32 * 3)()
        count = (C.c_int32 * 3)()
        if dst is None:
            out = np.zeros((n, 32), np.float32)
            k = check(self._lib.avbd_export_instances(self._h, out.ctypes.data, n, first, count), "export_instances")
            return out[:k], list(first), list(count)
        k = check(self._lib.avbd_export_instances(self._h, C.c_void_p(int(dst)), n, first, count),
                  "export_instances")
        return k, list(first), list(count)

    def make_tet_sphere(self, cx, cy, cz, radius, res, E, nu, particle_mass=1.0, friction=0.5):
        """GeometryHelpers::makeTetSphere (geometry.cpp:106-232). Returns the first particle id."""
        return check(self._lib.avbd_make_tet_sphere(self._h, float(cx), float(cy), float(cz), float(radius),
                                                    float(res), float(E), float(nu), float(particle_mass),
                                                    float(friction)), "make_tet_sphere")

    # ---- stepping ----
    def step(self):
        """Solver::Step(); returns the status name ('ok', 'exploded', ...)."""
        r = check(self._lib.avbd_step(self._h), "avbd_step")
        return STATUS.get(r, str(r))

    def step_dt(self, dt, iterations):
        r = check(self._lib.avbd_step_dt(self._h, float(dt), int(iterations)), "avbd_step_dt")
        self._p.step_value = float(dt)
        self._p.num_iterations = int(iterations)
        return STATUS.get(r, str(r))

    # ---- readback ----
    @property
    def num_bodies(self):
        return self._lib.avbd_num_bodies(self._h)

    @property
    def num_dynamic(self):
        return self._lib.avbd_num_dynamic_bodies(self._h)

    @property
    def emergency_stop(self):
        return bool(self._lib.avbd_emergency_stop(self._h))

    def force_live(self, force: int) -> bool:
        """False once a fracture disabled the joint/spring or it left with a body."""
        return bool(check(self._lib.avbd_force_live(self._h, int(force)), "force_live"))

    def get_state(self):
        n = self.num_bodies
        pos = np.zeros((n, 3), np.float32)
        quat = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 3), np.float32)
        omega = np.zeros((n, 3), np.float32)
        check(self._lib.avbd_get_state(self._h, _fp(pos), _fp(quat), _fp(vel), _fp(omega)), "get_state")
        return pos, quat, vel, omega

    def set_state(self, pos=None, quat=None, vel=None, omega=None):
        n = self.num_bodies
        arrs = [None if a is None else _f(a, n * k) for a, k in ((pos, 3), (quat, 4), (vel, 3), (omega, 3))]
        check(self._lib.avbd_set_state(self._h, *[None if a is None else _fp(a) for a in arrs]), "set_state")

    def contacts(self):
        """Live manifolds: {(A, B): (ids, data[n, 16])}, data as the oracle reports it."""
        n = check(self._lib.avbd_get_contacts(self._h, 0, None, None, None, None), "get_contacts")
        m = max(n, 1)
        pairs = np.zeros((m, 2), np.int32)
        counts = np.zeros(m, np.int32)
        ids = np.zeros((m, 8), np.uint32)
        data = np.zeros((m, 8, 16), np.float32)
        check(self._lib.avbd_get_contacts(self._h, n, pairs.ctypes.data_as(C.POINTER(C.c_int32)),
                                          counts.ctypes.data_as(C.POINTER(C.c_int32)),
                                          ids.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(data)), "get_contacts")
        return {(int(pairs[k, 0]), int(pairs[k, 1])): ([int(x) for x in ids[k, :counts[k]]], data[k, :counts[k]].copy())
                for k in range(n)}

    def colours(self):
        c = np.zeros(self.num_bodies, np.int32)
        k = check(self._lib.avbd_get_colours(self._h, c.ctypes.data_as(C.POINTER(C.c_int32))), "get_colours")
        return c, k

    def timings(self) -> dict:
        t = AvbdTimings()
        check(self._lib.avbd_get_timings(self._h, C.byref(t)), "get_timings")
        return {name: getattr(t, name) for name, _ in AvbdTimings._fields_}

    def collide(self, a, b):
        """CollisionSpace::CollisionBoxBox on the device for bodies a, b as they stand."""
        ids = np.zeros(8, np.uint32)
        data = np.zeros((8, 13), np.float32)
        n = check(self._lib.avbd_collide(self._h, int(a), int(b), ids.ctypes.data_as(C.POINTER(C.c_uint32)),
                                         _fp(data)), "collide")
        return [int(x) for x in ids[:n]], data[:n].copy()

    def collide_noalloc(self, body_a, body_b):
        """avbd_collide over many pairs without any device allocation (fixed
        device scratch). Returns (ids[n, 8], data[n, 8, 13], counts[n])."""
        a = np.ascontiguousarray(np.asarray(body_a, np.int32))
        b = np.ascontiguousarray(np.asarray(body_b, np.int32))
        n = a.size
        ids = np.zeros((n, 8), np.uint32)
        data = np.zeros((n, 8, 13), np.float32)
        counts = np.zeros(n, np.int32)
        ip = C.POINTER(C.c_int32)
        check(self._lib.avbd_collide_noalloc(self._h, n, a.ctypes.data_as(ip), b.ctypes.data_as(ip),
                                             ids.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(data),
                                             counts.ctypes.data_as(ip)), "collide_noalloc")
        return ids, data, counts

    def snapshot(self) -> np.ndarray:
        """Device state of a stepped world as a host byte array (see avbd_snapshot)."""
        n = check(self._lib.avbd_snapshot_bytes(self._h), "snapshot_bytes")
        buf = np.empty(n, np.uint8)
        check(self._lib.avbd_snapshot(self._h, buf.ctypes.data, n), "snapshot")
        return buf

    def restore(self, buf: np.ndarray):
        """Puts back a snapshot taken from this world (or one built the same way)."""
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        check(self._lib.avbd_restore(self._h, buf.ctypes.data, buf.size), "restore")

    def remove_body(self, body: int):
        """Solver::RemoveBody: the body and its forces and energies stop taking part (ids stay stable)."""
        check(self._lib.avbd_remove_body(self._h, int(body)), "remove_body")

    def remove_force(self, force: int):
        """Solver::RemoveForce for a joint or spring id."""
        check(self._lib.avbd_remove_force(self._h, int(force)), "remove_force")

    def remove_energy(self, energy: int, kind: str = "tet"):
        """Solver::RemoveEnergy for a Neo-Hookean tet ("tet") or StVK triangle ("tri") id."""
        fn = self._lib.avbd_remove_neohookean_tet if kind == "tet" else self._lib.avbd_remove_stvk_tri
        check(fn(self._h, int(energy)), "remove_energy")

    def set_group(self, group=0):
        """Lanes per body in the primal sweep (0 = by scene kind); before the first step."""
        check(self._lib.avbd_set_group(self._h, int(group)), "set_group")

    def footprint_bytes(self):
        return self._lib.avbd_scene_footprint_bytes(self._h)


class Batch:
    """Many independent scenes advanced by one persistent kernel per step."""

    def __init__(self, iterations=10, dt=1.0 / 60.0, device=0, **kw):
        self._lib = load()
        self._p = default_params(num_iterations=int(iterations), step_value=float(dt))
        for k, v in kw.items():
            setattr(self._p, k, v)
        h = C.c_void_p()
        check(self._lib.avbd_batch_create(C.byref(self._p), int(device), C.byref(h)), "avbd_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.avbd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, bodies, forces, tets, tris, scenes):
        """Allocates the device pools (bodies, joints+springs, tets, triangles, scene slots)."""
        check(self._lib.avbd_batch_reserve(self._h, int(bodies), int(forces), int(tets), int(tris), int(scenes)),
              "batch_reserve")

    def add_scene(self, solver: Solver) -> int:
        """Copies a staged (never stepped) Solver scene into the batch; returns its scene id."""
        return check(self._lib.avbd_batch_add_scene(self._h, solver.handle), "batch_add_scene")

    def try_add_scene(self, solver: Solver):
        """Like add_scene, but returns None when the scene does not fit in the free pool space."""
        r = self._lib.avbd_batch_add_scene(self._h, solver.handle)
        if r == -3:   # AVBD_ERR_NOMEM
            return None
        return check(r, "batch_add_scene")

    def body_offset(self, scene: int) -> int:
        return check(self._lib.avbd_batch_scene_body_offset(self._h, int(scene)), "scene_body_offset")

    def remove_scene(self, scene: int):
        check(self._lib.avbd_batch_remove_scene(self._h, int(scene)), "batch_remove_scene")

    def prepare(self):
        """Allocates the pools for the scenes added so far and stages them in
        page-locked host memory; the next step() copies them to the device.
        Optional (the first step() does it otherwise)."""
        check(self._lib.avbd_batch_prepare(self._h), "batch_prepare")

    @property
    def uploaded_bytes(self) -> int:
        """Host-to-device bytes the last upload of staged scenes copied."""
        return int(self._lib.avbd_batch_uploaded_bytes(self._h))

    def step(self, steps: int = 1) -> str:
        r = check(self._lib.avbd_batch_step(self._h, int(steps)), "batch_step")
        return STATUS.get(r, str(r))

    @property
    def num_scenes(self):
        return self._lib.avbd_batch_num_scenes(self._h)

    @property
    def dynamic_bodies(self) -> int:
        return int(self._lib.avbd_batch_dynamic_bodies(self._h))

    def scene_status(self, scene: int) -> str:
        r = check(self._lib.avbd_batch_scene_status(self._h, int(scene)), "scene_status")
        return STATUS.get(r, str(r))

    def scene_info(self, scene: int) -> dict:
        out = (C.c_int32 * 6)()
        check(self._lib.avbd_batch_scene_info(self._h, int(scene), out), "scene_info")
        keys = ("status", "colours", "candidates", "contacts", "incidence", "steps")
        return dict(zip(keys, list(out)))

    def get_state(self, scene: int):
        n = check(self._lib.avbd_batch_scene_bodies(self._h, int(scene)), "scene_bodies")
        pos = np.zeros((n, 3), np.float32)
        quat = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 3), np.float32)
        omega = np.zeros((n, 3), np.float32)
        check(self._lib.avbd_batch_get_state(self._h, int(scene), _fp(pos), _fp(quat), _fp(vel), _fp(omega)),
              "batch_get_state")
        return pos, quat, vel, omega

    def snapshot_scene(self, scene: int) -> np.ndarray:
        """Device state of one live scene as a host byte array (avbd_batch_scene_snapshot)."""
        n = check(self._lib.avbd_batch_scene_snapshot_bytes(self._h, int(scene)), "scene_snapshot_bytes")
        buf = np.empty(n, np.uint8)
        check(self._lib.avbd_batch_scene_snapshot(self._h, int(scene), buf.ctypes.data, n), "scene_snapshot")
        return buf

    def restore_scene(self, buf: np.ndarray) -> int:
        """Admits a scene snapshot wherever it fits; returns its new scene id."""
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        return check(self._lib.avbd_batch_scene_restore(self._h, buf.ctypes.data, buf.size), "scene_restore")

    def set_groups(self, rigid_group=4, fem_group=8):
        """Lanes per body in the primal sweep for rigid and FEM scenes (before the
        first step); fem_group may be GROUP_FLAT (one lane per particle-tet term)."""
        check(self._lib.avbd_batch_set_groups(self._h, int(rigid_group), int(fem_group)), "set_groups")

    def set_launch(self, threads_per_cta=0, ctas_per_sm=0):
        check(self._lib.avbd_batch_set_launch(self._h, int(threads_per_cta), int(ctas_per_sm)), "set_launch")

    def set_team_work(self, units_per_lane=0):
        """Scenes with at most this many (bodies + tets) per lane of half a team
        share a CTA with others (0: one scene per CTA); before stepping."""
        check(self._lib.avbd_batch_set_team_work(self._h, int(units_per_lane)), "set_team_work")

    def set_fem_team_work(self, units_per_lane=0):
        """The team split threshold for scenes with tets (0: one scene per CTA)."""
        check(self._lib.avbd_batch_set_fem_team_work(self._h, int(units_per_lane)), "set_fem_team_work")

    def set_grid_broadphase(self, min_bodies=128):
        """Scenes of at least min_bodies use the grid broadphase (0: all-pairs)."""
        check(self._lib.avbd_batch_set_grid_broadphase(self._h, int(min_bodies)), "set_grid_broadphase")

    def set_cluster(self, cluster_size=1, min_units=0):
        """Scenes of at least min_units bodies + tets run on a whole thread-block
        cluster of cluster_size CTAs (1 = off); before stepping."""
        check(self._lib.avbd_batch_set_cluster(self._h, int(cluster_size), int(min_units)), "set_cluster")

    def set_queue_weight(self, body_weight=1):
        """Queue order key: body_weight x bodies + tets, largest first."""
        check(self._lib.avbd_batch_set_queue_weight(self._h, int(body_weight)), "set_queue_weight")

    def set_scene_timing(self, on=True):
        """Per-scene device timing of each step (global timer stamps at the
        start and end of every scene's step)."""
        check(self._lib.avbd_batch_set_scene_timing(self._h, 1 if on else 0), "set_scene_timing")

    SCENE_STAMPS = 9   # AVBD_SCENE_STAMPS

    def scene_times(self):
        """(slots, 9) int64 array of global-timer ns through each slot's last
        step: start, after broadphase, narrowphase, warm start + incidence,
        colouring, prediction, iterations, velocities, end (0 for slots not
        stepped since timing was switched on)."""
        n = check(self._lib.avbd_batch_scene_times(self._h, None, 0), "scene_times")
        out = np.zeros((max(n, 1), self.SCENE_STAMPS), np.int64)
        k = check(self._lib.avbd_batch_scene_times(self._h, out.ctypes.data_as(C.POINTER(C.c_int64)), n),
                  "scene_times")
        return out[:k]

    def set_kernel(self, register_variant=1):
        """Build of the persistent kernel: 1..4 for CTAs of up to 256 threads
        (156, 128, 80 or 64 registers), 5/6 for 512 threads, 7 for 1024."""
        check(self._lib.avbd_batch_set_kernel(self._h, int(register_variant)), "set_kernel")

    def launch(self):
        t = C.c_int32()
        c = C.c_int32()
        check(self._lib.avbd_batch_get_launch(self._h, C.byref(t), C.byref(c)), "get_launch")
        return t.value, c.value

    @property
    def last_ms(self) -> float:
        return float(self._lib.avbd_batch_last_ms(self._h))


__all__ = ["Solver", "Batch", "AvbdError", "INF"]
