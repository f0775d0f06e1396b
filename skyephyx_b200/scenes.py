"""Seeded scene builders: the workloads and the reference's demo scenes.

Every builder takes a *solver-like* object exposing the reference's scene API
(``add_body``, ``add_particle``, ``add_spring``, ``add_joint``,
``add_neohookean_tet``, ``add_stvk_tri``, ``make_tet_volume``, ``set_static``)
and issues the same calls, in the same order, with the same float32 values,
whichever solver it is given.  Positions are rounded to float32 here, once, so
every consumer receives bit-identical inputs.

Workloads (sizes as stated in each docstring) are synthetic and seeded:
splitmix64-seeded numpy PCG64 streams, seed ``0x5EED0000 + config*1000 + scene``.
The demo scenes re-express SkyePhyX ``src/levels.h`` through this API.
"""
from __future__ import annotations

import math

import numpy as np

INF = float("inf")
CUBE = 0          # ModelType_Cube (geometry.hpp:17-22)
SPHERE = 1        # ModelType_Sphere (collides as a box, collision.hpp:28-31)
HINGE = (INF, INF, INF, INF, 0.0, 0.0)   # levels.h:207 hinge stiffness pattern


def f32(x):
    return np.float32(x)


def v3(x, y, z):
    """A 3-vector rounded to float32 once (a tuple of the float32 values)."""
    return (float(np.float32(x)), float(np.float32(y)), float(np.float32(z)))


def quat_axis_angle(axis, angle):
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    h = 0.5 * angle
    q = np.array([math.cos(h), *(math.sin(h) * axis)], np.float32)   # (w, x, y, z)
    return tuple(float(v) for v in q)


def rng_for(config: int, scene: int = 0) -> np.random.Generator:
    return np.random.default_rng(0x5EED0000 + config * 1000 + scene)


def _ground(s, half_x, half_z, top_y, friction=0.5):
    return s.add_body(CUBE, 1.0, friction, v3(0, top_y - 0.5, 0), v3(2 * half_x, 1, 2 * half_z), is_static=True)


# ---------------------------------------------------------------------------
# Workload configs
# ---------------------------------------------------------------------------
def pyramid_wall(s, rows=20, density=1000.0, friction=0.5, pitch=1.05, x0=0.0, z0=0.0, ground=True):
    """Plain rigid stack: `rows`-row 2-D pyramid of unit cubes (row r has
    rows-r cubes, 210 for 20 rows), pitch 1.05 m, resting on a static ground
    box (100 x 1 x 100 m, top at y = 0); the reference has no plane collider."""
    if ground:
        _ground(s, 50.0, 50.0, 0.0, friction)
    pos = []
    for r in range(rows):
        n = rows - r
        for k in range(n):
            pos.append((x0 + (k - 0.5 * (n - 1)) * pitch, 0.5 + r, z0))
    return _bulk_boxes(s, np.array(pos), np.ones((len(pos), 3)), None, density, friction)


def _bulk_boxes(s, pos, scale, yaw, density, friction):
    """Adds boxes (float32-rounded) through the solver's bulk insert; returns their ids."""
    n = len(pos)
    if n == 0:
        return []
    pos = np.asarray(pos, np.float32)
    scale = np.asarray(scale, np.float32)
    quat = np.zeros((n, 4), np.float32)
    quat[:, 0] = 1.0
    if yaw is not None:
        h = 0.5 * np.asarray(yaw, np.float64)
        quat[:, 0] = np.cos(h)
        quat[:, 2] = np.sin(h)
    first = s.add_bodies(CUBE, np.full(n, density, np.float32), np.full(n, friction, np.float32), pos, scale, quat,
                         np.zeros(n, np.int32))
    return list(range(first, first + n))


def fem_block(s, nx=41, ny=11, nz=11, cell=0.05, E=1e5, nu=0.3, density=1000.0, origin=(0.0, 0.0, 0.0),
              pin=True, friction=0.5):
    """Plain FEM block: makeTetVolume semantics (geometry.cpp:30-94), 5 tets per
    hex; 41x11x11 vertices (4,961; 20,000 tets) at 0.05 m; particle mass
    density*cell^3 (lumped uniform), min-x face pinned."""
    pm = density * cell ** 3
    return s.make_tet_volume(origin[0], origin[1], origin[2], nx, ny, nz, cell, E, nu, pm, friction, pin)


def mixed_large(s, n_boxes=32768, n_chains=64, links=32, n_springs=2048, seed_scene=0, nxz=50, config=3):
    """Plain large mixed rigid scene: `n_boxes` boxes with edges U[0.5, 1.5] m on
    a jittered lattice (`nxz` x `nxz` per layer) inside a 5-static-box
    container, `n_chains` hinge chains of `links` links anchored in the world,
    `n_springs` springs between random box pairs (k log-uniform [1e2, 1e5]
    N/m, rest = initial distance)."""
    rng = rng_for(config, seed_scene)
    # container: floor 84 x 1 x 84 (top at y = 0) + 4 walls 1 x 30 x 84
    s.add_body(CUBE, 1.0, 0.5, v3(0, -0.5, 0), v3(84, 1, 84), is_static=True)
    for (x, z, sx, sz) in ((-42.5, 0, 1, 84), (42.5, 0, 1, 84), (0, -42.5, 84, 1), (0, 42.5, 84, 1)):
        s.add_body(CUBE, 1.0, 0.5, v3(x, 15, z), v3(sx, 30, sz), is_static=True)
    pitch = 1.6
    idx = np.arange(n_boxes)
    i, k, j = idx % nxz, (idx // nxz) % nxz, idx // (nxz * nxz)
    edge = rng.uniform(0.5, 1.5, (n_boxes, 3))
    jit = rng.uniform(-0.05, 0.05, (n_boxes, 3))
    yaw = rng.uniform(-0.1, 0.1, n_boxes)
    pos = np.stack([(i - 0.5 * (nxz - 1)) * pitch + jit[:, 0], 0.8 + j * pitch + jit[:, 1],
                    (k - 0.5 * (nxz - 1)) * pitch + jit[:, 2]], axis=1)
    boxes = _bulk_boxes(s, pos, edge, yaw, 1000.0, 0.5)
    # horizontal hinge chains from world anchors at y = 45 (links 1.0 x 0.3 x 0.3 m)
    for c in range(n_chains):
        cx = -0.5 * links
        cz = -40.0 + c * (80.0 / max(1, n_chains - 1))
        prev = -1
        for l in range(links):
            pos = v3(cx + 0.5 + l * 1.0, 45.0, cz)
            b = s.add_body(CUBE, 1000.0, 0.5, pos, v3(1.0, 0.3, 0.3))
            if prev < 0:
                s.add_joint(-1, v3(cx, 45.0, cz), b, v3(-0.5, 0, 0), HINGE)
            else:
                s.add_joint(prev, v3(0.5, 0, 0), b, v3(-0.5, 0, 0), HINGE)
            prev = b
    for _ in range(n_springs):
        a, b = rng.choice(len(boxes), 2, replace=False)
        k = 10.0 ** rng.uniform(2.0, 5.0)
        s.add_spring(boxes[a], v3(0, 0, 0), boxes[b], v3(0, 0, 0), k, -1.0, False)
    return boxes


def stvk_block(s, nx=9, ny=4, nz=4, cell=0.2, E=1e5, nu=0.3, density=1000.0, pin=True, friction=0.5):
    """The Neo-Hookean block's particles and tets with StVK tets (config 2's
    StVK rerun; cell 0.2 m by default so particle boxes do not touch)."""
    pm = density * cell ** 3
    return s.make_stvk_tet_volume(0.0, 0.0, 0.0, nx, ny, nz, cell, E, nu, pm, friction, pin)


def served_scene(s, n_boxes, seed):
    """A served request: a scene of the batched mix's size composed like the
    large mixed scene: boxes in the container on a compact lattice (about 8
    layers), plus one world-anchored hinge link and one spring per 16 boxes."""
    nxz = max(2, int(math.ceil(math.sqrt(n_boxes / 8.0))))
    per = max(1, n_boxes // 16)
    return mixed_large(s, n_boxes=n_boxes, n_chains=per, links=1, n_springs=per, seed_scene=seed, nxz=nxz,
                       config=5)


def rigid_pile(s, n_boxes, rng, stack=True):
    """A batched rigid scene: `n_boxes` boxes as columns of unit cubes resting
    on each other (stack=True) or a loose jittered pile of boxes with edges
    U[0.6, 1.0] m and yaw U[-0.3, 0.3] rad dropped in place, on a static ground box."""
    _ground(s, 20.0, 20.0, 0.0)
    idx = np.arange(n_boxes)
    if stack:
        cols = max(1, int(math.ceil(math.sqrt(n_boxes / 8.0))))
        per = cols * cols
        lvl, c = idx // per, idx % per
        ci, cj = c // cols, c % cols
        pos = np.stack([(ci - 0.5 * (cols - 1)) * 1.1, 0.5 + lvl * 1.0, (cj - 0.5 * (cols - 1)) * 1.1], axis=1)
        return _bulk_boxes(s, pos, np.ones((n_boxes, 3)), None, 1000.0, 0.5)
    side = max(1, int(math.ceil(n_boxes ** (1.0 / 3.0))))
    i, k, j = idx % side, (idx // side) % side, idx // (side * side)
    e = rng.uniform(0.6, 1.0, (n_boxes, 3))
    jit = rng.uniform(-0.05, 0.05, (n_boxes, 3))
    yaw = rng.uniform(-0.3, 0.3, n_boxes)
    pos = np.stack([(i - 0.5 * (side - 1)) * 1.3 + jit[:, 0], 0.6 + j * 1.3 + jit[:, 1],
                    (k - 0.5 * (side - 1)) * 1.3 + jit[:, 2]], axis=1)
    return _bulk_boxes(s, pos, e, yaw, 1000.0, 0.5)


def fem_scene(s, n_tets, rng):
    """A batched FEM scene: a pinned block of about `n_tets` Neo-Hookean tets
    (aspect about 4:1:1, cell 0.2 m so vertex boxes do not touch)."""
    hexes = max(1, n_tets // 5)
    k = max(1, int(round((hexes / 4.0) ** (1.0 / 3.0))))
    nx = max(2, int(round(hexes / (k * k))) + 1)
    return s.make_tet_volume(0.0, 1.0, 0.0, nx, k + 1, k + 1, 0.2, 1e5, 0.3, 1000.0 * 0.2 ** 3, 0.5, True)


def batch_mix_specs(n_scenes=4096, fem_fraction=0.25, min_boxes=8, max_boxes=2048, min_tets=500, max_tets=5000,
                    config=4):
    """Scene mix of the batched workload: (kind, size, seed) per scene, box
    counts and tet counts log-uniform."""
    rng = rng_for(config, 0)
    specs = []
    for i in range(n_scenes):
        if rng.uniform() < fem_fraction:
            specs.append(("fem", int(math.exp(rng.uniform(math.log(min_tets), math.log(max_tets)))), i))
        else:
            specs.append(("stack" if i % 2 == 0 else "pile",
                          int(math.exp(rng.uniform(math.log(min_boxes), math.log(max_boxes)))), i))
    return specs


def build_spec(s, spec, config=4):
    kind, size, idx = spec
    rng = rng_for(config, idx)
    if kind == "fem":
        fem_scene(s, size, rng)
    else:
        rigid_pile(s, size, rng, stack=(kind == "stack"))


# ---------------------------------------------------------------------------
# Demo scenes of the reference (src/levels.h), re-expressed
# ---------------------------------------------------------------------------
def level_pyramid(s):
    """levels.h:28-82: 6-level 3-D pyramid of 2x1x2 blocks dropped on a ground box."""
    s.add_body(CUBE, 1.0, 0.5, v3(0, -10, 0), v3(20, 1, 20), is_static=True)
    levels, bw, bh, bd, sp = 6, 2.0, 1.0, 2.0, 0.3
    ground_top, drop = -9.5, 3.0
    for row in range(levels):
        n = levels - row
        span = n * bw + (n - 1) * sp
        sx = -span * 0.5 + bw * 0.5
        sz = -span * 0.5 + bd * 0.5
        y = ground_top + bh * 0.5 + row * (bh + sp) + drop
        for ix in range(n):
            for iz in range(n):
                s.add_body(CUBE, 1.0, 0.5, v3(sx + ix * (bw + sp), y, sz + iz * (bd + sp)), v3(bw, bh, bd))


def level_mass_stack(s):
    """levels.h:85-118: 5 boxes, each 1.5x larger than the one below."""
    s.add_body(CUBE, 1.0, 0.5, v3(0, -10, 0), v3(20, 1, 20), is_static=True)
    scale = 1.0
    for i in range(5):
        y = -9.5 + scale * 0.5 + i * (scale + 0.3) + 3.0
        s.add_body(CUBE, 1.0, 1.0, v3(0, y, 0), v3(scale, scale, scale))
        scale *= 1.5


def level_friction_slope(s):
    """levels.h:121-157: 10 blocks on a 30 degree slope, friction 0 .. 0.95."""
    q = quat_axis_angle((1, 0, 0), 30.0 * math.pi / 180.0)
    s.add_body(CUBE, 1.0, 0.5, v3(0, -10, 0), v3(35, 1, 10), quat=q, is_static=True)
    for i in range(10):
        fr = 0.95 * i / 9.0
        s.add_body(CUBE, 1.0, fr, v3(-15 + 3 * i, 1.0, 0), v3(2, 1, 2), quat=q)


def level_mass_springs(s):
    """levels.h:160-200: 8 blocks of growing density hanging on rope springs."""
    blocks = []
    for i in range(8):
        blocks.append(s.add_body(CUBE, 2.5 ** i, 0.5, v3(-7.0 + 2.0 * i, 0, 0), v3(1, 1, 1)))
    for i, b in enumerate(blocks):
        s.add_spring(-1, v3(-7.0 + 2.0 * i, 0, 0), b, v3(0, 0, 0), 1000.0, 3.0, True)


def level_joint_playground(s):
    """levels.h:203-329: hinge pendulum + rope bridge with one breakable link
    (fracture 2000) and three falling weights."""
    cs = np.array(v3(2.0, 0.7, 0.7), np.float32)
    anchor = np.array(v3(0, 5, 0), np.float32)
    last = -1
    spawn = np.array([anchor[0] + cs[0] / 2, anchor[1], anchor[2]], np.float32)
    for i in range(5):
        b = s.add_body(CUBE, 1.0, 0.5, spawn.copy(), cs)
        s.add_joint(last, v3(0.5, 0, 0) if last >= 0 else anchor, b, v3(-0.5, 0, 0), HINGE)
        last = b
        spawn[0] += cs[0]
    start = np.array(v3(-10, 5, -5), np.float32)
    cs = np.array(v3(2.0, 0.5, 3.0), np.float32)
    n_links, spacing = 12, 1.0
    last = -1
    spawn = np.array([start[0] + cs[0] / 2, start[1], start[2]], np.float32)
    z_edge, z_world = 0.5, 0.5 * cs[2]
    left = start - np.array(v3(spacing, 0, 0), np.float32)
    for i in range(n_links):
        b = s.add_body(CUBE, 1.0, 0.5, spawn.copy(), cs)
        fracture = 2000.0 if i == 6 else INF
        for side in range(2):
            zs = 1.0 if side == 0 else -1.0
            if last >= 0:
                ra, rb = v3(0.5, 0, zs * z_edge), v3(-0.5, 0, zs * z_edge)
            else:
                ra, rb = left + np.array(v3(0, 0, zs * z_world), np.float32), v3(-0.5, 0, zs * z_edge)
            s.add_spring(last, ra, b, rb, 5000.0, -1.0, False, fracture)
        last = b
        spawn[0] += cs[0] + spacing
    end = start + np.array(v3(cs[0] * n_links + (n_links - 1) * spacing, 0, 0), np.float32)
    right = end + np.array(v3(spacing, 0, 0), np.float32)
    for side in range(2):
        zs = 1.0 if side == 0 else -1.0
        s.add_spring(-1, right + np.array(v3(0, 0, zs * z_world), np.float32), last, v3(0.5, 0, zs * z_edge), INF,
                     -1.0, False)
    cx = float((start[0] + end[0]) * 0.5)
    bz = float(start[2])
    for (dx, y) in ((-0.5, 10.0), (0.5, 16.0), (0.0, 23.0)):
        s.add_body(CUBE, 1.0, 0.5, v3(cx + dx, y, bz), v3(3, 3, 3))


def make_tet(s, cx, cy, cz, edge, E, nu, mass=1.0, friction=0.5):
    """GeometryHelpers::makeTet (geometry.cpp:235-272): one regular tet of particles."""
    a = edge
    i3, i6, s23 = 1.0 / math.sqrt(3.0), 1.0 / math.sqrt(6.0), math.sqrt(2.0 / 3.0)
    vs = np.array([[0, 0, s23 * a], [-0.5 * a, -0.5 * i3 * a, -i6 * a], [0.5 * a, -0.5 * i3 * a, -i6 * a],
                   [0, i3 * a, -i6 * a]], np.float64)
    vs = vs - vs.mean(axis=0) + np.array([cx, cy, cz])
    ids = [s.add_particle(mass, friction, vs[i].astype(np.float32)) for i in range(4)]
    s.add_neohookean_tet(ids, E, nu)
    return ids


def level_neohookean_tets(s, E=8000.0, nu=0.3, particle_mass=1.0):
    """levels.h:332-372: 11 single tets of varying E and nu above a ground box."""
    s.add_body(CUBE, 1.0, 0.5, v3(0, -10, 0), v3(30, 1, 30), is_static=True)
    drop = -9.5 + 4.0
    for x, e in zip((-12, -6, 0, 6, 12), (50, 500, 3000, 8000, 20000)):
        make_tet(s, x, drop, 0, 3.0, e, 0.30, particle_mass)
    for x, n in zip((-12, -6, 0, 6, 12), (0.2, 0.25, 0.35, 0.42, 0.48)):
        make_tet(s, x, drop, -8.0, 3.0, 500, n, particle_mass)
    make_tet(s, 0, drop, 8.0, 3.0, E, nu, particle_mass)


def level_soft_beam(s, E=8000.0, nu=0.3, particle_mass=1.0):
    """levels.h:375-409: 9x3x3 pinned tet beam, cell 0.9 m."""
    n, cs = 3, 0.9
    return s.make_tet_volume(-3.0, 0.0, -(n - 1) * cs * 0.5, 3 * n, n, n, cs, E, nu, particle_mass, 0.5, True)


def level_cloth(s, E=8000.0, nu=0.3, particle_mass=1.0, N=10, M=15, spacing=1.5):
    """levels.h:442-491: StVK triangle cloth pinned at two corners."""
    sx = -(N - 1) * spacing * 0.5
    sz = -(M - 1) * spacing * 0.5
    parts = [0] * (N * M)
    for j in range(M):
        for i in range(N):
            parts[i + j * N] = s.add_particle(particle_mass, 0.5, v3(sx + i * spacing, 5.0, sz + j * spacing))
    s.set_static(parts[0], True)
    s.set_static(parts[N - 1], True)
    for j in range(M - 1):
        for i in range(N - 1):
            v00, v10 = parts[i + j * N], parts[i + 1 + j * N]
            v01, v11 = parts[i + (j + 1) * N], parts[i + 1 + (j + 1) * N]
            s.add_stvk_tri((v00, v10, v11), E, nu)
            s.add_stvk_tri((v00, v11, v01), E, nu)
    return parts


def level_soft_spheres(s, E=8000.0, nu=0.3, particle_mass=1.0):
    """levels.h:412-440: a makeTetSphere ball (radius 3, res 2: 149 particles,
    576 tets) dropped from 5 m above a static ground box."""
    s.add_body(CUBE, 1.0, 0.5, v3(0.0, -10.0, 0.0), v3(40.0, 1.0, 20.0), is_static=True)
    radius = 3.0
    return s.make_tet_sphere(0.0, -9.5 + radius + 5.0, 0.0, radius, 2.0, E, nu, particle_mass)


def level_safety_net(s, E=8000.0, nu=0.3, particle_mass=1.0, count=15, spacing=0.5):
    """levels.h:493-547: a 15x15 StVK triangle net pinned at its four corners."""
    sx = -(count - 1) * spacing * 0.5
    sz = -(count - 1) * spacing * 0.5
    parts = [0] * (count * count)
    for j in range(count):
        for i in range(count):
            parts[i + j * count] = s.add_particle(particle_mass, 0.5, v3(sx + i * spacing, -10.0, sz + j * spacing))
    for c in (0, count - 1, (count - 1) * count, count * count - 1):
        s.set_static(parts[c], True)
    for j in range(count - 1):
        for i in range(count - 1):
            v00, v10 = parts[i + j * count], parts[i + 1 + j * count]
            v01, v11 = parts[i + (j + 1) * count], parts[i + 1 + (j + 1) * count]
            s.add_stvk_tri((v00, v10, v11), E, nu)
            s.add_stvk_tri((v00, v11, v01), E, nu)
    return parts


LEVELS = {
    "pyramid": level_pyramid,
    "mass_stack": level_mass_stack,
    "friction_slope": level_friction_slope,
    "mass_springs": level_mass_springs,
    "joint_playground": level_joint_playground,
    "neohookean_tets": level_neohookean_tets,
    "soft_beam": level_soft_beam,
    "cloth": level_cloth,
    "soft_spheres": level_soft_spheres,
    "safety_net": level_safety_net,
}
