# SPDX-License-Identifier: MIT
"""Synthetic rigid scenes with the shapes and distributions of the benchmark
configurations: a cube pyramid, random box piles in a walled container,
capsule chains hanging from static anchors, and batches of independent
scenes. Every random draw comes from numpy's counter-based Philox generator,
so a seed fixes the scene bit for bit on any host.

A scene is a ``Scene`` of record arrays whose layouts are the C records of
``include/pmb200_core.h``: ``BODY_DTYPE`` (52 B, BodyParameters order),
``STATE_DTYPE`` (13 floats, PmRigidState order) and ``JOINT_DTYPE`` (220 B,
RigidConstraintOptions order with dense body indices). Rigid bodies are
triangle meshes, as in the reference: a box is a 12-triangle mesh
(tests/api/command_api_tests.cpp:339-350) and a capsule is a closed convex
tessellation small enough (<= 96 indices) for the convex face-contact path.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

STATIC, KINEMATIC, DYNAMIC = 0, 1, 2
FIXED, POINT, HINGE, SLIDER, PISTON, GENERIC, GENERIC_SPRING, MOTOR = range(8)

BODY_DTYPE = np.dtype([
    ("motion", "<u4"), ("mesh", "<u4"), ("inv_mass", "<f4"), ("inv_inertia", "<f4", 3),
    ("friction", "<f4"), ("restitution", "<f4"), ("linear_damping", "<f4"),
    ("angular_damping", "<f4"), ("max_linear_speed", "<f4"), ("max_angular_speed", "<f4"),
    ("margin", "<f4")])
assert BODY_DTYPE.itemsize == 52

STATE_DTYPE = np.dtype([("x", "<f4", 3), ("q", "<f4", 4), ("v", "<f4", 3), ("w", "<f4", 3)])
assert STATE_DTYPE.itemsize == 52

JOINT_DTYPE = np.dtype([
    ("type", "<u4"), ("body_a", "<u4"), ("body_b", "<u4"),
    ("anchor_a", "<f4", 3), ("anchor_b", "<f4", 3), ("frame_a", "<f4", 4), ("frame_b", "<f4", 4),
    ("lin_limit_axes", "<u4"), ("lin_lower", "<f4", 3), ("lin_upper", "<f4", 3),
    ("ang_limit_axes", "<u4"), ("ang_lower", "<f4", 3), ("ang_upper", "<f4", 3),
    ("lin_spring_axes", "<u4"), ("lin_stiffness", "<f4", 3), ("lin_damping", "<f4", 3),
    ("ang_spring_axes", "<u4"), ("ang_stiffness", "<f4", 3), ("ang_damping", "<f4", 3),
    ("motor_linear", "<u4"), ("motor_angular", "<u4"),
    ("motor_linear_velocity", "<f4"), ("motor_linear_max_impulse", "<f4"),
    ("motor_angular_velocity", "<f4"), ("motor_angular_max_impulse", "<f4"),
    ("enabled", "<u4"), ("disable_collisions", "<u4"), ("breaking_threshold", "<f4"),
    ("solver_iterations", "<u4")])
assert JOINT_DTYPE.itemsize == 220

STEP_DTYPE = np.dtype([
    ("dt", "<f4"), ("gravity", "<f4", 3), ("profile", "<u4"), ("requested_iterations", "<u4"),
    ("base_iterations", "<u4"), ("residual_tolerance", "<f4"), ("max_iterations", "<u4"),
    ("warm_start", "<u4"), ("collect_events", "<u4"), ("residual_norm", "<u4")])

STATS_DTYPE = np.dtype([
    ("candidate_pairs", "<u4"), ("active_pairs", "<u4"), ("contacts", "<u4"), ("colors", "<u4"),
    ("islands", "<u4"), ("iterations", "<u4"), ("impact", "<u4"), ("status", "<u4"),
    ("residual", "<f4"), ("residual_max", "<f4"), ("residual_over", "<f4")])

LEGACY, REALTIME = 0, 1
DT = np.float32(1.0 / 60.0)


@dataclasses.dataclass
class Scene:
    bodies: np.ndarray           # BODY_DTYPE[N]
    states: np.ndarray           # STATE_DTYPE[N]
    mesh_vertex_offsets: np.ndarray  # u32[M+1]
    vertices: np.ndarray         # f32[V, 3]
    mesh_index_offsets: np.ndarray   # u32[M+1]
    indices: np.ndarray          # u32[I]
    joints: np.ndarray           # JOINT_DTYPE[J]
    name: str = ""
    iterations: int = 10
    profile: int = LEGACY
    body_scene: np.ndarray | None = None        # batched worlds: scene of each body (u32, contiguous)
    scene_iterations: np.ndarray | None = None  # batched worlds: requested iterations per scene

    @property
    def n(self) -> int:
        return len(self.bodies)

    def step_desc(self, *, dt=DT, profile=None, iterations=None, residual_tolerance=0.0,
                  max_iterations=0, warm_start=0, collect_events=0, residual_norm=0) -> np.ndarray:
        s = np.zeros((), STEP_DTYPE)
        s["dt"] = dt
        s["gravity"] = (0.0, -9.81, 0.0)
        s["profile"] = self.profile if profile is None else profile
        s["requested_iterations"] = self.iterations if iterations is None else iterations
        s["base_iterations"] = 10
        s["residual_tolerance"] = residual_tolerance
        s["max_iterations"] = max_iterations
        s["warm_start"] = warm_start
        s["collect_events"] = collect_events
        s["residual_norm"] = residual_norm
        return s


class _Builder:
    def __init__(self):
        self.bodies, self.states, self.meshes, self.joints = [], [], [], []

    def mesh(self, vertices, indices) -> int:
        self.meshes.append((np.asarray(vertices, np.float32).reshape(-1, 3),
                            np.asarray(indices, np.uint32).reshape(-1)))
        return len(self.meshes) - 1

    def body(self, mesh, motion, x, q=(0, 0, 0, 1), v=(0, 0, 0), w=(0, 0, 0), mass=1.0,
             inertia=(1, 1, 1), friction=0.5, restitution=0.0, margin=0.005,
             max_speed=100.0, linear_damping=0.0, angular_damping=0.0) -> int:
        b = np.zeros((), BODY_DTYPE)
        b["motion"], b["mesh"] = motion, mesh
        if motion == DYNAMIC:
            b["inv_mass"] = np.float32(1.0) / np.float32(mass)
            b["inv_inertia"] = np.float32(1.0) / np.asarray(inertia, np.float32)
        b["friction"], b["restitution"], b["margin"] = friction, restitution, margin
        b["max_linear_speed"] = b["max_angular_speed"] = max_speed
        b["linear_damping"], b["angular_damping"] = linear_damping, angular_damping
        s = np.zeros((), STATE_DTYPE)
        s["x"], s["q"], s["v"], s["w"] = x, q, v, w
        self.bodies.append(b)
        self.states.append(s)
        return len(self.bodies) - 1

    def joint(self, kind, a, b, anchor_a, anchor_b, disable_collisions=True, iterations=0):
        j = np.zeros((), JOINT_DTYPE)
        j["type"], j["body_a"], j["body_b"] = kind, a, b
        j["anchor_a"], j["anchor_b"] = anchor_a, anchor_b
        j["frame_a"] = j["frame_b"] = (0, 0, 0, 1)
        j["enabled"] = 1
        j["disable_collisions"] = 1 if disable_collisions else 0
        j["solver_iterations"] = iterations
        self.joints.append(j)
        return len(self.joints) - 1

    def build(self, name, iterations, profile=LEGACY) -> Scene:
        voff = np.zeros(len(self.meshes) + 1, np.uint32)
        ioff = np.zeros(len(self.meshes) + 1, np.uint32)
        for k, (v, i) in enumerate(self.meshes):
            voff[k + 1] = voff[k] + len(v)
            ioff[k + 1] = ioff[k] + len(i)
        verts = np.concatenate([v for v, _ in self.meshes]) if self.meshes else np.zeros((0, 3), np.float32)
        idx = np.concatenate([i for _, i in self.meshes]) if self.meshes else np.zeros(0, np.uint32)
        return Scene(np.array(self.bodies, BODY_DTYPE), np.array(self.states, STATE_DTYPE), voff,
                     verts.astype(np.float32), ioff, idx.astype(np.uint32),
                     np.array(self.joints, JOINT_DTYPE).reshape(-1), name, iterations, profile)


# Outward-wound box triangles over the 8 corners (x fastest, then y, then z).
_BOX_TRIS = np.array([
    0, 2, 1, 1, 2, 3,  # -z
    4, 5, 6, 5, 7, 6,  # +z
    0, 1, 4, 1, 5, 4,  # -y
    2, 6, 3, 3, 6, 7,  # +y
    0, 4, 2, 2, 4, 6,  # -x
    1, 3, 5, 3, 7, 5,  # +x
], np.uint32)


def box_mesh(half):
    hx, hy, hz = (float(h) for h in half)
    v = np.array([[sx * hx, sy * hy, sz * hz] for sz in (-1, 1) for sy in (-1, 1) for sx in (-1, 1)],
                 np.float32)
    return v, _BOX_TRIS.copy()


def capsule_mesh(radius, length, segments=6):
    """Convex capsule tessellation along +y: a ``segments``-gon ring at each
    end of the cylinder and one pole per cap. 4*segments triangles (<= 96
    indices for segments <= 8)."""
    half = 0.5 * length
    ring = []
    for end in (-1, 1):
        for k in range(segments):
            a = 2.0 * math.pi * k / segments
            ring.append([radius * math.cos(a), end * half, radius * math.sin(a)])
    poles = [[0.0, -half - radius, 0.0], [0.0, half + radius, 0.0]]
    v = np.array(ring + poles, np.float32)
    lo, hi, pb, pt = 0, segments, 2 * segments, 2 * segments + 1
    tris = []
    for k in range(segments):
        k1 = (k + 1) % segments
        tris += [lo + k, hi + k, lo + k1, lo + k1, hi + k, hi + k1]   # side quad
        tris += [pb, lo + k, lo + k1]                                  # bottom cap
        tris += [pt, hi + k1, hi + k]                                  # top cap
    return v, np.array(tris, np.uint32)


def _fix_winding(v, t):
    """Orient every triangle outward from the centroid (convex meshes)."""
    t = t.reshape(-1, 3).copy()
    c = v.mean(axis=0)
    for row in t:
        a, b, d = v[row[0]], v[row[1]], v[row[2]]
        if np.dot(np.cross(b - a, d - a), a - c) < 0:
            row[1], row[2] = row[2], row[1]
    return t.reshape(-1)


def box_inertia(mass, half):
    h = np.asarray(half, np.float64)
    return (mass / 3.0 * (h[1] ** 2 + h[2] ** 2), mass / 3.0 * (h[0] ** 2 + h[2] ** 2),
            mass / 3.0 * (h[0] ** 2 + h[1] ** 2))


def _ground(b: _Builder, half_x, half_z, thickness=0.5, friction=0.5):
    m = b.mesh(*box_mesh((half_x, thickness, half_z)))
    return b.body(m, STATIC, (0.0, -thickness, 0.0), friction=friction)


def pyramid(levels=10, seed=1, jitter=1e-3, friction=0.5, density=1000.0, iterations=10,
            profile=LEGACY) -> Scene:
    """Planar pyramid of unit cubes (levels*(levels+1)/2 of them) on a static
    ground box; every cube centre jittered uniformly by +-jitter."""
    rng = np.random.Generator(np.random.Philox(seed))
    b = _Builder()
    _ground(b, 20.0, 20.0, friction=friction)
    cube = b.mesh(*box_mesh((0.5, 0.5, 0.5)))
    mass = density * 1.0
    inertia = box_inertia(mass, (0.5, 0.5, 0.5))
    for row in range(levels):
        count = levels - row
        for k in range(count):
            x = (k - 0.5 * (count - 1)) * 1.0
            y = 0.5 + row * 1.0
            d = rng.uniform(-jitter, jitter, 3)
            b.body(cube, DYNAMIC, (x + d[0], y + d[1], d[2]), mass=mass, inertia=inertia,
                   friction=friction)
    return b.build(f"pyramid{levels}", iterations, profile)


def box_pile(grid=(16, 16, 16), seed=2, spacing=1.8, iterations=10, profile=LEGACY,
             wall_height=None, count=None) -> Scene:
    """Random boxes (edges U[0.5,1.5] per axis, density U[500,2000], friction
    U[0.3,0.8]) on a jittered grid (gx along x, gy layers along y, gz along z)
    above a static walled container sized to the grid footprint. Walls are
    0.75 m per spawn layer high (at least 8 m) and the ground extends 10 m
    past them, so a settled pile stays on the ground."""
    gx, gy, gz = grid
    if wall_height is None:
        wall_height = max(8.0, 0.75 * gy)
    rng = np.random.Generator(np.random.Philox(seed))
    b = _Builder()
    half_x = 0.5 * gx * spacing + 1.0
    half_z = 0.5 * gz * spacing + 1.0
    _ground(b, half_x + 11.0, half_z + 11.0)
    wall_x = b.mesh(*box_mesh((0.5, 0.5 * wall_height, half_z + 1.0)))
    wall_z = b.mesh(*box_mesh((half_x + 1.0, 0.5 * wall_height, 0.5)))
    for s in (-1, 1):
        b.body(wall_x, STATIC, (s * (half_x + 0.5), 0.5 * wall_height, 0.0))
        b.body(wall_z, STATIC, (0.0, 0.5 * wall_height, s * (half_z + 0.5)))
    n = gx * gy * gz
    limit = n if count is None else min(n, count)
    edges = rng.uniform(0.5, 1.5, (n, 3)).astype(np.float32)
    density = rng.uniform(500.0, 2000.0, n)
    friction = rng.uniform(0.3, 0.8, n).astype(np.float32)
    jit = rng.uniform(-0.1, 0.1, (n, 3))
    k = 0
    for y in range(gy):
        for z in range(gz):
            for x in range(gx):
                if k >= limit:
                    break
                half = 0.5 * edges[k]
                m = b.mesh(*box_mesh(half))
                mass = float(density[k] * np.prod(edges[k].astype(np.float64)))
                pos = ((x - 0.5 * (gx - 1)) * spacing + jit[k, 0],
                       1.0 + y * spacing + jit[k, 1],
                       (z - 0.5 * (gz - 1)) * spacing + jit[k, 2])
                b.body(m, DYNAMIC, pos, mass=mass, inertia=box_inertia(mass, half),
                       friction=float(friction[k]))
                k += 1
    return b.build(f"pile{gx}x{gy}x{gz}", iterations, profile)


def joint_zoo(seed=6, profile=LEGACY, iterations=12, links=2) -> Scene:
    """One rig per joint type -- fixed, point, hinge (angular limit on its
    free axis), slider and piston (linear limit on the free axis; the piston
    also an angular limit), generic (equality and range limits on linear and
    angular axes), generic spring (springs on all six axes), motor (angular
    and linear drives) -- each a static anchor and `links` dynamic 0.4 m
    boxes in a chain started with seeded velocities, plus a point joint whose
    breaking threshold is below the impulse that holds its box."""
    rng = np.random.Generator(np.random.Philox(seed))
    b = _Builder()
    box = b.mesh(*box_mesh((0.2, 0.2, 0.2)))
    anchor = b.mesh(*box_mesh((0.1, 0.1, 0.1)))
    inertia = (0.32 / 12.0,) * 3

    def rig(kind, x0, setup=None, threshold=0.0):
        prev, prev_anchor = b.body(anchor, STATIC, (x0, 6.0, 0.0)), (0.0, -0.15, 0.0)
        for k in range(links):
            v = tuple(float(x) for x in rng.uniform(-1.0, 1.0, 3))
            w = tuple(float(x) for x in rng.uniform(-2.0, 2.0, 3))
            body = b.body(box, DYNAMIC, (x0, 6.0 - 0.45 - 0.5 * k, 0.0), v=v, w=w, mass=1.0, inertia=inertia)
            j = b.joint(kind, prev, body, prev_anchor, (0.0, 0.25, 0.0))
            o = b.joints[j]
            if setup:
                setup(o)
            o["breaking_threshold"] = threshold
            prev, prev_anchor = body, (0.0, -0.25, 0.0)

    def hinge(o):
        o["ang_limit_axes"] = 4
        o["ang_lower"], o["ang_upper"] = (0, 0, -0.5), (0, 0, 0.7)

    def slider(o):
        o["lin_limit_axes"] = 1
        o["lin_lower"], o["lin_upper"] = (-0.2, 0, 0), (0.3, 0, 0)

    def piston(o):
        slider(o)
        o["ang_limit_axes"] = 1
        o["ang_lower"], o["ang_upper"] = (-0.4, 0, 0), (0.4, 0, 0)

    def generic(o):
        o["lin_limit_axes"], o["ang_limit_axes"] = 7, 3
        o["lin_lower"], o["lin_upper"] = (-0.1, 0, 0), (0.2, 0, 0)
        o["ang_lower"], o["ang_upper"] = (-0.3, 0.0, 0), (0.3, 0.0, 0)

    def spring(o):
        o["lin_spring_axes"] = o["ang_spring_axes"] = 7
        o["lin_stiffness"], o["lin_damping"] = (200.0,) * 3, (5.0,) * 3
        o["ang_stiffness"], o["ang_damping"] = (50.0,) * 3, (1.0,) * 3

    def motor(o):
        o["motor_angular"] = o["motor_linear"] = 1
        o["motor_angular_velocity"], o["motor_angular_max_impulse"] = 2.0, 5.0
        o["motor_linear_velocity"], o["motor_linear_max_impulse"] = 0.5, 3.0

    kinds = [(FIXED, None), (POINT, None), (HINGE, hinge), (SLIDER, slider), (PISTON, piston),
             (GENERIC, generic), (GENERIC_SPRING, spring), (MOTOR, motor)]
    for k, (kind, setup) in enumerate(kinds):
        rig(kind, (k - 4.0) * 2.0, setup)
    rig(POINT, 8.0, threshold=0.12)
    b.body(b.mesh(*box_mesh((12.0, 0.5, 4.0))), STATIC, (0.0, -0.5, 0.0))
    return b.build("joint_zoo", iterations, profile)


def chains(count=512, links=64, seed=3, radius=0.05, length=0.4, spacing=1.0,
           iterations=20, profile=LEGACY, link_density=1000.0) -> Scene:
    """``count`` chains of ``links`` capsule links joined by point joints,
    the top link jointed to a static anchor, a box of 100x link mass on each
    free end, initial lateral velocity U(+-2) m/s per chain."""
    rng = np.random.Generator(np.random.Philox(seed))
    b = _Builder()
    cap_v, cap_t = capsule_mesh(radius, length)
    cap = b.mesh(cap_v, _fix_winding(cap_v, cap_t))
    anchor = b.mesh(*box_mesh((0.05, 0.05, 0.05)))
    link_mass = link_density * (math.pi * radius ** 2 * length + 4.0 / 3.0 * math.pi * radius ** 3)
    link_inertia = (link_mass * (3 * radius ** 2 + length ** 2) / 12.0, link_mass * radius ** 2 / 2.0,
                    link_mass * (3 * radius ** 2 + length ** 2) / 12.0)
    box_half = (0.2, 0.2, 0.2)
    end = b.mesh(*box_mesh(box_half))
    end_mass = 100.0 * link_mass
    side = int(math.ceil(math.sqrt(count)))
    top = 2.0 + links * length + 1.0
    vel = rng.uniform(-2.0, 2.0, (count, 2))
    pitch = length + 2 * radius
    for c in range(count):
        cx = (c % side - 0.5 * (side - 1)) * spacing
        cz = (c // side - 0.5 * (side - 1)) * spacing
        a = b.body(anchor, STATIC, (cx, top, cz))
        v0 = (float(vel[c, 0]), 0.0, float(vel[c, 1]))
        prev, prev_anchor = a, (0.0, 0.0, 0.0)
        for k in range(links):
            y = top - 0.5 * pitch - k * pitch
            link = b.body(cap, DYNAMIC, (cx, y, cz), v=v0, mass=link_mass, inertia=link_inertia,
                          friction=0.5)
            b.joint(POINT, prev, link, prev_anchor, (0.0, 0.5 * pitch, 0.0))
            prev, prev_anchor = link, (0.0, -0.5 * pitch, 0.0)
        y = top - links * pitch - box_half[1]
        box = b.body(end, DYNAMIC, (cx, y, cz), v=v0, mass=end_mass,
                     inertia=box_inertia(end_mass, box_half), friction=0.5)
        b.joint(POINT, prev, box, prev_anchor, (0.0, box_half[1], 0.0))
    return b.build(f"chains{count}x{links}", iterations, profile)


def prism_mesh(polygon, half_z):
    """A closed prism: the simple polygon ``polygon`` (x, y pairs, counter-
    clockwise) extruded over z in [-half_z, half_z], caps ear-clipped, every
    triangle wound outward. Concave polygons give concave meshes."""
    p = [(float(x), float(y)) for x, y in polygon]
    m = len(p)
    v = np.array([[x, y, -half_z] for x, y in p] + [[x, y, half_z] for x, y in p], np.float32)

    def cross2(o, a, b):
        return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])

    def inside(q, a, b, c):
        return cross2(a, b, q) > 0 and cross2(b, c, q) > 0 and cross2(c, a, q) > 0

    ring, cap = list(range(m)), []
    while len(ring) > 3:
        for k in range(len(ring)):
            i0, i1, i2 = ring[k - 1], ring[k], ring[(k + 1) % len(ring)]
            a, b, c = p[i0], p[i1], p[i2]
            if cross2(a, b, c) <= 0:
                continue
            if any(inside(p[j], a, b, c) for j in ring if j not in (i0, i1, i2)):
                continue
            cap.append((i0, i1, i2))
            ring.pop(k)
            break
        else:
            raise ValueError("polygon is not simple and counter-clockwise")
    cap.append(tuple(ring))
    tris = []
    for a, b, c in cap:
        tris += [m + a, m + b, m + c]   # +z cap: counter-clockwise seen from +z
        tris += [a, c, b]               # -z cap
    for k in range(m):
        k1 = (k + 1) % m
        tris += [k, k1, m + k1, k, m + k1, m + k]   # side quad, outward for a CCW polygon
    return v, np.array(tris, np.uint32)


def mesh_mix(profile=LEGACY, iterations=10, seed=11, margin=0.04) -> Scene:
    """Pairs the convex face path does not take: three boxes dropped into a
    static U-shaped trough (a closed concave prism), an L-shaped body (concave)
    resting on the ground with another dropped on it, and a capsule of 64
    triangles (convex but above the face path's 96 indices) lying down.
    Collision margins of 4 cm let the unswept contacts catch the falls; with
    the default 5 mm the falls need the swept (continuous) contacts."""
    rng = np.random.Generator(np.random.Philox(seed))
    b = _Builder()
    _ground(b, 5.0, 5.0)
    trough = b.mesh(*prism_mesh([(-1, 0), (1, 0), (1, 1), (0.8, 1), (0.8, 0.2), (-0.8, 0.2), (-0.8, 1), (-1, 1)],
                                1.0))
    b.body(trough, STATIC, (0.0, 0.0, 0.0), margin=margin)
    cube = b.mesh(*box_mesh((0.15, 0.15, 0.15)))
    for k in range(3):
        x = float(rng.uniform(-0.4, 0.4))
        b.body(cube, DYNAMIC, (x, 0.6 + 0.35 * k, float(rng.uniform(-0.3, 0.3))), mass=1.0,
               inertia=box_inertia(1.0, (0.15,) * 3), margin=margin)
    ell = [(0, 0), (0.6, 0), (0.6, 0.2), (0.2, 0.2), (0.2, 0.6), (0, 0.6)]
    cx, cy = 0.2, 0.2
    lmesh = b.mesh(*prism_mesh([(x - cx, y - cy) for x, y in ell], 0.15))
    l_inertia = box_inertia(2.0, (0.3, 0.3, 0.15))
    b.body(lmesh, DYNAMIC, (2.5, cy + 0.001, 0.0), mass=2.0, inertia=l_inertia, margin=margin)
    b.body(lmesh, DYNAMIC, (2.55, cy + 0.9, 0.05), mass=2.0, inertia=l_inertia, margin=margin)
    cap = b.mesh(*capsule_mesh(0.2, 0.8, segments=16))
    s = math.sqrt(0.5)
    b.body(cap, DYNAMIC, (-2.5, 0.25, 0.0), q=(0.0, 0.0, s, s), mass=1.5,
           inertia=box_inertia(1.5, (0.2, 0.6, 0.2)), margin=margin)
    return b.build("mesh mix", iterations, profile)


def guided_stop(kind=None, profile=LEGACY, iterations=10, speed=3.0) -> Scene:
    """Guided contacts: a box on an unbreakable piston (or slider) joint to a
    static anchor slides along the joint's axis into a static stop block.
    The box is the guide's only joint member, so the box-stop pair is guided:
    the face path skips it and the triangle-mesh path's swept ranges give its
    contacts, merged by guide direction and held at the guided offset."""
    kind = PISTON if kind is None else kind
    b = _Builder()
    anchor = b.mesh(*box_mesh((0.1, 0.1, 0.1)))
    box = b.mesh(*box_mesh((0.2, 0.2, 0.2)))
    a = b.body(anchor, STATIC, (0.0, 1.0, 0.0))
    body = b.body(box, DYNAMIC, (0.6, 1.0, 0.0), v=(speed, 0.0, 0.0), mass=1.0, inertia=box_inertia(1.0, (0.2,) * 3))
    b.body(box, STATIC, (2.0, 1.0, 0.0))
    b.joint(kind, a, body, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    return b.build("guided stop", iterations, profile)


def welded_groups(profile=LEGACY, iterations=10, disable_bc=True) -> Scene:
    """Fixed collision groups. Bars A, B, C (1.2 m long) in a row 0.5 m apart,
    welded A-B and B-C by collision-disabling fixed joints: A and C overlap
    but share a group, so they never touch. Boxes D and E overlap each other
    and are each welded to the static post P: the post joins them into one
    group. A free box F rests on C (an ordinary contact with a group member).
    disable_bc=False leaves the B-C weld colliding, which splits the first
    group, so A-C and B-C become candidate pairs."""
    b = _Builder()
    _ground(b, 4.0, 4.0)
    bar = b.mesh(*box_mesh((0.6, 0.1, 0.1)))
    small = b.mesh(*box_mesh((0.2, 0.1, 0.1)))
    post = b.mesh(*box_mesh((0.1, 1.0, 0.1)))
    cube = b.mesh(*box_mesh((0.15, 0.15, 0.15)))
    bar_inertia = box_inertia(1.0, (0.6, 0.1, 0.1))
    small_inertia = box_inertia(0.5, (0.2, 0.1, 0.1))
    bars = [b.body(bar, DYNAMIC, (-1.0 + 0.5 * k, 0.3, 0.0), mass=1.0, inertia=bar_inertia) for k in range(3)]
    b.joint(FIXED, bars[0], bars[1], (0.25, 0.0, 0.0), (-0.25, 0.0, 0.0))
    b.joint(FIXED, bars[1], bars[2], (0.25, 0.0, 0.0), (-0.25, 0.0, 0.0), disable_collisions=disable_bc)
    p = b.body(post, STATIC, (2.0, 1.0, 0.0))
    d = b.body(small, DYNAMIC, (2.25, 1.5, 0.0), mass=0.5, inertia=small_inertia)
    e = b.body(small, DYNAMIC, (2.3, 1.55, 0.0), mass=0.5, inertia=small_inertia)
    b.joint(FIXED, p, d, (0.15, 0.5, 0.0), (-0.1, 0.0, 0.0))
    b.joint(FIXED, p, e, (0.15, 0.55, 0.0), (-0.15, 0.0, 0.0))
    b.body(cube, DYNAMIC, (0.1, 0.56, 0.0), mass=0.5, inertia=box_inertia(0.5, (0.15,) * 3))
    return b.build("welded groups", iterations, profile)


def cube_pair(profile=REALTIME) -> Scene:
    """A static unit cube at y = -1 and a dynamic one at y = 2 (mass 1,
    inertia 1/6, friction 0.5, damping 0.05, speed limits 100, margin 5 mm):
    the scene the reference's command-API test steps
    (tests/api/command_api_tests.cpp:338-456)."""
    b = _Builder()
    m = b.mesh(*box_mesh((0.5, 0.5, 0.5)))
    common = dict(mass=1.0, inertia=(1.0 / 6.0,) * 3, friction=0.5, margin=0.005, max_speed=100.0,
                  linear_damping=0.05, angular_damping=0.05)
    b.body(m, STATIC, (0.0, -1.0, 0.0), **common)
    b.body(m, DYNAMIC, (0.0, 2.0, 0.0), **common)
    return b.build("cube pair", 10, profile)


def batch(parts, name="batch") -> Scene:
    """Independent scenes stepped as one batched world: bodies, meshes and
    joints concatenated (indices offset), each body tagged with its scene.
    All parts share one profile; each keeps its own requested iterations."""
    profile = parts[0].profile
    assert all(p.profile == profile for p in parts)
    bodies, states, joints, verts, idx, scene = [], [], [], [], [], []
    voff, ioff = [0], [0]
    mesh_base = body_base = 0
    for k, p in enumerate(parts):
        b = p.bodies.copy()
        b["mesh"] += mesh_base
        bodies.append(b)
        states.append(p.states)
        if len(p.joints):
            j = p.joints.copy()
            j["body_a"] += body_base
            j["body_b"] += body_base
            joints.append(j)
        for m in range(len(p.mesh_vertex_offsets) - 1):
            v0, v1 = p.mesh_vertex_offsets[m], p.mesh_vertex_offsets[m + 1]
            i0, i1 = p.mesh_index_offsets[m], p.mesh_index_offsets[m + 1]
            verts.append(p.vertices[v0:v1])
            idx.append(p.indices[i0:i1])
            voff.append(voff[-1] + int(v1 - v0))
            ioff.append(ioff[-1] + int(i1 - i0))
        scene.append(np.full(p.n, k, np.uint32))
        mesh_base += len(p.mesh_vertex_offsets) - 1
        body_base += p.n
    return Scene(np.concatenate(bodies), np.concatenate(states), np.array(voff, np.uint32),
                 np.concatenate(verts).astype(np.float32), np.array(ioff, np.uint32),
                 np.concatenate(idx).astype(np.uint32),
                 np.concatenate(joints) if joints else np.zeros(0, JOINT_DTYPE), name,
                 max(p.iterations for p in parts), profile, np.concatenate(scene),
                 np.array([p.iterations for p in parts], np.uint32))


def batched_plan(count=1024, seed=5, smallest=16, largest=2048):
    """Config-5 draw: body counts log-uniform in [smallest, largest] and the
    kind of each scene (True: box pile, False: joint chains), 50/50."""
    rng = np.random.Generator(np.random.Philox(seed))
    sizes = np.exp(rng.uniform(math.log(smallest), math.log(largest), count)).astype(int)
    kinds = rng.uniform(0.0, 1.0, count) < 0.5
    return sizes, kinds


def batched_part(k, size, kind, seed=5, profile=LEGACY) -> Scene:
    """Scene `k` of a config-5 batch: a random box pile (config-2
    distributions, 10 iterations) of `size` boxes, or `size // 17` joint
    chains (config-3 distributions, 16 links and an end box per chain, 20
    iterations). Depends only on (k, size, kind, seed), so any subset of the
    batch can be built on its own."""
    n = int(size)
    sub = seed * 100000 + int(k)
    if kind:
        side = max(1, int(round(n ** (1.0 / 3.0))))
        layers = int(math.ceil(n / (side * side)))
        return box_pile((side, layers, side), seed=sub, spacing=1.6, profile=profile,
                        wall_height=max(4.0, 0.75 * layers), count=n)
    return chains(count=max(1, n // 17), links=16, seed=sub, profile=profile)


def batched_scenes(count=1024, seed=5, smallest=16, largest=2048, profile=LEGACY, subset=None):
    """Config-5 mix: `count` independent scenes (batched_plan, batched_part)
    as one batched world; `subset` (scene indices) builds only those."""
    sizes, kinds = batched_plan(count, seed, smallest, largest)
    ids = range(count) if subset is None else subset
    parts = [batched_part(k, sizes[k], kinds[k], seed, profile) for k in ids]
    return batch(parts, f"batch{count}" if subset is None else f"batch{count}[{len(parts)}]")


def shard_scenes(weights, ranks):
    """Independent scenes bin-packed over `ranks` GPUs by weight (body
    count): longest-processing-time greedy -- heaviest scene first, each to
    the least-loaded rank, ties to the lower rank. Returns one ascending list
    of scene indices per rank; every scene appears exactly once."""
    weights = np.asarray(weights, np.int64)
    order = sorted(range(len(weights)), key=lambda k: (-int(weights[k]), k))
    load = [0] * ranks
    out = [[] for _ in range(ranks)]
    for k in order:
        r = min(range(ranks), key=lambda i: (load[i], i))
        out[r].append(k)
        load[r] += int(weights[k])
    return [sorted(x) for x in out]


def config(index: int) -> Scene:
    """The benchmark configurations 1-4 at full size (0-based ``index``)."""
    if index == 0:
        return pyramid()
    if index == 1:
        return box_pile((16, 16, 16), seed=2)
    if index == 2:
        return chains()
    if index == 3:
        return box_pile((64, 32, 32), seed=4)
    raise ValueError(index)


def pile_grid_for_config4():
    """64x32x32 spawn grid: 64 along x, 32 layers, 32 along z."""
    return (64, 32, 32)
