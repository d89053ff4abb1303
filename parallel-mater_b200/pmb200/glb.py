# SPDX-License-Identifier: MIT
"""Rigid part of the reference's authored-scene loader: a GLB (binary glTF
2.0) exported with the reference's Blender schema-2 extras, read into meshes,
rigid bodies and rigid constraints.

The rules restate the gallery loader (reference examples/support/scene.cpp,
load_glb_scene:636-1052, with read_metadata:156-217, node_state:225-237,
append_primitive:260-364 and finalize_body_geometry:484-527):

- nodes whose extras carry pm_system "collision_mesh" become collision
  proxies (their primitives, scaled by the node scale), keyed by pm_name;
- nodes with pm_system "rigid_body" become bodies: motion from pm_motion,
  mass (required when dynamic), friction, restitution, damping and collision
  margin from the extras over RigidBodyOptions' defaults (mass 1, friction
  0.5, damping 0.05, speeds 100, margin 0.005; a zero inertia diagonal, which
  asks the driver for the mesh box inertia); pose from the node's TRS, linear
  velocity from pm_initial_velocity_{x,y,z}; one triangle mesh per primitive,
  positions scaled by the node scale, then every vertex re-centred on the
  body's bounds centre and the position moved by the rotated centre; a body
  with pm_collision_proxy collides with that proxy's meshes (re-centred the
  same way); bodies that share a glTF mesh and scale share its meshes;
- nodes with pm_system "rigid_constraint" become constraints between the
  bodies named by pm_body_a / pm_body_b (pm_name or pm_source_name): the
  frame is the node's TRS with Blender's local Z restored (rotated by -90
  degrees about x), expressed in each body's frame; options from the extras
  (enabled, disable_collisions, breaking threshold, solver iterations, per
  axis linear / angular limits and springs, linear / angular motor).

Arithmetic is float32, in the loader's order.
"""
from __future__ import annotations

import json
import struct

import numpy as np

from . import scenes

f32 = np.float32

_COMPONENT = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_WIDTH = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4}
_MOTION = {"static": scenes.STATIC, "kinematic": scenes.KINEMATIC, "dynamic": scenes.DYNAMIC}
_JOINT_TYPES = {"fixed": scenes.FIXED, "point": scenes.POINT, "hinge": scenes.HINGE, "slider": scenes.SLIDER,
                "piston": scenes.PISTON, "generic": scenes.GENERIC, "generic_spring": scenes.GENERIC_SPRING,
                "motor": scenes.MOTOR}


class GlbError(ValueError):
    pass


def read_glb(data: bytes):
    """(document, binary chunk) of a GLB container."""
    magic, version, length = struct.unpack_from("<4sII", data, 0)
    if magic != b"glTF" or version != 2 or length > len(data):
        raise GlbError("not a glTF 2.0 binary")
    off, doc, blob = 12, None, b""
    while off + 8 <= length:
        size, kind = struct.unpack_from("<I4s", data, off)
        chunk = data[off + 8:off + 8 + size]
        if kind == b"JSON":
            doc = json.loads(chunk)
        elif kind == b"BIN\x00":
            blob = chunk
        off += 8 + size + (-size % 4)
    if doc is None:
        raise GlbError("GLB without a JSON chunk")
    return doc, blob


def accessor(doc, blob, index):
    """Accessor `index` as an array [count, width] (dense accessors)."""
    a = doc["accessors"][index]
    if "sparse" in a:
        raise GlbError("sparse accessors are not supported")
    dtype = np.dtype(_COMPONENT[a["componentType"]]).newbyteorder("<")
    width, count = _WIDTH[a["type"]], a["count"]
    view = doc["bufferViews"][a["bufferView"]]
    start = view.get("byteOffset", 0) + a.get("byteOffset", 0)
    row = dtype.itemsize * width
    stride = view.get("byteStride", 0) or row
    if stride == row:
        return np.frombuffer(blob, dtype, count=count * width, offset=start).reshape(count, width)
    return np.stack([np.frombuffer(blob, dtype, count=width, offset=start + k * stride) for k in range(count)]) \
        if count else np.zeros((0, width), dtype)


def _cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], f32)


def rotate(q, v):
    """v rotated by unit quaternion q (x, y, z, w): v + w t + q x t with
    t = 2 (q x v), in float32."""
    q = np.asarray(q, f32)
    v = np.asarray(v, f32)
    t = _cross(q[:3], v) * f32(2.0)
    return v + (t * q[3] + _cross(q[:3], t))


def qmul(a, b):
    a = np.asarray(a, f32)
    b = np.asarray(b, f32)
    return np.array([a[3] * b[0] + a[0] * b[3] + a[1] * b[2] - a[2] * b[1],
                     a[3] * b[1] - a[0] * b[2] + a[1] * b[3] + a[2] * b[0],
                     a[3] * b[2] + a[0] * b[1] - a[1] * b[0] + a[2] * b[3],
                     a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2]], f32)


def conj(q):
    q = np.asarray(q, f32)
    return np.array([-q[0], -q[1], -q[2], q[3]], f32)


def _node_state(node):
    x = np.array(node.get("translation", (0.0, 0.0, 0.0)), f32)
    q = np.array(node.get("rotation", (0.0, 0.0, 0.0, 1.0)), f32)
    return x, q


def _node_scale(node, name):
    s = np.array(node.get("scale", (1.0, 1.0, 1.0)), f32)
    if not np.all(np.isfinite(s)) or np.any(s < f32(1e-6)):
        raise GlbError(f"{name}: scale must be finite and positive")
    return s


def _primitive(doc, blob, prim, scale, name):
    if prim.get("mode", 4) != 4:
        raise GlbError(f"{name}: only triangle primitives are supported")
    if "POSITION" not in prim["attributes"]:
        raise GlbError(f"{name}: POSITION vec3 data is required")
    pos = accessor(doc, blob, prim["attributes"]["POSITION"]).astype(f32) * scale
    if "indices" in prim:
        idx = accessor(doc, blob, prim["indices"]).reshape(-1).astype(np.uint32)
    else:
        idx = np.arange(len(pos), dtype=np.uint32)
    if len(idx) % 3 or (len(idx) and int(idx.max()) >= len(pos)):
        raise GlbError(f"{name}: triangle index data is invalid")
    return [pos.astype(f32), idx]


def _root_trs(node, name):
    if "matrix" in node:
        raise GlbError(f"{name}: matrix transforms are unsupported; export TRS")


class GlbScene:
    """meshes: [[vertices float32 [n, 3], indices uint32]]; bodies and
    constraints: dicts of the loader's definitions (see load_glb_scene)."""

    def __init__(self):
        self.meshes, self.collision_meshes, self.bodies, self.constraints = [], [], [], []


def load_glb_scene(data: bytes) -> GlbScene:
    doc, blob = read_glb(data)
    nodes = doc.get("nodes", [])
    children = {c for n in nodes for c in n.get("children", [])}
    out = GlbScene()

    def extras(n):
        return n.get("extras") or {}

    proxies = {}
    for k, node in enumerate(nodes):
        e = extras(node)
        if e.get("pm_system") != "collision_mesh":
            continue
        name = e.get("pm_name", node.get("name", f"collision_node_{k}"))
        if e.get("pm_schema") != 2:
            raise GlbError(f"{name}: unsupported or missing pm_schema")
        if k in children or "matrix" in node:
            raise GlbError(f"{name}: collision proxies must be scene-root TRS nodes")
        scale = _node_scale(node, name)
        mesh = doc["meshes"][node["mesh"]]
        ids = []
        for p, prim in enumerate(mesh["primitives"]):
            ids.append(len(out.collision_meshes))
            out.collision_meshes.append(_primitive(doc, blob, prim, scale, f"{name}/primitive_{p}"))
        if name in proxies:
            raise GlbError(f"{name}: duplicate collision proxy name")
        proxies[name] = (_node_state(node), ids)

    shared = {}
    used_proxies = set()
    for k, node in enumerate(nodes):
        e = extras(node)
        system = e.get("pm_system")
        if system not in ("rigid_body", "sphere_cluster"):
            continue
        name = node.get("name", f"node_{k}")
        if e.get("pm_schema") != 2:
            raise GlbError(f"{name}: unsupported or missing pm_schema")
        motion = e.get("pm_motion")
        if motion not in _MOTION:
            raise GlbError(f"{name}: pm_motion is required" if motion is None else f"{name}: invalid pm_motion")
        if "pm_mass" not in e and motion == "dynamic":
            raise GlbError(f"{name}: dynamic bodies require pm_mass")
        body = {"name": e.get("pm_name", name), "motion": _MOTION[motion],
                "mass": f32(e.get("pm_mass", 1.0)), "inertia": (0.0, 0.0, 0.0),
                "friction": f32(e.get("pm_friction", 0.5)), "restitution": f32(e.get("pm_restitution", 0.0)),
                "linear_damping": f32(e.get("pm_linear_damping", 0.05)),
                "angular_damping": f32(e.get("pm_angular_damping", 0.05)),
                "margin": f32(e.get("pm_collision_margin", 0.005)), "max_speed": f32(100.0),
                "system": system}
        body["source_name"] = e.get("pm_source_name", body["name"])
        if k in children:
            raise GlbError(f"{body['name']}: physics objects must be scene-root nodes")
        _root_trs(node, body["name"])
        if "mesh" not in node or not doc["meshes"][node["mesh"]]["primitives"]:
            raise GlbError(f"{body['name']}: physics objects require render geometry")
        scale = _node_scale(node, body["name"])
        x, q = _node_state(node)
        body["velocity"] = np.array([e.get(f"pm_initial_velocity_{a}", 0.0) for a in "xyz"], f32)
        proxy = e.get("pm_collision_proxy")
        key = (node["mesh"], tuple(float(s) for s in scale))
        reuse = proxy is None and key in shared
        if reuse:
            body["mesh_indices"], center = shared[key]
        else:
            ids = []
            for p, prim in enumerate(doc["meshes"][node["mesh"]]["primitives"]):
                ids.append(len(out.meshes))
                out.meshes.append(_primitive(doc, blob, prim, scale, f"{body['name']}/primitive_{p}"))
            body["mesh_indices"] = ids
        body["collision_mesh_indices"] = []
        if proxy is not None:
            if proxy not in proxies:
                raise GlbError(f"{body['name']}: collision proxy '{proxy}' was not exported")
            if proxy in used_proxies:
                raise GlbError(f"{body['name']}: collision proxy '{proxy}' is already assigned to another body")
            used_proxies.add(proxy)
            (px, pq), pids = proxies[proxy]
            if np.max(np.abs(px - x)) > 1e-5 or abs(abs(float(np.dot(pq, q))) - 1.0) > 1e-5:
                raise GlbError(f"{body['name']}: collision proxy must share the rigid-body transform")
            body["collision_mesh_indices"] = list(pids)
        if not reuse:
            verts = np.concatenate([out.meshes[m][0] for m in body["mesh_indices"]])
            lo, hi = verts.min(axis=0), verts.max(axis=0)
            center = (lo + hi) * f32(0.5)
            half = (hi - lo) * f32(0.5)
            if not np.all(np.isfinite(center)) or half[0] < f32(1e-6) or half[2] < f32(1e-6):
                raise GlbError(f"{body['name']}: render bounds are invalid")
            for m in body["mesh_indices"]:
                out.meshes[m][0] = out.meshes[m][0] - center
            for m in body["collision_mesh_indices"]:
                out.collision_meshes[m][0] = out.collision_meshes[m][0] - center
            if proxy is None:
                shared[key] = (body["mesh_indices"], center)
        body["position"] = x + rotate(q, center)
        body["orientation"] = q
        if system == "rigid_body":
            out.bodies.append(body)

    half_pi = f32(1.5707963267948966)
    basis = np.array([np.sin(-half_pi * f32(0.5)), 0.0, 0.0, np.cos(-half_pi * f32(0.5))], f32)
    for k, node in enumerate(nodes):
        e = extras(node)
        if e.get("pm_system") != "rigid_constraint":
            continue
        name = e.get("pm_name", node.get("name", "rigid_constraint"))
        if e.get("pm_schema") != 2 or k in children or "matrix" in node:
            raise GlbError(f"{name}: rigid constraint needs schema 2 and a scene-root TRS node")
        kind = e.get("pm_constraint_type", "")
        if kind not in _JOINT_TYPES:
            raise GlbError(f"{name}: unsupported rigid constraint type")

        def find(key):
            target = e.get(key, "")
            hits = [b for b, body in enumerate(out.bodies) if target in (body["name"], body["source_name"])]
            return hits[0] if len(hits) == 1 else None
        a, b = find("pm_body_a"), find("pm_body_b")
        if a is None or b is None or a == b:
            raise GlbError(f"{name}: constraint body name is missing, ambiguous, or repeated")
        fx, fq = _node_state(node)
        fq = qmul(fq, basis)
        c = {"name": name, "type": _JOINT_TYPES[kind], "body_a": a, "body_b": b,
             "enabled": bool(e.get("pm_enabled", True)), "disable_collisions": bool(e.get("pm_disable_collisions", True)),
             "breaking_threshold": f32(e.get("pm_breaking_impulse_threshold", 0.0))}
        for side, idx in (("a", a), ("b", b)):
            inv = conj(out.bodies[idx]["orientation"])
            c[f"anchor_{side}"] = rotate(inv, fx - out.bodies[idx]["position"])
            c[f"frame_{side}"] = qmul(inv, fq)
        iters = e.get("pm_solver_iterations", 8.0)
        if not (1.0 <= iters <= 64.0) or iters != int(iters):
            raise GlbError(f"{name}: invalid constraint solver iterations")
        c["solver_iterations"] = int(iters)
        for field in ("lin_limit", "ang_limit", "lin_spring", "ang_spring"):
            c[field + "_axes"] = 0
        c.update({k2: np.zeros(3, f32) for k2 in ("lin_lower", "lin_upper", "ang_lower", "ang_upper", "lin_stiffness",
                                                  "lin_damping", "ang_stiffness", "ang_damping")})
        for ax, s in enumerate("xyz"):
            bit = 1 << ax
            if e.get(f"pm_use_limit_lin_{s}", False):
                c["lin_limit_axes"] |= bit
            c["lin_lower"][ax] = e.get(f"pm_limit_lin_{s}_lower", 0.0)
            c["lin_upper"][ax] = e.get(f"pm_limit_lin_{s}_upper", 0.0)
            if e.get(f"pm_use_limit_ang_{s}", False):
                c["ang_limit_axes"] |= bit
            c["ang_lower"][ax] = e.get(f"pm_limit_ang_{s}_lower", 0.0)
            c["ang_upper"][ax] = e.get(f"pm_limit_ang_{s}_upper", 0.0)
            if e.get(f"pm_use_spring_{s}", False):
                c["lin_spring_axes"] |= bit
            c["lin_stiffness"][ax] = e.get(f"pm_spring_stiffness_{s}", 0.0)
            c["lin_damping"][ax] = e.get(f"pm_spring_damping_{s}", 0.0)
            if e.get(f"pm_use_spring_ang_{s}", False):
                c["ang_spring_axes"] |= bit
            c["ang_stiffness"][ax] = e.get(f"pm_spring_stiffness_ang_{s}", 0.0)
            c["ang_damping"][ax] = e.get(f"pm_spring_damping_ang_{s}", 0.0)
        c["motor_linear"] = bool(e.get("pm_use_motor_lin", False))
        c["motor_linear_velocity"] = f32(e.get("pm_motor_lin_target_velocity", 0.0))
        c["motor_linear_max_impulse"] = f32(e.get("pm_motor_lin_max_impulse", 1.0))
        c["motor_angular"] = bool(e.get("pm_use_motor_ang", False))
        c["motor_angular_velocity"] = f32(e.get("pm_motor_ang_target_velocity", 0.0))
        c["motor_angular_max_impulse"] = f32(e.get("pm_motor_ang_max_impulse", 1.0))
        out.constraints.append(c)
    return out
