# SPDX-License-Identifier: MIT
"""Conformance runner for the reference's analytic rigid cases, through the
pm* driver.

The reference's conformance suite (conformance/v1: cases/*.json, the
runner in src/command_runner.cpp, the comparator compare.py) executes each
case through the public pm* command API and compares checkpoints against
its CUDA driver's results within per-case tolerances. This module does the
same for the three analytic rigid cases -- rigid-direct, constraint-breaking
and compound-weld-lifecycle -- against this project's driver:

- scenes restated from the runner's direct_scene / weld_scene
  (command_runner.cpp:230-305): the same box vertex and triangle order, body
  options with the defaults of RigidBodyOptions (authoring.hpp:127-143;
  mass 1, inertia from the mesh box when zero, friction 0.5, damping 0.05,
  speed limits 100, margin 0.005) and fixed welds with 8 solver iterations;
- the simulation set up as the gallery's CommandScene does
  (scene_builder_create.cpp.inc: contact capacity 65,536, rigid iterations
  10) and stepped one realtime tick at a time with contact events collected
  (scene_builder_output.cpp.inc:59-95);
- commands applied before the tick of their frame
  (command_runner.cpp:1122-1230, 2485-2510): impulses, kinematic targets,
  state replacement, constraint removal and re-addition;
- checkpoints in the runner's result layout (command_runner.cpp:1316-1350,
  2162-2410): rigid resources, constraint resources, canonical contacts and
  the invariants (momentum, joint errors, mechanical energy).

`compare` restates the comparator's rules (compare.py:248-453): every leaf
within abs + rel x max(|expected|, |actual|) of its tolerance class,
orientations by angle, counts/ids/flags exact, and contacts matched one to
one within each (body, collider) group. The backend's execution statistics
(dispatch counts and the like) are not physics and are not compared.
"""
from __future__ import annotations

import math

import numpy as np

from . import pm, scenes

# command_runner.cpp:230-242
_BOX_INDICES = [0, 1, 2, 0, 2, 3, 4, 6, 5, 4, 7, 6, 0, 4, 5, 0, 5, 1,
                1, 5, 6, 1, 6, 2, 2, 6, 7, 2, 7, 3, 3, 7, 4, 3, 4, 0]


def _box(half):
    x, y, z = (np.float32(h) for h in half)
    v = [(-x, -y, -z), (x, -y, -z), (x, y, -z), (-x, y, -z),
         (-x, -y, z), (x, -y, z), (x, y, z), (-x, y, z)]
    return np.array(v, np.float32), np.array(_BOX_INDICES, np.uint32)


class _Body:
    """RigidBodyOptions with the reference's defaults."""

    def __init__(self, name, mesh, position, motion=scenes.DYNAMIC, mass=1.0, inertia=(0.0, 0.0, 0.0),
                 linear_damping=0.05, angular_damping=0.05, orientation=(0.0, 0.0, 0.0, 1.0),
                 velocity=(0.0, 0.0, 0.0), friction=0.5, restitution=0.0, margin=0.005):
        self.name, self.mesh, self.position, self.motion = name, mesh, position, motion
        self.mass, self.inertia = mass, inertia
        self.linear_damping, self.angular_damping = linear_damping, angular_damping
        self.orientation, self.velocity = orientation, velocity
        self.friction, self.restitution, self.margin = friction, restitution, margin


def _direct_scene():
    meshes = [_box((0.25, 0.25, 0.25)), _box((3.0, 0.05, 3.0)), _box((0.2, 0.2, 0.2))]
    bodies = [_Body("dynamic-box", 0, (0.0, 2.0, 0.0), mass=2.0, inertia=(1.0 / 12.0,) * 3,
                    linear_damping=0.0, angular_damping=0.0),
              _Body("ground", 1, (0.0, -0.05, 0.0), motion=scenes.STATIC),
              _Body("kinematic-box", 2, (-1.0, 1.0, 0.0), motion=scenes.KINEMATIC)]
    return meshes, bodies, []


def _weld_scene(breaking):
    meshes = [_box((0.2, 0.2, 0.2))]
    count = 2 if breaking else 3
    bodies = [_Body(("break-a", "break-b")[k] if breaking else f"member-{k}", 0, (-0.4 + 0.4 * k, 1.0, 0.0),
                    linear_damping=0.0, angular_damping=0.0) for k in range(count)]
    joints = [("break-link" if breaking else f"weld-link-{k}", k, k + 1, 0.05 if breaking else 0.0)
              for k in range(count - 1)]
    return meshes, bodies, joints


SCENES = {"rigid-direct": lambda: _direct_scene(),
          "constraint-breaking": lambda: _weld_scene(True),
          "compound-weld-lifecycle": lambda: _weld_scene(False)}
ANCHOR_A, ANCHOR_B = (0.2, 0.0, 0.0), (-0.2, 0.0, 0.0)


def _scene(meshes, bodies, joints):
    b = scenes._Builder()
    ids = [b.mesh(v, i) for v, i in meshes]
    for body in bodies:
        inertia = tuple(body.inertia) if any(body.inertia) else (1.0, 1.0, 1.0)
        b.body(ids[body.mesh], body.motion, body.position, q=body.orientation, v=body.velocity, mass=body.mass,
               inertia=inertia, friction=body.friction, restitution=body.restitution, margin=body.margin,
               linear_damping=body.linear_damping, angular_damping=body.angular_damping)
    for joint in joints:
        if isinstance(joint, dict):  # an authored constraint (glb.load_glb_scene)
            k = b.joint(joint["type"], joint["body_a"], joint["body_b"], joint["anchor_a"], joint["anchor_b"],
                        disable_collisions=joint["disable_collisions"], iterations=joint["solver_iterations"])
            o = b.joints[k]
            o["frame_a"], o["frame_b"] = joint["frame_a"], joint["frame_b"]
            o["enabled"] = 1 if joint["enabled"] else 0
            o["breaking_threshold"] = joint["breaking_threshold"]
            for f in ("lin_limit_axes", "ang_limit_axes", "lin_spring_axes", "ang_spring_axes", "lin_lower",
                      "lin_upper", "ang_lower", "ang_upper", "lin_stiffness", "lin_damping", "ang_stiffness",
                      "ang_damping", "motor_linear_velocity", "motor_linear_max_impulse", "motor_angular_velocity",
                      "motor_angular_max_impulse"):
                o[f] = joint[f]
            o["motor_linear"] = 1 if joint["motor_linear"] else 0
            o["motor_angular"] = 1 if joint["motor_angular"] else 0
            continue
        name, a, c, threshold = joint
        k = b.joint(scenes.FIXED, a, c, ANCHOR_A, ANCHOR_B, disable_collisions=True, iterations=8)
        b.joints[k]["breaking_threshold"] = threshold
    return b.build("conformance", 8, scenes.REALTIME)


def glb_case_scene(gs):
    """(meshes, bodies, joints, body ids, constraint ids) of an authored scene
    (glb.load_glb_scene) as the conformance runner builds it
    (command_runner.cpp:1063-1095; scene_builder.cpp:393-433): each body's
    collision meshes -- its proxy's when it has one, else its render
    primitives -- merged into one geometry (shared by bodies with the same
    meshes), resource ids "rigid/<source name>/<index>" and
    "constraint/<name>/<index>"."""
    meshes, keys, bodies = [], {}, []
    for k, body in enumerate(gs.bodies):
        proxy = bool(body["collision_mesh_indices"])
        parts = body["collision_mesh_indices"] if proxy else body["mesh_indices"]
        key = (proxy, tuple(parts))
        if key not in keys:
            src = gs.collision_meshes if proxy else gs.meshes
            verts, idx, base = [], [], 0
            for m in parts:
                v, i = src[m]
                verts.append(v)
                idx.append(i + base)
                base += len(v)
            keys[key] = len(meshes)
            meshes.append((np.concatenate(verts).astype(np.float32), np.concatenate(idx).astype(np.uint32)))
        bodies.append(_Body(f"rigid/{body['source_name'] or body['name']}/{k}", keys[key],
                            tuple(float(x) for x in body["position"]), motion=body["motion"],
                            mass=float(body["mass"]), inertia=(0.0, 0.0, 0.0),
                            linear_damping=float(body["linear_damping"]),
                            angular_damping=float(body["angular_damping"]),
                            orientation=tuple(float(x) for x in body["orientation"]),
                            velocity=tuple(float(x) for x in body["velocity"]),
                            friction=float(body["friction"]), restitution=float(body["restitution"]),
                            margin=float(body["margin"])))
    joints = [dict(c) for c in gs.constraints]
    jnames = [f"constraint/{c['name']}/{k}" for k, c in enumerate(gs.constraints)]
    return meshes, bodies, joints, [b.name for b in bodies], jnames


def _rotate(q, p):
    x, y, z, w = (float(v) for v in q)
    px, py, pz = (float(v) for v in p)
    # q * (p, 0) * conj(q)
    tx = w * px + y * pz - z * py
    ty = w * py - x * pz + z * px
    tz = w * pz + x * py - y * px
    tw = -x * px - y * py - z * pz
    return (np.float32(tw * -x + tx * w + ty * -z - tz * -y),
            np.float32(tw * -y - tx * -z + ty * w + tz * -x),
            np.float32(tw * -z + tx * -y - ty * -x + tz * w))


def _angle(a, b):
    na = math.sqrt(sum(float(v) ** 2 for v in a))
    nb = math.sqrt(sum(float(v) ** 2 for v in b))
    if not (na > 0.0 and nb > 0.0):
        return 0.0
    d = abs(sum(float(x) * float(y) for x, y in zip(a, b)) / (na * nb))
    return 2.0 * math.acos(min(1.0, max(0.0, d)))


def _vec(v):
    return [float(x) for x in v]


def run_case(case, with_quality=False, authored=None):
    """Runs one case through the pm* driver; returns the result document
    {case_id, checkpoints: [...]} in the runner's layout. Analytic cases build
    their scene here; an integrated_glb case takes `authored`, the scene its
    GLB loads to (glb.load_glb_scene). with_quality adds the runner's
    rigid_quality invariants (joint anchor and angle errors, mechanical
    energy; analytic cases), which the recorded CUDA results lack."""
    cid = case["id"]
    if authored is not None:
        meshes, bodies, joints, names, jnames = glb_case_scene(authored)
        with_quality = False
    else:
        meshes, bodies, joints = SCENES[cid]()
        names = [body.name for body in bodies]
        jnames = [j[0] for j in joints]
    scene = _scene(meshes, bodies, joints)
    world = case["world"]
    gravity = tuple(float(g) for g in world["gravity"])
    infos = {i: {"mass": float(body.mass), "inertiaDiagonal": tuple(float(v) for v in body.inertia)}
             for i, body in enumerate(bodies)}
    session = pm.RigidSession(scene, iterations=10, contact_capacity=65536, body_infos=infos)
    present = [True] * len(joints)
    flags = {"generation_changed": False, "constraints_rebuilt": False}
    profile = case["tolerances"]["profile"]
    states = np.zeros(len(bodies), scenes.STATE_DTYPE)
    for i, body in enumerate(bodies):
        states[i]["x"] = body.position
        states[i]["q"] = body.orientation
        states[i]["v"] = body.velocity
    cstates = [(True, False, 0.0)] * len(joints)
    events = np.zeros(0, pm.PM_EVENT_DTYPE)

    def checkpoint(frame):
        res = []
        for i, name in enumerate(names):
            s = states[i]
            res.append({"angular_velocity": _vec(s["w"]), "id": name, "linear_velocity": _vec(s["v"]),
                        "orientation": _vec(s["q"]), "position": _vec(s["x"]), "present": True,
                        "tolerance_class": profile, "type": "rigid_body"})
        for k, name in enumerate(jnames):
            on = present[k]
            en, br, ap = cstates[k]
            res.append({"applied_impulse": float(ap) if on else 0.0, "broken": bool(on and br),
                        "enabled": bool(on and en), "id": name, "present": on,
                        "tolerance_class": "constraint_contact", "type": "rigid_constraint"})
        rigid = sorted(events, key=lambda e: (int(e["first"]), int(e["second"]), float(e["position"][0]),
                                              float(e["position"][1]), float(e["position"][2])))
        contacts = [{"body": names[int(e["first"])] if int(e["first"]) < len(names) else "unknown",
                     "collider": names[int(e["second"])] if int(e["second"]) < len(names) else "unknown",
                     "friction_impulse": _vec(e["frictionImpulse"]), "normal": _vec(e["normal"]),
                     "normal_impulse": float(e["normalImpulse"]), "penetration": float(e["penetration"]),
                     "position": _vec(e["position"])} for e in rigid[:256]]
        momentum = [np.float32(0.0)] * 3
        energy = 0.0
        for i, body in enumerate(bodies):
            if body.motion != scenes.DYNAMIC:
                continue
            v = states[i]["v"]
            momentum = [np.float32(momentum[k] + np.float32(body.mass * float(v[k]))) for k in range(3)]
            w = states[i]["w"]
            lin2 = sum(float(x) * float(x) for x in v)
            ang = 0.5 * sum(body.inertia[k] * float(w[k]) * float(w[k]) for k in range(3))
            pot = -body.mass * sum(gravity[k] * float(states[i]["x"][k]) for k in range(3))
            energy += 0.5 * body.mass * lin2 + ang + pot
        jpos = jang = 0.0
        for k, joint in enumerate(joints if with_quality else []):
            _, a, c, _ = joint
            if not present[k]:
                continue
            pa = [float(states[a]["x"][m]) + float(r) for m, r in enumerate(_rotate(states[a]["q"], ANCHOR_A))]
            pc = [float(states[c]["x"][m]) + float(r) for m, r in enumerate(_rotate(states[c]["q"], ANCHOR_B))]
            jpos = max(jpos, math.sqrt(sum((x - y) ** 2 for x, y in zip(pa, pc))))
            jang = max(jang, _angle(states[a]["q"], states[c]["q"]))
        invariants = {"cloth_count": 0, "combined_momentum": [float(m) for m in momentum], "complete_state": True,
                      "constraint_count": len(joints), "constraints_rebuilt": flags["constraints_rebuilt"],
                      "element_count": len(bodies), "finite": bool(np.isfinite(states["x"]).all()),
                      "fluid_count": 0, "generation_changed": flags["generation_changed"], "particle_count": 0,
                      "rigid_body_count": len(bodies), "rope_count": 0, "smoke_count": 0, "soft_body_count": 0}
        if with_quality:
            invariants["rigid_quality"] = {"maximum_joint_angle_error_rad": jang,
                                           "maximum_joint_position_error_m": jpos,
                                           "mechanical_energy_j": energy}
        return {"contacts": {"fluid_contact_count": 0, "fluid_contacts": [], "rigid_contact_count": len(rigid),
                             "rigid_contacts": contacts},
                "frame": frame, "invariants": invariants, "resources": res}

    out = []
    wanted = set(case["checkpoints"])
    try:
        if 0 in wanted:
            out.append(checkpoint(0))
        for frame in range(int(world["frames"])):
            inputs, targets = [], {}
            for cmd in case.get("commands", []):
                if cmd["frame"] != frame:
                    continue
                op, value = cmd["operation"], cmd.get("value")
                if op == "apply_impulse":
                    inputs.append((names.index(cmd["target"]), (0, 0, 0), (0, 0, 0), tuple(value), (0, 0, 0)))
                elif op == "set_kinematic_target":
                    i = names.index(cmd["target"])
                    t = np.zeros((), scenes.STATE_DTYPE)
                    t["x"], t["q"] = tuple(value), (0.0, 0.0, 0.0, 1.0)
                    targets[i] = t
                elif op == "replace_body":
                    i = names.index(cmd["target"])
                    r = np.zeros((), scenes.STATE_DTYPE)
                    r["x"], r["q"] = tuple(value), (0.0, 0.0, 0.0, 1.0)
                    pm.check(session.set_states(i, [r]), "replace body")
                    flags["generation_changed"] = True
                elif op == "set_constraints_enabled":
                    # every constraint rewritten with its enabled (active)
                    # option set to the value (command_runner.cpp:1221-1233)
                    pm.check(session.write_constraints([bool(value[0])] * len(present)), op)
                elif op in ("remove_constraints", "add_constraints"):
                    active = op == "add_constraints"
                    present[:] = [active] * len(present)
                    pm.check(session.write_constraints(present), op)
                    flags["constraints_rebuilt"] = flags["constraints_rebuilt"] or active
                else:
                    raise ValueError(f"unsupported command {op}")
            pm.check(session.step(gravity=gravity, inputs=inputs or None, targets=targets or None, events=True),
                     f"step {frame + 1}")
            states = session.states()
            (_, _, _), events = session.contact_events()
            cs = session.copy_constraint_states()
            cstates = [(bool(c["enabled"]), bool(c["broken"]), float(c["applied"])) for c in cs]
            if frame + 1 in wanted:
                out.append(checkpoint(frame + 1))
    finally:
        session.close()
    return {"case_id": cid, "checkpoints": out}


# ---------------------------------------------------------------- comparison
EXACT = {"case_id", "count", "enabled", "frame", "id", "type", "present", "broken", "finite",
         "complete_state", "generation_changed", "constraints_rebuilt", "tolerance_class"}


def _tolerance(case, cls, path):
    values = case["tolerances"]["values"]
    leaf = path.rsplit(".", 1)[-1].split("[", 1)[0]
    if leaf == "orientation":
        sel = values["quaternion_angular"]
    else:
        prof = values.get(cls) or values[case["tolerances"]["profile"]]
        q = "velocity" if any(k in leaf for k in ("velocity", "speed", "momentum", "vorticity")) else "position"
        sel = prof[q]
    return float(sel["abs"]), float(sel["rel"])


def _exact(key, value):
    return key in EXACT or key.endswith("_count") or isinstance(value, (bool, str)) or (
        isinstance(value, int) and not isinstance(value, bool)) or value is None


def compare(case, expected, actual, kinds=False):
    """Differences between two checkpoint lists (frame-aligned), as
    (path, message) pairs -- (path, message, kind) with kinds=True, kind
    "exact" (ids, flags, counts, types), "numeric" (a value outside its
    tolerance) or "contact" (a contact with no match within tolerance);
    empty when the result conforms."""
    fails = []

    def cmp(e, a, path, cls, exact):
        num = isinstance(e, (int, float)) and not isinstance(e, bool) and \
            isinstance(a, (int, float)) and not isinstance(a, bool)
        if type(e) is not type(a) and not num:
            fails.append((path, f"type {type(e).__name__} vs {type(a).__name__}", "exact"))
            return
        if isinstance(e, dict):
            child = str(e.get("tolerance_class", cls))
            for k in sorted(set(e) | set(a)):
                if k not in a or k not in e:
                    fails.append((f"{path}.{k}", "missing" if k not in a else "unexpected", "exact"))
                    continue
                cmp(e[k], a[k], f"{path}.{k}", child, exact or _exact(k, e[k]))
            return
        if isinstance(e, list):
            if path.endswith(".orientation"):
                ab, rel = _tolerance(case, cls, path)
                err = _angle(e, a)
                if err > ab + rel:
                    fails.append((path, f"angle {err:.3g} > {ab + rel:.3g}", "numeric"))
                return
            if len(e) != len(a):
                fails.append((path, f"length {len(e)} vs {len(a)}", "exact"))
                return
            if path.endswith(".rigid_contacts"):
                match_contacts(e, a, path, cls)
                return
            for k, (x, y) in enumerate(zip(e, a)):
                cmp(x, y, f"{path}[{k}]", cls, exact)
            return
        if num and not exact:
            ab, rel = _tolerance(case, cls, path)
            lim = ab + rel * max(abs(float(e)), abs(float(a)))
            if abs(float(e) - float(a)) > lim:
                fails.append((path, f"|{e} - {a}| > {lim:.3g}", "numeric"))
            return
        if e != a:
            fails.append((path, f"{e!r} != {a!r}", "exact"))

    def match_contacts(e, a, path, cls):
        # one-to-one matching within (body, collider) groups, every field of a
        # matched pair within its tolerance (augmenting paths)
        def ok(x, y):
            before = len(fails)
            cmp(x, y, path + "[?]", cls, False)
            good = len(fails) == before
            del fails[before:]
            return good
        edges = [[j for j, y in enumerate(a) if (y["body"], y["collider"]) == (x["body"], x["collider"]) and ok(x, y)]
                 for x in e]
        owner = {}

        def augment(i, seen):
            for j in edges[i]:
                if j in seen:
                    continue
                seen.add(j)
                if j not in owner or augment(owner[j], seen):
                    owner[j] = i
                    return True
            return False
        for i in range(len(e)):
            if not augment(i, set()):
                fails.append((f"{path}[{i}]", "no one-to-one contact match within tolerance", "contact"))

    profile = case["tolerances"]["profile"]
    frames = {cp["frame"]: cp for cp in actual}
    for cp in expected:
        got = frames.get(cp["frame"])
        if got is None:
            fails.append((f"frame {cp['frame']}", "missing checkpoint", "exact"))
            continue
        cmp(cp, got, f"$[frame {cp['frame']}]", profile, False)
    return fails if kinds else [(p, m) for p, m, _ in fails]
