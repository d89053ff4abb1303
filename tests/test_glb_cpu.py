# SPDX-License-Identifier: MIT
"""The authored-scene loader (pmb200.glb) on small GLBs built here: the
container and accessor reading, the loader's bounds re-centring and shared
meshes, the constraint frames (Blender's local Z restored, expressed in each
body's frame), option defaults, and its rejections."""
import json
import math
import struct

import numpy as np
import pytest

from pmb200 import glb, scenes

# A unit cube offset from its node origin: x in [1, 3], y in [0, 1], z in [-1, 1].
CUBE = np.array([[x, y, z] for z in (-1.0, 1.0) for y in (0.0, 1.0) for x in (1.0, 3.0)], np.float32)
TRIS = np.array([0, 2, 1, 1, 2, 3, 4, 5, 6, 5, 7, 6, 0, 1, 4, 1, 5, 4,
                 2, 6, 3, 3, 6, 7, 0, 4, 2, 2, 4, 6, 1, 3, 5, 3, 7, 5], np.uint16)


def make_glb(nodes, mesh_count=1):
    blob = CUBE.tobytes() + TRIS.tobytes()
    doc = {
        "asset": {"version": "2.0"},
        "buffers": [{"byteLength": len(blob)}],
        "bufferViews": [{"buffer": 0, "byteOffset": 0, "byteLength": CUBE.nbytes},
                        {"buffer": 0, "byteOffset": CUBE.nbytes, "byteLength": TRIS.nbytes}],
        "accessors": [{"bufferView": 0, "componentType": 5126, "count": 8, "type": "VEC3"},
                      {"bufferView": 1, "componentType": 5123, "count": 36, "type": "SCALAR"}],
        "meshes": [{"primitives": [{"attributes": {"POSITION": 0}, "indices": 1}]} for _ in range(mesh_count)],
        "nodes": nodes,
        "scenes": [{"nodes": list(range(len(nodes)))}],
    }
    js = json.dumps(doc).encode()
    js += b" " * (-len(js) % 4)
    blob += b"\0" * (-len(blob) % 4)
    body = struct.pack("<I4s", len(js), b"JSON") + js + struct.pack("<I4s", len(blob), b"BIN\0") + blob
    return struct.pack("<4sII", b"glTF", 2, 12 + len(body)) + body


def body_node(name, motion="dynamic", mesh=0, translation=(0.0, 0.0, 0.0), rotation=None, scale=None, **extras):
    e = {"pm_schema": 2, "pm_system": "rigid_body", "pm_name": name, "pm_motion": motion, "pm_mass": 2.0}
    e.update(extras)
    n = {"name": name, "mesh": mesh, "translation": list(translation), "extras": e}
    if rotation is not None:
        n["rotation"] = list(rotation)
    if scale is not None:
        n["scale"] = list(scale)
    return n


def test_bodies_are_recentred_on_their_bounds():
    s = math.sqrt(0.5)
    q = (0.0, 0.0, s, s)  # 90 degrees about z
    data = make_glb([body_node("Box", translation=(10.0, 0.0, 0.0), rotation=q, pm_friction=0.25,
                               pm_initial_velocity_x=1.5),
                     body_node("Ground", motion="static", scale=(2.0, 1.0, 1.0))], mesh_count=2)
    g = glb.load_glb_scene(data)
    assert len(g.bodies) == 2 and len(g.meshes) == 2
    box, ground = g.bodies
    # local bounds centre (2, 0.5, 0) rotated by q: (-0.5, 2, 0)
    assert np.allclose(box["position"], (9.5, 2.0, 0.0), atol=1e-6)
    v = g.meshes[box["mesh_indices"][0]][0]
    assert np.allclose(v.min(axis=0), (-1.0, -0.5, -1.0)) and np.allclose(v.max(axis=0), (1.0, 0.5, 1.0))
    assert box["motion"] == scenes.DYNAMIC and np.isclose(box["mass"], 2.0)
    assert np.isclose(box["friction"], 0.25) and np.isclose(box["linear_damping"], 0.05)
    assert np.allclose(box["velocity"], (1.5, 0.0, 0.0))
    # the ground's mesh is scaled by its node scale before centring
    vg = g.meshes[ground["mesh_indices"][0]][0]
    assert np.allclose(vg.max(axis=0) - vg.min(axis=0), (4.0, 1.0, 2.0))
    assert np.allclose(ground["position"], (4.0, 0.5, 0.0))


def test_bodies_sharing_a_mesh_share_its_geometry():
    data = make_glb([body_node("A", translation=(0.0, 0.0, 0.0)), body_node("B", translation=(5.0, 0.0, 0.0))])
    g = glb.load_glb_scene(data)
    assert len(g.meshes) == 1
    assert g.bodies[0]["mesh_indices"] == g.bodies[1]["mesh_indices"] == [0]
    assert np.allclose(g.bodies[1]["position"] - g.bodies[0]["position"], (5.0, 0.0, 0.0))


def test_constraint_frames_are_in_each_bodys_frame():
    s = math.sqrt(0.5)
    nodes = [body_node("A", translation=(0.0, 0.0, 0.0)), body_node("B", translation=(0.0, 3.0, 0.0)),
             {"name": "Hinge", "translation": [2.0, 2.0, 0.0], "rotation": [0.0, 0.0, 0.0, 1.0],
              "extras": {"pm_schema": 2, "pm_system": "rigid_constraint", "pm_name": "Hinge",
                         "pm_constraint_type": "hinge", "pm_body_a": "A", "pm_body_b": "B",
                         "pm_use_limit_ang_z": True, "pm_limit_ang_z_lower": -0.5, "pm_limit_ang_z_upper": 0.5,
                         "pm_solver_iterations": 12}}]
    g = glb.load_glb_scene(make_glb(nodes))
    (c,) = g.constraints
    assert c["type"] == scenes.HINGE and c["body_a"] == 0 and c["body_b"] == 1
    a, b = g.bodies
    for side, body in (("a", a), ("b", b)):
        world = body["position"] + glb.rotate(body["orientation"], c[f"anchor_{side}"])
        assert np.allclose(world, (2.0, 2.0, 0.0), atol=1e-6), side
        frame = glb.qmul(body["orientation"], c[f"frame_{side}"])
        assert np.allclose(np.abs(frame), (s, 0.0, 0.0, s), atol=1e-6), side  # -90 degrees about x
    assert c["ang_limit_axes"] == 4 and np.isclose(c["ang_lower"][2], -0.5) and c["lin_limit_axes"] == 0
    assert c["solver_iterations"] == 12 and c["enabled"] and c["disable_collisions"]
    assert np.isclose(c["motor_linear_max_impulse"], 1.0)


def test_loader_rejections():
    with pytest.raises(glb.GlbError):
        glb.load_glb_scene(b"not a glb at all....")
    with pytest.raises(glb.GlbError, match="pm_motion"):
        n = body_node("A")
        del n["extras"]["pm_motion"]
        glb.load_glb_scene(make_glb([n]))
    with pytest.raises(glb.GlbError, match="require pm_mass"):
        n = body_node("A")
        del n["extras"]["pm_mass"]
        glb.load_glb_scene(make_glb([n]))
    with pytest.raises(glb.GlbError, match="scale"):
        glb.load_glb_scene(make_glb([body_node("A", scale=(0.0, 1.0, 1.0))]))
    with pytest.raises(glb.GlbError, match="missing, ambiguous"):
        nodes = [body_node("A"), body_node("A", translation=(3.0, 0.0, 0.0)),
                 {"name": "J", "extras": {"pm_schema": 2, "pm_system": "rigid_constraint",
                                          "pm_constraint_type": "point", "pm_body_a": "A", "pm_body_b": "A"}}]
        glb.load_glb_scene(make_glb(nodes))
    with pytest.raises(glb.GlbError, match="solver iterations"):
        nodes = [body_node("A"), body_node("B", translation=(3.0, 0.0, 0.0)),
                 {"name": "J", "extras": {"pm_schema": 2, "pm_system": "rigid_constraint",
                                          "pm_constraint_type": "point", "pm_body_a": "A", "pm_body_b": "B",
                                          "pm_solver_iterations": 65}}]
        glb.load_glb_scene(make_glb(nodes))
