#!/usr/bin/env python3
# SPDX-License-Identifier: MIT
"""Extracts the reference's eight authored-scene (integrated_glb) rigid
constraint cases into conformance_glb.npz (test fixture): for each case the
case file, its CUDA driver's recorded result, and the scene its GLB loads to
through pmb200.glb.load_glb_scene (meshes as arrays, bodies and constraints
as JSON), plus the GLB's SHA-256 so a check against the checkout can tell
whether the asset changed.

Source: the reference checkout's conformance/v1/cases/constraint-*.json,
conformance/v1/golden/cuda/constraint-*.json and the GLBs they name under
examples/assets. Kept per checkpoint: frame, resources, contacts and
invariants (not the backend's execution statistics).

Usage: python tests/golden/make_conformance_glb.py /root/reference
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "parallel-mater_b200"))
from pmb200 import glb  # noqa: E402

CASES = ["constraint-fixed", "constraint-generic", "constraint-generic-spring", "constraint-hinge",
         "constraint-motor", "constraint-piston", "constraint-point", "constraint-slider"]
KEEP = ("frame", "resources", "contacts", "invariants")


def jsonable(value):
    if isinstance(value, dict):
        return {k: jsonable(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [jsonable(v) for v in value]
    if isinstance(value, np.ndarray):
        return [jsonable(v) for v in value.tolist()]
    if isinstance(value, (np.floating,)):
        return float(value)
    if isinstance(value, (np.integer,)):
        return int(value)
    if isinstance(value, (np.bool_,)):
        return bool(value)
    return value


def main(reference):
    root = os.path.join(reference, "conformance", "v1")
    arrays, meta = {}, {}
    for cid in CASES:
        with open(os.path.join(root, "cases", cid + ".json")) as f:
            case = json.load(f)
        with open(os.path.join(root, "golden", "cuda", cid + ".json")) as f:
            golden = json.load(f)
        asset = case["resources"][0]["definition"]["path"]
        with open(os.path.join(reference, asset), "rb") as f:
            data = f.read()
        scene = glb.load_glb_scene(data)
        for kind, meshes in (("mesh", scene.meshes), ("collision", scene.collision_meshes)):
            for k, (v, i) in enumerate(meshes):
                arrays[f"{cid}/{kind}{k}/v"] = np.asarray(v, np.float32)
                arrays[f"{cid}/{kind}{k}/i"] = np.asarray(i, np.uint32)
        meta[cid] = {
            "asset": asset, "sha256": hashlib.sha256(data).hexdigest(),
            "meshes": len(scene.meshes), "collision_meshes": len(scene.collision_meshes),
            "bodies": jsonable(scene.bodies), "constraints": jsonable(scene.constraints),
            "case": {k: case[k] for k in ("id", "kind", "world", "checkpoints", "commands", "tolerances",
                                          "comparison") if k in case},
            "golden": {"backend": golden.get("backend"),
                       "checkpoints": [{k: cp[k] for k in KEEP if k in cp} for cp in golden["checkpoints"]]},
        }
    arrays["meta"] = np.frombuffer(json.dumps(meta, sort_keys=True).encode(), np.uint8)
    path = os.path.join(HERE, "conformance_glb.npz")
    np.savez_compressed(path, **arrays)
    print(path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PMB_REFERENCE_ROOT", "/root/reference"))
