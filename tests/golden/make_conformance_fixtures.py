#!/usr/bin/env python3
# SPDX-License-Identifier: MIT
"""Extracts the reference's conformance inputs and CUDA results for the
analytic rigid cases into conformance_analytic.json (test fixture).

Source: the reference checkout's conformance/v1/cases/<id>.json (the case:
world, commands, checkpoints, tolerances) and conformance/v1/golden/cuda/
<id>.json (its CUDA driver's result). Kept per checkpoint: frame, resources,
contacts and invariants; dropped: the backend's execution statistics
(realtime_work, step), which describe how a driver ran, not the physics.

Usage: python tests/golden/make_conformance_fixtures.py /root/reference
"""
import json
import os
import sys

CASES = ["rigid-direct", "constraint-breaking", "compound-weld-lifecycle"]
KEEP = ("frame", "resources", "contacts", "invariants")


def main(reference):
    root = os.path.join(reference, "conformance", "v1")
    out = {}
    for cid in CASES:
        with open(os.path.join(root, "cases", cid + ".json")) as f:
            case = json.load(f)
        with open(os.path.join(root, "golden", "cuda", cid + ".json")) as f:
            golden = json.load(f)
        out[cid] = {
            "case": {k: case[k] for k in ("id", "kind", "world", "checkpoints", "commands", "tolerances",
                                          "comparison") if k in case},
            "golden": {"backend": golden.get("backend"),
                       "checkpoints": [{k: cp[k] for k in KEEP if k in cp} for cp in golden["checkpoints"]]},
        }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "conformance_analytic.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print(path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PMB_REFERENCE_ROOT", "/root/reference"))
