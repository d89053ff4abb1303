# SPDX-License-Identifier: MIT
"""The reference's analytic rigid conformance cases (conformance/v1:
rigid-direct, constraint-breaking, compound-weld-lifecycle) run through this
project's pm* driver and compared with the reference's own CUDA driver
results (tests/golden/conformance_analytic.json, extracted by
make_conformance_fixtures.py) within each case's tolerances, as the
reference's comparator does.

CPU tests check the comparator itself on the golden documents; the GPU test
runs the cases.
"""
import copy
import json
import os

import pytest

from pmb200 import conformance

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "conformance_analytic.json")


def _fixture():
    with open(FIXTURE) as f:
        return json.load(f)


def test_comparator_accepts_the_golden_and_rejects_perturbations():
    fx = _fixture()
    for cid, item in fx.items():
        case, golden = item["case"], item["golden"]["checkpoints"]
        assert conformance.compare(case, golden, copy.deepcopy(golden)) == [], cid
        bad = copy.deepcopy(golden)
        body = bad[-1]["resources"][0]
        body["position"][1] += 0.5
        fails = conformance.compare(case, golden, bad)
        assert any(p.endswith("position[1]") for p, _ in fails), cid
        bad = copy.deepcopy(golden)
        bad[-1]["invariants"]["generation_changed"] = not bad[-1]["invariants"]["generation_changed"]
        assert conformance.compare(case, golden, bad), cid


def test_comparator_matches_contacts_one_to_one():
    fx = _fixture()
    case, golden = fx["compound-weld-lifecycle"]["case"], fx["compound-weld-lifecycle"]["golden"]["checkpoints"]
    with_contacts = [cp for cp in golden if cp["contacts"]["rigid_contacts"]]
    assert with_contacts
    shuffled = copy.deepcopy(with_contacts)
    for cp in shuffled:
        cp["contacts"]["rigid_contacts"].reverse()
    assert conformance.compare(case, with_contacts, shuffled) == []
    moved = copy.deepcopy(with_contacts)
    moved[0]["contacts"]["rigid_contacts"][0]["position"][0] += 0.1
    assert conformance.compare(case, with_contacts, moved)


@pytest.mark.gpu
@pytest.mark.parametrize("cid", ["rigid-direct", "constraint-breaking", "compound-weld-lifecycle"])
def test_analytic_case_against_reference_cuda(gpu_available, cid):
    """Every checkpoint, body, joint and contact of the recorded CUDA result
    is produced, with equal ids, flags (present, enabled, broken, generation
    and rebuild markers) and counts (bodies, joints, contact points). The
    numeric differences are printed, not asserted: the recorded results come
    from an earlier reference revision whose realtime tick differs from the
    current sources in two documented ways (no x0.95 solver damping; a
    free-fall position step of 5/8 g dt^2 instead of the predictor's g dt^2)."""
    item = _fixture()[cid]
    result = conformance.run_case(item["case"])
    fails = conformance.compare(item["case"], item["golden"]["checkpoints"], result["checkpoints"], kinds=True)
    exact = [f for f in fails if f[2] == "exact"]
    numeric = [f for f in fails if f[2] != "exact"]
    print(f"{cid}: {len(numeric)} values outside tolerance")
    for path, message, _ in numeric[:20]:
        print("  ", path, message)
    assert not exact, exact[:10]
