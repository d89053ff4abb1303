# SPDX-License-Identifier: MIT
"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerances: pair sets, manifold point counts, colourings and island roots are
integer/index data and must match exactly; so must the poses: the tick
evaluates every expression in the oracle's order from IEEE-exact operations
(no contraction, IEEE division and square root, arctangent and cotangent from
series of basic operations), so positions, orientations and velocities are
compared bit for bit. Core math is compared with the golden vectors at rel
2e-5 / abs 2e-6 (the reference fixture validator's default tolerance).
"""
import json
import os

import numpy as np
import pytest

from pmb200 import core, scenes
import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "avbd_core_vectors.json")


def _num(v):
    if isinstance(v, str):
        return {"nan": np.nan, "inf": np.inf, "-inf": -np.inf}[v]
    return v


def _arr(rows):
    return np.array([[_num(x) for x in r] for r in rows], np.float32)


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _close(a, b, rel=2e-5, ab=2e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    ok = np.isclose(a, b, rtol=rel, atol=ab) | both_nan | (a == b)
    return ok


def test_device_block_solve_matches_golden(gpu_available, golden):
    blocks = golden["blocks"]
    inp = np.array([[_num(x) for x in b["h"]] + [_num(x) for x in b["g"]] for b in blocks], np.float32)
    out = core.math_eval(0, inp)
    solved = np.array([b["solved"] for b in blocks])
    assert np.array_equal(out[:, 6].astype(int), solved)
    ref = _arr([b["delta"] for b in blocks])
    ok = _close(out[solved == 1, :6], ref[solved == 1])
    # Ill-conditioned fixtures are validated by backward error in the
    # reference; compare componentwise only against the oracle there.
    orc = np.array([O.block_solve(i[:21], i[21:])[1] for i in inp])
    assert np.array_equal(out[:, :6], orc), "device block solve differs from the oracle bit pattern"
    assert ok.mean() > 0.97


def test_device_duals_contacts_rows_match_golden(gpu_available, golden):
    for kind, key in ((1, "duals"), (2, "contacts"), (3, "rows")):
        inp = _arr([e["in"] for e in golden[key]])
        ref = _arr([e["out"] for e in golden[key]])
        out = core.math_eval(kind, inp)
        assert _close(out, ref, rel=2e-5, ab=2e-6).all(), key


def _step_both(scene, frames, check_every=1):
    w = core.World(scene)
    o = O.OracleWorld(scene)
    worst = 0.0
    for f in range(frames):
        sg = w.step()
        so = o.step()
        assert sg["status"] == 0, core.status_names(int(sg["status"]))
        assert sg["candidate_pairs"] == so["candidate_pairs"], f
        assert np.array_equal(w.candidate_pairs(), o.candidate_pairs()), f
        cg, ng, kg = w.manifolds()
        co, no, ko = o.manifolds()
        assert np.array_equal(cg, co), f
        assert np.array_equal(ng, no), f
        colg, parg = w.graph()
        colo, paro = o.graph()
        dyn = scene.bodies["motion"] == scenes.DYNAMIC
        assert np.array_equal(colg[dyn], colo[dyn]), f
        assert np.array_equal(parg, paro), f
        assert sg["colors"] == so["colors"] and sg["islands"] == so["islands"]
        xg, xo = w.states(), o.states()
        err = max(np.abs(xg["x"] - xo["x"]).max(), np.abs(xg["v"] - xo["v"]).max(),
                  np.abs(xg["q"] - xo["q"]).max())
        worst = max(worst, err)
        assert np.array_equal(xg.view(np.uint8), xo.view(np.uint8)), (f, err)
    return w, o, worst


def test_pyramid_matches_oracle_legacy(gpu_available):
    _, _, worst = _step_both(scenes.pyramid(), 30)
    print("pyramid legacy worst |gpu-oracle| =", worst)


def test_pyramid_matches_oracle_realtime(gpu_available):
    s = scenes.pyramid(profile=scenes.REALTIME)
    _, _, worst = _step_both(s, 20)
    print("pyramid realtime worst |gpu-oracle| =", worst)


def test_small_pile_matches_oracle(gpu_available):
    s = scenes.box_pile((6, 4, 6), seed=7, spacing=1.6)
    _, _, worst = _step_both(s, 60)
    print("pile worst |gpu-oracle| =", worst)


def test_joint_zoo_matches_oracle(gpu_available):
    """All eight joint types with limits, springs, motors, breaking and hinge
    projection: poses equal the oracle's bits, joint flags and row counts
    equal every tick."""
    s = scenes.joint_zoo()
    w = core.World(s)
    o = O.OracleWorld(s)
    worst = 0.0
    for f in range(60):
        sg, so = w.step(), o.step()
        assert sg["status"] == 0, core.status_names(int(sg["status"]))
        assert sg["colors"] == so["colors"] and sg["islands"] == so["islands"], f
        fg, ag, cg = w.joints()
        fo, ao, co = o.joints()
        assert np.array_equal(fg, fo) and np.array_equal(cg, co), f
        xg, xo = w.states(), o.states()
        err = max(np.abs(xg["x"] - xo["x"]).max(), np.abs(xg["q"] - xo["q"]).max(),
                  np.abs(xg["v"] - xo["v"]).max())
        worst = max(worst, err)
        assert np.array_equal(xg.view(np.uint8), xo.view(np.uint8)), (f, err)
    print("joint zoo worst |gpu-oracle| =", worst)


def test_fixed_collision_groups_match_oracle(gpu_available):
    """Fixed collision groups on the GPU: the candidate pairs equal the
    oracle's every tick (no pair inside a group), and poses follow it."""
    s = scenes.welded_groups()
    w = core.World(s)
    o = O.OracleWorld(s)
    for f in range(60):
        sg, so = w.step(), o.step()
        assert sg["status"] == 0 and so["status"] == 0
        assert np.array_equal(w.candidate_pairs(), o.candidate_pairs()), f
        assert sg["contacts"] == so["contacts"], f
        xg, xo = w.states(), o.states()
        err = max(np.abs(xg[k] - xo[k]).max() for k in ("x", "q", "v"))
        assert err < 1e-4, (f, err)
    codes = set(int(c) for c in w.candidate_pairs())
    assert 1 * s.n + 3 not in codes and 5 * s.n + 6 not in codes


@pytest.mark.parametrize("margin", [0.04, 0.005])
def test_triangle_mesh_path_matches_oracle(gpu_available, margin):
    """The triangle-mesh narrowphase on the GPU (concave trough and L bodies,
    a 64-triangle capsule; with 5 mm margins the falls take the swept
    ranges): candidate pairs, contact counts and manifolds equal the oracle's
    every tick; poses follow it."""
    s = scenes.mesh_mix(margin=margin)
    w = core.World(s)
    o = O.OracleWorld(s)
    worst = 0.0
    for f in range(90):
        sg, so = w.step(), o.step()
        assert sg["status"] == 0 and so["status"] == 0
        assert np.array_equal(w.candidate_pairs(), o.candidate_pairs()), f
        assert sg["contacts"] == so["contacts"], f
        cg, ng, mg = w.manifolds()
        co, no, mo = o.manifolds()
        assert np.array_equal(cg, co) and np.array_equal(ng, no), f
        xg, xo = w.states(), o.states()
        err = max(np.abs(xg[k] - xo[k]).max() for k in ("x", "q", "v"))
        worst = max(worst, err)
        assert err < 1e-4, (f, err)
    print("mesh mix worst |gpu-oracle| =", worst)


@pytest.mark.parametrize("kind", [scenes.PISTON, scenes.SLIDER])
def test_guided_contacts_match_oracle(gpu_available, kind):
    """Guided contacts on the GPU (a piston or slider box sliding into a
    static stop): contact counts, manifolds and poses equal the oracle's every
    tick, and the box comes to rest at the guided offset."""
    s = scenes.guided_stop(kind)
    w = core.World(s)
    o = O.OracleWorld(s)
    for f in range(40):
        sg, so = w.step(), o.step()
        assert sg["status"] == 0 and so["status"] == 0
        assert sg["contacts"] == so["contacts"], f
        cg, ng, _ = w.manifolds()
        co, no, _ = o.manifolds()
        assert np.array_equal(cg, co) and np.array_equal(ng, no), f
        xg, xo = w.states(), o.states()
        err = max(np.abs(xg[k] - xo[k]).max() for k in ("x", "q", "v"))
        assert err < 1e-4, (f, err)
    assert 1.5998 <= w.states()["x"][1, 0] <= 1.6


def test_graph_replay_equals_steps(gpu_available):
    s = scenes.pyramid()
    a = core.World(s)
    b = core.World(s)
    for _ in range(4):
        a.step(stats=False)
    b.capture(steps=2)
    b.replay()
    b.replay()
    assert np.array_equal(a.states().view(np.uint8), b.states().view(np.uint8))


def test_snapshot_restore(gpu_available):
    s = scenes.pyramid()
    w = core.World(s)
    for _ in range(3):
        w.step()
    w.snapshot()
    for _ in range(3):
        w.step()
    x1 = w.states()
    w.restore()
    for _ in range(3):
        w.step()
    assert np.array_equal(x1.view(np.uint8), w.states().view(np.uint8))


@pytest.mark.parametrize("norm", [0, 1, 2], ids=["max", "rms", "p999"])
def test_residual_schedule_matches_oracle(gpu_available, norm):
    """The residual-driven schedule stops at the same sweep, with the same
    residual trace, on the GPU and the oracle, under each of its three rules
    (largest row, RMS, 99.9th percentile)."""
    s = scenes.box_pile((6, 4, 6), seed=11, spacing=1.6)
    w = core.World(s)
    o = O.OracleWorld(s)
    for f in range(40):
        sg = w.step(residual_tolerance=2e-4, max_iterations=40, residual_norm=norm)
        so = o.step(residual_tolerance=2e-4, max_iterations=40, residual_norm=norm)
        assert float(sg["residual_over"]) == float(so["residual_over"]), f
        assert sg["iterations"] == so["iterations"], f
        np.testing.assert_allclose(w.residual_trace(), o.residual_trace(), rtol=1e-5, atol=1e-9)
        assert abs(float(sg["residual_max"]) - float(so["residual_max"])) <= 1e-6 + 1e-5 * abs(float(so["residual_max"]))


def test_launch_plans_are_bit_identical(gpu_available):
    """Every solve launch plan (CTA size, lanes per body, the staged solve
    with fused duals) computes the same bits; the autotuner only picks among
    them and leaves the state as it found it."""
    s = scenes.box_pile((6, 4, 6), seed=13, spacing=1.6)
    ref = None
    plans = [(v, p) for v in range(3) for p in range(5)] + [(v, p) for v in (3, 4) for p in range(2)]
    for v, p in plans:
        w = core.World(s)
        w.set_launch_plan(v, p)
        for _ in range(12):
            w.step()
        x = w.states().view(np.uint8).copy()
        if ref is None:
            ref = x
        assert np.array_equal(x, ref), (v, p)
        w.close()
    w = core.World(s)
    for _ in range(5):
        w.step()
    before = w.states().view(np.uint8).copy()
    v, p, report = w.autotune(ticks=2)
    assert report.count("ms/tick") == len(plans)
    assert np.array_equal(w.states().view(np.uint8), before)


def test_launch_plans_are_bit_identical_on_the_settled_pile(gpu_available):
    """The same on the settled 65,536-box pile, where colours are large
    enough for the per-body width classes (8/16/32 lanes, heaviest first)."""
    s = scenes.box_pile((64, 32, 32), seed=4)
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "settled_pile_64x32x32.npz"))
    s.states = z["states"].astype(np.float32).view(scenes.STATE_DTYPE).reshape(-1).copy()
    ref = None
    for v, p in ((1, 0), (0, 1), (0, 2), (1, 2), (2, 2), (1, 3), (0, 3), (3, 0), (4, 0), (4, 1), (1, 4), (0, 4)):
        w = core.World(s)
        w.set_launch_plan(v, p)
        for _ in range(4):
            st = w.step()
            assert st["status"] == 0
        x = w.states().view(np.uint8).copy()
        if ref is None:
            ref = x
        assert np.array_equal(x, ref), (v, p)
        w.close()


def test_contact_events_match_oracle(gpu_available):
    """Contact events (every point of every active pair in order, penetration
    clamped at 0, the tick's normal and friction impulses): bodies, points,
    normals and penetrations equal the oracle's bits; impulses agree within
    the solver's float tolerance."""
    s = scenes.box_pile((4, 3, 4), seed=21, spacing=1.6, count=40)
    w = core.World(s, event_capacity=100000)
    o = O.OracleWorld(s)
    for t in range(40):
        w.step(collect_events=1)
        o.step()
        g, r = w.contact_events(), o.contact_events()
        assert len(g) == len(r), t
        for k in ("body", "collider", "position", "normal", "penetration"):
            assert np.array_equal(g[k].view(np.uint32), r[k].view(np.uint32)), (t, k)
        for k in ("normal_impulse", "friction_impulse"):
            assert np.allclose(g[k], r[k], rtol=2e-3, atol=2e-4), (t, k)
    w.step()
    assert len(w.contact_events()) == 0
    w.close()


def test_device_trig_equals_oracle_bits(gpu_available):
    """The tick's arctangent and x cot(x) evaluate to the oracle's bits."""
    rng = np.random.Generator(np.random.Philox(22))
    inp = np.zeros((5000, 3), np.float32)
    inp[:, :2] = rng.uniform(0.0, 1.0, (5000, 2))
    inp[:100, 1] = 0.0
    inp[:, 2] = rng.uniform(0.0, np.pi / 2, 5000)
    out = core.math_eval(4, inp)
    ref = np.array([O.trig_eval(r) for r in inp])
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))
