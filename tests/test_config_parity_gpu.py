# SPDX-License-Identifier: MIT
"""The benchmark configurations at their stated sizes: the CUDA path against
the CPU oracle frame by frame, then long runs on the GPU against the
reference's physical gates, and the error against an FP64 replay.

Parity (every compared frame): candidate pair sets, manifold pair codes and
point counts, colours of dynamic bodies and island roots are equal, and so
are the poses, bit for bit: the tick evaluates every expression in the
reference's order from IEEE-exact operations (no contraction, IEEE division
and square root, arctangent and cotangent from series of basic operations),
as the oracle does.

Physical gates (the reference's realtime stack gates,
tests/solver/rigid_realtime_cuda_tests.cu:362-370, with the measures of
conformance/v1/realtime/scenario-fixtures-v1.json:64-72): largest post-step
overlap of contact pairs <= 5 mm, settled translation drift <= 1 cm and
rotation drift <= 0.035 rad over the settled window, unforced energy growth
<= 5 %, no tunnelling (a body centre below the ground's top face).

FP64: the same scene stepped by the oracle in double precision; the largest
|FP32 GPU - FP64| position difference over the compared frames is printed
(chaotic divergence is expected; it is a measure, gated only loosely).
"""
import numpy as np
import pytest

from pmb200 import core, scenes
import oracle as O
import physics_gates as G

pytestmark = pytest.mark.gpu

def compare(scene, frames, fp64_frames=0, label="", joints=False):
    """GPU and FP32 oracle side by side for `frames` ticks (and the FP64
    oracle for the first `fp64_frames`); returns the GPU world, the worst
    FP32 pose difference and the worst FP64 position difference."""
    w = core.World(scene)
    o = O.OracleWorld(scene)
    o64 = O.OracleWorld(scene, fp64=True) if fp64_frames else None
    dyn = scene.bodies["motion"] == scenes.DYNAMIC
    worst, worst64, exact = 0.0, 0.0, 0
    for f in range(frames):
        sg = w.step()
        so = o.step()
        assert int(sg["status"]) == 0, (f, core.status_names(int(sg["status"])))
        assert np.array_equal(w.candidate_pairs(), o.candidate_pairs()), (label, f)
        cg, ng, _ = w.manifolds()
        co, no, _ = o.manifolds()
        assert np.array_equal(cg, co) and np.array_equal(ng, no), (label, f)
        colg, parg = w.graph()
        colo, paro = o.graph()
        assert np.array_equal(colg[dyn], colo[dyn]) and np.array_equal(parg, paro), (label, f)
        if joints:
            fg, _, rg = w.joints()
            fo, _, ro = o.joints()
            assert np.array_equal(fg, fo) and np.array_equal(rg, ro), (label, f)
        xg, xo = w.states(), o.states()
        err = max(float(np.abs(xg[k] - xo[k]).max()) for k in ("x", "q", "v"))
        exact += int(all(np.array_equal(xg[k], xo[k]) for k in ("x", "q", "v", "w")))
        worst = max(worst, err)
        assert np.array_equal(xg.view(np.uint8), xo.view(np.uint8)), (label, f, err)
        if o64 is not None and f < fp64_frames:
            o64.step()
            worst64 = max(worst64, float(np.abs(xg["x"].astype(np.float64) - o64.states()["x"]).max()))
    print(f"{label}: {frames} frames, worst |gpu - oracle| {worst:.3g}, bit-identical frames {exact}/{frames}, "
          f"max |fp32 gpu - fp64| position {worst64:.3g} m over {fp64_frames} frames")
    return w, worst, worst64


def stack_gates(scene, world, frames, settle, ground_top=0.0, label=""):
    """Step `world` `frames` more ticks on the GPU alone and measure the
    gates; the settled window starts `settle` ticks in."""
    dyn = scene.bodies["motion"] == scenes.DYNAMIC
    pen, pen_settled, tunnel = 0.0, 0.0, 0
    first = None
    drift = rot = 0.0
    e0 = emax = None
    for f in range(frames):
        st = world.step()
        assert int(st["status"]) == 0, (f, core.status_names(int(st["status"])))
        s = world.states()
        p = G.pair_penetration(scene, s, G.contact_pairs(world, scene.n))
        pen = max(pen, p)
        tunnel += int((s["x"][dyn, 1] < ground_top).sum())
        if f >= settle:
            pen_settled = max(pen_settled, p)
            e = G.energy(scene, s)
            if first is None:
                first = s
                e0 = emax = e
            emax = max(emax, e)
            drift = max(drift, float(np.linalg.norm(s["x"][dyn] - first["x"][dyn], axis=1).max()))
            dq = np.abs(np.einsum("pi,pi->p", s["q"][dyn].astype(np.float64), first["q"][dyn].astype(np.float64)))
            rot = max(rot, float((2 * np.arccos(np.clip(dq, 0, 1))).max()))
    growth = max(0.0, (emax - e0) / max(abs(e0), 1e-3))
    print(f"{label}: penetration {pen:.3g} m (settled window {pen_settled:.3g} m), settled drift {drift:.3g} m, "
          f"rotation drift {rot:.3g} rad, energy growth {growth:.3g}, tunnelling {tunnel}")
    return pen, pen_settled, drift, rot, growth, tunnel


@pytest.mark.parametrize("profile", [scenes.LEGACY, scenes.REALTIME], ids=["legacy", "realtime"])
def test_config1_pyramid_600_frames(gpu_available, profile):
    """Config 1 at its stated length: 55 jittered unit cubes, 600 frames
    compared with the oracle (and 600 with the FP64 replay), then the
    stack gates over the same trajectory re-run on the GPU."""
    s = scenes.pyramid(profile=profile)
    label = f"config 1 pyramid ({'legacy' if profile == scenes.LEGACY else 'realtime v1'})"
    compare(s, 600, fp64_frames=600, label=label)
    w = core.World(s)
    pen, _, drift, rot, growth, tunnel = stack_gates(s, w, 600, settle=120, label=label)
    assert pen <= 0.005 and drift <= 0.01 and rot <= 0.035 and growth <= 0.05 and tunnel == 0


def test_config2_pile_4096_first_frames(gpu_available):
    """Config 2 at its stated size (4,096 boxes, 16x16x16 grid, seed 2): the
    first 60 frames against the oracle (the bottom layers reach the ground
    and each other), 30 of them against the FP64 replay."""
    s = scenes.config(1)
    compare(s, 60, fp64_frames=30, label="config 2 pile 4096")


def test_config2_pile_300_frames_gates(gpu_available):
    """Config 2 over its stated 300 frames on the GPU: the pile falls, lands
    (boxes of up to 6.75 t hit the ground and each other at several m/s
    between frames 60 and 120) and settles. Once settled (frames 120-300)
    no pair overlaps by more than 2 mm (the reference's brick-stack gate,
    conformance/v1/quality/rigid-brick-penetration-v1.json); during the
    landing impacts the overlap stays under 1 cm (the serial oracle peaks at
    5.3 mm on this pile); energy never grows by more than 5 % over the
    settled window; nothing tunnels."""
    s = scenes.config(1)
    w = core.World(s)
    pen, settled, drift, rot, growth, tunnel = stack_gates(s, w, 300, settle=120,
                                                           label="config 2 pile 4096, 300 frames")
    assert settled <= 0.002 and pen <= 0.01 and growth <= 0.05 and tunnel == 0


def test_config3_chains_first_frames(gpu_available):
    """Config 3 at its stated size (512 chains x 64 capsule links, point
    joints, 100x end boxes, seed 3): the first 30 frames against the oracle,
    joint flags and row counts equal every frame, 8 against the FP64 replay."""
    s = scenes.config(2)
    compare(s, 30, fp64_frames=8, label="config 3 chains 512x64", joints=True)


def _joint_error(scene, states):
    """Largest world-anchor separation of the scene's joints (m)."""
    j = scene.joints
    x = states["x"].astype(np.float64)
    R = G.quat_matrix(states["q"])
    pa = x[j["body_a"]] + np.einsum("pij,pj->pi", R[j["body_a"]], j["anchor_a"].astype(np.float64))
    pb = x[j["body_b"]] + np.einsum("pij,pj->pi", R[j["body_b"]], j["anchor_b"].astype(np.float64))
    return float(np.linalg.norm(pa - pb, axis=1).max())


def test_config3_chains_600_frames_gates(gpu_available):
    """Config 3 over its stated 600 frames on the GPU: joint position error
    (largest world-anchor separation) stays within 1 cm, links and end boxes
    never interpenetrate by more than 5 mm, energy does not grow by more than
    5 % (the chains swing and collide; nothing drives them)."""
    s = scenes.config(2)
    w = core.World(s)
    jerr, pen, e0, emax = 0.0, 0.0, None, None
    for f in range(600):
        st = w.step()
        assert int(st["status"]) == 0, (f, core.status_names(int(st["status"])))
        x = w.states()
        jerr = max(jerr, _joint_error(s, x))
        if f % 10 == 0:
            pen = max(pen, G.pair_penetration(s, x, G.contact_pairs(w, s.n)))
        e = G.energy(s, x)
        e0 = e if e0 is None else e0
        emax = e if emax is None else max(emax, e)
    growth = max(0.0, (emax - e0) / max(abs(e0), 1e-3))
    print(f"config 3 chains 512x64, 600 frames: joint position error {jerr:.3g} m, penetration {pen:.3g} m, "
          f"energy growth {growth:.3g}")
    assert jerr <= 0.01 and pen <= 0.005 and growth <= 0.05
