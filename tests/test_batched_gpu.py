# SPDX-License-Identifier: MIT
"""Batched stepping of independent scenes (config-5 path) on the GPU.

A batched world steps several scenes in one tick: scene-keyed broadphase
buckets and per-scene large-body lists keep scenes apart, and every scene
sweeps its own iteration budget. Since no computation mixes data of two
scenes and the greedy colouring, island roots and Gauss-Seidel order of a
scene depend only on its own bodies, every scene of the batch must evolve
bit-identically to the same scene stepped alone -- that is the test. The
per-scene residual (float sums in any order) must match the lone world's
within 1e-4 relative.
"""
import numpy as np
import pytest

from pmb200 import core, scenes

pytestmark = pytest.mark.gpu


def _parts():
    return [scenes.pyramid(levels=5, seed=3),
            scenes.box_pile((4, 3, 4), seed=21, spacing=1.6, count=40),
            scenes.chains(count=2, links=6, seed=4),
            scenes.box_pile((3, 3, 3), seed=22, spacing=1.6),
            scenes.chains(count=1, links=9, seed=5, iterations=12),
            scenes.joint_zoo(seed=8),
            scenes.joint_zoo(seed=9, iterations=16)]


def test_batch_equals_scenes_stepped_alone(gpu_available):
    parts = _parts()
    batch = scenes.batch(parts)
    wb = core.World(batch)
    alone = [core.World(p) for p in parts]
    offs = np.concatenate([[0], np.cumsum([p.n for p in parts])])
    for t in range(30):
        sb = wb.step()
        assert sb["status"] == 0, core.status_names(int(sb["status"]))
        res = [w.step() for w in alone]
        xb = wb.states()
        for k, w in enumerate(alone):
            xa = w.states()
            assert np.array_equal(xb[offs[k]:offs[k + 1]].view(np.uint8), xa.view(np.uint8)), (t, k)
        rms, mx, its, cts = wb.scene_stats()
        for k, st in enumerate(res):
            assert its[k] == parts[k].iterations
            assert cts[k] == st["contacts"], (t, k)
            assert abs(rms[k] - st["residual"]) <= 1e-4 * abs(st["residual"]) + 1e-9, (t, k, rms[k], st["residual"])
    wb.close()
    for w in alone:
        w.close()


def test_batched_graph_replay_equals_steps(gpu_available):
    batch = scenes.batch(_parts())
    a = core.World(batch)
    b = core.World(batch)
    for _ in range(4):
        a.step(stats=False)
    b.capture(steps=2)
    b.replay()
    b.replay()
    assert np.array_equal(a.states().view(np.uint8), b.states().view(np.uint8))


def test_batched_learned_graph_replay_equals_steps(gpu_available):
    """The learned warm start (features, tensor-core inference, apply) is
    stream-ordered with no host decision, so a captured tick replays it
    exactly; a trained MLP (gate open or not) is read from device memory."""
    batch = scenes.batched_scenes(12, seed=5, smallest=16, largest=96)
    a = core.World(batch)
    b = core.World(batch)
    for w in (a, b):
        w.mlp_attach(seed=1)
        w.mlp_train(True, lr=3e-3, steps_per_tick=2)
        for _ in range(6):
            w.step(stats=False)
        w.mlp_train(False)
    assert np.array_equal(a.mlp_params()[0], b.mlp_params()[0])
    for _ in range(4):
        st = a.step(warm_start=1)
        assert st["status"] == 0
    b.capture(steps=2, warm_start=1)
    b.replay()
    b.replay()
    assert np.array_equal(a.states().view(np.uint8), b.states().view(np.uint8))
    a.close()
    b.close()


def test_batched_plans_are_bit_identical(gpu_available):
    """A batched world with joints (chains, every joint type) gives the same
    bits under every solve launch plan (CTA size, lanes per body, static or
    claimed body assignment)."""
    batch = scenes.batch(_parts())
    ref = None
    for v, p in ((1, 0), (1, 3), (0, 2), (2, 1), (0, 3), (4, 0), (3, 1), (1, 4)):
        w = core.World(batch)
        w.set_launch_plan(v, p)
        for _ in range(20):
            st = w.step()
            assert st["status"] == 0, core.status_names(int(st["status"]))
        x = w.states().view(np.uint8).copy()
        if ref is None:
            ref = x
        assert np.array_equal(x, ref), (v, p)
        w.close()


def test_batch_of_config5_scenes_equals_the_oracle(gpu_available):
    """Sixteen scenes drawn from the 1,024-scene batch (the config-5 mix of
    piles and chains, log-uniform sizes, seed 5) stepped as one batched world
    on the GPU for 20 ticks: every scene's states equal the CPU oracle
    stepping that scene alone, bit for bit, and every scene's contact count
    and sweep count match the oracle's."""
    import oracle as O
    ids = list(range(0, 1024, 64))
    sizes, kinds = scenes.batched_plan(1024, 5)
    parts = [scenes.batched_part(k, sizes[k], kinds[k], 5) for k in ids]
    batch = scenes.batch(parts)
    wb = core.World(batch)
    cpu = [O.OracleWorld(p) for p in parts]
    offs = np.concatenate([[0], np.cumsum([p.n for p in parts])])
    for t in range(20):
        sb = wb.step()
        assert sb["status"] == 0, core.status_names(int(sb["status"]))
        res = [o.step() for o in cpu]
        xb = wb.states()
        _, _, its, cts = wb.scene_stats()
        for k, o in enumerate(cpu):
            assert np.array_equal(xb[offs[k]:offs[k + 1]].view(np.uint8), o.states().view(np.uint8)), (t, ids[k])
            assert cts[k] == res[k]["contacts"] and its[k] == res[k]["iterations"], (t, ids[k])
    wb.close()
