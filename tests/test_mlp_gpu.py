# SPDX-License-Identifier: MIT
"""The warm-start MLP's tensor-core kernels against the CPU restatement.

- Forward outputs and every parameter gradient of the BF16 tcgen05 kernels
  (pmb_mlp_forward_backward) match oracle/mlp.py with BF16 rounding at the
  same points. Accumulation order inside the tensor cores differs from the
  oracle's float64 sums and ReLU masks can flip for pre-activations within
  rounding of zero, so the comparison is norm-wise: relative error <= 1e-2
  for the outputs and for each weight matrix's gradient.
- Batches that are not a multiple of the 128-row tile and batches spanning
  several tiles per CTA accumulate correctly.
- Online training inside the tick lowers the loss, and ticks run with the
  learned warm start reach the residual tolerance like plain ticks.
"""
import numpy as np
import pytest

import mlp as M
from pmb200 import core, scenes

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("n", [128, 1000, 40000])
def test_forward_backward_matches_oracle(gpu_available, n):
    rng = np.random.default_rng(n)
    f = rng.uniform(-1.0, 1.0, (n, M.FEATURES)).astype(np.float32)
    y = rng.uniform(-0.5, 1.5, (n, 2)).astype(np.float32)
    w = np.full(n, 1.0 / n, np.float32)
    p = M.init_params(n % 97)
    out, g, loss = core.mlp_forward_backward(f, y, w, p)
    o_ref, g_ref, loss_ref = M.forward_backward(f, y, w, p)
    assert _rel(out, o_ref) < 1e-2
    assert abs(loss - loss_ref) <= 1e-2 * abs(loss_ref)
    for lo, hi in ((M.W1, M.W2), (M.W2, M.W3), (M.W3, M.PARAMS)):
        assert _rel(g[lo:hi], g_ref[lo:hi]) < 1e-2, (n, lo)
    # padding parameters stay exactly zero
    w1 = g[M.W1:M.W2].reshape(M.HIDDEN, M.IN)
    w3 = g[M.W3:].reshape(M.OUT_N, M.HIDDEN_K)
    assert not w1[:, M.FEATURES + 1:].any() and not w3[M.OUT:].any()


def test_online_training_and_learned_ticks(gpu_available):
    scene = scenes.box_pile((8, 6, 8), seed=12, spacing=1.3)
    w = core.World(scene)
    # Training mechanics on ticks stopped by the RMS residual: the loss is
    # measured against each tick's converged rows, and under the row-max stop
    # the sweep count (and with it the converged penalties) of this small pile
    # varies from tick to tick, which no per-contact prediction can follow.
    kw = dict(residual_tolerance=2e-4, max_iterations=48, residual_norm=1)
    for _ in range(60):
        w.step(**kw)
    w.mlp_attach(seed=3)
    w.mlp_train(True, lr=3e-3, steps_per_tick=4)
    ratios = []
    for _ in range(40):
        st = w.step(**kw)
        assert st["status"] == 0
        _, loss, plain, gate = w.mlp_params()
        assert np.isfinite(loss) and plain > 0 and gate in (0.0, 1.0)
        ratios.append(loss / plain)
    # The model starts as the plain warm start (zero output layer: ratio 1
    # before the first update) and learns corrections that beat it.
    assert ratios[0] > 0.9, ratios[0]
    assert np.mean(ratios[-5:]) < 0.95, ratios
    w.mlp_train(False)
    for _ in range(10):
        st = w.step(warm_start=1, **kw)
        assert st["status"] == 0
        assert st["residual"] <= 2e-4 or st["iterations"] == 48
    assert np.isfinite(w.states()["x"]).all()


def test_trained_predictor_saves_sweeps_on_a_held_out_pile(gpu_available):
    """What the trained network gains. A predictor is trained online on one
    settled pile of 6,912 boxes (seed 12; 300 plain ticks, then 200 training
    frames), then applied to a held-out pile of the same size (seed 14, also
    settled 300 ticks) from one snapshot: at the same residual criterion --
    the 99.9th percentile of the row violations within 1e-4 m, at most 64
    sweeps -- the learned warm start needs fewer sweeps per tick on average
    than the plain warm start, and every tick of both arms that stops before
    the cap meets the criterion. (Piles of about a thousand boxes give too
    few contacts a frame for the model to beat the plain warm start within
    200 frames; its gate then stays closed.)"""
    kw = dict(residual_tolerance=1e-4, max_iterations=64, residual_norm=2)
    train = scenes.box_pile((24, 12, 24), seed=12, spacing=1.3)
    w = core.World(train)
    for _ in range(300):
        w.step(**kw)
    w.mlp_attach(seed=3)
    w.mlp_train(True, lr=3e-3, steps_per_tick=4)
    for _ in range(200):
        assert w.step(**kw)["status"] == 0
    params, loss, plain_loss, gate = w.mlp_params()
    w.close()
    assert gate == 1.0 and loss < 0.9 * plain_loss, (loss / plain_loss, gate)
    held = scenes.box_pile((24, 12, 24), seed=14, spacing=1.3)
    h = core.World(held)
    for _ in range(300):
        h.step(**kw)
    h.snapshot()
    h.mlp_attach(params=params)
    sweeps = {}
    for arm in (0, 1):
        h.restore()
        its = []
        for _ in range(40):
            st = h.step(warm_start=arm, **kw)
            assert st["status"] == 0
            its.append(int(st["iterations"]))
            if its[-1] < 64:
                assert float(st["residual_over"]) <= 1e-3, (arm, float(st["residual_over"]))
        sweeps[arm] = float(np.mean(its))
    h.close()
    print(f"held-out pile: training loss {loss / plain_loss:.3f} x plain; mean sweeps plain {sweeps[0]:.2f}, "
          f"learned {sweeps[1]:.2f}")
    assert sweeps[1] < sweeps[0], sweeps
