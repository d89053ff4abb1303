# SPDX-License-Identifier: MIT
"""ORACLE -- test infrastructure only. CPU restatement of the learned
warm-start MLP (8 -> 64 -> 64 -> 2) of parallel-mater_b200/csrc/pmb_mlp.cu,
for checking the tensor-core kernels. The model has no counterpart in the
reference (its warm start is constraint_math.slang:30-37, restated in
avbd_math.hpp); this file restates this project's own definition.

Parameter vector: W1 [64][16], W2 [64][80], W3 [16][80], row-major float32.
Bias terms are the weights of constant-one inputs: X[:, 8] = 1,
H1[:, 64] = H2[:, 64] = 1.

`forward_backward(..., bf16=True)` rounds to BF16 (round to nearest even)
exactly where the kernels store BF16 operands: X, the weights, both hidden
activations, and the backward operands dO, dZ2, dZ1; products and sums are
carried in float64 (the tensor cores accumulate exact BF16 products in
FP32). With bf16=False the same function is the plain float64 model, used
for finite-difference checks of the gradient formulas.
"""
import numpy as np

FEATURES, IN, HIDDEN, HIDDEN_K, OUT, OUT_N = 8, 16, 64, 80, 2, 16
W1, W2 = 0, HIDDEN * IN
W3 = W2 + HIDDEN * HIDDEN_K
PARAMS = W3 + OUT_N * HIDDEN_K


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    a = np.ascontiguousarray(a, np.float32)
    bits = a.view(np.uint32).astype(np.uint64)
    bits = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return bits.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    p = np.asarray(params, np.float64)
    return (p[W1:W2].reshape(HIDDEN, IN), p[W2:W3].reshape(HIDDEN, HIDDEN_K),
            p[W3:PARAMS].reshape(OUT_N, HIDDEN_K))


def forward_backward(features, targets, weights, params, bf16_round=True):
    """Returns (outputs [n,2], gradient [PARAMS], loss) of
    loss = sum_r w_r * ((o0 - y0)^2 + (o1 - y1)^2)."""
    rnd = bf16 if bf16_round else (lambda a: np.asarray(a, np.float64))
    f = np.asarray(features, np.float64).reshape(-1, FEATURES)
    n = len(f)
    y = np.asarray(targets, np.float64).reshape(n, 2)
    w = np.asarray(weights, np.float64).reshape(n)
    w1, w2, w3 = (rnd(m) for m in unpack(params))
    x = np.zeros((n, IN))
    x[:, :FEATURES] = f
    x[:, FEATURES] = 1.0
    x = rnd(x)
    z1 = x @ w1.T
    h1 = np.zeros((n, HIDDEN_K))
    h1[:, :HIDDEN] = rnd(np.maximum(z1, 0.0))
    h1[:, HIDDEN] = 1.0
    z2 = h1 @ w2.T
    h2 = np.zeros((n, HIDDEN_K))
    h2[:, :HIDDEN] = rnd(np.maximum(z2, 0.0))
    h2[:, HIDDEN] = 1.0
    o = (h2 @ w3.T)[:, :OUT]
    e = o - y
    loss = float(np.sum(w[:, None] * e * e))
    do = np.zeros((n, OUT_N))
    do[:, :OUT] = rnd(2.0 * w[:, None] * e)
    dw3 = do.T @ h2
    dz2 = rnd((do @ w3[:, :HIDDEN]) * (z2 > 0))
    dw2 = dz2.T @ h1
    dz1 = rnd((dz2 @ w2[:, :HIDDEN]) * (z1 > 0))
    dw1 = dz1.T @ x
    g = np.concatenate([dw1.ravel(), dw2.ravel(), dw3.ravel()])
    return o, g, loss


def init_params(seed=1):
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float64)
    w1, w2, w3 = (p[W1:W2].reshape(HIDDEN, IN), p[W2:W3].reshape(HIDDEN, HIDDEN_K),
                  p[W3:PARAMS].reshape(OUT_N, HIDDEN_K))
    w1[:, :FEATURES] = rng.uniform(-1, 1, (HIDDEN, FEATURES)) * np.sqrt(6.0 / FEATURES)
    w1[:, FEATURES] = rng.uniform(-0.1, 0.1, HIDDEN)
    w2[:, :HIDDEN] = rng.uniform(-1, 1, (HIDDEN, HIDDEN)) * np.sqrt(6.0 / HIDDEN)
    w2[:, HIDDEN] = rng.uniform(-0.1, 0.1, HIDDEN)
    w3[:OUT, :HIDDEN] = rng.uniform(-1, 1, (OUT, HIDDEN)) * np.sqrt(6.0 / HIDDEN)
    w3[:OUT, HIDDEN] = rng.uniform(-0.1, 0.1, OUT)
    return p.astype(np.float32)
