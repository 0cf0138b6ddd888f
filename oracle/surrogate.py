"""CPU oracle of the learned barostat's surrogate network.

Test infrastructure only: it checks the device forward and backward passes
(rainmd_b200/csrc/surrogate.cu); nothing in the product imports it. The reference has no
learned part, so there is no reference file to follow; this restates, in float64 numpy, the
network the device trains:

    h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2), y = x_0 (W3 . h2 + b3)

(the output gated by input 0, so it vanishes for a zero volume step) with 8 inputs, 64 units
per hidden layer, the weights W1, W2, W3 rounded to BF16 (round to
nearest even) in the forward pass and the biases kept in FP32, and the loss
L = mean_b (y_b - t_b)^2. Gradients are taken through the rounded weights (the gradient with
respect to a master weight is the gradient with respect to its BF16 value), as on the device.
Parameter layout (4801 floats): W1[64][8], b1[64], W2[64][64], b2[64], W3[64], b3.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H = 8, 64
W1 = 0
B1 = W1 + N_H * N_IN
W2 = B1 + N_H
B2 = W2 + N_H * N_H
W3 = B2 + N_H
B3 = W3 + N_H
PARAMS = B3 + 1


def bf16_round(values) -> np.ndarray:
    """float32 -> nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(values, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return (u & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def unpack(params, bf16: bool = True):
    """Weights (BF16-rounded when `bf16`, else taken as given) and biases, in float64."""
    p = np.asarray(params, dtype=np.float64)
    if bf16:
        def cast(v):
            return bf16_round(v.astype(np.float32)).astype(np.float64)
    else:
        def cast(v):
            return v
    w1 = cast(p[W1:B1]).reshape(N_H, N_IN)
    w2 = cast(p[W2:B2]).reshape(N_H, N_H)
    w3 = cast(p[W3:B3])
    return w1, p[B1:W2], w2, p[B2:W3], w3, float(p[B3])


def forward(params, x, bf16: bool = True):
    """Outputs y[count] and the hidden activations."""
    w1, b1, w2, b2, w3, b3 = unpack(params, bf16)
    x = np.asarray(x, dtype=np.float64).reshape(-1, N_IN)
    h1 = np.tanh(x @ w1.T + b1)
    h2 = np.tanh(h1 @ w2.T + b2)
    return x[:, 0] * (h2 @ w3 + b3), h1, h2


def loss_and_gradients(params, x, t, bf16: bool = True):
    """(loss, gradient[4801]) of the mean squared error."""
    w1, b1, w2, b2, w3, b3 = unpack(params, bf16)
    x = np.asarray(x, dtype=np.float64).reshape(-1, N_IN)
    t = np.asarray(t, dtype=np.float64)
    y, h1, h2 = forward(params, x, bf16)
    n = len(t)
    loss = float(np.mean((y - t) ** 2))
    dz = 2.0 * (y - t) / n * x[:, 0]  # through the gate
    g = np.zeros(PARAMS)
    g[W3:B3] = dz @ h2
    g[B3] = dz.sum()
    d2 = np.outer(dz, w3) * (1.0 - h2 ** 2)
    g[W2:B2] = (d2.T @ h1).reshape(-1)
    g[B2:W3] = d2.sum(0)
    d1 = (d2 @ w2) * (1.0 - h1 ** 2)
    g[W1:B1] = (d1.T @ x).reshape(-1)
    g[B1:W2] = d1.sum(0)
    return loss, g


def random_parameters(seed: int = 0, scale: float = 1.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    p[W1:B1] = rng.uniform(-1, 1, N_H * N_IN) * np.sqrt(6 / (N_IN + N_H)) * scale
    p[B1:W2] = rng.normal(0, 0.1, N_H)
    p[W2:B2] = rng.uniform(-1, 1, N_H * N_H) * np.sqrt(6 / (2 * N_H)) * scale
    p[B2:W3] = rng.normal(0, 0.1, N_H)
    p[W3:B3] = rng.uniform(-1, 1, N_H) * np.sqrt(6 / (N_H + 1)) * scale
    p[B3] = 0.05
    return p
