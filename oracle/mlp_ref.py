"""CPU reference of the learned preconditioner's MLP (numpy, float64 arithmetic).

TEST INFRASTRUCTURE: checks the library's forward and backward CUDA kernels
(risqgpu_mlp_grad, risqgpu_precond_factors).  The network has no counterpart in the
reference crate; it follows the definition in include/risqgpu.h:
o = W3 relu(W2 relu(W1 x + b1) + b2) + b3 with W1, W2, W3 rounded to BF16 (round to
nearest even), factor = clamp(exp((o(x) + o(x~)) / 2), 0.25, 4) with x~ the features with
the alpha and beta occupations exchanged and the first layer's activations rounded to
BF16 (inference); loss L = sum_b w_b (o_b - log t_b)^2 / sum_b w_b with FP32 activations
(training).
"""
from __future__ import annotations

import numpy as np


def bf16_round(a):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    special = (u & 0x7F800000) == 0x7F800000
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    r = np.where(special, u & 0xFFFF0000, r).astype(np.uint32)
    return r.view(np.float32)


def unpack(params, n_in, H):
    p = np.asarray(params, dtype=np.float32)
    o = 0
    W1 = p[o:o + H * n_in].reshape(H, n_in); o += H * n_in
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o:o + 1]
    return W1, b1, W2, b2, W3, b3


def forward(params, X, n_in, H, act_bf16=False):
    """Network output.  act_bf16: round the first layer's activations to BF16, as
    inference does (the trainer keeps them FP32)."""
    W1, b1, W2, b2, W3, b3 = unpack(params, n_in, H)
    W1r, W2r, W3r = (bf16_round(w).astype(np.float64) for w in (W1, W2, W3))
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ W1r.T + b1
    h1 = np.maximum(z1, 0.0)
    if act_bf16:
        h1 = bf16_round(h1.astype(np.float32)).astype(np.float64)
    z2 = h1 @ W2r.T + b2
    h2 = np.maximum(z2, 0.0)
    o = h2 @ W3r + b3[0]
    return o, (X, h1, h2, W2r, W3r)


def loss_and_grad(params, X, t, w, n_in, H):
    o, (X, h1, h2, W2r, W3r) = forward(params, X, n_in, H)
    t = np.asarray(t, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    W = w.sum()
    d = o - np.log(t)
    loss = np.sum(w * d ** 2) / W
    do = 2.0 * w * d / W
    dW3 = do @ h2
    db3 = do.sum()
    dh2 = np.outer(do, W3r) * (h2 > 0)
    dW2 = dh2.T @ h1
    db2 = dh2.sum(0)
    dh1 = (dh2 @ W2r) * (h1 > 0)
    dW1 = dh1.T @ X
    db1 = dh1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3, [db3]])
    return loss, g


def swap_spins(X, norb):
    """Features with the alpha and beta occupation blocks exchanged."""
    Xs = np.array(X, copy=True)
    Xs[:, :norb], Xs[:, norb:2 * norb] = X[:, norb:2 * norb], X[:, :norb]
    return Xs


def factors(params, X, n_in, H):
    norb = (n_in - 2) // 2
    o1, _ = forward(params, X, n_in, H, act_bf16=True)
    o2, _ = forward(params, swap_spins(X, norb), n_in, H, act_bf16=True)
    return np.clip(np.exp(0.5 * (o1 + o2)), 0.25, 4.0)
