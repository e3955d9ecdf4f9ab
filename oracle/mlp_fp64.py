"""FP64 CPU oracle of the leaf-value network: TEST INFRASTRUCTURE ONLY.

Only tests may import this module; the library's network runs on the GPU
(dcfr_mlp_* in libdcfr) and never calls it.

The network has no counterpart in the reference solver (it is the learned
leaf evaluator of depth-limited solves), so this oracle is pinned by
mathematics instead of reference vectors: its analytic gradients are checked
against central finite differences in float64 (tests/test_oracle_mlp.py).

Network (parameters in the library's layout, LeafNet.split):
    X_0 = x zero-padded to kin[0] columns
    Z_l = X_l W_l^T + b_l,  X_{l+1} = gelu(Z_l)      for l < L
    Y   = X_L W_L^T + b_L   (first out_dim columns)
    loss = sum(mask * (Y - t)^2) / sum(mask)
with gelu(z) = z * Phi(z) (the exact, erf form).

With bf16=True the operands are rounded to bfloat16 where the GPU kernels
store them in bfloat16: the input, the weights, each pre-activation Z_l
(kept for the backward pass), each activation X_{l+1}, and each output
gradient dY before it enters a GEMM. Everything else is float64.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

SQRT2 = np.sqrt(2.0)
INV_SQRT_2PI = 1.0 / np.sqrt(2.0 * np.pi)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even) via float32 bit patterns;
    returns float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return (r.astype(np.uint32).view(np.float32)).astype(np.float64)


def gelu(z: np.ndarray) -> np.ndarray:
    return 0.5 * z * (1.0 + erf(z / SQRT2))


def gelu_grad(z: np.ndarray) -> np.ndarray:
    return 0.5 * (1.0 + erf(z / SQRT2)) + z * np.exp(-0.5 * z * z) * INV_SQRT_2PI


def loss_and_gradients(layers, x, t, mask=None, bf16_points: bool = False):
    """layers: [(W [nout][kin], b [nout])] per layer (float arrays, padded as
    the library stores them); x [M][in_dim], t [M][out_dim], mask like t or
    None. Returns (loss, [(dW, db)] per layer), all float64."""
    rnd = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))
    W = [rnd(w) for w, _ in layers]
    B = [np.asarray(b, np.float64) for _, b in layers]
    M = x.shape[0]
    X0 = np.zeros((M, W[0].shape[1]))
    X0[:, :x.shape[1]] = x
    X = [rnd(X0)]
    Z = []
    for l in range(len(layers) - 1):
        pre = X[-1] @ W[l].T + B[l]
        Z.append(rnd(pre))
        X.append(rnd(gelu(pre)))
    Yfull = X[-1] @ W[-1].T + B[-1]
    out_dim = t.shape[1]
    Y = Yfull[:, :out_dim]
    m = np.ones_like(Y) if mask is None else np.asarray(mask, np.float64)
    cnt = m.sum()
    d = Y - np.asarray(t, np.float64)
    loss = float((m * d * d).sum() / cnt)
    dY = np.zeros_like(Yfull)
    dY[:, :out_dim] = 2.0 * m * d / cnt
    dY = rnd(dY)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        grads[l] = (dY.T @ X[l], dY.sum(0))
        if l > 0:
            dY = rnd((dY @ W[l]) * gelu_grad(Z[l - 1]))
    return loss, grads


def adam_step(w, g, m, v, step: int, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
    """One Adam step in float64 (bias-corrected, step counted from 1);
    returns (w, m, v)."""
    w, g, m, v = (np.asarray(a, np.float64) for a in (w, g, m, v))
    m = b1 * m + (1.0 - b1) * g
    v = b2 * v + (1.0 - b2) * g * g
    c1, c2 = 1.0 - b1 ** step, 1.0 - b2 ** step
    return w - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v
