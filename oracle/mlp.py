"""FP64 NumPy restatement of the warm-start network's forward and backward passes. TEST
INFRASTRUCTURE ONLY: the checker of the GPU tensor-core training kernels' gradients.

It mirrors where the GPU path rounds to BF16 (hidden activations, the BF16 copy of every gradient
that feeds a matrix product) so that the comparison isolates the products, the epilogues and the
operand layouts; everything else is FP64.
"""

from __future__ import annotations

import numpy as np


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    out = ((u + rounding) >> 16 << 16).astype(np.uint32)
    nan = np.isnan(f)
    out[nan] = 0x7FC00000
    return out.view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward_backward(weights, biases, x16, target, n_out):
    """weights[l] [out, in] and x16 [B, in0] hold BF16 values; biases FP32. Returns (loss, pred,
    dW list, db list) for the MSE over the first n_out outputs."""
    W = [np.asarray(w, np.float64) for w in weights]
    b = [np.asarray(v, np.float64) for v in biases]
    depth = len(W) - 1
    H = [np.asarray(x16, np.float64)]
    Z = []
    for l in range(depth + 1):
        z = H[-1] @ W[l].T + b[l]
        Z.append(z)
        if l < depth:
            H.append(bf16_round(silu(z)))
    pred = Z[-1]
    B = pred.shape[0]
    err = np.zeros_like(pred)
    err[:, :n_out] = pred[:, :n_out] - target[:, :n_out]
    loss = float((err[:, :n_out] ** 2).mean())
    d32 = 2.0 * err / (B * n_out)
    dW = [None] * (depth + 1)
    db = [None] * (depth + 1)
    for l in range(depth, -1, -1):
        d16 = bf16_round(d32)
        dW[l] = d16.T @ H[l]
        db[l] = d32.sum(axis=0)
        if l == 0:
            break
        d32 = (d16 @ W[l]) * silu_grad(Z[l - 1])
    return loss, pred, dW, db
