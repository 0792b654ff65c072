"""CPU FP64 restatement of the flux emulator's MLP (forward, loss, backward).

TEST INFRASTRUCTURE ONLY: the checker of libdsp_emu.so's tensor-core forward
and backward passes.  It follows the GPU's data flow -- BF16 inputs, weights,
activations and gradients, wide accumulation -- with FP64 arithmetic, so the
comparison isolates accumulation order and GELU rounding, not BF16 storage.
"""
from __future__ import annotations

import math

import numpy as np


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """BF16 bit patterns (uint16) of x, rounded to nearest even."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack_params(flat: np.ndarray, dims: list) -> list:
    """[(W [out_pad][in_pad], b [out_pad])] from the parameter order of dsp_emu_get_params."""
    out, off = [], 0
    for in_pad, out_pad in dims:
        W = flat[off:off + out_pad * in_pad].reshape(out_pad, in_pad).astype(np.float64)
        off += out_pad * in_pad
        b = flat[off:off + out_pad].astype(np.float64)
        off += out_pad
        out.append((W, b))
    return out


def forward(params: list, X: np.ndarray) -> np.ndarray:
    """Predictions [B][out_pad] of BF16 inputs X (BF16 weights and activations)."""
    H = bf16_round(X)
    for W, b in params[:-1]:
        H = bf16_round(gelu(H @ bf16_round(W).T + b))
    W, b = params[-1]
    return H @ bf16_round(W).T + b


def forward_backward(params: list, X: np.ndarray, Y: np.ndarray, HW: np.ndarray, n_out: int, n_heads: int):
    """Loss sum and gradients of one batch.  X: BF16 values [B][in_pad]; Y [B][n_out];
    HW [B][n_heads].  Returns (loss_sum, [(dW, db)])."""
    B = X.shape[0]
    nl = len(params)
    Wb = [bf16_round(W) for W, _ in params]
    H = [X]
    Z = []
    for i in range(nl - 1):
        z = H[-1] @ Wb[i].T + params[i][1]
        Z.append(z)
        H.append(bf16_round(gelu(z)))
    P = H[-1] @ Wb[-1].T + params[-1][1]
    nreal = n_out * n_heads
    d = np.zeros_like(P)
    loss = 0.0
    gscale = 2.0 / (n_out * B)
    for h in range(n_heads):
        diff = P[:, h * n_out:(h + 1) * n_out] - Y
        w = HW[:, h:h + 1]
        d[:, h * n_out:(h + 1) * n_out] = gscale * w * diff
        loss += float(np.sum(w * diff * diff))
    d[:, nreal:] = 0.0
    dZ = bf16_round(d)
    grads = [None] * nl
    for i in range(nl - 1, -1, -1):
        grads[i] = (dZ.T @ H[i], dZ.sum(axis=0))
        if i > 0:
            dH = dZ @ Wb[i]
            dZ = bf16_round(dH * gelu_grad(Z[i - 1]))
    return loss, grads
