"""FP64 reference of the surrogate MLP -- TEST INFRASTRUCTURE.

Checker for the tcgen05 kernels of walicxe3d_b200/csrc/wx3d_mlp.cu: forward
pass, mean-squared-error loss and its gradient in NumPy FP64.  With
quant=True the BF16 roundings of the GPU path (inputs, weights, activations
and the back-propagated gradients, at the points where they enter a tensor
core product) are applied, so the GPU result must match to FP32 round-off;
with quant=False the result is the exact FP64 gradient of the BF16-rounded
network.
"""
from __future__ import annotations

import numpy as np

from walicxe3d_b200.surrogate import unpack


def bf16(a) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    a32 = np.asarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x, quant: bool = True):
    w = unpack(p)
    q = bf16 if quant else (lambda a: np.asarray(a, np.float64))
    W1, W2, W3 = q(w["W1"]), q(w["W2"]), q(w["W3"])
    X = q(x)
    z1 = X @ W1 + w["b1"]
    h1 = q(_silu(z1))
    z2 = h1 @ W2 + w["b2"]
    h2 = q(_silu(z2))
    y = h2 @ W3 + w["b3"]
    return y, (X, z1, h1, z2, h2, W1, W2, W3)


def loss_grad(p, x, t, quant: bool = True):
    n = x.shape[0]
    q = bf16 if quant else (lambda a: np.asarray(a, np.float64))
    y, (X, z1, h1, z2, h2, W1, W2, W3) = forward(p, x, quant)
    e = y - t
    loss = (e * e).sum() / n
    dy = q(2.0 * e / n)
    dz2 = q((dy @ W3.T) * _dsilu(z2))
    dz1 = q((dz2 @ W2.T) * _dsilu(z1))
    g = np.concatenate([(X.T @ dz1).ravel(), dz1.sum(0), (h1.T @ dz2).ravel(), dz2.sum(0),
                        (h2.T @ dy).ravel(), dy.sum(0)])
    return loss, g
