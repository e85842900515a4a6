"""FP64 reference of the surrogate MLP -- TEST INFRASTRUCTURE.

Checker for the tcgen05 kernels of walicxe3d_b200/csrc/wx3d_mlp.cu: forward
pass, mean-squared-error loss and its gradient in NumPy FP64.  With
quant=True the roundings of the GPU path are applied: the forward hidden
layers as BF16 head/tail products (hi*hi + lo*hi + hi*lo), the FP32 output
layer unrounded, and the backward products with BF16 operands, so the GPU
result must match to FP32 round-off; with quant=False the result is the
exact FP64 forward pass and gradient of the network.
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


def split(a):
    """BF16 head and tail of a: hi = bf16(a), lo = bf16(a - hi)."""
    a32 = np.asarray(a, dtype=np.float32)
    hi = bf16(a32)
    lo = bf16((a32.astype(np.float64) - hi).astype(np.float32))
    return hi, lo


def _split_mm(a, w):
    """The three-product head/tail sum hi*hi + lo*hi + hi*lo of the GPU
    forward layers (the lo*lo product is not formed)."""
    ah, al = split(a)
    wh, wl = split(w)
    return ah @ wh + al @ wh + ah @ wl


def forward(p, x, quant: bool = True):
    w = unpack(p)
    if quant:
        z1 = _split_mm(x, w["W1"]) + w["b1"]
        h1 = _silu(z1)
        z2 = _split_mm(h1, w["W2"]) + w["b2"]
    else:
        X = np.asarray(x, np.float64)
        z1 = X @ w["W1"] + w["b1"]
        h1 = _silu(z1)
        z2 = h1 @ w["W2"] + w["b2"]
    h2 = _silu(z2)
    # the 64 -> 2 output layer runs in FP32 on the CUDA cores: no rounding
    y = h2 @ w["W3"] + w["b3"]
    return y, (np.asarray(x, np.float64), z1, h1, z2, h2, w["W1"], w["W2"], w["W3"])


def loss_grad(p, x, t, quant: bool = True):
    n = x.shape[0]
    q = bf16 if quant else (lambda a: np.asarray(a, np.float64))
    y, (X, z1, h1, z2, h2, W1, W2, W3) = forward(p, x, quant)
    e = y - t
    loss = (e * e).sum() / n
    # backward products are single BF16 tensor-core MMAs
    dy = q(2.0 * e / n)
    dz2 = q((dy @ q(W3).T) * _dsilu(z2))
    dz1 = q((dz2 @ q(W2).T) * _dsilu(z1))
    g = np.concatenate([(q(X).T @ dz1).ravel(), dz1.sum(0), (q(h1).T @ dz2).ravel(), dz2.sum(0),
                        (q(h2).T @ dy).ravel(), dy.sum(0)])
    return loss, g
