"""Learned surrogate of the hydrogen-rate + cooling_h update.

Host mirror of the wx3d_mlp_* entry points (include/wx3d.h): a 4-64-64-2
SiLU MLP, BF16 operands with FP32 accumulation, whose hidden layers (split
into BF16 head and tail in the forward pass), backward and weight-gradient
products run as tcgen05 tensor-core MMAs; the output layer is FP32.  Device buffers are
torch CUDA tensors (plumbing only); every computation runs in libwx3d.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .config import Config, WxConfig

NIN, NH, NOUT = 4, 64, 2
NPARAM = NIN * NH + NH + NH * NH + NH + NH * NOUT + NOUT

# Trust box of the surrogate (normalisation of its inputs)
LOG_N = (-3.0, 4.0)      # log10 n_H [cm^-3]
LOG_T = (2.0, 8.0)       # log10 T [K]
LOG_DT = (-2.0, 3.0)     # log10 dt [yr]
# Outputs: delta x_HII / SCALE_X and log10(cf) / SCALE_C, where the cooling
# factor cf = P1/P0 is the pressure ratio of the step
SCALE_X = 0.125
SCALE_C = 0.30102999566398120


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def unpack(p: np.ndarray) -> dict:
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = {}
    for name, shape in (("W1", (NIN, NH)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)),
                        ("W3", (NH, NOUT)), ("b3", (NOUT,))):
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


class Surrogate:
    """One MLP with its optimiser state on the current CUDA device."""

    def __init__(self, seed: int = 0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self.lib.wx3d_mlp_create(ctypes.c_uint64(seed), ctypes.byref(h)), "wx3d_mlp_create")
        self.h = h
        assert self.lib.wx3d_mlp_nparams() == NPARAM

    def close(self):
        if self.h:
            self.lib.wx3d_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(NPARAM, np.float32)
        _lib.check(self.lib.wx3d_mlp_get_params(self.h, _fp(p)), "wx3d_mlp_get_params")
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == NPARAM
        _lib.check(self.lib.wx3d_mlp_set_params(self.h, _fp(p)), "wx3d_mlp_set_params")

    def forward(self, x):
        import torch
        out = torch.empty((x.shape[0], NOUT), dtype=torch.float32, device=x.device)
        _lib.check(self.lib.wx3d_mlp_forward(self.h, x.shape[0], _vp(x), _vp(out), None), "wx3d_mlp_forward")
        return out

    def gradient(self, x, t):
        loss = ctypes.c_float()
        g = np.zeros(NPARAM, np.float32)
        _lib.check(self.lib.wx3d_mlp_gradient(self.h, x.shape[0], _vp(x), _vp(t), ctypes.byref(loss), _fp(g)),
                   "wx3d_mlp_gradient")
        return loss.value, g

    def train(self, x, t, epochs: int, batch: int = 16384, lr: float = 2e-3):
        losses = np.zeros(epochs, np.float32)
        _lib.check(self.lib.wx3d_mlp_train(self.h, x.shape[0], _vp(x), _vp(t), int(epochs), int(batch),
                                           ctypes.c_float(lr), _fp(losses)), "wx3d_mlp_train")
        return losses


def samples(cfg: Config, n: int, seed: int = 20261203, raw: bool = False):
    """n training samples from the plain FP64 integrator (GPU): normalised
    inputs [n,4], targets [n,2] and optionally raw (n_H, T, x_HII, dt[s])."""
    import torch
    lib = _lib.load()
    x = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    t = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    r = torch.empty((n, 4), dtype=torch.float64, device="cuda") if raw else None
    c = cfg.to_c()
    _lib.check(lib.wx3d_mlp_samples(ctypes.byref(c), n, ctypes.c_uint64(seed), _vp(x), _vp(t),
                                    _vp(r) if raw else None, None), "wx3d_mlp_samples")
    return (x, t, r) if raw else (x, t)
