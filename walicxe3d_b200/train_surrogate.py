"""Trains the hydrogen-rate + cooling_h surrogate and builds its trust table.

    python -m walicxe3d_b200.train_surrogate [--n-train 20000000] [--n-test 8000000]

Samples come from the plain FP64 integrator on the GPU (wx3d_mlp_samples:
log-uniform n_H in [1e-3, 1e4] cm^-3, T in [1e2, 1e8] K, dt in [1e-2, 1e3] yr,
uniform x_HII); training runs the tcgen05 forward/backward kernels with Adam
(wx3d_mlp_train).  The trained network is then judged against the plain
integrator on a held-out set: per bin of (log10 n_H dt/yr, log10 T, x_HII)
the largest ionisation-fraction and temperature errors decide whether the
bin is trusted.  A second, independent set (another seed, half the size)
measures the errors the trusted region shows on cells it has not seen.

Writes ``data/surrogate_h.npz`` (params, trust table) and
``data/surrogate_h.json`` (loss curve, error statistics, trusted fraction)
next to this file.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import config as C
from .surrogate import LOG_DT, LOG_N, LOG_T, SCALE_C, SCALE_X, Surrogate, samples

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "surrogate_h")

# Trust table geometry (wx3d_set_surrogate): log10(n_H dt/yr) in [-5, 7) by
# 0.25, log10 T in [2, 8) by 0.125, x_HII in eighths.
TRUST_ND, TRUST_T, TRUST_X = 48, 48, 8
ND_LO, ND_W = -5.0, 0.25
T_LO, T_W = 2.0, 0.125

X_TOL = 1.0e-3      # absolute ionisation-fraction error
T_TOL = 1.0e-2      # relative temperature error
SEED_TRAIN, SEED_TEST, SEED_VAL = 20261203, 20261204, 20261205


def training_config() -> C.Config:
    """EOS_H_RATE + COOL_H with the reference's cooling_limit (0.5); the
    integrator's result does not depend on the unit scalings."""
    return C.Config(npassive=1, eos_type=C.EOS_H_RATE, cooling_type=C.COOL_H)


def bins(raw: np.ndarray) -> np.ndarray:
    """Flat trust-table index of each raw sample (n_H, T, x_HII, dt[s]),
    computed as the device gate does."""
    lgn = np.log10(raw[:, 0])
    lgT = np.log10(raw[:, 1])
    lgd = np.log10(raw[:, 3] / C.YR)
    bn = np.clip(np.floor((lgn + lgd - ND_LO) / ND_W).astype(np.int64), 0, TRUST_ND - 1)
    bt = np.clip(np.floor((lgT - T_LO) / T_W).astype(np.int64), 0, TRUST_T - 1)
    bx = np.clip((raw[:, 2] * TRUST_X).astype(np.int64), 0, TRUST_X - 1)
    return (bn * TRUST_T + bt) * TRUST_X + bx


def errors(pred: np.ndarray, tgt: np.ndarray, raw: np.ndarray):
    """Ionisation-fraction (absolute) and temperature (relative) errors of
    the surrogate's update against the plain integrator's, with the clamps
    the fused kernel applies (neutral fraction in [0, 1 - 1e-4], cooling
    factor in [0.5, 1]).  T1 = cf P0 / (k n_H (2 - y1))."""
    x0 = raw[:, 2]
    y1p = np.clip(1.0 - (x0 + pred[:, 0].astype(np.float64) * SCALE_X), 0.0, 1.0 - 1.0e-4)
    y1t = 1.0 - (x0 + tgt[:, 0].astype(np.float64) * SCALE_X)
    ex = np.abs(y1p - y1t)
    cfp = np.clip(10.0 ** (pred[:, 1].astype(np.float64) * SCALE_C), 0.5, 1.0)
    cft = 10.0 ** (tgt[:, 1].astype(np.float64) * SCALE_C)
    eT = np.abs(cfp / cft * (2.0 - y1t) / (2.0 - y1p) - 1.0)
    return ex, eT


def bin_max(ex, eT, b):
    """Sample count and largest errors of every trust-table bin."""
    n = TRUST_ND * TRUST_T * TRUST_X
    cnt = np.bincount(b, minlength=n)
    mx = np.zeros(n)
    mt = np.zeros(n)
    np.maximum.at(mx, b, ex)
    np.maximum.at(mt, b, eT)
    return cnt, mx, mt


def trust_table(ex, eT, b, margin: float = 0.75, min_count: int = 100) -> np.ndarray:
    """A bin is trusted when it holds at least min_count held-out samples,
    its largest errors are within margin x the tolerances, and so are those
    of its neighbours in log10(n_H dt) and log10 T (the trusted region is
    eroded by one bin, where the error surface changes fastest)."""
    cnt, mx, mt = bin_max(ex, eT, b)
    ok = (cnt >= min_count) & (mx <= margin * X_TOL) & (mt <= margin * T_TOL)
    ok3 = ok.reshape(TRUST_ND, TRUST_T, TRUST_X)
    pad = np.pad(ok3, ((1, 1), (1, 1), (0, 0)), constant_values=True)
    er = ok3.copy()
    for d0, d1 in ((-1, 0), (1, 0), (0, -1), (0, 1)):
        er &= pad[1 + d0:1 + d0 + TRUST_ND, 1 + d1:1 + d1 + TRUST_T]
    return er.reshape(-1).astype(np.uint8)


# (epochs, learning rate): the whole box, then two rounds on the bins the
# network can learn; after each stage the bins whose errors exceed the
# factor x the tolerances leave the training set
SCHEDULE_ALL = ((40, 3e-3), (40, 1e-3))
SCHEDULE_FOCUS = (
    (10.0, ((60, 1e-3), (60, 3e-4))),
    (3.0, ((80, 3e-4), (80, 1e-4), (60, 3e-5))),
)
TRUST_MARGIN = 0.6


def _bins_device(raw):
    import torch
    lgn = torch.log10(raw[:, 0])
    lgT = torch.log10(raw[:, 1])
    lgd = torch.log10(raw[:, 3] / C.YR)
    bn = torch.clamp(torch.floor((lgn + lgd - ND_LO) / ND_W), 0, TRUST_ND - 1).long()
    bt = torch.clamp(torch.floor((lgT - T_LO) / T_W), 0, TRUST_T - 1).long()
    bx = torch.clamp((raw[:, 2] * TRUST_X).long(), 0, TRUST_X - 1)
    return (bn * TRUST_T + bt) * TRUST_X + bx


def train(n_train: int, n_test: int, out: str, seed: int = 1, batch: int = 16384):
    import torch

    cfg = training_config()
    t0 = time.time()
    x, t, r = samples(cfg, n_train, seed=SEED_TRAIN, raw=True)
    xt, tt, rt = samples(cfg, 2 * n_test, seed=SEED_TEST, raw=True)
    xv, tv, rv = samples(cfg, n_test, seed=SEED_VAL, raw=True)
    t_samples = time.time() - t0
    s = Surrogate(seed=seed)

    def evaluate(xs, ts, rs):
        pred = s.forward(xs).cpu().numpy()
        raw = rs.cpu().numpy()
        ex, eT = errors(pred, ts.cpu().numpy(), raw)
        return ex, eT, bins(raw)

    losses = []
    t0 = time.time()
    for epochs, lr in SCHEDULE_ALL:
        losses += [float(v) for v in s.train(x, t, epochs, batch=batch, lr=lr)]
    # focus: drop the bins the network cannot learn to a useful accuracy
    dropped = np.zeros(TRUST_ND * TRUST_T * TRUST_X, bool)
    rb = _bins_device(r)
    del r
    for factor, sched in SCHEDULE_FOCUS:
        ex, eT, b = evaluate(xt, tt, rt)
        cnt, mx, mt = bin_max(ex, eT, b)
        dropped |= (mx > factor * X_TOL) | (mt > factor * T_TOL)
        keep = ~torch.from_numpy(dropped).to(x.device)[rb]
        x, t, rb = x[keep].contiguous(), t[keep].contiguous(), rb[keep].contiguous()
        for epochs, lr in sched:
            losses += [float(v) for v in s.train(x, t, epochs, batch=batch, lr=lr)]
    n_focus = int(x.shape[0])
    hopeless = dropped
    torch.cuda.synchronize()
    t_train = time.time() - t0

    ex, eT, b = evaluate(xt, tt, rt)
    table = trust_table(ex, eT, b, margin=TRUST_MARGIN)
    cnt, mx, mt = bin_max(ex, eT, b)
    exv, eTv, bv = evaluate(xv, tv, rv)
    inside = table[bv] != 0
    stats = {
        "n_train": n_train,
        "n_train_focus": n_focus,
        "n_test": 2 * n_test,
        "n_validation": n_test,
        "schedule_all": [list(e) for e in SCHEDULE_ALL],
        "schedule_focus": [[f, [list(e) for e in sc]] for f, sc in SCHEDULE_FOCUS],
        "trust_margin": TRUST_MARGIN,
        "hopeless_bins": int(hopeless.sum()),
        "batch": batch,
        "seconds_sampling": t_samples,
        "seconds_training": t_train,
        "loss_per_epoch": losses,
        "test_rms_x": float(np.sqrt((ex ** 2).mean())),
        "test_rms_T": float(np.sqrt((eT ** 2).mean())),
        "test_max_x": float(ex.max()),
        "test_max_T": float(eT.max()),
        "trusted_bins": int(table.sum()),
        "bins": int(table.size),
        "validation_trusted_fraction": float(inside.mean()),
        "validation_max_x_trusted": float(exv[inside].max()) if inside.any() else 0.0,
        "validation_max_T_trusted": float(eTv[inside].max()) if inside.any() else 0.0,
        "validation_p999_x_trusted": float(np.quantile(exv[inside], 0.999)) if inside.any() else 0.0,
        "tolerances": {"x_abs": X_TOL, "T_rel": T_TOL},
        "box": {"log_n": LOG_N, "log_T": LOG_T, "log_dt_yr": LOG_DT},
    }
    os.makedirs(os.path.dirname(out), exist_ok=True)
    shape = (TRUST_ND, TRUST_T, TRUST_X)
    np.savez(out + ".npz", params=s.params, trust=table.reshape(shape),
             bin_max_x=mx.reshape(shape).astype(np.float32), bin_max_T=mt.reshape(shape).astype(np.float32))
    with open(out + ".json", "w") as f:
        json.dump(stats, f, indent=1)
    return s, table, stats


def load(path: str = DEFAULT_OUT):
    """(params float32[NPARAM], trust uint8[48,48,8]) of a trained surrogate."""
    d = np.load(path + ".npz")
    return d["params"].astype(np.float32), d["trust"].astype(np.uint8)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n-train", type=int, default=20_000_000)
    ap.add_argument("--n-test", type=int, default=8_000_000)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args()
    _, table, stats = train(a.n_train, a.n_test, a.out, seed=a.seed, batch=a.batch)
    print(json.dumps({k: v for k, v in stats.items() if k != "loss_per_epoch"}, indent=1))
    print("final loss", stats["loss_per_epoch"][-1])


if __name__ == "__main__":
    main()
