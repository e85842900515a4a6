"""Writes the golden fixtures of tests/test_golden.py.

    python tests/golden/make_golden.py

* sod_exact.npz -- the exact Riemann solution (Toro ch. 4, tests/exact_riemann.py)
  of the Sod problem at t = 0.15 on 128 cell centres: an analytic pin that
  no code path of the library or the oracle produced.
* oracle_cases.npz -- the CPU oracle's state after a fixed number of
  main-loop steps of four small configurations (single-level Sedov, Brio-Wu
  with HLLD, the radiative SNR with hrate + cooling_h, a three-level AMR
  blast): per-block and per-equation sums and L1 norms, one plane of one
  block, the SHA-256 of the whole state, and time/dt/it.  They pin the
  restatement against later changes; the GPU is compared with them at the
  parity bar.

The reference itself cannot run here (no Fortran compiler), so these are
the only recorded outputs.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from walicxe3d_b200 import problems  # noqa: E402

from exact_riemann import sample  # noqa: E402

SOD = dict(t=0.15, x0=0.5, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1), gamma=1.4, n=128)


def cases():
    """name -> (problem, steps)."""
    return {
        "sedov64": (problems.sedov(4), 20),
        "brio_wu": (problems.brio_wu(4), 20),
        "snr_h": (problems.snr_h(nroot=2, maxlev=2), 6),
        "amr3": (problems.blast_amr(nroot=3, maxlev=3, shell_radius=0.1, shell_width=0.02), 10),
    }


def summary(U: np.ndarray) -> dict:
    """Fixture entries of a state [nb, neq, 16, 16, 16]."""
    U = np.ascontiguousarray(U)
    nb = U.shape[0]
    return {
        "sum": U.sum(axis=(2, 3, 4)),
        "l1": np.abs(U).sum(axis=(2, 3, 4)),
        "plane": U[nb // 2, :, 8].copy(),
        "sha256": np.frombuffer(hashlib.sha256(U.tobytes()).digest(), np.uint8),
    }


def run_oracle(prob, steps: int, threads: int | None = None):
    o = oracle.from_problem(prob, threads=threads or os.cpu_count())
    for _ in range(steps):
        o.step()
    st = o.state
    return o.U[: prob.nblocks], np.array([st.time, st.dt, st.it], np.float64)


def sod_exact():
    n = SOD["n"]
    x = (np.arange(n) + 0.5) / n
    rho, u, p = sample(x, SOD["t"], SOD["x0"], *SOD["left"], *SOD["right"], SOD["gamma"])
    return x, rho, u, p


def main():
    x, rho, u, p = sod_exact()
    np.savez_compressed(os.path.join(HERE, "sod_exact.npz"), x=x, rho=rho, u=u, p=p)
    out = {}
    for name, (prob, steps) in cases().items():
        U, state = run_oracle(prob, steps)
        for k, v in summary(U).items():
            out[f"{name}/{k}"] = v
        out[f"{name}/state"] = state
        out[f"{name}/steps"] = np.array(steps)
    np.savez_compressed(os.path.join(HERE, "oracle_cases.npz"), **out)


if __name__ == "__main__":
    main()
