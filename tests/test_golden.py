"""Committed golden fixtures (tests/golden/, written by make_golden.py): the
exact Sod solution, and the oracle's state after fixed step counts of four
small configurations.  The oracle must reproduce its fixtures bit for bit;
the GPU path must match them at the parity bar (1e-10 relative L1)."""
import hashlib
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402

GOLD = os.path.join(HERE, "golden")


def _fixtures():
    return np.load(os.path.join(GOLD, "oracle_cases.npz"))


def test_exact_sod_fixture_is_the_exact_solution():
    f = np.load(os.path.join(GOLD, "sod_exact.npz"))
    x, rho, u, p = make_golden.sod_exact()
    assert np.array_equal(f["x"], x)
    assert np.array_equal(f["rho"], rho) and np.array_equal(f["u"], u) and np.array_equal(f["p"], p)


@pytest.mark.parametrize("name", sorted(make_golden.cases()))
def test_oracle_reproduces_its_fixture(name, ncpu):
    """The restatement is deterministic (each block on one thread): the same
    steps give the same bytes as when the fixture was written."""
    g = _fixtures()
    prob, steps = make_golden.cases()[name]
    assert int(g[f"{name}/steps"]) == steps
    U, state = make_golden.run_oracle(prob, steps, threads=ncpu)
    s = make_golden.summary(U)
    assert np.array_equal(s["sha256"], g[f"{name}/sha256"])
    assert np.array_equal(s["sum"], g[f"{name}/sum"])
    assert np.array_equal(state, g[f"{name}/state"])


def _rel_l1(a, b):
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(make_golden.cases()))
def test_gpu_matches_the_golden_fixture(name):
    from walicxe3d_b200.solver import from_problem
    g = _fixtures()
    prob, steps = make_golden.cases()[name]
    w = from_problem(prob)
    for _ in range(steps):
        w.step()
    U = w.download()
    assert np.all(np.isfinite(U))
    s = make_golden.summary(U)
    for e in range(U.shape[1]):
        assert _rel_l1(s["l1"][:, e], g[f"{name}/l1"][:, e]) <= 1e-10, (name, e)
        assert _rel_l1(s["plane"][e], g[f"{name}/plane"][e]) <= 1e-10, (name, e)
        ref = g[f"{name}/sum"][:, e]
        assert np.abs(s["sum"][:, e] - ref).sum() <= 1e-10 * g[f"{name}/l1"][:, e].sum(), (name, e)
    t, dt, it = g[f"{name}/state"]
    st = w.state
    assert st.it == int(it) and st.time == pytest.approx(t, rel=1e-12) and st.dt == pytest.approx(dt, rel=1e-10)


@pytest.mark.gpu
def test_gpu_sod_against_the_exact_fixture():
    """HLLC + minmod Sod tube on the GPU (8 blocks along x) against the exact
    solution at t = 0.15: density L1 error below the bar the oracle meets."""
    from walicxe3d_b200 import problems
    from walicxe3d_b200.solver import from_problem
    f = np.load(os.path.join(GOLD, "sod_exact.npz"))
    prob = problems.shock_tube(nblocks=8, axis=0, eta=0.0, t_end=0.15)
    w = from_problem(prob)
    for _ in range(5000):
        if w.state.time >= 0.15 - 1e-14:
            break
        w.step()
    assert abs(w.state.time - 0.15) < 1e-14
    U = w.download()
    order = np.argsort([prob.tree.coords(int(b))[1][0] for b in prob.local_blocks])
    rho = np.concatenate([U[n, 0].mean(axis=(0, 1)) for n in order])
    assert rho.shape == f["rho"].shape
    assert np.abs(rho - f["rho"]).mean() < 0.006
