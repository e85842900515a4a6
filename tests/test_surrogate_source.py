"""The surrogate inside the source step (wx3d_set_surrogate): gate and
per-cell fallback, accuracy of the trained network against the plain FP64
integrator, and the ablation of its speed against the plain source step."""
import os

import numpy as np
import pytest

from walicxe3d_b200 import config as C

pytestmark = pytest.mark.gpu

MU0 = 1.3
TRUST_SHAPE = (48, 48, 8)


def _cfg(nblocks, cooling=C.COOL_H):
    return C.Config(npassive=1, solver_type=C.SOLVER_HLLC, limiter_type=C.LIMITER_MINMOD,
                    eos_type=C.EOS_H_RATE, cooling_type=cooling, nbroot=(nblocks, 1, 1), maxlev=1,
                    l_sc=C.PC, d_sc=MU0 * C.AMU, v_sc=1.0e5, box=(float(nblocks) * C.PC, C.PC, C.PC))


def _cells(nblocks, seed, lo=(-3.0, 2.0), hi=(4.0, 8.0)):
    """nblocks blocks of cells at rest with log-uniform n_H, T and uniform x_HII."""
    rng = np.random.default_rng(seed)
    n = nblocks * C.BLOCK_CELLS
    lgn = rng.uniform(lo[0], hi[0], n)
    lgT = rng.uniform(lo[1], hi[1], n)
    x = rng.uniform(0.0, 1.0, n)
    return 10.0 ** lgn, 10.0 ** lgT, x


def _context(cfg, nblocks, n, T, x, dt_yr):
    from walicxe3d_b200 import problems
    from walicxe3d_b200.solver import Walicxe3D
    w = Walicxe3D(cfg, nblocks)
    w.set_mesh(np.arange(1, nblocks + 1))
    if cfg.cooling_type == C.COOL_TABLE:
        w.set_cooltable(*problems.cooling_table_synthetic())
    y = 1.0 - x
    U = np.zeros((nblocks, 6) + (16, 16, 16))
    sh = (nblocks, 16, 16, 16)
    U[:, 0] = (n * MU0).reshape(sh)
    U[:, 4] = (cfg.cv * T * C.KB * n * (2.0 - y) / cfg.p_sc).reshape(sh)
    U[:, 5] = (n * y).reshape(sh)
    w.upload(U)
    w.set_state(time=0.0, dt=dt_yr * C.YR / cfg.t_sc, it=10, nextout=1)
    return w


def _x_T(U, cfg):
    """(x_HII, T) of every cell of a state at rest."""
    rho, E, nh0 = U[:, 0].ravel(), U[:, 4].ravel(), U[:, 5].ravel()
    dh = rho / MU0
    y = nh0 / dh
    P = E / cfg.cv
    return 1.0 - y, P * cfg.p_sc / (C.KB * dh * (2.0 - y))


def _trained():
    from walicxe3d_b200.train_surrogate import DEFAULT_OUT, load
    if not os.path.exists(DEFAULT_OUT + ".npz"):
        pytest.fail("the trained surrogate (walicxe3d_b200/data/surrogate_h.npz) is missing")
    return load()


def test_all_fallback_is_the_plain_step():
    """With an all-zero trust table every cell takes the plain integrator:
    the fused surrogate kernel then reproduces the plain source step bit for
    bit, and counts every cell as a fallback."""
    from walicxe3d_b200.surrogate import NPARAM
    cfg = _cfg(2)
    n, T, x = _cells(2, seed=4)
    a = _context(cfg, 2, n, T, x, 10.0)
    b = _context(cfg, 2, n, T, x, 10.0)
    b.attach_surrogate(np.zeros(NPARAM, np.float32), np.zeros(TRUST_SHAPE, np.uint8))
    ma = a.sources()
    mb = b.sources()
    assert ma == mb
    assert np.array_equal(a.download(), b.download())
    st = b.status()
    assert st.surrogate_cells == 0 and st.fallback_cells == 2 * C.BLOCK_CELLS
    assert a.get_timestep() == b.get_timestep()


def test_all_fallback_run_matches_plain_run():
    """Full main-loop iterations (CUDA graph) of the radiative SNR with the
    surrogate attached but nothing trusted: identical to the plain run."""
    from walicxe3d_b200 import problems
    from walicxe3d_b200.solver import from_problem
    from walicxe3d_b200.surrogate import NPARAM
    prob = problems.snr_h(nroot=2, maxlev=2)
    a = from_problem(prob)
    b = from_problem(prob)
    b.attach_surrogate(np.zeros(NPARAM, np.float32), np.zeros(TRUST_SHAPE, np.uint8))
    sa = a.run(6)
    sb = b.run(6)
    assert sa.time == sb.time and sa.dt == sb.dt
    assert np.array_equal(a.download(), b.download())
    st = b.status()
    assert st.surrogate_cells == 0 and st.fallback_cells == 6 * prob.nblocks * C.BLOCK_CELLS


def test_invalid_surrogate_arguments():
    from walicxe3d_b200._lib import WxError
    from walicxe3d_b200.surrogate import NPARAM
    cfg = _cfg(1)
    n, T, x = _cells(1, seed=1)
    w = _context(cfg, 1, n, T, x, 1.0)
    with pytest.raises(WxError) as e:
        w.attach_surrogate(np.zeros(NPARAM, np.float32), np.zeros(10, np.uint8))
    assert e.value.code == 103
    adi = _context(C.Config(npassive=1, eos_type=C.EOS_ADIABATIC, nbroot=(1, 1, 1)), 1, n, T, x, 1.0)
    with pytest.raises(WxError) as e:
        adi.attach_surrogate(np.zeros(NPARAM, np.float32), np.zeros(TRUST_SHAPE, np.uint8))
    assert e.value.code == 104


@pytest.mark.parametrize("dt_yr", [0.03, 0.3, 3.0, 30.0, 300.0])
def test_trained_surrogate_within_tolerance(dt_yr):
    """Trained network against the plain FP64 integrator, cell by cell,
    over the whole input box: gated cells within |dx_HII| <= 1e-3 and
    |dT/T| <= 1 %, every other cell bit-identical to the plain step."""
    params, trust = _trained()
    nb = 4
    cfg = _cfg(nb)
    n, T, x = _cells(nb, seed=int(dt_yr * 1000) + 17)
    plain = _context(cfg, nb, n, T, x, dt_yr)
    sur = _context(cfg, nb, n, T, x, dt_yr)
    sur.attach_surrogate(params, trust)
    plain.sources()
    sur.sources()
    Up, Us = plain.download(), sur.download()
    xp, Tp = _x_T(Up, cfg)
    xs, Ts = _x_T(Us, cfg)
    ex = np.abs(xs - xp)
    eT = np.abs(Ts / Tp - 1.0)
    same = (Up == Us).all(axis=1).ravel()
    st = sur.status()
    assert st.surrogate_cells + st.fallback_cells == nb * C.BLOCK_CELLS
    assert st.fallback_cells <= int(same.sum())
    assert ex.max() <= 1.0e-3
    assert eT.max() <= 1.0e-2
    # density and momenta are never touched
    assert np.array_equal(Up[:, :4], Us[:, :4])


def test_trained_surrogate_covers_the_box():
    """The trust table admits a real share of the input box."""
    import json
    from walicxe3d_b200.train_surrogate import DEFAULT_OUT
    _, trust = _trained()
    with open(DEFAULT_OUT + ".json") as f:
        stats = json.load(f)
    assert trust.shape == TRUST_SHAPE
    assert stats["validation_max_x_trusted"] <= 1.0e-3
    assert stats["validation_max_T_trusted"] <= 1.0e-2
    assert stats["validation_trusted_fraction"] > 0.1


def test_surrogate_ablation_speed():
    """Ablation: the fused source step with and without the network on the
    same 1,024 blocks of hot cells (T from 3e4 to 3e7 K, where the plain
    step evaluates the full Biro et al. loss function), timed with CUDA
    events around the source kernel.  Prints both times and the share of
    cells the network handled; the surrogate path must stay within
    tolerance either way."""
    params, trust = _trained()
    nb = 1024
    cfg = _cfg(nb)
    n, T, x = _cells(nb, seed=99, lo=(-1.0, 4.5), hi=(2.0, 7.5))
    plain = _context(cfg, nb, n, T, x, 10.0)
    sur = _context(cfg, nb, n, T, x, 10.0)
    sur.attach_surrogate(params, trust)

    def timed(w, reps=5):
        w.set_timing(True)
        best = 1e30
        for _ in range(reps):
            w.upload(U0)
            w.set_state(time=0.0, dt=10.0 * C.YR / cfg.t_sc, it=10, nextout=1)
            w.sources()
            ms, cnt = w.kernel_times()
            best = min(best, ms[3])
        return best

    U0 = plain.download()
    tp = timed(plain)
    sur.reset_status()
    ts = timed(sur)
    st = sur.status()
    frac = st.surrogate_cells / max(1, st.surrogate_cells + st.fallback_cells)
    print(f"\nablation: plain {tp:.3f} ms, surrogate {ts:.3f} ms, gain {tp / ts:.2f}x, "
          f"surrogate share {frac:.3f}")
    # accuracy of the timed surrogate step against the plain one
    xp, Tp = _x_T(plain.download(), cfg)
    xs, Ts = _x_T(sur.download(), cfg)
    assert np.abs(xs - xp).max() <= 1.0e-3
    assert np.abs(Ts / Tp - 1.0).max() <= 1.0e-2


def test_ionisation_surrogate_all_fallback_is_the_plain_step():
    """EOS_H_RATE with table cooling (the colliding-winds physics): with an
    all-zero trust table the fused kernel runs the plain hrate update and
    the plain table cooling for every cell, bit for bit as the plain source
    step."""
    from walicxe3d_b200.surrogate import NPARAM
    cfg = _cfg(2, cooling=C.COOL_TABLE)
    n, T, x = _cells(2, seed=5)
    a = _context(cfg, 2, n, T, x, 10.0)
    b = _context(cfg, 2, n, T, x, 10.0)
    b.attach_surrogate(np.zeros(NPARAM, np.float32), np.zeros(TRUST_SHAPE, np.uint8))
    assert a.sources() == b.sources()
    assert np.array_equal(a.download(), b.download())
    st = b.status()
    assert st.surrogate_cells == 0 and st.fallback_cells == 2 * C.BLOCK_CELLS


@pytest.mark.parametrize("dt_yr", [0.3, 30.0])
def test_ionisation_surrogate_within_tolerance(dt_yr):
    """The trained network's x_HII output in place of the hrate update,
    followed by the plain table cooling: gated cells within |dx_HII| <= 1e-3
    and |dT/T| <= 1 % of the plain step, the others bit-identical."""
    params, trust = _trained()
    nb = 4
    cfg = _cfg(nb, cooling=C.COOL_TABLE)
    n, T, x = _cells(nb, seed=int(dt_yr * 100) + 3)
    plain = _context(cfg, nb, n, T, x, dt_yr)
    sur = _context(cfg, nb, n, T, x, dt_yr)
    sur.attach_surrogate(params, trust)
    plain.sources()
    sur.sources()
    Up, Us = plain.download(), sur.download()
    xp, Tp = _x_T(Up, cfg)
    xs, Ts = _x_T(Us, cfg)
    same = (Up == Us).all(axis=1).ravel()
    st = sur.status()
    assert st.surrogate_cells > 0
    assert st.fallback_cells <= int(same.sum())
    assert np.abs(xs - xp).max() <= 1.0e-3
    assert np.abs(Ts / Tp - 1.0).max() <= 1.0e-2
    assert np.array_equal(Up[:, :4], Us[:, :4])


@pytest.mark.parametrize("cooling", [C.COOL_H, C.COOL_TABLE])
def test_dt_outside_the_training_box_is_the_plain_step(cooling):
    """A time step below the training box (1e-3 yr, as in the reference's
    dt ramp of a fast-wind run): the trained network is attached but no cell
    is gated in; the kernel integrates every cell directly, bit for bit as
    the plain source step."""
    params, trust = _trained()
    cfg = _cfg(2, cooling=cooling)
    n, T, x = _cells(2, seed=8)
    a = _context(cfg, 2, n, T, x, 1.0e-3)
    b = _context(cfg, 2, n, T, x, 1.0e-3)
    b.attach_surrogate(params, trust)
    assert a.sources() == b.sources()
    assert np.array_equal(a.download(), b.download())
    st = b.status()
    assert st.surrogate_cells == 0 and st.fallback_cells == 2 * C.BLOCK_CELLS
