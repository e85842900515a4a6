"""GPU path (libwx3d.so through the C-ABI) against the CPU oracle.

Bar: relative L1 difference per conserved variable <= 1e-10 after the
stated step count (FP64 everywhere; differences come only from FMA
contraction and reciprocal-multiply rewrites of the same formulas).
"""
import numpy as np
import pytest

import oracle
from walicxe3d_b200 import config as C
from walicxe3d_b200 import problems
from walicxe3d_b200.mesh import BlockTree
from walicxe3d_b200.solver import Walicxe3D, from_problem

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel_l1(a, b):
    """Per-equation relative L1 difference, arrays [nb, neq, ...]."""
    out = []
    for e in range(a.shape[1]):
        den = np.abs(b[:, e]).sum()
        num = np.abs(a[:, e] - b[:, e]).sum()
        out.append(num / den if den > 0 else num)
    return np.array(out)


def run_both(prob, nsteps, ncpu, use_run=False):
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    for _ in range(nsteps):
        o.step()
    if use_run:
        g.run(nsteps)
    else:
        for _ in range(nsteps):
            g.step()
    return o, g


def check(o, g, prob, tol=TOL):
    Ug = g.download()
    Uo = o.U[: prob.nblocks]
    err = rel_l1(Ug, Uo)
    assert np.all(np.isfinite(Ug))
    assert err.max() <= tol, f"rel L1 per eq {err}"
    so, sg = o.state, g.state
    assert sg.it == so.it
    assert sg.time == pytest.approx(so.time, rel=1e-12)
    assert sg.dt == pytest.approx(so.dt, rel=1e-10)
    return err


def small_amr(nroot=3, levels=3, solver=C.SOLVER_HLLC, limiter=C.LIMITER_MINMOD):
    """A balanced three-level mesh around the box centre (132 blocks:
    20 / 48 / 64 per level)."""
    prob = problems.blast_amr(nroot=nroot, maxlev=levels, shell_radius=0.1, shell_width=0.02, solver=solver,
                              limiter=limiter)
    return prob


def inject(father):
    """refineBlock's copy (amr.f90:355-367) of a [neq,16,16,16] father block
    into its 8 children, natural order."""
    out = []
    for c in range(8):
        sx, sy, sz = c & 1, (c >> 1) & 1, c >> 2
        idx = lambda s: 8 * s + (np.arange(16) + 2) // 2 - 1   # 0-based of 8s + (i+1)/2
        out.append(father[:, idx(sz)][:, :, idx(sy)][:, :, :, idx(sx)])
    return out


def average8(kids):
    """coarseBlocks' average (amr.f90:1619): Fortran SUM over each 2x2x2
    section in array order (i fastest), divided by 8."""
    f = np.empty_like(kids[0])
    for c, a in enumerate(kids):
        sx, sy, sz = c & 1, (c >> 1) & 1, c >> 2
        s = a[:, 0::2, 0::2, 0::2].copy()
        for (dk, dj, di) in [(0, 0, 1), (0, 1, 0), (0, 1, 1), (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1)]:
            s = s + a[:, dk::2, dj::2, di::2]
        f[:, 8 * sz:8 * sz + 8, 8 * sy:8 * sy + 8, 8 * sx:8 * sx + 8] = s / 8.0
    return f


def test_sedov_hllc_minmod_50_steps(ncpu):
    prob = problems.sedov(4)
    o, g = run_both(prob, 50, ncpu)
    check(o, g, prob)


@pytest.mark.parametrize("limiter", [C.LIMITER_NO_AVERAGE, C.LIMITER_NONE, C.LIMITER_MINMOD, C.LIMITER_VANLEER,
                                     C.LIMITER_UMIST, C.LIMITER_WOODWARD, C.LIMITER_SUPERBEE])
def test_limiters_hllc(limiter, ncpu):
    prob = problems.smooth_pulse(2, limiter=limiter)
    o, g = run_both(prob, 15, ncpu)
    assert o.counters()[:3] == [0, 0, 0]
    check(o, g, prob)


@pytest.mark.parametrize("limiter", [C.LIMITER_MINMOD, C.LIMITER_VANLEER, C.LIMITER_SUPERBEE])
def test_limiters_on_strong_blast(limiter, ncpu):
    prob = problems.sedov(2, limiter=limiter)
    o, g = run_both(prob, 15, ncpu)
    check(o, g, prob)


def test_albada_limiter_fails_like_the_reference(ncpu):
    """The reference marks LIMITER_ALBADA "NOT WORKING" (hydro_core.f90:669):
    its formula is 0/0 where both slopes vanish.  The oracle goes non-finite
    and the GPU path reports WX_ERR_NAN instead of returning garbage."""
    from walicxe3d_b200 import WxError
    prob = problems.smooth_pulse(2, limiter=C.LIMITER_ALBADA)
    o = oracle.from_problem(prob, threads=ncpu)
    o.step()
    assert not np.all(np.isfinite(o.U))
    g = from_problem(prob)
    with pytest.raises(WxError) as ei:
        g.step()
    assert ei.value.code == 102


@pytest.mark.parametrize("solver", [C.SOLVER_HLL, C.SOLVER_HLL1, C.SOLVER_LAX])
def test_other_hydro_solvers(solver, ncpu):
    prob = problems.sedov(2, solver=solver, limiter=C.LIMITER_VANLEER)
    o, g = run_both(prob, 15, ncpu)
    check(o, g, prob)


@pytest.mark.parametrize("solver", [C.SOLVER_HLL, C.SOLVER_HLL1, C.SOLVER_LAX, C.SOLVER_HLLC])
def test_hydro_solvers_smooth(solver, ncpu):
    prob = problems.smooth_pulse(2, solver=solver, limiter=C.LIMITER_VANLEER)
    o, g = run_both(prob, 15, ncpu)
    check(o, g, prob)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_shock_tube_each_axis(axis, ncpu):
    prob = problems.shock_tube(nblocks=4, axis=axis, eta=5e-3, t_end=10.0)
    o, g = run_both(prob, 40, ncpu)
    check(o, g, prob)


@pytest.mark.parametrize("solver", [C.SOLVER_HLLD, C.SOLVER_HLLE, C.SOLVER_HLL])
def test_brio_wu_mhd(solver, ncpu):
    prob = problems.brio_wu(8)
    prob.cfg.solver_type = solver
    o, g = run_both(prob, 40, ncpu)
    check(o, g, prob)


def test_amr_three_levels_cross_level_ghosts(ncpu):
    prob = small_amr()
    levels = {prob.tree.level(int(b)) for b in prob.local_blocks}
    assert levels == {1, 2, 3}
    o, g = run_both(prob, 20, ncpu)
    check(o, g, prob)


def test_neighbour_table_matches_reference_queries(ncpu):
    prob = small_amr()
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    ft, fs = g.neighbours()
    slot = {int(b): s for s, b in enumerate(prob.local_blocks)}
    for s, b in enumerate(prob.local_blocks):
        for f in range(6):
            t, lst = o.neighbors(int(b), f + 1)
            assert ft[s, f] == t
            if t in (C.NEIGH_SAME, C.NEIGH_COARSER):
                assert fs[s, f, 0] == slot[int(lst[0])]
            elif t == C.NEIGH_FINER:
                assert list(fs[s, f]) == [slot[int(v)] for v in lst]


def test_reflective_boundaries(ncpu):
    prob = problems.sedov(2)
    prob.cfg.bc = (C.BC_REFLECTIVE,) * 6
    # move the blast off-centre so it hits the walls
    prob.U = np.roll(prob.U, 1, axis=0)
    o, g = run_both(prob, 25, ncpu)
    check(o, g, prob)


def test_graph_replay_equals_single_steps(ncpu):
    prob = problems.sedov(2)
    g1 = from_problem(prob)
    for _ in range(12):
        g1.step()
    g2 = from_problem(prob)
    g2.run(12)
    assert np.array_equal(g1.download(), g2.download())
    s1, s2 = g1.state, g2.state
    assert (s1.time, s1.dt, s1.it) == (s2.time, s2.dt, s2.it)


def test_run_matches_oracle(ncpu):
    prob = small_amr(solver=C.SOLVER_HLL, limiter=C.LIMITER_VANLEER)
    o, g = run_both(prob, 11, ncpu, use_run=True)
    check(o, g, prob)


def test_snr_hydrogen_rate_and_cooling_h(ncpu):
    prob = problems.snr_h(nroot=2, maxlev=2)
    o, g = run_both(prob, 12, ncpu)
    check(o, g, prob)


def test_table_cooling(ncpu):
    prob = problems.sedov(2)
    cfg = prob.cfg
    cfg.eos_type = C.EOS_SINGLE_SPECIE
    cfg.cooling_type = C.COOL_TABLE
    cfg.l_sc, cfg.d_sc, cfg.v_sc = C.PC, 1.3 * C.AMU, 1.0e5
    cfg.box = (C.PC,) * 3
    # temperatures from ~1e3 K to ~1e8 K across the blast
    prob.U = prob.U.copy()
    prob.U[:, 4] *= 1.0e2
    prob.U[:, 4] += 0.02
    prob.cooltable = problems.cooling_table_synthetic(200)
    o, g = run_both(prob, 10, ncpu)
    check(o, g, prob)


def test_separate_calls_equal_fused_step(ncpu):
    """hydroSolver; updatePrims; updateNeutralFraction; cooling as separate
    C-ABI calls (main.f90:91-100) against the oracle's main-loop body."""
    prob = problems.snr_h(nroot=2, maxlev=1)
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    for it in range(1, 6):
        o.step()
        st = g.state
        g.set_state(st.time, st.dt, st.it + 1, st.nextout, 0)
        g.hydro_solver()
        g.update_prims()
        g.update_neutral_fraction()
        g.cooling()
    err = rel_l1(g.download(), o.U[: prob.nblocks])
    assert err.max() <= TOL, err


def test_get_timestep_matches_oracle(ncpu):
    prob = small_amr()
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    for it in (1, 5, 11):
        o.set_state(0.0, 0.0, it, 1, 0)
        g.set_state(0.0, 0.0, it, 1, 0)
        assert g.get_timestep() == pytest.approx(o.get_timestep(), rel=1e-13)


def test_update_prims_matches_oracle(ncpu):
    prob = problems.snr_h(nroot=2, maxlev=1)
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    g.update_prims()
    err = rel_l1(g.prims(), o.PRIM[: prob.nblocks])
    assert err.max() <= 1e-14, err


def test_fortran_layout_roundtrip():
    prob = problems.sedov(2)
    g = from_problem(prob)
    nbmax = prob.nblocks + 3
    F = np.zeros((nbmax, 5, 20, 20, 20), order="F")
    F[:] = -7.0
    g.download_fortran(F)
    # physical cells equal the native array; ghosts untouched
    for s in range(prob.nblocks):
        for e in range(5):
            phys = F[s, e, 2:18, 2:18, 2:18]          # Fortran (i, j, k)
            assert np.array_equal(phys, prob.U[s, e].transpose(2, 1, 0))
    assert np.all(F[:, :, 0:2] == -7.0)
    g2 = Walicxe3D(prob.cfg, nbmax)
    g2.set_mesh(prob.local_blocks)
    g2.upload_fortran(F)
    assert np.array_equal(g2.download(prob.nblocks), prob.U)


def test_mark_refine_coarsen(ncpu):
    prob = small_amr()
    o = oracle.from_problem(prob, threads=ncpu, extra_slots=16)
    g = from_problem(prob, extra_slots=16)
    for _ in range(3):
        o.step()
        g.step()
    fo = o.mark()[: prob.nblocks]
    fg = g.mark()[: prob.nblocks]
    assert np.array_equal(fo, fg)
    assert set(np.unique(fg)) <= {0, 1, 2}
    # refine the first level-2 block into 8 free slots, then coarsen back
    lv = [prob.tree.level(int(b)) for b in prob.local_blocks]
    father = lv.index(2)
    kids = list(range(prob.nblocks, prob.nblocks + 8))
    n = prob.nblocks + 16
    Fg, Fo = g.download(n)[father], o.U[father]
    g.refine(father, kids)
    o.refine(father, kids)
    Ug, Uo = g.download(n), o.U
    for c, s in enumerate(kids):
        assert np.array_equal(Ug[s], inject(Fg)[c])   # device copy = reference copy rule
        assert np.array_equal(Uo[s], inject(Fo)[c])   # oracle obeys the same rule
    # perturb the children so the average is not a plain copy back
    Ug[kids] *= 1.0 + 1e-3 * np.arange(8)[:, None, None, None, None]
    g.upload(Ug)
    g.coarsen(kids, father)
    got = g.download(n)[father]
    assert np.array_equal(got, average8([Ug[s] for s in kids]))
    o.coarsen(kids, father)
    assert np.array_equal(o.U[father], average8([Uo[s] for s in kids]))


def test_sedov_256_conservation_and_symmetry():
    """Full-size property check (4096 blocks, 16.8M cells): with eta=0 mass
    and energy are conserved to round-off and the blast stays symmetric
    under the octant mirrors."""
    prob = problems.sedov(16, radius_cells=6.0)
    prob.cfg.visc_eta = 0.0
    g = from_problem(prob)
    U0 = prob.U
    g.run(20)
    U = g.download()
    for e in (0, 4):
        assert abs(U[:, e].sum() - U0[:, e].sum()) <= 1e-12 * abs(U0[:, e].sum())
    N = 256
    G = np.zeros((N, N, N))
    for n, b in enumerate(prob.local_blocks):
        _, x = prob.tree.coords(int(b))
        G[x[2] * 16:(x[2] + 1) * 16, x[1] * 16:(x[1] + 1) * 16, x[0] * 16:(x[0] + 1) * 16] = U[n, 0]
    scale = np.abs(G).max()
    assert np.abs(G - G[:, :, ::-1]).max() <= 1e-12 * scale
    assert np.abs(G - G.transpose(2, 1, 0)).max() <= 1e-12 * scale


SEDOV_XI0_GAMMA_5_3 = 1.15167   # E = alpha rho R^5 / t^2, alpha(5/3) = 0.4936 (Kamm & Timmes 2007)


def _sedov_radial_density(prob, U):
    """Mean density in radial shells of one cell width about the box centre:
    (shell centres, mean density)."""
    from walicxe3d_b200.mesh import cell_centres

    n = prob.cfg.nbroot[0] * 16
    xyz = cell_centres(prob.cfg, prob.tree, [int(b) for b in prob.local_blocks])
    r = np.sqrt(((xyz - 0.5) ** 2).sum(axis=1)).ravel()
    rho = U[:, 0].ravel()
    nbins = n // 2
    idx = np.minimum((r * n).astype(np.int64), nbins)
    ok = idx < nbins
    mean = np.bincount(idx[ok], weights=rho[ok], minlength=nbins) / np.maximum(
        np.bincount(idx[ok], minlength=nbins), 1)
    return (np.arange(nbins) + 0.5) / n, mean


def test_sedov_taylor_blast_radius_converges():
    """Physics check of the GPU path on a strong point blast: the shock radius
    approaches the Sedov-Taylor similarity solution R = xi0 (E t^2/rho)^(1/5)
    (gamma = 5/3, xi0 = 1.15167) as the mesh is refined (64^3, 128^3, 256^3
    cells), and the shell-averaged peak density rises towards the
    strong-shock limit (gamma+1)/(gamma-1) = 4 without passing it.  The run
    stops at the output time where R = 0.3 (the clip to dtout lands on it
    exactly); the shock is located where the shell-averaged density falls
    through the middle of ambient and peak, outside the peak."""
    r_target = 0.3
    t_target = (r_target / SEDOV_XI0_GAMMA_5_3) ** 2.5     # rho = E = 1
    errs, peaks = [], []
    for nroot in (4, 8, 16):
        prob = problems.sedov(nroot, radius_cells=3.0)
        prob.cfg.visc_eta = 0.0
        prob.cfg.dtout = t_target
        g = from_problem(prob)
        try:
            for _ in range(5000):
                s = g.step()
                if s.dumpout:
                    break
            assert s.dumpout and s.time == pytest.approx(t_target, rel=1e-14)
            U = g.download()
        finally:
            g.close()
        rc, prof = _sedov_radial_density(prob, U)
        ip = int(np.argmax(prof))
        half = 0.5 * (1.0 + prof[ip])
        j = ip + int(np.argmax(prof[ip:] < half))              # first shell outside the peak below half
        r_shock = rc[j - 1] + (half - prof[j - 1]) / (prof[j] - prof[j - 1]) * (rc[j] - rc[j - 1])
        errs.append(abs(r_shock / r_target - 1.0))
        peaks.append(prof[ip])
    assert errs[0] > errs[1] > errs[2], errs
    assert errs[2] < 0.02, errs
    assert peaks[0] < peaks[1] < peaks[2] < 4.0, peaks


def test_blast_amr_full_size_matches_oracle(ncpu):
    """The benchmark's headline mesh at full size (8^3 roots, 5 levels,
    11,600 blocks, 47.5M cells), stepped through the replayed CUDA graph of
    wx3d_run with the launch shape the mesh size selects (whole blocks, the
    viscous step fused into the corrector), against the oracle over all
    blocks."""
    prob = problems.blast_amr()
    assert prob.nblocks == 11600
    o, g = run_both(prob, 3, ncpu, use_run=True)
    check(o, g, prob)
    g.close()
    o.close()


def test_status_counts_and_zero_density_error():
    prob = problems.sedov(2)
    U = prob.U.copy()
    U[0, :, 3, 3, 3] = 0.0  # zero density cell -> reference aborts (hydro_core.f90:335)
    g = Walicxe3D(prob.cfg, prob.nblocks)
    g.set_mesh(prob.local_blocks)
    g.upload(U)
    from walicxe3d_b200 import WxError
    with pytest.raises(WxError) as ei:
        g.step()
    assert ei.value.code == 23


def test_fast_reciprocal_and_sqrt_within_two_ulp():
    """The Newton-refined reciprocal and square root of the flux kernels
    against the device's IEEE 1/x and sqrt(x), log-uniform over 600 decades
    plus powers of two and values next to them."""
    import ctypes

    from walicxe3d_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(12)
    x = 10.0 ** rng.uniform(-300, 300, 1_000_000)
    p2 = 2.0 ** np.arange(-1000, 1000, dtype=np.float64)
    x = np.concatenate([x, p2, np.nextafter(p2, 0), np.nextafter(p2, np.inf), [1.0, 1.4, 1e-30, 1e-40]])
    out = np.zeros(2, np.int64)
    rc = lib.wx3d_check_fast_math(x.size, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    assert rc == 0
    assert out[0] <= 2 and out[1] <= 2, out


def _shape(g, shape):
    g.set_zsplit(int(shape.split("-")[0]))
    g.set_fusion(shape.endswith("fused"))


@pytest.mark.parametrize("shape", ["1-fused", "1", "2", "8"])
def test_launch_shapes_match_oracle(shape, ncpu):
    """Every launch shape of the stage kernels (whole blocks with the viscous
    step fused into the corrector or separate, 2 and 8 z-slabs) against the
    CPU oracle on the three-level AMR mesh."""
    prob = small_amr()
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    _shape(g, shape)
    for _ in range(10):
        o.step()
        g.step()
    check(o, g, prob)


@pytest.mark.parametrize("name", ["amr", "brio-wu", "snr-h"])
def test_fused_viscous_step_equals_separate_kernel(name, ncpu):
    """The corrector with the viscous step fused reproduces the separate
    viscous kernel: hydro AMR (CFL from the viscous result), MHD with the
    8-wave source, and the radiative SNR (CFL from the source step)."""
    prob = {"amr": small_amr, "brio-wu": lambda: problems.brio_wu(4),
            "snr-h": lambda: problems.snr_h(nroot=2, maxlev=2)}[name]()
    a, b = from_problem(prob), from_problem(prob)
    _shape(a, "1-fused")
    _shape(b, "1")
    sa, sb = a.run(8), b.run(8)
    Ua, Ub = a.download(), b.download()
    assert np.all(np.isfinite(Ua))
    assert rel_l1(Ua, Ub).max() <= 1e-14
    assert sa.dt == pytest.approx(sb.dt, rel=1e-14) and sa.it == sb.it
    if name == "brio-wu":
        o = oracle.from_problem(prob, threads=ncpu)
        for _ in range(8):
            o.step()
        check(o, a, prob)


def test_autotune_picks_a_shape_and_keeps_the_state():
    prob = small_amr()
    g = from_problem(prob)
    U0 = g.download()
    z, fused, ms = g.autotune(2)
    assert z in (1, 2, 4, 8) and set(ms) == set(g.SHAPES) and all(v > 0 for v in ms.values())
    assert fused in (True, False)
    assert np.array_equal(g.download(), U0)


def test_autotune_between_steps_keeps_the_reference_time_step(ncpu):
    """The tuner's timed passes fold CFL minima and status counts of their
    scratch results into the control block; tuning between two steps must
    leave the next step's dt (the CFL minimum of U) and the counters as they
    were, so the run continues as the oracle's.  On a shock tube whose wave
    speeds still grow, the scratch results' CFL minimum lies below U's."""
    prob = problems.shock_tube(8)
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    try:
        for _ in range(2):
            o.step()
            g.step()
        before = g.status()
        g.autotune(2)
        after = g.status()
        for f in ("pressure_floor", "density_floor", "zero_density", "nan_cells", "max_cool_loss"):
            assert getattr(after, f) == getattr(before, f), f
        for _ in range(2):
            o.step()
            s = g.step()
            assert s.dt == pytest.approx(o.state.dt, rel=1e-12)
        check(o, g, prob)
    finally:
        g.close()
        o.close()


@pytest.mark.parametrize("shape", ["default", "1-fused"])
def test_colliding_winds_match_oracle(shape, ncpu):
    """Two spherical wind sources re-imposed before each stage (the
    userBoundary hook, winds.f90:123-240) with EOS_H_RATE and table
    cooling, on a two-level mesh, against the CPU oracle."""
    prob = problems.colliding_winds(nroot=2, maxlev=3, r_wind_cells=8)
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    if shape != "default":
        _shape(g, shape)
    for _ in range(6):
        o.step()
        g.step()
    check(o, g, prob)


WIND_EDGE_SEP = 1.0 - 18.0 / 128.0   # sources 9 finest cells (1/128 of the box) from the x boundaries


def test_wind_spheres_next_to_the_domain_boundary_match_oracle(ncpu):
    """Sources 9 finest cells from the x boundaries with spheres of 8: the
    spheres reach the physical cells next to the boundary but not its ghost
    layer.  The boundary ghosts then mirror those cells as they were before
    the wind -- the reference fills them before userBoundary imposes it --
    and the first stage reads them from U, not from the imposed copies."""
    prob = problems.colliding_winds(nroot=2, maxlev=3, r_wind_cells=8, sep_pc=WIND_EDGE_SEP)
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    try:
        for _ in range(6):
            o.step()
            g.step()
        check(o, g, prob)
    finally:
        g.close()
        o.close()


def test_wind_sphere_through_the_domain_boundary_ghosts_is_refused():
    """A sphere that reaches the ghost layer of the domain boundary would
    need the wind at the ghosts' own positions, which mirroring a physical
    cell does not give: refused, and the previous sources stay in force."""
    from walicxe3d_b200._lib import WxError
    prob = problems.colliding_winds(nroot=2, maxlev=3, r_wind_cells=8, sep_pc=WIND_EDGE_SEP)
    g = from_problem(prob)
    wider = [list(w) for w in prob.winds]
    for w in wider:
        w[6] *= 10.0 / 8.0                     # 10 finest cells: past the boundary 9 cells away
    with pytest.raises(WxError) as e:
        g.set_winds(wider)
    assert e.value.code == 104
    g.step()
    g.close()


def test_wind_sphere_on_a_level_transition_is_refused():
    """A sphere that reaches the ghost layer of a coarse/fine face would need
    the wind at ghost positions no same-level neighbour provides: refused."""
    from walicxe3d_b200._lib import WxError
    prob = problems.colliding_winds(nroot=2, maxlev=3, r_wind_cells=8)
    g = from_problem(prob)
    L = prob.cfg.box[0]
    bad = [[0.2 * L, 0.5 * L, 0.5 * L, 0, 0, 0, 0.3 * L, 1e20, 1e8, 1e5, 0.61, 0.0]]
    with pytest.raises(WxError) as e:
        g.set_winds(bad)
    assert e.value.code == 104
    g.step()   # the previous sources stay in force


def test_mesh_refused_for_a_wind_sphere_keeps_the_previous_mesh(tmp_path):
    """wx3d_set_mesh refusing a mesh with a coarse/fine face through a wind
    sphere (one level-2 block at the first source refined, its neighbours
    not) keeps the previous mesh whole, its slot registry included: a
    checkpoint written afterwards carries the previous mesh's bIDs."""
    from walicxe3d_b200._lib import WxError
    prob = problems.colliding_winds(nroot=2, maxlev=3, r_wind_cells=8)
    g = from_problem(prob)
    t = BlockTree(prob.cfg.nbroot, 3).roots()
    for b in sorted(t.leaves):
        t.refine(b)
    src = np.array([0.25, 0.5, 0.5]) + 1e-3          # just inside the block cornered at the first source
    inside = [b for b in t.leaves if np.all(t.bounds(b)[0] <= src) and np.all(src < t.bounds(b)[1])]
    assert len(inside) == 1
    t.refine(inside[0])
    with pytest.raises(WxError) as e:
        g.set_mesh(np.array(sorted(t.leaves), np.int32))
    assert e.value.code == 104
    g.write_bin(tmp_path / "b.bin")
    h = Walicxe3D(prob.cfg, g.max_blocks)
    lb = h.read_bin(tmp_path / "b.bin")
    assert sorted(int(b) for b in lb if b != -1) == sorted(int(b) for b in prob.local_blocks)
    g.step()


def test_small_wind_sphere_fails_at_the_same_step_as_the_reference(ncpu):
    """With wind spheres of 8 finest cells the reference algorithm goes
    non-finite next to the strong source at the end of the dt ramp; the GPU
    path reports WX_ERR_NAN at the same step as the CPU oracle turns
    non-finite."""
    from walicxe3d_b200._lib import WxError
    prob = problems.colliding_winds(nroot=2, maxlev=3, r_wind_cells=8)
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    step_o = step_g = None
    for s in range(16):
        if step_o is None:
            o.step()
            if not np.isfinite(o.U[: prob.nblocks]).all():
                step_o = s
        if step_g is None:
            try:
                g.step()
            except WxError as e:
                assert e.code == 102
                step_g = s
        if step_o is not None and step_g is not None:
            break
    assert step_o is not None and step_o == step_g


@pytest.mark.parametrize("ctype", [C.COOL_TABLE, C.COOL_TABLE_METAL, C.COOL_SCHURE])
def test_cooling_variants_match_oracle(ctype, ncpu):
    """Tabulated cooling (cooling.f90), metallicity-dependent 2-D tables
    (find_coef_metal, cooling.f90:435-519) and the Schure et al. tables
    (cooling_schure.f90) on a hot dense blob, 12 main-loop iterations, and
    the energy they remove."""
    prob = problems.cooling_blob(ctype, nroot=2)
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    E0 = prob.U[:, 4].sum()
    for _ in range(12):
        o.step()
        g.step()
    check(o, g, prob)
    assert g.download()[:, 4].sum() < (1.0 - 1e-4) * E0


@pytest.mark.parametrize("eos", [C.EOS_ADIABATIC, C.EOS_TWOTEMP])
def test_table_cooling_with_each_temperature_law(eos, ncpu):
    """calcTemp's other equations of state (hydro_core.f90:231-270) feeding
    the table cooling: ADIABATIC, and TWOTEMP, whose mean molecular weight
    switches from mu0 to mui above ion_thres (1e4 K; the blob spans 1e4 to
    3e7 K, so both branches are taken)."""
    prob = problems.cooling_blob(C.COOL_TABLE, nroot=2, eos=eos)
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    E0 = prob.U[:, 4].sum()
    for _ in range(12):
        o.step()
        g.step()
    check(o, g, prob)
    assert g.download()[:, 4].sum() < (1.0 - 1e-4) * E0


@pytest.mark.parametrize("shape", ["1-fused", "1", "2", "8"])
@pytest.mark.parametrize("solver", [C.SOLVER_HLLD, C.SOLVER_HLL1])
def test_field_cd_matches_oracle(shape, solver, ncpu):
    """The field-CD update of B (brio-wu/flux_cd.f90:52-86 with E = -v x B of
    the stage primitives) against the oracle on the 3-D Orszag-Tang vortex,
    in every launch shape (the carried E of the plane below crosses z-slab
    boundaries), for the two-stage and the first-order solver."""
    prob = problems.orszag_tang_3d(nroot=2, solver=solver)
    o = oracle.from_problem(prob, threads=ncpu)
    g = from_problem(prob)
    _shape(g, shape)
    for _ in range(12):
        o.step()
        g.step()
    check(o, g, prob)


@pytest.mark.parametrize("flux_cd", [True, False])
def test_field_cd_on_a_refined_mesh_matches_oracle(flux_cd, ncpu):
    """MHD on a two-level mesh, with field-CD or the Powell 8-wave source:
    the electric field (or div B) of the ghost cells comes through
    coarse/fine faces (injected or averaged primitives)."""
    prob = problems.orszag_tang_3d(nroot=4, maxlev=2, flux_cd=flux_cd)
    assert {prob.tree.level(int(b)) for b in prob.local_blocks} == {1, 2}
    o, g = run_both(prob, 10, ncpu)
    check(o, g, prob)


def test_field_cd_keeps_the_central_divergence_on_the_gpu():
    """4^3 blocks of the 3-D Orszag-Tang vortex, 20 steps through the CUDA
    graph: the central-difference divergence of B stays at its initial value
    to round-off with field-CD, and drifts with the 8-wave source."""
    from divergence import central_divergence
    drift = {}
    for flux_cd in (True, False):
        prob = problems.orszag_tang_3d(nroot=4, flux_cd=flux_cd)
        g = from_problem(prob)
        d0 = central_divergence(prob, g.download())
        g.run(20)
        U = g.download()
        assert np.all(np.isfinite(U))
        drift[flux_cd] = np.abs(central_divergence(prob, U) - d0).max()
        scale = np.abs(d0).max()
    assert drift[True] <= 1e-12 * scale
    assert drift[False] >= 1e-3 * scale


def test_admesh_matches_oracle(ncpu):
    """Live mesh: 12 main-loop steps past the dt ramp, each followed by admesh
    (amr.f90:44-133) on the device context and in the oracle.  The same
    blocks refine and coarsen into the same slots (first empty slot, as the
    reference's put), including slots freed earlier in the same call, and the
    state after the last step matches.  Before each admesh the marking flags
    are compared as well: from the second step on the device marking reads
    the ghost primitives the step's first-order stage left behind instead of
    gathering them."""
    prob = problems.amr_pulse()
    extra = 4 * prob.nblocks
    o = oracle.from_problem(prob, threads=ncpu, extra_slots=extra)
    g = from_problem(prob, extra_slots=extra)
    o.set_state(0.0, 0.0, 10, 1, 0)
    g.set_state(time=0.0, dt=0.0, it=10, nextout=1)
    total = np.zeros(2, int)
    for _ in range(12):
        o.step()
        g.step()
        fo, fg = o.mark(), g.mark()
        occ = g.local_blocks[:len(fg)] != -1
        assert np.array_equal(fo[:len(fg)][occ], fg[occ])
        no, ng = o.admesh(), g.admesh()
        assert no == ng
        assert np.array_equal(o.blocks, g.local_blocks)
        total += ng
    assert total[0] >= 5 and total[1] >= 5
    occ = g.local_blocks != -1
    Ug, Uo = g.download(g.max_blocks)[occ], o.U[occ]
    assert np.all(np.isfinite(Ug))
    err = rel_l1(Ug, Uo)
    assert err.max() <= TOL, f"rel L1 per eq {err}"
    so, sg = o.state, g.state
    assert sg.it == so.it and sg.time == pytest.approx(so.time, rel=1e-12)


def test_admesh_refuses_when_slots_run_out():
    """Too few free slots for the refinements: WX_ERR_INSUFICIENT_NBMAXPROC
    before any data moves; the block list and the state stay as they were.
    A list that differs from the mesh last set is refused too."""
    from walicxe3d_b200._lib import WxError
    prob = problems.amr_pulse()
    g = from_problem(prob, extra_slots=4)
    g.set_state(time=0.0, dt=0.0, it=10, nextout=1)
    g.step()
    U0, lb0 = g.download(g.max_blocks), g.local_blocks.copy()
    with pytest.raises(WxError) as e:
        g.admesh()
    assert e.value.code == 7
    assert np.array_equal(g.local_blocks, lb0)
    assert np.array_equal(g.download(g.max_blocks), U0)
    g.local_blocks = lb0[::-1].copy()
    with pytest.raises(WxError) as e:
        g.admesh()
    assert e.value.code == 106


def test_admesh_with_sources_matches_oracle(ncpu):
    """Live mesh with hydrogen ionisation and cooling_h: marking after the
    source step (the reference marks on primitives computed before it), then
    ten more steps with sources on the adapted mesh."""
    prob = problems.cooling_pulse(width_pc=2.5)
    extra = 4 * prob.nblocks
    o = oracle.from_problem(prob, threads=ncpu, extra_slots=extra)
    g = from_problem(prob, extra_slots=extra)
    o.set_state(0.0, 0.0, 10, 1, 0)
    g.set_state(time=0.0, dt=0.0, it=10, nextout=1)
    total = np.zeros(2, int)
    for _ in range(10):
        o.step()
        g.step()
        no, ng = o.admesh(), g.admesh()
        assert no == ng
        assert np.array_equal(o.blocks, g.local_blocks)
        total += ng
    assert total[0] >= 1 and total[1] >= 1
    occ = g.local_blocks != -1
    Ug, Uo = g.download(g.max_blocks)[occ], o.U[occ]
    err = rel_l1(Ug, Uo)
    assert err.max() <= TOL, f"rel L1 per eq {err}"


def test_invalid_meshes_are_refused():
    """wx3d_set_mesh refuses what the reference's tree queries would not
    resolve (WX_ERR_MESH): a bID registered twice, a bID outside the tree, a
    face with a level jump of two, a region no block covers; more slots than
    the context holds is WX_ERR_INSUFICIENT_NBMAXPROC; stepping with no mesh
    is WX_ERR_MESH.  A refused mesh leaves the previous one in place."""
    from walicxe3d_b200._lib import WxError
    cfg = C.Config(nbroot=(2, 2, 2), maxlev=3)
    tree = BlockTree(cfg.nbroot, 3).roots()
    roots = sorted(tree.leaves)
    w = Walicxe3D(cfg, 64)
    with pytest.raises(WxError) as e:
        w.step()
    assert e.value.code == 106
    good = np.array(roots, np.int32)
    w.set_mesh(good)
    U = problems.smooth_pulse(nroot=2).U
    w.upload(U)

    def refused(lb, code):
        with pytest.raises(WxError) as e:
            w.set_mesh(np.asarray(lb, np.int32))
        assert e.value.code == code

    refused(list(roots[:-1]) + [roots[0]], 106)             # registered twice
    refused(list(roots[:-1]) + [tree.maxid + 5], 106)        # outside the tree
    refused(roots[1:], 106)                                  # a hole: root 1's region is uncovered
    # level jump of two: root 1 refined twice in one octant, its neighbours left at level 1
    t = BlockTree(cfg.nbroot, 3).roots()
    t.refine(roots[0])
    first = t.children(roots[0])[7]                          # the child touching the other roots
    t.refine(first)
    refused(sorted(t.leaves), 106)
    refused(list(range(1, 66)), 7)                           # 65 slots > max_blocks 64
    # the previous mesh is still in place: a step runs
    w.set_state(time=0.0, dt=0.0, it=10, nextout=1)
    w.step()
    assert np.all(np.isfinite(w.download()))


@pytest.mark.parametrize("use_run", [False, True])
def test_an_empty_mesh_steps_like_the_reference(use_run):
    """A process whose localBlocks are all -1 (more processes than blocks):
    its loops find no block, its local dt is 1e30*CFL (getTimestep,
    hydro_solver.f90:145-192), clamped to the next output time, and each step
    advances time, it and nextout as the oracle's does, through wx3d_step and
    through the graph replay of wx3d_run."""
    prob = problems.brio_wu(4)
    empty = np.full(4, -1, np.int32)
    o = oracle.Oracle(prob.cfg, 4)
    o.set_blocks(empty)
    w = Walicxe3D(prob.cfg, 4)
    w.set_mesh(empty)
    for x in (o, w):
        x.set_state(time=0.0, dt=0.0, it=3, nextout=1)
    for _ in range(3):
        o.step()
    if use_run:
        w.run(3)
    else:
        for _ in range(3):
            w.step()
    so, sg = o.state, w.state
    assert (sg.time, sg.dt, sg.it, sg.nextout) == (so.time, so.dt, so.it, so.nextout)
    assert so.it == 6 and so.time > 0.0
    o.close()
    w.close()


@pytest.mark.parametrize("solver", [C.SOLVER_LAX, C.SOLVER_HLL1, C.SOLVER_HLL])
def test_other_solvers_on_a_three_level_mesh(solver, ncpu):
    """Lax-Friedrichs (one-deep ghosts of U, lax.f90:39-99), the first-order
    HLL1 stage, and HLL on the three-level AMR blast: coarse/fine ghost
    fills under each solver's own stencil, and the zero UP ghosts the
    single-stage solvers give the viscous step."""
    prob = small_amr(solver=solver)
    o, g = run_both(prob, 10, ncpu)
    check(o, g, prob)
