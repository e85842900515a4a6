"""Problem setups (initial conditions and meshes) for the benchmark workloads.

Each builder returns a ``Problem`` with the configuration, the localBlocks
registry (bID per slot, Morton-ordered) and the conserved variables in the
native layout ``U[slot][eq][k][j][i]`` (16^3 physical cells per block).

The reference builds its ICs in Fortran user modules; the ones restated
here are the Sedov-type blast (uniform medium plus a thermal-energy sphere),
the Brio-Wu shock tube (brio-wu/brio-wu.f90:53-132), the uniform ISM
(source/uniformISM.f90:87-185), the supernova remnant (source/snr.f90:90-218)
and spherical winds (source/winds.f90:123-240).  The benchmark meshes are
synthetic snapshots with the shapes named by the workloads (root grids,
refinement levels, leaf counts).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import config as C
from .config import NCELLS, Config
from .mesh import BlockTree, cell_centres


@dataclass
class Problem:
    name: str
    cfg: Config
    tree: BlockTree
    local_blocks: np.ndarray      # int32 bID per slot
    U: np.ndarray                 # float64 [nslots, neq, 16, 16, 16]
    cooltable: tuple | None = None
    cooltable_metal: tuple | None = None    # (nptsT, nptsZ, table[(nptsT+1)*(nptsZ+1)])
    cooltable_schure: tuple | None = None   # (data[180, 5], dmc_f)
    winds: list = field(default_factory=list)
    steps: int = 50

    @property
    def nblocks(self) -> int:
        return len(self.local_blocks)

    @property
    def cells(self) -> int:
        return self.nblocks * NCELLS ** 3


def prim2flow(cfg: Config, prim: np.ndarray) -> np.ndarray:
    """Vectorised prim2flow (source/hydro_core.f90:278-313) over axis 1."""
    u = np.empty_like(prim)
    rho = prim[:, 0]
    u[:, 0] = rho
    u[:, 1] = rho * prim[:, 1]
    u[:, 2] = rho * prim[:, 2]
    u[:, 3] = rho * prim[:, 3]
    v2 = prim[:, 1] ** 2 + prim[:, 2] ** 2 + prim[:, 3] ** 2
    u[:, 4] = 0.5 * rho * v2 + cfg.cv * prim[:, 4]
    if cfg.bfield:
        if cfg.mhd:
            u[:, 4] = u[:, 4] + 0.5 * (prim[:, 5] ** 2 + prim[:, 6] ** 2 + prim[:, 7] ** 2)
        u[:, 5:8] = prim[:, 5:8]
    if cfg.npassive:
        u[:, cfg.firstpas:] = prim[:, cfg.firstpas:]
    return u


def _finish(name, cfg, tree, prim_fn, steps, chunk: int = 512, **kw) -> Problem:
    bids = tree.morton_order()
    U = np.empty((len(bids), cfg.neqtot, NCELLS, NCELLS, NCELLS))
    for s in range(0, len(bids), chunk):
        part = bids[s:s + chunk]
        xyz = cell_centres(cfg, tree, part)
        U[s:s + len(part)] = prim2flow(cfg, prim_fn(xyz))
    return Problem(name, cfg, tree, np.asarray(bids, dtype=np.int32), U, steps=steps, **kw)


# ---------------------------------------------------------------------------
def sedov(nroot: int = 4, steps: int = 50, solver=C.SOLVER_HLLC, limiter=C.LIMITER_MINMOD,
          radius_cells: float = 3.0, energy: float = 1.0) -> Problem:
    """Sedov-type blast, adiabatic hydro, single level: nroot^3 root blocks
    of 16^3 in the unit box, gamma=5/3, ambient rho=1 p=1e-5 v=0, energy E
    deposited as thermal energy in the cells whose centres lie within
    radius_cells cells of the box centre; free-flow boundaries."""
    cfg = Config(solver_type=solver, limiter_type=limiter, nbroot=(nroot,) * 3, maxlev=1,
                 gamma=5.0 / 3.0, cfl=0.4, visc_eta=5.0e-3)
    tree = BlockTree(cfg.nbroot, 1).roots()
    dx = cfg.dx(1)[0]

    # cells whose centres lie inside the sphere: offsets (a+1/2, b+1/2, c+1/2) dx
    a = np.arange(-int(radius_cells) - 1, int(radius_cells) + 1) + 0.5
    n_in = int(((a[:, None, None] ** 2 + a[None, :, None] ** 2 + a[None, None, :] ** 2) < radius_cells ** 2).sum())

    def prim_fn(xyz):
        r = np.sqrt(((xyz - 0.5) ** 2).sum(axis=1))
        inside = r < radius_cells * dx
        p = np.full(r.shape, 1.0e-5)
        p[inside] = (cfg.gamma - 1.0) * energy / (n_in * dx ** 3)
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        prim[:, 0] = 1.0
        prim[:, 4] = p
        return prim

    return _finish(f"sedov{nroot * NCELLS}", cfg, tree, prim_fn, steps)


def brio_wu(nblocks_x: int = 16, steps: int = 0) -> Problem:
    """Brio-Wu shock tube extruded to 3-D: nblocks_x x 1 x 1 blocks of 16^3,
    box 1 x 1/16 x 1/16, gamma=2, Bx=0.75, left rho=1 p=1 By=1, right
    rho=0.125 p=0.1 By=-1 (brio-wu/brio-wu.f90:87-105), HLLD + minmod,
    CFL 0.4, no viscosity, Powell 8-wave source; the y/z-invariant problem
    makes free-flow y/z boundaries equivalent to periodic ones."""
    cfg = Config(bfield=True, mhd=True, solver_type=C.SOLVER_HLLD, limiter_type=C.LIMITER_MINMOD,
                 eight_wave=True, nbroot=(nblocks_x, 1, 1), maxlev=1, gamma=2.0, cfl=0.4, visc_eta=0.0,
                 box=(1.0, 1.0 / nblocks_x, 1.0 / nblocks_x), tfin=0.1, dtout=0.01)
    tree = BlockTree(cfg.nbroot, 1).roots()

    def prim_fn(xyz):
        x = xyz[:, 0]
        left = x <= 0.5
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        prim[:, 0] = np.where(left, 1.0, 0.125)
        prim[:, 4] = np.where(left, 1.0, 0.1)
        prim[:, 5] = 0.75
        prim[:, 6] = np.where(left, 1.0, -1.0)
        return prim

    return _finish("brio-wu", cfg, tree, prim_fn, steps or 200)


def orszag_tang_3d(nroot: int = 2, flux_cd: bool = True, solver=C.SOLVER_HLLD, steps: int = 20,
                   maxlev: int = 1) -> Problem:
    """Orszag-Tang vortex (the reference's orzag-tang example; its problem
    file is not in the tree) extended to 3-D: unit box of nroot^3 root
    blocks, gamma=5/3, rho=25/(36 pi), p=5/(12 pi),
    v=(-sin 2 pi y, sin 2 pi x, 0.2 sin 2 pi (x+z)),
    B=B0 (-sin 2 pi y, sin 4 pi x, 0.3 sin 2 pi (x+y+z)) with B0=1/sqrt(4 pi)
    (B_z depends on z, so the field starts with a non-zero divergence),
    minmod, CFL 0.4, no viscosity, free-flow boundaries.  With flux_cd the
    magnetic field takes the field-CD update (brio-wu/flux_cd.f90:52-86)
    instead of the 8-wave source.  With maxlev > 1 the blocks within 0.2 of
    the box centre are refined to maxlev (face-balanced), so the electric
    field also crosses coarse/fine faces."""
    cfg = Config(bfield=True, mhd=True, solver_type=solver, limiter_type=C.LIMITER_MINMOD,
                 eight_wave=not flux_cd, enable_flux_cd=flux_cd, nbroot=(nroot,) * 3, maxlev=maxlev,
                 gamma=5.0 / 3.0, cfl=0.4, visc_eta=0.0)
    tree = BlockTree(cfg.nbroot, maxlev).roots()
    if maxlev > 1:
        tree.refine_where(lambda lev, lo, hi: np.sqrt(((np.clip(0.5, lo, hi) - 0.5) ** 2).sum()) < 0.2, maxlev)
    b0 = 1.0 / np.sqrt(4.0 * np.pi)

    def prim_fn(xyz):
        x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
        tp = 2.0 * np.pi
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        prim[:, 0] = 25.0 / (36.0 * np.pi)
        prim[:, 1] = -np.sin(tp * y)
        prim[:, 2] = np.sin(tp * x)
        prim[:, 3] = 0.2 * np.sin(tp * (x + z))
        prim[:, 4] = 5.0 / (12.0 * np.pi)
        prim[:, 5] = -b0 * np.sin(tp * y)
        prim[:, 6] = b0 * np.sin(2.0 * tp * x)
        prim[:, 7] = 0.3 * b0 * np.sin(tp * (x + y + z))
        return prim

    return _finish("orszag-tang-3d", cfg, tree, prim_fn, steps)


def amr_pulse(nroot: int = 2, maxlev: int = 3, centre=(0.15, 0.15, 0.15), width: float = 0.03,
              amplitude: float = 10.0, steps: int = 20, refine_roots=None) -> Problem:
    """Live-mesh test: a Gaussian pressure and density pulse in one corner of
    a uniform medium at rest (rho = p = 1), on nroot^3 root blocks all
    refined once (level 2), or only the roots listed in refine_roots (bIDs).
    The first admesh coarsens the quiet families and refines the blocks
    around the pulse; as the pulse spreads, refinement follows it.  HLLC +
    minmod, CFL 0.4, eta 5e-3, free-flow boundaries."""
    cfg = Config(solver_type=C.SOLVER_HLLC, limiter_type=C.LIMITER_MINMOD, nbroot=(nroot,) * 3, maxlev=maxlev,
                 gamma=5.0 / 3.0, cfl=0.4, visc_eta=5.0e-3)
    tree = BlockTree(cfg.nbroot, maxlev).roots()
    for b in sorted(tree.leaves) if refine_roots is None else list(refine_roots):
        tree.refine(b)
    c = np.array(centre)

    def prim_fn(xyz):
        r2 = ((xyz - c[None, :, None, None, None]) ** 2).sum(axis=1)
        g = amplitude * np.exp(-r2 / width ** 2)
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        prim[:, 0] = 1.0 + 0.5 * g
        prim[:, 4] = 1.0 + g
        return prim

    return _finish("amr-pulse", cfg, tree, prim_fn, steps)


def cooling_pulse(nroot: int = 2, maxlev: int = 3, width_pc: float = 1.5, amplitude: float = 30.0,
                  steps: int = 20) -> Problem:
    """Live-mesh test with source terms: the ISM of snr_h (n = 1 cm^-3,
    T = 1e4 K, neutral fraction 0.99; EOS_H_RATE + COOL_H, HLLC + minmod,
    box 50 pc) with a Gaussian overpressure (peak amplitude x the ISM
    pressure, half-width width_pc) in one corner, on nroot^3 root blocks all
    refined once.  The first admesh coarsens the quiet families and refines
    around the pulse; hydrogen ionisation and cooling act on the hot gas."""
    mu0 = 1.3
    cfg = Config(npassive=1, solver_type=C.SOLVER_HLLC, limiter_type=C.LIMITER_MINMOD,
                 eos_type=C.EOS_H_RATE, cooling_type=C.COOL_H, nbroot=(nroot,) * 3, maxlev=maxlev,
                 gamma=5.0 / 3.0, cfl=0.4, visc_eta=5.0e-3, l_sc=C.PC, d_sc=mu0 * C.AMU, v_sc=1.0e5,
                 box=(50.0 * C.PC,) * 3, tfin=5.0e4 * C.YR, dtout=1.0e4 * C.YR)
    tree = BlockTree(cfg.nbroot, maxlev).roots()
    for b in sorted(tree.leaves):
        tree.refine(b)
    centre = np.array([7.5, 7.5, 7.5])  # pc, code units

    def prim_fn(xyz):
        dens_ism = 1.0 * C.AMU * mu0
        pres_ism = dens_ism / (mu0 * C.AMU) * C.KB * 1.0e4
        r2 = ((xyz - centre[None, :, None, None, None]) ** 2).sum(axis=1)
        g = amplitude * np.exp(-r2 / width_pc ** 2)
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        prim[:, 0] = mu0 * dens_ism / cfg.d_sc
        prim[:, 4] = pres_ism * (1.0 + g) / cfg.p_sc
        prim[:, 5] = 0.99 * dens_ism / cfg.d_sc
        return prim

    return _finish("cooling-pulse", cfg, tree, prim_fn, steps)


def smooth_pulse(nroot: int = 2, amplitude: float = 0.2, width: float = 0.15, solver=C.SOLVER_HLLC,
                 limiter=C.LIMITER_MINMOD) -> Problem:
    """Smooth Gaussian density/pressure pulse at rest in a uniform medium
    (rho = p = 1), nroot^3 root blocks: a low-Mach test where no floor or
    limiter switch is hit, for solver and limiter parity."""
    cfg = Config(solver_type=solver, limiter_type=limiter, nbroot=(nroot,) * 3, maxlev=1)
    tree = BlockTree(cfg.nbroot, 1).roots()

    def prim_fn(xyz):
        r2 = ((xyz - np.array([0.45, 0.5, 0.55])[None, :, None, None, None]) ** 2).sum(axis=1)
        g = amplitude * np.exp(-r2 / width ** 2)
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        prim[:, 0] = 1.0 + g
        prim[:, 1] = 0.1 * g
        prim[:, 4] = 1.0 + 1.5 * g
        return prim

    return _finish("pulse", cfg, tree, prim_fn, 20)


def shock_tube(nblocks: int = 16, axis: int = 0, gamma: float = 1.4, left=(1.0, 0.0, 1.0),
               right=(0.125, 0.0, 0.1), solver=C.SOLVER_HLLC, limiter=C.LIMITER_MINMOD, eta: float = 0.0,
               t_end: float = 0.2) -> Problem:
    """Sod-type shock tube along `axis` (0, 1, 2): nblocks blocks of 16^3 in
    a box of length 1 along the axis and 1/nblocks across; (rho, u, p) left
    and right of the mid-plane; free-flow boundaries.  dtout = t_end so the
    reference's output clipping (hydro_solver.f90:204-207) lands a step
    exactly on t_end."""
    nb = [1, 1, 1]
    nb[axis] = nblocks
    box = [1.0 / nblocks] * 3
    box[axis] = 1.0
    cfg = Config(solver_type=solver, limiter_type=limiter, nbroot=tuple(nb), maxlev=1, gamma=gamma,
                 visc_eta=eta, box=tuple(box), tfin=t_end, dtout=t_end)
    tree = BlockTree(cfg.nbroot, 1).roots()

    def prim_fn(xyz):
        x = xyz[:, axis]
        lft = x <= 0.5
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        prim[:, 0] = np.where(lft, left[0], right[0])
        prim[:, 1 + axis] = np.where(lft, left[1], right[1])
        prim[:, 4] = np.where(lft, left[2], right[2])
        return prim

    return _finish(f"shocktube{axis}", cfg, tree, prim_fn, 0)


def blast_amr(nroot: int = 8, maxlev: int = 5, shell_radius: float = 0.1, shell_width: float = 0.004,
              steps: int = 200, solver=C.SOLVER_HLLC, limiter=C.LIMITER_MINMOD) -> Problem:
    """Batched AMR blast snapshot: the Sedov setup on nroot^3 root blocks with
    maxlev levels; the blocks crossing the blast shell (radius shell_radius,
    half-width shell_width) are refined to maxlev and the face-proximity rule
    fills the intermediate levels, giving uneven leaf counts per level.  The
    state is a smooth blast profile: hot rarefied interior, compressed shell
    moving outwards, cold ambient medium."""
    cfg = Config(solver_type=solver, limiter_type=limiter, nbroot=(nroot,) * 3, maxlev=maxlev,
                 gamma=5.0 / 3.0, cfl=0.4, visc_eta=5.0e-3)
    tree = BlockTree(cfg.nbroot, maxlev).roots()
    c = np.array([0.5, 0.5, 0.5])

    def crosses(lev, lo, hi):
        near = np.clip(c, lo, hi)
        dmin = np.sqrt(((near - c) ** 2).sum())
        corners = np.array([[lo[0] if a else hi[0], lo[1] if b else hi[1], lo[2] if d else hi[2]]
                            for a in (0, 1) for b in (0, 1) for d in (0, 1)])
        dmax = np.sqrt(((corners - c) ** 2).sum(axis=1)).max()
        return dmin <= shell_radius + shell_width and dmax >= shell_radius - shell_width

    tree.refine_where(crosses, maxlev)

    def prim_fn(xyz):
        r = np.sqrt(((xyz - c[None, :, None, None, None]) ** 2).sum(axis=1))
        s = (r - shell_radius) / shell_width
        shell = np.exp(-s * s)
        inside = 0.5 * (1.0 - np.tanh(s))
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        prim[:, 0] = 1.0 + 3.0 * shell - 0.9 * inside * (1 - shell)
        prim[:, 4] = 1.0e-5 + 0.5 * inside + 0.8 * shell
        vr = 0.6 * shell + 0.3 * inside * (r / shell_radius)
        rr = np.maximum(r, 1e-12)
        for d in range(3):
            prim[:, 1 + d] = vr * (xyz[:, d] - c[d]) / rr
        return prim

    return _finish(f"blast-amr-l{maxlev}", cfg, tree, prim_fn, steps)


def cooling_table_synthetic(n: int = 200) -> tuple:
    """A monotone, smooth Lambda(T) table in loadcooldata format
    (source/cooling.f90:135-184): n rows of (log10 T, -log10 Lambda) for
    log T in 4..9, Lambda peaking near 1e5.3 K."""
    logT = np.linspace(4.0, 9.0, n)
    logL = -21.6 - 0.9 * (logT - 5.3) ** 2 / (1.0 + 0.35 * np.abs(logT - 5.3)) + 0.25 * np.tanh(logT - 7.5)
    return logT, -logL


def snr_h(nroot: int = 4, maxlev: int = 2, steps: int = 20) -> Problem:
    """Radiative supernova remnant with hydrogen ionisation (snr/user.f90):
    uniform ISM n=1 cm^-3, T=1e4 K, neutral fraction 0.99, ejecta 2 Msun and
    1e51 erg (chi=0.5) inside 1 pc, box 50 pc, EOS_H_RATE + COOL_H, HLLC +
    minmod, one passive scalar (neutral H density)."""
    mu0 = 1.3
    cfg = Config(npassive=1, solver_type=C.SOLVER_HLLC, limiter_type=C.LIMITER_MINMOD,
                 eos_type=C.EOS_H_RATE, cooling_type=C.COOL_H, nbroot=(nroot,) * 3, maxlev=maxlev,
                 gamma=5.0 / 3.0, cfl=0.4, visc_eta=5.0e-3, l_sc=C.PC, d_sc=mu0 * C.AMU, v_sc=1.0e5,
                 box=(50.0 * C.PC,) * 3, tfin=5.0e4 * C.YR, dtout=1.0e4 * C.YR)
    tree = BlockTree(cfg.nbroot, maxlev).roots()
    xc = 25.0  # pc, code units
    rsn = 1.0

    def near(lev, lo, hi):
        p = np.clip(np.full(3, xc / 50.0), lo, hi)
        return np.sqrt(((p - xc / 50.0) ** 2).sum()) * 50.0 <= 6.0 * rsn

    tree.refine_where(near, maxlev)

    def prim_fn(xyz):
        # impose_uniform_ism (uniformISM.f90:124-158)
        dens_ism = 1.0 * C.AMU * mu0
        temp_ism, y0 = 1.0e4, 0.99
        pres_ism = dens_ism / (mu0 * C.AMU) * C.KB * temp_ism
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        prim[:, 0] = mu0 * dens_ism / cfg.d_sc
        prim[:, 4] = pres_ism / cfg.p_sc
        prim[:, 5] = y0 * dens_ism / cfg.d_sc
        # detonateSNR (snr.f90:127-206), linear velocity profile
        msn, esn, chi = 2.0 * C.MSUN, 1.0e51, 0.5
        R = rsn * C.PC
        ek, et = chi * esn, (1.0 - chi) * esn
        dens = msn / (4.0 / 3.0 * C.PI * R ** 3)
        vmax = np.sqrt(10.0 / 3.0 * ek / msn)
        pres = (1.0 / cfg.cv) * et / (4.0 / 3.0 * C.PI * R ** 3)
        pos = xyz * cfg.l_sc
        d = pos - xc * C.PC
        dist = np.sqrt((d ** 2).sum(axis=1))
        m = dist < R
        vel = np.where(m, dist / R * vmax, 0.0)
        safe = np.maximum(dist, 1.0)
        prim[:, 0] = np.where(m, dens / cfg.d_sc, prim[:, 0])
        for a in range(3):
            prim[:, 1 + a] = np.where(m, vel * d[:, a] / safe / cfg.v_sc, 0.0)
        prim[:, 4] = np.where(m, pres / cfg.p_sc, prim[:, 4])
        prim[:, 5] = np.where(m, 0.0, prim[:, 5])
        return prim

    return _finish("snr-h", cfg, tree, prim_fn, steps)


def colliding_winds(nroot: int = 8, maxlev: int = 6, box_pc: float = 1.0, sep_pc: float = 0.5,
                    r_wind_cells: float = 16.0, r_wind_pc: float | None = None, steps: int = 500,
                    shell_width: float = 0.25) -> Problem:
    """Colliding stellar winds with table cooling: two spherical wind
    sources (imposeSphericalWind, winds.f90:123-240; Mdot 1e-6 and 1e-7
    Msun/yr, vinf 2000 and 1000 km/s, T 1e5 K, radius r_wind_cells finest
    cells unless r_wind_pc is given) sep_pc apart on the x axis of a cubic
    box_pc box, in a uniform n=1 cm^-3, 1e4 K ISM of neutral fraction 0.99;
    EOS_H_RATE with the neutral-H passive scalar, COOL_TABLE with a 200-row
    table, HLLC + minmod.  The snapshot has each wind streaming freely out
    to the contact surface at the momentum-balance stand-off distance of the
    weaker wind; the zone around each source is refined to maxlev (as
    refineZone does at it=0, with a margin of one finest block so no
    coarse/fine face meets a wind sphere's ghost layer) and the bow-shaped
    contact region around the weaker source to maxlev-1.  The winds are
    ionised (their passive scalar, which the reference leaves undefined, is
    0).  With spheres of 8 finest cells or fewer the reference algorithm
    goes non-finite next to the strong source once the dt ramp ends (the
    stage-1 fluxes of the imposed cells use their primitives from before
    the imposition); 16 cells run stably."""
    mu0, mu_wind = 1.3, 0.61
    cfg = Config(npassive=1, solver_type=C.SOLVER_HLLC, limiter_type=C.LIMITER_MINMOD,
                 eos_type=C.EOS_H_RATE, cooling_type=C.COOL_TABLE, nbroot=(nroot,) * 3, maxlev=maxlev,
                 gamma=5.0 / 3.0, cfl=0.4, visc_eta=5.0e-3, l_sc=C.PC, d_sc=mu0 * C.AMU, v_sc=1.0e5,
                 box=(box_pc * C.PC,) * 3, tfin=1.0e4 * C.YR, dtout=1.0e3 * C.YR)
    L = box_pc * C.PC
    srcs = [np.array([0.5 * L - 0.5 * sep_pc * C.PC, 0.5 * L, 0.5 * L]),
            np.array([0.5 * L + 0.5 * sep_pc * C.PC, 0.5 * L, 0.5 * L])]
    mdot = [1.0e-6 * C.MSUN / C.YR, 1.0e-7 * C.MSUN / C.YR]
    vinf = [2000.0 * C.KPS, 1000.0 * C.KPS]
    dx_fine = L / (NCELLS * nroot * 2 ** (maxlev - 1))
    R = r_wind_pc * C.PC if r_wind_pc is not None else r_wind_cells * dx_fine
    winds = [[s[0], s[1], s[2], 0.0, 0.0, 0.0, R, m, v, 1.0e5, mu_wind, 0.0] for s, m, v in zip(srcs, mdot, vinf)]
    eta = (mdot[1] * vinf[1]) / (mdot[0] * vinf[0])
    r2 = sep_pc * C.PC * np.sqrt(eta) / (1.0 + np.sqrt(eta))   # stand-off of the weaker wind

    tree = BlockTree(cfg.nbroot, maxlev).roots()
    fine_block = 1.0 / (nroot * 2 ** (maxlev - 1))              # normalised finest block size
    sn = [s / L for s in srcs]

    def box_dist(p, lo, hi):
        near = np.clip(p, lo, hi)
        return np.sqrt(((near - p) ** 2).sum())

    def shell(lev, lo, hi):
        p = sn[1]
        corners = np.array([[lo[0] if a else hi[0], lo[1] if b else hi[1], lo[2] if d else hi[2]]
                            for a in (0, 1) for b in (0, 1) for d in (0, 1)])
        dmax = np.sqrt(((corners - p) ** 2).sum(axis=1)).max()
        w = shell_width * r2 / L
        return box_dist(p, lo, hi) <= r2 / L + w and dmax >= r2 / L - w

    def zone(lev, lo, hi):
        return any(box_dist(p, lo, hi) <= R / L + fine_block for p in sn)

    tree.refine_where(shell, maxlev - 1)
    tree.refine_where(zone, maxlev)

    def wind_prim(xyz_cm, k, nvar):
        d = xyz_cm - srcs[k][None, :, None, None, None]
        dist = np.maximum(np.sqrt((d ** 2).sum(axis=1)), 1.0e-3 * R)
        dens = mdot[k] / vinf[k] / dist / dist / (4.0 * C.PI)
        out = np.zeros((xyz_cm.shape[0], nvar) + xyz_cm.shape[2:])
        out[:, 0] = dens / cfg.d_sc
        for a in range(3):
            out[:, 1 + a] = vinf[k] * d[:, a] / dist / cfg.v_sc
        out[:, 4] = dens / (mu_wind * C.AMU) * C.KB * 1.0e5 / cfg.p_sc
        return out, dist

    def prim_fn(xyz):
        xyz_cm = xyz * cfg.l_sc
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        n_ism, T_ism, y_ism = 1.0, 1.0e4, 0.99
        dens = n_ism * mu0 * C.AMU
        prim[:, 0] = dens / cfg.d_sc
        prim[:, 4] = dens / (mu0 * C.AMU) * C.KB * T_ism * (2.0 - y_ism) / cfg.p_sc
        prim[:, 5] = y_ism * dens / cfg.d_sc
        w1, d1 = wind_prim(xyz_cm, 0, cfg.neqtot)
        w2, d2 = wind_prim(xyz_cm, 1, cfg.neqtot)
        in2 = (d2 < r2)[:, None]
        in1 = ((d1 < sep_pc * C.PC - r2) & ~(d2 < r2))[:, None]
        return np.where(in2, w2, np.where(in1, w1, prim))

    return _finish(f"winds-l{maxlev}", cfg, tree, prim_fn, steps, cooltable=cooling_table_synthetic(200),
                   winds=winds)


def metal_table_synthetic(nT: int = 60, Z=(0.1, 0.3, 1.0, 3.0)) -> tuple:
    """A COOL_TABLE_METAL table in loadcooldata_metal layout
    (source/cooling.f90:193-265): log T from 4 to 8.5, log Lambda rising
    with log Z and peaking near 1e5.3 K."""
    logT = np.linspace(4.0, 8.5, nT)
    tab = np.zeros((nT + 1, len(Z) + 1))
    tab[0, 0] = -1.0
    tab[0, 1:] = Z
    tab[1:, 0] = logT
    base = -21.8 - 0.8 * (logT - 5.3) ** 2 / (1.0 + 0.4 * np.abs(logT - 5.3))
    for j, z in enumerate(Z):
        tab[1:, j + 1] = base + 0.6 * np.log10(z) * np.exp(-0.5 * (logT - 5.5) ** 2)
    return nT, len(Z), tab.ravel()


def schure_table_synthetic() -> np.ndarray:
    """A Schure et al. style table (source/cooling_schure.f90:52-95): 180
    rows of log T (1.0 to 8.16 by 0.04) and -log Lambda for four ionisation
    fractions of the low-temperature branch."""
    logT = 1.0 + 0.04 * np.arange(180)
    data = np.zeros((180, 5))
    data[:, 0] = logT
    hot = 21.7 + 0.8 * (logT - 5.3) ** 2 / (1.0 + 0.4 * np.abs(logT - 5.3))
    for c, fi in enumerate((1e-4, 1e-3, 1e-2, 1e-1)):
        cold = 26.0 - 0.5 * np.log10(fi) - 0.6 * (logT - 4.0)
        w = 0.5 * (1.0 + np.tanh((logT - 4.2) / 0.15))
        data[:, 1 + c] = w * hot + (1.0 - w) * np.minimum(cold, 29.0)
    return data


def cooling_blob(cooling_type: int, nroot: int = 4, steps: int = 10, eos: int = C.EOS_SINGLE_SPECIE) -> Problem:
    """A hot, dense blob in a warm medium, in physical units (box 1 pc,
    l_sc = pc, d_sc = 1.3 amu, v_sc = 1 km/s): n from 10 to 1000 cm^-3 and T
    from 1e4 to 3e7 K, smooth, with a metallicity passive scalar of 0.05 to
    4 times the density (COOL_TABLE_METAL reads it), slow expansion.  For
    COOL_TABLE, COOL_TABLE_METAL and COOL_SCHURE with synthetic tables;
    cooling removes percents of the thermal energy per step.  `eos` selects
    the temperature calcTemp gives the cooling (single specie by default)."""
    mu0 = 1.3
    cfg = Config(npassive=1, solver_type=C.SOLVER_HLLC, limiter_type=C.LIMITER_MINMOD,
                 eos_type=eos, cooling_type=cooling_type, nbroot=(nroot,) * 3, maxlev=1,
                 gamma=5.0 / 3.0, cfl=0.4, visc_eta=5.0e-3, l_sc=C.PC, d_sc=mu0 * C.AMU, v_sc=1.0e5,
                 box=(C.PC,) * 3, tfin=1.0e9 * C.YR, dtout=1.0e9 * C.YR)
    tree = BlockTree(cfg.nbroot, 1).roots()
    c = np.array([0.5, 0.5, 0.5])

    def prim_fn(xyz):
        r = np.sqrt(((xyz - c[None, :, None, None, None]) ** 2).sum(axis=1))
        prim = np.zeros((xyz.shape[0], cfg.neqtot) + xyz.shape[2:])
        n = 10.0 + 990.0 * np.exp(-(r / 0.15) ** 2)
        T = 1.0e4 + 3.0e7 * np.exp(-(r / 0.12) ** 2)
        prim[:, 0] = n
        prim[:, 4] = n * mu0 * C.AMU / (mu0 * C.AMU) * C.KB * T / cfg.p_sc
        rr = np.maximum(r, 1e-12)
        for d in range(3):
            prim[:, 1 + d] = 3.0 * r * (xyz[:, d] - c[d]) / rr
        prim[:, 5] = n * (0.05 + 3.95 * 0.5 * (1.0 + np.sin(12.0 * xyz[:, 0]) * np.cos(9.0 * xyz[:, 1])))
        return prim

    kw = {}
    if cooling_type == C.COOL_TABLE:
        kw["cooltable"] = cooling_table_synthetic(200)
    elif cooling_type == C.COOL_TABLE_METAL:
        kw["cooltable_metal"] = metal_table_synthetic()
    elif cooling_type == C.COOL_SCHURE:
        kw["cooltable_schure"] = (schure_table_synthetic(), 2)
    return _finish(f"cooling-blob-{cooling_type}", cfg, tree, prim_fn, steps, **kw)
