"""Run-time configuration mirroring the reference's compile-time parameters.

``WxConfig`` is the ctypes image of ``wx_config`` in ``include/wx3d.h``.  Its
fields are the parameters of ``source/parameters.f90`` that the hot path
reads (solver, limiter, BCs, gamma, CFL, viscosity, EOS, cooling, unit
scalings, root-block geometry); BFIELD, a Makefile switch in the reference,
is the ``bfield`` field.  Derived values follow ``source/parameters.f90``:
``cv = 1/(gamma-1)`` (:373), ``p_sc = d_sc*v_sc**2`` (:379), ``e_sc = p_sc``
(:380), ``t_sc = l_sc/v_sc`` (:381).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field, fields

# Enumerations of source/constants.f90:52-119
LEFT, RIGHT, FRONT, BACK, BOTTOM, TOP = 1, 2, 3, 4, 5, 6
BC_REFLECTIVE, BC_FREE_FLOW, BC_PERIODIC = 1, 2, 3
NEIGH_SAME, NEIGH_COARSER, NEIGH_FINER, NEIGH_BOUNDARY = 1, 2, 3, 4
FLAG_NONE, FLAG_REFINE, FLAG_COARSE = 0, 1, 2
SOLVER_LAX, SOLVER_HLL1, SOLVER_HLL, SOLVER_HLLC, SOLVER_HLLE, SOLVER_HLLD = 1, 2, 3, 4, 5, 6
(LIMITER_NO_AVERAGE, LIMITER_NONE, LIMITER_MINMOD, LIMITER_VANLEER, LIMITER_ALBADA,
 LIMITER_UMIST, LIMITER_WOODWARD, LIMITER_SUPERBEE) = -1, 0, 1, 2, 3, 4, 5, 6
EOS_ADIABATIC, EOS_SINGLE_SPECIE, EOS_TWOTEMP, EOS_H_RATE = 0, 1, 2, 3
COOL_NONE, COOL_TABLE, COOL_TABLE_METAL, COOL_H, COOL_SCHURE = 0, 1, 2, 3, 4

NCELLS = 16          # ncells_block (source/parameters.f90:113)
NGHOST = 2           # nghost (source/parameters.f90:209)
BLOCK_CELLS = NCELLS ** 3

# Physical constants (source/constants.f90:37-47)
AMU = 1.660538782e-24
KB = 1.380650400e-16
PC = 3.085677588e+18
YR = 3.155673600e+7
MSUN = 1.988920000e+33
KPS = 1.0e5
PI = 3.14159265358979


class WxConfig(ctypes.Structure):
    """ctypes image of ``wx_config`` (include/wx3d.h)."""

    _fields_ = [
        ("neqtot", ctypes.c_int32),
        ("npassive", ctypes.c_int32),
        ("bfield", ctypes.c_int32),
        ("mhd", ctypes.c_int32),
        ("solver_type", ctypes.c_int32),
        ("limiter_type", ctypes.c_int32),
        ("eos_type", ctypes.c_int32),
        ("cooling_type", ctypes.c_int32),
        ("bc", ctypes.c_int32 * 6),
        ("eight_wave", ctypes.c_int32),
        ("user_source_terms", ctypes.c_int32),
        ("enable_flux_cd", ctypes.c_int32),
        ("pad0", ctypes.c_int32),
        ("nbrootx", ctypes.c_int32),
        ("nbrooty", ctypes.c_int32),
        ("nbrootz", ctypes.c_int32),
        ("maxlev", ctypes.c_int32),
        ("gamma", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("visc_eta", ctypes.c_double),
        ("cooling_limit", ctypes.c_double),
        ("mu0", ctypes.c_double),
        ("mui", ctypes.c_double),
        ("ion_thres", ctypes.c_double),
        ("l_sc", ctypes.c_double),
        ("d_sc", ctypes.c_double),
        ("v_sc", ctypes.c_double),
        ("xphystot", ctypes.c_double),
        ("yphystot", ctypes.c_double),
        ("zphystot", ctypes.c_double),
        ("tfin", ctypes.c_double),
        ("dtout", ctypes.c_double),
        ("refine_thres", ctypes.c_double),
        ("coarse_thres", ctypes.c_double),
    ]


class WxState(ctypes.Structure):
    """ctypes image of ``wx_state`` (source/globals.f90:52-56)."""

    _fields_ = [
        ("time", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("it", ctypes.c_int32),
        ("nextout", ctypes.c_int32),
        ("dumpout", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]


class WxStatus(ctypes.Structure):
    """ctypes image of ``wx_status``."""

    _fields_ = [
        ("pressure_floor", ctypes.c_int64),
        ("density_floor", ctypes.c_int64),
        ("zero_density", ctypes.c_int64),
        ("nan_cells", ctypes.c_int64),
        ("max_cool_loss", ctypes.c_double),
        ("kernels_launched", ctypes.c_int64),
        ("surrogate_cells", ctypes.c_int64),
        ("fallback_cells", ctypes.c_int64),
    ]


@dataclass
class Config:
    """Python-side parameters; defaults are those of source/parameters.f90
    except the unit scalings (1 = code units) and the box (unit cube)."""

    npassive: int = 0
    bfield: bool = False
    mhd: bool = False
    solver_type: int = SOLVER_HLLC
    limiter_type: int = LIMITER_VANLEER
    eos_type: int = EOS_ADIABATIC
    cooling_type: int = COOL_NONE
    bc: tuple = (BC_FREE_FLOW,) * 6
    eight_wave: bool = False
    enable_flux_cd: bool = False
    nbroot: tuple = (1, 1, 1)
    maxlev: int = 1
    gamma: float = 5.0 / 3.0
    cfl: float = 0.4
    visc_eta: float = 5.0e-3
    cooling_limit: float = 0.5
    mu0: float = 1.3
    mui: float = 0.61
    ion_thres: float = 1.0e4
    l_sc: float = 1.0
    d_sc: float = 1.0
    v_sc: float = 1.0
    box: tuple = (1.0, 1.0, 1.0)
    tfin: float = 1.0e30
    dtout: float = 1.0e30
    refine_thres: float = 0.3
    coarse_thres: float = 0.03

    @property
    def neqtot(self) -> int:
        return 5 + (3 if self.bfield else 0) + self.npassive

    @property
    def firstpas(self) -> int:
        """0-based index of the first passive scalar (firstpas-1)."""
        return 5 + (3 if self.bfield else 0)

    @property
    def cv(self) -> float:
        return 1.0 / (self.gamma - 1.0)

    @property
    def p_sc(self) -> float:
        return self.d_sc * self.v_sc ** 2

    @property
    def t_sc(self) -> float:
        return self.l_sc / self.v_sc

    def dx(self, level: int) -> tuple:
        """Cell size per level (source/init.f90:726-730)."""
        s = float(2 ** (level - 1))
        return tuple(self.box[d] / (NCELLS * self.nbroot[d] * s) / self.l_sc for d in range(3))

    def to_c(self) -> WxConfig:
        c = WxConfig()
        c.neqtot = self.neqtot
        c.npassive = self.npassive
        c.bfield = int(self.bfield)
        c.mhd = int(self.mhd)
        c.solver_type = self.solver_type
        c.limiter_type = self.limiter_type
        c.eos_type = self.eos_type
        c.cooling_type = self.cooling_type
        for i in range(6):
            c.bc[i] = self.bc[i]
        c.eight_wave = int(self.eight_wave)
        c.user_source_terms = 0
        c.enable_flux_cd = int(self.enable_flux_cd)
        c.nbrootx, c.nbrooty, c.nbrootz = self.nbroot
        c.maxlev = self.maxlev
        c.gamma = self.gamma
        c.cfl = self.cfl
        c.visc_eta = self.visc_eta
        c.cooling_limit = self.cooling_limit
        c.mu0, c.mui, c.ion_thres = self.mu0, self.mui, self.ion_thres
        c.l_sc, c.d_sc, c.v_sc = self.l_sc, self.d_sc, self.v_sc
        c.xphystot, c.yphystot, c.zphystot = self.box
        c.tfin, c.dtout = self.tfin, self.dtout
        c.refine_thres, c.coarse_thres = self.refine_thres, self.coarse_thres
        return c
