"""CPU oracle of the per-block Godunov update -- TEST INFRASTRUCTURE.

A ctypes binding of oracle/_build/liboracle.so, the FP64 C++ restatement of
the reference Fortran routines (oracle/wx_oracle.cpp).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it, always as the
checker or the timed CPU reference, never as part of the product path.

PARITY UNPINNED: the reference ships no tests or golden data and no Fortran
compiler is available, so the restatement is pinned by physics checks
(exact Riemann solutions, conservation, symmetry) rather than by outputs of
the reference binary.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

from walicxe3d_b200.config import Config, WxConfig, WxState

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_lib = None


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < (HERE / "wx_oracle.cpp").stat().st_mtime:
        subprocess.run(["sh", str(HERE / "build.sh")], check=True)
    return LIB


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB))
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        sig = {
            "orc_create": (vp, [ctypes.POINTER(WxConfig), ctypes.c_int, ctypes.c_int]),
            "orc_destroy": (None, [vp]),
            "orc_set_threads": (None, [vp, ctypes.c_int]),
            "orc_set_blocks": (ctypes.c_int, [vp, ctypes.c_int, ip]),
            "orc_neighbors": (None, [vp, ctypes.c_int, ctypes.c_int, ip, ip]),
            "orc_sibling_coords": (None, [vp, ctypes.c_int, ip]),
            "orc_meshlevel": (ctypes.c_int, [vp, ctypes.c_int]),
            "orc_children": (None, [vp, ctypes.c_int, ip]),
            "orc_father": (ctypes.c_int, [vp, ctypes.c_int]),
            "orc_cell_pos": (None, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]),
            "orc_set_array": (None, [vp, ctypes.c_int, ctypes.c_int, dp]),
            "orc_get_array": (None, [vp, ctypes.c_int, ctypes.c_int, dp]),
            "orc_set_state": (None, [vp, ctypes.POINTER(WxState)]),
            "orc_get_state": (None, [vp, ctypes.POINTER(WxState)]),
            "orc_get_counters": (None, [vp, ctypes.POINTER(ctypes.c_longlong)]),
            "orc_update_prims": (None, [vp]),
            "orc_calc_prims": (None, [vp, ctypes.c_int, ctypes.c_int]),
            "orc_boundary": (None, [vp, ctypes.c_int, ctypes.c_int]),
            "orc_get_timestep": (ctypes.c_double, [vp]),
            "orc_hydro_solver": (None, [vp]),
            "orc_update_neutral_fraction": (None, [vp]),
            "orc_cooling": (ctypes.c_double, [vp]),
            "orc_step": (None, [vp]),
            "orc_set_cooltable": (ctypes.c_int, [vp, ctypes.c_int, dp, dp]),
            "orc_set_cooltable_metal": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, dp]),
            "orc_set_cooltable_schure": (ctypes.c_int, [vp, dp, ctypes.c_int]),
            "orc_add_wind": (ctypes.c_int, [vp, dp]),
            "orc_mark": (None, [vp, ip]),
            "orc_refine": (None, [vp, ctypes.c_int, ip]),
            "orc_coarsen": (None, [vp, ip, ctypes.c_int]),
            "orc_admesh": (ctypes.c_int, [vp, ip]),
            "orc_get_blocks": (None, [vp, ip]),
        }
        for n, (r, a) in sig.items():
            f = getattr(lib, n)
            f.restype = r
            f.argtypes = a
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


U_, UP_, PRIM_ = 0, 1, 2


class Oracle:
    """Reference-semantics state: U, UP, PRIM with two ghost layers per block."""

    def __init__(self, cfg: Config, nbmax: int, threads: int | None = None):
        self.lib = load()
        self.cfg = cfg
        self._c = cfg.to_c()
        self.nbmax = nbmax
        self.neq = cfg.neqtot
        self.h = self.lib.orc_create(ctypes.byref(self._c), nbmax, threads or 1)

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, n: int):
        self.lib.orc_set_threads(self.h, n)

    def set_blocks(self, bids):
        b = np.ascontiguousarray(bids, dtype=np.int32)
        assert self.lib.orc_set_blocks(self.h, len(b), _ip(b)) == 0

    def set_U(self, U: np.ndarray):
        """Physical cells of U in the native layout [nb][eq][k][j][i]."""
        full = np.zeros((self.nbmax, self.neq, 16, 16, 16))
        full[: U.shape[0]] = U
        self.lib.orc_set_array(self.h, U_, 0, _dp(np.ascontiguousarray(full)))

    def get(self, which: int = U_, full: bool = False) -> np.ndarray:
        shape = (self.nbmax, self.neq) + ((20, 20, 20) if full else (16, 16, 16))
        out = np.empty(shape)
        self.lib.orc_get_array(self.h, which, int(full), _dp(out))
        return out

    @property
    def U(self):
        return self.get(U_)

    @property
    def PRIM(self):
        return self.get(PRIM_)

    def set_state(self, time=0.0, dt=0.0, it=0, nextout=1, dumpout=0):
        s = WxState(time, dt, it, nextout, dumpout, 0)
        self.lib.orc_set_state(self.h, ctypes.byref(s))

    @property
    def state(self) -> WxState:
        s = WxState()
        self.lib.orc_get_state(self.h, ctypes.byref(s))
        return s

    def counters(self):
        a = (ctypes.c_longlong * 4)()
        self.lib.orc_get_counters(self.h, a)
        return list(a)

    def update_prims(self):
        self.lib.orc_update_prims(self.h)

    def boundary(self, depth: int, which: int = U_):
        self.lib.orc_boundary(self.h, depth, which)

    def get_timestep(self) -> float:
        return self.lib.orc_get_timestep(self.h)

    def hydro_solver(self):
        self.lib.orc_hydro_solver(self.h)

    def update_neutral_fraction(self):
        self.lib.orc_update_neutral_fraction(self.h)

    def cooling(self) -> float:
        return self.lib.orc_cooling(self.h)

    def step(self):
        self.lib.orc_step(self.h)

    def set_cooltable(self, logT, b):
        lt = np.ascontiguousarray(logT, dtype=np.float64)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        assert self.lib.orc_set_cooltable(self.h, len(lt), _dp(lt), _dp(bb)) == 0

    def set_cooltable_metal(self, nptsT, nptsZ, table):
        t = np.ascontiguousarray(table, dtype=np.float64)
        assert self.lib.orc_set_cooltable_metal(self.h, int(nptsT), int(nptsZ), _dp(t)) == 0

    def set_cooltable_schure(self, data, dmc_f):
        d = np.ascontiguousarray(np.asarray(data).reshape(-1), dtype=np.float64)
        assert self.lib.orc_set_cooltable_schure(self.h, _dp(d), int(dmc_f)) == 0

    def add_wind(self, params12):
        p = np.ascontiguousarray(params12, dtype=np.float64)
        self.lib.orc_add_wind(self.h, _dp(p))

    def mark(self) -> np.ndarray:
        f = np.zeros(self.nbmax, np.int32)
        self.lib.orc_mark(self.h, _ip(f))
        return f

    def refine(self, father, children):
        c = np.ascontiguousarray(children, dtype=np.int32)
        self.lib.orc_refine(self.h, int(father), _ip(c))

    def coarsen(self, children, father):
        c = np.ascontiguousarray(children, dtype=np.int32)
        self.lib.orc_coarsen(self.h, _ip(c), int(father))

    def admesh(self):
        """admesh (amr.f90:44-133) with one process; returns (blocks refined,
        families coarsened).  Raises on the reference's abort codes."""
        n = np.zeros(2, np.int32)
        rc = self.lib.orc_admesh(self.h, _ip(n))
        if rc:
            raise RuntimeError(f"oracle admesh aborted with code {rc}")
        return int(n[0]), int(n[1])

    @property
    def blocks(self) -> np.ndarray:
        """localBlocks (nbmax entries, -1 = empty slot)."""
        b = np.zeros(self.nbmax, np.int32)
        self.lib.orc_get_blocks(self.h, _ip(b))
        return b

    def neighbors(self, bid: int, direction: int):
        t = ctypes.c_int()
        lst = np.zeros(4, np.int32)
        self.lib.orc_neighbors(self.h, bid, direction, ctypes.byref(t), _ip(lst))
        return t.value, lst

    def sibling_coords(self, bid):
        s = np.zeros(3, np.int32)
        self.lib.orc_sibling_coords(self.h, bid, _ip(s))
        return tuple(int(v) for v in s)


def from_problem(prob, threads: int | None = None, extra_slots: int = 0) -> Oracle:
    """Oracle loaded with a Problem, primitives updated as main.f90:69 does."""
    o = Oracle(prob.cfg, prob.nblocks + extra_slots, threads=threads or os.cpu_count())
    o.set_blocks(prob.local_blocks)
    o.set_U(prob.U)
    if prob.cooltable is not None:
        o.set_cooltable(*prob.cooltable)
    if prob.cooltable_metal is not None:
        o.set_cooltable_metal(*prob.cooltable_metal)
    if prob.cooltable_schure is not None:
        o.set_cooltable_schure(*prob.cooltable_schure)
    for w in prob.winds:
        o.add_wind(w)
    o.set_state(0.0, 0.0, 0, 1, 0)
    o.update_prims()
    return o
