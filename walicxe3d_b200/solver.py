"""Host-side mirror of the reference's hot-path module interface.

The reference drives the hot path through argument-less module subroutines
acting on globals (source/main.f90:79-122):

    hydroSolver()            -> Walicxe3D.hydro_solver()
    updatePrims()            -> Walicxe3D.update_prims()
    updateNeutralFraction()  -> Walicxe3D.update_neutral_fraction()
    cooling()                -> Walicxe3D.cooling()
    getTimestep(dt)          -> Walicxe3D.get_timestep()
    markByPhysical / refineBlock / coarseBlocks (data parts)
                             -> Walicxe3D.mark() / refine() / coarsen()

``Walicxe3D`` owns one wx3d context: the conserved variables of every block
live on the GPU; ``upload``/``download`` move them between host arrays
(native layout ``[slot][eq][k][j][i]``) and HBM.  Errors raise ``WxError``
carrying the reference's error code (source/constants.f90:135-162).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .config import BLOCK_CELLS, Config, WxState, WxStatus


def _i32(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Walicxe3D:
    """One GPU context of the per-block Godunov update."""

    def __init__(self, cfg: Config, max_blocks: int):
        self.lib = _lib.load()
        self.cfg = cfg
        self.max_blocks = int(max_blocks)
        self._c = cfg.to_c()
        h = ctypes.c_void_p()
        _lib.check(self.lib.wx3d_init(ctypes.byref(self._c), self.max_blocks, ctypes.byref(h)), "wx3d_init")
        self.ctx = h
        self.nslots = 0

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if self.ctx:
            self.lib.wx3d_finalize(self.ctx)
            self.ctx = None
        sur = getattr(self, "_surrogate", None)
        if sur is not None:
            sur.close()
            self._surrogate = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, code, where):
        _lib.check(code, where, self.ctx)

    # -- mesh and state -------------------------------------------------------
    def set_stream(self, stream_handle: int | None):
        self._chk(self.lib.wx3d_set_stream(self.ctx, ctypes.c_void_p(stream_handle or 0)), "wx3d_set_stream")

    def set_mesh(self, local_blocks):
        lb, p = _i32(local_blocks)
        self._chk(self.lib.wx3d_set_mesh(self.ctx, len(lb), p), "wx3d_set_mesh")
        self.nslots = len(lb)
        self.local_blocks = np.full(self.max_blocks, -1, np.int32)
        self.local_blocks[:len(lb)] = lb

    def admesh(self):
        """admesh (amr.f90:44-133): mark, proximity rule, refine and coarsen
        in the reference's slot order; updates ``local_blocks`` (all
        max_blocks slots, -1 = empty) and returns (blocks refined, families
        coarsened)."""
        lb = np.ascontiguousarray(self.local_blocks, dtype=np.int32)
        n = np.zeros(2, np.int32)
        self._chk(self.lib.wx3d_admesh(self.ctx, self.max_blocks, lb.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                       n.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))), "wx3d_admesh")
        self.local_blocks = lb
        self.nslots = self.max_blocks
        return int(n[0]), int(n[1])

    def set_zsplit(self, z: int):
        self._chk(self.lib.wx3d_set_zsplit(self.ctx, int(z)), "wx3d_set_zsplit")

    def set_winds(self, winds):
        """Spherical wind sources (rows of 12: xc yc zc vx vy vz radius mdot
        vinf temp mu y0, cgs), re-imposed after every ghost exchange as the
        reference's userBoundary does."""
        w = np.ascontiguousarray(np.asarray(winds, dtype=np.float64).reshape(-1, 12))
        self._chk(self.lib.wx3d_set_winds(self.ctx, len(w), w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                  "wx3d_set_winds")

    def set_fusion(self, on: bool):
        self._chk(self.lib.wx3d_set_fusion(self.ctx, int(bool(on))), "wx3d_set_fusion")

    SHAPES = ("1-fused", "1", "2", "4", "8")

    def autotune(self, reps: int = 3):
        """Measured choice of the stage launch shape (z-slab split, and for
        whole blocks whether the corrector carries the viscous step) for the
        current mesh; returns (split, fused, {shape: ms per solver pass})."""
        ms = (ctypes.c_double * 5)()
        best = (ctypes.c_int32 * 2)()
        self._chk(self.lib.wx3d_autotune(self.ctx, int(reps), ms, best), "wx3d_autotune")
        return best[0], bool(best[1]), dict(zip(self.SHAPES, list(ms)))

    def neighbours(self):
        n = self.nslots
        ft = np.zeros(n * 6, np.int32)
        fs = np.zeros(n * 24, np.int32)
        self._chk(self.lib.wx3d_get_neighbours(self.ctx, n, ft.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                               fs.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
                  "wx3d_get_neighbours")
        return ft.reshape(n, 6), fs.reshape(n, 6, 4)

    def upload(self, U: np.ndarray):
        U, p = _f64(U)
        assert U.shape[1] == self.cfg.neqtot and U.shape[2:] == (16, 16, 16)
        self._chk(self.lib.wx3d_upload_blocks(self.ctx, U.shape[0], p), "wx3d_upload_blocks")

    def download(self, nslots: int | None = None) -> np.ndarray:
        n = self.nslots if nslots is None else nslots
        out = np.empty((n, self.cfg.neqtot, 16, 16, 16))
        self._chk(self.lib.wx3d_download_blocks(self.ctx, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                  "wx3d_download_blocks")
        return out

    def upload_fortran(self, U: np.ndarray):
        """U in the reference's layout U(nbMaxProc, neq, -1:18, -1:18, -1:18)
        (Fortran order)."""
        a = np.asfortranarray(U, dtype=np.float64)
        p = a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self._chk(self.lib.wx3d_upload_U_fortran(self.ctx, a.shape[0], p), "wx3d_upload_U_fortran")

    def download_fortran(self, U: np.ndarray):
        assert U.flags.f_contiguous and U.dtype == np.float64
        p = U.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self._chk(self.lib.wx3d_download_U_fortran(self.ctx, U.shape[0], p), "wx3d_download_U_fortran")

    @property
    def state(self) -> WxState:
        s = WxState()
        self._chk(self.lib.wx3d_get_state(self.ctx, ctypes.byref(s)), "wx3d_get_state")
        return s

    def set_state(self, time=0.0, dt=0.0, it=0, nextout=1, dumpout=0):
        s = WxState(time, dt, it, nextout, dumpout, 0)
        self._chk(self.lib.wx3d_set_state(self.ctx, ctypes.byref(s)), "wx3d_set_state")

    def status(self) -> WxStatus:
        s = WxStatus()
        self._chk(self.lib.wx3d_get_status(self.ctx, ctypes.byref(s)), "wx3d_get_status")
        return s

    def reset_status(self):
        self._chk(self.lib.wx3d_reset_status(self.ctx), "wx3d_reset_status")

    # -- the reference's hot-path subroutines ---------------------------------
    def get_timestep(self) -> float:
        dt = ctypes.c_double()
        self._chk(self.lib.wx3d_get_timestep(self.ctx, ctypes.byref(dt)), "wx3d_get_timestep")
        return dt.value

    def hydro_solver(self):
        self._chk(self.lib.wx3d_hydro_solver(self.ctx), "wx3d_hydro_solver")

    def update_prims(self):
        self._chk(self.lib.wx3d_update_prims(self.ctx), "wx3d_update_prims")

    def prims(self) -> np.ndarray:
        out = np.empty((self.nslots, self.cfg.neqtot, 16, 16, 16))
        self._chk(self.lib.wx3d_download_prims(self.ctx, self.nslots,
                                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                  "wx3d_download_prims")
        return out

    def update_neutral_fraction(self):
        self._chk(self.lib.wx3d_update_neutral_fraction(self.ctx), "wx3d_update_neutral_fraction")

    def cooling(self) -> float:
        m = ctypes.c_double()
        self._chk(self.lib.wx3d_cooling(self.ctx, ctypes.byref(m)), "wx3d_cooling")
        return m.value

    # -- checkpoints (writeBin / writeState / warmstart) ----------------------
    def write_bin(self, path):
        self._chk(self.lib.wx3d_write_bin(self.ctx, str(path).encode()), "wx3d_write_bin")

    def read_bin(self, path) -> np.ndarray:
        """warmstart's block read: returns the new localBlocks registry."""
        lb = np.full(self.max_blocks, -1, np.int32)
        n = ctypes.c_int32()
        self._chk(self.lib.wx3d_read_bin(self.ctx, str(path).encode(), self.max_blocks,
                                         lb.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(n)),
                  "wx3d_read_bin")
        self.nslots = int(n.value)
        return lb

    def write_state(self, path, noutput: int, datadir: str = ""):
        self._chk(self.lib.wx3d_write_state(self.ctx, str(path).encode(), int(noutput), datadir.encode()),
                  "wx3d_write_state")

    def read_state(self, path):
        """warmstart's state read; returns (noutput, datadir)."""
        n = ctypes.c_int32()
        buf = ctypes.create_string_buffer(512)
        self._chk(self.lib.wx3d_read_state(self.ctx, str(path).encode(), ctypes.byref(n), buf, 512),
                  "wx3d_read_state")
        return int(n.value), buf.value.decode()

    def set_cooltable_metal(self, nptsT, nptsZ, table):
        t, p = _f64(table)
        self._chk(self.lib.wx3d_set_cooltable_metal(self.ctx, int(nptsT), int(nptsZ), p), "wx3d_set_cooltable_metal")

    def set_cooltable_schure(self, data, dmc_f):
        d, p = _f64(np.asarray(data).reshape(-1))
        self._chk(self.lib.wx3d_set_cooltable_schure(self.ctx, p, int(dmc_f)), "wx3d_set_cooltable_schure")

    def sources(self) -> float:
        """updatePrims + updateNeutralFraction + cooling in one fused pass
        (the surrogate's, when attached); returns maxloss."""
        m = ctypes.c_double()
        self._chk(self.lib.wx3d_sources(self.ctx, ctypes.byref(m)), "wx3d_sources")
        return m.value

    def set_cooltable(self, logT, b):
        logT, p1 = _f64(logT)
        b, p2 = _f64(b)
        self._chk(self.lib.wx3d_set_cooltable(self.ctx, len(logT), p1, p2), "wx3d_set_cooltable")

    def step(self) -> WxState:
        s = WxState()
        self._chk(self.lib.wx3d_step(self.ctx, ctypes.byref(s)), "wx3d_step")
        return s

    def run(self, nsteps: int) -> WxState:
        s = WxState()
        self._chk(self.lib.wx3d_run(self.ctx, int(nsteps), ctypes.byref(s)), "wx3d_run")
        return s

    def run_async(self, nsteps: int):
        self._chk(self.lib.wx3d_run_async(self.ctx, int(nsteps)), "wx3d_run_async")

    def mark(self) -> np.ndarray:
        f = np.zeros(self.nslots, np.int32)
        self._chk(self.lib.wx3d_mark(self.ctx, self.nslots, f.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
                  "wx3d_mark")
        return f

    def refine(self, father_slot: int, child_slots):
        ch, p = _i32(child_slots)
        self._chk(self.lib.wx3d_refine(self.ctx, int(father_slot), p), "wx3d_refine")

    def coarsen(self, child_slots, father_slot: int):
        ch, p = _i32(child_slots)
        self._chk(self.lib.wx3d_coarsen(self.ctx, p, int(father_slot)), "wx3d_coarsen")

    def attach_surrogate(self, params=None, trust=None):
        """Source steps of step()/run() use the trained MLP where its trust
        table allows and the plain integrator elsewhere.  Defaults to the
        network shipped in walicxe3d_b200/data."""
        from .surrogate import Surrogate
        if params is None or trust is None:
            from .train_surrogate import load
            p0, t0 = load()
            params = p0 if params is None else params
            trust = t0 if trust is None else trust
        self._surrogate = Surrogate()
        self._surrogate.params = params
        tb = np.ascontiguousarray(trust, dtype=np.uint8).ravel()
        self._chk(self.lib.wx3d_set_surrogate(self.ctx, self._surrogate.h, tb.ctypes.data_as(ctypes.c_void_p),
                                              tb.size, 1), "wx3d_set_surrogate")

    def detach_surrogate(self):
        self._chk(self.lib.wx3d_set_surrogate(self.ctx, None, None, 0, 0), "wx3d_set_surrogate")

    def set_timing(self, on: bool):
        self._chk(self.lib.wx3d_set_timing(self.ctx, int(bool(on))), "wx3d_set_timing")

    def kernel_times(self):
        """(ms, count) per kernel kind: predictor, corrector, viscous, sources."""
        ms = (ctypes.c_double * 4)()
        cnt = (ctypes.c_int32 * 4)()
        self._chk(self.lib.wx3d_kernel_times(self.ctx, ms, cnt), "wx3d_kernel_times")
        return list(ms), list(cnt)

    @property
    def kernels_launched(self) -> int:
        return int(self.status().kernels_launched)


def from_problem(prob, extra_slots: int = 0) -> Walicxe3D:
    """Context loaded with a Problem's mesh, state and tables."""
    w = Walicxe3D(prob.cfg, prob.nblocks + extra_slots)
    w.set_mesh(prob.local_blocks)
    w.upload(prob.U)
    if prob.cooltable is not None:
        w.set_cooltable(*prob.cooltable)
    if prob.cooltable_metal is not None:
        w.set_cooltable_metal(*prob.cooltable_metal)
    if prob.cooltable_schure is not None:
        w.set_cooltable_schure(*prob.cooltable_schure)
    if prob.winds:
        w.set_winds(prob.winds)
    w.set_state(time=0.0, dt=0.0, it=0, nextout=1)
    return w


__all__ = ["Walicxe3D", "from_problem", "BLOCK_CELLS"]
