"""ctypes binding of libwx3d.so (include/wx3d.h).

The shared library is built in-tree (``walicxe3d_b200/libwx3d.so``) by
``walicxe3d_b200/csrc/build.sh``.  There is no fallback: if the library is
missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

from .config import WxConfig, WxState, WxStatus

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libwx3d.so"

_lib = None

c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_float_p = ctypes.POINTER(ctypes.c_float)
c_void_p = ctypes.c_void_p

_SIGNATURES = {
    "wx3d_config_defaults": (ctypes.c_int, [ctypes.POINTER(WxConfig)]),
    "wx3d_init": (ctypes.c_int, [ctypes.POINTER(WxConfig), ctypes.c_int32, ctypes.POINTER(c_void_p)]),
    "wx3d_finalize": (ctypes.c_int, [c_void_p]),
    "wx3d_set_stream": (ctypes.c_int, [c_void_p, c_void_p]),
    "wx3d_set_mesh": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_int32_p]),
    "wx3d_set_mesh_halo": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_int32_p, ctypes.c_int32, c_int32_p]),
    "wx3d_step_part": (ctypes.c_int, [c_void_p, ctypes.c_int32]),
    "wx3d_get_dtmin": (ctypes.c_int, [c_void_p, c_double_p]),
    "wx3d_set_dtmin": (ctypes.c_int, [c_void_p, ctypes.c_double]),
    "wx3d_pack_blocks": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_void_p]),
    "wx3d_unpack_blocks": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_void_p]),
    "wx3d_pack_faces": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_void_p]),
    "wx3d_unpack_faces": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_void_p]),
    "wx3d_set_zsplit": (ctypes.c_int, [c_void_p, ctypes.c_int32]),
    "wx3d_set_fusion": (ctypes.c_int, [c_void_p, ctypes.c_int32]),
    "wx3d_set_winds": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_double_p]),
    "wx3d_autotune": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_double_p, c_int32_p]),
    "wx3d_get_neighbours": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_int32_p, c_int32_p]),
    "wx3d_write_bin": (ctypes.c_int, [c_void_p, ctypes.c_char_p]),
    "wx3d_read_bin": (ctypes.c_int, [c_void_p, ctypes.c_char_p, ctypes.c_int32, c_int32_p, c_int32_p]),
    "wx3d_write_state": (ctypes.c_int, [c_void_p, ctypes.c_char_p, ctypes.c_int32, ctypes.c_char_p]),
    "wx3d_read_state": (ctypes.c_int, [c_void_p, ctypes.c_char_p, c_int32_p, ctypes.c_char_p, ctypes.c_int32]),
    "wx3d_upload_blocks": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_double_p]),
    "wx3d_download_blocks": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_double_p]),
    "wx3d_upload_U_fortran": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_double_p]),
    "wx3d_download_U_fortran": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_double_p]),
    "wx3d_update_prims": (ctypes.c_int, [c_void_p]),
    "wx3d_download_prims": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_double_p]),
    "wx3d_set_state": (ctypes.c_int, [c_void_p, ctypes.POINTER(WxState)]),
    "wx3d_get_state": (ctypes.c_int, [c_void_p, ctypes.POINTER(WxState)]),
    "wx3d_get_timestep": (ctypes.c_int, [c_void_p, c_double_p]),
    "wx3d_hydro_solver": (ctypes.c_int, [c_void_p]),
    "wx3d_update_neutral_fraction": (ctypes.c_int, [c_void_p]),
    "wx3d_cooling": (ctypes.c_int, [c_void_p, c_double_p]),
    "wx3d_step": (ctypes.c_int, [c_void_p, ctypes.POINTER(WxState)]),
    "wx3d_run": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.POINTER(WxState)]),
    "wx3d_run_async": (ctypes.c_int, [c_void_p, ctypes.c_int32]),
    "wx3d_set_cooltable_metal": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, c_double_p]),
    "wx3d_set_cooltable_schure": (ctypes.c_int, [c_void_p, c_double_p, ctypes.c_int32]),
    "wx3d_set_cooltable": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_double_p, c_double_p]),
    "wx3d_mark": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_int32_p]),
    "wx3d_refine": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_int32_p]),
    "wx3d_coarsen": (ctypes.c_int, [c_void_p, c_int32_p, ctypes.c_int32]),
    "wx3d_admesh": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_int32_p, c_int32_p]),
    "wx3d_set_timing": (ctypes.c_int, [c_void_p, ctypes.c_int32]),
    "wx3d_kernel_times": (ctypes.c_int, [c_void_p, c_double_p, c_int32_p]),
    "wx3d_get_status": (ctypes.c_int, [c_void_p, ctypes.POINTER(WxStatus)]),
    "wx3d_reset_status": (ctypes.c_int, [c_void_p]),
    "wx3d_hydro_step_noalloc": (ctypes.c_int, [ctypes.POINTER(WxConfig), ctypes.c_int32, c_int32_p, c_void_p,
                                                c_void_p, ctypes.POINTER(WxState), c_void_p]),
    "wx3d_mlp_create": (ctypes.c_int, [ctypes.c_uint64, ctypes.POINTER(c_void_p)]),
    "wx3d_mlp_destroy": (ctypes.c_int, [c_void_p]),
    "wx3d_mlp_nparams": (ctypes.c_int, []),
    "wx3d_mlp_get_params": (ctypes.c_int, [c_void_p, c_float_p]),
    "wx3d_mlp_set_params": (ctypes.c_int, [c_void_p, c_float_p]),
    "wx3d_mlp_samples": (ctypes.c_int, [ctypes.POINTER(WxConfig), ctypes.c_int64, ctypes.c_uint64, c_void_p, c_void_p,
                                        c_void_p, c_void_p]),
    "wx3d_mlp_forward": (ctypes.c_int, [c_void_p, ctypes.c_int64, c_void_p, c_void_p, c_void_p]),
    "wx3d_mlp_gradient": (ctypes.c_int, [c_void_p, ctypes.c_int64, c_void_p, c_void_p, c_float_p, c_float_p]),
    "wx3d_mlp_train": (ctypes.c_int, [c_void_p, ctypes.c_int64, c_void_p, c_void_p, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_float, c_float_p]),
    "wx3d_check_fast_math": (ctypes.c_int, [ctypes.c_int32, c_double_p, ctypes.POINTER(ctypes.c_int64)]),
    "wx3d_measure_fp64_peak": (ctypes.c_int, [c_double_p]),
    "wx3d_check_wait_timeout": (ctypes.c_int, [ctypes.c_int32]),
    "wx3d_sources": (ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "wx3d_set_surrogate": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    "wx3d_error_string": (ctypes.c_char_p, [ctypes.c_int32]),
    "wx3d_last_error": (ctypes.c_int, [c_void_p, ctypes.c_char_p, ctypes.c_int32]),
}

EXPORTED = tuple(_SIGNATURES)


class WxError(RuntimeError):
    """A non-zero status returned by a wx3d_* entry point."""

    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        msg = f"{where} failed with status {code}"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load libwx3d.so (raises OSError if it is missing: there is no CPU path)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise OSError(
            f"{p} not found: build the CUDA library with walicxe3d_b200/csrc/build.sh "
            "(the package has no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(code: int, where: str, ctx=None) -> None:
    if code != 0:
        detail = ""
        lib = load()
        if ctx is not None:
            buf = ctypes.create_string_buffer(512)
            lib.wx3d_last_error(ctx, buf, 512)
            detail = buf.value.decode(errors="replace")
        if not detail:
            detail = (lib.wx3d_error_string(code) or b"").decode()
        raise WxError(code, where, detail)
