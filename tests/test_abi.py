"""The C-ABI library loads and exports every entry point include/wx3d.h
declares; no compute call is made here."""
import ctypes
import re
from pathlib import Path

import pytest

from conftest import ROOT, gpu_available
from walicxe3d_b200 import _lib
from walicxe3d_b200.config import WxConfig, WxState, WxStatus

HEADER = ROOT / "include" / "wx3d.h"


def declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wx3d_[A-Za-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), f"{n} not exported by {_lib.LIB_PATH}"
    assert set(names) == set(_lib.EXPORTED)


def test_struct_sizes_match_header():
    # wx_config: 17 int32 fields (+ 5 for bc[6] beyond one) then 17 doubles
    assert ctypes.sizeof(WxConfig) == 4 * 22 + 8 * 17
    assert ctypes.sizeof(WxState) == 32
    assert ctypes.sizeof(WxStatus) == 64


def test_config_defaults_match_parameters_f90():
    lib = _lib.load()
    c = WxConfig()
    assert lib.wx3d_config_defaults(ctypes.byref(c)) == 0
    assert c.solver_type == 4 and c.limiter_type == 2 and c.cfl == 0.4 and c.visc_eta == 5.0e-3
    assert c.gamma == 5.0 / 3.0 and c.neqtot == 5 and list(c.bc) == [2] * 6


def test_error_strings():
    lib = _lib.load()
    assert lib.wx3d_error_string(0) == b"ok"
    assert lib.wx3d_error_string(23) == b"zero density"


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_init_fails_loudly_without_a_gpu():
    lib = _lib.load()
    c = WxConfig()
    lib.wx3d_config_defaults(ctypes.byref(c))
    h = ctypes.c_void_p()
    assert lib.wx3d_init(ctypes.byref(c), 8, ctypes.byref(h)) == 105  # WX_ERR_NO_DEVICE
    assert not h.value


def test_unsupported_configs_rejected_before_device_use():
    lib = _lib.load()
    h = ctypes.c_void_p()
    c = WxConfig()
    lib.wx3d_config_defaults(ctypes.byref(c))
    c.bc[0] = 3  # BC_PERIODIC: not implemented by the reference
    assert lib.wx3d_init(ctypes.byref(c), 8, ctypes.byref(h)) == 104
    lib.wx3d_config_defaults(ctypes.byref(c))
    c.mhd = 1  # mhd without BFIELD computes no time step in the reference
    assert lib.wx3d_init(ctypes.byref(c), 8, ctypes.byref(h)) == 104
    lib.wx3d_config_defaults(ctypes.byref(c))
    c.eos_type = 3  # H_RATE needs a passive scalar
    assert lib.wx3d_init(ctypes.byref(c), 8, ctypes.byref(h)) == 26
    # the field-CD update of B needs an active field, excludes the 8-wave
    # source and applies to the Godunov solvers only
    lib.wx3d_config_defaults(ctypes.byref(c))
    c.enable_flux_cd = 1
    assert lib.wx3d_init(ctypes.byref(c), 8, ctypes.byref(h)) == 104
    c.bfield, c.mhd, c.neqtot, c.npassive, c.solver_type = 1, 1, 8, 0, 6  # HLLD
    c.eight_wave = 1
    assert lib.wx3d_init(ctypes.byref(c), 8, ctypes.byref(h)) == 104
    c.eight_wave, c.solver_type = 0, 1  # Lax-Friedrichs
    assert lib.wx3d_init(ctypes.byref(c), 8, ctypes.byref(h)) == 104


def test_package_has_no_cpu_fallback(tmp_path):
    with pytest.raises(OSError):
        _lib.load(tmp_path / "missing.so")
