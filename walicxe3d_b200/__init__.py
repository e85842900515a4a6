"""walicxe3d_b200 -- B200-native (sm_100a) per-block Godunov update of
Walicxe3D-style block-structured AMR hydro/MHD.

The compute path is libwx3d.so (CUDA C++, built by csrc/build.sh) behind the
C-ABI of include/wx3d.h; this package is its host-side Python mirror.
"""
from . import config, mesh, problems
from .config import Config
from ._lib import LIB_PATH, WxError, load
from .solver import Walicxe3D, from_problem

__all__ = ["config", "mesh", "problems", "Config", "Walicxe3D", "from_problem", "WxError", "load", "LIB_PATH"]
