"""B200-native fractional time step of TOSCA (momentum RHS, pressure Poisson
solve, projection) behind the C-ABI of include/tosca_gpu.h.

`load()` returns the bound entry points of the in-tree CUDA library
tosca_b200/_build/libtosca_gpu.so. There is no CPU fallback: if the library is
missing, loading raises.
"""
from __future__ import annotations

import ctypes
import os

from . import api
from .api import Config, Solver, TgError, TgStats  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libtosca_gpu.so")
_FNS = None


def load() -> dict:
    """Load and bind the CUDA library (prefix tg_)."""
    global _FNS
    if _FNS is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library not built: {LIB_PATH} (run __graft_entry__.build())")
        lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
        _FNS = api.bind(lib, "tg_")
    return _FNS


def gpu_solver(cfg: Config) -> Solver:
    """A Solver context on the CUDA library."""
    return Solver(cfg, load())
