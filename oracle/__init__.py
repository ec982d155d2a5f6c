"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU restatement of TOSCA's
time step (tosca_oracle.cpp). Imported by tests/, the smoke check and the
CPU-baseline leg of bench.py; never by the product package."""
from __future__ import annotations

import ctypes
import os
import subprocess

from tosca_b200 import api

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libtosca_oracle.so")
_FNS = None
_LIB = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def load():
    global _FNS, _LIB
    if _FNS is None:
        if not os.path.exists(LIB_PATH):
            build()
        _LIB = ctypes.CDLL(LIB_PATH)
        _FNS = api.bind(_LIB, "tor_")
        _LIB.tor_poisson_size.restype = ctypes.c_int64
        _LIB.tor_poisson_size.argtypes = [ctypes.c_void_p]
        _LIB.tor_poisson_nnz.restype = ctypes.c_int64
        _LIB.tor_poisson_nnz.argtypes = [ctypes.c_void_p]
        _LIB.tor_poisson_matrix.restype = ctypes.c_int
        _LIB.tor_poisson_matrix.argtypes = [ctypes.c_void_p] * 4
        _LIB.tor_poisson_symmetric.restype = ctypes.c_int32
        _LIB.tor_poisson_symmetric.argtypes = [ctypes.c_void_p]
        _LIB.tor_num_threads.restype = ctypes.c_int32
        _LIB.tor_mo_ustar.restype = ctypes.c_double
        _LIB.tor_mo_ustar.argtypes = [ctypes.c_double] * 7
        _LIB.tor_mo_qwall.restype = ctypes.c_double
        _LIB.tor_mo_qwall.argtypes = [ctypes.c_double] * 9
    return _FNS


def lib():
    load()
    return _LIB


def solver(cfg: api.Config) -> api.Solver:
    return api.Solver(cfg, load())


def poisson_matrix(s: api.Solver):
    """Assembled pressure matrix of an oracle context as scipy CSR."""
    import numpy as np
    import scipy.sparse as sp
    L = lib()
    n = L.tor_poisson_size(s.h)
    nnz = L.tor_poisson_nnz(s.h)
    rp = np.zeros(n + 1, np.int64)
    col = np.zeros(nnz, np.int64)
    val = np.zeros(nnz)
    L.tor_poisson_matrix(s.h, rp.ctypes.data_as(ctypes.c_void_p), col.ctypes.data_as(ctypes.c_void_p),
                         val.ctypes.data_as(ctypes.c_void_p))
    return sp.csr_matrix((val, col, rp), shape=(n, n))


def mo_ustar(U, dist, z0, gamma_m, kappa, qwall, theta_ref) -> float:
    """The restatement's uStarShumann (friction velocity for a wall heat flux)."""
    return lib().tor_mo_ustar(U, dist, z0, gamma_m, kappa, qwall, theta_ref)


def mo_qwall(U, dist, z0, gamma_m, gamma_h, alpha_h, theta_ref, delta_theta, kappa) -> float:
    """The restatement's qWallShumann (wall heat flux for a temperature difference)."""
    return lib().tor_mo_qwall(U, dist, z0, gamma_m, gamma_h, alpha_h, theta_ref, delta_theta, kappa)
