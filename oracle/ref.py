"""TEST INFRASTRUCTURE ONLY: ctypes access to TOSCA's own stage functions,
compiled from the reference sources against single-rank PETSc/HYPRE/MPI
stand-ins (oracle/refstub, built into oracle/_ref/libtosca_ref.so). The
harness exports the C-ABI of include/tosca_gpu.h with the prefix "ref_", so a
`Solver` on it runs the reference's FormU, GradP, UpdateNut, SetCoeffMatrix,
SolvePEqn, ProjectVelocity, ... on the same inputs as the oracle restatement.
Imported only by tests/."""
from __future__ import annotations

import ctypes
import os
import subprocess

from tosca_b200 import api

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libtosca_ref.so")
_FNS = None
_LIB = None


def reference_src(root: str | None = None) -> str | None:
    """The reference checkout whose sources the harness compiles, if present."""
    root = root or os.environ.get("TOSCA_REFERENCE_ROOT") or "/root/reference"
    return root if os.path.isdir(os.path.join(root, "src")) else None


def build(root: str | None = None) -> str | None:
    """Compile the harness from the reference sources (None: no reference here)."""
    root = reference_src(root)
    if root is None:
        return None
    subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "refstub"), f"REF={root}", "-j8"], check=True)
    return LIB_PATH


def available(prebuilt_only: bool = False) -> bool:
    if prebuilt_only:
        return os.path.exists(LIB_PATH)
    return os.path.exists(LIB_PATH) or reference_src() is not None


def load(prebuilt_only: bool = False):
    """Bind the harness. prebuilt_only: use oracle/_ref as built, never look
    for (or rebuild from) a reference checkout."""
    global _FNS, _LIB
    if _FNS is None:
        if not prebuilt_only and (not os.path.exists(LIB_PATH) or reference_src() is not None):
            build()
        _LIB = ctypes.CDLL(LIB_PATH)
        _FNS = api.bind(_LIB, "ref_")
        _LIB.ref_poisson_size.restype = ctypes.c_int64
        _LIB.ref_poisson_size.argtypes = [ctypes.c_void_p]
        _LIB.ref_poisson_nnz.restype = ctypes.c_int64
        _LIB.ref_poisson_nnz.argtypes = [ctypes.c_void_p]
        _LIB.ref_poisson_matrix.restype = ctypes.c_int
        _LIB.ref_poisson_matrix.argtypes = [ctypes.c_void_p] * 4
        _LIB.ref_mo_ustar.restype = ctypes.c_double
        _LIB.ref_mo_ustar.argtypes = [ctypes.c_double] * 7
        _LIB.ref_mo_qwall.restype = ctypes.c_double
        _LIB.ref_mo_qwall.argtypes = [ctypes.c_double] * 9
    return _FNS


def solver(cfg: api.Config, prebuilt_only: bool = False) -> api.Solver:
    return api.Solver(cfg, load(prebuilt_only))


def poisson_matrix(s: api.Solver):
    """The matrix the reference's SetCoeffMatrix assembled, as scipy CSR."""
    import numpy as np
    import scipy.sparse as sp
    L = _LIB
    n = L.ref_poisson_size(s.h)
    nnz = L.ref_poisson_nnz(s.h)
    rp = np.zeros(n + 1, np.int64)
    col = np.zeros(nnz, np.int64)
    val = np.zeros(nnz)
    L.ref_poisson_matrix(s.h, rp.ctypes.data_as(ctypes.c_void_p), col.ctypes.data_as(ctypes.c_void_p),
                         val.ctypes.data_as(ctypes.c_void_p))
    return sp.csr_matrix((val, col, rp), shape=(n, n))


def mo_ustar(U, dist, z0, gamma_m, kappa, qwall, theta_ref) -> float:
    """TOSCA's uStarShumann (wallfunctions.c:12-130)."""
    load()
    return _LIB.ref_mo_ustar(U, dist, z0, gamma_m, kappa, qwall, theta_ref)


def mo_qwall(U, dist, z0, gamma_m, gamma_h, alpha_h, theta_ref, delta_theta, kappa) -> float:
    """TOSCA's qWallShumann (wallfunctions.c:133-290)."""
    load()
    return _LIB.ref_mo_qwall(U, dist, z0, gamma_m, gamma_h, alpha_h, theta_ref, delta_theta, kappa)
