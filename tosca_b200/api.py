"""ctypes mirror of the C-ABI in include/tosca_gpu.h.

`Solver` wraps one context of a library that exports the tg_* entry points
(the CUDA library, prefix "tg_") or the same entry points under another prefix.
Arrays are numpy float64 in TOSCA's DMDA layout: shape (mz, my, mx) for scalars
and (mz, my, mx, 3) for Cmpnts vectors, i fastest (base.h:80-84).

The stage methods carry the names of the reference functions they replace so a
test reads like the reference's time loop (src/main.c:54-327).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

# ------------------------------------------------------------------ constants
TG_OK, TG_ERR_CUDA, TG_ERR_BAD_ARG, TG_ERR_NOT_CONVERGED, TG_ERR_NAN, TG_ERR_ALLOC, TG_ERR_STATE = range(7)

BC_PERIODIC, BC_NOSLIP, BC_SLIP, BC_WALL_SHUMANN, BC_FIXED_VALUE, BC_ZERO_GRADIENT, BC_INLET_LOG = 0, 1, 2, 3, 4, 5, 6
NUTBC_PERIODIC, NUTBC_ZEROGRADIENT, NUTBC_FIXEDVALUE = 0, 1, 2
DIV_CENTRAL, DIV_QUICK = 0, 1
DDT_FE, DDT_RK4, DDT_CN, DDT_ABCN, DDT_RK3WCN, DDT_RK3SOCN = 0, 1, 2, 3, 4, 5
TDDT_RK4, TDDT_ABBE, TDDT_BE, TDDT_BDF2 = 0, 1, 2, 3
TBC_ZERO_GRADIENT, TBC_FIXED_VALUE, TBC_FIXED_GRADIENT, TBC_PERIODIC, TBC_WALL_FUNCTION = 0, 1, 2, 3, 4
TWALL_FIXED_FLUX, TWALL_SHUMANN, TWALL_SURFACE_SERIES = -2, -3, -4
PREC_FP64, PREC_MIXED = 0, 1

FIELDS = [
    "CENT", "CSI", "ETA", "ZET", "ICSI", "IETA", "IZET", "JCSI", "JETA", "JZET",
    "KCSI", "KETA", "KZET", "AJ", "IAJ", "JAJ", "KAJ",
    "UCONT", "UCAT", "UCONT_O", "RHS", "DP", "BTHETA",
    "P", "PHI", "NUT", "TMPRT", "TAUWALL", "SOURCE",
    "UCONT_ADJ", "UCAT_ADJ", "P_ADJ", "SOURCE_ADJ",
    "FARM_FORCE", "FARM_CONT", "WALL_ADJ",
    "QWALL", "SURF_THETA",
]
F = {name: i for i, name in enumerate(FIELDS)}
SCALAR_FIELDS = {"AJ", "IAJ", "JAJ", "KAJ", "P", "PHI", "NUT", "TMPRT", "P_ADJ"}


class TgConfig(C.Structure):
    _fields_ = [
        ("mx", C.c_int32), ("my", C.c_int32), ("mz", C.c_int32),
        ("bc", C.c_int32 * 6),
        ("nut_bc", C.c_int32 * 6),
        ("nut_bc_value", C.c_double * 6),
        ("curvilinear", C.c_int32),
        ("les", C.c_int32),
        ("cs", C.c_double),
        ("nu", C.c_double),
        ("div_scheme", C.c_int32),
        ("ddt_scheme", C.c_int32),
        ("dt", C.c_double),
        ("buoyancy", C.c_int32),
        ("t_ref", C.c_double),
        ("mean_grad_p", C.c_int32),
        ("mean_grad_p_value", C.c_double * 3),
        ("wall_roughness", C.c_double),
        ("wall_kappa", C.c_double),
        ("poisson_rtol", C.c_double),
        ("poisson_div_tol", C.c_double),
        ("poisson_maxit", C.c_int32),
        ("precision", C.c_int32),
        ("it_start", C.c_int32),
        ("device", C.c_int32),
        ("source", C.c_int32),
        ("teqn", C.c_int32),
        ("t_bc", C.c_int32 * 6),
        ("prandtl", C.c_double),
        ("t_bc_value", C.c_double * 6),
        ("snes_atol", C.c_double),
        ("snes_rtol", C.c_double),
        ("snes_maxit", C.c_int32),
        ("gmres_restart", C.c_int32),
        ("t_ddt_scheme", C.c_int32),
        ("t_gmres_restart", C.c_int32),
        ("t_atol", C.c_double),
        ("t_rtol", C.c_double),
        ("p_tilde", C.c_int32),
        ("poisson_guess", C.c_int32),
        ("t_wall_type", C.c_int32),
        ("t_wall_localized", C.c_int32),
        ("t_wall_qwall", C.c_double),
        ("t_wall_heating_rate", C.c_double),
        ("t_wall_kappa", C.c_double),
        ("t_wall_theta_ref", C.c_double),
        ("t_wall_roughness", C.c_double),
        ("t_wall_gamma_m", C.c_double),
        ("t_wall_gamma_h", C.c_double),
        ("t_wall_alpha_h", C.c_double),
        ("wall_gamma_m", C.c_double),
        ("wall_theta_ref", C.c_double),
        ("t_start", C.c_double),
        ("bc_value", C.c_double * 18),
        ("inlet_u_tau", C.c_double),
        ("inlet_z0", C.c_double),
        ("inlet_h_inv", C.c_double),
        ("inlet_dir", C.c_double * 3),
    ]


class TgTurbine(C.Structure):
    """tg_turbine: one uniform actuator disk (C_T', sampled on the rotor disk)."""
    _fields_ = [
        ("center", C.c_double * 3),
        ("axis", C.c_double * 3),
        ("up", C.c_double * 3),
        ("r_tip", C.c_double),
        ("r_hub", C.c_double),
        ("epsilon", C.c_double),
        ("ct", C.c_double),
        ("n_radial", C.c_int32),
        ("n_azimuth", C.c_int32),
    ]

    @classmethod
    def make(cls, center, axis=(-1.0, 0.0, 0.0), up=(0.0, 0.0, 1.0), r_tip=63.0, r_hub=1.5, epsilon=20.0,
             ct=1.33, n_radial=10, n_azimuth=24):
        t = cls()
        t.center[:] = center
        t.axis[:] = axis
        t.up[:] = up
        t.r_tip, t.r_hub, t.epsilon, t.ct = r_tip, r_hub, epsilon, ct
        t.n_radial, t.n_azimuth = n_radial, n_azimuth
        return t


class TgAdjointStats(C.Structure):
    _fields_ = [
        ("steps", C.c_int64),
        ("forward_steps", C.c_int64),
        ("snapshots", C.c_int32),
        ("poisson_iterations", C.c_int32),
        ("seconds", C.c_double),
    ]


class TgStats(C.Structure):
    _fields_ = [
        ("steps", C.c_int64),
        ("poisson_iterations", C.c_int32),
        ("poisson_total_iterations", C.c_int32),
        ("poisson_initial_residual", C.c_double),
        ("poisson_final_residual", C.c_double),
        ("max_divergence", C.c_double),
        ("seconds", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


@dataclass
class Config:
    """Python view of tg_config (include/tosca_gpu.h)."""
    mx: int
    my: int
    mz: int
    bc: tuple = (BC_PERIODIC,) * 6
    nut_bc: tuple = (NUTBC_PERIODIC,) * 6
    nut_bc_value: tuple = (0.0,) * 6
    curvilinear: int = 0
    les: int = 0
    cs: float = 0.0289
    nu: float = 1.0 / 1600.0
    div_scheme: int = DIV_CENTRAL
    ddt_scheme: int = DDT_FE
    dt: float = 0.005
    buoyancy: int = 0
    t_ref: float = 300.0
    mean_grad_p: int = 0
    mean_grad_p_value: tuple = (0.0, 0.0, 0.0)
    wall_roughness: float = 0.1
    wall_kappa: float = 0.4
    poisson_rtol: float = 1e-14
    poisson_div_tol: float = 0.0
    poisson_maxit: int = 5000
    precision: int = PREC_FP64
    it_start: int = 0
    device: int = 0
    source: int = 0
    teqn: int = 0
    t_bc: tuple = (TBC_PERIODIC,) * 6
    prandtl: float = 0.7
    t_bc_value: tuple = (0.0,) * 6
    snes_atol: float = 1e-5
    snes_rtol: float = 1e-30
    snes_maxit: int = 20
    gmres_restart: int = 30
    t_ddt_scheme: int = 0
    t_gmres_restart: int = 30
    t_atol: float = 1e-5
    t_rtol: float = 1e-30
    p_tilde: int = 0
    poisson_guess: int = 2
    # thetaWallFunction on the jLeft temperature patch (t_bc[2] = TBC_WALL_FUNCTION)
    t_wall_type: int = TWALL_SHUMANN
    t_wall_localized: int = 0
    t_wall_qwall: float = 0.0
    t_wall_heating_rate: float = 0.0
    t_wall_kappa: float = 0.4
    t_wall_theta_ref: float = 300.0
    t_wall_roughness: float = 0.1
    t_wall_gamma_m: float = 4.8
    t_wall_gamma_h: float = 7.8
    t_wall_alpha_h: float = 1.0
    # stability correction of the velocity wall function (with a thetaWallFunction)
    wall_gamma_m: float = 4.8
    wall_theta_ref: float = 300.0
    t_start: float = 0.0
    # TG_BC_FIXED_VALUE patches: Cartesian velocity of patch p at [3p, 3p + 2]
    bc_value: tuple = (0.0,) * 18
    # BC_INLET_LOG on kLeft (inletFunction type 2): uTau, roughness, hInv, Udir
    inlet_u_tau: float = 0.4
    inlet_z0: float = 0.1
    inlet_h_inv: float = 1.0e30
    inlet_dir: tuple = (1.0, 0.0, 0.0)

    def to_c(self) -> TgConfig:
        c = TgConfig()
        for name, _ in TgConfig._fields_:
            v = getattr(self, name)
            if isinstance(v, (tuple, list)):
                arr = getattr(c, name)
                for q, x in enumerate(v):
                    arr[q] = x
            else:
                setattr(c, name, v)
        return c

    @property
    def cells(self) -> int:
        return (self.mx - 2) * (self.my - 2) * (self.mz - 2)


_SIGS = {
    "create": (C.c_int, [C.POINTER(TgConfig), C.POINTER(C.c_void_p)]),
    "destroy": (C.c_int, [C.c_void_p]),
    "last_error": (C.c_char_p, [C.c_void_p]),
    "status_string": (C.c_char_p, [C.c_int]),
    "set_mesh_nodes": (C.c_int, [C.c_void_p, C.c_void_p]),
    "set_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]),
    "get_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]),
    "init_from_cartesian": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "contravariant_to_cartesian": (C.c_int, [C.c_void_p]),
    "update_nut": (C.c_int, [C.c_void_p]),
    "update_wall_models": (C.c_int, [C.c_void_p]),
    "grad_p": (C.c_int, [C.c_void_p]),
    "buoyancy": (C.c_int, [C.c_void_p]),
    "update_wall_models_t": (C.c_int, [C.c_void_p]),
    "update_temperature_bcs": (C.c_int, [C.c_void_p]),
    "set_surface_temperature": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "form_u": (C.c_int, [C.c_void_p, C.c_double, C.c_int32]),
    "explicit_rhs": (C.c_int, [C.c_void_p]),
    "solve_u": (C.c_int, [C.c_void_p]),
    "solve_p": (C.c_int, [C.c_void_p, C.POINTER(TgStats)]),
    "continuity_error": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "update_cartesian_bcs": (C.c_int, [C.c_void_p]),
    "update_contravariant_bcs": (C.c_int, [C.c_void_p]),
    "sync_pressure": (C.c_int, [C.c_void_p]),
    "step": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(TgStats)]),
    "step_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(TgStats)]),
    "write_field_petsc": (C.c_int, [C.c_void_p, C.c_int32, C.c_char_p]),
    "read_field_petsc": (C.c_int, [C.c_void_p, C.c_int32, C.c_char_p]),
    "set_turbines": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(TgTurbine), C.c_double]),
    "set_turbine_ct": (C.c_int, [C.c_void_p, C.c_void_p]),
    "turbine_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_int32]),
    "set_farm_objective": (C.c_int, [C.c_void_p, C.c_int32]),
    "ct_gradient": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "momentum_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
}

# adjoint entry points (the CPU restatement exports tor_adjoint_step only) and
# the step-replay switch of the CUDA library
_ADJ_SIGS = {
    "adjoint_step": (C.c_int, [C.c_void_p]),
    "adjoint_forward": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(TgStats)]),
    "adjoint_reverse": (C.c_int, [C.c_void_p, C.POINTER(TgAdjointStats)]),
    "adjoint_set_tapes": (C.c_int, [C.c_void_p, C.c_int32]),
    "set_graphs": (C.c_int, [C.c_void_p, C.c_int32]),
    "graph_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "mesh_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
}

ENTRY_POINTS = tuple(_SIGS) + tuple(_ADJ_SIGS)


def bind(lib: C.CDLL, prefix: str) -> dict:
    """Attach argument/return types to every entry point of `lib` and return
    them keyed by their unprefixed name. Raises AttributeError if one is missing."""
    out = {}
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
        out[name] = fn
    for name, (res, args) in _ADJ_SIGS.items():
        fn = getattr(lib, prefix + name, None)
        if fn is not None:
            fn.restype = res
            fn.argtypes = args
            out[name] = fn
    return out


class TgError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Solver:
    """One tg_ctx. `fns` comes from bind(); the CUDA library is bound by
    tosca_b200.load()."""

    def __init__(self, cfg: Config, fns: dict):
        self.cfg = cfg
        self.fns = fns
        self._c = cfg.to_c()
        h = C.c_void_p()
        st = fns["create"](C.byref(self._c), C.byref(h))
        if st != TG_OK:
            raise TgError(st, "create failed: " + fns["status_string"](st).decode())
        self.h = h
        self.last_stats = TgStats()

    # ---------------------------------------------------------------- helpers
    def _check(self, st: int, what: str):
        if st != TG_OK:
            msg = self.fns["last_error"](self.h)
            raise TgError(st, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "h", None):
            self.fns["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def shape(self):
        return (self.cfg.mz, self.cfg.my, self.cfg.mx)

    # ------------------------------------------------------------------ data
    def set_mesh_nodes(self, nodes: np.ndarray):
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        assert nodes.shape == self.shape + (3,)
        self._check(self.fns["set_mesh_nodes"](self.h, _ptr(nodes)), "set_mesh_nodes")

    def field_shape(self, name: str, halo: int = 0) -> tuple:
        """Host array shape of a field: planes (mz, mx[, 3]) for the wall-model
        fields, (mz, my, mx[, 3]) plus 2*halo per direction otherwise."""
        mz, my, mx = self.shape
        if name in ("TAUWALL", "WALL_ADJ"):
            return (mz, mx, 3)
        if name in ("QWALL", "SURF_THETA"):
            return (mz, mx)
        shp = (mz + 2 * halo, my + 2 * halo, mx + 2 * halo)
        return shp if name in SCALAR_FIELDS else shp + (3,)

    def get(self, name: str, halo: int = 0) -> np.ndarray:
        out = np.zeros(self.field_shape(name, halo))
        self._check(self.fns["get_field"](self.h, F[name], _ptr(out), halo), f"get_field {name}")
        return out

    def set(self, name: str, arr: np.ndarray, halo: int = 0):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        want = self.field_shape(name, halo)
        if arr.size != int(np.prod(want)):
            raise ValueError(f"set_field {name}: {arr.shape} does not match {want}")
        self._check(self.fns["set_field"](self.h, F[name], _ptr(arr), halo), f"set_field {name}")

    # ----------------------------------------------------- TOSCA field files
    # file names of readFields / writeFields (io.c:247-420, 2261)
    FILE_FIELDS = {"V": "UCONT", "U": "UCAT", "p": "P", "nut": "NUT", "T": "TMPRT"}

    def write_field_petsc(self, name: str, path: str):
        self._check(self.fns["write_field_petsc"](self.h, F[name], path.encode()), f"write_field_petsc {name}")

    def read_field_petsc(self, name: str, path: str):
        self._check(self.fns["read_field_petsc"](self.h, F[name], path.encode()), f"read_field_petsc {name}")

    def write_fields(self, directory: str):
        """V, U, p (and nut with LES, T with the temperature equation) as TOSCA writes
        them into a time directory."""
        import os
        os.makedirs(directory, exist_ok=True)
        for fname, field in self.FILE_FIELDS.items():
            if (fname == "nut" and not self.cfg.les) or (fname == "T" and not getattr(self.cfg, "teqn", 0)):
                continue
            self.write_field_petsc(field, os.path.join(directory, fname))

    def read_fields(self, directory: str):
        """The fields of a TOSCA time directory that this configuration uses."""
        import os
        for fname, field in self.FILE_FIELDS.items():
            path = os.path.join(directory, fname)
            if os.path.exists(path):
                self.read_field_petsc(field, path)

    def init_from_cartesian(self, ucat: np.ndarray, halo: int = 0):
        ucat = np.ascontiguousarray(ucat, dtype=np.float64)
        self._check(self.fns["init_from_cartesian"](self.h, _ptr(ucat), halo), "init_from_cartesian")

    # ---------------------------------------------------------------- stages
    def contravariantToCartesian(self):
        self._check(self.fns["contravariant_to_cartesian"](self.h), "contravariantToCartesian")

    def UpdateNut(self):
        self._check(self.fns["update_nut"](self.h), "UpdateNut")

    def UpdateWallModelsU(self):
        self._check(self.fns["update_wall_models"](self.h), "UpdateWallModelsU")

    def GradP(self):
        self._check(self.fns["grad_p"](self.h), "GradP")

    def Buoyancy(self):
        self._check(self.fns["buoyancy"](self.h), "Buoyancy")

    def UpdateWallModelsT(self):
        self._check(self.fns["update_wall_models_t"](self.h), "UpdateWallModelsT")

    def UpdateTemperatureBCs(self):
        self._check(self.fns["update_temperature_bcs"](self.h), "UpdateTemperatureBCs")

    def set_surface_temperature(self, time, temp):
        """The surface temperature series of thetaWallFunction -4."""
        t = np.ascontiguousarray(time, dtype=np.float64)
        v = np.ascontiguousarray(temp, dtype=np.float64)
        if t.shape != v.shape or t.ndim != 1:
            raise ValueError("time and temperature must be 1-D arrays of one length")
        self._check(self.fns["set_surface_temperature"](self.h, int(t.size), _ptr(t), _ptr(v)), "set_surface_temperature")

    def FormU(self, scale: float = 1.0, zero_rhs: bool = True):
        self._check(self.fns["form_u"](self.h, scale, 1 if zero_rhs else 0), "FormU")

    def ExplicitRhsU(self):
        self._check(self.fns["explicit_rhs"](self.h), "ExplicitRhsU")

    def SolveUEqn(self):
        self._check(self.fns["solve_u"](self.h), "SolveUEqn")

    def SolvePEqn(self) -> TgStats:
        st = TgStats()
        self._check(self.fns["solve_p"](self.h, C.byref(st)), "SolvePEqn")
        return st

    def ContinuityErrorsOptimized(self) -> float:
        v = C.c_double()
        self._check(self.fns["continuity_error"](self.h, C.byref(v)), "ContinuityErrorsOptimized")
        return v.value

    def UpdateCartesianBCs(self):
        self._check(self.fns["update_cartesian_bcs"](self.h), "UpdateCartesianBCs")

    def UpdateContravariantBCs(self):
        self._check(self.fns["update_contravariant_bcs"](self.h), "UpdateContravariantBCs")

    def SyncPressureAcrossDomains(self):
        self._check(self.fns["sync_pressure"](self.h), "SyncPressureAcrossDomains")

    def step(self, n: int = 1) -> TgStats:
        st = TgStats()
        self._check(self.fns["step"](self.h, n, C.byref(st)), "step")
        self.last_stats = st
        return st

    # --------------------------------------------------------------- adjoint
    def adjoint_step(self):
        """VJP of one step at the current state (adjoint fields in, adjoint fields out)."""
        self._check(self.fns["adjoint_step"](self.h), "adjoint_step")

    def adjoint_forward(self, n: int, nsnap: int) -> TgStats:
        st = TgStats()
        self._check(self.fns["adjoint_forward"](self.h, n, nsnap, C.byref(st)), "adjoint_forward")
        return st

    def adjoint_set_tapes(self, max_tapes: int):
        """Cap the step tapes of the segment checkpoint schedule (-1: memory decides, 0: none)."""
        self._check(self.fns["adjoint_set_tapes"](self.h, max_tapes), "adjoint_set_tapes")

    def adjoint_reverse(self) -> TgAdjointStats:
        st = TgAdjointStats()
        self._check(self.fns["adjoint_reverse"](self.h, C.byref(st)), "adjoint_reverse")
        return st

    # -------------------------------------------------------------- turbines
    def set_turbines(self, turbines, rho: float = 1.225):
        """Define the actuator-disk farm (a sequence of TgTurbine; empty removes it)."""
        n = len(turbines)
        arr = (TgTurbine * max(n, 1))(*turbines)
        self._check(self.fns["set_turbines"](self.h, n, arr, rho), "set_turbines")
        self.n_turbines = n

    def set_turbine_ct(self, ct):
        ct = np.ascontiguousarray(ct, dtype=np.float64)
        self._check(self.fns["set_turbine_ct"](self.h, _ptr(ct)), "set_turbine_ct")

    def turbine_state(self, reset: bool = False) -> dict:
        """Last step's disk speed, thrust and power per turbine, and the summed farm power."""
        n = self.n_turbines
        u, th, pw = np.zeros(n), np.zeros(n), np.zeros(n)
        ps = C.c_double()
        self._check(self.fns["turbine_state"](self.h, _ptr(u), _ptr(th), _ptr(pw), C.byref(ps), 1 if reset else 0),
                    "turbine_state")
        return {"uref": u, "thrust": th, "power": pw, "power_sum": ps.value}

    def set_farm_objective(self, on: bool):
        self._check(self.fns["set_farm_objective"](self.h, 1 if on else 0), "set_farm_objective")

    def ct_gradient(self, reset: bool = False) -> np.ndarray:
        g = np.zeros(self.n_turbines)
        self._check(self.fns["ct_gradient"](self.h, _ptr(g), 1 if reset else 0), "ct_gradient")
        return g

    def set_graphs(self, on: bool):
        """Replay steps as CUDA graphs (default on) or launch them kernel by kernel."""
        self._check(self.fns["set_graphs"](self.h, 1 if on else 0), "set_graphs")

    def graph_info(self) -> tuple:
        """(steps replayed from the captured graph, capture failed)."""
        n, f = C.c_int64(), C.c_int32()
        self._check(self.fns["graph_info"](self.h, C.byref(n), C.byref(f)), "graph_info")
        return n.value, bool(f.value)

    def mesh_info(self) -> tuple:
        """(orthogonal, axis_aligned): the CUDA library's classification of the mesh."""
        a, b = C.c_int32(), C.c_int32()
        self._check(self.fns["mesh_info"](self.h, C.byref(a), C.byref(b)), "mesh_info")
        return bool(a.value), bool(b.value)

    def momentum_info(self) -> tuple:
        """(Newton steps or IMEX stages, Krylov operator products, last Krylov
        residual estimate) of the last implicit momentum solve."""
        a, b, r = C.c_int32(), C.c_int32(), C.c_double()
        self._check(self.fns["momentum_info"](self.h, C.byref(a), C.byref(b), C.byref(r)), "momentum_info")
        return a.value, b.value, r.value

    def step_host(self, ucont, ucat, p, nut=None, halo: int = 0) -> TgStats:
        st = TgStats()
        for a in (ucont, ucat, p) + ((nut,) if nut is not None else ()):
            assert a.flags.c_contiguous and a.dtype == np.float64
        self._check(self.fns["step_host"](self.h, _ptr(ucont), _ptr(ucat), _ptr(p),
                                          _ptr(nut) if nut is not None else None, halo, C.byref(st)),
                    "step_host")
        return st
