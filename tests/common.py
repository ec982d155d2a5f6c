"""Shared helpers of the parity tests: build both the CUDA solver and the CPU
restatement (oracle) on the same case and compare fields."""
from __future__ import annotations

import numpy as np

import oracle
import tosca_b200
from tosca_b200 import cases


def interior(a: np.ndarray) -> np.ndarray:
    return a[1:-1, 1:-1, 1:-1]


def rel_l2(a: np.ndarray, b: np.ndarray, region=interior) -> float:
    a, b = region(a), region(b)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)


def div_roundoff_floor(ucont: np.ndarray, aj: np.ndarray, ulps: float = 256.0) -> float:
    """Round-off level of ContinuityErrorsOptimized (peqn.c:4148-4157) on this
    state: `ulps` units of FP64 rounding of the largest per-cell sum of face
    flux magnitudes times aj. Below about this level the divergence after the
    projection no longer follows the solver tolerance (measured on the ABL at
    64 x 64 x 32: 1e-15 to 5.5e-14 for relative tolerances 1e-13 to 1e-15, on
    the GPU and on the oracle alike, against 256 ulps = 9.9e-14)."""
    V = np.abs(ucont)
    s = (V[1:-1, 1:-1, 1:-1, 0] + V[1:-1, 1:-1, :-2, 0] + V[1:-1, 1:-1, 1:-1, 1] + V[1:-1, :-2, 1:-1, 1]
         + V[1:-1, 1:-1, 1:-1, 2] + V[:-2, 1:-1, 1:-1, 2]) * np.abs(aj[1:-1, 1:-1, 1:-1])
    return float(ulps * np.finfo(np.float64).eps * s.max())


def max_abs(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))))


def build_case(name: str, **kw):
    if name == "tgv":
        cfg, nodes, ucat, p = cases.tgv_case(**kw)
        return cfg, nodes, ucat, p, None
    if name == "abl":
        cfg, nodes, ucat, p = cases.abl_case(**kw)
        return cfg, nodes, ucat, p, None
    if name == "hill":
        return cases.hill_case(**kw)
    if name == "channel":
        cfg, nodes, ucat, p = cases.channel_case(**kw)
        return cfg, nodes, ucat, p, None
    if name == "ohill":
        # the hill with the inflow/outflow pair of TOSCA's CosineHillCurvTest deck
        cfg, nodes, ucat, p, T = cases.hill_case(**kw)
        cases.open_x(cfg, 8.0)
        return cfg, nodes, ucat, p, T
    raise ValueError(name)


def pair(name: str, cfg_over=None, **kw):
    """(gpu_solver, oracle_solver) set up identically."""
    cfg, nodes, ucat, p, T = build_case(name, **kw)
    if cfg_over:
        for k, v in cfg_over.items():
            setattr(cfg, k, v)
    g = tosca_b200.gpu_solver(cfg)
    o = oracle.solver(cfg)
    for s in (g, o):
        cases.setup(s, nodes, ucat, p, T)
    return g, o


SMALL = {
    "tgv": dict(n=16),
    "abl": dict(nx=16, ny=16, nz=12, Lx=160.0, Ly=160.0, H=100.0),
    "hill": dict(nx=24, ny=12, nz=12),
    # inflow at x = 0, outflow at x = Lx, noSlip ground (cases.channel_case)
    "channel": dict(nx=20, ny=12, nz=10, Lx=200.0, Ly=120.0, H=100.0),
    "ohill": dict(nx=24, ny=12, nz=12),
}
