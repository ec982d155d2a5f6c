"""Grids whose sizes do not halve evenly: the multigrid preconditioner
aggregates pairs of cells and keeps a single-cell aggregate at the end of an
odd direction, so every size coarsens (HYPRE's BoomerAMG, peqn.c:357-429,
takes any grid). The CUDA step against the oracle after a few steps at odd
sizes: the 75 x 75 x 25 shape of TOSCA's CNBL scaling decks scaled down by 4
(the 300 x 300 x 100 deck itself stopped at 75 x 75 x 25 = 140,625 coarsest
cells before), odd sizes in every direction on the ABL and on the
curvilinear hill (BiCGStab path), and a Taylor-Green box of 18^3 cells
(18 -> 9 -> 5 -> 3)."""
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases
from tests.common import rel_l2

pytestmark = pytest.mark.gpu


def _pair(name, steps, tol_u=1e-10, tol_p=1e-10, prec=api.PREC_FP64, **kw):
    if name == "abl":
        cfg, nodes, ucat, p = cases.abl_case(ddt=api.DDT_RK4, **kw)
        T = None
    elif name == "hill":
        cfg, nodes, ucat, p, T = cases.hill_case(ddt=api.DDT_RK4, **kw)
    else:
        cfg, nodes, ucat, p = cases.tgv_case(ddt=api.DDT_RK4, **kw)
        T = None
    cfg.poisson_rtol = 1e-13
    o = oracle.solver(cfg)
    cases.setup(o, nodes, ucat, p, T)
    cfg.precision = prec
    g = tosca_b200.gpu_solver(cfg)
    cases.setup(g, nodes, ucat, p, T)
    sg = g.step(steps)
    o.step(steps)
    u_g, u_o = g.get("UCAT"), o.get("UCAT")
    for c in range(3):
        assert rel_l2(u_g[..., c], u_o[..., c]) < tol_u, c
    assert rel_l2(g.get("P"), o.get("P")) < tol_p
    assert sg.max_divergence < (1e-8 if prec == api.PREC_MIXED else 1e-10)
    g.close(); o.close()


def test_cnbl_shape_75x75x25():
    _pair("abl", 3, nx=75, ny=75, nz=25, Lx=750.0, Ly=750.0, H=250.0)


def test_abl_odd_every_direction():
    _pair("abl", 5, nx=45, ny=27, nz=15, Lx=450.0, Ly=270.0, H=150.0)


def test_abl_odd_mixed_precision():
    _pair("abl", 5, tol_u=1e-6, tol_p=1e-6, prec=api.PREC_MIXED, nx=45, ny=27, nz=15, Lx=450.0, Ly=270.0, H=150.0)


def test_hill_odd_sizes():
    _pair("hill", 3, tol_p=1e-9, nx=27, ny=15, nz=13)


def test_tgv_18():
    _pair("tgv", 5, n=18)
