"""Sizes that do not fill the kernels' blocks (18 x 10 x 14 interior cells:
partial blocks of the 32 x 4 x 2 face-flux tile in i and j, of the line
smoother's chunks and of the reductions): FormU, ExplicitRhsU and three steps
against the oracle, on an axis-aligned ABL mesh and on the curvilinear hill."""
import numpy as np
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases
from tests.common import rel_l2

pytestmark = pytest.mark.gpu


def _full(a):
    return a


def _case(name):
    if name == "abl":
        cfg, nodes, ucat, p = cases.abl_case(nx=14, ny=18, nz=10, Lx=140.0, Ly=180.0, H=100.0, ddt=api.DDT_RK4)
        T = None
    else:
        cfg, nodes, ucat, p, T = cases.hill_case(nx=14, ny=18, nz=10, ddt=api.DDT_RK4)
    cfg.poisson_rtol = 1e-13
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        out.append(s)
    return out


@pytest.mark.parametrize("name", ["abl", "hill"])
def test_ragged_stages_and_steps(name):
    g, o = _case(name)
    assert g.mesh_info()[1] == (name == "abl")
    for s in (g, o):
        if s.cfg.les:
            s.UpdateNut(); s.UpdateWallModelsU()
        s.FormU(1.0, True)
    assert rel_l2(g.get("RHS"), o.get("RHS"), _full) < 1e-12
    for s in (g, o):
        s.GradP()
        if s.cfg.buoyancy:
            s.Buoyancy()
        s.ExplicitRhsU()
    assert rel_l2(g.get("RHS"), o.get("RHS"), _full) < 1e-12
    for s in (g, o):
        s.step(3)
    for f in ("UCAT", "UCONT"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    assert rel_l2(g.get("P"), o.get("P")) < 1e-9
    g.close(); o.close()
