"""Temperature transport on the GPU against the oracle: the stratified hill
case with the temperature advanced every step (RK4, WENO3, Smagorinsky with
the stability-corrected Pr_t) and feeding the buoyancy of the next step."""
import numpy as np
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases
from tests.common import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("les", [1, 0])
def test_teqn_steps_match_oracle(les):
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, t_amp=0.5, nx=24, ny=12, nz=12)
    cfg.poisson_rtol = 1e-13
    cfg.les = les
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.step(5)
        out.append(s)
    g, o = out
    for f in ("TMPRT", "UCAT", "UCONT", "P"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    # ghost values from UpdateTemperatureBCs
    a, b = g.get("TMPRT"), o.get("TMPRT")
    assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()
    g.close(); o.close()


def test_teqn_replay_and_mixed():
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, t_amp=0.5, nx=24, ny=12, nz=12)
    res = []
    for prec, graphs in ((api.PREC_FP64, False), (api.PREC_FP64, True), (api.PREC_MIXED, True)):
        cfg.precision = prec
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.set_graphs(graphs)
        s.step(6)
        res.append((s, s.get("TMPRT"), s.get("UCAT")))
    (e, te, ue), (r, tr, ur), (m, tm, um) = res
    assert np.array_equal(te, tr) and np.array_equal(ue, ur)
    assert r.graph_info()[0] == 5
    assert rel_l2(tm, te) < 1e-6 and rel_l2(um, ue) < 1e-6
    for s, _, _ in res:
        s.close()


@pytest.mark.parametrize("scheme,rtol", [(api.TDDT_ABBE, 1e-13), (api.TDDT_BE, 1e-10), (api.TDDT_BDF2, 1e-10)])
@pytest.mark.parametrize("les", [1, 0])
def test_implicit_temperature_matches_oracle(les, scheme, rtol):
    # ABBE: AB2 convection and backward-Euler diffusion by GMRES (TeqnABBE),
    # GMRES converged to 1e-13 of |b|; BE / BDF2: Newton-Krylov (TeqnSNES) to
    # 1e-10 of |F_0| (the differenced Jacobian limits the Newton iteration)
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, t_amp=0.5, nx=24, ny=12, nz=12)
    cfg.poisson_rtol = 1e-13
    cfg.les = les
    cfg.t_ddt_scheme = scheme
    cfg.t_atol, cfg.t_rtol = 0.0, rtol
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.step(5)
        out.append(s)
    g, o = out
    for f in ("TMPRT", "UCAT", "UCONT"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    assert rel_l2(g.get("P"), o.get("P")) < 1e-9
    assert g.graph_info()[0] == 0          # the Krylov loops run on the host
    g.close(); o.close()


@pytest.mark.parametrize("ddt,tddt", [(api.DDT_CN, api.TDDT_BDF2), (api.DDT_ABCN, api.TDDT_ABBE)])
def test_temperature_with_implicit_momentum(ddt, tddt):
    # the temperature and momentum schemes are independent (-dTdtScheme,
    # -dUdtScheme): implicit pairs against the oracle after 3 steps
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, t_amp=0.5, nx=24, ny=12, nz=12)
    cfg.poisson_rtol = 1e-13
    cfg.ddt_scheme, cfg.t_ddt_scheme = ddt, tddt
    cfg.snes_atol, cfg.snes_rtol, cfg.snes_maxit = 0.0, 1e-13, 30
    cfg.t_atol, cfg.t_rtol = 0.0, 1e-10 if tddt == api.TDDT_BDF2 else 1e-13
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.step(3)
        out.append(s)
    g, o = out
    for f in ("TMPRT", "UCAT", "UCONT"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    assert rel_l2(g.get("P"), o.get("P")) < 1e-9
    g.close(); o.close()


@pytest.mark.parametrize("teqn", [False, True])
def test_p_tilde_buoyancy_matches_oracle(teqn):
    # -pTildeBuoyancy 1: ghGradRhoK (teqn.c:278-652) in place of Buoyancy, on
    # the stratified curvilinear hill, frozen or transported temperature
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=teqn, t_amp=0.5, nx=24, ny=12, nz=12)
    cfg.poisson_rtol = 1e-13
    cfg.p_tilde = 1
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.Buoyancy()
        out.append((s, s.get("BTHETA")))
    (g, bg), (o, bo) = out
    assert rel_l2(bg, bo) < 1e-12 and np.abs(bo).max() > 0
    for s in (g, o):
        s.step(5)
    for f in ("UCAT", "UCONT") + (("TMPRT",) if teqn else ()):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    assert rel_l2(g.get("P"), o.get("P")) < 1e-9
    g.close(); o.close()
