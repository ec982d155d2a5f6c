"""CPU checks of the IMEX momentum schemes in the oracle (UeqnABCN,
UeqnRK3CN_W, UeqnRK3CN_SO with GMRES on IMEXMatVec, ueqn_solvers.c:1508-1799):
temporal behaviour against RK4 on the Taylor-Green vortex, restart
independence of the tightly converged GMRES, and the configuration checks."""
import numpy as np
import pytest

import oracle
from tosca_b200 import api, cases
from tests.common import rel_l2


def _run(ddt, dt, steps, n=8, nu=None, restart=30, rtol=1e-13):
    cfg, nodes, ucat, p = cases.tgv_case(n, ddt=ddt, dt=dt)
    if nu is not None:
        cfg.nu = nu
    cfg.poisson_rtol = 1e-14
    cfg.snes_atol, cfg.snes_rtol, cfg.gmres_restart = 0.0, rtol, restart
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p)
    st = s.step(steps)
    out = {f: s.get(f) for f in ("UCAT", "UCONT", "P")}
    info = s.momentum_info()
    s.close()
    return out, st, info


def _errors(ddt):
    errs = []
    for dt, steps in ((0.02, 5), (0.01, 10)):
        a, st, info = _run(ddt, dt, steps)
        assert st.max_divergence < 1e-12
        assert info[0] == (1 if ddt == api.DDT_ABCN else 3)   # stages of the last step
        r, _, _ = _run(api.DDT_RK4, dt, steps)
        errs.append(rel_l2(a["UCAT"], r["UCAT"]))
    return errs


def test_rk3wcn_is_second_order():
    e = _errors(api.DDT_RK3WCN)
    assert e[0] < 1e-8 and e[0] / e[1] > 3.0, e


def test_rk3socn_viscous_part_is_first_order():
    # the stage weights of the implicit viscous part (gamma = 1/2, 1/8, 1/3)
    # match the Shu-Osher weights to first order only: on the viscous decay
    # of the vortex the error halves with dt
    e = _errors(api.DDT_RK3SOCN)
    assert e[0] < 1e-6 and 1.8 < e[0] / e[1] < 2.2, e


def test_abcn_first_step_adds_rhs_twice():
    # ueqn_solvers.c:1697-1700 adds Rhs to the copy of Rhs on the first step,
    # an O(dt) error carried by every later step: the error halves with dt
    e = _errors(api.DDT_ABCN)
    assert 1e-4 < e[0] < 1e-2 and 1.8 < e[0] / e[1] < 2.2, e


@pytest.mark.parametrize("ddt", [api.DDT_ABCN, api.DDT_RK3WCN, api.DDT_RK3SOCN])
def test_gmres_restart_independent(ddt):
    # a viscous case that needs several Krylov iterations per stage
    a, _, ia = _run(ddt, 0.05, 2, nu=0.2, restart=30)
    b, _, ib = _run(ddt, 0.05, 2, nu=0.2, restart=2)
    assert ia[1] >= 3 * ia[0], ia
    assert ib[1] >= ia[1]
    for f in ("UCAT", "P"):
        assert rel_l2(b[f], a[f]) < 1e-11, f


def test_abs_tolerance_stops_early():
    a, _, ia = _run(api.DDT_RK3WCN, 0.05, 1, nu=0.05, rtol=1e-13)
    b, _, ib = _run(api.DDT_RK3WCN, 0.05, 1, nu=0.05, rtol=1e-4)
    assert ib[1] < ia[1]
    assert rel_l2(b["UCAT"], a["UCAT"]) < 1e-4


def test_config_checks():
    cfg, nodes, ucat, p = cases.tgv_case(8, ddt=api.DDT_RK3SOCN, dt=0.01)
    cfg.gmres_restart = 61
    with pytest.raises(api.TgError):
        oracle.solver(cfg)
    cfg.gmres_restart = 30
    cfg.ddt_scheme = 6
    with pytest.raises(api.TgError):
        oracle.solver(cfg)
