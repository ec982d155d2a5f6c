"""CPU checks of the Crank-Nicolson momentum step in the oracle: the
implicit solve converges, and on the Taylor-Green vortex the CN and RK4
solutions agree to the order of the time step squared."""
import numpy as np
import pytest

import oracle
from tosca_b200 import api, cases
from tests.common import rel_l2


def _run(ddt, dt, steps, n=8):
    cfg, nodes, ucat, p = cases.tgv_case(n, ddt=ddt, dt=dt)
    cfg.poisson_rtol = 1e-14
    cfg.snes_atol, cfg.snes_rtol, cfg.snes_maxit = 0.0, 1e-13, 30
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p)
    st = s.step(steps)
    out = {f: s.get(f) for f in ("UCAT", "P")}
    s.close()
    return out, st


def test_cn_converges_and_is_second_order():
    errs = []
    for dt, steps in ((0.02, 5), (0.01, 10)):
        cn, st = _run(api.DDT_CN, dt, steps)
        rk, _ = _run(api.DDT_RK4, dt, steps)
        assert st.max_divergence < 1e-12
        errs.append(rel_l2(cn["UCAT"], rk["UCAT"]))
    # the CN-RK4 difference is the CN error: O(dt^2)
    assert errs[0] < 1e-3 and 2.5 < errs[0] / errs[1] < 5.5, errs
