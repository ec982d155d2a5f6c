"""Crank-Nicolson momentum step (Jacobian-free Newton-Krylov) on the GPU
against the oracle's: both converge the implicit equation to 1e-13 relative
residual, so the steps agree to 1e-10 whatever the Krylov path."""
import numpy as np
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases
from tests.common import SMALL, build_case, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["tgv", "abl"])
def test_cn_steps_match_oracle(name):
    cfg, nodes, ucat, p, T = build_case(name, **SMALL[name])
    cfg.ddt_scheme = api.DDT_CN
    cfg.poisson_rtol = 1e-13
    cfg.snes_atol, cfg.snes_rtol, cfg.snes_maxit = 0.0, 1e-13, 30
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.step(3)
        out.append(s)
    g, o = out
    for f in ("UCAT", "UCONT", "P"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    assert g.graph_info()[0] == 0          # the Newton loop runs on the host
    g.close(); o.close()


def test_cn_reports_iteration_cap():
    cfg, nodes, ucat, p, T = build_case("tgv", **SMALL["tgv"])
    cfg.ddt_scheme = api.DDT_CN
    cfg.snes_atol, cfg.snes_rtol, cfg.snes_maxit = 0.0, 1e-30, 1
    s = tosca_b200.gpu_solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    with pytest.raises(api.TgError) as e:
        s.step(1)
    assert e.value.status == api.TG_ERR_NOT_CONVERGED
    s.close()


def test_cn_mixed_close_to_fp64():
    # the Newton residual is evaluated in FP64 in the mixed mode too (the
    # differenced Jacobian needs it); the rest of the step runs mixed
    cfg, nodes, ucat, p, T = build_case("abl", **SMALL["abl"])
    cfg.ddt_scheme = api.DDT_CN
    cfg.snes_atol, cfg.snes_rtol, cfg.snes_maxit = 0.0, 1e-12, 30
    res = []
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        cfg.precision = prec
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p, T)
        st = s.step(3)
        res.append((s.get("UCAT"), st.max_divergence, s.momentum_info()))
        s.close()
    assert rel_l2(res[1][0], res[0][0]) < 1e-6
    assert res[1][1] < 1e-8
    assert res[1][2][0] <= res[0][2][0] + 1          # Newton steps as in FP64
