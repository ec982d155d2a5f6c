"""IMEX momentum schemes (ABCN, RK3WCN, RK3SOCN: GMRES on the implicit
viscous operator IMEXMatVec, ueqn_solvers.c:1508-1799) on the GPU against the
oracle's. Both converge the Krylov solves to 1e-13 of |b|, so the steps
agree to 1e-10 whatever the Krylov path."""
import numpy as np
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases
from tests.common import SMALL, build_case, rel_l2

pytestmark = pytest.mark.gpu

SCHEMES = [api.DDT_ABCN, api.DDT_RK3WCN, api.DDT_RK3SOCN]


def _pair(name, ddt, steps, restart=30, **over):
    cfg, nodes, ucat, p, T = build_case(name, **SMALL[name])
    cfg.ddt_scheme = ddt
    cfg.poisson_rtol = 1e-13
    cfg.snes_atol, cfg.snes_rtol, cfg.gmres_restart = 0.0, 1e-13, restart
    for k, v in over.items():
        setattr(cfg, k, v)
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.step(steps)
        out.append(s)
    return out


@pytest.mark.parametrize("ddt", SCHEMES)
@pytest.mark.parametrize("name", ["tgv", "abl", "hill"])
def test_imex_steps_match_oracle(name, ddt):
    g, o = _pair(name, ddt, 3)
    for f in ("UCAT", "UCONT"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    # the projection corrects the small divergence of the predicted field, so
    # the 1e-13 Krylov stopping differences of the momentum solve reach phi
    # amplified; on the non-symmetric hill operator they leave ~3e-10 in P
    assert rel_l2(g.get("P"), o.get("P")) < (1e-9 if name == "hill" else 1e-10)
    gi, oi = g.momentum_info(), o.momentum_info()
    assert gi[0] == oi[0] == (1 if ddt == api.DDT_ABCN else 3)
    assert abs(gi[1] - oi[1]) <= gi[0], (gi, oi)
    assert g.graph_info()[0] == 0          # the Krylov loop runs on the host
    g.close(); o.close()


@pytest.mark.parametrize("ddt", SCHEMES)
def test_imex_restarted_gmres_matches_oracle(ddt):
    g, o = _pair("tgv", ddt, 2, restart=2, nu=0.2, dt=0.05)
    assert g.momentum_info()[1] > 2 * g.momentum_info()[0]   # restarts happened
    for f in ("UCAT", "P"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    g.close(); o.close()


def test_imex_mixed_precision_close_to_fp64():
    cfg, nodes, ucat, p, T = build_case("abl", **SMALL["abl"])
    cfg.ddt_scheme = api.DDT_RK3WCN
    cfg.snes_atol, cfg.snes_rtol = 0.0, 1e-12
    res = []
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        cfg.precision = prec
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p, T)
        st = s.step(3)
        res.append((s.get("UCAT"), st.max_divergence))
        s.close()
    assert rel_l2(res[1][0], res[0][0]) < 1e-6
    assert res[1][1] < 1e-8
