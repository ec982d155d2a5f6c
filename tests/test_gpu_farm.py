"""Actuator-disk farm on the GPU against the oracle: step fields, turbine
forces and state, the adjoint with respect to C_T' (field by field and
against central differences of the CUDA step), and step replay."""
import ctypes

import numpy as np
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases
from tests.common import rel_l2
from tests.test_oracle_farm import small_farm

pytestmark = pytest.mark.gpu
EPS = 1e-6


def _pair(wall=api.BC_NOSLIP, ddt=api.DDT_RK4, les=1):
    cfg, nodes, ucat, p, tb = small_farm(ddt=ddt, wall=wall)
    cfg.les = les
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p)
        s.set_turbines(tb, 1.225)
        out.append(s)
    return out, tb


@pytest.mark.parametrize("wall,ddt", [(api.BC_NOSLIP, api.DDT_RK4), (api.BC_WALL_SHUMANN, api.DDT_RK4),
                                      (api.BC_NOSLIP, api.DDT_FE)])
def test_farm_steps_match_oracle(wall, ddt):
    (g, o), tb = _pair(wall, ddt)
    for s in (g, o):
        s.step(5)
    for f in ("UCAT", "UCONT", "P"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    for f in ("FARM_FORCE", "FARM_CONT"):
        a, b = g.get(f), o.get(f)
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), f
    sg, so = g.turbine_state(), o.turbine_state()
    for k in ("uref", "thrust", "power"):
        assert np.allclose(sg[k], so[k], rtol=1e-11, atol=0), k
    assert abs(sg["power_sum"] - so["power_sum"]) <= 1e-11 * abs(so["power_sum"])
    g.close(); o.close()


def test_farm_adjoint_step_matches_oracle():
    (g, o), tb = _pair()
    for s in (g, o):
        s.step(1)
        s.set_farm_objective(True)
    rng = np.random.default_rng(9)
    shape = g.get("UCAT").shape
    interior = np.zeros(shape[:3], bool)
    interior[1:-1, 1:-1, 1:-1] = True
    seeds = {"UCONT_ADJ": rng.standard_normal(shape), "UCAT_ADJ": rng.standard_normal(shape) * interior[..., None],
             "P_ADJ": rng.standard_normal(shape[:3]), "SOURCE_ADJ": np.zeros(shape)}
    L = oracle.lib()
    L.tor_adjoint_step.argtypes = [ctypes.c_void_p]
    for s in (g, o):
        for k, v in seeds.items():
            s.set(k, v)
    g.adjoint_step()
    assert L.tor_adjoint_step(o.h) == 0
    for k in ("UCONT_ADJ", "UCAT_ADJ", "P_ADJ"):
        assert rel_l2(g.get(k), o.get(k), lambda a: a) < 1e-8, k
    gg, go = g.ct_gradient(), o.ct_gradient()
    assert np.allclose(gg, go, rtol=1e-8, atol=0), (gg, go)
    g.close(); o.close()


@pytest.mark.parametrize("nsnap", [4, 2])
def test_farm_power_gradient_matches_central_differences(nsnap):
    cfg, nodes, ucat, p, tb = small_farm()
    nsteps = 4
    ct0 = np.array([t.ct for t in tb])

    def start(ct=None):
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p)
        s.set_turbines(tb, 1.225)
        s.step(1)
        if ct is not None:
            s.set_turbine_ct(ct)
        s.turbine_state(reset=True)
        return s

    def J(ct):
        s = start(ct)
        s.step(nsteps)
        v = s.turbine_state()["power_sum"]
        s.close()
        return v

    s = start()
    s.set_farm_objective(True)
    s.adjoint_forward(nsteps, nsnap)
    for k in ("UCONT_ADJ", "UCAT_ADJ", "SOURCE_ADJ"):
        s.set(k, np.zeros(ucat.shape))
    s.set("P_ADJ", np.zeros(p.shape))
    s.ct_gradient(reset=True)
    st = s.adjoint_reverse()
    grad = s.ct_gradient()
    assert st.steps == nsteps
    s.close()
    for t in range(len(tb)):
        e = np.zeros(len(tb))
        e[t] = EPS
        fd = (J(ct0 + e) - J(ct0 - e)) / (2 * EPS)
        assert abs(grad[t] - fd) <= 1e-5 * abs(fd), (t, grad[t], fd)


def test_farm_replay_bitwise_and_mixed_precision():
    cfg, nodes, ucat, p, tb = small_farm(wall=api.BC_WALL_SHUMANN)
    runs = []
    for prec, graphs in ((api.PREC_FP64, False), (api.PREC_FP64, True), (api.PREC_MIXED, True)):
        cfg.precision = prec
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p)
        s.set_graphs(graphs)
        s.set_turbines(tb, 1.225)
        s.step(6)
        runs.append((s, {f: s.get(f) for f in ("UCAT", "UCONT", "P")}, s.turbine_state()))
    (e, fe, te), (r, fr, tr), (m, fm, tm) = runs
    for f in fe:
        assert np.array_equal(fe[f], fr[f]), f
        assert rel_l2(fm[f], fe[f]) < 1e-6, f
    assert te["power_sum"] == tr["power_sum"]
    assert r.graph_info()[0] == 5
    for s, _, _ in runs:
        s.close()
