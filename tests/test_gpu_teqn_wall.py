"""The jLeft thetaWallFunction on the GPU against the oracle (which the
reference-pin tests hold to TOSCA's own UpdateWallModelsT and wall
functions): Schumann-Grotzbach (-3) with a cooling or heating surface,
plane-averaged or per cell, and the fixed heat flux (-2), on the stratified
ABL and the stratified hill; the wall heat flux enters the temperature step
and, through its plane mean, the friction velocity of the next step."""
import numpy as np
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases
from tests.common import rel_l2

pytestmark = pytest.mark.gpu


def _case(case, kind, heating_rate=-0.01, localized=False, qwall=0.0, **kw):
    if case == "sabl":
        cfg, nodes, ucat, p, T = cases.stratified_abl_case(16, 12, 12, heating_rate=heating_rate, localized=localized,
                                                           t_amp=0.5, **kw)
    else:
        cfg, nodes, ucat, p, T = cases.hill_case(24, 12, 12, teqn=True, t_amp=0.5, **kw)
        cases.thermal_wall(cfg, api.TWALL_SHUMANN, heating_rate=heating_rate, localized=localized)
    cfg.t_wall_type, cfg.t_wall_qwall = kind, qwall
    cfg.poisson_rtol = 1e-13
    return cfg, nodes, ucat, p, T


def _pair(cfg, nodes, ucat, p, T, steps, surf=None):
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        if surf is not None:
            s.set("SURF_THETA", surf)
        s.step(steps)
        out.append(s)
    return out


def _check(g, o, p_tol=1e-9):
    for f in ("TMPRT", "UCAT", "UCONT"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    assert rel_l2(g.get("P"), o.get("P")) < p_tol
    qg, qo = g.get("QWALL"), o.get("QWALL")
    assert np.abs(qo).max() > 0
    assert np.abs(qg - qo).max() <= 1e-8 * np.abs(qo).max()
    assert np.abs(g.get("SURF_THETA") - o.get("SURF_THETA")).max() <= 1e-12 * 300.0
    assert rel_l2(g.get("TAUWALL"), o.get("TAUWALL"), lambda a: a) < 1e-10


@pytest.mark.parametrize("case,kind,localized,heating_rate,qwall", [
    ("sabl", api.TWALL_SHUMANN, False, -0.01, 0.0),
    ("sabl", api.TWALL_SHUMANN, True, 0.02, 0.0),
    ("sabl", api.TWALL_FIXED_FLUX, False, 0.0, 0.05),
    ("hill", api.TWALL_SHUMANN, False, -0.01, 0.0),
    ("hill", api.TWALL_SHUMANN, True, -0.01, 0.0),
])
def test_thermal_wall_steps_match_oracle(case, kind, localized, heating_rate, qwall):
    g, o = _pair(*_case(case, kind, heating_rate, localized, qwall), steps=5)
    _check(g, o)
    g.close(); o.close()


def test_calm_stable_surface_bisects():
    """Weak wind over a surface 4 K colder than the air: the Monin-Obukhov
    iteration has no root (u* < 1e-2) and both sides take the bisection
    branch, per cell."""
    cfg, nodes, ucat, p, T = _case("sabl", api.TWALL_SHUMANN, heating_rate=0.0, localized=True, ustar=0.02)
    surf = np.full((cfg.mz, cfg.mx), 296.0)
    g, o = _pair(cfg, nodes, ucat, p, T, steps=3, surf=surf)
    _check(g, o)
    g.close(); o.close()


@pytest.mark.parametrize("scheme", [api.TDDT_ABBE, api.TDDT_BE])
def test_thermal_wall_with_implicit_temperature(scheme):
    """The wall flux is part of FormT's diffusive budget, so it enters the
    ABBE operator and the BE residual as in the reference."""
    cfg, nodes, ucat, p, T = _case("sabl", api.TWALL_SHUMANN, heating_rate=-0.01)
    cfg.t_ddt_scheme = scheme
    cfg.t_atol, cfg.t_rtol = 0.0, (1e-13 if scheme == api.TDDT_ABBE else 1e-10)
    g, o = _pair(cfg, nodes, ucat, p, T, steps=4)
    _check(g, o)
    g.close(); o.close()


def test_thermal_wall_stage_matches_oracle():
    cfg, nodes, ucat, p, T = _case("hill", api.TWALL_SHUMANN, heating_rate=0.03, localized=True)
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.UpdateWallModelsT()
        s.UpdateWallModelsT()                  # surface seeded once, raised twice
        out.append((s, s.get("QWALL"), s.get("SURF_THETA")))
    (g, qg, sg), (o, qo, so) = out
    assert np.abs(qg - qo).max() <= 1e-8 * np.abs(qo).max() and np.abs(qo).max() > 0
    assert np.abs(sg - so).max() <= 1e-12 * 300.0
    g.close(); o.close()


def test_thermal_wall_replay_and_mixed():
    """Graph replay is bitwise the eager step (the surface temperature is seeded
    before the first captured step); the mixed-precision step stays close."""
    cfg, nodes, ucat, p, T = _case("sabl", api.TWALL_SHUMANN, heating_rate=-0.02)
    res = []
    for prec, graphs in ((api.PREC_FP64, False), (api.PREC_FP64, True), (api.PREC_MIXED, True)):
        cfg.precision = prec
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.set_graphs(graphs)
        s.step(6)
        res.append((s, s.get("TMPRT"), s.get("UCAT"), s.get("QWALL")))
    (e, te, ue, qe), (r, tr, ur, qr), (m, tm, um, qm) = res
    assert np.array_equal(te, tr) and np.array_equal(ue, ur) and np.array_equal(qe, qr)
    assert r.graph_info()[0] == 5
    assert rel_l2(tm, te) < 1e-6 and rel_l2(um, ue) < 1e-6
    for s, *_ in res:
        s.close()


def test_thermal_wall_configuration_checked():
    cfg, *_ = _case("sabl", api.TWALL_SHUMANN)
    for bad in (dict(les=0), dict(t_wall_type=-5), dict(t_wall_kappa=0.0), dict(wall_theta_ref=-1.0)):
        with pytest.raises(api.TgError):
            tosca_b200.gpu_solver(api.Config(**{**cfg.__dict__, **bad}))


def test_drop_in_step_with_temperature():
    """The drop-in step with the state in host arrays and the temperature
    handed over around it (tg_set_field / tg_get_field TG_F_TMPRT), as a host
    that keeps T in its own vector does, against three oracle steps."""
    cfg, nodes, ucat, p, T = _case("sabl", api.TWALL_SHUMANN, heating_rate=-0.01)
    g = tosca_b200.gpu_solver(cfg)
    o = oracle.solver(cfg)
    for s in (g, o):
        cases.setup(s, nodes, ucat, p, T)
    uc, ut, pp, tt = (np.ascontiguousarray(o.get(f)) for f in ("UCONT", "UCAT", "P", "TMPRT"))
    for _ in range(3):
        g.set("TMPRT", tt)
        g.step_host(uc, ut, pp)
        tt = g.get("TMPRT")
        o.step(1)
    assert rel_l2(tt, o.get("TMPRT")) < 1e-10
    assert rel_l2(ut, o.get("UCAT")) < 1e-10 and rel_l2(uc, o.get("UCONT")) < 1e-10
    assert rel_l2(pp, o.get("P")) < 1e-9
    g.close(); o.close()


SERIES = (np.array([0.0, 50.0, 100.0, 100.5, 101.0, 102.0]), np.array([302.0, 301.0, 300.5, 299.8, 299.0, 298.0]))


@pytest.mark.parametrize("case,localized", [("sabl", False), ("sabl", True), ("hill", False)])
def test_surface_temperature_series_matches_oracle(case, localized):
    """thetaWallFunction -4 (surface temperature interpolated in time from a
    series, ground ghost 2 T_s - T(j=1) after the first step) after 5 steps
    from t_start = 100 s, through and beyond the series' points."""
    cfg, nodes, ucat, p, T = _case(case, api.TWALL_SURFACE_SERIES, localized=localized)
    cfg.t_start = 100.0
    out = []
    for make in (tosca_b200.gpu_solver, oracle.solver):
        s = make(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.set_surface_temperature(*SERIES)
        s.step(5)
        out.append(s)
    g, o = out
    for f in ("TMPRT", "UCAT", "UCONT"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    assert rel_l2(g.get("P"), o.get("P")) < 1e-9
    assert np.abs(g.get("TMPRT") - o.get("TMPRT")).max() <= 1e-10 * 300.0     # ghosts included
    qg, qo = g.get("QWALL"), o.get("QWALL")
    assert np.abs(qg - qo).max() <= 1e-8 * np.abs(qo).max() and np.abs(qo).max() > 0
    g.close(); o.close()


def test_surface_temperature_series_replay_and_refusal():
    """The -4 step replays from its graph bitwise (the surface temperature is
    interpolated on the device from the step counter), a new series of another
    length rebuilds the graph, and a step without a series is refused."""
    cfg, nodes, ucat, p, T = _case("sabl", api.TWALL_SURFACE_SERIES)
    cfg.t_start = 100.0
    res = []
    for graphs in (False, True):
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p, T)
        if graphs:
            with pytest.raises(api.TgError):
                s.step(1)
        s.set_surface_temperature(*SERIES)
        s.set_graphs(graphs)
        s.step(3)
        s.set_surface_temperature(np.array([0.0, 200.0]), np.array([301.0, 297.0]))
        s.step(3)
        res.append((s, s.get("TMPRT"), s.get("QWALL")))
    (e, te, qe), (r, tr, qr) = res
    assert np.array_equal(te, tr) and np.array_equal(qe, qr)
    assert r.graph_info()[0] >= 3
    e.close(); r.close()
