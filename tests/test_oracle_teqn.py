"""CPU checks of the temperature-transport restatement in the oracle:
uniform temperature is preserved by the WENO3 convection and the diffusion
(up to the projected divergence), and the temperature changes where the
flow advects a perturbation."""
import numpy as np
import pytest

import oracle
from tosca_b200 import api, cases
from tests.common import rel_l2

SMALL = dict(nx=24, ny=12, nz=12)


def test_uniform_temperature_is_preserved():
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, **SMALL)
    cfg.poisson_rtol = 1e-14
    cfg.t_bc_value = (0.0,) * 6            # zero gradient at the top too
    T[...] = 300.0
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    s.step(3)
    t = s.get("TMPRT")[1:-1, 1:-1, 1:-1]
    assert np.abs(t - 300.0).max() <= 1e-10 * 300.0
    s.close()


def test_perturbation_is_transported():
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, t_amp=0.5, **SMALL)
    cfg.poisson_rtol = 1e-14
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    t0 = s.get("TMPRT")
    s.step(3)
    t1 = s.get("TMPRT")
    d = np.abs(t1 - t0)[1:-1, 1:-1, 1:-1]
    assert d.max() > 1e-3 and np.isfinite(t1).all()
    # fixed gradient at the top ghost (UpdateTemperatureBCs)
    aj = s.get("AJ")
    eta = s.get("ETA")
    top = cfg.my - 2
    area = np.linalg.norm(eta[1:-1, top, 1:-1], axis=-1)
    dd = (1.0 / aj[1:-1, top, 1:-1]) / area
    assert np.allclose(t1[1:-1, top + 1, 1:-1], dd * cfg.t_bc_value[3] + t1[1:-1, top, 1:-1], rtol=0, atol=1e-12)
    # zero gradient at the terrain
    assert np.array_equal(t1[1:-1, 0, 1:-1], t1[1:-1, 1, 1:-1])
    s.close()


def _abbe_run(dt, steps, scheme, rtol=1e-13, restart=30, les=1):
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, t_amp=0.5, nx=16, ny=8, nz=8, dt=dt)
    cfg.les = les
    cfg.poisson_rtol = 1e-13
    cfg.t_ddt_scheme = scheme
    cfg.t_atol, cfg.t_rtol, cfg.t_gmres_restart = 0.0, rtol, restart
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    s.step(steps)
    t = s.get("TMPRT")
    s.close()
    return t


def test_abbe_temperature_converges_to_rk4():
    # ABBE (AB2 convection, backward-Euler diffusion, forward Euler on the
    # first step) against the explicit RK4 temperature: first order in dt
    errs = []
    for dt, steps in ((0.5, 4), (0.25, 8)):
        a = _abbe_run(dt, steps, api.TDDT_ABBE)
        r = _abbe_run(dt, steps, api.TDDT_RK4)
        assert np.isfinite(a).all()
        errs.append(rel_l2(a, r))
    assert errs[0] < 1e-4 and 1.6 < errs[0] / errs[1] < 4.5, errs


def test_abbe_gmres_restart_independent():
    a = _abbe_run(0.5, 2, api.TDDT_ABBE, restart=30, les=0)
    b = _abbe_run(0.5, 2, api.TDDT_ABBE, restart=1, les=0)
    assert rel_l2(b, a) < 1e-11


@pytest.mark.parametrize("scheme,lo,hi", [(api.TDDT_BE, 1.8, 2.2), (api.TDDT_BDF2, 3.0, 5.0)])
def test_implicit_temperature_order(scheme, lo, hi):
    # TeqnSNES: backward Euler is first order, BDF2 (BE on the first step)
    # second order against the explicit RK4 temperature
    errs = []
    for dt, steps in ((0.5, 4), (0.25, 8)):
        a = _abbe_run(dt, steps, scheme, rtol=1e-10)
        r = _abbe_run(dt, steps, api.TDDT_RK4)
        errs.append(rel_l2(a, r))
    assert errs[0] < 1e-5 and lo < errs[0] / errs[1] < hi, errs


def test_temperature_scheme_checked():
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, t_amp=0.5, nx=16, ny=8, nz=8)
    cfg.t_ddt_scheme = 4
    with pytest.raises(api.TgError):
        oracle.solver(cfg)


def test_p_tilde_buoyancy():
    # ghGradRhoK vanishes for T = tRef, is finite and non-zero for the
    # stratified hill, and needs the buoyancy switch
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, t_amp=0.5, nx=16, ny=8, nz=8)
    cfg.p_tilde = 1
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, np.full_like(T, cfg.t_ref))
    s.Buoyancy()
    # the top patch has a fixed lapse-rate gradient: its ghosts differ from tRef
    assert np.abs(s.get("BTHETA")[:, 1:-3]).max() == 0.0
    s.set("TMPRT", T)
    s.Buoyancy()
    b = s.get("BTHETA")
    assert np.isfinite(b).all() and np.abs(b).max() > 0
    s.step(2)
    s.close()
    cfg.buoyancy = 0
    with pytest.raises(api.TgError):
        oracle.solver(cfg)


# ------------------------------------------------------ thermal wall function
def _sabl(**kw):
    cfg, nodes, ucat, p, T = cases.stratified_abl_case(16, 12, 12, t_amp=0.5, **kw)
    cfg.poisson_rtol = 1e-14
    return cfg, nodes, ucat, p, T


def test_fixed_heat_flux_enters_the_heat_budget():
    """qWall = q (-2) at the ground, zero-gradient top and periodic sides: the
    volume integral of T grows by q * (ground area) * dt per step; the RK4
    convection and the interior diffusion telescope (wall-normal fluxes
    vanish). The air above the 100 m perturbed layer is uniform (no lapse
    rate), so that the top ghosts, which the RK4 stages do not update, carry
    no flux within the three steps."""
    cfg, nodes, ucat, p, T = _sabl(lapse=0.0)
    cases.thermal_wall(cfg, api.TWALL_FIXED_FLUX, qwall=0.08)
    cfg.t_bc_value = (0.0,) * 6
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    vol = 1.0 / s.get("AJ")[1:-1, 1:-1, 1:-1]
    area = s.get("JETA")[1:-1, 0, 1:-1, 2].sum()
    heat = lambda: float((s.get("TMPRT")[1:-1, 1:-1, 1:-1] * vol).sum())
    h0 = heat()
    s.step(3)
    expect = 3 * cfg.dt * 0.08 * area
    assert abs(heat() - h0 - expect) <= 1e-9 * expect
    assert np.all(s.get("QWALL")[1:-1, 1:-1] == 0.08)
    s.close()


@pytest.mark.parametrize("heating_rate,sign", [(-0.02, -1.0), (0.02, 1.0)])
def test_surface_temperature_and_heat_flux_sign(heating_rate, sign):
    """-3: the surface starts at the wall value and moves by heatingRate * dt
    per step; a cooling surface draws heat out of the air (qWall < 0, stable),
    a heating one puts heat in (qWall > 0, unstable); averaged: one value."""
    cfg, nodes, ucat, p, T = _sabl(heating_rate=heating_rate)
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    t_wall = 0.5 * (T[1:-1, 1, 1:-1] + T[1:-1, 0, 1:-1])
    s.step(4)
    st = s.get("SURF_THETA")[1:-1, 1:-1]
    assert np.abs(st - (t_wall + 4 * heating_rate * cfg.dt)).max() <= 1e-12 * 300.0
    q = s.get("QWALL")[1:-1, 1:-1]
    assert np.all(q == q[0, 0]) and sign * q[0, 0] > 0
    s.close()


def test_localized_heat_flux_varies_per_cell():
    cfg, nodes, ucat, p, T = _sabl(heating_rate=0.02, localized=True)
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    s.step(2)
    q = s.get("QWALL")[1:-1, 1:-1]
    assert q.std() > 0 and np.all(q > 0)
    s.close()


def test_stratification_changes_the_friction_velocity():
    """The velocity wall function reads the plane mean of the last qWall: the
    wall stress of a stable step differs from the neutral one, and is
    neutral on the first step (qWall still zero)."""
    taus = []
    for kind in (None, api.TWALL_SHUMANN):
        cfg, nodes, ucat, p, T = _sabl(heating_rate=-0.05)
        if kind is None:
            bc = list(cfg.t_bc); bc[2] = api.TBC_ZERO_GRADIENT; cfg.t_bc = tuple(bc)
        s = oracle.solver(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.set("SURF_THETA", np.full((cfg.mz, cfg.mx), 299.0))    # 1 K below the air: unstable
        out = []
        for _ in range(2):
            s.step(1)
            out.append(s.get("TAUWALL"))
        taus.append(out)
        s.close()
    assert np.array_equal(taus[0][0], taus[1][0])
    assert rel_l2(taus[1][1], taus[0][1], lambda a: a) > 1e-3


def test_thermal_wall_configuration_checked():
    cfg, nodes, ucat, p, T = _sabl()
    for bad in (dict(les=0), dict(t_wall_type=-1), dict(t_wall_theta_ref=0.0), dict(wall_theta_ref=0.0),
                dict(t_wall_localized=2), dict(t_bc=(api.TBC_PERIODIC, api.TBC_PERIODIC, api.TBC_ZERO_GRADIENT,
                                                     api.TBC_WALL_FUNCTION, api.TBC_PERIODIC, api.TBC_PERIODIC))):
        c = api.Config(**{**cfg.__dict__, **bad})
        with pytest.raises(api.TgError):
            oracle.solver(c)


def test_surface_temperature_series_ghost_rule():
    """-4: the ground ghost is zero-gradient after the first step and 2 T_s -
    T(j=1) after the later ones (boundary.c:2392-2408); qWall follows the
    series' surface temperature; without a series the step is refused."""
    cfg, nodes, ucat, p, T = _sabl()
    cfg.t_wall_type, cfg.t_start = api.TWALL_SURFACE_SERIES, 0.0
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    with pytest.raises(api.TgError):
        s.step(1)
    ts = 299.5
    s.set_surface_temperature([0.0, 10.0], [ts, ts])
    s.step(1)
    t = s.get("TMPRT")
    assert np.array_equal(t[1:-1, 0, 1:-1], t[1:-1, 1, 1:-1])
    s.step(1)
    t = s.get("TMPRT")
    assert np.abs(t[1:-1, 0, 1:-1] + t[1:-1, 1, 1:-1] - 2 * ts).max() <= 1e-12 * ts
    q = s.get("QWALL")[1:-1, 1:-1]
    assert np.all(q == q[0, 0]) and q[0, 0] < 0        # air at ~300 K over a 299.5 K surface: stable
    s.close()
