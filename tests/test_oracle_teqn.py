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
