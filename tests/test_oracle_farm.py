"""CPU checks of the actuator-disk farm restatement in the oracle (the checker
of the CUDA farm): known answers for a uniform inflow (disk speed, thrust,
power, integral of the projected force) and central finite differences of
the summed farm power with respect to the turbines' C_T'."""
import ctypes

import numpy as np
import pytest

import oracle
from tosca_b200 import api, cases

EPS = 1e-6


def _lib():
    L = oracle.lib()
    L.tor_adjoint_step.argtypes = [ctypes.c_void_p]
    L.tor_adjoint_step.restype = ctypes.c_int
    return L


def small_farm(ddt=api.DDT_RK4, wall=api.BC_NOSLIP, ct=1.33):
    cfg, nodes, ucat, p, tb = cases.farm_case(nx=16, ny=12, nz=12, Lx=160.0, Ly=120.0, H=120.0, dz1=6.0,
                                              rows=2, cols=1, D=40.0, hub=55.0, sx=1.5, epsilon=15.0, ct=ct,
                                              r_hub=1.0, n_radial=4, n_azimuth=8, ddt=ddt, wall=wall)
    cfg.poisson_rtol = 1e-14
    return cfg, nodes, ucat, p, tb


def test_uniform_inflow_known_answers():
    cfg, nodes, ucat, p, tb = small_farm()
    tb = tb[:1]
    U0, rho = 7.5, 1.2
    ucat[...] = 0.0
    ucat[1:-1, 1:-1, 1:-1, 0] = U0
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p)
    s.set_turbines(tb, rho)
    s.step(1)
    st = s.turbine_state()
    t = tb[0]
    area = np.pi * t.r_tip ** 2
    thrust = rho * 0.5 * U0 * U0 * t.ct * area
    # (the rotor axis is normalised as nUnit does, |v| + 1e-12: relative 4e-12 in the thrust)
    assert abs(st["uref"][0] - U0) <= 1e-12 * U0
    assert abs(st["thrust"][0] - thrust) <= 1e-11 * thrust
    assert abs(st["power"][0] - thrust * U0) <= 1e-11 * thrust * U0
    assert abs(st["power_sum"] - thrust * U0) <= 1e-11 * thrust * U0
    # the projected force integrates to the thrust per unit density along the
    # axis (Gaussian truncated at 2.63 epsilon and sampled at the cell centres)
    f = s.get("FARM_FORCE")
    vol = 1.0 / s.get("AJ")
    total = (f[..., 0] * vol)[1:-1, 1:-1, 1:-1].sum()
    assert total < 0 and abs(-total - thrust / rho) <= 0.03 * thrust / rho
    assert np.abs(f[..., 1:]).max() <= 1e-12 * np.abs(f[..., 0]).max()
    s.close()


def test_disk_points_cover_the_rotor_area():
    # the area weights sum to pi r_tip^2 whatever the sampling resolution
    cfg, nodes, ucat, p, tb = small_farm()
    ucat[...] = 0.0
    ucat[1:-1, 1:-1, 1:-1, 0] = 3.0
    for nr, na in ((2, 1), (5, 7)):
        for t in tb:
            t.n_radial, t.n_azimuth = nr, na
        s = oracle.solver(cfg)
        cases.setup(s, nodes, ucat, p)
        s.set_turbines(tb, 1.0)
        s.step(1)
        st = s.turbine_state()
        for t, th in zip(tb, st["thrust"]):
            assert abs(th - 0.5 * 9.0 * t.ct * np.pi * t.r_tip ** 2) <= 1e-11 * th
        s.close()


def _state_after(cfg, nodes, ucat, p, tb, n, ct=None):
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p)
    s.set_turbines(tb, 1.225)
    s.step(1)                      # a state produced by the step itself
    if ct is not None:
        s.set_turbine_ct(ct)
    s.turbine_state(reset=True)
    if n:
        s.step(n)
    return s


@pytest.mark.parametrize("ddt,les", [(api.DDT_RK4, 1), (api.DDT_FE, 0)])
def test_power_gradient_matches_central_differences(ddt, les):
    cfg, nodes, ucat, p, tb = small_farm(ddt=ddt)
    cfg.les = les
    nsteps = 3
    ct0 = np.array([t.ct for t in tb])

    def J(ct):
        s = _state_after(cfg, nodes, ucat, p, tb, nsteps, ct)
        v = s.turbine_state()["power_sum"]
        s.close()
        return v

    L = _lib()
    shape = ucat.shape
    adj = {"UCONT_ADJ": np.zeros(shape), "UCAT_ADJ": np.zeros(shape), "P_ADJ": np.zeros(shape[:3]),
           "SOURCE_ADJ": np.zeros(shape)}
    grad = np.zeros(len(tb))
    for n in reversed(range(nsteps)):
        r = _state_after(cfg, nodes, ucat, p, tb, n)
        r.set_farm_objective(True)
        for k, v in adj.items():
            r.set(k, v)
        assert L.tor_adjoint_step(r.h) == 0
        adj = {k: r.get(k) for k in adj}
        grad += r.ct_gradient()
        r.close()
    for t in range(len(tb)):
        e = np.zeros(len(tb))
        e[t] = EPS
        fd = (J(ct0 + e) - J(ct0 - e)) / (2 * EPS)
        assert abs(grad[t] - fd) <= 1e-5 * abs(fd), (t, grad[t], fd)


def test_state_functional_gradient_matches_central_differences():
    # J = <wc, Ucat_N> + <wu, Ucont_N>: C_T' acts only through the flow (the
    # projected forces and, from the second step on, the sampled disk speed)
    cfg, nodes, ucat, p, tb = small_farm()
    nsteps = 3
    ct0 = np.array([t.ct for t in tb])
    rng = np.random.default_rng(5)
    interior = np.zeros(p.shape, bool)
    interior[1:-1, 1:-1, 1:-1] = True
    wc = rng.standard_normal(ucat.shape) * interior[..., None]
    wu = rng.standard_normal(ucat.shape)

    def J(ct):
        s = _state_after(cfg, nodes, ucat, p, tb, nsteps, ct)
        v = (wc * s.get("UCAT")).sum() + (wu * s.get("UCONT")).sum()
        s.close()
        return v

    L = _lib()
    adj = {"UCONT_ADJ": wu, "UCAT_ADJ": wc, "P_ADJ": np.zeros(p.shape), "SOURCE_ADJ": np.zeros(ucat.shape)}
    grad = np.zeros(len(tb))
    for n in reversed(range(nsteps)):
        r = _state_after(cfg, nodes, ucat, p, tb, n)
        for k, v in adj.items():
            r.set(k, v)
        assert L.tor_adjoint_step(r.h) == 0
        adj = {k: r.get(k) for k in adj}
        grad += r.ct_gradient()
        r.close()
    for t in range(len(tb)):
        e = np.zeros(len(tb))
        e[t] = EPS
        fd = (J(ct0 + e) - J(ct0 - e)) / (2 * EPS)
        assert abs(grad[t] - fd) <= 1e-5 * abs(fd), (t, grad[t], fd)
