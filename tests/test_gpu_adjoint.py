"""Adjoint of the CUDA step (tg_adjoint_*), checked three ways:

* against the adjoint restatement in the oracle, field by field, after one
  step (both transpose the same discrete step);
* dot-product test: <w, J v> with the tangent J v from central differences of
  the CUDA step equals <J^T w, v> from the CUDA adjoint;
* gradient of J = <wu, Ucont_N> + <wc, Ucat_N> with respect to the body force
  over N steps (revolve checkpointing with fewer snapshots than steps) against
  central differences of the CUDA step and of the oracle's (CPU) step.

Central differences use eps = 1e-6 (relative tolerance 1e-5); the field
comparison with the oracle uses 1e-8 relative L2 (both pressure solves are
converged to <= 1e-12)."""
import ctypes

import numpy as np
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases
from tests.common import interior, rel_l2

pytestmark = pytest.mark.gpu
EPS = 1e-6
ADJ = ("UCONT_ADJ", "UCAT_ADJ", "P_ADJ", "SOURCE_ADJ")


def _case(name, ddt, div=api.DIV_CENTRAL, les=None):
    if name == "tgv":
        cfg, nodes, ucat, p = cases.tgv_case(12, ddt=ddt)
    else:
        # "abl_wall": the Schumann wall function on the ground (its filter
        # state is part of the state, adjoint field WALL_ADJ)
        cfg, nodes, ucat, p = cases.abl_case(nx=12, ny=10, nz=8, Lx=120.0, Ly=100.0, H=80.0, dz1=4.0, ddt=ddt,
                                             wall=api.BC_WALL_SHUMANN if name == "abl_wall" else api.BC_NOSLIP)
    cfg.div_scheme = div
    if les is not None:
        cfg.les = les
    cfg.poisson_rtol = 1e-13
    cfg.source = 1
    return cfg, nodes, ucat, p


def _start(make, cfg, nodes, ucat, p, f0, steps=1):
    s = make(cfg)
    cases.setup(s, nodes, ucat, p)
    s.set("SOURCE", f0)
    s.step(steps)
    return s


def _olib():
    L = oracle.lib()
    L.tor_adjoint_step.argtypes = [ctypes.c_void_p]
    L.tor_adjoint_step.restype = ctypes.c_int
    return L


def _seeds(rng, shape3, shape1):
    inside = np.zeros(shape1, bool)
    inside[1:-1, 1:-1, 1:-1] = True
    return (rng.standard_normal(shape3), rng.standard_normal(shape3) * inside[..., None],
            rng.standard_normal(shape1))


@pytest.mark.parametrize("name,ddt,div", [
    ("tgv", api.DDT_FE, api.DIV_CENTRAL),
    ("tgv", api.DDT_RK4, api.DIV_CENTRAL),
    ("abl", api.DDT_FE, api.DIV_CENTRAL),
    ("abl", api.DDT_RK4, api.DIV_CENTRAL),
    ("abl", api.DDT_RK4, api.DIV_QUICK),
    ("abl_wall", api.DDT_FE, api.DIV_CENTRAL),
    ("abl_wall", api.DDT_RK4, api.DIV_QUICK),
])
def test_adjoint_step_matches_oracle(name, ddt, div):
    rng = np.random.default_rng(7)
    cfg, nodes, ucat, p = _case(name, ddt, div)
    f0 = rng.standard_normal(ucat.shape) * 0.01
    g = _start(tosca_b200.gpu_solver, cfg, nodes, ucat, p, f0)
    o = _start(oracle.solver, cfg, nodes, ucat, p, f0)
    wu, wc, wp = _seeds(rng, ucat.shape, p.shape)
    keys = ADJ
    for s in (g, o):
        s.set("UCONT_ADJ", wu); s.set("UCAT_ADJ", wc); s.set("P_ADJ", wp); s.set("SOURCE_ADJ", np.zeros_like(f0))
    if name == "abl_wall":
        ww = rng.standard_normal((cfg.mz, cfg.mx, 3))
        for s in (g, o):
            s.set("WALL_ADJ", ww)
        keys = ADJ + ("WALL_ADJ",)
    g.adjoint_step()
    L = _olib()
    assert L.tor_adjoint_step(o.h) == 0, L.tor_last_error(o.h)
    for k in keys:
        a, b = g.get(k), o.get(k)
        nb = np.linalg.norm(b)
        if nb < 1e-12:
            assert np.linalg.norm(a) < 1e-9, k
            continue
        assert np.linalg.norm(a - b) <= 1e-8 * nb, (k, np.linalg.norm(a - b) / nb)
    # the state is the one at the start of the step again
    o2 = _start(oracle.solver, cfg, nodes, ucat, p, f0)
    assert rel_l2(g.get("UCONT"), o2.get("UCONT")) < 1e-10
    g.close(); o.close(); o2.close()


@pytest.mark.parametrize("name", ["abl", "abl_wall"])
def test_dot_product_with_central_difference_tangent(name):
    """<w, (F(x + eps v) - F(x - eps v)) / 2 eps> = <J^T w, v> for the one-step
    map F on Ucont (ABL, RK4, Smagorinsky; with the wall function, F also
    carries the wall filter state, so every evaluation starts from a context
    with the same history)."""
    rng = np.random.default_rng(11)
    cfg, nodes, ucat, p = _case(name, api.DDT_RK4)
    f0 = rng.standard_normal(ucat.shape) * 0.01
    g = _start(tosca_b200.gpu_solver, cfg, nodes, ucat, p, f0)
    x0 = {k: g.get(k) for k in ("UCONT", "UCAT", "P")}
    wu, wc, wp = _seeds(rng, ucat.shape, p.shape)
    v = rng.standard_normal(ucat.shape) * np.abs(x0["UCONT"]).max() * 1e-3

    def F(du):
        t = _start(tosca_b200.gpu_solver, cfg, nodes, ucat, p, f0)
        t.set("UCONT", x0["UCONT"] + du); t.set("UCAT", x0["UCAT"]); t.set("P", x0["P"])
        t.step(1)
        out = (wu * t.get("UCONT")).sum() + (wc * t.get("UCAT")).sum() + (wp * t.get("P")).sum()
        t.close()
        return out

    lhs = (F(EPS * v) - F(-EPS * v)) / (2 * EPS)
    g.set("UCONT_ADJ", wu); g.set("UCAT_ADJ", wc); g.set("P_ADJ", wp); g.set("SOURCE_ADJ", np.zeros_like(f0))
    g.adjoint_step()
    rhs = (g.get("UCONT_ADJ") * v).sum()
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs)), (lhs, rhs)
    g.close()


@pytest.mark.parametrize("name,nsteps,nsnap,tapes", [("abl", 4, 2, 0), ("abl", 5, 5, -1), ("abl_wall", 4, 2, 0),
                                                     ("abl_wall", 5, 5, -1), ("abl_wall", 5, 3, 2), ("abl", 6, 3, -1)])
def test_gradient_with_checkpointing_matches_central_differences(name, nsteps, nsnap, tapes):
    """dJ/df . v over N steps, reversed with a binomial checkpoint schedule
    (tapes = 0), every tape kept (nsnap = N) or the segment schedule (tapes of
    k steps: each step re-run once in the reversal), against central
    differences of the CUDA step and of the oracle's CPU step (the reference
    gradient)."""
    rng = np.random.default_rng(5)
    cfg, nodes, ucat, p = _case(name, api.DDT_RK4)
    f0 = rng.standard_normal(ucat.shape) * 0.01
    g = _start(tosca_b200.gpu_solver, cfg, nodes, ucat, p, f0)
    x0 = {k: g.get(k) for k in ("UCONT", "UCAT", "P")}
    wu, wc, _ = _seeds(rng, ucat.shape, p.shape)

    def J(make, f):
        s = _start(make, cfg, nodes, ucat, p, f0)
        s.set("SOURCE", f)
        s.step(nsteps)
        out = (wu * s.get("UCONT")).sum() + (wc * s.get("UCAT")).sum()
        s.close()
        return out

    g.adjoint_set_tapes(tapes)
    st = g.adjoint_forward(nsteps, nsnap)
    assert st.steps == nsteps
    g.set("UCONT_ADJ", wu); g.set("UCAT_ADJ", wc); g.set("P_ADJ", np.zeros_like(p))
    g.set("SOURCE_ADJ", np.zeros_like(f0))
    if cfg.bc[2] == api.BC_WALL_SHUMANN:
        g.set("WALL_ADJ", np.zeros((cfg.mz, cfg.mx, 3)))
    ast = g.adjoint_reverse()
    assert ast.steps == nsteps
    if nsnap < nsteps and tapes == 0:
        assert ast.forward_steps > nsteps           # binomial schedule: recomputation happened
    elif nsnap < nsteps:
        assert ast.forward_steps == nsteps          # segment schedule: each step re-run once
    grad = g.get("SOURCE_ADJ")
    # the context is back at the initial state
    assert rel_l2(g.get("UCONT"), x0["UCONT"]) < 1e-14
    v = rng.standard_normal(f0.shape)
    ad = (grad * v).sum()
    fd_gpu = (J(tosca_b200.gpu_solver, f0 + EPS * v) - J(tosca_b200.gpu_solver, f0 - EPS * v)) / (2 * EPS)
    fd_cpu = (J(oracle.solver, f0 + EPS * v) - J(oracle.solver, f0 - EPS * v)) / (2 * EPS)
    assert abs(ad - fd_gpu) <= 1e-5 * abs(fd_gpu), (ad, fd_gpu)
    assert abs(ad - fd_cpu) <= 1e-5 * abs(fd_cpu), (ad, fd_cpu)
    g.close()


def test_unsupported_configurations_are_rejected():
    # the curvilinear hill: non-symmetric pressure operator
    cfg, nodes, ucat, p, T = cases.hill_case(nx=12, ny=8, nz=8)
    g = tosca_b200.gpu_solver(cfg)
    cases.setup(g, nodes, ucat, p, T)
    with pytest.raises(api.TgError) as e:
        g.adjoint_step()
    assert e.value.status == api.TG_ERR_BAD_ARG
    g.close()
