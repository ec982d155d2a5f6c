"""CPU checks of the adjoint restatement in the oracle (the checker of the
CUDA adjoint): central finite differences of a linear functional of the
state after one or more steps, J = <wu, Ucont> + <wc, Ucat> + <wp, P>, with
respect to the body force, the initial Ucont, Ucat and P. Runs on the CPU."""
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


def _case(name, ddt, div):
    if name == "tgv":
        cfg, nodes, ucat, p = cases.tgv_case(8, ddt=ddt)
    else:
        # "abl_wall": the Schumann wall function (-3) on the ground
        cfg, nodes, ucat, p = cases.abl_case(nx=8, ny=6, nz=6, Lx=80.0, Ly=60.0, H=60.0, dz1=4.0, ddt=ddt,
                                             wall=api.BC_WALL_SHUMANN if name == "abl_wall" else api.BC_NOSLIP)
    cfg.div_scheme = div
    cfg.poisson_rtol = 1e-14
    cfg.source = 1
    return cfg, nodes, ucat, p


def _start(cfg, nodes, ucat, p, f0, extra_steps=0):
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p)
    s.set("SOURCE", f0)
    s.step(1 + extra_steps)      # a state produced by the step itself
    return s


def adjoint_vs_fd(name, ddt, div=api.DIV_CENTRAL, nsteps=1, seed=3):
    rng = np.random.default_rng(seed)
    cfg, nodes, ucat, p = _case(name, ddt, div)
    f0 = rng.standard_normal(ucat.shape) * 0.01
    s = _start(cfg, nodes, ucat, p, f0)
    st0 = {k: s.get(k) for k in ("UCONT", "UCAT", "P")}
    s.close()
    interior = np.zeros(st0["P"].shape, bool)
    interior[1:-1, 1:-1, 1:-1] = True
    wu = rng.standard_normal(st0["UCONT"].shape)
    wc = rng.standard_normal(st0["UCAT"].shape) * interior[..., None]
    wp = rng.standard_normal(st0["P"].shape)

    def J(f, du=0.0, dc=0.0, dp=0.0):
        t = _start(cfg, nodes, ucat, p, f0)
        t.set("UCONT", st0["UCONT"] + du)
        t.set("UCAT", st0["UCAT"] + dc)
        t.set("P", st0["P"] + dp)
        t.set("SOURCE", f)
        t.step(nsteps)
        v = (wu * t.get("UCONT")).sum() + (wc * t.get("UCAT")).sum() + (wp * t.get("P")).sum()
        t.close()
        return v

    L = _lib()
    adj = {"UCONT_ADJ": wu, "UCAT_ADJ": wc, "P_ADJ": wp, "SOURCE_ADJ": np.zeros_like(f0)}
    if cfg.bc[2] == api.BC_WALL_SHUMANN:
        adj["WALL_ADJ"] = np.zeros((cfg.mz, cfg.mx, 3))   # the filter state after the last step feeds no functional
    for n in reversed(range(nsteps)):
        r = _start(cfg, nodes, ucat, p, f0, extra_steps=n)
        for k, v in adj.items():
            r.set(k, v)
        assert L.tor_adjoint_step(r.h) == 0, L.tor_last_error(r.h)
        adj = {k: r.get(k) for k in adj}
        r.close()
    out = {}
    for what, key in (("source", "SOURCE_ADJ"), ("ucont", "UCONT_ADJ"), ("ucat", "UCAT_ADJ"), ("p", "P_ADJ")):
        v = rng.standard_normal(adj[key].shape)
        if what in ("ucat", "p"):
            v = v * (interior[..., None] if what == "ucat" else interior)
        if what == "source":
            fd = (J(f0 + EPS * v) - J(f0 - EPS * v)) / (2 * EPS)
        else:
            kw = {"ucont": "du", "ucat": "dc", "p": "dp"}[what]
            fd = (J(f0, **{kw: EPS * v}) - J(f0, **{kw: -EPS * v})) / (2 * EPS)
        out[what] = (float((adj[key] * v).sum()), float(fd))
    return out


def _check(out, skip=()):
    for what, (ad, fd) in out.items():
        if what in skip:
            continue
        scale = max(abs(fd), abs(ad), 1e-12)
        assert abs(ad - fd) <= 2e-5 * scale, (what, ad, fd)


@pytest.mark.parametrize("name,ddt,div", [
    ("tgv", api.DDT_FE, api.DIV_CENTRAL),
    ("tgv", api.DDT_RK4, api.DIV_CENTRAL),
    ("abl", api.DDT_FE, api.DIV_CENTRAL),
    ("abl", api.DDT_RK4, api.DIV_QUICK),
])
def test_one_step_gradient_matches_finite_differences(name, ddt, div):
    # without LES the interior Ucat at the start of a step is read by nothing: its gradient is zero
    _check(adjoint_vs_fd(name, ddt, div), skip=("ucat",) if name == "tgv" else ())


def test_three_steps_gradient_matches_finite_differences():
    _check(adjoint_vs_fd("abl", api.DDT_RK4, nsteps=3))


@pytest.mark.parametrize("ddt,nsteps", [(api.DDT_FE, 1), (api.DDT_RK4, 1), (api.DDT_RK4, 3)])
def test_wall_function_gradient_matches_finite_differences(ddt, nsteps):
    """The Schumann wall stress (UpdateWallModelsU, boundary.c:3257-3600) and
    its time-filtered wall velocity differentiated: the filter state passes
    between reversed steps through TG_F_WALL_ADJ."""
    _check(adjoint_vs_fd("abl_wall", ddt, nsteps=nsteps))
