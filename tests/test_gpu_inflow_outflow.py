"""Inflow and outflow velocity patches on the GPU against the oracle, whose
restatement of them is pinned to TOSCA's own code (tests/test_ref_pin.py).

The open channel (cases.channel_case: fixedValue inflow at x = 0,
zeroGradient outflow at x = Lx, noSlip or Schumann-wall ground, slip top,
periodic y) exercises UpdateCartesianBCs for both patch types
(boundary.c:1632-1673, 1897-1970), the reverse-flow clip of
UpdateContravariantBCs (boundary.c:718-741), the outflow faces kept by
resetNonResolvedCellFaces (inline.h:1674-1835) and adjustFluxesLocal
(ueqn.c:748-1135) at the end of the momentum solve. FP64 bar: 1e-10 relative
L2 on u, v, w and p after ten steps, the largest divergence at or below the
oracle's up to the round-off floor; mixed precision within 1e-6."""
import numpy as np
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases
from tests.common import SMALL, build_case, div_roundoff_floor, pair, rel_l2

pytestmark = pytest.mark.gpu

TIGHT = {"poisson_rtol": 1e-13}


def _bc(wall=api.BC_NOSLIP):
    return (api.BC_PERIODIC, api.BC_PERIODIC, wall, api.BC_SLIP, api.BC_FIXED_VALUE, api.BC_ZERO_GRADIENT)


@pytest.mark.parametrize("ddt,wall,div", [(api.DDT_FE, api.BC_NOSLIP, api.DIV_CENTRAL),
                                          (api.DDT_RK4, api.BC_NOSLIP, api.DIV_CENTRAL),
                                          (api.DDT_RK4, api.BC_WALL_SHUMANN, api.DIV_CENTRAL),
                                          (api.DDT_RK4, api.BC_NOSLIP, api.DIV_QUICK)])
def test_channel_ten_steps(ddt, wall, div):
    g, o = pair("channel", dict(TIGHT, ddt_scheme=ddt, div_scheme=div, bc=_bc(wall)), **SMALL["channel"])
    div_g = [g.step(1).max_divergence for _ in range(10)]
    div_o = [o.step(1).max_divergence for _ in range(10)]
    u_g, u_o = g.get("UCAT"), o.get("UCAT")
    for c in range(3):
        assert rel_l2(u_g[..., c], u_o[..., c]) < 1e-10, c
    assert rel_l2(g.get("UCONT"), o.get("UCONT")) < 1e-10
    assert rel_l2(g.get("P"), o.get("P")) < 1e-10
    floor = div_roundoff_floor(o.get("UCONT"), o.get("AJ"))
    assert max(div_g) <= max(div_o) + floor, (div_g, div_o, floor)
    g.close(); o.close()


@pytest.mark.parametrize("localized", [False, True])
def test_stratified_channel(localized):
    """The stratified ABL opened in x (cases.open_x: 8 m/s at 301 K through
    the fixedValue inflow, zeroGradient outflow for velocity and temperature)
    with the RK4 temperature equation, Boussinesq buoyancy and the
    Schumann-Grotzbach thermal wall function on the ground: ten steps, GPU
    against the oracle (itself pinned to TOSCA's own code on this case)."""
    cfg, nodes, ucat, p, T = cases.stratified_abl_case(16, 12, 12, heating_rate=-0.01, localized=localized, t_amp=0.5)
    cases.open_x(cfg, 8.0, 301.0)
    cfg.poisson_rtol = 1e-13
    g = tosca_b200.gpu_solver(cfg)
    o = oracle.solver(cfg)
    for s in (g, o):
        cases.setup(s, nodes, ucat, p, T)
        s.step(10)
    for f in ("UCAT", "P", "TMPRT"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
    qg, qo = g.get("QWALL"), o.get("QWALL")
    assert np.abs(qg - qo).max() <= 1e-9 * np.abs(qo).max()
    g.close(); o.close()


@pytest.mark.parametrize("prec", [api.PREC_FP64, api.PREC_MIXED])
def test_open_hill(prec):
    """The curvilinear QUICK hill with the inflow/outflow pair of TOSCA's
    CosineHillCurvTest deck (fixedValue inflow, zeroGradient outflow; the
    general-metric kernels and the BiCGStab pressure solve), RK4 with the
    transported temperature (inflow at 301 K), ten steps: FP64 within 1e-10
    of the oracle (P 1e-9, as on the periodic hill), mixed within 1e-6."""
    cfg, nodes, ucat, p, T = cases.hill_case(24, 12, 12, ddt=api.DDT_RK4, teqn=True, t_amp=0.5)
    cases.open_x(cfg, 8.0, 301.0)
    cfg.poisson_rtol = 1e-13
    cfg.precision = prec
    g = tosca_b200.gpu_solver(cfg)
    o = oracle.solver(cfg)
    for s in (g, o):
        cases.setup(s, nodes, ucat, p, T)
        s.step(10)
    tol = 1e-10 if prec == api.PREC_FP64 else 1e-6
    for f in ("UCAT", "TMPRT"):
        assert rel_l2(g.get(f), o.get(f)) < tol, f
    assert rel_l2(g.get("P"), o.get("P")) < (1e-9 if prec == api.PREC_FP64 else 1e-6)
    g.close(); o.close()


def test_channel_multiblock_mixed():
    """A channel spanning several blocks of every kernel (48 x 40 x 16 cells:
    two blocks of the face-flux kernel in i), RK4, FP64 within 1e-10 and
    mixed precision within 1e-6 of the FP64 oracle after ten steps."""
    size = dict(nx=48, ny=40, nz=16, Lx=480.0, Ly=400.0, H=100.0)
    g, o = pair("channel", dict(TIGHT, ddt_scheme=api.DDT_RK4), **size)
    cfg, nodes, ucat, p, T = build_case("channel", **size)
    cfg.poisson_rtol = 1e-13
    cfg.ddt_scheme = api.DDT_RK4
    cfg.precision = api.PREC_MIXED
    m = tosca_b200.gpu_solver(cfg)
    cases.setup(m, nodes, ucat, p, T)
    for s in (g, o, m):
        s.step(10)
    for f in ("UCAT", "P"):
        assert rel_l2(g.get(f), o.get(f)) < 1e-10, f
        assert rel_l2(m.get(f), o.get(f)) < 1e-6, f
    g.close(); o.close(); m.close()


def test_reverse_flow_and_ghosts():
    """UpdateCartesianBCs and UpdateContravariantBCs on a velocity field that
    flows back in through part of the outflow patch: the zeroGradient faces
    with inflow are clipped to zero, the fixedValue ghosts hold the patch
    value; GPU and oracle agree to round-off."""
    g, o = pair("channel", TIGHT, **SMALL["channel"])
    u = o.get("UCAT")
    rng = np.random.default_rng(5)
    u[1:-1, 1:-1, 1:-1] += rng.standard_normal(u[1:-1, 1:-1, 1:-1].shape) * 4.0
    for s in (g, o):
        s.set("UCAT", u)
        s.UpdateCartesianBCs()
        s.UpdateContravariantBCs()
    assert rel_l2(g.get("UCAT"), o.get("UCAT")) < 1e-14
    assert rel_l2(g.get("UCONT"), o.get("UCONT")) < 1e-14
    uc = g.get("UCONT")[-2, 1:-1, 1:-1, 2]
    assert (uc >= 0.0).all() and (uc == 0.0).any()
    ghost = g.get("UCAT")[0, 1:-1, 1:-1]
    assert np.array_equal(ghost, np.broadcast_to(np.array(g.cfg.bc_value[12:15]), ghost.shape))
    g.close(); o.close()


def test_solve_u_balances_the_boundary_flux():
    """SolveUEqn from the step-start state: after adjustFluxesLocal the
    outflow through the zeroGradient patch equals the inflow through the
    fixedValue patch, on the GPU as on the oracle."""
    g, o = pair("channel", dict(TIGHT, ddt_scheme=api.DDT_RK4), **SMALL["channel"])
    for s in (g, o):
        s.set("UCONT_O", s.get("UCONT"))
        s.UpdateNut(); s.UpdateWallModelsU(); s.GradP()
        s.SolveUEqn()
        w = s.get("UCONT")[..., 2]
        fin, fout = w[0, 1:-1, 1:-1].sum(), w[-2, 1:-1, 1:-1].sum()
        assert abs(fin - fout) <= 1e-12 * abs(fin)
    assert rel_l2(g.get("UCONT"), o.get("UCONT")) < 1e-13
    g.close(); o.close()


def test_channel_replay_bitwise():
    """Steps replayed from the captured CUDA graph equal the kernel-by-kernel
    steps bit for bit with the inflow/outflow patches (adjustFluxesLocal runs
    on device scalars inside the graph)."""
    cfg, nodes, ucat, p, T = build_case("channel", **SMALL["channel"])
    cfg.ddt_scheme = api.DDT_RK4
    out = []
    for graphs in (False, True):
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.set_graphs(graphs)
        s.step(5)
        out.append(s)
    e, r = out
    for f in ("UCONT", "UCAT", "P", "NUT"):
        assert np.array_equal(e.get(f), r.get(f)), f
    assert r.graph_info()[0] == 4
    e.close(); r.close()


@pytest.mark.parametrize("name,prec", [("channel", api.PREC_FP64), ("channel", api.PREC_MIXED),
                                       ("ohill", api.PREC_FP64)])
def test_log_inlet(name, prec):
    """The kLeft log-law inletFunction (type 2, cases.log_inlet) in place of
    the fixedValue inflow, hInv = 60 m on the 100 m channel (both branches of
    the profile) and none on the open hill, a direction with x and y
    components: ten RK4 steps against the oracle (itself pinned to TOSCA's
    own code on these cases), FP64 within 1e-10 (P 1e-9 on the hill), mixed
    within 1e-6; the ghosts after UpdateCartesianBCs within 1e-14."""
    cfg, nodes, ucat, p, T = build_case(name, **SMALL[name])
    cases.log_inlet(cfg, 0.4, 0.1, 60.0 if name == "channel" else 1e30, (0.96, 0.28, 0.0))
    cfg.poisson_rtol = 1e-13
    cfg.ddt_scheme = api.DDT_RK4
    cfg.precision = prec
    g = tosca_b200.gpu_solver(cfg)
    o = oracle.solver(cfg)
    for s in (g, o):
        cases.setup(s, nodes, ucat, p, T)
        s.UpdateCartesianBCs()
    assert rel_l2(g.get("UCAT")[0], o.get("UCAT")[0]) < 1e-14
    for s in (g, o):
        s.step(10)
    tol = 1e-10 if prec == api.PREC_FP64 else 1e-6
    assert rel_l2(g.get("UCAT"), o.get("UCAT")) < tol
    assert rel_l2(g.get("P"), o.get("P")) < (1e-9 if name == "ohill" and prec == api.PREC_FP64 else tol)
    g.close(); o.close()


def test_unsupported_combinations_are_refused():
    cfg, *_ = build_case("channel", **SMALL["channel"])
    for ddt in (api.DDT_CN, api.DDT_ABCN, api.DDT_RK3WCN, api.DDT_RK3SOCN):
        cfg.ddt_scheme = ddt
        with pytest.raises(api.TgError):
            tosca_b200.gpu_solver(cfg)
        with pytest.raises(api.TgError):
            oracle.solver(cfg)
    # the log-law inletFunction on kLeft only, with a unit direction
    for bad in ({"bc": _bc()[:5] + (api.BC_INLET_LOG,)}, {"inlet_dir": (1.0, 1.0, 0.0)}, {"inlet_z0": -1.0}):
        cfg, *_ = build_case("channel", **SMALL["channel"])
        cases.log_inlet(cfg)
        for k, v in bad.items():
            setattr(cfg, k, v)
        with pytest.raises(api.TgError):
            tosca_b200.gpu_solver(cfg)
    # the adjoint of the inflow/outflow patches is not built
    for log in (False, True):
        cfg, nodes, ucat, p, T = build_case("channel", **SMALL["channel"])
        cfg.ddt_scheme = api.DDT_RK4
        if log:
            cases.log_inlet(cfg)
        g = tosca_b200.gpu_solver(cfg)
        cases.setup(g, nodes, ucat, p, T)
        with pytest.raises(api.TgError):
            g.adjoint_forward(2, 2)
        g.close()
