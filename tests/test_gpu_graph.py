"""Step replay from a captured CUDA graph against the same steps launched
kernel by kernel: the graph runs the same kernels in the same order with the
pressure-solver loop controlled on the device, so the fields are bitwise
equal, and so are the solver statistics."""
import numpy as np
import pytest

import tosca_b200
from tosca_b200 import api, cases
from tests.common import SMALL, build_case

pytestmark = pytest.mark.gpu

FIELDS = ["UCONT", "UCAT", "P", "NUT"]


def twin(name, over=None, **kw):
    """Two CUDA solvers on the same case: eager (graphs off) and replayed."""
    cfg, nodes, ucat, p, T = build_case(name, **kw)
    for k, v in (over or {}).items():
        setattr(cfg, k, v)
    out = []
    for graphs in (False, True):
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p, T)
        s.set_graphs(graphs)
        out.append(s)
    return out


def assert_same(e, r):
    for f in FIELDS:
        a, b = e.get(f), r.get(f)
        assert np.array_equal(a, b), (f, float(np.max(np.abs(a - b))))


@pytest.mark.parametrize("name,prec", [("tgv", api.PREC_FP64), ("abl", api.PREC_FP64),
                                       ("abl", api.PREC_MIXED), ("hill", api.PREC_FP64)])
def test_replay_bitwise(name, prec):
    e, r = twin(name, {"precision": prec}, **SMALL[name])
    se, sr = e.step(6), r.step(6)
    assert_same(e, r)
    assert se.poisson_total_iterations == sr.poisson_total_iterations
    assert se.poisson_iterations == sr.poisson_iterations
    assert se.poisson_final_residual == sr.poisson_final_residual
    assert se.max_divergence == sr.max_divergence
    assert se.steps == sr.steps == 6
    replays, failed = r.graph_info()
    assert not failed
    # the first step runs eagerly (first-step branches)
    assert replays == 5
    assert e.graph_info()[0] == 0
    e.close(); r.close()


def test_replay_across_calls_and_field_writes():
    e, r = twin("abl", **SMALL["abl"])
    for s in (e, r):
        s.step(2)
    rng = np.random.default_rng(7)
    dp = rng.standard_normal(e.shape + (3,)) * 1e-3
    for s in (e, r):
        s.set("DP", dp)        # a caller-written dP: the next step clears it eagerly
        s.step(1)
        s.step(3)
    assert_same(e, r)
    assert r.graph_info()[0] == 4
    e.close(); r.close()


def test_replay_iteration_cap_reported():
    e, r = twin("tgv", {"poisson_maxit": 1, "poisson_rtol": 1e-14}, **SMALL["tgv"])
    for s in (e, r):
        with pytest.raises(api.TgError) as ei:
            s.step(4)
        assert ei.value.status == api.TG_ERR_NOT_CONVERGED
    assert_same(e, r)
    assert r.graph_info()[0] == 3
    e.close(); r.close()


def test_step_host_replayed():
    e, r = twin("tgv", **SMALL["tgv"])
    states = []
    for s in (e, r):
        s.step(1)
        u, c, p = s.get("UCONT"), s.get("UCAT"), s.get("P")
        for _ in range(3):
            st = s.step_host(u, c, p)
        states.append((u, c, p, st))
    for a, b in zip(states[0][:3], states[1][:3]):
        assert np.array_equal(a, b)
    assert states[0][3].poisson_iterations == states[1][3].poisson_iterations
    assert r.graph_info()[0] == 3
    e.close(); r.close()


def test_step_host_nut_copied_during_the_step():
    """tg_step_host copies nut out on its own stream from the event recorded
    after UpdateNut (an external event node inside the replayed step graph):
    the eager and the replayed drop-in steps return the same nut, bit for
    bit, equal to the context's own nut after the step (UpdateNut is its only
    writer), on the LES ABL with the wall function."""
    e, r = twin("abl", **SMALL["abl"])
    outs = []
    for s in (e, r):
        s.step(1)
        u, c, p = s.get("UCONT"), s.get("UCAT"), s.get("P")
        nut = np.full(s.shape, -1.0)
        for _ in range(4):
            s.step_host(u, c, p, nut)
            assert np.array_equal(nut, s.get("NUT"))
        outs.append((u, c, p, nut))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    assert r.graph_info()[0] == 4
    e.close(); r.close()


def test_graphs_off_then_on():
    e, r = twin("tgv", **SMALL["tgv"])
    e.step(2)
    r.step(2)
    r.set_graphs(False)
    r.step(2)
    r.set_graphs(True)
    r.step(2)
    e.step(4)
    assert_same(e, r)
    e.close(); r.close()



def _adjoint_twin(ddt):
    from tests.test_gpu_adjoint import _case
    rng = np.random.default_rng(11)
    cfg, nodes, ucat, p = _case("abl", ddt)
    f0 = rng.standard_normal(ucat.shape) * 0.01
    out = []
    for graphs in (False, True):
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p)
        s.set_graphs(graphs)
        s.set("SOURCE", f0)
        s.step(1)
        out.append(s)
    inside = np.zeros(p.shape, bool)
    inside[1:-1, 1:-1, 1:-1] = True
    seeds = (rng.standard_normal(ucat.shape), rng.standard_normal(ucat.shape) * inside[..., None],
             rng.standard_normal(p.shape))
    return out, seeds


ADJ = ("UCONT_ADJ", "UCAT_ADJ", "P_ADJ", "SOURCE_ADJ")


def _seed(s, seeds):
    s.set("UCONT_ADJ", seeds[0]); s.set("UCAT_ADJ", seeds[1]); s.set("P_ADJ", seeds[2])
    s.set("SOURCE_ADJ", np.zeros(seeds[0].shape))


def _same_adjoint(e, r):
    # the forward state is restored bitwise; the transposed face fluxes and
    # gradients scatter with FP64 atomics, whose summation order varies (the
    # adjoint seeds are O(1); P_ADJ itself can be at round-off level)
    for f in ("UCONT", "UCAT", "P"):
        assert np.array_equal(e.get(f), r.get(f)), f
    for f in ADJ:
        a, b = e.get(f), r.get(f)
        assert np.linalg.norm(a - b) <= 1e-11 * max(np.linalg.norm(b), 1.0), f


@pytest.mark.parametrize("ddt", [api.DDT_FE, api.DDT_RK4])
def test_adjoint_step_replay(ddt):
    (e, r), seeds = _adjoint_twin(ddt)
    for s in (e, r):
        _seed(s, seeds)
        for _ in range(3):
            s.adjoint_step()
    _same_adjoint(e, r)
    assert r.graph_info()[0] == 3     # the taped forward steps
    e.close(); r.close()


@pytest.mark.parametrize("nsnap", [5, 2])
def test_adjoint_reverse_replay(nsnap):
    # nsnap = steps keeps every tape; fewer snapshots re-run forward steps
    (e, r), seeds = _adjoint_twin(api.DDT_RK4)
    stats = []
    for s in (e, r):
        s.adjoint_forward(5, nsnap)
        _seed(s, seeds)
        stats.append(s.adjoint_reverse())
    _same_adjoint(e, r)
    assert abs(stats[0].poisson_iterations - stats[1].poisson_iterations) <= 5
    assert stats[0].forward_steps == stats[1].forward_steps
    assert r.graph_info()[0] > 0
    e.close(); r.close()
