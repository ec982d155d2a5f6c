"""The adjoint configuration end to end: the gradient of the hub-height probe
misfit J = sum (u - u_obs)^2 (64 x 64 probes) after 20 steps of the ABL
with its Schumann wall function, with respect to the 3-D body force, taken
through the torch.autograd.Function harness of tests/c4_harness.py (forward:
tg_adjoint_forward with 10 snapshots for 20 steps; backward:
tg_adjoint_reverse), and checked against central differences of J:

* FP64 at 128 x 64 x 64 cells against central differences of the CUDA step
  (eps = 1e-6 relative to the body force);
* FP64 at 64 x 32 x 32 cells against central differences of the oracle's CPU
  step (the reference gradient);
* the mixed-precision forward (FP32 stencils and multigrid): the FP64 adjoint
  along the mixed trajectory against central differences of the mixed step,
  with a step (1e-3) above the FP32 rounding of J."""
import numpy as np
import pytest
import torch

import oracle
import tosca_b200
from tests import c4_harness as H
from tosca_b200 import api, cases

pytestmark = pytest.mark.gpu
STEPS, SNAPS = 20, 10


def _fresh(make, cfg, nodes, ucat, p, warm=2):
    """A solver at the start state (two steps in: wall filter seeded)."""
    s = make(cfg)
    cases.setup(s, nodes, ucat, p)
    s.set("SOURCE", np.zeros(ucat.shape))
    s.step(warm)
    return s


def _objective(make, cfg, nodes, ucat, p, idx, u_obs, f):
    s = _fresh(make, cfg, nodes, ucat, p)
    s.set("SOURCE", f)
    s.step(STEPS)
    u = H.probes(s.get("UCAT"), idx)
    s.close()
    return float(((u - u_obs) ** 2).sum())


def _gradient(cfg, nodes, ucat, p, idx, u_obs, f):
    s = _fresh(tosca_b200.gpu_solver, cfg, nodes, ucat, p)
    x0 = {k: s.get(k) for k in ("UCONT", "UCAT", "P")}
    ft = torch.tensor(f, requires_grad=True)
    U = H.StepsFunction.apply(ft, s, x0, STEPS, SNAPS)
    J = H.misfit(U, idx, u_obs)
    J.backward()
    back = {k: s.get(k) for k in ("UCONT", "UCAT", "P")}
    s.close()
    return float(J.detach()), ft.grad.numpy(), x0, back


def _setup(size, precision=api.PREC_FP64):
    cfg, nodes, ucat, p = H.c4_case(*size, precision=precision)
    idx = H.probe_index(nodes, cfg)
    f_obs = H.body_force(ucat.shape, seed=4)
    s = _fresh(tosca_b200.gpu_solver, cfg, nodes, ucat, p)
    s.set("SOURCE", f_obs)
    s.step(STEPS)
    u_obs = H.probes(s.get("UCAT"), idx)
    s.close()
    f0 = H.body_force(ucat.shape, seed=21)
    return cfg, nodes, ucat, p, idx, u_obs, f0


def test_probe_plane_is_64_by_64():
    cfg, nodes, ucat, p = H.c4_case()
    j, ks, is_ = H.probe_index(nodes, cfg)
    assert len(ks) == 64 and len(is_) == 64
    zc = 0.5 * (nodes[0, j - 1, 0, 2] + nodes[0, j, 0, 2])
    assert abs(zc - H.HUB) < 10.0


def test_c4_gradient_against_cuda_central_differences():
    cfg, nodes, ucat, p, idx, u_obs, f0 = _setup((128, 64, 64))
    J, grad, x0, back = _gradient(cfg, nodes, ucat, p, idx, u_obs, f0)
    assert J > 0.0
    # the reversal leaves the context at the start state
    for k in x0:
        assert np.linalg.norm(back[k] - x0[k]) <= 1e-14 * np.linalg.norm(x0[k]), k
    v = np.random.default_rng(9).standard_normal(f0.shape) * np.abs(f0).max()
    eps = 1e-6
    Jp = _objective(tosca_b200.gpu_solver, cfg, nodes, ucat, p, idx, u_obs, f0 + eps * v)
    Jm = _objective(tosca_b200.gpu_solver, cfg, nodes, ucat, p, idx, u_obs, f0 - eps * v)
    fd = (Jp - Jm) / (2 * eps)
    ad = float((grad * v).sum())
    assert abs(ad - fd) <= 1e-5 * abs(fd), (ad, fd)


def test_c4_gradient_against_cpu_reference_gradient():
    """The reference gradient: central differences of the oracle's CPU step
    (64 x 32 x 32 cells to keep the CPU time bounded)."""
    cfg, nodes, ucat, p, idx, u_obs, f0 = _setup((64, 32, 32))
    J, grad, _, _ = _gradient(cfg, nodes, ucat, p, idx, u_obs, f0)
    v = np.random.default_rng(9).standard_normal(f0.shape) * np.abs(f0).max()
    eps = 1e-6
    Jp = _objective(oracle.solver, cfg, nodes, ucat, p, idx, u_obs, f0 + eps * v)
    Jm = _objective(oracle.solver, cfg, nodes, ucat, p, idx, u_obs, f0 - eps * v)
    fd = (Jp - Jm) / (2 * eps)
    ad = float((grad * v).sum())
    assert abs(ad - fd) <= 1e-5 * abs(fd), (ad, fd)
    # the oracle's J itself agrees with the CUDA step's
    assert abs(_objective(oracle.solver, cfg, nodes, ucat, p, idx, u_obs, f0) - J) <= 1e-6 * J


def test_c4_gradient_mixed_precision_forward():
    cfg, nodes, ucat, p, idx, u_obs, f0 = _setup((128, 64, 64), precision=api.PREC_MIXED)
    J, grad, _, _ = _gradient(cfg, nodes, ucat, p, idx, u_obs, f0)
    v = np.random.default_rng(9).standard_normal(f0.shape) * np.abs(f0).max()
    eps = 1e-3
    Jp = _objective(tosca_b200.gpu_solver, cfg, nodes, ucat, p, idx, u_obs, f0 + eps * v)
    Jm = _objective(tosca_b200.gpu_solver, cfg, nodes, ucat, p, idx, u_obs, f0 - eps * v)
    fd = (Jp - Jm) / (2 * eps)
    ad = float((grad * v).sum())
    assert abs(ad - fd) <= 1e-3 * abs(fd), (ad, fd)
