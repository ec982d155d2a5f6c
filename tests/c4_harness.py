"""Test harness of the adjoint configuration: the gradient of a hub-height
velocity misfit with respect to a 3-D body force, through the C-ABI.

Workload (ABL 128 x 64 x 64 cells, Cartesian, Schumann wall function,
Smagorinsky, RK4, 20 steps): J = sum over a 64 x 64 probe plane of
(u - u_obs)^2, with u the streamwise Ucat component at the cell centres of
the DMDA j-plane nearest to hub height (90 m), every second x-cell (DMDA k)
and every y-cell (DMDA i); u_obs is the same probe plane after the same 20
steps driven by a seeded perturbation of the body force (seed 4).

`StepsFunction` wraps the CUDA solver in a torch.autograd.Function: forward
runs the steps with binomial checkpointing (tg_adjoint_forward) and returns
the final Ucat; backward seeds the Ucat adjoint with the incoming gradient,
reverses the steps (tg_adjoint_reverse) and returns the gradient with respect
to the body force (TG_F_SOURCE_ADJ). It is a test harness: the solver itself
is driven through the C-ABI, not through torch."""
from __future__ import annotations

import numpy as np
import torch

from tosca_b200 import api, cases

HUB = 90.0


def c4_case(nx=128, ny=64, nz=64, ddt=api.DDT_RK4, precision=api.PREC_FP64, rtol=1e-13):
    """The adjoint ABL scaled from the 256 x 256 x 128 one (10 m in x and y,
    H = 1000 m * nz / 128), with its wall function and a body force channel."""
    cfg, nodes, ucat, p = cases.abl_case(nx=nx, ny=ny, nz=nz, Lx=10.0 * nx, Ly=10.0 * ny, H=1000.0 * nz / 128.0,
                                         ddt=ddt)
    cfg.source = 1
    cfg.poisson_rtol = rtol
    cfg.precision = precision
    return cfg, nodes, ucat, p


def probe_index(nodes, cfg):
    """(j_hub, k cells, i cells) of the probe plane."""
    zc = 0.5 * (nodes[0, :-2, 0, 2] + nodes[0, 1:-1, 0, 2])      # centre height of the cells j = 1 .. my-2
    j_hub = 1 + int(np.argmin(np.abs(zc - HUB)))
    ks = np.arange(1, cfg.mz - 1, 2)
    is_ = np.arange(1, cfg.mx - 1)
    return j_hub, ks, is_


def probes(ucat, idx):
    j, ks, is_ = idx
    return ucat[ks][:, j][:, is_, 0]


def body_force(shape, seed, scale=1e-3):
    return np.random.default_rng(seed).standard_normal(shape) * scale


class StepsFunction(torch.autograd.Function):
    """Ucat after `nsteps` steps of `solver` from the state `x0`, as a function
    of the body force f (float64 CPU tensor, DMDA shape (mz, my, mx, 3))."""

    @staticmethod
    def forward(ctx, f, solver, x0, nsteps, nsnap):
        for k, v in x0.items():
            solver.set(k, v)
        solver.set("SOURCE", f.detach().numpy())
        solver.adjoint_forward(nsteps, nsnap)
        ctx.solver = solver
        ctx.shape = tuple(f.shape)
        return torch.from_numpy(solver.get("UCAT"))

    @staticmethod
    def backward(ctx, grad_ucat):
        s = ctx.solver
        zeros = np.zeros(ctx.shape)
        s.set("UCAT_ADJ", np.ascontiguousarray(grad_ucat.detach().numpy()))
        s.set("UCONT_ADJ", zeros)
        s.set("P_ADJ", zeros[..., 0].copy())
        s.set("SOURCE_ADJ", zeros)
        if s.cfg.bc[2] == api.BC_WALL_SHUMANN and s.cfg.les:
            s.set("WALL_ADJ", np.zeros((s.cfg.mz, s.cfg.mx, 3)))
        s.adjoint_reverse()
        return torch.from_numpy(s.get("SOURCE_ADJ")), None, None, None, None


def misfit(ucat_t: torch.Tensor, idx, u_obs: np.ndarray) -> torch.Tensor:
    j, ks, is_ = idx
    u = ucat_t[torch.as_tensor(ks)][:, j][:, torch.as_tensor(is_), 0]
    return ((u - torch.as_tensor(u_obs)) ** 2).sum()
