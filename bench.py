"""Benchmark of the B200 TOSCA fractional time step.

Workload (default): the neutral pressure-driven ABL, 256 x 256 x 128 cells
(DMDA extent 258 x 130 x 258), RK4 momentum, Smagorinsky LES, Schumann wall
stress, slip top, periodic x/y, pressure solved until the divergence bound
dt * max|r aj| <= 5e-9 holds (ContinuityErrorsOptimized definition).
Synthetic seeded inputs (log-law + splitmix64 perturbations); every field is
larger than the 126 MB L2, so no flush is needed between steps.

One JSON line is printed by rank 0. `--impl reference` times the CPU
restatement of the reference step on the full workload (TOSCA's own stage
functions compile against single-rank stand-ins and pin the restatement, but
its MPI/PETSc/HYPRE runtime is absent); the `cpu_baseline` of the GPU line is
the same restatement on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s mixed vs FP64 GPU at div≤1e-8; adjoint/forward time ratio"
UNIT = "Mcell-steps/s"
DIV_TOL = 5e-9

# algorithmic bytes per interior cell of one launch, by storage precision of
# the arrays the kernel reads (each array counted once per read and once per
# write; metrics re-read every launch). The mixed mode reads FP32 copies of the
# metrics (4 B) and keeps the state, fluxes and Krylov vectors in FP64. On an
# axis-aligned mesh (tg_mesh_info) the stencil kernels read one component of
# each metric vector.
def bytes_per_cell(kernel, precision, axis=False):
    m = 4 if precision == "mixed" else 8      # metric storage
    g = 4 if precision == "mixed" else 8      # multigrid storage
    if axis:
        table = {
            # ucat 3, ucont 3, nut 1; per face the normal metric component of
            # csi, eta, zet and aj (12) -> fluxes 9
            "formu_face_fluxes": 7 * 8 + 12 * m + 9 * 8,
            # fp 3, dP 3, and the RK4 update applied in place (U_o, Utmp -> Utmp,
            # U: 9, 12, 12, 6 values over the four stages); csi.y, eta.z, zet.x,
            # face aj 3, icsi.y, jeta.z, kzet.x
            "formu_rhs_faces": (6 + 39 / 4) * 8 + 9 * m,
            # ucont 3 -> ucat 3; csi.y, eta.z, zet.x
            "contra_to_cart": 6 * 8 + 3 * m,
            # ucat 3 -> nut 1; csi.y, eta.z, zet.x, aj
            "smagorinsky": 4 * 8 + 4 * m,
            # p 1 -> dP 3; icsi.y, jeta.z, kzet.x and the face aj 3
            "grad_p": 4 * 8 + 6 * m,
            # phi 1, ucont 3 -> ucont 3; icsi.y, jeta.z, kzet.x and the face aj 3
            "project": 7 * 8 + 6 * m,
            # T 1, nut 1, ucont 3; icsi.y, jeta.z, kzet.x and the face aj 3 (FP64
            # in every mode) -> convective and diffusive fluxes 6
            "teqn_face_fluxes": (5 + 6 + 6) * 8,
        }
        if kernel in table:
            return table[kernel]
    table = {
        # ucat 3, ucont 3, nut 1 (FP64); face metrics 27 + face aj 3; -> fluxes 9 (FP64)
        "formu_face_fluxes": 7 * 8 + 30 * m + 9 * 8,
        # fluxes 9 -> fp 3
        "formu_cell_fp": 12 * 8,
        # fp 3, dP 3 and the RK4 update in place (9.75 values per stage, FP64);
        # csi/eta/zet 9, face aj 3, icsi/jeta/kzet 9 (metrics)
        "formu_rhs_faces": (6 + 39 / 4) * 8 + 21 * m,
        # ucont 3 -> ucat 3 (FP64); csi/eta/zet 9
        "contra_to_cart": 6 * 8 + 9 * m,
        # ucat 3 -> nut 1 (FP64); csi/eta/zet 9, aj 1
        "smagorinsky": 4 * 8 + 10 * m,
        # p 1 -> dP 3 (FP64); face metrics 27 + 3
        "grad_p": 4 * 8 + 30 * m,
        # phi 1, ucont 3 -> ucont 3 (FP64); face metrics 27 + 3
        "project": 7 * 8 + 30 * m,
        # one zebra colour (half the cells): r, minv, aN, c', aE, aT, x of the
        # other colour -> x: 8 values per cell of the colour
        "mg_smooth_line_L0": 8 * g / 2,
        # r, x, 3 coefficients -> coarse r (1/8 of the cells)
        "mg_restrict_L0": 5 * g + g / 8,
        # x read/write, coarse x (1/8)
        "mg_prolong_L0": 2 * g + g / 8,
        "pois_apply7": 5 * 8,          # x 1, 3 coefficients -> y 1
        "pois_apply19": 11 * 8,        # x 1, 9 coefficients -> y 1
        "pois_cg_update": 48,          # x, r read/write; p, q read
        "pois_cg_dir": 24,             # z, p read; p write
        "pois_dot": 16,                # two vectors
        # T 1, nut 1, ucont 3; face metrics 27 + 3 (FP64) -> fluxes 6
        "teqn_face_fluxes": (5 + 30 + 6) * 8,
    }
    return table.get(kernel)


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None
        self.skip = 0          # samples written before the region began

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        # nvidia-smi takes a moment to start: wait (at most 5 s) for its first
        # sample so that the sampling covers the region from its start; that
        # sample, taken before the region, is used only if no later one exists
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            with open(self.path) as f:
                n = sum(1 for _ in f)
            if n > 0:
                self.skip = n
                break
            time.sleep(0.02)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = open(self.path).read().splitlines()
        if len(lines) > self.skip:
            lines = lines[self.skip:]
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(name, precision, seed_offset=0, small=False, cells=None, ddt="rk4", open_x=False):
    from tosca_b200 import api, cases
    if name == "abl":
        kw = dict(nx=64, ny=64, nz=32, Lx=640.0, Ly=640.0, H=250.0) if small else {}
        if cells:
            nx, ny, nz = cells
            kw = dict(nx=nx, ny=ny, nz=nz, Lx=10.0 * nx, Ly=10.0 * ny, H=1000.0 * nz / 128.0)
        cfg, nodes, ucat, p = cases.abl_case(ddt=api.DDT_RK4, seed=20261203 + seed_offset, **kw)
        T = None
        desc = "ABL %dx%dx%d cells, RK4, Smagorinsky, Schumann wall, dt=0.25 s" % (
            cfg.mz - 2, cfg.mx - 2, cfg.my - 2)
    elif name == "sabl":
        kw = dict(nx=64, ny=64, nz=32, Lx=640.0, Ly=640.0, H=250.0) if small else {}
        if cells:
            nx, ny, nz = cells
            kw = dict(nx=nx, ny=ny, nz=nz, Lx=10.0 * nx, Ly=10.0 * ny, H=1000.0 * nz / 128.0)
        cfg, nodes, ucat, p, T = cases.stratified_abl_case(ddt=api.DDT_RK4, **kw)
        desc = ("stable ABL %dx%dx%d cells, RK4, Smagorinsky, Schumann wall with Monin-Obukhov stability, "
                "transported potential temperature (RK4, WENO3) with Boussinesq buoyancy and a "
                "Schumann-Grotzbach thetaWallFunction (surface cooling 0.25 K/h), dt=0.25 s" % (cfg.mz - 2, cfg.mx - 2, cfg.my - 2))
    elif name == "channel":
        kw = dict(nx=64, ny=64, nz=32, Lx=640.0, Ly=640.0, H=250.0) if small else dict(
            nx=256, ny=256, nz=128, Lx=2560.0, Ly=2560.0, H=1000.0)
        if cells:
            nx, ny, nz = cells
            kw = dict(nx=nx, ny=ny, nz=nz, Lx=10.0 * nx, Ly=10.0 * ny, H=1000.0 * nz / 128.0)
        cfg, nodes, ucat, p = cases.channel_case(ddt=api.DDT_RK4, seed=20261203 + seed_offset,
                                                 wall=api.BC_WALL_SHUMANN, **kw)
        T = None
        desc = ("open channel %dx%dx%d cells (the ABL grid): fixedValue inflow 8 m/s at x = 0, zeroGradient "
                "outflow at x = Lx (adjustFluxesLocal), RK4, Smagorinsky, Schumann wall, dt=0.25 s" % (
                    cfg.mz - 2, cfg.mx - 2, cfg.my - 2))
    elif name == "tgv":
        cfg, nodes, ucat, p = cases.tgv_case(32 if small else 64, ddt=api.DDT_RK4)
        T = None
        desc = "Taylor-Green vortex %d^3, RK4, dt=0.005" % (cfg.mx - 2)
    elif name == "hill":
        kw = dict(nx=48, ny=24, nz=24) if small else {}
        cfg, nodes, ucat, p, T = cases.hill_case(ddt=api.DDT_RK4, teqn=True, **kw)
        desc = ("cosine hill %dx%dx%d cells, QUICK, Smagorinsky, Schumann wall, Boussinesq buoyancy of the "
                "transported temperature (RK4, WENO3), RK4" % (cfg.mz - 2, cfg.mx - 2, cfg.my - 2))
    elif name == "farm":
        kw = (dict(nx=96, ny=64, nz=32, Lx=960.0, Ly=640.0, H=250.0, rows=2, cols=2, D=63.0, hub=60.0)
              if small else {})
        cfg, nodes, ucat, p, turbines = cases.farm_case(ddt=api.DDT_RK4, seed=20261203 + seed_offset, **kw)
        T = None
        desc = ("ABL %dx%dx%d cells with %d uniform actuator disks (C_T' %.3f, D %.0f m, %d points each), RK4, "
                "Smagorinsky, Schumann wall, dt=0.25 s" % (cfg.mz - 2, cfg.mx - 2, cfg.my - 2, len(turbines),
                                                          turbines[0].ct, 2 * turbines[0].r_tip,
                                                          turbines[0].n_radial * turbines[0].n_azimuth))
    else:
        raise SystemExit(f"unknown workload {name}")
    if name != "farm":
        turbines = None
    if open_x and name != "channel":
        # the inflow/outflow pair of TOSCA's hill and turbine decks
        # (CosineHillCurvTest, NREL5MWTest: kLeft fixedValue, kRight zeroGradient)
        cases.open_x(cfg, 8.0, None)
        desc += "; x open: fixedValue inflow 8 m/s, zeroGradient outflow (adjustFluxesLocal)"
    if ddt == "cn":                   # ddtScheme CN with the reference's SNES defaults (ueqn.c:128-130)
        cfg.ddt_scheme = api.DDT_CN
        cfg.snes_atol, cfg.snes_rtol, cfg.snes_maxit = 1e-5, 1e-30, 20
        desc = desc.replace("RK4", "Crank-Nicolson (JFNK, absTolU 1e-5)", 1)
    elif ddt in IMEX:                 # IMEX schemes with the reference's KSP defaults (ueqn.c:249-282)
        cfg.ddt_scheme = getattr(api, IMEX[ddt][0])
        cfg.snes_atol, cfg.snes_rtol, cfg.gmres_restart = 1e-5, 1e-30, 30
        desc = desc.replace("RK4", IMEX[ddt][1] + " (GMRES(30), absTolU 1e-5)", 1)
    cfg.poisson_rtol = 1e-30
    cfg.poisson_div_tol = DIV_TOL
    cfg.poisson_maxit = 400
    cfg.precision = api.PREC_MIXED if precision == "mixed" else api.PREC_FP64
    return cfg, nodes, ucat, p, T, desc, turbines


IMEX = {"abcn": ("DDT_ABCN", "ABCN IMEX"), "rk3wcn": ("DDT_RK3WCN", "RK3WCN IMEX"),
        "rk3socn": ("DDT_RK3SOCN", "RK3SOCN IMEX")}


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), or the platform string."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def cpu_baseline(workload, steps, full=False, cells=None, open_x=False):
    """CPU restatement of the reference step (the oracle, OpenMP on all host
    threads) on the workload: the full configuration (`full`), or a bounded
    sample of it (the ABL at 128 x 128 x 64 cells with the same 10 m spacing
    and aspect, the other workloads at their small size). The pressure solve
    is CG preconditioned by the oracle's aggregation multigrid (the reference
    uses HYPRE with BoomerAMG) to the reference's default poissonTol 1e-8; one
    untimed warm-up step builds the multigrid hierarchy."""
    import oracle
    from tosca_b200 import cases
    if full:
        cfg, nodes, ucat, p, T, desc, turbines = make_workload(workload, "fp64", cells=cells, open_x=open_x)
    elif workload == "abl":
        cfg, nodes, ucat, p, T, desc, turbines = make_workload(workload, "fp64", cells=(128, 128, 64), open_x=open_x)
    else:
        cfg, nodes, ucat, p, T, desc, turbines = make_workload(workload, "fp64", small=True, open_x=open_x)
    cfg.poisson_rtol = 1e-8          # the reference's default poissonTol (peqn.c:54)
    cfg.poisson_div_tol = 0.0
    cfg.poisson_maxit = 20000
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    if turbines:
        s.set_turbines(turbines, 1.225)
    s.step(1)                        # warm-up
    t0 = time.perf_counter()
    st = s.step(steps)
    dt = time.perf_counter() - t0
    cells = cfg.cells
    ncores = oracle.lib().tor_num_threads()
    s.close()
    return {
        "value": cells * steps / dt / 1e6, "unit": UNIT, "cores": int(ncores), "cpu_model": cpu_model(),
        "kind": "port",
        "sample": f"{desc}; {'the full configuration' if full else 'bounded sample'}; {steps} timed steps after "
                  f"1 warm-up; CG preconditioned by aggregation multigrid (V(1,1), j-line Gauss-Seidel) to the "
                  f"reference's poissonTol 1e-8, {st.poisson_iterations} iterations in the last step "
                  f"(oracle, OpenMP)",
        "seconds": dt, "max_divergence": st.max_divergence, "workload": desc, "cells": cells,
    }


def max_over_ranks_of(dist, x):
    """The largest of the ranks' values of x (device time of the timed steps):
    all_reduce(MAX) on the process group (a CUDA tensor under NCCL, a CPU one
    under gloo); x itself without a process group."""
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(cells, steps, world, seconds):
    """Whole-job Mcell-steps/s of `world` replicas that each advanced `cells`
    cells by `steps` steps, timed by the slowest rank."""
    return cells * steps * world / seconds / 1e6


def run_reference(args, rank, world):
    """The reference arm: the CPU restatement on the full workload (at most
    two timed steps: about 10 to 30 s each on 16 host threads at the ABL's
    8.4 M cells), rank 0 only."""
    if rank != 0:
        return 0
    steps = max(1, min(args.steps, 2))
    base = cpu_baseline(args.workload, steps, full=True, cells=args.cells, open_x=args.open_x)
    line = {
        "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
        "warmup": 1, "ms_per_step": base["seconds"] / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": base["workload"], "cells": base["cells"]},
        "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "cpu_model", "kind", "sample")},
        "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("TOSCA's own stage functions compile from its sources against single-rank PETSc/HYPRE/MPI "
                 "stand-ins (oracle/_ref) and pin the restatement to round-off, but its MPI, PETSc 3.15 and "
                 "HYPRE 2.20 runtime is absent, so the timed arm is the OpenMP restatement of the step"),
    }
    print(json.dumps(line), flush=True)
    return 0


def adjoint_ratio(dev, steps=20, warmup=8, cells=(128, 64, 64)):
    """Adjoint/forward time on the adjoint configuration: ABL 128 x 64 x 64
    cells, Cartesian, Schumann wall function, Smagorinsky, RK4, 3-D body force;
    objective J = sum (u - u_obs)^2 over the 64 x 64 hub-height probe plane
    after `steps` steps (u_obs from a run with a seeded body-force
    perturbation, seed 4). Device time of tg_step per step against the device
    time per step of tg_adjoint_reverse seeded with dJ/dUcat: (a) every step's
    tape kept (no forward step in the reversal), (b) the segment schedule
    (a snapshot every 10 steps, each segment re-run taped once in the
    reversal), (c) binomial checkpointing with half as many snapshots as steps
    and no tapes (each reversed step re-runs its forward step to record the
    stages, plus the schedule's recomputation)."""
    import tosca_b200
    from tosca_b200 import api, cases
    nx, ny, nz = cells
    cfg, nodes, ucat, p = cases.abl_case(nx=nx, ny=ny, nz=nz, Lx=10.0 * nx, Ly=10.0 * ny, H=1000.0 * nz / 128.0,
                                         ddt=api.DDT_RK4)
    cfg.poisson_rtol = 1e-30
    cfg.poisson_div_tol = DIV_TOL
    cfg.poisson_maxit = 400
    cfg.source = 1
    cfg.device = dev
    # probe plane: the j-plane of cell centres nearest 90 m, every second x cell, every y cell
    zc = 0.5 * (nodes[0, :-2, 0, 2] + nodes[0, 1:-1, 0, 2])
    jh, ks, is_ = 1 + int(np.argmin(np.abs(zc - 90.0))), np.arange(1, cfg.mz - 1, 2), np.arange(1, cfg.mx - 1)

    def start(f):
        s = tosca_b200.gpu_solver(cfg)
        cases.setup(s, nodes, ucat, p)
        s.set("SOURCE", f)
        s.step(warmup)
        return s

    rng = np.random.default_rng(4)
    f_obs = rng.standard_normal(ucat.shape) * 1e-3
    f0 = np.random.default_rng(21).standard_normal(ucat.shape) * 1e-3
    s = start(f_obs)
    s.step(steps)
    u_obs = s.get("UCAT")[ks][:, jh][:, is_, 0]
    s.close()
    s = start(f0)
    x0 = {k: s.get(k) for k in ("UCONT", "UCAT", "P")}
    fwd = s.step(steps)
    for k, v in x0.items():
        s.set(k, v)
    out = {"workload": "adjoint ABL %dx%dx%d cells, RK4, Smagorinsky, Schumann wall function, body force, FP64; "
                       "J = hub-height 64x64 probe misfit after %d steps" % (nx, ny, nz, steps),
           "forward_ms_per_step": fwd.seconds / steps * 1e3, "steps": steps,
           "forward_poisson_iterations_per_step": fwd.poisson_total_iterations / steps}
    # (a) every tape kept; (b) snapshots every 10 steps, the tapes of one
    # segment re-recorded in the reversal (each step re-run once); (c) the
    # binomial schedule over half as many snapshots as steps, no tapes. A first
    # untimed pass captures the reversal's CUDA graphs.
    for key, nsnap, tapes in (("warmup", steps, -1), ("tapes_kept", steps, -1), ("segments", max(1, steps // 10), 10),
                              ("checkpointed", max(1, steps // 2), 0)):
        s.adjoint_set_tapes(tapes)
        tst = s.adjoint_forward(steps, nsnap)
        u = s.get("UCAT")
        seed = np.zeros(ucat.shape)
        seed[np.ix_(ks, [jh], is_, [0])] = 2.0 * (u[np.ix_(ks, [jh], is_, [0])] - u_obs[:, None, :, None])
        J = float(((u[ks][:, jh][:, is_, 0] - u_obs) ** 2).sum())
        s.set("UCAT_ADJ", seed)
        s.set("UCONT_ADJ", np.zeros(ucat.shape)); s.set("P_ADJ", np.zeros(p.shape)); s.set("SOURCE_ADJ", np.zeros(ucat.shape))
        s.set("WALL_ADJ", np.zeros((cfg.mz, cfg.mx, 3)))
        ast = s.adjoint_reverse()
        a_ms = ast.seconds / steps * 1e3
        g = s.get("SOURCE_ADJ")
        if key == "warmup":
            continue
        out[key] = {"snapshots": int(ast.snapshots), "forward_steps_in_reversal": int(ast.forward_steps),
                    "adjoint_poisson_iterations_per_step": ast.poisson_iterations / steps,
                    "taped_forward_ms_per_step": tst.seconds / steps * 1e3,
                    "adjoint_ms_per_step": a_ms, "adjoint_over_forward": a_ms / out["forward_ms_per_step"],
                    "J": J, "grad_norm": float(np.linalg.norm(g))}
    s.close()
    out["adjoint_over_forward"] = out["tapes_kept"]["adjoint_over_forward"]
    out["adjoint_over_forward_segments"] = out["segments"]["adjoint_over_forward"]
    out["adjoint_over_forward_checkpointed"] = out["checkpointed"]["adjoint_over_forward"]
    return out


def farm_adjoint(dev, precision, steps, warmup=5, fwd_steps=10):
    """Gradient of the farm power summed over `steps` steps with respect to the
    turbines' C_T' (tg_set_farm_objective) on the farm workload (Schumann wall
    function on the ground), forward in
    `precision`: tg_adjoint_forward offered as many device snapshots as half
    the free HBM holds (the library then takes the segment schedule when the
    tapes of a segment fit beside them: a snapshot per segment, each segment
    re-run once taped in the reversal; binomial checkpointing otherwise),
    then tg_adjoint_reverse from zero adjoint fields. Device time per reversed
    step against the device time of a plain step of the same solver."""
    import torch
    import tosca_b200
    from tosca_b200 import api, cases
    cfg, nodes, ucat, p, turbines = cases.farm_case(ddt=api.DDT_RK4)
    cfg.poisson_rtol = 1e-30
    cfg.poisson_div_tol = DIV_TOL
    cfg.poisson_maxit = 400
    cfg.precision = api.PREC_MIXED if precision == "mixed" else api.PREC_FP64
    cfg.device = dev
    solver = tosca_b200.gpu_solver(cfg)
    cases.setup(solver, nodes, ucat, p)
    solver.set_turbines(turbines, 1.225)
    solver.step(warmup)
    fwd_ms = solver.step(fwd_steps).seconds / fwd_steps * 1e3
    free, _ = torch.cuda.mem_get_info()
    G = cfg.mx * cfg.my * cfg.mz
    snap = 8 * (7 * G + 3 * cfg.cells)               # Ucont, Ucat, P and the last three Poisson solutions
    work = 8 * (49 + 31) * G                       # adjoint work arrays and the work tape
    nsnap = int(max(2, min(steps, 0.5 * (free - work) // snap)))
    solver.set_farm_objective(True)
    solver.ct_gradient(reset=True)
    solver.turbine_state(reset=True)
    fw = solver.adjoint_forward(steps, nsnap)
    J = solver.turbine_state()["power_sum"]
    shape = (cfg.mz, cfg.my, cfg.mx)
    for k in ("UCONT_ADJ", "UCAT_ADJ", "SOURCE_ADJ"):
        solver.set(k, np.zeros(shape + (3,)))
    solver.set("P_ADJ", np.zeros(shape))
    solver.set("WALL_ADJ", np.zeros((cfg.mz, cfg.mx, 3)))
    rv = solver.adjoint_reverse()
    g = solver.ct_gradient()
    solver.close()
    adj_ms = rv.seconds / steps * 1e3
    return {"workload": "farm workload (Schumann wall function), %s forward" % precision, "steps": steps, "snapshots": int(rv.snapshots), "forward_steps_in_reversal": int(rv.forward_steps),
            "recorded_forward_ms_per_step": fw.seconds / steps * 1e3, "adjoint_ms_per_step": adj_ms,
            "forward_ms_per_step": fwd_ms, "adjoint_over_forward": adj_ms / fwd_ms,
            "adjoint_poisson_iterations_per_step": rv.poisson_iterations / steps,
            "objective": "farm power summed over the steps (W)", "J": J,
            "dJ_dCt": [float(v) for v in g]}


def kernel_table(L, h):
    import ctypes
    kernels = {}
    nb = ctypes.create_string_buffer(64)
    for q in range(L.tg_prof_count(h)):
        n = ctypes.c_int64()
        ms = ctypes.c_double()
        L.tg_prof_get(h, q, nb, ctypes.byref(n), ctypes.byref(ms))
        kernels[nb.value.decode()] = {"launches": int(n.value), "ms": float(ms.value)}
    total = sum(v["ms"] for v in kernels.values())
    for v in kernels.values():
        v["share"] = v["ms"] / total if total > 0 else 0.0
    return kernels


def roofline_of(kernels, precision, cells, axis=False):
    """Roofline of the dominant kernel with a known byte count: algorithmic
    bytes per launch / average launch time (library events on its stream)."""
    ranked = sorted(kernels.items(), key=lambda kv: -kv[1]["ms"])
    dom = next((k for k, v in ranked if bytes_per_cell(k, precision, axis) is not None), None)
    if dom is None:
        return None
    peak, peak_src = load_peaks()
    kv = kernels[dom]
    per_launch_ms = kv["ms"] / kv["launches"]
    algo_bytes = bytes_per_cell(dom, precision, axis) * cells
    achieved = algo_bytes / (per_launch_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_per_cell.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f).get(precision + ("_axis" if axis else ""), {})
        if dom in tj:
            traffic = tj[dom] * cells
    return {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
            "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
            "algorithmic_bytes_per_launch": algo_bytes, "avg_launch_ms": per_launch_ms,
            "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else peak_src)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="abl", choices=["abl", "tgv", "hill", "farm", "sabl", "channel"])
    ap.add_argument("--open-x", action="store_true",
                    help="replace the periodic x direction by a fixedValue inflow and a zeroGradient outflow")
    ap.add_argument("--ddt", default="rk4", choices=["rk4", "cn", "abcn", "rk3wcn", "rk3socn"], help="momentum time scheme of the workload")
    ap.add_argument("--farm-adjoint-steps", type=int, default=200,
                    help="farm workload: steps of the C_T' gradient of the summed farm power")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="both: the mixed step is the headline value, the FP64 step is timed beside it")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--profile-steps", type=int, default=2,
                    help="untimed steps after the timed region with per-kernel events on")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward timing")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--profile-json", default=None, help="write per-kernel timings here (one file per arm)")
    ap.add_argument("--cells", type=int, nargs=3, default=None, metavar=("NX", "NY", "NZ"),
                    help="override the ABL size (profiling captures of a smaller case)")
    args = ap.parse_args()

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import ctypes
    import torch
    import tosca_b200
    from tosca_b200 import cases

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    L = ctypes.CDLL(tosca_b200.LIB_PATH)
    L.tg_prof_enable.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.tg_prof_reset.argtypes = [ctypes.c_void_p]
    L.tg_prof_count.argtypes = [ctypes.c_void_p]
    L.tg_prof_count.restype = ctypes.c_int32
    L.tg_prof_get.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_char_p,
                              ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)]

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return max_over_ranks_of(dist, x)

    def arm(precision):
        cfg, nodes, ucat, p, T, desc, turbines = make_workload(args.workload, precision, seed_offset=rank, cells=args.cells,
                                                               ddt=args.ddt, open_x=args.open_x)
        cfg.device = dev
        solver = tosca_b200.gpu_solver(cfg)
        cases.setup(solver, nodes, ucat, p, T)
        axis = solver.mesh_info()[1]
        if turbines:
            solver.set_turbines(turbines, 1.225)
        if args.warmup > 0:
            solver.step(args.warmup)
        # timed region: device time between events on the library's stream
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(dev) as clk:
            r0 = solver.graph_info()[0]
            st = solver.step(args.steps)
            torch.cuda.synchronize()
        barrier()
        replayed = solver.graph_info()[0] - r0
        mom = solver.momentum_info()
        t_dev = max_over_ranks(st.seconds)
        # per-kernel events on a few further steps (outside the timed region)
        L.tg_prof_reset(solver.h)
        L.tg_prof_enable(solver.h, 1)
        solver.step(args.profile_steps)
        torch.cuda.synchronize()
        L.tg_prof_enable(solver.h, 0)
        kernels = kernel_table(L, solver.h)
        return {"cfg": cfg, "desc": desc, "solver": solver, "st": st, "t_dev": t_dev, "clocks": clk.summary(),
                "replayed": replayed, "momentum": mom,
                "value": replica_throughput(cfg.cells, args.steps, world, t_dev), "kernels": kernels,
                "roofline": roofline_of(kernels, precision, cfg.cells, axis), "axis_aligned": axis}

    arms = {}
    order = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    for prec in order:
        arms[prec] = arm(prec)
    head_prec = order[-1]
    head = arms[head_prec]
    cfg, cells = head["cfg"], head["cfg"].cells

    # mixed against FP64 after the same number of steps from the same state
    field_err = None
    if len(arms) == 2:
        def rel(a, b):
            a, b = a[1:-1, 1:-1, 1:-1], b[1:-1, 1:-1, 1:-1]
            d = float(np.linalg.norm(b.ravel()))
            return float(np.linalg.norm((a - b).ravel()) / d) if d > 0 else float(np.linalg.norm(a.ravel()))
        ua, ub = arms["mixed"]["solver"].get("UCAT"), arms["fp64"]["solver"].get("UCAT")
        field_err = {"u": rel(ua[..., 0], ub[..., 0]), "v": rel(ua[..., 1], ub[..., 1]),
                     "w": rel(ua[..., 2], ub[..., 2]),
                     "p": rel(arms["mixed"]["solver"].get("P"), arms["fp64"]["solver"].get("P")),
                     "steps": args.warmup + args.steps + args.profile_steps,
                     "against": "FP64 GPU step (itself within 1e-10 of the FP64 oracle in the parity tests)"}
        arms["fp64"]["solver"].close()

    # end-to-end through the C-ABI with host buffers (drop-in call per step)
    solver = head["solver"]
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else max(2, args.steps // 2)
    mz, my, mx = cfg.mz, cfg.my, cfg.mx
    h_ucont = torch.empty((mz, my, mx, 3), dtype=torch.float64, pin_memory=True).numpy()
    h_ucat = torch.empty((mz, my, mx, 3), dtype=torch.float64, pin_memory=True).numpy()
    h_p = torch.empty((mz, my, mx), dtype=torch.float64, pin_memory=True).numpy()
    h_nut = torch.empty((mz, my, mx), dtype=torch.float64, pin_memory=True).numpy()
    h_ucont[...] = solver.get("UCONT")
    h_ucat[...] = solver.get("UCAT")
    h_p[...] = solver.get("P")
    h_nut[...] = solver.get("NUT")
    nut_arg = h_nut if cfg.les else None
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        se = solver.step_host(h_ucont, h_ucat, h_p, nut_arg)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    barrier()
    bytes_in = h_ucont.nbytes + h_ucat.nbytes + h_p.nbytes          # nut is output only
    bytes_out = bytes_in + (h_nut.nbytes if cfg.les else 0)
    # what bounds it: the step's device time against the wall time per call;
    # the rest is the exposed host<->device copies (and the layout
    # conversions): nut's copy overlaps the step, so it is not counted there
    e2e_ms = t_e2e / e2e_steps * 1e3
    dev_ms = head["t_dev"] / args.steps * 1e3
    copy_ms = max(e2e_ms - dev_ms, 1e-9)
    e2e = {"value": cells * e2e_steps * world / t_e2e / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": int(bytes_in), "d2h_bytes_per_step": int(bytes_out),
           "steps": e2e_steps, "precision": head_prec, "max_divergence": se.max_divergence,
           "ms_per_step": e2e_ms, "device_step_ms": dev_ms, "transfer_ms_per_step": copy_ms,
           "transfer_gbs": (bytes_in + bytes_out) / (copy_ms * 1e-3) / 1e9,
           "limiter": "host<->device copies of the state (PCIe), %.0f %% of the call" % (100.0 * copy_ms / e2e_ms)}

    adj = None
    if rank == 0 and not args.no_adjoint and args.workload == "abl":
        adj = adjoint_ratio(dev)
    farm_adj = None
    if rank == 0 and not args.no_adjoint and args.workload == "farm" and args.farm_adjoint_steps > 0:
        solver.close()                               # its HBM goes to the checkpoints
        farm_adj = farm_adjoint(dev, head_prec, args.farm_adjoint_steps)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(args.workload, args.cpu_steps, open_x=args.open_x)
        cpu = {k: base[k] for k in ("value", "unit", "cores", "cpu_model", "kind", "sample")}

    if rank == 0:
        st = head["st"]
        kernels = head["kernels"]
        ranked = sorted(kernels.items(), key=lambda kv: -kv[1]["ms"])
        launches_per_step = sum(v["launches"] for v in kernels.values()) / max(1, args.profile_steps)
        line = {
            "metric": METRIC, "value": round(head["value"], 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["t_dev"] / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if head_prec == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": head["desc"], "cells": cells, "dmda_extent": [mx, my, mz],
                       "precision": head_prec, "divergence_bound": DIV_TOL,
                       "l2": "every field exceeds the 126 MB L2; no flush",
                       "mesh_axis_aligned": head["axis_aligned"],
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "poisson_iterations_per_step": st.poisson_total_iterations / max(1, args.steps),
                       "max_divergence": st.max_divergence,
                       "steps_replayed_from_cuda_graph": head["replayed"]},
            "clocks": head["clocks"],
            "e2e": e2e,
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "gpu_launches_note": "per-step count of the library's timed launches in the profiled steps x timed steps",
            "roofline": head["roofline"],
            "adjoint": adj,
            "farm_adjoint": farm_adj,
            "cpu_baseline": cpu,
            "kernels_top": {k: {"ms_per_step": round(v["ms"] / max(1, args.profile_steps), 3),
                                "launches_per_step": v["launches"] / max(1, args.profile_steps),
                                "share": round(v["share"], 4)} for k, v in ranked[:12]},
        }
        if args.ddt != "rk4":
            o, k, r = head["momentum"]
            line["config"]["momentum_solve_last_step"] = {
                "newton_steps" if args.ddt == "cn" else "stages": o, "krylov_operator_products": k, "last_residual": r}
        if "fp64" in arms and head_prec != "fp64":
            a = arms["fp64"]
            line["fp64"] = {"value": round(a["value"], 3), "ms_per_step": a["t_dev"] / args.steps * 1e3,
                            "poisson_iterations_per_step": a["st"].poisson_total_iterations / max(1, args.steps),
                            "max_divergence": a["st"].max_divergence, "clocks": a["clocks"],
                            "roofline": a["roofline"]}
            line["mixed_over_fp64"] = round(head["value"] / a["value"], 4)
            line["mixed_field_error"] = field_err
        print(json.dumps(line), flush=True)
        if args.profile_json:
            for prec, a in arms.items():
                path = args.profile_json if len(arms) == 1 else args.profile_json.replace(".json", "_%s.json" % prec)
                with open(path, "w") as f:
                    json.dump({"kernels": a["kernels"], "cells": a["cfg"].cells, "steps": args.profile_steps,
                               "precision": prec}, f, indent=1)
    solver.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
