"""Input generators for the workloads: grid nodes in TOSCA's DMDA layout,
initial fields and configurations.

Axis mapping (mesh.c:92-94): DMDA i <-> physical y, j <-> physical z,
k <-> physical x. A grid of nx x ny x nz cells therefore has the DMDA extent
(mx, my, mz) = (ny+2, nz+2, nx+2); node (k, j, i) sits at DMDA point (k, j, i)
for k < mz-1, j < my-1, i < mx-1 and the last point of each direction carries
no node (mesh.c:190-290).

Workloads (synthetic, seeded; no dataset is involved):
  tgv        Taylor-Green vortex, [0,2pi]^3, all-periodic, central, no LES
  abl        neutral pressure-driven ABL: periodic x/y, Schumann wall function
             (type -3) at the ground, slip top, Smagorinsky, tanh-stretched z
  hill       terrain-following mesh over a 2-D cosine hill, QUICK, stable
             Boussinesq stratification, frozen or transported temperature
  farm       abl with uniform actuator disks
  sabl       stratified abl: transported potential temperature with Boussinesq
             buoyancy and a thetaWallFunction at the ground (thermal_wall)
"""
from __future__ import annotations

import math

import numpy as np

from .api import (BC_FIXED_VALUE, BC_INLET_LOG, BC_NOSLIP, BC_PERIODIC, BC_SLIP, BC_WALL_SHUMANN, BC_ZERO_GRADIENT, DDT_FE,
                  DDT_RK4, DIV_CENTRAL, DIV_QUICK, NUTBC_FIXEDVALUE, NUTBC_PERIODIC, NUTBC_ZEROGRADIENT, TBC_FIXED_GRADIENT, TBC_FIXED_VALUE, TBC_PERIODIC, TBC_WALL_FUNCTION,
                  TBC_ZERO_GRADIENT, TWALL_FIXED_FLUX, TWALL_SHUMANN, Config)


# --------------------------------------------------------------------- grids
def cartesian_nodes(X: np.ndarray, Y: np.ndarray, Z: np.ndarray) -> np.ndarray:
    """Nodes of a Cartesian grid from its 1-D node coordinates (mesh.c:70-95,
    'cartesian' mesh file). Returns (mz, my, mx, 3)."""
    nx, ny, nz = len(X), len(Y), len(Z)
    mx, my, mz = ny + 1, nz + 1, nx + 1
    nodes = np.zeros((mz, my, mx, 3))
    nodes[: mz - 1, : my - 1, : mx - 1, 0] = X[:, None, None]
    nodes[: mz - 1, : my - 1, : mx - 1, 1] = Y[None, None, :]
    nodes[: mz - 1, : my - 1, : mx - 1, 2] = Z[None, :, None]
    return nodes


def tanh_stretch(n: int, H: float, dz1: float, max_ratio: float = 1.05) -> np.ndarray:
    """n+1 nodes on [0, H] clustered at 0 by z = H(1 - tanh(d(1-s))/tanh(d)).
    d is the clustering that gives a first spacing of dz1, reduced if needed so
    that the largest ratio of consecutive spacings stays <= max_ratio."""
    s = np.linspace(0.0, 1.0, n + 1)

    def nodes(d):
        return H * (1.0 - np.tanh(d * (1.0 - s)) / math.tanh(d))

    def ratio(d):
        dz = np.diff(nodes(d))
        return float(np.max(dz[1:] / dz[:-1]))

    def bisect(pred):
        # largest d in (0, 30] with pred(d) true (pred is monotone: true for small d)
        lo, hi = 1e-6, 30.0
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if pred(mid):
                lo = mid
            else:
                hi = mid
        return lo

    d = min(bisect(lambda dd: nodes(dd)[1] >= dz1), bisect(lambda dd: ratio(dd) <= max_ratio))
    z = nodes(d)
    z[0], z[-1] = 0.0, H
    return z


def cell_centres(nodes: np.ndarray) -> np.ndarray:
    """8-node average at interior cells (mesh.c:713-743); zero elsewhere."""
    mz, my, mx, _ = nodes.shape
    c = np.zeros_like(nodes)
    n = nodes
    c[1:-1, 1:-1, 1:-1] = 0.125 * (
        n[1:-1, 1:-1, 1:-1] + n[1:-1, :-2, 1:-1] + n[:-2, 1:-1, 1:-1] + n[:-2, :-2, 1:-1]
        + n[1:-1, 1:-1, :-2] + n[1:-1, :-2, :-2] + n[:-2, 1:-1, :-2] + n[:-2, :-2, :-2])
    return c


def hill_nodes(nx: int, ny: int, nz: int, Lx: float = 6000.0, Ly: float = 3000.0, H: float = 1500.0,
               h0: float = 100.0, half_width: float = 500.0, dz1: float = 3.0) -> np.ndarray:
    """Terrain-following grid over a 2-D cosine hill centred in x:
    h(x) = h0/2 (1 + cos(pi (x-xc) / (2 L))) for |x-xc| < 2L (L = half-width at
    half height), z = h(x) + zeta (H - h(x)) / H with zeta tanh-stretched."""
    X = np.linspace(0.0, Lx, nx + 1)
    Y = np.linspace(0.0, Ly, ny + 1)
    zeta = tanh_stretch(nz, H, dz1)
    xc = 0.5 * Lx
    r = X - xc
    h = np.where(np.abs(r) < 2 * half_width, 0.5 * h0 * (1.0 + np.cos(np.pi * r / (2 * half_width))), 0.0)
    mx, my, mz = ny + 2, nz + 2, nx + 2
    nodes = np.zeros((mz, my, mx, 3))
    zz = h[:, None] + zeta[None, :] * (H - h[:, None]) / H          # (nx+1, nz+1)
    nodes[: mz - 1, : my - 1, : mx - 1, 0] = X[:, None, None]
    nodes[: mz - 1, : my - 1, : mx - 1, 1] = Y[None, None, :]
    nodes[: mz - 1, : my - 1, : mx - 1, 2] = zz[:, :, None]
    return nodes


# ------------------------------------------------------------------- noise
_M64 = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser on uint64 arrays (Steele, Lea, Flood 2014)."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform_noise(seed: int, n: int, stream: int) -> np.ndarray:
    """n deterministic uniforms in [-1, 1) for (seed, stream, global index)."""
    idx = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        key = idx * np.uint64(3) + np.uint64(stream) + np.uint64(seed) * np.uint64(0x632BE59BD9B4E019)
    r = splitmix64(key)
    return (r >> np.uint64(11)).astype(np.float64) * (2.0 / 2.0 ** 53) - 1.0


# -------------------------------------------------------------------- cases
def tgv_case(n: int = 64, ddt: int = DDT_FE, dt: float = 0.005, nu: float = 1.0 / 1600.0):
    """Taylor-Green vortex on [0,2pi]^3 with n^3 cells; initial fields as
    SetTaylorGreenFieldU/P (initialField.c:1061-1204, 1959-2030) with the
    pressure p = (cos2x + cos2y)(cos2z + 2)/16 (unit density)."""
    L = 2.0 * math.pi
    X = np.linspace(0.0, L, n + 1)
    nodes = cartesian_nodes(X, X.copy(), X.copy())
    cfg = Config(mx=n + 2, my=n + 2, mz=n + 2, bc=(BC_PERIODIC,) * 6, les=0, nu=nu,
                 div_scheme=DIV_CENTRAL, ddt_scheme=ddt, dt=dt)
    cent = cell_centres(nodes)
    x, y, z = cent[..., 0], cent[..., 1], cent[..., 2]
    ucat = np.zeros_like(cent)
    ucat[..., 0] = np.sin(x) * np.cos(y) * np.cos(z)
    ucat[..., 1] = -np.cos(x) * np.sin(y) * np.cos(z)
    p = np.zeros(cent.shape[:3])
    p[1:-1, 1:-1, 1:-1] = ((np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0)[1:-1, 1:-1, 1:-1]
    interior = np.zeros(cent.shape[:3], bool)
    interior[1:-1, 1:-1, 1:-1] = True
    ucat[~interior] = 0.0
    return cfg, nodes, ucat, p


def abl_case(nx: int = 256, ny: int = 256, nz: int = 128, Lx: float = 2560.0, Ly: float = 2560.0,
             H: float = 1000.0, dz1: float = 2.0, ustar: float = 0.4, z0: float = 0.1,
             kappa: float = 0.4, cs: float = 0.01, nu: float = 1.5e-5, dt: float = 0.25,
             ddt: int = DDT_FE, seed: int = 20261203, amp: float = 0.05, wall: int = BC_WALL_SHUMANN):
    """Neutral pressure-driven ABL on a tanh-clustered vertical grid (first
    cell dz1, largest consecutive spacing ratio <= 1.05). Log-law initial profile u = (u*/kappa)
    ln(z/z0) with seeded uniform +-amp perturbations: Ucat = U(z)(1+e_x, e_y,
    e_z), e from splitmix64 over (seed, component, global cell index). Mean
    pressure gradient u*^2/H drives the flow (meanGradPForcing,
    ueqn_sources.c:3735-3822). `wall` is the bottom patch type: the Schumann
    wall function, or noSlip for the adjoint configuration."""
    X = np.linspace(0.0, Lx, nx + 1)
    Y = np.linspace(0.0, Ly, ny + 1)
    Z = tanh_stretch(nz, H, dz1)
    nodes = cartesian_nodes(X, Y, Z)
    mx, my, mz = ny + 2, nz + 2, nx + 2
    cfg = Config(mx=mx, my=my, mz=mz,
                 bc=(BC_PERIODIC, BC_PERIODIC, wall, BC_SLIP, BC_PERIODIC, BC_PERIODIC),
                 nut_bc=(NUTBC_PERIODIC, NUTBC_PERIODIC, NUTBC_FIXEDVALUE, NUTBC_FIXEDVALUE, NUTBC_PERIODIC, NUTBC_PERIODIC),
                 les=1, cs=cs, nu=nu, div_scheme=DIV_CENTRAL, ddt_scheme=ddt, dt=dt,
                 mean_grad_p=1, mean_grad_p_value=(ustar * ustar / H, 0.0, 0.0),
                 wall_roughness=z0, wall_kappa=kappa)
    cent = cell_centres(nodes)
    zc = np.maximum(cent[..., 2], z0 * 1.0001)
    U = (ustar / kappa) * np.log(zc / z0)
    G = mx * my * mz
    e = [uniform_noise(seed, G, s).reshape(mz, my, mx) * amp for s in range(3)]
    ucat = np.zeros_like(cent)
    ucat[..., 0] = U * (1.0 + e[0])
    ucat[..., 1] = U * e[1]
    ucat[..., 2] = U * e[2]
    interior = np.zeros((mz, my, mx), bool)
    interior[1:-1, 1:-1, 1:-1] = True
    ucat[~interior] = 0.0
    p = np.zeros((mz, my, mx))
    return cfg, nodes, ucat, p


def channel_case(nx: int = 256, ny: int = 128, nz: int = 64, Lx: float = 2560.0, Ly: float = 1280.0,
                 H: float = 500.0, u_in: float = 8.0, wall: int = BC_NOSLIP, **kw):
    """Open channel with an inflow and an outflow (flow along +x, the k
    direction): a fixedValue patch (BC_FIXED_VALUE, uniform Cartesian
    velocity (u_in, 0, 0)) at x = 0, a zeroGradient outflow patch
    (BC_ZERO_GRADIENT) at x = Lx, the bottom patch `wall` (noSlip or the
    Schumann wall function), slip top, periodic y; zero-gradient nut on the
    inflow and outflow patches, no mean pressure gradient. Grid and initial
    field as abl_case."""
    cfg, nodes, ucat, p = abl_case(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, H=H, wall=wall, **kw)
    open_x(cfg, u_in)
    return cfg, nodes, ucat, p


def log_inlet(cfg: Config, u_tau: float = 0.4, z0: float = 0.1, h_inv: float = 1.0e30,
              direction=(1.0, 0.0, 0.0)) -> Config:
    """Replaces the x = 0 inflow of an opened case (open_x) by TOSCA's
    inletFunction type 2: the log-law ghost (u_tau/0.4) ln(h/z0) along
    `direction` (a unit vector), constant above h_inv."""
    b = list(cfg.bc); b[4] = BC_INLET_LOG
    cfg.bc = tuple(b)
    cfg.inlet_u_tau, cfg.inlet_z0, cfg.inlet_h_inv, cfg.inlet_dir = u_tau, z0, h_inv, tuple(direction)
    return cfg


def open_x(cfg: Config, u_in: float = 8.0, t_in: float = None) -> Config:
    """Turns the periodic x (k) direction of a case into an inflow/outflow
    pair: fixedValue velocity (u_in, 0, 0) at x = 0, zeroGradient at x = Lx,
    zero-gradient nut on both; with the temperature equation, a fixedValue
    temperature t_in at the inflow and zeroGradient at the outflow. The mean
    pressure gradient is switched off."""
    b = list(cfg.bc); b[4], b[5] = BC_FIXED_VALUE, BC_ZERO_GRADIENT
    nb = list(cfg.nut_bc); nb[4], nb[5] = NUTBC_ZEROGRADIENT, NUTBC_ZEROGRADIENT
    v = [0.0] * 18; v[12] = u_in
    cfg.bc, cfg.nut_bc, cfg.bc_value = tuple(b), tuple(nb), tuple(v)
    cfg.mean_grad_p, cfg.mean_grad_p_value = 0, (0.0, 0.0, 0.0)
    if cfg.teqn:
        tb = list(cfg.t_bc); tb[4], tb[5] = TBC_FIXED_VALUE, TBC_ZERO_GRADIENT
        tv = list(cfg.t_bc_value); tv[4] = cfg.t_ref if t_in is None else t_in
        cfg.t_bc, cfg.t_bc_value = tuple(tb), tuple(tv)
    return cfg


def farm_case(nx: int = 384, ny: int = 256, nz: int = 128, Lx: float = 3840.0, Ly: float = 2560.0,
              H: float = 1000.0, rows: int = 4, cols: int = 4, D: float = 126.0, hub: float = 90.0,
              sx: float = 7.0, sy: float = 5.0, epsilon: float = None, ct: float = 4.0 / 3.0,
              r_hub: float = 1.5, n_radial: int = 16, n_azimuth: int = 48, **kw):
    """ABL (abl_case, flow along +x) with rows x cols uniform actuator disks:
    diameter D at hub height `hub`, spaced sx D along x and sy D along y and
    centred in the domain, axes facing the wind (-x), C_T' = ct, Gaussian
    width epsilon (default twice the x spacing). Returns the abl_case tuple and
    the list of TgTurbine."""
    from .api import TgTurbine
    cfg, nodes, ucat, p = abl_case(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, H=H, **kw)
    eps = 2.0 * Lx / nx if epsilon is None else epsilon
    turbines = []
    for r in range(rows):
        for c in range(cols):
            x = 0.5 * Lx + (r - 0.5 * (rows - 1)) * sx * D
            y = 0.5 * Ly + (c - 0.5 * (cols - 1)) * sy * D
            turbines.append(TgTurbine.make((x, y, hub), axis=(-1.0, 0.0, 0.0), up=(0.0, 0.0, 1.0), r_tip=0.5 * D,
                                           r_hub=r_hub, epsilon=eps, ct=ct, n_radial=n_radial, n_azimuth=n_azimuth))
    return cfg, nodes, ucat, p, turbines


def hill_case(nx: int = 192, ny: int = 96, nz: int = 96, dt: float = 0.5, ustar: float = 0.3,
              z0: float = 0.1, kappa: float = 0.4, cs: float = 0.01, nu: float = 1.5e-5,
              theta0: float = 300.0, lapse: float = 0.001, ddt: int = DDT_FE, seed: int = 7, amp: float = 0.02,
              teqn: bool = False, t_amp: float = 0.0, **kw):
    """Terrain-following cosine-hill case: periodic x/y, Schumann wall stress on
    the terrain (curvilinear branch), slip top, QUICK convection, Smagorinsky,
    Boussinesq buoyancy from a stable stratification theta = theta0 + lapse * z
    (tRef = theta0), frozen, or with `teqn` transported (SolveTEqn, RK4:
    adiabatic terrain, the lapse rate as the fixed gradient at the top, Pr 0.7)
    with seeded +-t_amp K perturbations of the initial theta."""
    nodes = hill_nodes(nx, ny, nz, **kw)
    mx, my, mz = ny + 2, nz + 2, nx + 2
    H = float(nodes[0, my - 2, 0, 2])
    cfg = Config(mx=mx, my=my, mz=mz,
                 bc=(BC_PERIODIC, BC_PERIODIC, BC_WALL_SHUMANN, BC_SLIP, BC_PERIODIC, BC_PERIODIC),
                 nut_bc=(NUTBC_PERIODIC, NUTBC_PERIODIC, NUTBC_FIXEDVALUE, NUTBC_FIXEDVALUE, NUTBC_PERIODIC, NUTBC_PERIODIC),
                 curvilinear=1, les=1, cs=cs, nu=nu, div_scheme=DIV_QUICK, ddt_scheme=ddt, dt=dt,
                 buoyancy=1, t_ref=theta0, mean_grad_p=1, mean_grad_p_value=(ustar * ustar / H, 0.0, 0.0),
                 wall_roughness=z0, wall_kappa=kappa)
    cent = cell_centres(nodes)
    # height above the local terrain
    ground = np.zeros((mz, mx))
    ground[1:-1, 1:-1] = 0.25 * (nodes[1:-1, 0, 1:-1, 2] + nodes[:-2, 0, 1:-1, 2] + nodes[1:-1, 0, :-2, 2] + nodes[:-2, 0, :-2, 2])
    hz = np.maximum(cent[..., 2] - ground[:, None, :], z0 * 1.0001)
    U = (ustar / kappa) * np.log(hz / z0)
    G = mx * my * mz
    e = [uniform_noise(seed, G, s).reshape(mz, my, mx) * amp for s in range(3)]
    ucat = np.zeros_like(cent)
    ucat[..., 0] = U * (1.0 + e[0])
    ucat[..., 1] = U * e[1]
    ucat[..., 2] = U * e[2]
    interior = np.zeros((mz, my, mx), bool)
    interior[1:-1, 1:-1, 1:-1] = True
    ucat[~interior] = 0.0
    # frozen temperature with ghost values: interior from the centres, ghosts
    # by linear extrapolation in j and periodic copies in i, k
    T = theta0 + lapse * cent[..., 2]
    T[:, 0, :] = 2 * T[:, 1, :] - T[:, 2, :]
    T[:, -1, :] = 2 * T[:, -2, :] - T[:, -3, :]
    T[:, :, 0] = T[:, :, -2]
    T[:, :, -1] = T[:, :, 1]
    T[0] = T[-2]
    T[-1] = T[1]
    if teqn:
        cfg.ddt_scheme = DDT_RK4
        cfg.teqn = 1
        cfg.t_bc = (TBC_PERIODIC, TBC_PERIODIC, TBC_ZERO_GRADIENT, TBC_FIXED_GRADIENT, TBC_PERIODIC, TBC_PERIODIC)
        cfg.t_bc_value = (0.0, 0.0, 0.0, lapse, 0.0, 0.0)
        cfg.prandtl = 0.7
        if t_amp:
            T = T + t_amp * uniform_noise(seed + 11, G, 0).reshape(mz, my, mx) * interior
    p = np.zeros((mz, my, mx))
    return cfg, nodes, ucat, p, T


def thermal_wall(cfg: Config, kind: int = TWALL_SHUMANN, heating_rate: float = 0.0, qwall: float = 0.0,
                 localized: bool = False, gamma_m: float = 4.8, gamma_h: float = 7.8, alpha_h: float = 1.0) -> Config:
    """Puts a thetaWallFunction on the ground (jLeft) temperature patch of a
    configuration with transported temperature and LES: Schumann-Grotzbach
    with a surface heating rate (K/s), or a fixed heat flux qwall (K m/s).
    The roughness, kappa and thetaRef follow the velocity wall function and
    tRef; the same gammaM and thetaRef correct the velocity wall function."""
    bc = list(cfg.t_bc)
    bc[2] = TBC_WALL_FUNCTION
    cfg.t_bc = tuple(bc)
    cfg.t_wall_type = kind
    cfg.t_wall_localized = int(localized)
    cfg.t_wall_qwall = qwall
    cfg.t_wall_heating_rate = heating_rate
    cfg.t_wall_kappa = cfg.wall_kappa
    cfg.t_wall_theta_ref = cfg.t_ref
    cfg.t_wall_roughness = cfg.wall_roughness
    cfg.t_wall_gamma_m, cfg.t_wall_gamma_h, cfg.t_wall_alpha_h = gamma_m, gamma_h, alpha_h
    cfg.wall_gamma_m, cfg.wall_theta_ref = gamma_m, cfg.t_ref
    return cfg


def stratified_abl_case(nx: int = 256, ny: int = 256, nz: int = 128, theta0: float = 300.0, lapse: float = 0.01,
                        inversion: float = 100.0, t_amp: float = 0.1, heating_rate: float = -0.25 / 3600.0,
                        localized: bool = False, seed: int = 31, **kw):
    """Stably stratified ABL (abl_case grid and flow) with transported
    potential temperature: theta0 up to `inversion` m, then rising by `lapse`
    K/m, seeded +-t_amp K perturbations below the inversion, Boussinesq
    buoyancy (tRef = theta0), RK4 for both equations, Pr 0.7, the lapse rate
    as the fixed gradient at the top and a Schumann-Grotzbach
    thetaWallFunction at the ground whose surface cools at `heating_rate`
    K/s (the GABLS1 rate by default). Returns cfg, nodes, ucat, p, T."""
    cfg, nodes, ucat, p = abl_case(nx=nx, ny=ny, nz=nz, **kw)
    cfg.ddt_scheme = DDT_RK4
    cfg.buoyancy, cfg.t_ref = 1, theta0
    cfg.teqn, cfg.prandtl = 1, 0.7
    cfg.t_bc = (TBC_PERIODIC, TBC_PERIODIC, TBC_ZERO_GRADIENT, TBC_FIXED_GRADIENT, TBC_PERIODIC, TBC_PERIODIC)
    cfg.t_bc_value = (0.0, 0.0, 0.0, lapse, 0.0, 0.0)
    thermal_wall(cfg, TWALL_SHUMANN, heating_rate=heating_rate, localized=localized)
    cent = cell_centres(nodes)
    z = cent[..., 2]
    mz, my, mx = z.shape
    T = theta0 + lapse * np.maximum(z - inversion, 0.0)
    below = (z < inversion)
    T = T + t_amp * uniform_noise(seed, mx * my * mz, 0).reshape(mz, my, mx) * below
    T[:, 0, :] = T[:, 1, :]
    dz_top = nodes[:, my - 2, :, 2] - nodes[:, my - 3, :, 2]          # height of the top cells
    T[:, -1, :] = T[:, -2, :] + lapse * dz_top
    T[:, :, 0] = T[:, :, -2]
    T[:, :, -1] = T[:, :, 1]
    T[0] = T[-2]
    T[-1] = T[1]
    return cfg, nodes, ucat, p, T


def setup(solver, nodes, ucat, p, T=None):
    """Mesh, initial velocity and pressure into a Solver (SetInitialField)."""
    solver.set_mesh_nodes(nodes)
    if T is not None:
        solver.set("TMPRT", T)
    solver.init_from_cartesian(ucat)
    solver.set("P", p)
