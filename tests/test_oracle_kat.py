"""Known-answer checks that pin the CPU restatement (oracle) of TOSCA's step.

The reference ships no golden outputs (its tests are input decks only). Its
own code pins the restatement stage by stage in tests/test_ref_pin.py; the
checks here hold independently of it: properties the discretisation must
satisfy, i.e. Cartesian metric identities with TOSCA's axis mapping, exact
projection to a divergence-free field, symmetry of the pressure operator on
orthogonal grids, free-stream preservation on the curvilinear hill, and the
analytic decay rate of the 2-D Taylor-Green vortex."""
import math

import numpy as np
import pytest
import scipy.sparse.linalg as spla

import oracle
from tosca_b200 import api, cases
from tests.common import interior


def test_cartesian_metrics_axis_mapping():
    # mesh.c:92-94: i <-> y, j <-> z, k <-> x; csi = (0, dy dz, 0), aj = 1/(dx dy dz)
    X = np.linspace(0, 3.0, 7)      # dx = 0.5
    Y = np.linspace(0, 1.2, 7)      # dy = 0.2
    Z = np.linspace(0, 0.6, 7)      # dz = 0.1
    nodes = cases.cartesian_nodes(X, Y, Z)
    cfg = api.Config(mx=8, my=8, mz=8, bc=(api.BC_SLIP,) * 6)
    s = oracle.solver(cfg)
    s.set_mesh_nodes(nodes)
    dx, dy, dz = 0.5, 0.2, 0.1
    np.testing.assert_allclose(interior(s.get("CSI")), np.broadcast_to([0, dz * dx, 0], (6, 6, 6, 3)), atol=1e-14)
    np.testing.assert_allclose(interior(s.get("ETA")), np.broadcast_to([0, 0, dx * dy], (6, 6, 6, 3)), atol=1e-14)
    np.testing.assert_allclose(interior(s.get("ZET")), np.broadcast_to([dy * dz, 0, 0], (6, 6, 6, 3)), atol=1e-14)
    np.testing.assert_allclose(interior(s.get("AJ")), 1.0 / (dx * dy * dz), rtol=1e-13)
    cent = s.get("CENT")
    np.testing.assert_allclose(cent[3, 2, 4], [2.5 * dx, 3.5 * dy, 1.5 * dz], atol=1e-14)
    # face metrics on the boundary face 0 and ghost mirroring (mesh.c:1100-1180)
    np.testing.assert_allclose(s.get("ICSI")[3, 3, 0], [0, dz * dx, 0], atol=1e-14)
    np.testing.assert_allclose(s.get("IAJ")[3, 3, 0], 1.0 / (dx * dy * dz), rtol=1e-13)
    np.testing.assert_allclose(s.get("AJ")[0, 0, 0], 1.0 / (dx * dy * dz), rtol=1e-13)


def test_projection_is_divergence_free_tgv():
    cfg, nodes, ucat, p = cases.tgv_case(16)
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p)
    st = s.step(1)
    assert st.max_divergence < 1e-12
    assert st.poisson_final_residual < 1e-12


def test_pressure_operator_symmetric_orthogonal_and_pinned():
    cfg, nodes, ucat, p = cases.abl_case(12, 12, 8, Lx=120, Ly=120, H=80)
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p)
    A = oracle.poisson_matrix(s)
    assert oracle.lib().tor_poisson_symmetric(s.h) == 1
    A = A.toarray()
    # pinned first row (peqn.c:883-887)
    assert A[0, 0] == 1.0 and np.count_nonzero(A[0]) == 1
    B = A[1:, 1:]
    np.testing.assert_allclose(B, B.T, atol=1e-12 * np.abs(B).max())
    # rows annihilate constants except where they touch the pinned cell
    rs = A[1:].sum(axis=1)
    touching = A[1:, 0] != 0
    assert np.all(np.abs(rs[~touching]) < 1e-12 * np.abs(B).max())


def test_hill_operator_nonsymmetric_19pt():
    cfg, nodes, ucat, p, T = cases.hill_case(16, 8, 8)
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    A = oracle.poisson_matrix(s)
    nnz_per_row = np.diff(A.indptr)
    # the hill varies in x (DMDA k) only: cross terms couple k and j, giving
    # 7 + 4 entries per interior row
    assert nnz_per_row.max() == 11
    assert oracle.lib().tor_poisson_symmetric(s.h) == 0


def test_free_stream_preservation_hill():
    # a uniform horizontal stream: interpolated face fluxes are divergence free
    # on the terrain-following grid (metric identity of the face bases)
    cfg, nodes, ucat, p, T = cases.hill_case(24, 8, 8)
    s = oracle.solver(cfg)
    s.set_mesh_nodes(nodes)
    u = np.zeros_like(ucat)
    u[1:-1, 1:-1, 1:-1, 0] = 5.0
    s.init_from_cartesian(u)
    aj = s.get("AJ")
    uc = s.get("UCONT")
    div = (uc[1:-1, 1:-1, 1:-1, 0] - uc[1:-1, 1:-1, :-2, 0] + uc[1:-1, 1:-1, 1:-1, 1] - uc[1:-1, :-2, 1:-1, 1]
           + uc[1:-1, 1:-1, 1:-1, 2] - uc[:-2, 1:-1, 1:-1, 2]) * aj[1:-1, 1:-1, 1:-1]
    # the bottom row sees the wall (zero flux) -- check away from walls
    assert np.max(np.abs(div[:, 1:-1, :])) < 1e-10 * 5.0 / 15.0


def _tgv2d_rate(n, nsteps, dt, nu):
    """Measured / analytic energy decay rate of the 2-D Taylor-Green vortex
    (u = sin x cos y, v = -cos x sin y; energy ~ exp(-4 nu t)), taken after
    the first step so that the initial projection of the interpolated field
    does not enter."""
    L = 2 * math.pi
    X = np.linspace(0, L, n + 1)
    Z = np.linspace(0, L / n * 4, 5)          # 4 cells in z (the DMDA j direction)
    nodes = cases.cartesian_nodes(X, X.copy(), Z)
    cfg = api.Config(mx=n + 2, my=4 + 2, mz=n + 2, nu=nu, dt=dt, ddt_scheme=api.DDT_RK4)
    cent = cases.cell_centres(nodes)
    x, y = cent[..., 0], cent[..., 1]
    u = np.zeros_like(cent)
    u[..., 0] = np.sin(x) * np.cos(y)
    u[..., 1] = -np.cos(x) * np.sin(y)
    u[0] = u[-1] = 0; u[:, 0] = u[:, -1] = 0; u[:, :, 0] = u[:, :, -1] = 0
    p = np.zeros(cent.shape[:3])
    p[1:-1, 1:-1, 1:-1] = (0.25 * (np.cos(2 * x) + np.cos(2 * y)))[1:-1, 1:-1, 1:-1]
    s = oracle.solver(cfg)
    cases.setup(s, nodes, u, p)
    s.step(1)
    e0 = np.sum(interior(s.get("UCAT"))[..., :2] ** 2)
    s.step(nsteps)
    e1 = np.sum(interior(s.get("UCAT"))[..., :2] ** 2)
    return math.log(e1 / e0) / (-4 * nu * nsteps * dt)


def test_taylor_green_2d_decay_rate_second_order():
    r16 = _tgv2d_rate(16, 20, 0.01, 0.05)
    r32 = _tgv2d_rate(32, 20, 0.01, 0.05)
    e16, e32 = abs(r16 - 1.0), abs(r32 - 1.0)
    assert e32 < 0.01
    # second-order convergence of the decay rate
    assert 3.0 < e16 / e32 < 5.0
