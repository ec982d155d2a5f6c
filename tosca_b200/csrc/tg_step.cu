// Stage kernels of the fractional time step: momentum right-hand side
// (FormU and its sources), explicit integrators, boundary/ghost updates,
// projection and divergence. Each kernel restates one loop of the reference
// (file:line at the kernel). All fields are SoA FP64 on the global DMDA extent.
#include <cmath>
#include <type_traits>

#include "tg_internal.cuh"
#include "tg_mo.cuh"

namespace tg {
namespace {

__device__ __forceinline__ bool is_wall(int t) { return t == TG_BC_NOSLIP || t == TG_BC_SLIP || t == TG_BC_WALL_SHUMANN; }

// 2-D plane launch helper
inline dim3 g2(int na, int nb) { return dim3((na + 31) / 32, (nb + 7) / 8); }
const dim3 b2(32, 8);

// element-type conversion of a vector triple
template <class To, class From>
__device__ __forceinline__ R3<To> cvta(R3<From> a) { return R3<To>{(To)a.x, (To)a.y, (To)a.z}; }

// ------------------------------------------------------------------------
// contravariantToCartesian (ueqn.c:528-635): average face fluxes to the
// centre and solve [csi;eta;zet] u = q by Cramer's rule. Interior cells.
// MS is the storage type of the metrics (FP32 copies in the mixed-precision
// mode), A the arithmetic type; Ucont and Ucat stay FP64.
// ------------------------------------------------------------------------
template <class A, class MS>
__device__ __forceinline__ void contra_cell(const Grid &g, const FaceMet<MS> &m, const State &s, int c, bool ax)
{
    using M = A;
    if (ax) {
        // axis-aligned mesh: [csi; eta; zet] = [0 cs 0; 0 0 et; ze 0 0], the
        // same Cramer products without the vanishing ones
        const M cs = (M)m.csi.y[c], et = (M)m.eta.z[c], ze = (M)m.zet.x[c];
        const M q0 = (M)(0.5 * (s.ucont.x[c - 1] + s.ucont.x[c]));
        const M q1 = (M)(0.5 * (s.ucont.y[c - g.mx] + s.ucont.y[c]));
        const M q2 = (M)(0.5 * (s.ucont.z[c - g.mx * g.my] + s.ucont.z[c]));
        const M det = cs * (et * ze);
        s.ucat.x[c] = (double)((q2 * (cs * et)) / det);
        s.ucat.y[c] = (double)((q0 * (et * ze)) / det);
        s.ucat.z[c] = (double)((q1 * (cs * ze)) / det);
        return;
    }
    R3<M> sc = cvta<M>(ld3(m.csi, c)), e = cvta<M>(ld3(m.eta, c)), z = cvta<M>(ld3(m.zet, c));
    M m00 = sc.x, m01 = sc.y, m02 = sc.z, m10 = e.x, m11 = e.y, m12 = e.z, m20 = z.x, m21 = z.y, m22 = z.z;
    M q0 = (M)(0.5 * (s.ucont.x[c - 1] + s.ucont.x[c]));
    M q1 = (M)(0.5 * (s.ucont.y[c - g.mx] + s.ucont.y[c]));
    M q2 = (M)(0.5 * (s.ucont.z[c - g.mx * g.my] + s.ucont.z[c]));
    M det  =  m00 * (m11 * m22 - m12 * m21) - m01 * (m10 * m22 - m12 * m20) + m02 * (m10 * m21 - m11 * m20);
    M det0 =  q0 * (m11 * m22 - m12 * m21) - q1 * (m01 * m22 - m02 * m21) + q2 * (m01 * m12 - m02 * m11);
    M det1 = -q0 * (m10 * m22 - m12 * m20) + q1 * (m00 * m22 - m02 * m20) - q2 * (m00 * m12 - m02 * m10);
    M det2 =  q0 * (m10 * m21 - m11 * m20) - q1 * (m00 * m21 - m01 * m20) + q2 * (m00 * m11 - m01 * m10);
    s.ucat.x[c] = (double)(det0 / det); s.ucat.y[c] = (double)(det1 / det); s.ucat.z[c] = (double)(det2 / det);
}

template <class A, class MS>
__global__ void k_contra_to_cart(Grid g, FaceMet<MS> m, State s, bool ax)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    contra_cell<A>(g, m, s, g.lin(k, j, i), ax);
}

// the same on the interior cells next to the boundary only: the cells whose
// Cartesian velocity reaches the ghost cells through the periodic copies.
// blockIdx.z selects the boundary plane.
__global__ void k_contra_to_cart_shell(Grid g, FaceMet<double> m, State s, bool ax)
{
    int patch = blockIdx.z;
    int dir = patch >> 1, right = patch & 1;
    int a = blockIdx.x * blockDim.x + threadIdx.x + 1, b = blockIdx.y * blockDim.y + threadIdx.y + 1;
    int na = (dir == 0 ? g.my : g.mx) - 2, nb = (dir == 2 ? g.my : g.mz) - 2;
    if (a > na || b > nb) return;
    int i, j, k;
    if (dir == 0) { k = b; j = a; i = right ? g.mx - 2 : 1; }
    else if (dir == 1) { k = b; i = a; j = right ? g.my - 2 : 1; }
    else { j = b; i = a; k = right ? g.mz - 2 : 1; }
    contra_cell<double>(g, m, s, g.lin(k, j, i), ax);
}

// FP32 copies of the stencil metrics
__global__ void k_to_f32(int64_t n, const double *a, float *b)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) b[q] = (float)a[q];
}

// ------------------------------------------------------------------------
// resetCellPeriodicFluxes (inline.h:5453-5606): periodic ghost cells take the
// first interior cell of the opposite side. One direction per launch; applied
// i, then j, then k, which composes to the reference's simultaneous remap.
// left_only: resetFacePeriodicFluxesVector (inline.h:5357-5451), face 0 <- m-2.
// ------------------------------------------------------------------------
template <int NC, class T>
__global__ void k_periodic_copy(Grid g, T *a0, T *a1, T *a2, int dir, int left_only)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = dir == 0 ? g.my : g.mx, nb = dir == 2 ? g.my : g.mz;
    if (a >= na || b >= nb) return;
    for (int side = 0; side < (left_only ? 1 : 2); side++) {
        int d, s;
        if (dir == 0) { d = g.lin(b, a, side ? g.mx - 1 : 0); s = g.lin(b, a, side ? 1 : g.mx - 2); }
        else if (dir == 1) { d = g.lin(b, side ? g.my - 1 : 0, a); s = g.lin(b, side ? 1 : g.my - 2, a); }
        else { d = g.lin(side ? g.mz - 1 : 0, b, a); s = g.lin(side ? 1 : g.mz - 2, b, a); }
        a0[d] = a0[s];
        if (NC == 3) { a1[d] = a1[s]; a2[d] = a2[s]; }
    }
}

template <int NC, class T>
void periodic_copy(tg_ctx *C, T *a0, T *a1, T *a2, int left_only)
{
    const Grid g = C->g;
    if (g.pi) TG_PROF(C, "bc_periodic_copy", k_periodic_copy<NC, T><<<g2(g.my, g.mz), b2, 0, C->stream>>>(g, a0, a1, a2, 0, left_only));
    if (g.pj) TG_PROF(C, "bc_periodic_copy", k_periodic_copy<NC, T><<<g2(g.mx, g.mz), b2, 0, C->stream>>>(g, a0, a1, a2, 1, left_only));
    if (g.pk) TG_PROF(C, "bc_periodic_copy", k_periodic_copy<NC, T><<<g2(g.mx, g.my), b2, 0, C->stream>>>(g, a0, a1, a2, 2, left_only));
}

// ------------------------------------------------------------------------
// resetNoPenetrationFluxes (inline.h:5262-5355): zero wall-normal fluxes on
// wall patches. Plane launch per direction; range [0, m-2] in the others.
// ------------------------------------------------------------------------
__global__ void k_no_penetration(Grid g, State s, int dir, int left, int right)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = (dir == 0 ? g.my : g.mx) - 1, nb = (dir == 2 ? g.my : g.mz) - 1;
    if (a >= na || b >= nb) return;
    if (dir == 0) {
        if (left) s.ucont.x[g.lin(b, a, 0)] = 0.0;
        if (right) s.ucont.x[g.lin(b, a, g.mx - 2)] = 0.0;
    } else if (dir == 1) {
        if (left) s.ucont.y[g.lin(b, 0, a)] = 0.0;
        if (right) s.ucont.y[g.lin(b, g.my - 2, a)] = 0.0;
    } else {
        if (left) s.ucont.z[g.lin(0, b, a)] = 0.0;
        if (right) s.ucont.z[g.lin(g.mz - 2, b, a)] = 0.0;
    }
}

// ------------------------------------------------------------------------
// UpdateCartesianBCs (boundary.c:824-2050): face-adjacent ghost cells.
// blockIdx.z selects the patch; threads cover the interior of that patch.
// Reads interior cells only, writes ghost cells only.
// ------------------------------------------------------------------------
__global__ void k_cartesian_bcs(Grid g, Metrics m, State s, Params p)
{
    int patch = blockIdx.z;
    int dir = patch >> 1, right = patch & 1;
    int a = blockIdx.x * blockDim.x + threadIdx.x + 1, b = blockIdx.y * blockDim.y + threadIdx.y + 1;
    int na = (dir == 0 ? g.my : g.mx) - 2, nb = (dir == 2 ? g.my : g.mz) - 2;
    if (a > na || b > nb) return;
    int type = p.bc[patch];
    int i, j, k;
    if (dir == 0) { k = b; j = a; i = right ? g.mx - 2 : 1; }
    else if (dir == 1) { k = b; i = a; j = right ? g.my - 2 : 1; }
    else { j = b; i = a; k = right ? g.mz - 2 : 1; }
    int c = g.lin(k, j, i);
    int step = dir == 0 ? 1 : (dir == 1 ? g.mx : g.mx * g.my);
    int ghost = right ? c + step : c - step;
    R3<double> U = ld3(s.ucat, c);
    if (type == TG_BC_WALL_SHUMANN) {
        // slip preserving the wall-normal gradient, boundary.c:1155-1226 (jLeft)
        R3<double> Uc = ld3(s.ucat, right ? c - step : c + step);
        R3<double> n; calc_normal(ld3(m.csi, c), ld3(m.eta, c), ld3(m.zet, c), 1, n);
        R3<double> UbN = dot3(U, n) * n, UcN = dot3(Uc, n) * n;
        R3<double> UbP = U - UbN, UcP = Uc - UcN;
        R3<double> Ug{2. * UbP.x - UcP.x, 2. * UbP.y - UcP.y, 2. * UbP.z - UcP.z};
        st3(s.ucat, ghost, Ug - UbN);
    } else if (type == TG_BC_SLIP) {
        // boundary.c:1677-1853
        R3<double> n; calc_normal(ld3(m.csi, c), ld3(m.eta, c), ld3(m.zet, c), dir, n);
        R3<double> Un2 = (2.0 * dot3(U, n)) * n;
        st3(s.ucat, ghost, U - Un2);
    } else if (type == TG_BC_NOSLIP) {
        // boundary.c:1855-1895
        st3(s.ucat, ghost, -1.0 * U);
    } else if (type == TG_BC_FIXED_VALUE) {
        // fixedValue, boundary.c:1632-1673: the ghost takes the patch value
        st3(s.ucat, ghost, R3<double>{p.bc_value[3 * patch], p.bc_value[3 * patch + 1], p.bc_value[3 * patch + 2]});
    } else if (type == TG_BC_INLET_LOG) {
        // inletFunction type 2 (kLeft), boundary.c:1253-1283: the log law in
        // the first cell centre's height above the ground, at least 1e-5,
        // constant above hInv, along the unit direction
        const double h = m.cent.z[c] - p.grnd, ks = p.inlet_u_tau / 0.4;
        const double um = h <= p.inlet_h_inv ? fmax(ks * log(h / p.inlet_z0), 1e-5) : ks * log(p.inlet_h_inv / p.inlet_z0);
        st3(s.ucat, ghost, R3<double>{um * p.inlet_dir[0], um * p.inlet_dir[1], um * p.inlet_dir[2]});
    } else if (type == TG_BC_ZERO_GRADIENT) {
        // zeroGradient (outflow), boundary.c:1897-1970: linear extrapolation
        // from the first two cells
        st3(s.ucat, ghost, 2.0 * U - ld3(s.ucat, right ? c - step : c + step));
    } else {
        // periodic, boundary.c:1990-2018: ghost <- first interior cell of the opposite side
        int src;
        if (dir == 0) src = g.lin(k, j, right ? 1 : g.mx - 2);
        else if (dir == 1) src = g.lin(k, right ? 1 : g.my - 2, i);
        else src = g.lin(right ? 1 : g.mz - 2, j, i);
        st3(s.ucat, ghost, ld3(s.ucat, src));
    }
}

// ------------------------------------------------------------------------
// UpdateContravariantBCs (boundary.c:614-822). Two passes: periodic left
// faces take the solved right face (from the pre-call values), then the
// right/left faces of non-wall patches are re-interpolated from Ucat and
// wall faces zeroed.
// ------------------------------------------------------------------------
__global__ void k_contra_bc_periodic(Grid g, State s, int dir)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = (dir == 0 ? g.my : g.mx) - 1, nb = (dir == 2 ? g.my : g.mz) - 1;
    if (a >= na || b >= nb) return;
    if (dir == 0) s.ucont.x[g.lin(b, a, 0)] = s.ucont.x[g.lin(b, a, g.mx - 2)];
    else if (dir == 1) s.ucont.y[g.lin(b, 0, a)] = s.ucont.y[g.lin(b, g.my - 2, a)];
    else s.ucont.z[g.lin(0, b, a)] = s.ucont.z[g.lin(g.mz - 2, b, a)];
}

__global__ void k_contra_bc_faces(Grid g, Metrics m, State s, Params p, int dir)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = (dir == 0 ? g.my : g.mx) - 1, nb = (dir == 2 ? g.my : g.mz) - 1;
    if (a >= na || b >= nb) return;
    for (int side = 0; side < 2; side++) {
        int patch = 2 * dir + side;
        int type = p.bc[patch];
        bool periodic = type == TG_BC_PERIODIC;
        if (periodic && side == 0) continue;   // left periodic face handled by the copy pass
        int f, step;
        if (dir == 0) { f = g.lin(b, a, side ? g.mx - 2 : 0); step = 1; }
        else if (dir == 1) { f = g.lin(b, side ? g.my - 2 : 0, a); step = g.mx; }
        else { f = g.lin(side ? g.mz - 2 : 0, b, a); step = g.mx * g.my; }
        double *u = dir == 0 ? s.ucont.x : (dir == 1 ? s.ucont.y : s.ucont.z);
        if (is_wall(type)) { u[f] = 0.0; continue; }
        R3<double> un = ld3(s.ucat, f + step), uc = ld3(s.ucat, f);
        R3<double> S = dir == 0 ? ld3(m.icsi, f) : (dir == 1 ? ld3(m.jeta, f) : ld3(m.kzet, f));
        double v = 0.5 * (un.x + uc.x) * S.x + 0.5 * (un.y + uc.y) * S.y + 0.5 * (un.z + uc.z) * S.z;
        // zeroGradient: no flow back in through the face, boundary.c:718-741
        if (type == TG_BC_ZERO_GRADIENT && (side ? v < 0.0 : v > 0.0)) v = 0.0;
        u[f] = v;
    }
}

// ------------------------------------------------------------------------
// UpdatePhiBCs (boundary.c:3168-3255) / UpdatePressureBCs (boundary.c:3051-3166):
// ghost cells copy the first interior cell (zero gradient) or the opposite
// interior cell (periodic). Sequential per-direction passes compose to the
// reference's simultaneous remap because every source is interior in the
// remapped direction.
// ------------------------------------------------------------------------
__global__ void k_scalar_ghosts(Grid g, double *v, int dir)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = dir == 0 ? g.my : g.mx, nb = dir == 2 ? g.my : g.mz;
    if (a >= na || b >= nb) return;
    int per = dir == 0 ? g.pi : (dir == 1 ? g.pj : g.pk);
    int m = dir == 0 ? g.mx : (dir == 1 ? g.my : g.mz);
    for (int side = 0; side < 2; side++) {
        int dd = side ? m - 1 : 0;
        int ss = side ? (per ? 1 : m - 2) : (per ? m - 2 : 1);
        int d, s;
        if (dir == 0) { d = g.lin(b, a, dd); s = g.lin(b, a, ss); }
        else if (dir == 1) { d = g.lin(b, dd, a); s = g.lin(b, ss, a); }
        else { d = g.lin(dd, b, a); s = g.lin(ss, b, a); }
        v[d] = v[s];
    }
}

// ------------------------------------------------------------------------
// Smagorinsky eddy viscosity: UpdateCs (les.c:172-178) + UpdateNut
// (les.c:2119-2514) with Compute_du_center (inline.h:3344-3418) and
// Compute_du_dxyz (inline.h:3635-3663). Interior cells.
// ------------------------------------------------------------------------
template <class M>
__global__ void k_smagorinsky(Grid g, FaceMet<M> m, State s, Params p, bool ax)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int c = g.lin(k, j, i);
    // the +-1 neighbours of an interior cell lie inside the DMDA: no wrap
    auto U = [&](int kk, int jj, int ii) { return ld3(s.ucat, g.lin(kk, jj, ii)); };
    M ajc = m.aj[c];
    R3<M> sc = ld3(m.csi, c), e = ld3(m.eta, c), z = ld3(m.zet, c);
    R3<double> dc, de, dz;
    if (!g.pi && i == g.mx - 2) dc = U(k, j, i) - U(k, j, i - 1);
    else if (!g.pi && i == 1)   dc = U(k, j, i + 1) - U(k, j, i);
    else                        dc = 0.5 * (U(k, j, i + 1) - U(k, j, i - 1));
    if (!g.pj && j == g.my - 2) de = U(k, j, i) - U(k, j - 1, i);
    else if (!g.pj && j == 1)   de = U(k, j + 1, i) - U(k, j, i);
    else                        de = 0.5 * (U(k, j + 1, i) - U(k, j - 1, i));
    if (!g.pk && k == g.mz - 2) dz = U(k, j, i) - U(k - 1, j, i);
    else if (!g.pk && k == 1)   dz = U(k + 1, j, i) - U(k, j, i);
    else                        dz = 0.5 * (U(k + 1, j, i) - U(k - 1, j, i));
    const R3<M> a = cvta<M>(dc), b = cvta<M>(de), d = cvta<M>(dz);
    const M h = M(0.5);
    M du_dx, du_dy, du_dz, dv_dx, dv_dy, dv_dz, dw_dx, dw_dy, dw_dz;
    if (ax) {
        // axis-aligned mesh: csi = (0, cs, 0), eta = (0, 0, et), zet = (ze, 0, 0)
        du_dx = (d.x * z.x) * ajc; du_dy = (a.x * sc.y) * ajc; du_dz = (b.x * e.z) * ajc;
        dv_dx = (d.y * z.x) * ajc; dv_dy = (a.y * sc.y) * ajc; dv_dz = (b.y * e.z) * ajc;
        dw_dx = (d.z * z.x) * ajc; dw_dy = (a.z * sc.y) * ajc; dw_dz = (b.z * e.z) * ajc;
    } else {
        du_dx = (a.x * sc.x + b.x * e.x + d.x * z.x) * ajc;
        du_dy = (a.x * sc.y + b.x * e.y + d.x * z.y) * ajc;
        du_dz = (a.x * sc.z + b.x * e.z + d.x * z.z) * ajc;
        dv_dx = (a.y * sc.x + b.y * e.x + d.y * z.x) * ajc;
        dv_dy = (a.y * sc.y + b.y * e.y + d.y * z.y) * ajc;
        dv_dz = (a.y * sc.z + b.y * e.z + d.y * z.z) * ajc;
        dw_dx = (a.z * sc.x + b.z * e.x + d.z * z.x) * ajc;
        dw_dy = (a.z * sc.y + b.z * e.y + d.z * z.y) * ajc;
        dw_dz = (a.z * sc.z + b.z * e.z + d.z * z.z) * ajc;
    }
    M S00 = h * (du_dx + du_dx), S01 = h * (du_dy + dv_dx), S02 = h * (du_dz + dw_dx);
    M S10 = h * (dv_dx + du_dy), S11 = h * (dv_dy + dv_dy), S12 = h * (dv_dz + dw_dy);
    M S20 = h * (dw_dx + du_dz), S21 = h * (dw_dy + dv_dz), S22 = h * (dw_dz + dw_dz);
    M Sabs = sqrt(M(2) * (S00 * S00 + S01 * S01 + S02 * S02 + S10 * S10 + S11 * S11 + S12 * S12 + S20 * S20 + S21 * S21 + S22 * S22));
    // filter width squared pow(pow(1/aj, 1/3), 2), evaluated once per mesh (k_filter2)
    s.nut[c] = (double)((M)p.cs * m.flt2[c] * Sabs);
}

// UpdateNutBCs (boundary.c:2630-2930): face-adjacent ghosts of nut
__global__ void k_nut_bcs(Grid g, State s, Params p)
{
    int patch = blockIdx.z;
    int dir = patch >> 1, right = patch & 1;
    int a = blockIdx.x * blockDim.x + threadIdx.x + 1, b = blockIdx.y * blockDim.y + threadIdx.y + 1;
    int na = (dir == 0 ? g.my : g.mx) - 2, nb = (dir == 2 ? g.my : g.mz) - 2;
    if (a > na || b > nb) return;
    int i, j, k;
    if (dir == 0) { k = b; j = a; i = right ? g.mx - 2 : 1; }
    else if (dir == 1) { k = b; i = a; j = right ? g.my - 2 : 1; }
    else { j = b; i = a; k = right ? g.mz - 2 : 1; }
    int c = g.lin(k, j, i);
    int step = dir == 0 ? 1 : (dir == 1 ? g.mx : g.mx * g.my);
    int ghost = right ? c + step : c - step;
    int t = p.nut_bc[patch];
    if (t == TG_NUTBC_ZEROGRADIENT) s.nut[ghost] = s.nut[c];
    else if (t == TG_NUTBC_FIXEDVALUE) s.nut[ghost] = p.nut_bc_value[patch];
    else {
        int src;
        if (dir == 0) src = g.lin(k, j, right ? 1 : g.mx - 2);
        else if (dir == 1) src = g.lin(k, right ? 1 : g.my - 2, i);
        else src = g.lin(right ? 1 : g.mz - 2, j, i);
        s.nut[ghost] = s.nut[src];
    }
}

// ------------------------------------------------------------------------
// UpdateWallModelsU for jLeft wall function -3 (boundary.c:3257-3600):
// plane averages, friction velocity (uStarShumann, wallfunctions.c:12-130:
// neutral, or corrected by the plane mean of the thetaWallFunction's last
// heat flux when the temperature jLeft patch has one), filtered
// wall-parallel velocity and the contravariant wall stress.
// ------------------------------------------------------------------------
__device__ __forceinline__ void wall_parallel(Grid g, Metrics m, State s, int k, int i, R3<double> &Up, R3<double> &n)
{
    int c = g.lin(k, 1, i);
    calc_normal(ld3(m.csi, c), ld3(m.eta, c), ld3(m.zet, c), 1, n);
    R3<double> U = ld3(s.ucat, c);
    Up = U - dot3(U, n) * n;
}

// per-block partial sums of |U_par|, the wall distance and (coupled) qWall
// over the j=1 plane
__global__ void __launch_bounds__(256) k_wall_plane_sums(Grid g, Metrics m, State s, Params p, double *part)
{
    int nI = g.mx - 2, nK = g.mz - 2;
    double su = 0.0, sd = 0.0, sq = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nI * nK; t += gridDim.x * blockDim.x) {
        int i = t % nI + 1, k = t / nI + 1;
        int c = g.lin(k, 1, i);
        double area = sqrt(dot3(ld3(m.eta, c), ld3(m.eta, c)));
        R3<double> Up, n; wall_parallel(g, m, s, k, i, Up, n);
        su += sqrt(dot3(Up, Up));
        sd += 0.5 / m.aj[c] / area;
        if (p.wall_coupled) sq += s.qwall[k * g.mx + i];
    }
    double v[3] = {su, sd, sq};
    block_reduce<256>(v, RedSum{}, RedSum{}, RedSum{});
    if (threadIdx.x == 0) { part[3 * blockIdx.x] = v[0]; part[3 * blockIdx.x + 1] = v[1]; part[3 * blockIdx.x + 2] = v[2]; }
}

// final sums (deterministic order) and u* = uStarShumann(<|U_par|>, <s>, qWall)
__global__ void k_wall_ustar(Grid g, Params p, const double *part, int nb, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double su = 0.0, sd = 0.0, sq = 0.0;
    for (int b = 0; b < nb; b++) { su += part[3 * b]; sd += part[3 * b + 1]; sq += part[3 * b + 2]; }
    double cnt = (double)(g.mx - 2) * (double)(g.mz - 2);
    double Umean = su / cnt, dist = sd / cnt, q = sq / cnt;
    double us = mo::ustar(Umean, dist, p.z0, p.wall_gamma_m, p.kappa, p.wall_coupled ? q : 0.0, p.wall_theta_ref);
    out[0] = Umean; out[1] = dist; out[2] = us;
}

__global__ void k_wall_init_filter(Grid g, Metrics m, State s)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, k = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.mx - 2 || k > g.mz - 2) return;
    R3<double> Up, n; wall_parallel(g, m, s, k, i, Up, n);
    int w = k * g.mx + i;
    s.ufx[w] = Up.x; s.ufy[w] = Up.y; s.ufz[w] = Up.z;
}

// d_it: the step counter (the running mean of |U_parallel| weights the old
// mean by it / (it + 1))
__global__ void k_wall_stress(Grid g, Metrics m, State s, Params p, const double *wsc, const double *d_it)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, k = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.mx - 2 || k > g.mz - 2) return;
    const double Umean = wsc[0], uStar = wsc[2];
    const double aN = d_it[0], m1 = aN / (aN + 1.0), m2 = 1.0 / (aN + 1.0);
    int c = g.lin(k, 1, i), w = k * g.mx + i;
    R3<double> Up, n; wall_parallel(g, m, s, k, i, Up, n);
    double upm = sqrt(dot3(Up, Up));
    R3<double> e1{Up.x / (upm + 1.e-12), Up.y / (upm + 1.e-12), Up.z / (upm + 1.e-12)};   // nUnit, inline.h:870-890
    R3<double> e3 = n;
    double um = m1 * s.umean[w] + m2 * upm;
    s.umean[w] = um;
    R3<double> zz = ld3(m.zet, c), cc = ld3(m.csi, c);
    double lx = 1.0 / m.aj[c] / sqrt(dot3(zz, zz)), ly = 1.0 / m.aj[c] / sqrt(dot3(cc, cc));
    double T = fmax(sqrt(lx * lx + ly * ly) / um, p.dt);
    s.ufx[w] = (1.0 - p.dt / T) * s.ufx[w] + (p.dt / T) * Up.x;
    s.ufy[w] = (1.0 - p.dt / T) * s.ufy[w] + (p.dt / T) * Up.y;
    R3<double> je = ld3(m.jeta, g.lin(k, 0, i));
    if (p.curvilinear) {
        // rotation to the local (e1, e2 = e3 x e1, e3) frame; only the e1 and e3 columns enter the stress
        double a11 = e1.x, a13 = e3.x;
        double a21 = e1.y, a23 = e3.y;
        double a31 = e1.z, a33 = e3.z;
        double u2 = uStar * uStar;
        double t11 = -2.0 * a11 * a13 * u2, t12 = -(a13 * a21 + a11 * a23) * u2, t13 = -(a13 * a31 + a11 * a33) * u2;
        double t21 = -(a23 * a11 + a21 * a13) * u2, t22 = -2.0 * a23 * a21 * u2, t23 = -(a23 * a31 + a21 * a33) * u2;
        double t31 = -(a33 * a11 + a31 * a13) * u2, t32 = -(a33 * a21 + a31 * a23) * u2, t33 = -2.0 * a33 * a31 * u2;
        s.twx[w] = t11 * je.x + t12 * je.y + t13 * je.z;
        s.twy[w] = t21 * je.x + t22 * je.y + t23 * je.z;
        s.twz[w] = t31 * je.x + t32 * je.y + t33 * je.z;
    } else {
        double TauXZ = -uStar * uStar * (s.ufx[w] / fmax(Umean, 1e-5));
        double TauYZ = -uStar * uStar * (s.ufy[w] / fmax(Umean, 1e-5));
        s.twx[w] = je.z * TauXZ;
        s.twy[w] = je.z * TauYZ;
        s.twz[w] = je.x * TauXZ + je.y * TauYZ;
    }
}

// ------------------------------------------------------------------------
// GradP (peqn.c:3437-3773): face pressure gradient with the metric tensor,
// one-sided cross derivatives only at the corner faces. Interior cells.
// ------------------------------------------------------------------------
// GH = true: ghGradRhoK (teqn.c:278-652, -pTildeBuoyancy 1), the same
// stencil applied to rho_k = (tRef - T) / tRef and scaled by g z of the cell's
// node (g = -9.81), stored negated in bTheta so that ExplicitRhsU's AB2
// buoyancy sum +3/2 b - 1/2 b_o reads -3/2 ghGradRhok + 1/2 ghGradRhok_o
// (ueqn_solvers.c:1314-1324); the products are associated as (g z) (grad .
// S) aj, the reference's g z (grad . S) aj up to rounding
template <class M, bool GH = false>
__global__ void k_grad_p(Grid g, FaceMet<M> m, State s, bool ax, const double *node_z = nullptr, double t_ref = 0.0)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int c = g.lin(k, j, i);
    auto P = [&](int kk, int jj, int ii) {
        const double v = GH ? s.tmprt[g.id(kk, jj, ii)] : s.p[g.id(kk, jj, ii)];
        return GH ? (t_ref - v) / t_ref : v;
    };
    const int mx = g.mx, my = g.my, mz = g.mz;
    if (ax && !GH) {
        // axis-aligned mesh: the cross terms g12, g13, g21, g23, g31, g32 vanish
        // the + neighbours lie inside the DMDA except across a periodic seam,
        // where index m + 1 wraps to 1
        const M ic = m.icsi.y[c], je = m.jeta.z[c], kz = m.kzet.x[c];
        const double pc = s.p[c];
        const double dpdc = ((i == mx - 2 && g.pi) ? s.p[g.lin(k, j, 1)] : s.p[c + 1]) - pc;
        const double dpde = ((j == my - 2 && g.pj) ? s.p[g.lin(k, 1, i)] : s.p[c + mx]) - pc;
        const double dpdz = ((k == mz - 2 && g.pk) ? s.p[g.lin(1, j, i)] : s.p[c + mx * my]) - pc;
        M ox = ((M)dpdc * (ic * ic)) * m.iaj[c], oy = ((M)dpde * (je * je)) * m.jaj[c], oz = ((M)dpdz * (kz * kz)) * m.kaj[c];
        if (!g.pi && i == mx - 2) ox = 0;
        if (!g.pj && j == my - 2) oy = 0;
        if (!g.pk && k == mz - 2) oz = 0;
        s.dp.x[c] = (double)ox; s.dp.y[c] = (double)oy; s.dp.z[c] = (double)oz;
        return;
    }
    R3<M> ic = ld3(m.icsi, c), ie = ld3(m.ieta, c), iz = ld3(m.izet, c);
    R3<M> jc = ld3(m.jcsi, c), je = ld3(m.jeta, c), jz = ld3(m.jzet, c);
    R3<M> kc = ld3(m.kcsi, c), ke = ld3(m.keta, c), kz = ld3(m.kzet, c);
    M g11 = dot3(ic, ic), g12 = dot3(ie, ic), g13 = dot3(iz, ic);
    M g21 = dot3(jc, je), g22 = dot3(je, je), g23 = dot3(jz, je);
    M g31 = dot3(kc, kz), g32 = dot3(ke, kz), g33 = dot3(kz, kz);
    double dpdc, dpde, dpdz;
    M ox, oy, oz;
    dpdc = (i == mx - 2 && g.pi) ? P(k, j, mx + 1) - P(k, j, i) : P(k, j, i + 1) - P(k, j, i);
    if (j == my - 2 && i == mx - 2)  dpde = (P(k, j, i) - P(k, j - 1, i) + P(k, j, i + 1) - P(k, j - 1, i + 1)) * 0.5;
    else if (j == 1 && i == mx - 2)  dpde = (P(k, j + 1, i) - P(k, j, i) + P(k, j + 1, i + 1) - P(k, j, i + 1)) * 0.5;
    else                             dpde = (P(k, j + 1, i) - P(k, j - 1, i) + P(k, j + 1, i + 1) - P(k, j - 1, i + 1)) * 0.25;
    if (k == mz - 2 && i == mx - 2)  dpdz = (P(k, j, i) - P(k - 1, j, i) + P(k, j, i + 1) - P(k - 1, j, i + 1)) * 0.5;
    else if (k == 1 && i == mx - 2)  dpdz = (P(k + 1, j, i) - P(k, j, i) + P(k + 1, j, i + 1) - P(k, j, i + 1)) * 0.5;
    else                             dpdz = (P(k + 1, j, i) - P(k - 1, j, i) + P(k + 1, j, i + 1) - P(k - 1, j, i + 1)) * 0.25;
    ox = ((M)dpdc * g11 + (M)dpde * g12 + (M)dpdz * g13) * m.iaj[c];
    if (i == mx - 2 && j == my - 2)  dpdc = (P(k, j, i) - P(k, j, i - 1) + P(k, j + 1, i) - P(k, j + 1, i - 1)) * 0.5;
    else if (i == 1 && j == my - 2)  dpdc = (P(k, j, i + 1) - P(k, j, i) + P(k, j + 1, i + 1) - P(k, j + 1, i)) * 0.5;
    else                             dpdc = (P(k, j, i + 1) - P(k, j, i - 1) + P(k, j + 1, i + 1) - P(k, j + 1, i - 1)) * 0.25;
    dpde = (j == my - 2 && g.pj) ? P(k, my + 1, i) - P(k, j, i) : P(k, j + 1, i) - P(k, j, i);
    if (k == mz - 2 && j == my - 2)  dpdz = (P(k, j, i) - P(k - 1, j, i) + P(k, j + 1, i) - P(k - 1, j + 1, i)) * 0.5;
    else if (k == 1 && j == my - 2)  dpdz = (P(k + 1, j, i) - P(k, j, i) + P(k + 1, j + 1, i) - P(k, j + 1, i)) * 0.5;
    else                             dpdz = (P(k + 1, j, i) - P(k - 1, j, i) + P(k + 1, j + 1, i) - P(k - 1, j + 1, i)) * 0.25;
    oy = ((M)dpdc * g21 + (M)dpde * g22 + (M)dpdz * g23) * m.jaj[c];
    if (i == mx - 2 && k == mz - 2)  dpdc = (P(k, j, i) - P(k, j, i - 1) + P(k + 1, j, i) - P(k + 1, j, i - 1)) * 0.5;
    else if (i == 1 && k == mz - 2)  dpdc = (P(k, j, i + 1) - P(k, j, i) + P(k + 1, j, i + 1) - P(k + 1, j, i)) * 0.5;
    else                             dpdc = (P(k, j, i + 1) - P(k, j, i - 1) + P(k + 1, j, i + 1) - P(k + 1, j, i - 1)) * 0.25;
    if (j == my - 2 && k == mz - 2)  dpde = (P(k, j, i) - P(k, j - 1, i) + P(k + 1, j, i) - P(k + 1, j - 1, i)) * 0.5;
    else if (j == 1 && k == mz - 2)  dpde = (P(k, j + 1, i) - P(k, j, i) + P(k + 1, j + 1, i) - P(k + 1, j, i)) * 0.5;
    else                             dpde = (P(k, j + 1, i) - P(k, j - 1, i) + P(k + 1, j + 1, i) - P(k + 1, j - 1, i)) * 0.25;
    dpdz = (k == mz - 2 && g.pk) ? P(mz + 1, j, i) - P(k, j, i) : P(k + 1, j, i) - P(k, j, i);
    oz = ((M)dpdc * g31 + (M)dpde * g32 + (M)dpdz * g33) * m.kaj[c];
    if (!g.pi && i == mx - 2) ox = 0;
    if (!g.pj && j == my - 2) oy = 0;
    if (!g.pk && k == mz - 2) oz = 0;
    if (GH) {
        const double gz = -9.81 * node_z[c];
        s.btheta.x[c] = -(gz * (double)ox); s.btheta.y[c] = -(gz * (double)oy); s.btheta.z[c] = -(gz * (double)oz);
        return;
    }
    s.dp.x[c] = (double)ox; s.dp.y[c] = (double)oy; s.dp.z[c] = (double)oz;
}

// ------------------------------------------------------------------------
// Buoyancy (ueqn_sources.c:2726-2880), frozen temperature: g_cont = g.S_face
// and bTheta = g_cont (tRef - T_face)/tRef at faces of interior cells.
// ------------------------------------------------------------------------
__global__ void k_buoyancy(Grid g, Metrics m, State s, Params p)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    int c = g.lin(k, j, i);
    const double gz = -9.81, tRef = p.t_ref;
    if (i <= g.mx - 2 && j <= g.my - 2 && k <= g.mz - 2) {
        if (j > 0 && k > 0) { R3<double> S = ld3(m.icsi, c); s.gcont.x[c] = 0 * S.x + 0 * S.y + gz * S.z; }
        if (i > 0 && k > 0) { R3<double> S = ld3(m.jeta, c); s.gcont.y[c] = 0 * S.x + 0 * S.y + gz * S.z; }
        if (i > 0 && j > 0) { R3<double> S = ld3(m.kzet, c); s.gcont.z[c] = 0 * S.x + 0 * S.y + gz * S.z; }
    }
    double bx = 0.0, by = 0.0, bz = 0.0;
    if (i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2) {
        double T = s.tmprt[c];
        double tI = 0.5 * (T + s.tmprt[g.id(k, j, i + 1)]);
        double tJ = 0.5 * (T + s.tmprt[g.id(k, j + 1, i)]);
        double tK = 0.5 * (T + s.tmprt[g.id(k + 1, j, i)]);
        bx += 1.0 * (s.gcont.x[c] * (tRef - tI) / tRef);
        by += 1.0 * (s.gcont.y[c] * (tRef - tJ) / tRef);
        bz += 1.0 * (s.gcont.z[c] * (tRef - tK) / tRef);
    }
    s.btheta.x[c] = bx; s.btheta.y[c] = by; s.btheta.z[c] = bz;
}

// ------------------------------------------------------------------------
// FormU (ueqn_solvers.c:6-1083), every formMode (pass 1 selects the terms).
// Pass 1: per face the convective (central or QUICK) plus viscous flux,
// stored summed per direction in f1 (i faces), f2 (j faces), f3 (k faces).
// ------------------------------------------------------------------------
__device__ __forceinline__ R3<double> quick(R3<double> f0, R3<double> f1, R3<double> f2, R3<double> f3, double w)
{
    // quadraticUpwindVec, inline.h:5089-5109
    R3<double> fUU, fU, fD;
    if (w > 0) { fUU = f0; fU = f1; fD = f2; } else { fUU = f3; fU = f2; fD = f1; }
    return 0.5 * (fU + fD) + (1. / 8.) * (2.0 * fU - (fD + fUU));
}

// viscous flux (g . grad u + R . n) * ajc * nuEff, ueqn_solvers.c:180-216, 392-394
template <class M>
__device__ __forceinline__ R3<M> visc_flux(R3<M> s0, R3<M> s1, R3<M> s2, int dir, R3<M> dc, R3<M> de, R3<M> dz, M ajc, M nuEff)
{
    M csi0 = s0.x, csi1 = s0.y, csi2 = s0.z, eta0 = s1.x, eta1 = s1.y, eta2 = s1.z, zet0 = s2.x, zet1 = s2.y, zet2 = s2.z;
    M g11, g21, g31, n0, n1, n2;
    if (dir == 0) { g11 = csi0 * csi0 + csi1 * csi1 + csi2 * csi2; g21 = eta0 * csi0 + eta1 * csi1 + eta2 * csi2; g31 = zet0 * csi0 + zet1 * csi1 + zet2 * csi2; n0 = csi0; n1 = csi1; n2 = csi2; }
    else if (dir == 1) { g11 = csi0 * eta0 + csi1 * eta1 + csi2 * eta2; g21 = eta0 * eta0 + eta1 * eta1 + eta2 * eta2; g31 = zet0 * eta0 + zet1 * eta1 + zet2 * eta2; n0 = eta0; n1 = eta1; n2 = eta2; }
    else { g11 = csi0 * zet0 + csi1 * zet1 + csi2 * zet2; g21 = eta0 * zet0 + eta1 * zet1 + eta2 * zet2; g31 = zet0 * zet0 + zet1 * zet1 + zet2 * zet2; n0 = zet0; n1 = zet1; n2 = zet2; }
    M r11 = dc.x * csi0 + de.x * eta0 + dz.x * zet0, r21 = dc.y * csi0 + de.y * eta0 + dz.y * zet0, r31 = dc.z * csi0 + de.z * eta0 + dz.z * zet0;
    M r12 = dc.x * csi1 + de.x * eta1 + dz.x * zet1, r22 = dc.y * csi1 + de.y * eta1 + dz.y * zet1, r32 = dc.z * csi1 + de.z * eta1 + dz.z * zet1;
    M r13 = dc.x * csi2 + de.x * eta2 + dz.x * zet2, r23 = dc.y * csi2 + de.y * eta2 + dz.y * zet2, r33 = dc.z * csi2 + de.z * eta2 + dz.z * zet2;
    R3<M> v;
    v.x = (g11 * dc.x + g21 * de.x + g31 * dz.x + r11 * n0 + r21 * n1 + r31 * n2) * ajc * (nuEff);
    v.y = (g11 * dc.y + g21 * de.y + g31 * dz.y + r12 * n0 + r22 * n1 + r32 * n2) * ajc * (nuEff);
    v.z = (g11 * dc.z + g21 * de.z + g31 * dz.z + r13 * n0 + r23 * n1 + r33 * n2) * ajc * (nuEff);
    return v;
}

// Pass 1 runs one thread per interior cell (k, j, i): it forms the i, j and
// k faces on the cell's + side, and a cell next to a non-periodic 0 boundary
// also the face on its - side (face 0, which a periodic direction does not
// form). Ucat and nut are staged in a shared-memory tile covering the block's
// cells with one cell below and two above in every direction, loaded once
// with the periodic wrap of the DMDA index (g.id); every stencil read then is
// a fixed tile offset. Tile points outside a non-periodic extent hold 0 and
// are never read; the QUICK points of the boundary faces, which may lie
// outside the tile (the periodic wrap reads i = mx + 2 and i = -3), are read
// from global memory.
//
// visc_flux on an axis-aligned mesh (csi || y, eta || z, zet || x, the
// reference's i -> y, j -> z, k -> x axes): cs = csi.y, et = eta.z, ze = zet.x
// of the face. Every other metric component is zero up to the round-off of
// the metric evaluation (at most 1e-12 of the largest, tg_set_mesh_nodes), so
// the products left out change the flux by that relative amount at most; the
// terms kept are the same products.
template <class M>
__device__ __forceinline__ R3<M> visc_flux_ax(M cs, M et, M ze, int dir, R3<M> dc, R3<M> de, R3<M> dz, M ajc, M nuEff)
{
    R3<M> v;
    if (dir == 0) {          // n = csi: g11 = cs^2, r21 = dz.y ze, r22 = dc.y cs, r23 = de.y et
        const M g11 = cs * cs;
        v.x = (g11 * dc.x + (dz.y * ze) * cs) * ajc * (nuEff);
        v.y = (g11 * dc.y + (dc.y * cs) * cs) * ajc * (nuEff);
        v.z = (g11 * dc.z + (de.y * et) * cs) * ajc * (nuEff);
    } else if (dir == 1) {   // n = eta: g21 = et^2, r31 = dz.z ze, r32 = dc.z cs, r33 = de.z et
        const M g21 = et * et;
        v.x = (g21 * de.x + (dz.z * ze) * et) * ajc * (nuEff);
        v.y = (g21 * de.y + (dc.z * cs) * et) * ajc * (nuEff);
        v.z = (g21 * de.z + (de.z * et) * et) * ajc * (nuEff);
    } else {                 // n = zet: g31 = ze^2, r11 = dz.x ze, r12 = dc.x cs, r13 = de.x et
        const M g31 = ze * ze;
        v.x = (g31 * dz.x + (dz.x * ze) * ze) * ajc * (nuEff);
        v.y = (g31 * dz.y + (dc.x * cs) * ze) * ajc * (nuEff);
        v.z = (g31 * dz.z + (de.x * et) * ze) * ajc * (nuEff);
    }
    return v;
}

// M: storage and arithmetic type of the metrics in the viscous flux; F: storage
// type of the face fluxes. The convective flux is formed in FP64 from the FP64
// Ucont and Ucat. mode is FormU's formMode (ueqn_solvers.c:17, 105-106):
// 0 convection + viscosity, 1 convection only, 2 viscosity (with the wall
// stress) only; the skipped part of each face flux is zero. AX: the mesh is
// axis-aligned (visc_flux_ax reads 3 of the 9 face metric components).
constexpr int FBX = 32, FBY = 4, FBZ = 2, FBN = FBX * FBY * FBZ, FMINB = 4;   // block of k_face_fluxes
constexpr int FTX = FBX + 3, FTY = FBY + 3, FTZ = FBZ + 3, FTN = FTX * FTY * FTZ;

template <class M, class F, int mode, bool AX>
__global__ void __launch_bounds__(FBN, FMINB) k_face_fluxes(Grid g, FaceMet<M> m, State s, FluxWork<F> w, Params p)
{
    __shared__ double su[3][FTN];
    __shared__ double sn[FTN];
    const int mx = g.mx, my = g.my, mz = g.mz;
    const int i0 = 1 + blockIdx.x * FBX, j0 = 1 + blockIdx.y * FBY, k0 = 1 + blockIdx.z * FBZ;
    const bool les = p.les;
    // staging: tile point (tx, ty, tz) <- DMDA (i0-1+tx, j0-1+ty, k0-1+tz),
    // wrapped; 0 outside a non-periodic extent
    auto stage = [&](int tx, int ty, int tz, int gi) {
        const int gj = g.wj(j0 - 1 + ty), gk = g.wk(k0 - 1 + tz), q = (tz * FTY + ty) * FTX + tx;
        double ux = 0.0, uy = 0.0, uz = 0.0, nt = 0.0;
        if (gi >= 0 && gi < mx && gj >= 0 && gj < my && gk >= 0 && gk < mz) {
            const int c = (gk * my + gj) * mx + gi;
            ux = s.ucat.x[c]; uy = s.ucat.y[c]; uz = s.ucat.z[c];
            if (mode != 1 && les) nt = s.nut[c];
        }
        su[0][q] = ux; su[1][q] = uy; su[2][q] = uz; sn[q] = nt;
    };
    {
        // each warp stages whole tile rows (its lane is tx, the row index is
        // warp-uniform), then every thread at most one of the 3 x FTY x FTZ
        // points of the last three columns
        static_assert(FBX == 32 && FBN % 32 == 0 && 3 * FTY * FTZ <= FBN, "one warp per tile row, one pass for the last columns");
        const int lane = threadIdx.x, wid = threadIdx.z * FBY + threadIdx.y;
        const int gi = g.wi(i0 - 1 + lane);
        for (int r = wid; r < FTY * FTZ; r += FBN / 32) stage(lane, r % FTY, r / FTY, gi);
        const int q = wid * 32 + lane;
        if (q < 3 * FTY * FTZ) {
            const int r = q / 3, tx = FBX + (q - 3 * r);
            stage(tx, r % FTY, r / FTY, g.wi(i0 - 1 + tx));
        }
    }
    __syncthreads();
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y, k = k0 + threadIdx.z;
    if (i > mx - 2 || j > my - 2 || k > mz - 2) return;
    const bool npi = !g.pi, npj = !g.pj, npk = !g.pk;
    const bool quickDiv = p.div_scheme == TG_DIV_QUICK;
    const double nu = p.nu;
    const int t0 = ((threadIdx.z + 1) * FTY + threadIdx.y + 1) * FTX + threadIdx.x + 1;   // tile index of (k, j, i)
    auto S = [&](int dk, int dj, int di) { const int q = t0 + (dk * FTY + dj) * FTX + di; return R3<double>{su[0][q], su[1][q], su[2][q]}; };
    auto SN = [&](int dk, int dj, int di) { return sn[t0 + (dk * FTY + dj) * FTX + di]; };
    auto U = [&](int kk, int jj, int ii) { return ld3(s.ucat, g.id(kk, jj, ii)); };

    // ---- i face (k, j, fi), fi = i + e: ueqn_solvers.c:173-395 with Compute_du_i (inline.h:2748-2807)
    auto iface = [&](int fi, int e) {
        const int f = g.lin(k, j, fi);
        const bool edge = (fi == 0 || fi == mx - 2);
        R3<double> dv{0, 0, 0}, vv{0, 0, 0}, dc, de, dz;
        if (mode != 1) {
            dc = S(0, 0, e + 1) - S(0, 0, e);
            if (j == my - 2 && edge && (npj || npi))      de = 0.5 * (S(0, 0, e + 1) + S(0, 0, e) - S(0, -1, e + 1) - S(0, -1, e));
            else if (j == 1 && edge && (npj || npi))      de = 0.5 * (S(0, 1, e + 1) + S(0, 1, e) - S(0, 0, e + 1) - S(0, 0, e));
            else                                          de = 0.25 * (S(0, 1, e + 1) + S(0, 1, e) - S(0, -1, e + 1) - S(0, -1, e));
            if (k == mz - 2 && edge && (npk || npi))      dz = 0.5 * (S(0, 0, e + 1) + S(0, 0, e) - S(-1, 0, e + 1) - S(-1, 0, e));
            else if (k == 1 && edge && (npk || npi))      dz = 0.5 * (S(1, 0, e + 1) + S(1, 0, e) - S(0, 0, e + 1) - S(0, 0, e));
            else                                          dz = 0.25 * (S(1, 0, e + 1) + S(1, 0, e) - S(-1, 0, e + 1) - S(-1, 0, e));
        }
        if (mode != 2) {
            const double uc = s.ucont.x[f];
            if (quickDiv) {
                if (edge) {
                    int iL, iR;
                    if (g.pi && fi == mx - 2) { iR = mx + 2; iL = fi - 1; }
                    else if (fi == 0) { iL = fi; iR = fi + 2; }
                    else { iL = fi - 1; iR = fi + 1; }
                    dv = (-uc) * quick(U(k, j, iL), U(k, j, fi), U(k, j, fi + 1), U(k, j, iR), uc);
                } else dv = (-uc) * quick(S(0, 0, e - 1), S(0, 0, e), S(0, 0, e + 1), S(0, 0, e + 2), uc);
            } else dv = (-uc) * (0.5 * (S(0, 0, e) + S(0, 0, e + 1)));
        }
        if (mode != 1) {
            M nuEff;
            if (p.les) {
                const double nt = 0.5 * (SN(0, 0, e) + SN(0, 0, e + 1));
                if ((p.bc[TG_ILEFT] == TG_BC_SLIP && fi == 0) || (p.bc[TG_IRIGHT] == TG_BC_SLIP && fi == mx - 2)) nuEff = M(0);
                else nuEff = (M)(nu + nt);
            } else nuEff = (M)nu;
            if (AX) vv = cvta<double>(visc_flux_ax<M>(m.icsi.y[f], m.ieta.z[f], m.izet.x[f], 0, cvta<M>(dc), cvta<M>(de), cvta<M>(dz), m.iaj[f], nuEff));
            else vv = cvta<double>(visc_flux<M>(ld3(m.icsi, f), ld3(m.ieta, f), ld3(m.izet, f), 0, cvta<M>(dc), cvta<M>(de), cvta<M>(dz), m.iaj[f], nuEff));
        }
        st3(w.f1, f, cvta<F>(dv + vv));
    };
    // ---- j face (k, fj, i), fj = j + e: ueqn_solvers.c:397-602 with Compute_du_j (inline.h:2809-2869)
    auto jface = [&](int fj, int e) {
        const int f = g.lin(k, fj, i);
        const bool edge = (fj == 0 || fj == my - 2);
        R3<double> dv{0, 0, 0}, vv{0, 0, 0}, dc, de, dz;
        if (mode != 1) {
            de = S(0, e + 1, 0) - S(0, e, 0);
            if (i == mx - 2 && edge && (npi || npj))      dc = 0.5 * (S(0, e + 1, 0) + S(0, e, 0) - S(0, e + 1, -1) - S(0, e, -1));
            else if (i == 1 && edge && (npi || npj))      dc = 0.5 * (S(0, e + 1, 1) + S(0, e, 1) - S(0, e + 1, 0) - S(0, e, 0));
            else                                          dc = 0.25 * (S(0, e + 1, 1) + S(0, e, 1) - S(0, e + 1, -1) - S(0, e, -1));
            if (k == mz - 2 && edge && (npk || npj))      dz = 0.5 * (S(0, e + 1, 0) + S(0, e, 0) - S(-1, e + 1, 0) - S(-1, e, 0));
            else if (k == 1 && edge && (npk || npj))      dz = 0.5 * (S(1, e + 1, 0) + S(1, e, 0) - S(0, e + 1, 0) - S(0, e, 0));
            else                                          dz = 0.25 * (S(1, e + 1, 0) + S(1, e, 0) - S(-1, e + 1, 0) - S(-1, e, 0));
        }
        if (mode != 2) {
            const double uc = s.ucont.y[f];
            if (quickDiv) {
                if (edge) {
                    int jL, jR;
                    if (g.pj && fj == my - 2) { jR = my + 2; jL = fj - 1; }
                    else if (fj == 0) { jL = fj; jR = fj + 2; }
                    else { jL = fj - 1; jR = fj + 1; }
                    dv = (-uc) * quick(U(k, jL, i), U(k, fj, i), U(k, fj + 1, i), U(k, jR, i), uc);
                } else dv = (-uc) * quick(S(0, e - 1, 0), S(0, e, 0), S(0, e + 1, 0), S(0, e + 2, 0), uc);
            } else dv = (-uc) * (0.5 * (S(0, e, 0) + S(0, e + 1, 0)));
        }
        if (mode != 1) {
            M nuEff;
            R3<double> base{0, 0, 0};
            if (p.les) {
                const double nt = 0.5 * (SN(0, e, 0) + SN(0, e + 1, 0));
                // both j patches read the jLeft wall stress, ueqn_solvers.c:548-558
                if ((p.bc[TG_JLEFT] == TG_BC_WALL_SHUMANN && fj == 0) || (p.bc[TG_JRIGHT] == TG_BC_WALL_SHUMANN && fj == my - 2)) {
                    const int q = k * mx + i;
                    base = R3<double>{-s.twx[q], -s.twy[q], -s.twz[q]};
                    nuEff = (M)nu;
                } else if ((p.bc[TG_JLEFT] == TG_BC_SLIP && fj == 0) || (p.bc[TG_JRIGHT] == TG_BC_SLIP && fj == my - 2)) nuEff = M(0);
                else nuEff = (M)(nu + nt);
            } else nuEff = (M)nu;
            if (AX) vv = base + cvta<double>(visc_flux_ax<M>(m.jcsi.y[f], m.jeta.z[f], m.jzet.x[f], 1, cvta<M>(dc), cvta<M>(de), cvta<M>(dz), m.jaj[f], nuEff));
            else vv = base + cvta<double>(visc_flux<M>(ld3(m.jcsi, f), ld3(m.jeta, f), ld3(m.jzet, f), 1, cvta<M>(dc), cvta<M>(de), cvta<M>(dz), m.jaj[f], nuEff));
        }
        st3(w.f2, f, cvta<F>(dv + vv));
    };
    // ---- k face (fk, j, i), fk = k + e: ueqn_solvers.c:604-778 with Compute_du_k (inline.h:2871-2931)
    auto kface = [&](int fk, int e) {
        const int f = g.lin(fk, j, i);
        const bool edge = (fk == 0 || fk == mz - 2);
        R3<double> dv{0, 0, 0}, vv{0, 0, 0}, dc, de, dz;
        if (mode != 1) {
            dz = S(e + 1, 0, 0) - S(e, 0, 0);
            if (i == mx - 2 && edge && (npi || npk))      dc = 0.5 * (S(e + 1, 0, 0) + S(e, 0, 0) - S(e + 1, 0, -1) - S(e, 0, -1));
            else if (i == 1 && edge && (npi || npk))      dc = 0.5 * (S(e + 1, 0, 1) + S(e, 0, 1) - S(e + 1, 0, 0) - S(e, 0, 0));
            else                                          dc = 0.25 * (S(e + 1, 0, 1) + S(e, 0, 1) - S(e + 1, 0, -1) - S(e, 0, -1));
            if (j == my - 2 && edge && (npj || npk))      de = 0.5 * (S(e + 1, 0, 0) + S(e, 0, 0) - S(e + 1, -1, 0) - S(e, -1, 0));
            else if (j == 1 && edge && (npj || npk))      de = 0.5 * (S(e + 1, 1, 0) + S(e, 1, 0) - S(e + 1, 0, 0) - S(e, 0, 0));
            else                                          de = 0.25 * (S(e + 1, 1, 0) + S(e, 1, 0) - S(e + 1, -1, 0) - S(e, -1, 0));
        }
        if (mode != 2) {
            const double uc = s.ucont.z[f];
            if (quickDiv) {
                if (edge) {
                    int kL, kR;
                    if (g.pk && fk == mz - 2) { kR = mz + 2; kL = fk - 1; }
                    else if (fk == 0) { kL = fk; kR = fk + 2; }
                    else { kL = fk - 1; kR = fk + 1; }
                    dv = (-uc) * quick(U(kL, j, i), U(fk, j, i), U(fk + 1, j, i), U(kR, j, i), uc);
                } else dv = (-uc) * quick(S(e - 1, 0, 0), S(e, 0, 0), S(e + 1, 0, 0), S(e + 2, 0, 0), uc);
            } else dv = (-uc) * (0.5 * (S(e, 0, 0) + S(e + 1, 0, 0)));
        }
        if (mode != 1) {
            M nuEff;
            if (p.les) {
                const double nt = 0.5 * (SN(e, 0, 0) + SN(e + 1, 0, 0));
                if ((p.bc[TG_KLEFT] == TG_BC_SLIP && fk == 0) || (p.bc[TG_KRIGHT] == TG_BC_SLIP && fk == mz - 2)) nuEff = M(0);
                else nuEff = (M)(nu + nt);
            } else nuEff = (M)nu;
            if (AX) vv = cvta<double>(visc_flux_ax<M>(m.kcsi.y[f], m.keta.z[f], m.kzet.x[f], 2, cvta<M>(dc), cvta<M>(de), cvta<M>(dz), m.kaj[f], nuEff));
            else vv = cvta<double>(visc_flux<M>(ld3(m.kcsi, f), ld3(m.keta, f), ld3(m.kzet, f), 2, cvta<M>(dc), cvta<M>(de), cvta<M>(dz), m.kaj[f], nuEff));
        }
        st3(w.f3, f, cvta<F>(dv + vv));
    };
    // one emitted body per direction: the second pass is the face on the -
    // side of a cell next to a non-periodic 0 boundary
    const int ni = (i == 1 && npi) ? 2 : 1, nj = (j == 1 && npj) ? 2 : 1, nk = (k == 1 && npk) ? 2 : 1;
#pragma unroll 1
    for (int e = 0; e > -ni; e--) iface(i + e, e);
#pragma unroll 1
    for (int e = 0; e > -nj; e--) jface(j + e, e);
#pragma unroll 1
    for (int e = 0; e > -nk; e--) kface(k + e, e);
}

// Pass 2 (ueqn_solvers.c:825-947): divergence of the face fluxes of interior
// cell (k, j, i). A periodic direction reads its face 0 from face m-2
// (resetFacePeriodicFluxesVector, inline.h:5357-5451, applied to the fluxes).
template <class M>
__device__ __forceinline__ R3<M> cell_fp(const Grid &g, const FluxWork<M> &w, int k, int j, int i)
{
    const int c = g.lin(k, j, i), pl = g.mx * g.my;
    const int iw = (i == 1 && g.pi) ? c + g.mx - 3 : c - 1;
    const int js = (j == 1 && g.pj) ? c + (g.my - 3) * g.mx : c - g.mx;
    const int kb = (k == 1 && g.pk) ? c + (g.mz - 3) * pl : c - pl;
    R3<M> F;
    F.x = w.f1.x[c] - w.f1.x[iw] + w.f2.x[c] - w.f2.x[js] + w.f3.x[c] - w.f3.x[kb];
    F.y = w.f1.y[c] - w.f1.y[iw] + w.f2.y[c] - w.f2.y[js] + w.f3.y[c] - w.f3.y[kb];
    F.z = w.f1.z[c] - w.f1.z[iw] + w.f2.z[c] - w.f2.z[js] + w.f3.z[c] - w.f3.z[kb];
    return F;
}

template <class F>
__global__ void k_cell_fp(Grid g, FluxWork<F> w)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    st3(w.fp, g.lin(k, j, i), cell_fp(g, w, k, j, i));
}

// Explicit time update of one face value u with right-hand side r (UeqnFE,
// ueqn_solvers.c:1411-1442: U = r dt + U_o; UeqnRK4, ueqn_solvers.c:1446-1504,
// stage st: Utmp = U_o + b_st dt r (st = 0) or Utmp + b_st dt r, U = U_o +
// a_{st+1} dt r, after the last stage U = Utmp + b_3 dt r), in the order of
// the reference's VecScale / VecAXPY / VecWAXPY calls.
struct RkArgs {
    double cb, ca;      // b_st dt (FE: dt), a_{st+1} dt
    int first, last, fe;
};
__device__ __forceinline__ void rk_point(double *uc, double *ut, const double *uo, double r, const RkArgs &a)
{
    if (a.fe) { *uc = r * a.cb + *uo; return; }
    if (a.last) { *uc = a.cb * r + *ut; return; }
    const double o = *uo;
    if (a.first) *ut = a.cb * r + o;
    else *ut = *ut + a.cb * r;
    *uc = a.ca * r + o;
}

// Pass 3 (ueqn_solvers.c:1008-1035): rhs_face += scale * aj_face *
// central(S . fp) at the faces of interior cells, fp of the cell and of its
// +i, +j, +k neighbours read from pass 2. The neighbour beyond the last
// interior cell is the ghost cell, which holds the opposite first interior
// cell (periodic, resetCellPeriodicFluxes) or a copy of this cell
// (ueqn_solvers.c:949-990). With `fused` the kernel also forms
// the rest of ExplicitRhsU at these faces in the reference's order:
// Rhs = -dP (+ AB2 buoyancy) (ueqn_solvers.c:1305-1338), += turbine body
// force (ueqn_solvers.c:1340-1344), += FormU, += sourceU (body force), +=
// meanGradPForcing (ueqn_sources.c:3735-3822). MR:
// metric storage type; F: face-flux storage type. kind: 0 R += scale FormU;
// 1 the ExplicitRhsU value is stored in R; 2 it is not stored but masked at
// the non-resolved faces and applied at once by the explicit time update
// (rk_point, one RK4 stage or the FE step).
template <class MR, class F, int kind, bool AX>
__global__ void __launch_bounds__(256) k_rhs_faces(Grid g, FaceMet<MR> m, State s, FluxWork<F> w, V3f<double> R, double scale, Params p, int ab2, RkArgs rk)
{
    constexpr bool fused = kind >= 1;
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int c = g.lin(k, j, i);
    // the value of the three faces: stored, or masked and applied (kind 2)
    auto finish = [&](double ox, double oy, double oz) {
        if (kind == 2) {
            // resetNonResolvedCellFaces (inline.h:1674-1835) on the + faces of
            // the last interior cells of a non-periodic direction (kept for
            // outflow and on a zeroGradient patch)
            if (!g.pi && i == g.mx - 2 && !(p.bc[TG_IRIGHT] == TG_BC_ZERO_GRADIENT || s.ucont_o.x[c] > 0)) ox = 0.0;
            if (!g.pj && j == g.my - 2 && !(p.bc[TG_JRIGHT] == TG_BC_ZERO_GRADIENT || s.ucont_o.y[c] > 0)) oy = 0.0;
            if (!g.pk && k == g.mz - 2 && !(p.bc[TG_KRIGHT] == TG_BC_ZERO_GRADIENT || s.ucont_o.z[c] > 0)) oz = 0.0;
            rk_point(s.ucont.x + c, s.utmp.x + c, s.ucont_o.x + c, ox, rk);
            rk_point(s.ucont.y + c, s.utmp.y + c, s.ucont_o.y + c, oy, rk);
            rk_point(s.ucont.z + c, s.utmp.z + c, s.ucont_o.z + c, oz, rk);
        } else {
            R.x[c] = ox; R.y[c] = oy; R.z[c] = oz;
        }
    };
    R3<double> base;
    if (fused) {
        base = R3<double>{0.0 - s.dp.x[c], 0.0 - s.dp.y[c], 0.0 - s.dp.z[c]};
        if (p.buoyancy) {
            R3<double> b = ld3(s.btheta, c);
            if (ab2) {
                R3<double> bo = ld3(s.btheta_o, c);
                base = base + (3.0 / 2.0) * b;
                base = base + (-1.0 / 2.0) * bo;
            } else {
                base = base + 1.0 * b;
            }
        }
        if (p.farm) base = base + 1.0 * ld3(s.farmcont, c);
    } else {
        base = ld3(R, c);
    }
    // arithmetic in FP32 only when both the metrics and the fluxes are FP32
    using M = typename std::conditional<std::is_same<MR, float>::value && std::is_same<F, float>::value, float, double>::type;
    auto FP = [&](int kk, int jj, int ii) { return cvta<M>(ld3(w.fp, g.lin(kk, jj, ii))); };
    auto MT = [&](const V3f<MR> &v, int q) { return cvta<M>(ld3(v, q)); };
    const M sc = (M)scale, h = M(0.5);
    M v1, v2;
    double ox, oy, oz;
    if (AX) {
        // axis-aligned mesh: S . fp is csi.y fp.y, eta.z fp.z, zet.x fp.x
        const int pl = g.mx * g.my;
        const int ie = i < g.mx - 2 ? c + 1 : (g.pi ? g.lin(k, j, 1) : c);
        const int jn = j < g.my - 2 ? c + g.mx : (g.pj ? g.lin(k, 1, i) : c);
        const int kt = k < g.mz - 2 ? c + pl : (g.pk ? g.lin(1, j, i) : c);
        v1 = (M)m.csi.y[c] * (M)w.fp.y[c]; v2 = (M)m.csi.y[c + 1] * (M)w.fp.y[ie];
        ox = base.x + (double)(sc * (M)m.iaj[c] * (h * (v1 + v2)));
        v1 = (M)m.eta.z[c] * (M)w.fp.z[c]; v2 = (M)m.eta.z[c + g.mx] * (M)w.fp.z[jn];
        oy = base.y + (double)(sc * (M)m.jaj[c] * (h * (v1 + v2)));
        v1 = (M)m.zet.x[c] * (M)w.fp.x[c]; v2 = (M)m.zet.x[c + pl] * (M)w.fp.x[kt];
        oz = base.z + (double)(sc * (M)m.kaj[c] * (h * (v1 + v2)));
        if (fused && p.source) {
            const V3f<double> &f = s.source;
            ox += 1.0 * (0.5 * (f.y[c] + f.y[c + 1]) * (double)m.icsi.y[c]);
            oy += 1.0 * (0.5 * (f.z[c] + f.z[c + g.mx]) * (double)m.jeta.z[c]);
            oz += 1.0 * (0.5 * (f.x[c] + f.x[c + pl]) * (double)m.kzet.x[c]);
        }
        if (fused && p.mean_grad_p) {
            ox += (double)((M)p.mgp[1] * (M)m.icsi.y[c]);
            oy += (double)((M)p.mgp[2] * (M)m.jeta.z[c]);
            oz += (double)((M)p.mgp[0] * (M)m.kzet.x[c]);
        }
        finish(ox, oy, oz);
        return;
    }
    const R3<M> fpc = FP(k, j, i);
    { R3<M> fb = i < g.mx - 2 ? FP(k, j, i + 1) : (g.pi ? FP(k, j, 1) : fpc);
      R3<M> a = MT(m.csi, c), b = MT(m.csi, c + 1);
      v1 = a.x * fpc.x + a.y * fpc.y + a.z * fpc.z; v2 = b.x * fb.x + b.y * fb.y + b.z * fb.z;
      ox = base.x + (double)(sc * (M)m.iaj[c] * (h * (v1 + v2))); }
    { R3<M> fb = j < g.my - 2 ? FP(k, j + 1, i) : (g.pj ? FP(k, 1, i) : fpc);
      int n = c + g.mx; R3<M> a = MT(m.eta, c), b = MT(m.eta, n);
      v1 = a.x * fpc.x + a.y * fpc.y + a.z * fpc.z; v2 = b.x * fb.x + b.y * fb.y + b.z * fb.z;
      oy = base.y + (double)(sc * (M)m.jaj[c] * (h * (v1 + v2))); }
    { R3<M> fb = k < g.mz - 2 ? FP(k + 1, j, i) : (g.pk ? FP(1, j, i) : fpc);
      int n = c + g.mx * g.my; R3<M> a = MT(m.zet, c), b = MT(m.zet, n);
      v1 = a.x * fpc.x + a.y * fpc.y + a.z * fpc.z; v2 = b.x * fb.x + b.y * fb.y + b.z * fb.z;
      oz = base.z + (double)(sc * (M)m.kaj[c] * (h * (v1 + v2))); }
    if (fused && p.source) {
        // sourceU (ueqn_solvers.c:1369, ueqn_sources.c:2884-2980): central body force . face area, FP64
        const V3f<double> &f = s.source;
        const int ie = c + 1, jn = c + g.mx, kt = c + g.mx * g.my;
        R3<double> a = cvta<double>(ld3(m.icsi, c)), b = cvta<double>(ld3(m.jeta, c)), d = cvta<double>(ld3(m.kzet, c));
        ox += 1.0 * (0.5 * (f.x[c] + f.x[ie]) * a.x + 0.5 * (f.y[c] + f.y[ie]) * a.y + 0.5 * (f.z[c] + f.z[ie]) * a.z);
        oy += 1.0 * (0.5 * (f.x[c] + f.x[jn]) * b.x + 0.5 * (f.y[c] + f.y[jn]) * b.y + 0.5 * (f.z[c] + f.z[jn]) * b.z);
        oz += 1.0 * (0.5 * (f.x[c] + f.x[kt]) * d.x + 0.5 * (f.y[c] + f.y[kt]) * d.y + 0.5 * (f.z[c] + f.z[kt]) * d.z);
    }
    if (fused && p.mean_grad_p) {
        R3<M> a = MT(m.icsi, c), b = MT(m.jeta, c), d = MT(m.kzet, c);
        const M g0 = (M)p.mgp[0], g1 = (M)p.mgp[1], g2 = (M)p.mgp[2];
        ox += (double)(g0 * a.x + g1 * a.y + g2 * a.z);
        oy += (double)(g0 * b.x + g1 * b.y + g2 * b.z);
        oz += (double)(g0 * d.x + g1 * d.y + g2 * d.z);
    }
    finish(ox, oy, oz);
}

// the explicit time update of the points outside the interior cells, whose
// right-hand side is zero (never formed, or reset at the non-resolved faces):
// rk_point with r = 0 on the six boundary planes of the DMDA box, each point
// once
__global__ void k_rk_shell(Grid g, State s, RkArgs rk)
{
    const int patch = blockIdx.z, dir = patch >> 1, right = patch & 1;
    const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int i, j, k;
    if (dir == 0) { if (a >= g.my || b >= g.mz) return; i = right ? g.mx - 1 : 0; j = a; k = b; }
    else if (dir == 1) { if (a >= g.mx - 2 || b >= g.mz) return; j = right ? g.my - 1 : 0; i = a + 1; k = b; }
    else { if (a >= g.mx - 2 || b >= g.my - 2) return; k = right ? g.mz - 1 : 0; i = a + 1; j = b + 1; }
    const int c = g.lin(k, j, i);
    rk_point(s.ucont.x + c, s.utmp.x + c, s.ucont_o.x + c, 0.0, rk);
    rk_point(s.ucont.y + c, s.utmp.y + c, s.ucont_o.y + c, 0.0, rk);
    rk_point(s.ucont.z + c, s.utmp.z + c, s.ucont_o.z + c, 0.0, rk);
}

// ------------------------------------------------------------------------
// adjustFluxesLocal (ueqn.c:748-1135) on the inflow/outflow patches
// (fixedValue, zeroGradient: the non-periodic, non-wall patch type 0). The
// faces of a patch are split by the sign of their flux into inflow (into the
// domain) and outflow; the outflow faces take the imbalance FluxOut - FluxIn
// in proportion to their own flux, so that the boundary fluxes sum to zero.
// Pass 1 (blockIdx.y = patch): per-block inflow/outflow sums, faces of zero
// (or non-finite) flux set to zero; pass 2 (one block): the totals in a fixed
// order into sc[0] (in) and sc[1] (out); pass 3: the outflow correction.
// ------------------------------------------------------------------------
constexpr int AF_BLOCKS = 32;   // pass-1 blocks per patch

__device__ __forceinline__ bool inout_patch(const Params &p, int patch)
{
    return p.bc[patch] >= TG_BC_FIXED_VALUE;
}
// the boundary face (a, b) of a patch (interior range 1..m-2 in both plane
// directions): its contravariant component array and index
__device__ __forceinline__ double *patch_face(const Grid &g, const State &s, int dir, int right, int a, int b, int &f)
{
    if (dir == 2) { f = g.lin(right ? g.mz - 2 : 0, b, a); return s.ucont.z; }
    if (dir == 1) { f = g.lin(b, right ? g.my - 2 : 0, a); return s.ucont.y; }
    f = g.lin(b, a, right ? g.mx - 2 : 0);
    return s.ucont.x;
}
__device__ __forceinline__ void patch_extent(const Grid &g, int dir, int &na, int &nb)
{
    na = (dir == 0 ? g.my : g.mx) - 2;
    nb = (dir == 2 ? g.my : g.mz) - 2;
}

__global__ void __launch_bounds__(256) k_flux_sums(Grid g, State s, Params p, double *part)
{
    const int patch = blockIdx.y, dir = patch >> 1, right = patch & 1;
    double v[2] = {0.0, 0.0};    // inflow, outflow
    if (inout_patch(p, patch)) {
        int na, nb;
        patch_extent(g, dir, na, nb);
        for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na * nb; t += gridDim.x * blockDim.x) {
            int f;
            double *u = patch_face(g, s, dir, right, t % na + 1, t / na + 1, f);
            const double x = u[f];
            if (x > 0.0) v[right ? 1 : 0] += x;
            else if (x < 0.0) v[right ? 0 : 1] += -x;
            else u[f] = 0.0;
        }
    }
    block_reduce<256>(v, RedSum{}, RedSum{});
    if (threadIdx.x == 0) {
        const int q = patch * gridDim.x + blockIdx.x;
        part[2 * q] = v[0];
        part[2 * q + 1] = v[1];
    }
}

__global__ void __launch_bounds__(256) k_flux_total(const double *part, int n, double *sc)
{
    double v[2] = {0.0, 0.0};
    for (int q = threadIdx.x; q < n; q += blockDim.x) { v[0] += part[2 * q]; v[1] += part[2 * q + 1]; }
    block_reduce<256>(v, RedSum{}, RedSum{});
    if (threadIdx.x == 0) { sc[0] = v[0]; sc[1] = v[1]; }
}

__global__ void k_flux_correct(Grid g, State s, Params p, const double *sc)
{
    const int patch = blockIdx.y, dir = patch >> 1, right = patch & 1;
    if (!inout_patch(p, patch)) return;
    int na, nb;
    patch_extent(g, dir, na, nb);
    const double in = sc[0], out = sc[1], gf = out - in;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na * nb; t += gridDim.x * blockDim.x) {
        int f;
        double *u = patch_face(g, s, dir, right, t % na + 1, t / na + 1, f);
        const double x = u[f];
        if (!right && x < 0.0) u[f] = x + gf * (-x / out);
        if (right && x > 0.0) u[f] = x - gf * (x / out);
    }
}

// resetNonResolvedCellFaces (inline.h:1674-1835) on the boundary planes of one
// direction: face 0 kept only for outflow or on a zeroGradient patch, face m-1
// unused, face m-2 of a non-periodic direction kept only for outflow or on a
// zeroGradient patch.
__global__ void k_non_resolved(Grid g, State s, Params p, int dir)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = dir == 0 ? g.my : g.mx, nb = dir == 2 ? g.my : g.mz;
    if (a >= na || b >= nb) return;
    int m = dir == 0 ? g.mx : (dir == 1 ? g.my : g.mz);
    int per = dir == 0 ? g.pi : (dir == 1 ? g.pj : g.pk);
    double *v = dir == 0 ? s.rhs.x : (dir == 1 ? s.rhs.y : s.rhs.z);
    const double *uo = dir == 0 ? s.ucont_o.x : (dir == 1 ? s.ucont_o.y : s.ucont_o.z);
    auto at = [&](int l) { return dir == 0 ? g.lin(b, a, l) : (dir == 1 ? g.lin(b, l, a) : g.lin(l, b, a)); };
    const bool zgl = p.bc[2 * dir] == TG_BC_ZERO_GRADIENT, zgr = p.bc[2 * dir + 1] == TG_BC_ZERO_GRADIENT;
    { int q = at(0); if (!(zgl || uo[q] < 0)) v[q] = 0.0; }
    { int q = at(m - 1); v[q] = 0.0; }
    if (!per) { int q = at(m - 2); if (!(zgr || uo[q] > 0)) v[q] = 0.0; }
}


// ------------------------------------------------------------------------
// ProjectVelocity (peqn.c:2495-2905): V = V* - dt G(phi) with the full
// metric tensor; faces 0 and m-2 skipped unless periodic.
// ------------------------------------------------------------------------
template <class M>
__global__ void k_project(Grid g, FaceMet<M> m, State s, double dt, bool ax)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    const int mx = g.mx, my = g.my, mz = g.mz;
    int f = g.lin(k, j, i);
    auto F = [&](int kk, int jj, int ii) { return s.phi[g.id(kk, jj, ii)]; };
    if (ax) {
        // axis-aligned mesh: only the normal derivative of phi has a metric weight
        if (j > 0 && k > 0 && ((i > 0 && i < mx - 2) || g.pi)) {
            const double c1 = (double)m.icsi.y[f];
            s.ucont.x[f] -= ((F(k, j, i + 1) - F(k, j, i)) * (c1 * c1) * (double)m.iaj[f]) * dt;
        }
        if (i > 0 && k > 0 && ((j > 0 && j < my - 2) || g.pj)) {
            const double e2 = (double)m.jeta.z[f];
            s.ucont.y[f] -= ((F(k, j + 1, i) - F(k, j, i)) * (e2 * e2) * (double)m.jaj[f]) * dt;
        }
        if (i > 0 && j > 0 && ((k > 0 && k < mz - 2) || g.pk)) {
            const double z3 = (double)m.kzet.x[f];
            s.ucont.z[f] -= ((F(k + 1, j, i) - F(k, j, i)) * (z3 * z3) * (double)m.kaj[f]) * dt;
        }
        return;
    }
    if (j > 0 && k > 0 && ((i > 0 && i < mx - 2) || g.pi)) {
        double dpdc = F(k, j, i + 1) - F(k, j, i), dpde, dpdz;
        if (j == my - 2)      dpde = (F(k, j, i) + F(k, j, i + 1) - F(k, j - 1, i) - F(k, j - 1, i + 1)) * 0.5;
        else if (j == 1)      dpde = (F(k, j + 1, i) + F(k, j + 1, i + 1) - F(k, j, i) - F(k, j, i + 1)) * 0.5;
        else                  dpde = (F(k, j + 1, i) + F(k, j + 1, i + 1) - F(k, j - 1, i) - F(k, j - 1, i + 1)) * 0.25;
        if (k == mz - 2)      dpdz = (F(k, j, i) + F(k, j, i + 1) - F(k - 1, j, i) - F(k - 1, j, i + 1)) * 0.5;
        else if (k == 1)      dpdz = (F(k + 1, j, i) + F(k + 1, j, i + 1) - F(k, j, i) - F(k, j, i + 1)) * 0.5;
        else                  dpdz = (F(k + 1, j, i) + F(k + 1, j, i + 1) - F(k - 1, j, i) - F(k - 1, j, i + 1)) * 0.25;
        R3<double> c1 = cvta<double>(ld3(m.icsi, f)), e1 = cvta<double>(ld3(m.ieta, f)), z1 = cvta<double>(ld3(m.izet, f));
        double a = (double)m.iaj[f];
        s.ucont.x[f] -= (dpdc * (c1.x * c1.x + c1.y * c1.y + c1.z * c1.z) * a
                       + dpde * (e1.x * c1.x + e1.y * c1.y + e1.z * c1.z) * a
                       + dpdz * (z1.x * c1.x + z1.y * c1.y + z1.z * c1.z) * a) * dt;
    }
    if (i > 0 && k > 0 && ((j > 0 && j < my - 2) || g.pj)) {
        double dpdc, dpde = F(k, j + 1, i) - F(k, j, i), dpdz;
        if (i == mx - 2)      dpdc = (F(k, j, i) + F(k, j + 1, i) - F(k, j, i - 1) - F(k, j + 1, i - 1)) * 0.5;
        else if (i == 1)      dpdc = (F(k, j, i + 1) + F(k, j + 1, i + 1) - F(k, j, i) - F(k, j + 1, i)) * 0.5;
        else                  dpdc = (F(k, j, i + 1) + F(k, j + 1, i + 1) - F(k, j, i - 1) - F(k, j + 1, i - 1)) * 0.25;
        if (k == mz - 2)      dpdz = (F(k, j, i) + F(k, j + 1, i) - F(k - 1, j, i) - F(k - 1, j + 1, i)) * 0.5;
        else if (k == 1)      dpdz = (F(k + 1, j, i) + F(k + 1, j + 1, i) - F(k, j, i) - F(k, j + 1, i)) * 0.5;
        else                  dpdz = (F(k + 1, j, i) + F(k + 1, j + 1, i) - F(k - 1, j, i) - F(k - 1, j + 1, i)) * 0.25;
        R3<double> c2 = cvta<double>(ld3(m.jcsi, f)), e2 = cvta<double>(ld3(m.jeta, f)), z2 = cvta<double>(ld3(m.jzet, f));
        double a = (double)m.jaj[f];
        s.ucont.y[f] -= (dpdc * (c2.x * e2.x + c2.y * e2.y + c2.z * e2.z) * a
                       + dpde * (e2.x * e2.x + e2.y * e2.y + e2.z * e2.z) * a
                       + dpdz * (z2.x * e2.x + z2.y * e2.y + z2.z * e2.z) * a) * dt;
    }
    if (i > 0 && j > 0 && ((k > 0 && k < mz - 2) || g.pk)) {
        double dpdc, dpde, dpdz = F(k + 1, j, i) - F(k, j, i);
        if (i == mx - 2)      dpdc = (F(k, j, i) + F(k + 1, j, i) - F(k, j, i - 1) - F(k + 1, j, i - 1)) * 0.5;
        else if (i == 1)      dpdc = (F(k, j, i + 1) + F(k + 1, j, i + 1) - F(k, j, i) - F(k + 1, j, i)) * 0.5;
        else                  dpdc = (F(k, j, i + 1) + F(k + 1, j, i + 1) - F(k, j, i - 1) - F(k + 1, j, i - 1)) * 0.25;
        if (j == my - 2)      dpde = (F(k, j, i) + F(k + 1, j, i) - F(k, j - 1, i) - F(k + 1, j - 1, i)) * 0.5;
        else if (j == 1)      dpde = (F(k, j + 1, i) + F(k + 1, j + 1, i) - F(k, j, i) - F(k + 1, j, i)) * 0.5;
        else                  dpde = (F(k, j + 1, i) + F(k + 1, j + 1, i) - F(k, j - 1, i) - F(k + 1, j - 1, i)) * 0.25;
        R3<double> c3 = cvta<double>(ld3(m.kcsi, f)), e3 = cvta<double>(ld3(m.keta, f)), z3 = cvta<double>(ld3(m.kzet, f));
        double a = (double)m.kaj[f];
        s.ucont.z[f] -= (dpdc * (c3.x * z3.x + c3.y * z3.y + c3.z * z3.z) * a
                       + dpde * (e3.x * z3.x + e3.y * z3.y + e3.z * z3.z) * a
                       + dpdz * (z3.x * z3.x + z3.y * z3.y + z3.z * z3.z) * a) * dt;
    }
}

// UpdatePressure (peqn.c:2909-2962): p += phi at interior cells
__global__ void k_update_pressure(Grid g, State s)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int c = g.lin(k, j, i);
    s.p[c] += s.phi[c];
}

// SyncPressureAcrossDomains (overset.c:263-315): p -= p[1][1][1] everywhere
__global__ void k_gauge(int64_t n, double *p, const double *ref_cell)
{
    double ref = *ref_cell;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) p[q] -= ref;
}
__global__ void k_copy1(const double *src, double *dst) { dst[0] = src[0]; }

// ContinuityErrorsOptimized (peqn.c:4114-4181): max |div(V)| * aj, block partials
__global__ void __launch_bounds__(256) k_div_partial(Grid g, Metrics m, State s, double *part)
{
    int nI = g.mx - 2, nJ = g.my - 2, nK = g.mz - 2;
    int64_t n = (int64_t)nI * nJ * nK;
    double mm = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(t % nI) + 1; int64_t r = t / nI; int j = (int)(r % nJ) + 1; int k = (int)(r / nJ) + 1;
        int c = g.lin(k, j, i);
        double d = fabs((s.ucont.x[c] - s.ucont.x[c - 1] + s.ucont.y[c] - s.ucont.y[c - g.mx]
                        + s.ucont.z[c] - s.ucont.z[c - g.mx * g.my]) * m.aj[c]);
        mm = nanmax(mm, d);
    }
    double v[1] = {mm};
    block_reduce<256>(v, RedNanMax{});
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}
__global__ void __launch_bounds__(256) k_max_final(const double *part, int nb, double *out)
{
    double v[1] = {0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v[0] = nanmax(v[0], part[b]);
    block_reduce<256>(v, RedNanMax{});
    if (threadIdx.x == 0) out[0] = v[0];
}

// initial face fluxes from the cell-centre velocity (initialField.c:1140-1190)
__global__ void k_init_faces(Grid g, Metrics m, State s)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int f = g.lin(k, j, i);
    R3<double> a = ld3(s.ucat, f);
    if (j >= 1 && k >= 1) {
        R3<double> b = ld3(s.ucat, f + 1), S = ld3(m.icsi, f);
        R3<double> uf{0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z)};
        s.ucont.x[f] = uf.x * S.x + uf.y * S.y + uf.z * S.z;
    }
    if (i >= 1 && k >= 1) {
        R3<double> b = ld3(s.ucat, f + g.mx), S = ld3(m.jeta, f);
        R3<double> uf{0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z)};
        s.ucont.y[f] = uf.x * S.x + uf.y * S.y + uf.z * S.z;
    }
    if (i >= 1 && j >= 1) {
        R3<double> b = ld3(s.ucat, f + g.mx * g.my), S = ld3(m.kzet, f);
        R3<double> uf{0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z)};
        s.ucont.z[f] = uf.x * S.x + uf.y * S.y + uf.z * S.z;
    }
}

inline dim3 gi(const Grid &g) { return grid3(g.mx - 2, g.my - 2, g.mz - 2); }
inline dim3 ga(const Grid &g) { return grid3(g.mx, g.my, g.mz); }
inline dim3 gf(const Grid &g) { return grid3(g.mx - 1, g.my - 1, g.mz - 1); }
inline int nblk(int64_t n) { int64_t b = (n + 255) / 256; return (int)(b < 148 * 16 ? b : 148 * 16); }

}  // namespace

// ============================================================================ host wrappers
// contravariantToCartesian of the stage entry point and of the end of the
// step, in FP64 in every mode: with FP32 metric copies here the relative L2
// error of p against the FP64 oracle rose to 3.3e-6 in 5 steps (ABL 16x16x12)
void contra_to_cart(tg_ctx *C)
{
    TG_PROF(C, "contra_to_cart_final", k_contra_to_cart<double, double><<<gi(C->g), block3(), 0, C->stream>>>(C->g, C->fm64, C->s, C->axis_aligned));
}

// contravariantToCartesian inside the momentum stages, at the precision the
// context's policy gives it
void contra_to_cart_stage(tg_ctx *C)
{
    const dim3 gr = gi(C->g);
    if (C->pol.contra_a32) TG_PROF(C, "contra_to_cart", k_contra_to_cart<float, float><<<gr, block3(), 0, C->stream>>>(C->g, C->fm32, C->s, C->axis_aligned));
    else if (C->pol.contra_m32) TG_PROF(C, "contra_to_cart", k_contra_to_cart<double, float><<<gr, block3(), 0, C->stream>>>(C->g, C->fm32, C->s, C->axis_aligned));
    else TG_PROF(C, "contra_to_cart", k_contra_to_cart<double, double><<<gr, block3(), 0, C->stream>>>(C->g, C->fm64, C->s, C->axis_aligned));
}

// Precision of each momentum stage in the mixed mode. Every momentum stencil
// reads the FP32 metric copies (half the metric bytes, which dominate the
// stencils' traffic). Two things stay FP64 because the pressure field is set by
// the divergence of the momentum right-hand side, in which the convective
// fluxes nearly cancel: the arithmetic of contravariantToCartesian, FormU's
// convective fluxes and the face assembly, and the storage of the face-flux
// planes. The projection keeps FP64 metrics too: with FP32 metric copies its
// correction is no longer the exact gradient whose divergence the FP64 Poisson
// operator balanced, and the left-over divergence raised the relative L2 error
// of p to 3.3e-6 in 5 steps (ABL 16x16x12). Measured against the FP64 oracle
// (ABL 48x48x32, 20 steps) FP32
// storage of the face fluxes alone raised the relative L2 error of p from
// 1.3e-7 to 4.9e-6; FP32 Cramer arithmetic raised it to 6e-7 in 5 steps.
static void set_policy(tg_ctx *C)
{
    C->pol.contra_m32 = C->mixed;
    C->pol.contra_a32 = false;
    C->pol.visc32 = C->mixed;
    C->pol.flux32 = false;
    C->pol.rhs32 = C->mixed;
    C->pol.smag32 = C->mixed;
    C->pol.gradp32 = C->mixed;
    C->pol.proj32 = false;
}

// Smagorinsky filter width squared of every cell from its Jacobian, in the
// arithmetic of the eddy-viscosity kernel (les.c:2204-2514)
template <class T>
__global__ void k_filter2(int64_t n, const T *aj, T *out)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const T filter = pow(T(1) / aj[q], T(1) / T(3));
        out[q] = pow(filter, T(2));
    }
}

void refresh_filter(tg_ctx *C)
{
    const int64_t G = C->g.size();
    k_filter2<double><<<nblk(G), 256, 0, C->stream>>>(G, C->fm64.aj, C->fm64.flt2);
}

void alloc_precision_work(tg_ctx *C)
{
    const size_t G = (size_t)C->g.size();
    const Metrics &m = C->m;
    C->fm64 = FaceMet<double>{m.csi, m.eta, m.zet, m.icsi, m.ieta, m.izet, m.jcsi, m.jeta, m.jzet,
                              m.kcsi, m.keta, m.kzet, m.aj, m.iaj, m.jaj, m.kaj, dallocd(C, G)};
    set_policy(C);
    if (!C->pol.flux32) C->fw64 = FluxWork<double>{dalloc3(C, G), dalloc3(C, G), dalloc3(C, G), dalloc3(C, G)};
    if (!C->mixed) return;
    auto f3 = [&]() {
        float *a = (float *)dalloc(C, 3 * G * sizeof(float));
        return V3f<float>{a, a + G, a + 2 * G};
    };
    FaceMet<float> &f = C->fm32;
    V3f<float> *vv[] = {&f.csi, &f.eta, &f.zet, &f.icsi, &f.ieta, &f.izet, &f.jcsi, &f.jeta, &f.jzet, &f.kcsi, &f.keta, &f.kzet};
    for (auto *v : vv) *v = f3();
    float **ss[] = {&f.aj, &f.iaj, &f.jaj, &f.kaj, &f.flt2};
    for (auto **v : ss) *v = (float *)dalloc(C, G * sizeof(float));
    if (C->pol.flux32) C->fw32 = FluxWork<float>{f3(), f3(), f3(), f3()};
    C->met32_stale = true;
}

void refresh_met32(tg_ctx *C)
{
    if (!C->mixed || !C->met32_stale) return;
    const int64_t G = C->g.size();
    const FaceMet<double> &a = C->fm64;
    const FaceMet<float> &b = C->fm32;
    const V3f<double> va[] = {a.csi, a.eta, a.zet, a.icsi, a.ieta, a.izet, a.jcsi, a.jeta, a.jzet, a.kcsi, a.keta, a.kzet};
    const V3f<float> vb[] = {b.csi, b.eta, b.zet, b.icsi, b.ieta, b.izet, b.jcsi, b.jeta, b.jzet, b.kcsi, b.keta, b.kzet};
    for (int q = 0; q < 12; q++) {
        k_to_f32<<<nblk(G), 256, 0, C->stream>>>(G, va[q].x, vb[q].x);
        k_to_f32<<<nblk(G), 256, 0, C->stream>>>(G, va[q].y, vb[q].y);
        k_to_f32<<<nblk(G), 256, 0, C->stream>>>(G, va[q].z, vb[q].z);
    }
    const double *sa[] = {a.aj, a.iaj, a.jaj, a.kaj};
    float *sb[] = {b.aj, b.iaj, b.jaj, b.kaj};
    for (int q = 0; q < 4; q++) k_to_f32<<<nblk(G), 256, 0, C->stream>>>(G, sa[q], sb[q]);
    k_filter2<float><<<nblk(G), 256, 0, C->stream>>>(G, b.aj, b.flt2);
    TG_CUDA(cudaGetLastError());
    C->met32_stale = false;
}

void reset_cell_periodic(tg_ctx *C, V3f<double> v) { periodic_copy<3, double>(C, v.x, v.y, v.z, 0); }
void reset_cell_periodic_s(tg_ctx *C, double *v) { periodic_copy<1, double>(C, v, nullptr, nullptr, 0); }
void reset_face_periodic(tg_ctx *C, V3f<double> v) { periodic_copy<3, double>(C, v.x, v.y, v.z, 1); }

void reset_no_penetration(tg_ctx *C)
{
    const Grid g = C->g;
    const int *bc = C->prm.bc;
    auto w = [](int t) { return t == TG_BC_NOSLIP || t == TG_BC_SLIP || t == TG_BC_WALL_SHUMANN; };
    for (int d = 0; d < 3; d++) {
        int l = w(bc[2 * d]), r = w(bc[2 * d + 1]);
        if (!l && !r) continue;
        int na = d == 0 ? g.my : g.mx, nb = d == 2 ? g.my : g.mz;
        TG_PROF(C, "bc_no_penetration", k_no_penetration<<<g2(na, nb), b2, 0, C->stream>>>(g, C->s, d, l, r));
    }
}

void update_cartesian_bcs(tg_ctx *C)
{
    const Grid g = C->g;
    int na = std::max(g.mx, g.my) - 2, nb = std::max(g.my, g.mz) - 2;
    dim3 grid((na + 31) / 32, (nb + 7) / 8, 6);
    TG_PROF(C, "bc_cartesian", k_cartesian_bcs<<<grid, b2, 0, C->stream>>>(g, C->m, C->s, C->prm));
}

void update_contravariant_bcs(tg_ctx *C)
{
    const Grid g = C->g;
    for (int d = 0; d < 3; d++) {
        int na = d == 0 ? g.my : g.mx, nb = d == 2 ? g.my : g.mz;
        if (C->prm.bc[2 * d] == TG_BC_PERIODIC) k_contra_bc_periodic<<<g2(na, nb), b2, 0, C->stream>>>(g, C->s, d);
        TG_PROF(C, "bc_contravariant", k_contra_bc_faces<<<g2(na, nb), b2, 0, C->stream>>>(g, C->m, C->s, C->prm, d));
    }
}

void adjust_fluxes(tg_ctx *C)
{
    bool any = false;
    for (int q = 0; q < 6; q++) any |= C->prm.bc[q] >= TG_BC_FIXED_VALUE;
    if (!any) return;
    const Grid g = C->g;
    static_assert(6 * AF_BLOCKS * 2 <= 4 * 148 * 4, "partials fit the reduction scratch");
    TG_PROF(C, "bc_adjust_fluxes", k_flux_sums<<<dim3(AF_BLOCKS, 6), 256, 0, C->stream>>>(g, C->s, C->prm, C->d_red));
    k_flux_total<<<1, 256, 0, C->stream>>>(C->d_red, 6 * AF_BLOCKS, C->d_scal + SC_FLUX);
    TG_PROF(C, "bc_adjust_fluxes", k_flux_correct<<<dim3(AF_BLOCKS, 6), 256, 0, C->stream>>>(g, C->s, C->prm, C->d_scal + SC_FLUX));
}

void update_scalar_ghosts(tg_ctx *C, double *v)
{
    const Grid g = C->g;
    TG_PROF(C, "bc_scalar_ghosts", k_scalar_ghosts<<<g2(g.my, g.mz), b2, 0, C->stream>>>(g, v, 0));
    TG_PROF(C, "bc_scalar_ghosts", k_scalar_ghosts<<<g2(g.mx, g.mz), b2, 0, C->stream>>>(g, v, 1));
    TG_PROF(C, "bc_scalar_ghosts", k_scalar_ghosts<<<g2(g.mx, g.my), b2, 0, C->stream>>>(g, v, 2));
}

void update_nut(tg_ctx *C)
{
    const Grid g = C->g;
    TG_CUDA(cudaMemsetAsync(C->s.nut, 0, sizeof(double) * g.size(), C->stream));
    refresh_met32(C);
    if (C->pol.smag32) TG_PROF(C, "smagorinsky", k_smagorinsky<float><<<gi(g), block3(), 0, C->stream>>>(g, C->fm32, C->s, C->prm, C->axis_aligned));
    else TG_PROF(C, "smagorinsky", k_smagorinsky<double><<<gi(g), block3(), 0, C->stream>>>(g, C->fm64, C->s, C->prm, C->axis_aligned));
    int na = std::max(g.mx, g.my) - 2, nb = std::max(g.my, g.mz) - 2;
    dim3 grid((na + 31) / 32, (nb + 7) / 8, 6);
    TG_PROF(C, "bc_nut", k_nut_bcs<<<grid, b2, 0, C->stream>>>(g, C->s, C->prm));
}

void update_wall_models(tg_ctx *C)
{
    if (!C->prm.les || C->prm.bc[TG_JLEFT] != TG_BC_WALL_SHUMANN) return;
    const Grid g = C->g;
    const int nb = 148;
    TG_PROF(C, "wall_plane_sums", k_wall_plane_sums<<<nb, 256, 0, C->stream>>>(g, C->m, C->s, C->prm, C->d_red));
    k_wall_ustar<<<1, 32, 0, C->stream>>>(g, C->prm, C->d_red, nb, C->d_scal + 8);
    dim3 grid((g.mx - 2 + 31) / 32, (g.mz - 2 + 7) / 8);
    if (!C->ufilt_set) {
        k_wall_init_filter<<<grid, b2, 0, C->stream>>>(g, C->m, C->s);
        C->ufilt_set = true;
    }
    TG_PROF(C, "wall_stress", k_wall_stress<<<grid, b2, 0, C->stream>>>(g, C->m, C->s, C->prm, C->d_scal + 8, C->d_scal + SC_IT));
}

// GradP writes the faces of interior cells; dP is zero elsewhere from its
// allocation unless a caller wrote it
void grad_p(tg_ctx *C)
{
    if (C->clear_dp) {
        TG_CUDA(cudaMemsetAsync(C->s.dp.x, 0, 3 * sizeof(double) * C->g.size(), C->stream));
        C->clear_dp = false;
    }
    refresh_met32(C);
    if (C->pol.gradp32) TG_PROF(C, "grad_p", k_grad_p<float><<<gi(C->g), block3(), 0, C->stream>>>(C->g, C->fm32, C->s, C->axis_aligned));
    else TG_PROF(C, "grad_p", k_grad_p<double><<<gi(C->g), block3(), 0, C->stream>>>(C->g, C->fm64, C->s, C->axis_aligned));
}

void buoyancy(tg_ctx *C)
{
    if (C->cfg.p_tilde)   // ghGradRhoK (teqn.c:278), FP64
        TG_PROF(C, "gh_grad_rhok", (k_grad_p<double, true><<<gi(C->g), block3(), 0, C->stream>>>(C->g, C->fm64, C->s, false, C->node_z, C->prm.t_ref)));
    else
        k_buoyancy<<<ga(C->g), block3(), 0, C->stream>>>(C->g, C->m, C->s, C->prm);
}

// FormU pass 1 (face fluxes) at the precision of the context's policy.
// Pass 2 (k_cell_fp) follows; the flux planes are only read at the points
// pass 1 writes, fp only at interior cells.
template <int mode, bool AX>
static void face_fluxes(tg_ctx *C, dim3 gr)
{
    const Grid g = C->g;
    const auto &P = C->pol;
    if (P.visc32 && P.flux32) TG_PROF(C, "formu_face_fluxes", (k_face_fluxes<float, float, mode, AX><<<gr, dim3(FBX, FBY, FBZ), 0, C->stream>>>(g, C->fm32, C->s, C->fw32, C->prm)));
    else if (P.visc32) TG_PROF(C, "formu_face_fluxes", (k_face_fluxes<float, double, mode, AX><<<gr, dim3(FBX, FBY, FBZ), 0, C->stream>>>(g, C->fm32, C->s, C->fw64, C->prm)));
    else if (P.flux32) TG_PROF(C, "formu_face_fluxes", (k_face_fluxes<double, float, mode, AX><<<gr, dim3(FBX, FBY, FBZ), 0, C->stream>>>(g, C->fm64, C->s, C->fw32, C->prm)));
    else TG_PROF(C, "formu_face_fluxes", (k_face_fluxes<double, double, mode, AX><<<gr, dim3(FBX, FBY, FBZ), 0, C->stream>>>(g, C->fm64, C->s, C->fw64, C->prm)));
}

static void form_u_faces(tg_ctx *C, int mode)
{
    const Grid g = C->g;
    refresh_met32(C);
    // one thread per interior cell (k_face_fluxes)
    const dim3 gr((g.mx - 2 + FBX - 1) / FBX, (g.my - 2 + FBY - 1) / FBY, (g.mz - 2 + FBZ - 1) / FBZ);
    const auto &P = C->pol;
    const bool ax = C->axis_aligned;
    if (mode == 1) { if (ax) face_fluxes<1, true>(C, gr); else face_fluxes<1, false>(C, gr); }
    else if (mode == 2) { if (ax) face_fluxes<2, true>(C, gr); else face_fluxes<2, false>(C, gr); }
    else { if (ax) face_fluxes<0, true>(C, gr); else face_fluxes<0, false>(C, gr); }
    if (P.flux32) TG_PROF(C, "formu_cell_fp", k_cell_fp<float><<<gi(g), block3(), 0, C->stream>>>(g, C->fw32));
    else TG_PROF(C, "formu_cell_fp", k_cell_fp<double><<<gi(g), block3(), 0, C->stream>>>(g, C->fw64));
}

template <int fused, bool AX>
static void rhs_faces_t(tg_ctx *C, V3f<double> rhs, double scale, int ab2, RkArgs rk)
{
    const Grid g = C->g;
    const dim3 gr = gi(g);
    const auto &P = C->pol;
    if (P.rhs32 && P.flux32) TG_PROF(C, "formu_rhs_faces", k_rhs_faces<float, float, fused, AX><<<gr, block3(), 0, C->stream>>>(g, C->fm32, C->s, C->fw32, rhs, scale, C->prm, ab2, rk));
    else if (P.rhs32) TG_PROF(C, "formu_rhs_faces", k_rhs_faces<float, double, fused, AX><<<gr, block3(), 0, C->stream>>>(g, C->fm32, C->s, C->fw64, rhs, scale, C->prm, ab2, rk));
    else if (P.flux32) TG_PROF(C, "formu_rhs_faces", k_rhs_faces<double, float, fused, AX><<<gr, block3(), 0, C->stream>>>(g, C->fm64, C->s, C->fw32, rhs, scale, C->prm, ab2, rk));
    else TG_PROF(C, "formu_rhs_faces", k_rhs_faces<double, double, fused, AX><<<gr, block3(), 0, C->stream>>>(g, C->fm64, C->s, C->fw64, rhs, scale, C->prm, ab2, rk));
}

template <int fused>
static void rhs_faces(tg_ctx *C, V3f<double> rhs, double scale, int ab2, RkArgs rk = RkArgs{})
{
    if (C->axis_aligned) rhs_faces_t<fused, true>(C, rhs, scale, ab2, rk);
    else rhs_faces_t<fused, false>(C, rhs, scale, ab2, rk);
}

void form_u(tg_ctx *C, V3f<double> rhs, double scale, int mode)
{
    form_u_faces(C, mode);
    rhs_faces<0>(C, rhs, scale, 0);
}

// rhs += scale * FormU again from the cell sums the last FormU left (same
// state and formMode)
void form_u_again(tg_ctx *C, V3f<double> rhs, double scale)
{
    rhs_faces<0>(C, rhs, scale, 0);
}

// ExplicitRhsU up to the face fluxes: resets, Cartesian velocity, FormU passes 1-2
static void explicit_rhs_head(tg_ctx *C, int mode)
{
    const Grid g = C->g;
    reset_no_penetration(C);
    reset_face_periodic(C, C->s.ucont);
    contra_to_cart_stage(C);
    reset_cell_periodic(C, C->s.ucat);
    if (C->taping) tape_stage(C);
    form_u_faces(C, mode);
    // every point outside the interior faces keeps Rhs = -dP + b = 0: zero from
    // the allocation, rewritten here only after a caller wrote Rhs
    if (C->clear_rhs) {
        TG_CUDA(cudaMemsetAsync(C->s.rhs.x, 0, 3 * sizeof(double) * g.size(), C->stream));
        C->clear_rhs = false;
    }
}

void explicit_rhs(tg_ctx *C, int mode)
{
    const Grid g = C->g;
    explicit_rhs_head(C, mode);
    rhs_faces<1>(C, C->s.rhs, 1.0, C->it > C->cfg.it_start ? 1 : 0);
    TG_PROF(C, "bc_non_resolved", k_non_resolved<<<g2(g.my, g.mz), b2, 0, C->stream>>>(g, C->s, C->prm, 0));
    TG_PROF(C, "bc_non_resolved", k_non_resolved<<<g2(g.mx, g.mz), b2, 0, C->stream>>>(g, C->s, C->prm, 1));
    TG_PROF(C, "bc_non_resolved", k_non_resolved<<<g2(g.mx, g.my), b2, 0, C->stream>>>(g, C->s, C->prm, 2));
}

// ExplicitRhsU followed by one explicit update (an RK4 stage or the FE step)
// without storing Rhs: the face assembly applies the update at the faces of
// the interior cells, k_rk_shell at every other point (zero right-hand side)
static void explicit_rhs_update(tg_ctx *C, RkArgs rk)
{
    const Grid g = C->g;
    explicit_rhs_head(C, 0);
    rhs_faces<2>(C, C->s.rhs, 1.0, C->it > C->cfg.it_start ? 1 : 0, rk);
    dim3 grid((std::max(g.mx, g.my) + 31) / 32, (std::max(g.my, g.mz) + 7) / 8, 6);
    TG_PROF(C, "rk_shell", k_rk_shell<<<grid, dim3(32, 8), 0, C->stream>>>(g, C->s, rk));
}

// resetNonResolvedCellFaces (inline.h:1674-1835) on an arbitrary face vector
void mask_non_resolved(tg_ctx *C, V3f<double> v)
{
    const Grid g = C->g;
    State s = C->s;
    s.rhs = v;
    k_non_resolved<<<g2(g.my, g.mz), b2, 0, C->stream>>>(g, s, C->prm, 0);
    k_non_resolved<<<g2(g.mx, g.mz), b2, 0, C->stream>>>(g, s, C->prm, 1);
    k_non_resolved<<<g2(g.mx, g.my), b2, 0, C->stream>>>(g, s, C->prm, 2);
}

// constant part of the Crank-Nicolson residual (UeqnSNES, ueqn_solvers.c:1097-1163):
// bU = -dP (+ AB2 buoyancy) (+ 1/2 Rhs_o) (+ turbine force) + sourceU, and the
// mean pressure gradient (see tg_cn.cu)
__global__ void k_cn_bu(Grid g, Metrics m, State s, Params p, V3f<double> bu, int ab2, int half_rhs_o)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    const int c = g.lin(k, j, i);
    R3<double> b = -1.0 * ld3(s.dp, c);
    if (p.buoyancy) {
        if (ab2) { b = b + (3.0 / 2.0) * ld3(s.btheta, c); b = b + (-1.0 / 2.0) * ld3(s.btheta_o, c); }
        else b = b + 1.0 * ld3(s.btheta, c);
    }
    if (half_rhs_o) b = b + 0.5 * ld3(s.rhs_o, c);
    if (p.farm) b = b + 1.0 * ld3(s.farmcont, c);
    if (i >= 1 && j >= 1 && k >= 1 && i <= g.mx - 2 && j <= g.my - 2 && k <= g.mz - 2) {
        if (p.source) {
            const V3f<double> &f = s.source;
            const int ie = c + 1, jn = c + g.mx, kt = c + g.mx * g.my;
            const R3<double> a = ld3(m.icsi, c), e = ld3(m.jeta, c), d = ld3(m.kzet, c);
            b.x += 1.0 * (0.5 * (f.x[c] + f.x[ie]) * a.x + 0.5 * (f.y[c] + f.y[ie]) * a.y + 0.5 * (f.z[c] + f.z[ie]) * a.z);
            b.y += 1.0 * (0.5 * (f.x[c] + f.x[jn]) * e.x + 0.5 * (f.y[c] + f.y[jn]) * e.y + 0.5 * (f.z[c] + f.z[jn]) * e.z);
            b.z += 1.0 * (0.5 * (f.x[c] + f.x[kt]) * d.x + 0.5 * (f.y[c] + f.y[kt]) * d.y + 0.5 * (f.z[c] + f.z[kt]) * d.z);
        }
        if (p.mean_grad_p) {
            const R3<double> a = ld3(m.icsi, c), e = ld3(m.jeta, c), d = ld3(m.kzet, c);
            b.x += p.mgp[0] * a.x + p.mgp[1] * a.y + p.mgp[2] * a.z;
            b.y += p.mgp[0] * e.x + p.mgp[1] * e.y + p.mgp[2] * e.z;
            b.z += p.mgp[0] * d.x + p.mgp[1] * d.y + p.mgp[2] * d.z;
        }
    }
    st3(bu, c, b);
}

void cn_build_bu(tg_ctx *C, V3f<double> bu, bool half_rhs_o)
{
    const Grid g = C->g;
    k_cn_bu<<<ga(g), block3(), 0, C->stream>>>(g, C->m, C->s, C->prm, bu, C->it > C->cfg.it_start ? 1 : 0, half_rhs_o ? 1 : 0);
}


// SolveUEqn (ueqn.c:397-440). cart_tail: finish with contravariantToCartesian
// on every interior cell as the reference does; the full step converts only
// the boundary shell, which gives the same Ucat at the end of the step because
// the projection is followed by its own conversion.
static int solve_u_impl(tg_ctx *C, bool cart_tail, tg_stats *st = nullptr)
{
    const int64_t G = C->g.size();
    const double dt = C->prm.dt;
    int rc = 0;
    if (C->cfg.ddt_scheme == TG_DDT_CN) {
        // UeqnSNES, ueqn_solvers.c:1087-1199
        rc = solve_u_cn(C, st);
    } else if (imex_scheme(C->cfg.ddt_scheme)) {
        // UeqnABCN / UeqnRK3CN_W / UeqnRK3CN_SO, ueqn_solvers.c:1508-1735
        rc = solve_u_imex(C);
    } else if (C->cfg.ddt_scheme == TG_DDT_FE) {
        // UeqnFE, ueqn_solvers.c:1411-1442
        explicit_rhs_update(C, RkArgs{dt, 0.0, 0, 0, 1});
    } else {
        // UeqnRK4, ueqn_solvers.c:1446-1504
        const double b[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
        const double a[4] = {0.0, 0.5, 0.5, 1.0};
        for (int st = 0; st < 4; st++)
            explicit_rhs_update(C, RkArgs{dt * b[st], st < 3 ? a[st + 1] * dt : 0.0, st == 0 ? 1 : 0, st == 3 ? 1 : 0, 0});
    }
    // SolveUEqn tail, ueqn.c:413-437
    reset_no_penetration(C);
    reset_face_periodic(C, C->s.ucont);
    if (cart_tail) {
        contra_to_cart(C);
    } else {
        // the full step converts again after the projection, which rewrites
        // every interior cell and the face ghosts; only the edge and corner
        // ghosts keep what the periodic copies below bring from the shell
        const Grid g = C->g;
        int na = std::max(g.mx, g.my) - 2, nb = std::max(g.my, g.mz) - 2;
        dim3 grid((na + 31) / 32, (nb + 7) / 8, 6);
        TG_PROF(C, "contra_to_cart_shell", k_contra_to_cart_shell<<<grid, b2, 0, C->stream>>>(g, C->fm64, C->s, C->axis_aligned));
    }
    reset_cell_periodic(C, C->s.ucat);
    adjust_fluxes(C);                  // ueqn.c:437
    return rc;
}

void solve_u(tg_ctx *C) { solve_u_impl(C, true); }

// SolvePEqn (peqn.c:3777-3971) after the Poisson solve: phi ghosts, pressure
// update and ghosts, projection
void pressure_update_and_project(tg_ctx *C)
{
    const Grid g = C->g;
    update_scalar_ghosts(C, C->s.phi);
    TG_PROF(C, "update_pressure", k_update_pressure<<<gi(g), block3(), 0, C->stream>>>(g, C->s));
    update_scalar_ghosts(C, C->s.p);
    refresh_met32(C);
    if (C->pol.proj32) TG_PROF(C, "project", k_project<float><<<gf(g), block3(), 0, C->stream>>>(g, C->fm32, C->s, C->prm.dt, C->axis_aligned));
    else TG_PROF(C, "project", k_project<double><<<gf(g), block3(), 0, C->stream>>>(g, C->fm64, C->s, C->prm.dt, C->axis_aligned));
}

int solve_p(tg_ctx *C, tg_stats *st)
{
    int rc = poisson_solve(C, st);
    pressure_update_and_project(C);
    return rc;
}

void reduce_max_abs_div(tg_ctx *C, double *d_out)
{
    const int nb = C->red_blocks;
    TG_PROF(C, "div_max", k_div_partial<<<nb, 256, 0, C->stream>>>(C->g, C->m, C->s, C->d_red));
    k_max_final<<<1, 256, 0, C->stream>>>(C->d_red, nb, d_out);
}

double continuity_error(tg_ctx *C)
{
    reduce_max_abs_div(C, C->d_scal + 16);
    TG_CUDA(cudaMemcpyAsync(C->h_scal + 16, C->d_scal + 16, sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaStreamSynchronize(C->stream));
    return C->h_scal[16];
}

void sync_pressure(tg_ctx *C)
{
    const Grid g = C->g;
    const int64_t G = g.size();
    k_copy1<<<1, 1, 0, C->stream>>>(C->s.p + g.lin(1, 1, 1), C->d_scal + 17);
    TG_PROF(C, "gauge", k_gauge<<<nblk(G), 256, 0, C->stream>>>(G, C->s.p, C->d_scal + 17));
}

void init_from_cartesian(tg_ctx *C)
{
    const Grid g = C->g;
    if (C->prm.teqn) update_temperature_bcs(C);
    update_cartesian_bcs(C);
    k_init_faces<<<gf(g), block3(), 0, C->stream>>>(g, C->m, C->s);
    update_contravariant_bcs(C);
}

__global__ void k_set_scalar(double *a, double v) { a[0] = v; }
__global__ void k_incr_scalar(double *a) { a[0] += 1.0; }

void set_device_step(tg_ctx *C) { k_set_scalar<<<1, 1, 0, C->stream>>>(C->d_scal + SC_IT, (double)C->it); }

// one time step in the order of main.c:54-327; capture: the step is being
// recorded into a CUDA graph (device-side Poisson loop, statistics in the
// SC_G* device slots)
static int step_body(tg_ctx *C, tg_stats *st, bool capture)
{
    const int64_t G = C->g.size();
    TG_CUDA(cudaMemcpyAsync(C->s.ucont_o.x, C->s.ucont.x, 3 * sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
    if (C->taping) tape_step_start(C);
    if (C->prm.teqn) {                  // main.c:83-99: (BDF2: Tmprt_oo = Tmprt_o,) Tmprt_o = Tmprt
        if (C->cfg.t_ddt_scheme == TG_TDDT_BDF2)
            TG_CUDA(cudaMemcpyAsync(C->tmprt_oo, C->s.tmprt_o, sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
        TG_CUDA(cudaMemcpyAsync(C->s.tmprt_o, C->s.tmprt, sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
    }
    if (C->prm.les) {
        update_nut(C);
        // nut is final for the step: tg_step_host copies it out from here
        if (C->ev_nut)
            TG_CUDA(cudaEventRecordWithFlags(C->ev_nut, C->stream, capture ? cudaEventRecordExternal : cudaEventRecordDefault));
        update_wall_models(C);
    }
    if (C->taping) tape_nut(C);
    if (C->prm.farm) farm_update(C);
    grad_p(C);
    if (C->prm.buoyancy) {
        if (C->it > C->cfg.it_start)
            TG_CUDA(cudaMemcpyAsync(C->s.btheta_o.x, C->s.btheta.x, 3 * sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
        buoyancy(C);
    }
    const int urc = solve_u_impl(C, false, st);
    int rc = 0;
    if (capture) poisson_solve_capture(C);
    else rc = poisson_solve(C, st);
    if (urc == 2) rc = 2;
    else if (rc != 2) rc |= urc;
    pressure_update_and_project(C);
    contra_to_cart(C);
    if (C->prm.teqn) {                  // main.c:194-205
        update_wall_models_t(C);
        const int trc = solve_t(C);
        if (trc == 2) rc = 2;
        else if (rc != 2) rc |= trc;
    }
    reduce_max_abs_div(C, C->d_scal + 16);
    if (C->cfg.ddt_scheme == TG_DDT_CN) {   // main.c:214-272: Rhs_o for the next step
        TG_CUDA(cudaMemsetAsync(C->s.rhs_o.x, 0, 3 * sizeof(double) * G, C->stream));
        form_u(C, C->s.rhs_o, 1.0);
    }
    if (C->prm.teqn) update_temperature_bcs(C);   // main.c:274-278
    update_cartesian_bcs(C);
    update_contravariant_bcs(C);
    sync_pressure(C);
    k_incr_scalar<<<1, 1, 0, C->stream>>>(C->d_scal + SC_IT);
    return rc;
}

// A step replays as one CUDA graph once every choice the host makes in it is
// fixed: after the first step (Adams-Bashforth flag, btheta_o copy), with the
// wall filter (and thetaWallFunction surface temperature) seeded, no pending clear of a caller-written Rhs or dP, the FP32
// metric copies current, and profiling and taping off. The Krylov loop of the
// captured step runs under device control (poisson_solve_capture).
static bool graph_eligible(const tg_ctx *C)
{
    const bool wall = C->prm.les && C->prm.bc[TG_JLEFT] == TG_BC_WALL_SHUMANN;
    return C->graphs && !C->graph_failed && !C->prof.on && (!C->taping || tape_in_work(C)) && C->pois &&
           C->cfg.ddt_scheme != TG_DDT_CN && !imex_scheme(C->cfg.ddt_scheme) &&   // host-driven Krylov loops
           !(C->prm.teqn && C->cfg.t_ddt_scheme != TG_TDDT_RK4) &&
           C->it > C->cfg.it_start && (!wall || C->ufilt_set) &&
           !(C->prm.les && C->prm.t_wall == TG_TWALL_SHUMANN && !C->surf_set) &&   // surfaceTheta seeded
           !C->clear_rhs && !C->clear_dp && !(C->mixed && C->met32_stale);
}

void graph_destroy(tg_ctx *C)
{
    if (C->step_exec) cudaGraphExecDestroy(C->step_exec);
    if (C->step_exec_taped) cudaGraphExecDestroy(C->step_exec_taped);
    C->step_exec = C->step_exec_taped = nullptr;
    adj_graph_destroy(C);
}

bool capture_graph(tg_ctx *C, cudaGraphExec_t *out, const std::function<void()> &body)
{
    *out = nullptr;
    for (cudaStream_t &a : C->aux)
        if (!a) TG_CUDA(cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking));
    cudaStream_t s = C->stream;
    cudaGraph_t graph = nullptr;
    TG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
        body();
    } catch (const CudaError &) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t part = nullptr;
        for (int q = 1; q >= 0; q--)   // body graphs belong to their conditional nodes
            if (cudaStreamIsCapturing(C->aux[q], &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
                cudaStreamEndCapture(C->aux[q], &part);
        part = nullptr;
        C->stream = s;
        cudaStreamEndCapture(s, &part);
        if (part) cudaGraphDestroy(part);
        cudaGetLastError();
        return false;
    }
    if (cudaStreamEndCapture(s, &graph) != cudaSuccess) { cudaGetLastError(); return false; }
    cudaError_t e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { *out = nullptr; cudaGetLastError(); return false; }
    return true;
}

void step_stats_reset(tg_ctx *C)
{
    TG_CUDA(cudaMemsetAsync(C->d_scal + SC_G, 0, sizeof(double) * ST_COUNT, C->stream));
    TG_CUDA(cudaMemsetAsync(C->d_scal + SC_ADJ, 0, sizeof(double) * ST_COUNT, C->stream));
}

int step_stats_read(tg_ctx *C, tg_stats *s, bool any, bool last)
{
    TG_CUDA(cudaMemcpyAsync(C->h_scal + 16, C->d_scal + 16, sizeof(double) * (SC_IT - 16), cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaStreamSynchronize(C->stream));
    if (!any) return 0;
    const double *h = C->h_scal;
    s->poisson_total_iterations += (int32_t)h[SC_GTOT];
    if (last) {
        s->poisson_iterations = (int32_t)h[SC_GIT];
        s->poisson_initial_residual = h[SC_GRES0];
        s->poisson_final_residual = h[SC_GRES];
    }
    if (h[SC_GNAN] != 0.0) return 2;
    return h[SC_GNOCONV] > 0.0 ? 1 : 0;
}

// One step: a replay of the captured step graph when the step qualifies,
// else the eager sequence with a host-side Poisson loop. Returns 0, or for an
// eager step 1 (iteration cap) / 2 (non-finite residual); a replayed step
// reports through the SC_G* slots read by the caller.
int step(tg_ctx *C, tg_stats *st, bool *replayed)
{
    if (replayed) *replayed = false;
    if (graph_eligible(C)) {
        // the taped step records its stages into the work tape
        cudaGraphExec_t &ex = C->taping ? C->step_exec_taped : C->step_exec;
        if (!ex && !capture_graph(C, &ex, [&]() { step_body(C, nullptr, true); })) {
            // capture is unsupported for this configuration: stay eager
            graph_destroy(C);
            C->graph_failed = true;
        }
        if (ex) {
            TG_CUDA(cudaGraphLaunch(ex, C->stream));
            C->it++;
            C->replays++;
            if (replayed) *replayed = true;
            return 0;
        }
    }
    int rc = step_body(C, st, false);
    C->it++;
    return rc;
}

}  // namespace tg
