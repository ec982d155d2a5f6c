// Discrete adjoint of the fractional time step (TOSCA has no adjoint; this is
// new). tg_adjoint_step computes the vector-Jacobian product of one step of
// tg_step: given the adjoints of the state after the step (Ucont, the full
// Ucat array, P) it returns the adjoints of the state before it and adds the
// step's contribution to the gradient with respect to the body force of
// sourceU. The step is re-run once with its stage states recorded (the tape),
// then every forward kernel is transposed in reverse order:
//
//   gauge, UpdateContravariantBCs, UpdateCartesianBCs, contravariantToCartesian,
//   ProjectVelocity, UpdatePressure (+ ghosts), the pressure solve (its own
//   Krylov/multigrid solve of the transposed operator), SetRHS, the RK4 (or FE)
//   combination, and per stage resetNonResolvedCellFaces, sourceU, FormU (face
//   assembly, cell divergence, face fluxes), the periodic ghost copies,
//   contravariantToCartesian and the flux resets; then GradP and Smagorinsky.
//
// Transposes that gather (each output written by one thread) are used for the
// volume operators with simple stencils; the stencil scatters of FormU, GradP,
// ProjectVelocity and Smagorinsky and the boundary routines accumulate with
// FP64 atomics. Switches of the forward step (QUICK's upwind choice, the
// outflow masks of resetNonResolvedCellFaces) are frozen at the forward state.
//
// Scope: orthogonal grids (symmetric pressure operator), FE and RK4, central
// and QUICK convection, constant or Smagorinsky viscosity, noSlip, slip and
// periodic patches, the Schumann wall function on jLeft (neutral, plane-
// averaged u*, Cartesian branch: its time-filter state is part of the state,
// adjoint TG_F_WALL_ADJ); the body force, frozen-temperature buoyancy and the
// mean pressure gradient enter as forcings. The curvilinear (non-symmetric)
// pressure operator and the curvilinear wall-stress branch are rejected with
// TG_ERR_BAD_ARG. The adjoint arithmetic is FP64 in every precision mode.
//
// Checkpointing: tg_adjoint_forward runs the forward steps keeping device
// snapshots of the state at the positions of a binomial (revolve) schedule;
// tg_adjoint_reverse walks the steps backwards, restoring the nearest
// snapshot and recomputing forward where the schedule says so (each reversed
// step re-runs its own forward step once to record its stages). When there is
// a snapshot per step and the tapes of all steps fit in 60 % of the free
// device memory, the forward pass keeps every step's tape instead and the
// reversal runs no forward step at all.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "tg_internal.cuh"

namespace tg {

struct Snapshot {
    V3f<double> ucont, ucat, btheta, btheta_o;
    double *p, *px, *pxp, *pxp2; // P, the last three Poisson solutions (initial guess of the next solve)
    double phist = 0.0;          // solutions in that history (device slot SC_PHIST)
    double *wum = nullptr, *wfx = nullptr, *wfy = nullptr;   // wall-model state (planes), with the wall function
    bool ufilt_set = false;
    int it;
    int pos;       // step index of the state held (-1: free)
};

// forward intermediates of one step
struct Tape {
    V3f<double> u_o, ucat_n, ut[4], uc[4];
    double *nut = nullptr;
    // wall-model state at the step start (planes mz x mx) and, on the device,
    // [0] the step counter of the step, [1] 1 when the step seeded the filter
    double *wum = nullptr, *wfx = nullptr, *wfy = nullptr, *meta = nullptr;
    int nst = 0;
};

struct AdjState {
    // public adjoint fields
    V3f<double> ua, ca, fa;
    double *pa = nullptr;
    double *wxa = nullptr, *wya = nullptr, *wma = nullptr;   // TG_F_WALL_ADJ (planes)
    // wall reverse work: tauWall adjoint, Up and |Up| adjoints, block partials, scalars
    double *twa[3] = {nullptr, nullptr, nullptr}, *upa[4] = {nullptr, nullptr, nullptr, nullptr};
    double *wpart = nullptr, *wsc = nullptr;
    // work
    V3f<double> uoa, usa, uta, cta, ra, dpa, fpa, f1a, f2a, f3a, qa;
    double *pha = nullptr, *na = nullptr, *lam = nullptr, *rhsc = nullptr;
    double *lam_prev = nullptr, *lam_prev2 = nullptr;   // solutions of the two steps reversed before
    // tape of the step being reversed: the work tape, or one of the stored
    // tapes of a forward run that kept every step's tape
    Tape work_tape;
    std::vector<Tape> store;
    Tape *cur = nullptr;
    bool stored = false;                 // the last forward run kept every tape
    bool work = false;
    // checkpoints (the last one is the scratch state of an adjoint step)
    std::vector<Snapshot> snaps;
    Snapshot single{};                  // scratch state of tg_adjoint_step
    bool has_single = false;
    int base_it = 0, nsteps = 0, fwd_steps = 0;
    int max_tapes = -1;                 // cap of the segment schedule's tapes (-1: memory decides)
    int seg = 0;                        // segment length of the last forward run (0: other schedule)
    int64_t adj_iters = 0;                // Krylov iterations of the transposed solves
    bool recorded = false;
    // CUDA graphs of a reversed step: reading the work tape, and reading each
    // of the first stored tapes (no copy into the work tape)
    cudaGraphExec_t rev_exec = nullptr;
    std::vector<cudaGraphExec_t> rev_store;
    bool rev_failed = false;
    // bounds of the recorded forward run
    int start_pos = 0;
};

namespace {

constexpr int TB = 256;
inline int nblk1(int64_t n) { int64_t b = (n + TB - 1) / TB; return (int)std::min<int64_t>(b, 148 * 16); }
inline dim3 g2(int na, int nb) { return dim3((na + 31) / 32, (nb + 7) / 8); }
const dim3 b2(32, 8);
inline dim3 gall(const Grid &g) { return grid3(g.mx, g.my, g.mz); }
inline dim3 gint(const Grid &g) { return grid3(g.mx - 2, g.my - 2, g.mz - 2); }
inline dim3 gfc(const Grid &g) { return grid3(g.mx - 1, g.my - 1, g.mz - 1); }

__device__ __forceinline__ bool is_wall(int t) { return t == TG_BC_NOSLIP || t == TG_BC_SLIP || t == TG_BC_WALL_SHUMANN; }
__device__ __forceinline__ void aadd(double *p, double v) { if (v != 0.0) atomicAdd(p, v); }
__device__ __forceinline__ void aadd3(const V3f<double> &f, int q, double w, R3<double> v)
{
    aadd(f.x + q, w * v.x); aadd(f.y + q, w * v.y); aadd(f.z + q, w * v.z);
}
__device__ __forceinline__ bool interior(const Grid &g, int k, int j, int i)
{
    return i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2;
}

// ------------------------------------------------------------- elementwise
__global__ void k_axpy3(int64_t n, V3f<double> y, double a, V3f<double> x)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        y.x[q] += a * x.x[q]; y.y[q] += a * x.y[q]; y.z[q] += a * x.z[q];
    }
}
__global__ void k_sum_partial(int64_t n, const double *a, double *part)
{
    __shared__ double sh[TB];
    double s = 0.0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) s += a[q];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = TB / 2; w > 0; w >>= 1) { if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w]; __syncthreads(); }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
// syncPressure transpose: p_adj[ref] -= sum(p_adj)
__global__ void k_gauge_adj(const double *part, int nb, double *pa, int ref)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += part[b];
    pa[ref] -= s;
}

// ------------------------------------------------ periodic / ghost copies
// one direction of the forward copies (tg_step.cu k_periodic_copy /
// k_scalar_ghosts): dst <- src, transposed: adj[src] += adj[dst], adj[dst] = 0
__device__ __forceinline__ void plane_idx(const Grid &g, int dir, int a, int b, int l, int &q)
{
    if (dir == 0) q = g.lin(b, a, l); else if (dir == 1) q = g.lin(b, l, a); else q = g.lin(l, b, a);
}
// cell periodic copies (both sides) or face copies (left only) of a vector
__global__ void k_adj_periodic(Grid g, V3f<double> v, int dir, int left_only)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = dir == 0 ? g.my : g.mx, nb = dir == 2 ? g.my : g.mz;
    if (a >= na || b >= nb) return;
    int m = dir == 0 ? g.mx : (dir == 1 ? g.my : g.mz);
    for (int side = left_only ? 0 : 1; side >= 0; side--) {
        int d, s;
        plane_idx(g, dir, a, b, side ? m - 1 : 0, d);
        plane_idx(g, dir, a, b, side ? 1 : m - 2, s);
        v.x[s] += v.x[d]; v.y[s] += v.y[d]; v.z[s] += v.z[d];
        v.x[d] = 0.0; v.y[d] = 0.0; v.z[d] = 0.0;
    }
}
// scalar ghosts (periodic or zero-gradient), UpdatePhiBCs / UpdatePressureBCs
__global__ void k_adj_scalar_ghosts(Grid g, double *v, int dir)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = dir == 0 ? g.my : g.mx, nb = dir == 2 ? g.my : g.mz;
    if (a >= na || b >= nb) return;
    int per = dir == 0 ? g.pi : (dir == 1 ? g.pj : g.pk);
    int m = dir == 0 ? g.mx : (dir == 1 ? g.my : g.mz);
    for (int side = 1; side >= 0; side--) {
        int dd = side ? m - 1 : 0;
        int ss = side ? (per ? 1 : m - 2) : (per ? m - 2 : 1);
        int d, s;
        plane_idx(g, dir, a, b, dd, d);
        plane_idx(g, dir, a, b, ss, s);
        v[s] += v[d];
        v[d] = 0.0;
    }
}
// nut BC ghosts (k_nut_bcs): fixed values have no source
__global__ void k_adj_nut_bcs(Grid g, double *na, Params p)
{
    int patch = blockIdx.z;
    int dir = patch >> 1, right = patch & 1;
    int a = blockIdx.x * blockDim.x + threadIdx.x + 1, b = blockIdx.y * blockDim.y + threadIdx.y + 1;
    int nA = (dir == 0 ? g.my : g.mx) - 2, nB = (dir == 2 ? g.my : g.mz) - 2;
    if (a > nA || b > nB) return;
    int i, j, k;
    if (dir == 0) { k = b; j = a; i = right ? g.mx - 2 : 1; }
    else if (dir == 1) { k = b; i = a; j = right ? g.my - 2 : 1; }
    else { j = b; i = a; k = right ? g.mz - 2 : 1; }
    int c = g.lin(k, j, i);
    int step = dir == 0 ? 1 : (dir == 1 ? g.mx : g.mx * g.my);
    int ghost = right ? c + step : c - step;
    int t = p.nut_bc[patch];
    double v = na[ghost];
    na[ghost] = 0.0;
    if (t == TG_NUTBC_ZEROGRADIENT) aadd(na + c, v);
    else if (t != TG_NUTBC_FIXEDVALUE) {
        int src;
        if (dir == 0) src = g.lin(k, j, right ? 1 : g.mx - 2);
        else if (dir == 1) src = g.lin(k, right ? 1 : g.my - 2, i);
        else src = g.lin(right ? 1 : g.mz - 2, j, i);
        aadd(na + src, v);
    }
}
// resetNoPenetrationFluxes: wall-normal faces of wall patches zeroed
__global__ void k_adj_no_penetration(Grid g, V3f<double> a, Params p)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int q = g.lin(k, j, i);
    if ((i == 0 && is_wall(p.bc[TG_ILEFT])) || (i == g.mx - 2 && is_wall(p.bc[TG_IRIGHT]))) a.x[q] = 0.0;
    if ((j == 0 && is_wall(p.bc[TG_JLEFT])) || (j == g.my - 2 && is_wall(p.bc[TG_JRIGHT]))) a.y[q] = 0.0;
    if ((k == 0 && is_wall(p.bc[TG_KLEFT])) || (k == g.mz - 2 && is_wall(p.bc[TG_KRIGHT]))) a.z[q] = 0.0;
}

// ------------------------------------------------- contravariantToCartesian
// (a) per interior cell: q_adj = M^-T ucat_adj (Cramer on the transpose), ucat_adj = 0
__global__ void k_adj_contra_cells(Grid g, Metrics m, V3f<double> ca, V3f<double> qa)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int c = g.lin(k, j, i);
    R3<double> gv = ld3(ca, c);
    st3(ca, c, R3<double>{0.0, 0.0, 0.0});
    R3<double> s = ld3(m.csi, c), e = ld3(m.eta, c), z = ld3(m.zet, c);
    double a00 = s.x, a01 = e.x, a02 = z.x, a10 = s.y, a11 = e.y, a12 = z.y, a20 = s.z, a21 = e.z, a22 = z.z;
    double det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
    double q0 = ( gv.x * (a11 * a22 - a12 * a21) - gv.y * (a01 * a22 - a02 * a21) + gv.z * (a01 * a12 - a02 * a11)) / det;
    double q1 = (-gv.x * (a10 * a22 - a12 * a20) + gv.y * (a00 * a22 - a02 * a20) - gv.z * (a00 * a12 - a02 * a10)) / det;
    double q2 = ( gv.x * (a10 * a21 - a11 * a20) - gv.y * (a00 * a21 - a01 * a20) + gv.z * (a00 * a11 - a01 * a10)) / det;
    st3(qa, c, R3<double>{q0, q1, q2});
}
// (b) per face: ucont_adj += 0.5 (q_adj of the two cells); q_adj is zero off the interior
__global__ void k_adj_contra_faces(Grid g, V3f<double> qa, V3f<double> ua)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int f = g.lin(k, j, i);
    ua.x[f] += 0.5 * (qa.x[f] + qa.x[f + 1]);
    ua.y[f] += 0.5 * (qa.y[f] + qa.y[f + g.mx]);
    ua.z[f] += 0.5 * (qa.z[f] + qa.z[f + g.mx * g.my]);
}

// ------------------------------------------------------ UpdateCartesianBCs
__device__ void calc_normal_adj(R3<double> csi, R3<double> eta, R3<double> zet, int dir, R3<double> &n)
{
    const double a11 = csi.x, a12 = csi.y, a13 = csi.z;
    const double a21 = eta.x, a22 = eta.y, a23 = eta.z;
    const double a31 = zet.x, a32 = zet.y, a33 = zet.z;
    double det = a11 * (a33 * a22 - a32 * a23) - a21 * (a33 * a12 - a32 * a13) + a31 * (a23 * a12 - a22 * a13);
    double x, y, z;
    if (dir == 0) { x = (a33 * a22 - a32 * a23) / det; y = -(a33 * a21 - a31 * a23) / det; z = (a32 * a21 - a31 * a22) / det; }
    else if (dir == 1) { x = -(a33 * a12 - a32 * a13) / det; y = (a33 * a11 - a31 * a13) / det; z = -(a32 * a11 - a31 * a12) / det; }
    else { x = (a23 * a12 - a22 * a13) / det; y = -(a23 * a11 - a21 * a13) / det; z = (a22 * a11 - a21 * a12) / det; }
    double sm = sqrt(x * x + y * y + z * z);
    n = R3<double>{x / sm, y / sm, z / sm};
}
// ghost <- f(interior) per patch: adj of the ghost moves to its source
__global__ void k_adj_cartesian_bcs(Grid g, Metrics m, V3f<double> ca, Params p)
{
    int patch = blockIdx.z;
    int dir = patch >> 1, right = patch & 1;
    int a = blockIdx.x * blockDim.x + threadIdx.x + 1, b = blockIdx.y * blockDim.y + threadIdx.y + 1;
    int nA = (dir == 0 ? g.my : g.mx) - 2, nB = (dir == 2 ? g.my : g.mz) - 2;
    if (a > nA || b > nB) return;
    int type = p.bc[patch];
    int i, j, k;
    if (dir == 0) { k = b; j = a; i = right ? g.mx - 2 : 1; }
    else if (dir == 1) { k = b; i = a; j = right ? g.my - 2 : 1; }
    else { j = b; i = a; k = right ? g.mz - 2 : 1; }
    int c = g.lin(k, j, i);
    int step = dir == 0 ? 1 : (dir == 1 ? g.mx : g.mx * g.my);
    int ghost = right ? c + step : c - step;
    R3<double> ga = ld3(ca, ghost);
    st3(ca, ghost, R3<double>{0.0, 0.0, 0.0});
    if (type == TG_BC_SLIP) {
        R3<double> n; calc_normal_adj(ld3(m.csi, c), ld3(m.eta, c), ld3(m.zet, c), dir, n);
        aadd3(ca, c, 1.0, ga - (2.0 * dot3(ga, n)) * n);
    } else if (type == TG_BC_NOSLIP) {
        aadd3(ca, c, -1.0, ga);
    } else if (type == TG_BC_WALL_SHUMANN && dir == 1 && !right) {
        // ghost = 2 Ub - 3 (Ub.n) n - Uc + (Uc.n) n, Ub = (k, 1, i), Uc = (k, 2, i)
        R3<double> n; calc_normal_adj(ld3(m.csi, c), ld3(m.eta, c), ld3(m.zet, c), 1, n);
        const double gn = dot3(ga, n);
        aadd3(ca, c, 1.0, 2.0 * ga - (3.0 * gn) * n);
        aadd3(ca, c + g.mx, 1.0, gn * n - ga);
    } else if (type == TG_BC_PERIODIC) {
        int src;
        if (dir == 0) src = g.lin(k, j, right ? 1 : g.mx - 2);
        else if (dir == 1) src = g.lin(k, right ? 1 : g.my - 2, i);
        else src = g.lin(right ? 1 : g.mz - 2, j, i);
        aadd3(ca, src, 1.0, ga);
    }
}

// ----------------------------------------------------- UpdateContravariantBCs
// per direction (the forward runs k_contra_bc_periodic then k_contra_bc_faces):
// periodic left faces <- pre-call face m-2; faces of non-wall patches
// re-interpolated from Ucat; faces of wall patches zeroed
__global__ void k_adj_contra_bcs(Grid g, Metrics m, V3f<double> ua, V3f<double> ca, Params p, int dir)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int nA = (dir == 0 ? g.my : g.mx) - 1, nB = (dir == 2 ? g.my : g.mz) - 1;
    if (a >= nA || b >= nB) return;
    double *u = dir == 0 ? ua.x : (dir == 1 ? ua.y : ua.z);
    int step = dir == 0 ? 1 : (dir == 1 ? g.mx : g.mx * g.my);
    int f0, fr;
    if (dir == 0) { f0 = g.lin(b, a, 0); fr = g.lin(b, a, g.mx - 2); }
    else if (dir == 1) { f0 = g.lin(b, 0, a); fr = g.lin(b, g.my - 2, a); }
    else { f0 = g.lin(0, b, a); fr = g.lin(g.mz - 2, b, a); }
    const bool periodic = p.bc[2 * dir] == TG_BC_PERIODIC;
    double gl = u[f0], gr = u[fr];
    double pre_l = 0.0, pre_r = 0.0;       // adjoints of the pre-call values at the two faces
    // right face (fr): interp (non-wall) or zero (wall): overwritten either way
    if (!is_wall(p.bc[2 * dir + 1])) {
        R3<double> S = dir == 0 ? ld3(m.icsi, fr) : (dir == 1 ? ld3(m.jeta, fr) : ld3(m.kzet, fr));
        aadd3(ca, fr + step, 0.5 * gr, S);
        aadd3(ca, fr, 0.5 * gr, S);
    }
    // left face (f0)
    if (periodic) {
        pre_r += gl;                          // copy of the pre-call right face
    } else if (!is_wall(p.bc[2 * dir])) {
        R3<double> S = dir == 0 ? ld3(m.icsi, f0) : (dir == 1 ? ld3(m.jeta, f0) : ld3(m.kzet, f0));
        aadd3(ca, f0 + step, 0.5 * gl, S);
        aadd3(ca, f0, 0.5 * gl, S);
    }
    u[f0] = pre_l;
    u[fr] = pre_r;
}

// ------------------------------------------------------------ ProjectVelocity
__global__ void k_adj_project(Grid g, Metrics m, V3f<double> ua, double *fa, double dt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    const int mx = g.mx, my = g.my, mz = g.mz;
    int f = g.lin(k, j, i);
    auto F = [&](int kk, int jj, int ii, double w) { aadd(fa + g.id(kk, jj, ii), w); };
    if (j > 0 && k > 0 && ((i > 0 && i < mx - 2) || g.pi)) {
        R3<double> c1 = ld3(m.icsi, f), e1 = ld3(m.ieta, f), z1 = ld3(m.izet, f);
        double a = m.iaj[f], gg = -dt * ua.x[f];
        double wc = gg * dot3(c1, c1) * a, we = gg * dot3(e1, c1) * a, wz = gg * dot3(z1, c1) * a;
        F(k, j, i + 1, wc); F(k, j, i, -wc);
        if (j == my - 2)      { double w = 0.5 * we; F(k, j, i, w); F(k, j, i + 1, w); F(k, j - 1, i, -w); F(k, j - 1, i + 1, -w); }
        else if (j == 1)      { double w = 0.5 * we; F(k, j + 1, i, w); F(k, j + 1, i + 1, w); F(k, j, i, -w); F(k, j, i + 1, -w); }
        else                  { double w = 0.25 * we; F(k, j + 1, i, w); F(k, j + 1, i + 1, w); F(k, j - 1, i, -w); F(k, j - 1, i + 1, -w); }
        if (k == mz - 2)      { double w = 0.5 * wz; F(k, j, i, w); F(k, j, i + 1, w); F(k - 1, j, i, -w); F(k - 1, j, i + 1, -w); }
        else if (k == 1)      { double w = 0.5 * wz; F(k + 1, j, i, w); F(k + 1, j, i + 1, w); F(k, j, i, -w); F(k, j, i + 1, -w); }
        else                  { double w = 0.25 * wz; F(k + 1, j, i, w); F(k + 1, j, i + 1, w); F(k - 1, j, i, -w); F(k - 1, j, i + 1, -w); }
    }
    if (i > 0 && k > 0 && ((j > 0 && j < my - 2) || g.pj)) {
        R3<double> c2 = ld3(m.jcsi, f), e2 = ld3(m.jeta, f), z2 = ld3(m.jzet, f);
        double a = m.jaj[f], gg = -dt * ua.y[f];
        double wc = gg * dot3(c2, e2) * a, we = gg * dot3(e2, e2) * a, wz = gg * dot3(z2, e2) * a;
        F(k, j + 1, i, we); F(k, j, i, -we);
        if (i == mx - 2)      { double w = 0.5 * wc; F(k, j, i, w); F(k, j + 1, i, w); F(k, j, i - 1, -w); F(k, j + 1, i - 1, -w); }
        else if (i == 1)      { double w = 0.5 * wc; F(k, j, i + 1, w); F(k, j + 1, i + 1, w); F(k, j, i, -w); F(k, j + 1, i, -w); }
        else                  { double w = 0.25 * wc; F(k, j, i + 1, w); F(k, j + 1, i + 1, w); F(k, j, i - 1, -w); F(k, j + 1, i - 1, -w); }
        if (k == mz - 2)      { double w = 0.5 * wz; F(k, j, i, w); F(k, j + 1, i, w); F(k - 1, j, i, -w); F(k - 1, j + 1, i, -w); }
        else if (k == 1)      { double w = 0.5 * wz; F(k + 1, j, i, w); F(k + 1, j + 1, i, w); F(k, j, i, -w); F(k, j + 1, i, -w); }
        else                  { double w = 0.25 * wz; F(k + 1, j, i, w); F(k + 1, j + 1, i, w); F(k - 1, j, i, -w); F(k - 1, j + 1, i, -w); }
    }
    if (i > 0 && j > 0 && ((k > 0 && k < mz - 2) || g.pk)) {
        R3<double> c3 = ld3(m.kcsi, f), e3 = ld3(m.keta, f), z3 = ld3(m.kzet, f);
        double a = m.kaj[f], gg = -dt * ua.z[f];
        double wc = gg * dot3(c3, z3) * a, we = gg * dot3(e3, z3) * a, wz = gg * dot3(z3, z3) * a;
        F(k + 1, j, i, wz); F(k, j, i, -wz);
        if (i == mx - 2)      { double w = 0.5 * wc; F(k, j, i, w); F(k + 1, j, i, w); F(k, j, i - 1, -w); F(k + 1, j, i - 1, -w); }
        else if (i == 1)      { double w = 0.5 * wc; F(k, j, i + 1, w); F(k + 1, j, i + 1, w); F(k, j, i, -w); F(k + 1, j, i, -w); }
        else                  { double w = 0.25 * wc; F(k, j, i + 1, w); F(k + 1, j, i + 1, w); F(k, j, i - 1, -w); F(k + 1, j, i - 1, -w); }
        if (j == my - 2)      { double w = 0.5 * we; F(k, j, i, w); F(k + 1, j, i, w); F(k, j - 1, i, -w); F(k + 1, j - 1, i, -w); }
        else if (j == 1)      { double w = 0.5 * we; F(k, j + 1, i, w); F(k + 1, j + 1, i, w); F(k, j, i, -w); F(k + 1, j, i, -w); }
        else                  { double w = 0.25 * we; F(k, j + 1, i, w); F(k + 1, j + 1, i, w); F(k, j - 1, i, -w); F(k + 1, j - 1, i, -w); }
    }
}

// UpdatePressure (interior p += phi): phi_adj += p_adj; phi interior -> compact rhs
__global__ void k_adj_update_pressure(Grid g, const double *pa, double *pha, double *rhsc)
{
    int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y * blockDim.y + threadIdx.y, kc = blockIdx.z * blockDim.z + threadIdx.z;
    int nx = g.mx - 2, ny = g.my - 2, nz = g.mz - 2;
    if (ic >= nx || jc >= ny || kc >= nz) return;
    int c = g.lin(kc + 1, jc + 1, ic + 1);
    pha[c] += pa[c];
}
__global__ void k_adj_phi_compact(Grid g, const double *pha, double *rhsc)
{
    int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y * blockDim.y + threadIdx.y, kc = blockIdx.z * blockDim.z + threadIdx.z;
    int nx = g.mx - 2, ny = g.my - 2, nz = g.mz - 2;
    if (ic >= nx || jc >= ny || kc >= nz) return;
    rhsc[(kc * ny + jc) * nx + ic] = pha[g.lin(kc + 1, jc + 1, ic + 1)];
}
// SetRHS transpose (rows other than the pinned cell (1,1,1)): per face
// u*_adj += (lam(left cell) - lam(right cell)) / dt
__global__ void k_adj_set_rhs(Grid g, const double *lam, V3f<double> usa, double dt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    const int nx = g.mx - 2, ny = g.my - 2;
    auto L = [&](int kk, int jj, int ii) -> double {
        if (!interior(g, kk, jj, ii) || (ii == 1 && jj == 1 && kk == 1)) return 0.0;
        return lam[((kk - 1) * ny + (jj - 1)) * nx + (ii - 1)];
    };
    int f = g.lin(k, j, i);
    const double idt = 1.0 / dt;
    usa.x[f] += (L(k, j, i) - L(k, j, i + 1)) * idt;
    usa.y[f] += (L(k, j, i) - L(k, j + 1, i)) * idt;
    usa.z[f] += (L(k, j, i) - L(k + 1, j, i)) * idt;
}

// ----------------------------------------------------------------- RK stage
// rhs adjoint of stage s: dt b_s u*_adj (+ a_{s+1} dt adjoint of the next
// stage's Ucont), masked as resetNonResolvedCellFaces (frozen at Ucont_o);
// dP_adj -= it
__global__ void k_adj_stage_rhs(Grid g, V3f<double> ra, V3f<double> usa, V3f<double> nxt, double cb, double cn,
                                V3f<double> uo, V3f<double> dpa)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    int q = g.lin(k, j, i);
    R3<double> r{cb * usa.x[q], cb * usa.y[q], cb * usa.z[q]};
    if (cn != 0.0) { r.x += cn * nxt.x[q]; r.y += cn * nxt.y[q]; r.z += cn * nxt.z[q]; }
    R3<double> o = ld3(uo, q);
    if (i == 0) { if (!(o.x < 0)) r.x = 0.0; } else if (i == g.mx - 1) r.x = 0.0; else if (i == g.mx - 2 && !g.pi) { if (!(o.x > 0)) r.x = 0.0; }
    if (j == 0) { if (!(o.y < 0)) r.y = 0.0; } else if (j == g.my - 1) r.y = 0.0; else if (j == g.my - 2 && !g.pj) { if (!(o.y > 0)) r.y = 0.0; }
    if (k == 0) { if (!(o.z < 0)) r.z = 0.0; } else if (k == g.mz - 1) r.z = 0.0; else if (k == g.mz - 2 && !g.pk) { if (!(o.z > 0)) r.z = 0.0; }
    st3(ra, q, r);
    if (interior(g, k, j, i)) { dpa.x[q] -= r.x; dpa.y[q] -= r.y; dpa.z[q] -= r.z; }
}

// sourceU transpose (gather): f_adj(p) = 0.5 sum over the faces of interior
// cells that read f(p) of rhs_adj * face area
__global__ void k_adj_source(Grid g, Metrics m, V3f<double> ra, V3f<double> fa)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    int q = g.lin(k, j, i), pl = g.mx * g.my;
    R3<double> acc{0, 0, 0};
    if (interior(g, k, j, i)) {
        acc = acc + (0.5 * ra.x[q]) * ld3(m.icsi, q);
        acc = acc + (0.5 * ra.y[q]) * ld3(m.jeta, q);
        acc = acc + (0.5 * ra.z[q]) * ld3(m.kzet, q);
    }
    if (interior(g, k, j, i - 1)) acc = acc + (0.5 * ra.x[q - 1]) * ld3(m.icsi, q - 1);
    if (interior(g, k, j - 1, i)) acc = acc + (0.5 * ra.y[q - g.mx]) * ld3(m.jeta, q - g.mx);
    if (interior(g, k - 1, j, i)) acc = acc + (0.5 * ra.z[q - pl]) * ld3(m.kzet, q - pl);
    fa.x[q] += acc.x; fa.y[q] += acc.y; fa.z[q] += acc.z;
}

// ---------------------------------------------------------------- FormU
// pass 3 transpose (gather): fp_adj of interior cell p from the face assembly
// of its own faces and of the faces of the -i/-j/-k cells, plus the remapped
// neighbour reads at the boundary (periodic: first interior cell; otherwise the
// cell itself)
__global__ void k_adj_rhs_faces(Grid g, Metrics m, V3f<double> ra, double scale, V3f<double> fpa)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    const int mx = g.mx, my = g.my, mz = g.mz, pl = mx * my;
    int c = g.lin(k, j, i);
    auto tx = [&](int q) { return scale * m.iaj[q] * 0.5 * ra.x[q]; };
    auto ty = [&](int q) { return scale * m.jaj[q] * 0.5 * ra.y[q]; };
    auto tz = [&](int q) { return scale * m.kaj[q] * 0.5 * ra.z[q]; };
    R3<double> acc = tx(c) * ld3(m.csi, c) + ty(c) * ld3(m.eta, c) + tz(c) * ld3(m.zet, c);
    // i: cell c-1 reads fp(c) with csi(c); at the last cell the neighbour read is remapped
    if (i >= 2) acc = acc + tx(c - 1) * ld3(m.csi, c);
    if (g.pi && i == 1) { int q = g.lin(k, j, mx - 2); acc = acc + tx(q) * ld3(m.csi, q + 1); }
    if (!g.pi && i == mx - 2) acc = acc + tx(c) * ld3(m.csi, c + 1);
    if (j >= 2) acc = acc + ty(c - mx) * ld3(m.eta, c);
    if (g.pj && j == 1) { int q = g.lin(k, my - 2, i); acc = acc + ty(q) * ld3(m.eta, q + mx); }
    if (!g.pj && j == my - 2) acc = acc + ty(c) * ld3(m.eta, c + mx);
    if (k >= 2) acc = acc + tz(c - pl) * ld3(m.zet, c);
    if (g.pk && k == 1) { int q = g.lin(mz - 2, j, i); acc = acc + tz(q) * ld3(m.zet, q + pl); }
    if (!g.pk && k == mz - 2) acc = acc + tz(c) * ld3(m.zet, c + pl);
    st3(fpa, c, acc);
}
// pass 2 transpose (gather per face): flux_adj(f) = fp_adj(left cell) -
// fp_adj(right cell), with the periodic face-0 read of cell 1 remapped to
// face m-2
__global__ void k_adj_cell_fp(Grid g, V3f<double> fpa, V3f<double> f1a, V3f<double> f2a, V3f<double> f3a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    const int mx = g.mx, my = g.my, mz = g.mz, pl = mx * my;
    int f = g.lin(k, j, i);
    R3<double> z{0, 0, 0};
    auto FP = [&](int kk, int jj, int ii) { return interior(g, kk, jj, ii) ? ld3(fpa, g.lin(kk, jj, ii)) : z; };
    // i faces
    {
        R3<double> a = FP(k, j, i);
        if (!(g.pi && i == 0)) a = a - FP(k, j, i + 1);
        if (g.pi && i == mx - 2) a = a - FP(k, j, 1);
        if (g.pi && i == 0) a = z;
        st3(f1a, f, a);
    }
    {
        R3<double> a = FP(k, j, i);
        if (!(g.pj && j == 0)) a = a - FP(k, j + 1, i);
        if (g.pj && j == my - 2) a = a - FP(k, 1, i);
        if (g.pj && j == 0) a = z;
        st3(f2a, f, a);
    }
    {
        R3<double> a = FP(k, j, i);
        if (!(g.pk && k == 0)) a = a - FP(k + 1, j, i);
        if (g.pk && k == mz - 2) a = a - FP(1, j, i);
        if (g.pk && k == 0) a = z;
        st3(f3a, f, a);
    }
    (void)pl;
}

// viscous flux per unit nuEff is v_a = ajc [sum_m g_m d_m[a] + sum_m s_m[a] (d_m . n)]
// (s_m = face csi, eta, zet; n = s_dir; g_m = s_m . n); transpose:
// d_m_adj = ajc [g_m v_adj + (s_m . v_adj) n]
__device__ __forceinline__ void visc_adj(R3<double> s0, R3<double> s1, R3<double> s2, int dir, R3<double> va, double ajc, R3<double> dd[3])
{
    R3<double> sm[3] = {s0, s1, s2};
    R3<double> n = sm[dir];
    for (int q = 0; q < 3; q++) dd[q] = ajc * (dot3(sm[q], n) * va + dot3(sm[q], va) * n);
}

// the transpose of the axis-aligned viscous flux (visc_flux_ax of the forward
// step: cs = csi.y, et = eta.z, ze = zet.x of the face, the other metric
// components left out), term by term
__device__ __forceinline__ void visc_adj_ax(double cs, double et, double ze, int dir, R3<double> va, double ajc, R3<double> dd[3])
{
    if (dir == 0) {
        const double g11 = cs * cs;
        dd[0] = ajc * R3<double>{g11 * va.x, g11 * va.y + (cs * va.y) * cs, g11 * va.z};
        dd[1] = ajc * R3<double>{0.0, (et * va.z) * cs, 0.0};
        dd[2] = ajc * R3<double>{0.0, (ze * va.x) * cs, 0.0};
    } else if (dir == 1) {
        const double g21 = et * et;
        dd[0] = ajc * R3<double>{0.0, 0.0, (cs * va.y) * et};
        dd[1] = ajc * R3<double>{g21 * va.x, g21 * va.y, g21 * va.z + (et * va.z) * et};
        dd[2] = ajc * R3<double>{0.0, 0.0, (ze * va.x) * et};
    } else {
        const double g31 = ze * ze;
        dd[0] = ajc * R3<double>{(cs * va.y) * ze, 0.0, 0.0};
        dd[1] = ajc * R3<double>{(et * va.z) * ze, 0.0, 0.0};
        dd[2] = ajc * R3<double>{g31 * va.x + (ze * va.x) * ze, g31 * va.y, g31 * va.z};
    }
}

// pass 1 transpose: per face, scatter to Ucat (atomics), Ucont (own face) and
// nut. AX: the mesh is axis-aligned and the forward step formed the
// axis-aligned viscous flux, whose exact transpose reads 3 of the 9 face
// metric components
template <bool AX>
__global__ void k_adj_face_fluxes(Grid g, Metrics m, V3f<double> ut, V3f<double> uc, const double *nut, Params p,
                                  V3f<double> f1a, V3f<double> f2a, V3f<double> f3a,
                                  V3f<double> uta, V3f<double> cta, double *na, V3f<double> twa)
{
    // Ucat and nut of the block's faces with one point below and two above
    // in every direction, staged in shared memory as in the forward pass 1
    // (rows per warp, wrapped DMDA index, 0 outside a non-periodic extent);
    // the QUICK points of the periodic boundary faces that fall outside the
    // tile are read from global memory.
    constexpr int ATX = BX + 3, ATY = BY + 3, ATZ = BZ + 3, ATN = ATX * ATY * ATZ;
    static_assert(BX == 32 && (BX * BY * BZ) % 32 == 0 && 3 * ATY * ATZ <= BX * BY * BZ, "tile staging layout");
    __shared__ double su[3][ATN];
    __shared__ double sn[ATN];
    const int mx = g.mx, my = g.my, mz = g.mz;
    const int i0 = blockIdx.x * BX, j0 = blockIdx.y * BY, k0 = blockIdx.z * BZ;
    {
        auto stage = [&](int tx, int ty, int tz, int gi) {
            const int gj = g.wj(j0 - 1 + ty), gk = g.wk(k0 - 1 + tz), q = (tz * ATY + ty) * ATX + tx;
            double ux = 0.0, uy = 0.0, uz = 0.0, nt = 0.0;
            if (gi >= 0 && gi < mx && gj >= 0 && gj < my && gk >= 0 && gk < mz) {
                const int c = (gk * my + gj) * mx + gi;
                ux = uc.x[c]; uy = uc.y[c]; uz = uc.z[c];
                if (p.les) nt = nut[c];
            }
            su[0][q] = ux; su[1][q] = uy; su[2][q] = uz; sn[q] = nt;
        };
        const int lane = threadIdx.x, wid = threadIdx.z * BY + threadIdx.y;
        const int gi = g.wi(i0 - 1 + lane);
        for (int r = wid; r < ATY * ATZ; r += BX * BY * BZ / 32) stage(lane, r % ATY, r / ATY, gi);
        const int q = wid * 32 + lane;
        if (q < 3 * ATY * ATZ) {
            const int r = q / 3, tx = BX + (q - 3 * r);
            stage(tx, r % ATY, r / ATY, g.wi(i0 - 1 + tx));
        }
    }
    __syncthreads();
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y, k = k0 + threadIdx.z;
    if (i > mx - 2 || j > my - 2 || k > mz - 2) return;
    const bool npi = !g.pi, npj = !g.pj, npk = !g.pk;
    const bool quickDiv = p.div_scheme == TG_DIV_QUICK;
    const double nu = p.nu;
    int f = g.lin(k, j, i);
    // tile index of (kk, jj, ii), or -1 outside the tile
    auto tq = [&](int kk, int jj, int ii) {
        const int tx = ii - i0 + 1, ty = jj - j0 + 1, tz = kk - k0 + 1;
        return ((unsigned)tx < (unsigned)ATX && (unsigned)ty < (unsigned)ATY && (unsigned)tz < (unsigned)ATZ) ? (tz * ATY + ty) * ATX + tx : -1;
    };
    auto U = [&](int kk, int jj, int ii) {
        const int q = tq(kk, jj, ii);
        return q >= 0 ? R3<double>{su[0][q], su[1][q], su[2][q]} : ld3(uc, g.id(kk, jj, ii));
    };
    auto UA = [&](int kk, int jj, int ii, double w, R3<double> v) { aadd3(cta, g.id(kk, jj, ii), w, v); };
    auto NUT = [&](int kk, int jj, int ii) { const int q = tq(kk, jj, ii); return q >= 0 ? sn[q] : nut[g.id(kk, jj, ii)]; };
    auto NA = [&](int kk, int jj, int ii, double v) { aadd(na + g.id(kk, jj, ii), v); };
    auto quickW = [](double w, double q[4]) {
        if (w > 0) { q[0] = -0.125; q[1] = 0.75; q[2] = 0.375; q[3] = 0.0; }
        else       { q[0] = 0.0; q[1] = 0.375; q[2] = 0.75; q[3] = -0.125; }
    };
    // ---- i faces (the periodic face 0 is not read by the forward step)
    if (j != 0 && k != 0 && !(g.pi && i == 0)) {
        R3<double> gv = ld3(f1a, f);
        double ucv = ut.x[f];
        R3<double> ga = (-ucv) * gv;
        R3<double> uface;
        if (quickDiv) {
            int iL, iR;
            if (i == 0 || i == mx - 2) {
                if (g.pi && i == mx - 2) { iR = mx + 2; iL = i - 1; }
                else if (g.pi && i == 0) { iL = -3; iR = i + 2; }
                else if (i == 0) { iL = i; iR = i + 2; }
                else { iL = i - 1; iR = i + 1; }
            } else { iL = i - 1; iR = i + 2; }
            double w[4]; quickW(ucv, w);
            uface = w[0] * U(k, j, iL) + w[1] * U(k, j, i) + w[2] * U(k, j, i + 1) + w[3] * U(k, j, iR);
            UA(k, j, iL, w[0], ga); UA(k, j, i, w[1], ga); UA(k, j, i + 1, w[2], ga); UA(k, j, iR, w[3], ga);
        } else {
            uface = 0.5 * (U(k, j, i) + U(k, j, i + 1));
            UA(k, j, i, 0.5, ga); UA(k, j, i + 1, 0.5, ga);
        }
        uta.x[f] += -dot3(gv, uface);
        double nuEff; bool vnut = false;
        if (p.les) {
            if ((p.bc[TG_ILEFT] == TG_BC_SLIP && i == 0) || (p.bc[TG_IRIGHT] == TG_BC_SLIP && i == mx - 2)) nuEff = 0.0;
            else { nuEff = nu + 0.5 * (NUT(k, j, i) + NUT(k, j, i + 1)); vnut = true; }
        } else nuEff = nu;
        R3<double> dd[3];
        if (AX) visc_adj_ax(m.icsi.y[f], m.ieta.z[f], m.izet.x[f], 0, gv, m.iaj[f], dd);
        else visc_adj(ld3(m.icsi, f), ld3(m.ieta, f), ld3(m.izet, f), 0, gv, m.iaj[f], dd);
        bool edge = (i == 0 || i == mx - 2);
        // stencil weights of (dc, de, dz): dc = U(i+1) - U(i)
        int jo = (j == my - 2 && edge && (npj || npi)) ? 1 : ((j == 1 && edge && (npj || npi)) ? 2 : 0);
        int ko = (k == mz - 2 && edge && (npk || npi)) ? 1 : ((k == 1 && edge && (npk || npi)) ? 2 : 0);
        if (vnut) {
            R3<double> dc = U(k, j, i + 1) - U(k, j, i), de, dz;
            if (jo == 1) de = 0.5 * (U(k, j, i + 1) + U(k, j, i) - U(k, j - 1, i + 1) - U(k, j - 1, i));
            else if (jo == 2) de = 0.5 * (U(k, j + 1, i + 1) + U(k, j + 1, i) - U(k, j, i + 1) - U(k, j, i));
            else de = 0.25 * (U(k, j + 1, i + 1) + U(k, j + 1, i) - U(k, j - 1, i + 1) - U(k, j - 1, i));
            if (ko == 1) dz = 0.5 * (U(k, j, i + 1) + U(k, j, i) - U(k - 1, j, i + 1) - U(k - 1, j, i));
            else if (ko == 2) dz = 0.5 * (U(k + 1, j, i + 1) + U(k + 1, j, i) - U(k, j, i + 1) - U(k, j, i));
            else dz = 0.25 * (U(k + 1, j, i + 1) + U(k + 1, j, i) - U(k - 1, j, i + 1) - U(k - 1, j, i));
            double ne = dot3(dd[0], dc) + dot3(dd[1], de) + dot3(dd[2], dz);
            NA(k, j, i, 0.5 * ne); NA(k, j, i + 1, 0.5 * ne);
        }
        for (int q = 0; q < 3; q++) dd[q] = nuEff * dd[q];
        UA(k, j, i + 1, 1.0, dd[0]); UA(k, j, i, -1.0, dd[0]);
        if (jo == 1)      { UA(k, j, i + 1, 0.5, dd[1]); UA(k, j, i, 0.5, dd[1]); UA(k, j - 1, i + 1, -0.5, dd[1]); UA(k, j - 1, i, -0.5, dd[1]); }
        else if (jo == 2) { UA(k, j + 1, i + 1, 0.5, dd[1]); UA(k, j + 1, i, 0.5, dd[1]); UA(k, j, i + 1, -0.5, dd[1]); UA(k, j, i, -0.5, dd[1]); }
        else              { UA(k, j + 1, i + 1, 0.25, dd[1]); UA(k, j + 1, i, 0.25, dd[1]); UA(k, j - 1, i + 1, -0.25, dd[1]); UA(k, j - 1, i, -0.25, dd[1]); }
        if (ko == 1)      { UA(k, j, i + 1, 0.5, dd[2]); UA(k, j, i, 0.5, dd[2]); UA(k - 1, j, i + 1, -0.5, dd[2]); UA(k - 1, j, i, -0.5, dd[2]); }
        else if (ko == 2) { UA(k + 1, j, i + 1, 0.5, dd[2]); UA(k + 1, j, i, 0.5, dd[2]); UA(k, j, i + 1, -0.5, dd[2]); UA(k, j, i, -0.5, dd[2]); }
        else              { UA(k + 1, j, i + 1, 0.25, dd[2]); UA(k + 1, j, i, 0.25, dd[2]); UA(k - 1, j, i + 1, -0.25, dd[2]); UA(k - 1, j, i, -0.25, dd[2]); }
    }
    // ---- j faces
    if (i != 0 && k != 0 && !(g.pj && j == 0)) {
        R3<double> gv = ld3(f2a, f);
        double ucv = ut.y[f];
        R3<double> ga = (-ucv) * gv;
        R3<double> uface;
        if (quickDiv) {
            int jL, jR;
            if (j == 0 || j == my - 2) {
                if (g.pj && j == my - 2) { jR = my + 2; jL = j - 1; }
                else if (g.pj && j == 0) { jL = -3; jR = j + 2; }
                else if (j == 0) { jL = j; jR = j + 2; }
                else { jL = j - 1; jR = j + 1; }
            } else { jL = j - 1; jR = j + 2; }
            double w[4]; quickW(ucv, w);
            uface = w[0] * U(k, jL, i) + w[1] * U(k, j, i) + w[2] * U(k, j + 1, i) + w[3] * U(k, jR, i);
            UA(k, jL, i, w[0], ga); UA(k, j, i, w[1], ga); UA(k, j + 1, i, w[2], ga); UA(k, jR, i, w[3], ga);
        } else {
            uface = 0.5 * (U(k, j, i) + U(k, j + 1, i));
            UA(k, j, i, 0.5, ga); UA(k, j + 1, i, 0.5, ga);
        }
        uta.y[f] += -dot3(gv, uface);
        double nuEff; bool vnut = false;
        if (p.les) {
            if ((p.bc[TG_JLEFT] == TG_BC_WALL_SHUMANN && j == 0) || (p.bc[TG_JRIGHT] == TG_BC_WALL_SHUMANN && j == my - 2)) {
                // the face flux holds -tauWall (ueqn_solvers.c:548-558)
                aadd3(twa, k * mx + i, -1.0, gv);
                nuEff = nu;
            } else if ((p.bc[TG_JLEFT] == TG_BC_SLIP && j == 0) || (p.bc[TG_JRIGHT] == TG_BC_SLIP && j == my - 2)) nuEff = 0.0;
            else { nuEff = nu + 0.5 * (NUT(k, j, i) + NUT(k, j + 1, i)); vnut = true; }
        } else nuEff = nu;
        R3<double> dd[3];
        if (AX) visc_adj_ax(m.jcsi.y[f], m.jeta.z[f], m.jzet.x[f], 1, gv, m.jaj[f], dd);
        else visc_adj(ld3(m.jcsi, f), ld3(m.jeta, f), ld3(m.jzet, f), 1, gv, m.jaj[f], dd);
        bool edge = (j == 0 || j == my - 2);
        int io = (i == mx - 2 && edge && (npi || npj)) ? 1 : ((i == 1 && edge && (npi || npj)) ? 2 : 0);
        int ko = (k == mz - 2 && edge && (npk || npj)) ? 1 : ((k == 1 && edge && (npk || npj)) ? 2 : 0);
        if (vnut) {
            R3<double> dc, de = U(k, j + 1, i) - U(k, j, i), dz;
            if (io == 1) dc = 0.5 * (U(k, j + 1, i) + U(k, j, i) - U(k, j + 1, i - 1) - U(k, j, i - 1));
            else if (io == 2) dc = 0.5 * (U(k, j + 1, i + 1) + U(k, j, i + 1) - U(k, j + 1, i) - U(k, j, i));
            else dc = 0.25 * (U(k, j + 1, i + 1) + U(k, j, i + 1) - U(k, j + 1, i - 1) - U(k, j, i - 1));
            if (ko == 1) dz = 0.5 * (U(k, j + 1, i) + U(k, j, i) - U(k - 1, j + 1, i) - U(k - 1, j, i));
            else if (ko == 2) dz = 0.5 * (U(k + 1, j + 1, i) + U(k + 1, j, i) - U(k, j + 1, i) - U(k, j, i));
            else dz = 0.25 * (U(k + 1, j + 1, i) + U(k + 1, j, i) - U(k - 1, j + 1, i) - U(k - 1, j, i));
            double ne = dot3(dd[0], dc) + dot3(dd[1], de) + dot3(dd[2], dz);
            NA(k, j, i, 0.5 * ne); NA(k, j + 1, i, 0.5 * ne);
        }
        for (int q = 0; q < 3; q++) dd[q] = nuEff * dd[q];
        UA(k, j + 1, i, 1.0, dd[1]); UA(k, j, i, -1.0, dd[1]);
        if (io == 1)      { UA(k, j + 1, i, 0.5, dd[0]); UA(k, j, i, 0.5, dd[0]); UA(k, j + 1, i - 1, -0.5, dd[0]); UA(k, j, i - 1, -0.5, dd[0]); }
        else if (io == 2) { UA(k, j + 1, i + 1, 0.5, dd[0]); UA(k, j, i + 1, 0.5, dd[0]); UA(k, j + 1, i, -0.5, dd[0]); UA(k, j, i, -0.5, dd[0]); }
        else              { UA(k, j + 1, i + 1, 0.25, dd[0]); UA(k, j, i + 1, 0.25, dd[0]); UA(k, j + 1, i - 1, -0.25, dd[0]); UA(k, j, i - 1, -0.25, dd[0]); }
        if (ko == 1)      { UA(k, j + 1, i, 0.5, dd[2]); UA(k, j, i, 0.5, dd[2]); UA(k - 1, j + 1, i, -0.5, dd[2]); UA(k - 1, j, i, -0.5, dd[2]); }
        else if (ko == 2) { UA(k + 1, j + 1, i, 0.5, dd[2]); UA(k + 1, j, i, 0.5, dd[2]); UA(k, j + 1, i, -0.5, dd[2]); UA(k, j, i, -0.5, dd[2]); }
        else              { UA(k + 1, j + 1, i, 0.25, dd[2]); UA(k + 1, j, i, 0.25, dd[2]); UA(k - 1, j + 1, i, -0.25, dd[2]); UA(k - 1, j, i, -0.25, dd[2]); }
    }
    // ---- k faces
    if (i != 0 && j != 0 && !(g.pk && k == 0)) {
        R3<double> gv = ld3(f3a, f);
        double ucv = ut.z[f];
        R3<double> ga = (-ucv) * gv;
        R3<double> uface;
        if (quickDiv) {
            int kL, kR;
            if (k == 0 || k == mz - 2) {
                if (g.pk && k == mz - 2) { kR = mz + 2; kL = k - 1; }
                else if (g.pk && k == 0) { kL = -3; kR = k + 2; }
                else if (k == 0) { kL = k; kR = k + 2; }
                else { kL = k - 1; kR = k + 1; }
            } else { kL = k - 1; kR = k + 2; }
            double w[4]; quickW(ucv, w);
            uface = w[0] * U(kL, j, i) + w[1] * U(k, j, i) + w[2] * U(k + 1, j, i) + w[3] * U(kR, j, i);
            UA(kL, j, i, w[0], ga); UA(k, j, i, w[1], ga); UA(k + 1, j, i, w[2], ga); UA(kR, j, i, w[3], ga);
        } else {
            uface = 0.5 * (U(k, j, i) + U(k + 1, j, i));
            UA(k, j, i, 0.5, ga); UA(k + 1, j, i, 0.5, ga);
        }
        uta.z[f] += -dot3(gv, uface);
        double nuEff; bool vnut = false;
        if (p.les) {
            if ((p.bc[TG_KLEFT] == TG_BC_SLIP && k == 0) || (p.bc[TG_KRIGHT] == TG_BC_SLIP && k == mz - 2)) nuEff = 0.0;
            else { nuEff = nu + 0.5 * (NUT(k, j, i) + NUT(k + 1, j, i)); vnut = true; }
        } else nuEff = nu;
        R3<double> dd[3];
        if (AX) visc_adj_ax(m.kcsi.y[f], m.keta.z[f], m.kzet.x[f], 2, gv, m.kaj[f], dd);
        else visc_adj(ld3(m.kcsi, f), ld3(m.keta, f), ld3(m.kzet, f), 2, gv, m.kaj[f], dd);
        bool edge = (k == 0 || k == mz - 2);
        int io = (i == mx - 2 && edge && (npi || npk)) ? 1 : ((i == 1 && edge && (npi || npk)) ? 2 : 0);
        int jo = (j == my - 2 && edge && (npj || npk)) ? 1 : ((j == 1 && edge && (npj || npk)) ? 2 : 0);
        if (vnut) {
            R3<double> dc, de, dz = U(k + 1, j, i) - U(k, j, i);
            if (io == 1) dc = 0.5 * (U(k + 1, j, i) + U(k, j, i) - U(k + 1, j, i - 1) - U(k, j, i - 1));
            else if (io == 2) dc = 0.5 * (U(k + 1, j, i + 1) + U(k, j, i + 1) - U(k + 1, j, i) - U(k, j, i));
            else dc = 0.25 * (U(k + 1, j, i + 1) + U(k, j, i + 1) - U(k + 1, j, i - 1) - U(k, j, i - 1));
            if (jo == 1) de = 0.5 * (U(k + 1, j, i) + U(k, j, i) - U(k + 1, j - 1, i) - U(k, j - 1, i));
            else if (jo == 2) de = 0.5 * (U(k + 1, j + 1, i) + U(k, j + 1, i) - U(k + 1, j, i) - U(k, j, i));
            else de = 0.25 * (U(k + 1, j + 1, i) + U(k, j + 1, i) - U(k + 1, j - 1, i) - U(k, j - 1, i));
            double ne = dot3(dd[0], dc) + dot3(dd[1], de) + dot3(dd[2], dz);
            NA(k, j, i, 0.5 * ne); NA(k + 1, j, i, 0.5 * ne);
        }
        for (int q = 0; q < 3; q++) dd[q] = nuEff * dd[q];
        UA(k + 1, j, i, 1.0, dd[2]); UA(k, j, i, -1.0, dd[2]);
        if (io == 1)      { UA(k + 1, j, i, 0.5, dd[0]); UA(k, j, i, 0.5, dd[0]); UA(k + 1, j, i - 1, -0.5, dd[0]); UA(k, j, i - 1, -0.5, dd[0]); }
        else if (io == 2) { UA(k + 1, j, i + 1, 0.5, dd[0]); UA(k, j, i + 1, 0.5, dd[0]); UA(k + 1, j, i, -0.5, dd[0]); UA(k, j, i, -0.5, dd[0]); }
        else              { UA(k + 1, j, i + 1, 0.25, dd[0]); UA(k, j, i + 1, 0.25, dd[0]); UA(k + 1, j, i - 1, -0.25, dd[0]); UA(k, j, i - 1, -0.25, dd[0]); }
        if (jo == 1)      { UA(k + 1, j, i, 0.5, dd[1]); UA(k, j, i, 0.5, dd[1]); UA(k + 1, j - 1, i, -0.5, dd[1]); UA(k, j - 1, i, -0.5, dd[1]); }
        else if (jo == 2) { UA(k + 1, j + 1, i, 0.5, dd[1]); UA(k, j + 1, i, 0.5, dd[1]); UA(k + 1, j, i, -0.5, dd[1]); UA(k, j, i, -0.5, dd[1]); }
        else              { UA(k + 1, j + 1, i, 0.25, dd[1]); UA(k, j + 1, i, 0.25, dd[1]); UA(k + 1, j - 1, i, -0.25, dd[1]); UA(k, j - 1, i, -0.25, dd[1]); }
    }
}

// ------------------------------------------------------------------- GradP
__global__ void k_adj_grad_p(Grid g, Metrics m, V3f<double> dpa, double *pa)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    const int mx = g.mx, my = g.my, mz = g.mz;
    int c = g.lin(k, j, i);
    auto P = [&](int kk, int jj, int ii, double w) { aadd(pa + g.id(kk, jj, ii), w); };
    R3<double> ic = ld3(m.icsi, c), ie = ld3(m.ieta, c), iz = ld3(m.izet, c);
    R3<double> jc = ld3(m.jcsi, c), je = ld3(m.jeta, c), jz = ld3(m.jzet, c);
    R3<double> kc = ld3(m.kcsi, c), ke = ld3(m.keta, c), kz = ld3(m.kzet, c);
    double g11 = dot3(ic, ic), g12 = dot3(ie, ic), g13 = dot3(iz, ic);
    double g21 = dot3(jc, je), g22 = dot3(je, je), g23 = dot3(jz, je);
    double g31 = dot3(kc, kz), g32 = dot3(ke, kz), g33 = dot3(kz, kz);
    R3<double> o = ld3(dpa, c);
    if (!g.pi && i == mx - 2) o.x = 0;
    if (!g.pj && j == my - 2) o.y = 0;
    if (!g.pk && k == mz - 2) o.z = 0;
    {
        double a = o.x * m.iaj[c], wc = a * g11, we = a * g12, wz = a * g13;
        if (i == mx - 2 && g.pi) { P(k, j, mx + 1, wc); P(k, j, i, -wc); } else { P(k, j, i + 1, wc); P(k, j, i, -wc); }
        if (j == my - 2 && i == mx - 2)  { double w = 0.5 * we; P(k, j, i, w); P(k, j - 1, i, -w); P(k, j, i + 1, w); P(k, j - 1, i + 1, -w); }
        else if (j == 1 && i == mx - 2)  { double w = 0.5 * we; P(k, j + 1, i, w); P(k, j, i, -w); P(k, j + 1, i + 1, w); P(k, j, i + 1, -w); }
        else                             { double w = 0.25 * we; P(k, j + 1, i, w); P(k, j - 1, i, -w); P(k, j + 1, i + 1, w); P(k, j - 1, i + 1, -w); }
        if (k == mz - 2 && i == mx - 2)  { double w = 0.5 * wz; P(k, j, i, w); P(k - 1, j, i, -w); P(k, j, i + 1, w); P(k - 1, j, i + 1, -w); }
        else if (k == 1 && i == mx - 2)  { double w = 0.5 * wz; P(k + 1, j, i, w); P(k, j, i, -w); P(k + 1, j, i + 1, w); P(k, j, i + 1, -w); }
        else                             { double w = 0.25 * wz; P(k + 1, j, i, w); P(k - 1, j, i, -w); P(k + 1, j, i + 1, w); P(k - 1, j, i + 1, -w); }
    }
    {
        double a = o.y * m.jaj[c], wc = a * g21, we = a * g22, wz = a * g23;
        if (i == mx - 2 && j == my - 2)  { double w = 0.5 * wc; P(k, j, i, w); P(k, j, i - 1, -w); P(k, j + 1, i, w); P(k, j + 1, i - 1, -w); }
        else if (i == 1 && j == my - 2)  { double w = 0.5 * wc; P(k, j, i + 1, w); P(k, j, i, -w); P(k, j + 1, i + 1, w); P(k, j + 1, i, -w); }
        else                             { double w = 0.25 * wc; P(k, j, i + 1, w); P(k, j, i - 1, -w); P(k, j + 1, i + 1, w); P(k, j + 1, i - 1, -w); }
        if (j == my - 2 && g.pj) { P(k, my + 1, i, we); P(k, j, i, -we); } else { P(k, j + 1, i, we); P(k, j, i, -we); }
        if (k == mz - 2 && j == my - 2)  { double w = 0.5 * wz; P(k, j, i, w); P(k - 1, j, i, -w); P(k, j + 1, i, w); P(k - 1, j + 1, i, -w); }
        else if (k == 1 && j == my - 2)  { double w = 0.5 * wz; P(k + 1, j, i, w); P(k, j, i, -w); P(k + 1, j + 1, i, w); P(k, j + 1, i, -w); }
        else                             { double w = 0.25 * wz; P(k + 1, j, i, w); P(k - 1, j, i, -w); P(k + 1, j + 1, i, w); P(k - 1, j + 1, i, -w); }
    }
    {
        double a = o.z * m.kaj[c], wc = a * g31, we = a * g32, wz = a * g33;
        if (i == mx - 2 && k == mz - 2)  { double w = 0.5 * wc; P(k, j, i, w); P(k, j, i - 1, -w); P(k + 1, j, i, w); P(k + 1, j, i - 1, -w); }
        else if (i == 1 && k == mz - 2)  { double w = 0.5 * wc; P(k, j, i + 1, w); P(k, j, i, -w); P(k + 1, j, i + 1, w); P(k + 1, j, i, -w); }
        else                             { double w = 0.25 * wc; P(k, j, i + 1, w); P(k, j, i - 1, -w); P(k + 1, j, i + 1, w); P(k + 1, j, i - 1, -w); }
        if (j == my - 2 && k == mz - 2)  { double w = 0.5 * we; P(k, j, i, w); P(k, j - 1, i, -w); P(k + 1, j, i, w); P(k + 1, j - 1, i, -w); }
        else if (j == 1 && k == mz - 2)  { double w = 0.5 * we; P(k, j + 1, i, w); P(k, j, i, -w); P(k + 1, j + 1, i, w); P(k + 1, j, i, -w); }
        else                             { double w = 0.25 * we; P(k, j + 1, i, w); P(k, j - 1, i, -w); P(k + 1, j + 1, i, w); P(k + 1, j - 1, i, -w); }
        if (k == mz - 2 && g.pk) { P(mz + 1, j, i, wz); P(k, j, i, -wz); } else { P(k + 1, j, i, wz); P(k, j, i, -wz); }
    }
}

// -------------------------------------------------------------- Smagorinsky
__global__ void k_adj_smagorinsky(Grid g, Metrics m, V3f<double> ucat, const double *na, Params p, V3f<double> ca)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int c = g.lin(k, j, i);
    double nav = na[c];
    if (nav == 0.0) return;
    double ajc = m.aj[c];
    R3<double> s = ld3(m.csi, c), e = ld3(m.eta, c), z = ld3(m.zet, c);
    int tq[3][2]; double tw[3][2];
    auto set = [&](int d, int qa, double wa, int qb, double wb) { tq[d][0] = qa; tw[d][0] = wa; tq[d][1] = qb; tw[d][1] = wb; };
    if (!g.pi && i == g.mx - 2)  set(0, g.id(k, j, i), 1.0, g.id(k, j, i - 1), -1.0);
    else if (!g.pi && i == 1)    set(0, g.id(k, j, i + 1), 1.0, g.id(k, j, i), -1.0);
    else                         set(0, g.id(k, j, i + 1), 0.5, g.id(k, j, i - 1), -0.5);
    if (!g.pj && j == g.my - 2)  set(1, g.id(k, j, i), 1.0, g.id(k, j - 1, i), -1.0);
    else if (!g.pj && j == 1)    set(1, g.id(k, j + 1, i), 1.0, g.id(k, j, i), -1.0);
    else                         set(1, g.id(k, j + 1, i), 0.5, g.id(k, j - 1, i), -0.5);
    if (!g.pk && k == g.mz - 2)  set(2, g.id(k, j, i), 1.0, g.id(k - 1, j, i), -1.0);
    else if (!g.pk && k == 1)    set(2, g.id(k + 1, j, i), 1.0, g.id(k, j, i), -1.0);
    else                         set(2, g.id(k + 1, j, i), 0.5, g.id(k - 1, j, i), -0.5);
    R3<double> d[3];
    for (int q = 0; q < 3; q++) d[q] = tw[q][0] * ld3(ucat, tq[q][0]) + tw[q][1] * ld3(ucat, tq[q][1]);
    const R3<double> mm[3] = {s, e, z};
    auto comp = [](const R3<double> &v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); };
    double G[3][3];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double acc = 0.0;
            for (int q = 0; q < 3; q++) acc += comp(d[q], a) * comp(mm[q], b);
            G[a][b] = acc * ajc;
        }
    double S[3][3], ss = 0.0;
    for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) { S[a][b] = 0.5 * (G[a][b] + G[b][a]); ss += S[a][b] * S[a][b]; }
    double Sabs = sqrt(2.0 * ss);
    if (!(Sabs > 0.0)) return;
    double filter = pow(1. / ajc, 1. / 3.);
    double coef = p.cs * pow(filter, 2.0) * nav;
    double dd[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double gb = coef * 2.0 * S[a][b] / Sabs * ajc;
            for (int q = 0; q < 3; q++) dd[q][a] += gb * comp(mm[q], b);
        }
    for (int q = 0; q < 3; q++)
        for (int t = 0; t < 2; t++) {
            R3<double> v{dd[q][0], dd[q][1], dd[q][2]};
            aadd3(ca, tq[q][t], tw[q][t], v);
        }
}

}  // namespace

// ===================================================================== host
// ------------------------------------------------- UpdateWallModelsU reverse
// Forward (k_wall_stress, Cartesian branch): per plane cell w at j = 1,
// Up = U - (U.n) n, Umean = mean |Up|, u* = max(0, kappa Umean / ln(d/z0)),
// S = u*^2, D = max(Umean, 1e-5); umean' = m1 umean + m2 |Up|;
// r = dt / max(L/umean', dt); uf' = (1-r) uf + r Up (x, y; uf = Up on the
// seeding step); tau = -S uf' / D; tw = (je.z tau_x, je.z tau_y, je.x tau_x +
// je.y tau_y). The reverse maps the tauWall adjoint (from FormU) and the
// adjoint of the state after the step (wxa, wya, wma) to the adjoint of the
// step-start Ucat at j = 1 and of the step-start wall state. Plane sums are
// per-block trees summed in a fixed order (bitwise reproducible).
constexpr int WNB = 148;     // blocks of the plane reductions

__device__ __forceinline__ void wall_par(const Grid &g, const Metrics &m, const V3f<double> &ucat, int k, int i,
                                         R3<double> &Up, R3<double> &n)
{
    const int c = g.lin(k, 1, i);
    calc_normal_adj(ld3(m.csi, c), ld3(m.eta, c), ld3(m.zet, c), 1, n);
    const R3<double> U = ld3(ucat, c);
    Up = U - dot3(U, n) * n;
}

// block sums of (a, b) into part[2 blockIdx], part[2 blockIdx + 1]
// (blocks of 256 threads)
__device__ __forceinline__ void block_sum2(double a, double b, double *part)
{
    double v[2] = {a, b};
    block_reduce<256>(v, RedSum{}, RedSum{});
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = v[0]; part[2 * blockIdx.x + 1] = v[1]; }
}

// forward plane sums of |Up| and the wall distance (the step-start Ucat)
__global__ void __launch_bounds__(256) k_adj_wall_fwd(Grid g, Metrics m, V3f<double> ucat, double *part)
{
    const int nI = g.mx - 2, nK = g.mz - 2;
    double su = 0.0, sd = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nI * nK; t += gridDim.x * blockDim.x) {
        const int i = t % nI + 1, k = t / nI + 1, c = g.lin(k, 1, i);
        const double area = sqrt(dot3(ld3(m.eta, c), ld3(m.eta, c)));
        R3<double> Up, n; wall_par(g, m, ucat, k, i, Up, n);
        su += sqrt(dot3(Up, Up));
        sd += 0.5 / m.aj[c] / area;
    }
    block_sum2(su, sd, part);
}
// wsc <- Umean, dist, u*, S, D, logLaw
__global__ void k_adj_wall_fwd_final(Grid g, Params p, const double *part, double *wsc)
{
    double su = 0.0, sd = 0.0;
    for (int b = 0; b < WNB; b++) { su += part[2 * b]; sd += part[2 * b + 1]; }
    const double cnt = (double)(g.mx - 2) * (double)(g.mz - 2);
    const double Umean = su / cnt, dist = sd / cnt, logLaw = log(dist / p.z0);
    const double us = fmax(0.0, (p.kappa * Umean) / logLaw);
    wsc[0] = Umean; wsc[1] = dist; wsc[2] = us; wsc[3] = us * us; wsc[4] = fmax(Umean, 1e-5); wsc[5] = logLaw;
}
// per cell: filter and running-mean reverse; block sums of the S and D adjoints
__global__ void __launch_bounds__(256) k_adj_wall_local(Grid g, Metrics m, Params p, V3f<double> ucat, const double *wum0,
                                                        const double *wfx0, const double *wfy0, const double *meta,
                                                        V3f<double> twa, double *wxa, double *wya, double *wma,
                                                        V3f<double> upa, double *upma, const double *wsc, double *part)
{
    const int nI = g.mx - 2, nK = g.mz - 2;
    const double aN = meta[0], m1 = aN / (aN + 1.0), m2 = 1.0 / (aN + 1.0);
    const bool seed = meta[1] != 0.0;
    const double S = wsc[3], D = wsc[4], dt = p.dt;
    double sa = 0.0, da = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nI * nK; t += gridDim.x * blockDim.x) {
        const int i = t % nI + 1, k = t / nI + 1, c = g.lin(k, 1, i), w = k * g.mx + i;
        R3<double> Up, n; wall_par(g, m, ucat, k, i, Up, n);
        const double upm = sqrt(dot3(Up, Up));
        const double um = m1 * wum0[w] + m2 * upm;
        const R3<double> zz = ld3(m.zet, c), cc = ld3(m.csi, c);
        const double lx = 1.0 / m.aj[c] / sqrt(dot3(zz, zz)), ly = 1.0 / m.aj[c] / sqrt(dot3(cc, cc));
        const double L = sqrt(lx * lx + ly * ly);
        const bool filt = L / um > dt;
        const double r = dt / (filt ? L / um : dt);
        const double fx0 = seed ? Up.x : wfx0[w], fy0 = seed ? Up.y : wfy0[w];
        const double fx = (1.0 - r) * fx0 + r * Up.x, fy = (1.0 - r) * fy0 + r * Up.y;
        const R3<double> je = ld3(m.jeta, g.lin(k, 0, i));
        const double txa = je.z * twa.x[w] + je.x * twa.z[w];
        const double tya = je.z * twa.y[w] + je.y * twa.z[w];
        const double fxa = wxa[w] + txa * (-S / D), fya = wya[w] + tya * (-S / D);
        sa += txa * (-fx / D) + tya * (-fy / D);
        da += txa * (S * fx / (D * D)) + tya * (S * fy / (D * D));
        double fx0a = (1.0 - r) * fxa, fy0a = (1.0 - r) * fya;
        R3<double> pa{r * fxa, r * fya, 0.0};
        const double ra = (Up.x - fx0) * fxa + (Up.y - fy0) * fya;
        const double uma = wma[w] + (filt ? ra * dt / L : 0.0);
        if (seed) { pa.x += fx0a; pa.y += fy0a; fx0a = 0.0; fy0a = 0.0; }
        wxa[w] = fx0a; wya[w] = fy0a; wma[w] = m1 * uma;
        upma[w] = m2 * uma;
        st3(upa, w, pa);
    }
    block_sum2(sa, da, part);
}
// wsc[6] <- adjoint of Umean
__global__ void k_adj_wall_mean(Grid g, Params p, const double *part, double *wsc)
{
    double sa = 0.0, da = 0.0;
    for (int b = 0; b < WNB; b++) { sa += part[2 * b]; da += part[2 * b + 1]; }
    const double Umean = wsc[0], us = wsc[2], logLaw = wsc[5];
    wsc[6] = (us > 0.0 ? sa * 2.0 * us * p.kappa / logLaw : 0.0) + (Umean > 1e-5 ? da : 0.0);
}
// Up and |Up| adjoints (with the plane mean's share) into the Ucat adjoint at j = 1
__global__ void k_adj_wall_scatter(Grid g, Metrics m, V3f<double> ucat, V3f<double> upa, const double *upma,
                                   const double *wsc, V3f<double> ca)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, k = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.mx - 2 || k > g.mz - 2) return;
    const int c = g.lin(k, 1, i), w = k * g.mx + i;
    const double cnt = (double)(g.mx - 2) * (double)(g.mz - 2);
    R3<double> Up, n; wall_par(g, m, ucat, k, i, Up, n);
    const double upm = sqrt(dot3(Up, Up));
    const double ma = upma[w] + wsc[6] / cnt;
    R3<double> pa = ld3(upa, w);
    if (upm > 0.0) pa = pa + (ma / upm) * Up;
    aadd3(ca, c, 1.0, pa - dot3(pa, n) * n);
}
__global__ void k_tape_wall_meta(double *meta, const double *d_it, double seed) { meta[0] = d_it[0]; meta[1] = seed; }

struct ApiFail { tg_status s; std::string msg; };

static V3f<double> alloc3(tg_ctx *C) { return dalloc3(C, (size_t)C->g.size()); }

static size_t wall_plane(const tg_ctx *C) { return (size_t)C->g.mx * C->g.mz; }
static bool wall_on(const tg_ctx *C) { return C->prm.les && C->prm.bc[TG_JLEFT] == TG_BC_WALL_SHUMANN; }

static AdjState &adj_state(tg_ctx *C)
{
    if (!C->adj) {
        AdjState *A = new AdjState();
        C->adj = A;
        A->ua = alloc3(C); A->ca = alloc3(C); A->fa = alloc3(C);
        A->pa = dallocd(C, (size_t)C->g.size());
        A->wxa = dallocd(C, wall_plane(C)); A->wya = dallocd(C, wall_plane(C)); A->wma = dallocd(C, wall_plane(C));
    }
    return *C->adj;
}

static Tape make_tape(tg_ctx *C)
{
    Tape t;
    t.u_o = alloc3(C); t.ucat_n = alloc3(C);
    for (int q = 0; q < 4; q++) { t.ut[q] = alloc3(C); t.uc[q] = alloc3(C); }
    t.nut = dallocd(C, (size_t)C->g.size());
    t.wum = dallocd(C, wall_plane(C)); t.wfx = dallocd(C, wall_plane(C)); t.wfy = dallocd(C, wall_plane(C));
    t.meta = dallocd(C, 2);
    return t;
}
static size_t tape_bytes(tg_ctx *C) { return (size_t)C->g.size() * sizeof(double) * (3 * 10 + 1); }

static void adj_work(tg_ctx *C)
{
    AdjState &A = adj_state(C);
    if (A.work) return;
    const size_t G = (size_t)C->g.size();
    V3f<double> *v[] = {&A.uoa, &A.usa, &A.uta, &A.cta, &A.ra, &A.dpa, &A.fpa, &A.f1a, &A.f2a, &A.f3a, &A.qa};
    for (auto *p : v) *p = alloc3(C);
    A.pha = dallocd(C, G); A.na = dallocd(C, G);
    A.lam = dallocd(C, (size_t)poisson_n(C)); A.rhsc = dallocd(C, (size_t)poisson_n(C));
    A.lam_prev = dallocd(C, (size_t)poisson_n(C)); A.lam_prev2 = dallocd(C, (size_t)poisson_n(C));
    A.work_tape = make_tape(C);
    A.cur = &A.work_tape;
    for (int q = 0; q < 3; q++) A.twa[q] = dallocd(C, wall_plane(C));
    for (int q = 0; q < 4; q++) A.upa[q] = dallocd(C, wall_plane(C));
    A.wpart = dallocd(C, 2 * WNB);
    A.wsc = dallocd(C, 8);
    A.work = true;
}

bool adj_wall_field(tg_ctx *C, double *&x, double *&y, double *&m)
{
    AdjState &A = adj_state(C);
    x = A.wxa; y = A.wya; m = A.wma;
    return true;
}

bool adj_field(tg_ctx *C, int w, V3f<double> &v, double *&s)
{
    if (w != TG_F_UCONT_ADJ && w != TG_F_UCAT_ADJ && w != TG_F_P_ADJ && w != TG_F_SOURCE_ADJ) return false;
    AdjState &A = adj_state(C);
    s = nullptr;
    if (w == TG_F_UCONT_ADJ) v = A.ua;
    else if (w == TG_F_UCAT_ADJ) v = A.ca;
    else if (w == TG_F_SOURCE_ADJ) v = A.fa;
    else s = A.pa;
    return true;
}

void adj_graph_destroy(tg_ctx *C)
{
    if (!C->adj) return;
    if (C->adj->rev_exec) cudaGraphExecDestroy(C->adj->rev_exec);
    for (cudaGraphExec_t e : C->adj->rev_store) if (e) cudaGraphExecDestroy(e);
    C->adj->rev_store.clear();
    C->adj->rev_exec = nullptr;
    C->adj->rev_failed = false;
}

void adj_destroy(tg_ctx *C)
{
    adj_graph_destroy(C);
    delete C->adj;       // device buffers are owned by the context allocation list
    C->adj = nullptr;
}

bool tape_in_work(const tg_ctx *C) { return C->adj && C->adj->cur == &C->adj->work_tape; }

static void copy3(tg_ctx *C, V3f<double> dst, V3f<double> src)
{
    TG_CUDA(cudaMemcpyAsync(dst.x, src.x, 3 * sizeof(double) * (size_t)C->g.size(), cudaMemcpyDeviceToDevice, C->stream));
}
static void zero3(tg_ctx *C, V3f<double> v)
{
    TG_CUDA(cudaMemsetAsync(v.x, 0, 3 * sizeof(double) * (size_t)C->g.size(), C->stream));
}

static void copy_plane(tg_ctx *C, double *dst, const double *src, size_t n)
{
    TG_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
}

static void copy_tape(tg_ctx *C, Tape &dst, const Tape &src)
{
    copy_plane(C, dst.wum, src.wum, wall_plane(C));
    copy_plane(C, dst.wfx, src.wfx, wall_plane(C));
    copy_plane(C, dst.wfy, src.wfy, wall_plane(C));
    copy_plane(C, dst.meta, src.meta, 2);
    copy3(C, dst.u_o, src.u_o);
    copy3(C, dst.ucat_n, src.ucat_n);
    for (int q = 0; q < src.nst; q++) { copy3(C, dst.ut[q], src.ut[q]); copy3(C, dst.uc[q], src.uc[q]); }
    TG_CUDA(cudaMemcpyAsync(dst.nut, src.nut, sizeof(double) * (size_t)C->g.size(), cudaMemcpyDeviceToDevice, C->stream));
    dst.nst = src.nst;
}

void tape_step_start(tg_ctx *C)
{
    Tape &T = *C->adj->cur;
    copy3(C, T.u_o, C->s.ucont);
    copy3(C, T.ucat_n, C->s.ucat);
    if (wall_on(C)) {
        copy_plane(C, T.wum, C->s.umean, wall_plane(C));
        copy_plane(C, T.wfx, C->s.ufx, wall_plane(C));
        copy_plane(C, T.wfy, C->s.ufy, wall_plane(C));
        k_tape_wall_meta<<<1, 1, 0, C->stream>>>(T.meta, C->d_scal + SC_IT, C->ufilt_set ? 0.0 : 1.0);
    }
    T.nst = 0;
}
void tape_nut(tg_ctx *C)
{
    Tape &T = *C->adj->cur;
    TG_CUDA(cudaMemcpyAsync(T.nut, C->s.nut, sizeof(double) * (size_t)C->g.size(), cudaMemcpyDeviceToDevice, C->stream));
}
void tape_stage(tg_ctx *C)
{
    Tape &T = *C->adj->cur;
    if (T.nst >= 4) return;
    copy3(C, T.ut[T.nst], C->s.ucont);
    copy3(C, T.uc[T.nst], C->s.ucat);
    T.nst++;
}

// reverse per-direction copies
static void adj_periodic(tg_ctx *C, V3f<double> v, int left_only)
{
    const Grid g = C->g;
    if (g.pk) k_adj_periodic<<<g2(g.mx, g.my), b2, 0, C->stream>>>(g, v, 2, left_only);
    if (g.pj) k_adj_periodic<<<g2(g.mx, g.mz), b2, 0, C->stream>>>(g, v, 1, left_only);
    if (g.pi) k_adj_periodic<<<g2(g.my, g.mz), b2, 0, C->stream>>>(g, v, 0, left_only);
}
static void adj_scalar_ghosts(tg_ctx *C, double *v)
{
    const Grid g = C->g;
    k_adj_scalar_ghosts<<<g2(g.mx, g.my), b2, 0, C->stream>>>(g, v, 2);
    k_adj_scalar_ghosts<<<g2(g.mx, g.mz), b2, 0, C->stream>>>(g, v, 1);
    k_adj_scalar_ghosts<<<g2(g.my, g.mz), b2, 0, C->stream>>>(g, v, 0);
}
static void adj_contra(tg_ctx *C, V3f<double> ca, V3f<double> ua)
{
    AdjState &A = *C->adj;
    const Grid g = C->g;
    k_adj_contra_cells<<<gint(g), block3(), 0, C->stream>>>(g, C->m, ca, A.qa);
    k_adj_contra_faces<<<gfc(g), block3(), 0, C->stream>>>(g, A.qa, ua);
}

static bool adjoint_supported(tg_ctx *C, std::string &why)
{
    if (C->prm.bc[TG_JLEFT] == TG_BC_WALL_SHUMANN && C->prm.curvilinear) {
        why = "the adjoint of the curvilinear wall-stress branch is not implemented"; return false;
    }
    if (!C->orthogonal) { why = "the adjoint needs the symmetric (orthogonal-grid) pressure operator"; return false; }
    if (C->prm.teqn) { why = "the adjoint of the temperature equation is not implemented"; return false; }
    if (C->cfg.ddt_scheme == TG_DDT_CN) { why = "the adjoint of the Crank-Nicolson scheme is not implemented"; return false; }
    if (imex_scheme(C->cfg.ddt_scheme)) { why = "the adjoint of the IMEX schemes is not implemented"; return false; }
    for (int q = 0; q < 6; q++)
        if (C->prm.bc[q] >= TG_BC_FIXED_VALUE) {
            why = "the adjoint of the inflow/outflow patches (fixedValue, zeroGradient, inletFunction) is not implemented"; return false;
        }
    return true;
}

// reverse sweep of one recorded step (tape filled by a taped forward step from
// the state at its start); capture: the sweep is being recorded into a CUDA
// graph (device-side transposed-solve loop, statistics in the SC_ADJ slots)
static int adjoint_reverse_body(tg_ctx *C, bool capture)
{
    AdjState &A = *C->adj;
    const Tape &T = *A.cur;
    const Grid g = C->g;
    const int64_t G = g.size();
    cudaStream_t st = C->stream;
    const double dt = C->prm.dt;
    TG_PROF(C, "adj_misc", k_sum_partial<<<C->red_blocks, TB, 0, st>>>(G, A.pa, C->d_red));
    k_gauge_adj<<<1, 1, 0, st>>>(C->d_red, C->red_blocks, A.pa, g.lin(1, 1, 1));
    // UpdateContravariantBCs, UpdateCartesianBCs, contravariantToCartesian
    for (int d = 2; d >= 0; d--) {
        int na = d == 0 ? g.my : g.mx, nb = d == 2 ? g.my : g.mz;
        k_adj_contra_bcs<<<g2(na, nb), b2, 0, st>>>(g, C->m, A.ua, A.ca, C->prm, d);
    }
    {
        int na = std::max(g.mx, g.my) - 2, nb = std::max(g.my, g.mz) - 2;
        dim3 grid((na + 31) / 32, (nb + 7) / 8, 6);
        k_adj_cartesian_bcs<<<grid, b2, 0, st>>>(g, C->m, A.ca, C->prm);
    }
    adj_contra(C, A.ca, A.ua);
    zero3(C, A.ca);                                      // edge and corner ghosts: not read by any stencil
    // ProjectVelocity
    TG_CUDA(cudaMemsetAsync(A.pha, 0, sizeof(double) * G, st));
    TG_PROF(C, "adj_project", k_adj_project<<<gfc(g), block3(), 0, st>>>(g, C->m, A.ua, A.pha, dt));
    // UpdatePressure + ghosts, phi ghosts, phiToPhi
    adj_scalar_ghosts(C, A.pa);
    k_adj_update_pressure<<<gint(g), block3(), 0, st>>>(g, A.pa, A.pha, A.rhsc);
    adj_scalar_ghosts(C, A.pha);
    k_adj_phi_compact<<<gint(g), block3(), 0, st>>>(g, A.pha, A.rhsc);
    // started from the solutions of the previously reversed steps,
    // extrapolated like the forward solve's guess, to the context's
    // relative tolerance when that lies in [1e-14, 1e-8]; when the forward
    // solve stops on the divergence bound instead, to 1e-7, the relative
    // residual that bound leaves in the forward solve; else to 1e-8
    const double rt = C->cfg.poisson_rtol;
    const double artol = (rt >= 1e-14 && rt <= 1e-8) ? rt : (C->cfg.poisson_div_tol > 0.0 ? 1e-7 : 1e-8);
    int rc = 0;
    if (capture) {
        adjoint_guess(C, A.lam, A.lam_prev, A.lam_prev2, C->d_scal + SC_LHIST);
        poisson_solve_adjoint_capture(C, A.rhsc, A.lam, artol);
    } else {
        tg_stats ps{};
        adjoint_guess(C, A.lam, A.lam_prev, A.lam_prev2, C->d_scal + SC_LHIST);
        rc = poisson_solve_adjoint(C, A.rhsc, A.lam, artol, &ps);
        A.adj_iters += ps.poisson_iterations;
        if (rc == 3) return 3;
    }
    // SetRHS; u* = utmp after the tail flux resets
    copy3(C, A.usa, A.ua);
    TG_PROF(C, "adj_set_rhs", k_adj_set_rhs<<<gfc(g), block3(), 0, st>>>(g, A.lam, A.usa, dt));
    adj_periodic(C, A.usa, 1);
    k_adj_no_penetration<<<gfc(g), block3(), 0, st>>>(g, A.usa, C->prm);
    // stages
    copy3(C, A.uoa, A.usa);
    zero3(C, A.dpa);
    const bool wall = wall_on(C);
    if (wall) for (int q = 0; q < 3; q++) TG_CUDA(cudaMemsetAsync(A.twa[q], 0, sizeof(double) * wall_plane(C), st));
    const V3f<double> twa{A.twa[0], A.twa[1], A.twa[2]};
    TG_CUDA(cudaMemsetAsync(A.na, 0, sizeof(double) * G, st));
    const double bw[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    const double aw[4] = {0.0, 0.5, 0.5, 1.0};
    const bool rk = T.nst == 4;
    if (C->prm.farm) farm_adj_begin(C);
    for (int s = T.nst - 1; s >= 0; s--) {
        double cb = dt * (rk ? bw[s] : 1.0);
        double cn = (rk && s < 3) ? aw[s + 1] * dt : 0.0;
        TG_PROF(C, "adj_stage_rhs", k_adj_stage_rhs<<<gall(g), block3(), 0, st>>>(g, A.ra, A.usa, A.uta, cb, cn, T.u_o, A.dpa));
        if (C->prm.source) TG_PROF(C, "adj_source", k_adj_source<<<gall(g), block3(), 0, st>>>(g, C->m, A.ra, A.fa));
        if (C->prm.farm) farm_adj_stage(C, A.ra);
        // FormU transposed
        TG_PROF(C, "adj_rhs_faces", k_adj_rhs_faces<<<gint(g), block3(), 0, st>>>(g, C->m, A.ra, 1.0, A.fpa));
        TG_PROF(C, "adj_cell_fp", k_adj_cell_fp<<<gfc(g), block3(), 0, st>>>(g, A.fpa, A.f1a, A.f2a, A.f3a));
        zero3(C, A.uta);
        zero3(C, A.cta);
        if (C->axis_aligned)
            TG_PROF(C, "adj_face_fluxes", k_adj_face_fluxes<true><<<gfc(g), block3(), 0, st>>>(g, C->m, T.ut[s], T.uc[s], T.nut,
                                                          C->prm, A.f1a, A.f2a, A.f3a, A.uta, A.cta, A.na, twa));
        else
            TG_PROF(C, "adj_face_fluxes", k_adj_face_fluxes<false><<<gfc(g), block3(), 0, st>>>(g, C->m, T.ut[s], T.uc[s], T.nut,
                                                           C->prm, A.f1a, A.f2a, A.f3a, A.uta, A.cta, A.na, twa));
        // stage Ucat: periodic copies, interior from contravariantToCartesian, other ghosts from the state Ucat
        adj_periodic(C, A.cta, 0);
        adj_contra(C, A.cta, A.uta);
        TG_PROF(C, "adj_misc", k_axpy3<<<nblk1(G), TB, 0, st>>>(G, A.ca, 1.0, A.cta));
        // stage Ucont = Pf(Pnp(pre))
        adj_periodic(C, A.uta, 1);
        k_adj_no_penetration<<<gfc(g), block3(), 0, st>>>(g, A.uta, C->prm);
        TG_PROF(C, "adj_misc", k_axpy3<<<nblk1(G), TB, 0, st>>>(G, A.uoa, 1.0, A.uta));
    }
    // GradP
    TG_PROF(C, "adj_grad_p", k_adj_grad_p<<<gint(g), block3(), 0, st>>>(g, C->m, A.dpa, A.pa));
    // Smagorinsky
    if (C->prm.les) {
        int na = std::max(g.mx, g.my) - 2, nb = std::max(g.my, g.mz) - 2;
        dim3 grid((na + 31) / 32, (nb + 7) / 8, 6);
        k_adj_nut_bcs<<<grid, b2, 0, st>>>(g, A.na, C->prm);
        TG_PROF(C, "adj_smagorinsky", k_adj_smagorinsky<<<gint(g), block3(), 0, st>>>(g, C->m, T.ucat_n, A.na, C->prm, A.ca));
    }
    // the wall model (its stress feeds every stage; it reads the step-start Ucat)
    if (wall) {
        const V3f<double> upa{A.upa[0], A.upa[1], A.upa[2]};
        dim3 grid((g.mx - 2 + 31) / 32, (g.mz - 2 + 7) / 8);
        TG_PROF(C, "adj_wall", k_adj_wall_fwd<<<WNB, 256, 0, st>>>(g, C->m, T.ucat_n, A.wpart));
        k_adj_wall_fwd_final<<<1, 1, 0, st>>>(g, C->prm, A.wpart, A.wsc);
        TG_PROF(C, "adj_wall", k_adj_wall_local<<<WNB, 256, 0, st>>>(g, C->m, C->prm, T.ucat_n, T.wum, T.wfx, T.wfy, T.meta,
                                                                      twa, A.wxa, A.wya, A.wma, upa, A.upa[3], A.wsc, A.wpart));
        k_adj_wall_mean<<<1, 1, 0, st>>>(g, C->prm, A.wpart, A.wsc);
        TG_PROF(C, "adj_wall", k_adj_wall_scatter<<<grid, b2, 0, st>>>(g, C->m, T.ucat_n, upa, A.upa[3], A.wsc, A.ca));
    }
    // turbines: C_T' gradient and the adjoint of the Ucat they sampled
    if (C->prm.farm) farm_adj_finish(C, T.ucat_n, A.ca);
    copy3(C, A.ua, A.uoa);
    TG_CUDA(cudaGetLastError());
    return rc;
}

// One reversed step: a replay of the captured sweep (the tape is first copied
// into the work tape when it is a stored one), or the sweep launched kernel by
// kernel when profiling or step replay is off. A replayed sweep returns 0 and
// reports through the SC_ADJ slots.
constexpr int REV_STORE_GRAPHS = 64;   // stored tapes with their own reverse graph

static int adjoint_reverse_step(tg_ctx *C)
{
    AdjState &A = *C->adj;
    if (!C->graphs || C->prof.on || A.rev_failed) return adjoint_reverse_body(C, false);
    cudaGraphExec_t *ex = &A.rev_exec;
    if (A.cur != &A.work_tape) {
        const long q = A.cur - A.store.data();
        if (q >= 0 && q < (long)A.store.size() && q < REV_STORE_GRAPHS) {
            if ((long)A.rev_store.size() <= q) A.rev_store.resize(q + 1, nullptr);
            ex = &A.rev_store[q];
        } else {
            copy_tape(C, A.work_tape, *A.cur);
            A.cur = &A.work_tape;
        }
    }
    if (!*ex && !capture_graph(C, ex, [&]() { adjoint_reverse_body(C, true); })) {
        A.rev_failed = true;
        return adjoint_reverse_body(C, false);
    }
    TG_CUDA(cudaGraphLaunch(*ex, C->stream));
    return 0;
}

// statistics of replayed steps and sweeps since step_stats_reset: throws on a
// non-finite residual or a transposed solve at its iteration cap
static void adj_replay_check(tg_ctx *C)
{
    TG_CUDA(cudaMemcpyAsync(C->h_scal + SC_G, C->d_scal + SC_G, sizeof(double) * (SC_ADJ + ST_COUNT - SC_G),
                            cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaStreamSynchronize(C->stream));
    const double *h = C->h_scal;
    C->adj->adj_iters += (int64_t)h[SC_ADJ + ST_TOT];
    if (h[SC_G + ST_NAN] != 0.0) throw ApiFail{TG_ERR_NAN, "non-finite residual in a forward step"};
    if (h[SC_ADJ + ST_NAN] != 0.0) throw ApiFail{TG_ERR_NAN, "non-finite residual in a transposed pressure solve"};
    if (h[SC_ADJ + ST_NOCONV] != 0.0) throw ApiFail{TG_ERR_NOT_CONVERGED, "adjoint step failed"};
}

// ---------------------------------------------------------- snapshots
static Snapshot make_snapshot(tg_ctx *C)
{
    Snapshot s{};
    s.ucont = alloc3(C); s.ucat = alloc3(C);
    if (C->prm.buoyancy) { s.btheta = alloc3(C); s.btheta_o = alloc3(C); }   // the AB2 history
    s.p = dallocd(C, (size_t)C->g.size());
    s.px = dallocd(C, (size_t)poisson_n(C));
    s.pxp = dallocd(C, (size_t)poisson_n(C));
    s.pxp2 = dallocd(C, (size_t)poisson_n(C));
    if (wall_on(C)) { s.wum = dallocd(C, wall_plane(C)); s.wfx = dallocd(C, wall_plane(C)); s.wfy = dallocd(C, wall_plane(C)); }
    s.pos = -1;
    return s;
}
__global__ void k_set_phist(double *a, double v) { a[0] = v; }

static void save_state(tg_ctx *C, Snapshot &s, int pos)
{
    copy3(C, s.ucont, C->s.ucont); copy3(C, s.ucat, C->s.ucat);
    if (s.btheta.x) { copy3(C, s.btheta, C->s.btheta); copy3(C, s.btheta_o, C->s.btheta_o); }
    TG_CUDA(cudaMemcpyAsync(s.p, C->s.p, sizeof(double) * (size_t)C->g.size(), cudaMemcpyDeviceToDevice, C->stream));
    TG_CUDA(cudaMemcpyAsync(s.px, poisson_x(C), sizeof(double) * (size_t)poisson_n(C), cudaMemcpyDeviceToDevice, C->stream));
    TG_CUDA(cudaMemcpyAsync(s.pxp, poisson_xprev(C), sizeof(double) * (size_t)poisson_n(C), cudaMemcpyDeviceToDevice, C->stream));
    TG_CUDA(cudaMemcpyAsync(s.pxp2, poisson_xprev2(C), sizeof(double) * (size_t)poisson_n(C), cudaMemcpyDeviceToDevice, C->stream));
    TG_CUDA(cudaMemcpyAsync(&s.phist, C->d_scal + SC_PHIST, sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    if (s.wum) {
        copy_plane(C, s.wum, C->s.umean, wall_plane(C));
        copy_plane(C, s.wfx, C->s.ufx, wall_plane(C));
        copy_plane(C, s.wfy, C->s.ufy, wall_plane(C));
    }
    TG_CUDA(cudaStreamSynchronize(C->stream));
    s.ufilt_set = C->ufilt_set;
    s.it = C->it;
    s.pos = pos;
}
static void restore_state(tg_ctx *C, const Snapshot &s)
{
    copy3(C, C->s.ucont, s.ucont); copy3(C, C->s.ucat, s.ucat);
    if (s.btheta.x) { copy3(C, C->s.btheta, s.btheta); copy3(C, C->s.btheta_o, s.btheta_o); }
    TG_CUDA(cudaMemcpyAsync(C->s.p, s.p, sizeof(double) * (size_t)C->g.size(), cudaMemcpyDeviceToDevice, C->stream));
    TG_CUDA(cudaMemcpyAsync(poisson_x(C), s.px, sizeof(double) * (size_t)poisson_n(C), cudaMemcpyDeviceToDevice, C->stream));
    TG_CUDA(cudaMemcpyAsync(poisson_xprev(C), s.pxp, sizeof(double) * (size_t)poisson_n(C), cudaMemcpyDeviceToDevice, C->stream));
    TG_CUDA(cudaMemcpyAsync(poisson_xprev2(C), s.pxp2, sizeof(double) * (size_t)poisson_n(C), cudaMemcpyDeviceToDevice, C->stream));
    k_set_phist<<<1, 1, 0, C->stream>>>(C->d_scal + SC_PHIST, s.phist);
    if (s.wum) {
        copy_plane(C, C->s.umean, s.wum, wall_plane(C));
        copy_plane(C, C->s.ufx, s.wfx, wall_plane(C));
        copy_plane(C, C->s.ufy, s.wfy, wall_plane(C));
        C->ufilt_set = s.ufilt_set;
    }
    C->it = s.it;
    set_device_step(C);
}

// one adjoint step at the current state: taped forward step, restore, reverse
static int adjoint_step_here(tg_ctx *C, Snapshot &scratch)
{
    C->adj->cur = &C->adj->work_tape;
    save_state(C, scratch, -2);
    C->taping = true;
    tg_stats fs{};
    int frc = step(C, &fs);
    C->taping = false;
    restore_state(C, scratch);
    if (frc == 2) return 2;
    return adjoint_reverse_step(C);
}

// binomial checkpointing: minimal forward recomputation to reverse l steps
// with c free snapshots (Griewank-Walther), p(l, 0) = l(l-1)/2, p(1, c) = 0,
// p(l, c) = min_m m + p(l-m, c-1) + p(m, c); split[l][c] = the best m
struct Revolve {
    int L = 0, Cmax = 0;
    std::vector<int64_t> cost;
    std::vector<int> split;
    void build(int l, int c)
    {
        L = l; Cmax = c;
        cost.assign((size_t)(l + 1) * (c + 1), 0);
        split.assign((size_t)(l + 1) * (c + 1), 1);
        auto at = [&](int a, int b) -> int64_t & { return cost[(size_t)a * (c + 1) + b]; };
        for (int a = 1; a <= l; a++) at(a, 0) = (int64_t)a * (a - 1) / 2;
        for (int b = 1; b <= c; b++) {
            at(1, b) = 0;
            for (int a = 2; a <= l; a++) {
                int64_t best = INT64_MAX; int bm = 1;
                // large problems: bisection instead of the full search
                int lo = 1, hi = a - 1;
                if ((int64_t)l * l * c > 200000000LL) { lo = hi = std::max(1, a / 2); }
                for (int m2 = lo; m2 <= hi; m2++) {
                    int64_t v = m2 + at(a - m2, b - 1) + at(m2, b);
                    if (v < best) { best = v; bm = m2; }
                }
                at(a, b) = best;
                split[(size_t)a * (c + 1) + b] = bm;
            }
        }
    }
    int best_split(int a, int b) const { return split[(size_t)a * (Cmax + 1) + b]; }
};

}  // namespace tg

using namespace tg;

namespace {

template <class F>
tg_status adj_guard(tg_ctx *C, F &&f)
{
    if (!C) return TG_ERR_BAD_ARG;
    try {
        cudaError_t e = cudaSetDevice(C->cfg.device);
        if (e != cudaSuccess) { C->err = std::string("cudaSetDevice: ") + cudaGetErrorString(e); return TG_ERR_CUDA; }
        tg_status s = f();
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) { C->err = std::string("kernel launch: ") + cudaGetErrorString(le); return TG_ERR_CUDA; }
        return s;
    } catch (const CudaError &e) {
        C->err = std::string(e.what) + ": " + cudaGetErrorString(e.e);
        return e.e == cudaErrorMemoryAllocation ? TG_ERR_ALLOC : TG_ERR_CUDA;
    } catch (const ApiFail &e) {
        C->err = e.msg;
        return e.s;
    } catch (const std::bad_alloc &) {
        C->err = "host allocation failed";
        return TG_ERR_ALLOC;
    }
}

tg_status check_adjoint(tg_ctx *C)
{
    if (!C->has_mesh) { C->err = "mesh not set"; return TG_ERR_STATE; }
    std::string why;
    if (!adjoint_supported(C, why)) { C->err = why; return TG_ERR_BAD_ARG; }
    return TG_OK;
}

// recursive reversal of steps [a, a+l) with the state at a in snaps[slot];
// free slots are slots > slot up to the end
void reverse_range(tg_ctx *C, const Revolve &R, int a, int l, int slot, tg_adjoint_stats *st)
{
    AdjState &A = *C->adj;
    Snapshot &base = A.snaps[slot];
    const int c = (int)A.snaps.size() - 2 - slot;     // free slots (the last slot is scratch)
    if (l == 1) {
        restore_state(C, base);
        int rc = adjoint_step_here(C, A.snaps.back());
        if (rc) throw ApiFail{rc == 3 ? TG_ERR_BAD_ARG : TG_ERR_NOT_CONVERGED, "adjoint step failed"};
        st->forward_steps += 1;
        st->steps += 1;
        return;
    }
    if (c <= 0) {
        // no free snapshot: recompute from the base for every step, last first
        for (int q = l - 1; q >= 0; q--) {
            restore_state(C, base);
            for (int r = 0; r < q; r++) { tg_stats fs{}; step(C, &fs); st->forward_steps += 1; }
            int rc = adjoint_step_here(C, A.snaps.back());
            if (rc) throw ApiFail{rc == 3 ? TG_ERR_BAD_ARG : TG_ERR_NOT_CONVERGED, "adjoint step failed"};
            st->forward_steps += 1;
            st->steps += 1;
        }
        return;
    }
    int m = std::min(l - 1, std::max(1, R.best_split(std::min(l, R.L), std::min(c, R.Cmax))));
    Snapshot &nxt = A.snaps[slot + 1];
    if (nxt.pos != a + m) {
        restore_state(C, base);
        for (int r = 0; r < m; r++) { tg_stats fs{}; step(C, &fs); st->forward_steps += 1; }
        save_state(C, nxt, a + m);
    }
    reverse_range(C, R, a + m, l - m, slot + 1, st);
    nxt.pos = -1;
    reverse_range(C, R, a, m, slot, st);
}
}  // namespace

extern "C" {

tg_status tg_adjoint_step(tg_ctx *C)
{
    return adj_guard(C, [&]() -> tg_status {
        tg_status s = check_adjoint(C);
        if (s != TG_OK) return s;
        AdjState &A = adj_state(C);
        adj_work(C);
        if (!A.has_single) { A.single = make_snapshot(C); A.has_single = true; }
        step_stats_reset(C);
        int rc = adjoint_step_here(C, A.single);
        adj_replay_check(C);
        if (rc == 3) { C->err = "adjoint of the non-symmetric pressure operator is not implemented"; return TG_ERR_BAD_ARG; }
        if (rc == 2) { C->err = "non-finite residual in the forward step"; return TG_ERR_NAN; }
        if (rc == 1) { C->err = "transposed pressure solve reached its iteration cap"; return TG_ERR_NOT_CONVERGED; }
        return TG_OK;
    });
}

tg_status tg_adjoint_forward(tg_ctx *C, int32_t nsteps, int32_t nsnap, tg_stats *stats)
{
    return adj_guard(C, [&]() -> tg_status {
        tg_status s = check_adjoint(C);
        if (s != TG_OK) return s;
        if (nsteps < 1 || nsnap < 1) { C->err = "nsteps and nsnap must be positive"; return TG_ERR_BAD_ARG; }
        AdjState &A = adj_state(C);
        adj_work(C);
        // With a snapshot per step and room in device memory, every step's tape
        // is kept during this pass and the reversal re-runs no forward step.
        bool store = nsnap >= nsteps;
        if (store) {
            size_t freeb = 0, totalb = 0;
            TG_CUDA(cudaMemGetInfo(&freeb, &totalb));
            const size_t need = tape_bytes(C) * (size_t)std::max(0, nsteps - (int)A.store.size());
            store = need <= freeb / 10 * 6;
        }
        if (store) while ((int)A.store.size() < nsteps) A.store.push_back(make_tape(C));
        A.stored = store;
        // segment schedule: snapshots every seg steps, the tapes of one segment
        int seg = 0;
        if (!store && A.max_tapes != 0 && nsteps >= 2) {
            size_t freeb = 0, totalb = 0;
            TG_CUDA(cudaMemGetInfo(&freeb, &totalb));
            const int64_t budget = (int64_t)(freeb / 10 * 6);
            int fit = (int)A.store.size() + (int)std::max<int64_t>(0, budget / (int64_t)tape_bytes(C));
            if (A.max_tapes > 0) fit = std::min(fit, A.max_tapes);
            fit = std::min(fit, nsteps);
            if (fit >= 2 && (nsteps + fit - 1) / fit <= nsnap) seg = fit;
        }
        if (seg) while ((int)A.store.size() < seg) A.store.push_back(make_tape(C));
        A.seg = seg;
        // snapshots of the schedule plus one scratch state of the adjoint step
        const int want = store ? 2 : (seg ? (nsteps + seg - 1) / seg + 1 : std::min(nsnap, nsteps) + 1);
        while ((int)A.snaps.size() < want) A.snaps.push_back(make_snapshot(C));
        while ((int)A.snaps.size() > want) A.snaps.pop_back();     // buffers stay owned by the context
        for (auto &sp : A.snaps) sp.pos = -1;
        Revolve R;
        R.build(nsteps, (int)A.snaps.size() - 2);
        // forward pass: keep the snapshots the first descent of the schedule uses
        std::vector<int> keep;
        {
            int a = 0, l = nsteps, slot = 0;
            while (l > 1 && slot + 1 < (int)A.snaps.size() - 1) {
                int c = (int)A.snaps.size() - 2 - slot;
                int m = std::min(l - 1, std::max(1, R.best_split(std::min(l, R.L), std::min(c, R.Cmax))));
                keep.push_back(a + m);
                a += m; l -= m; slot++;
            }
        }
        tg_stats local{};
        tg_stats *st = stats ? stats : &local;
        *st = tg_stats{};
        step_stats_reset(C);
        TG_CUDA(cudaEventRecord(C->ev0, C->stream));
        save_state(C, A.snaps[0], 0);
        size_t next = 0;
        if (store || seg) keep.clear();
        bool any = false, last = false;
        for (int n = 0; n < nsteps; n++) {
            // a kept tape is recorded into the work tape and copied out
            if (store) { A.cur = &A.work_tape; C->taping = true; }
            int rc = step(C, st, &last);
            any |= last;
            C->taping = false;
            if (store) copy_tape(C, A.store[n], A.work_tape);
            st->steps += 1;
            if (rc == 2) { C->err = "non-finite residual in the pressure solve"; return TG_ERR_NAN; }
            if (next < keep.size() && keep[next] == n + 1) { save_state(C, A.snaps[next + 1], n + 1); next++; }
            if (seg && (n + 1) % seg == 0 && n + 1 < nsteps) save_state(C, A.snaps[(n + 1) / seg], n + 1);
        }
        TG_CUDA(cudaEventRecord(C->ev1, C->stream));
        if (step_stats_read(C, st, any, last) == 2) { C->err = "non-finite residual in the pressure solve"; return TG_ERR_NAN; }
        float ms = 0.f;
        TG_CUDA(cudaEventElapsedTime(&ms, C->ev0, C->ev1));
        st->seconds = ms * 1e-3;
        A.nsteps = nsteps;
        A.recorded = true;
        return TG_OK;
    });
}

tg_status tg_adjoint_set_tapes(tg_ctx *C, int32_t max_tapes)
{
    return adj_guard(C, [&]() -> tg_status {
        if (max_tapes < -1) { C->err = "max_tapes must be -1, 0 or positive"; return TG_ERR_BAD_ARG; }
        adj_state(C).max_tapes = max_tapes;
        return TG_OK;
    });
}

tg_status tg_adjoint_reverse(tg_ctx *C, tg_adjoint_stats *stats)
{
    return adj_guard(C, [&]() -> tg_status {
        tg_status s = check_adjoint(C);
        if (s != TG_OK) return s;
        AdjState &A = adj_state(C);
        if (!A.recorded) { C->err = "no recorded forward run (call tg_adjoint_forward first)"; return TG_ERR_STATE; }
        tg_adjoint_stats local{};
        tg_adjoint_stats *st = stats ? stats : &local;
        *st = tg_adjoint_stats{};
        st->snapshots = (int32_t)A.snaps.size() - 1;
        Revolve R;
        R.build(A.nsteps, (int)A.snaps.size() - 2);
        A.adj_iters = 0;
        step_stats_reset(C);
        // a new reversal: its first transposed solve starts from the last
        // solution without extrapolating across the two reversals
        TG_CUDA(cudaMemsetAsync(C->d_scal + SC_LHIST, 0, sizeof(double), C->stream));
        TG_CUDA(cudaEventRecord(C->ev0, C->stream));
        if (A.stored) {
            for (int n = A.nsteps - 1; n >= 0; n--) {
                A.cur = &A.store[n];
                int rc = adjoint_reverse_step(C);
                if (rc) { C->err = "adjoint pressure solve failed"; return rc == 3 ? TG_ERR_BAD_ARG : TG_ERR_NOT_CONVERGED; }
                st->steps += 1;
            }
        } else if (A.seg) {
            // per segment, last first: re-run its steps taped from its snapshot, then reverse them
            const int nseg = (A.nsteps + A.seg - 1) / A.seg;
            for (int b = nseg - 1; b >= 0; b--) {
                const int len = std::min(A.seg, A.nsteps - b * A.seg);
                restore_state(C, A.snaps[b]);
                for (int q = 0; q < len; q++) {
                    // recorded into the work tape (a replayed taped step) and copied out
                    A.cur = &A.work_tape;
                    C->taping = true;
                    tg_stats fs{};
                    const int frc = step(C, &fs);
                    C->taping = false;
                    copy_tape(C, A.store[q], A.work_tape);
                    st->forward_steps += 1;
                    if (frc == 2) { C->err = "non-finite residual in a re-run forward step"; return TG_ERR_NAN; }
                }
                for (int q = len - 1; q >= 0; q--) {
                    A.cur = &A.store[q];
                    int rc = adjoint_reverse_step(C);
                    if (rc) { C->err = "adjoint pressure solve failed"; return rc == 3 ? TG_ERR_BAD_ARG : TG_ERR_NOT_CONVERGED; }
                    st->steps += 1;
                }
            }
        } else {
            reverse_range(C, R, 0, A.nsteps, 0, st);
        }
        restore_state(C, A.snaps[0]);
        TG_CUDA(cudaEventRecord(C->ev1, C->stream));
        adj_replay_check(C);
        float ms = 0.f;
        TG_CUDA(cudaEventElapsedTime(&ms, C->ev0, C->ev1));
        st->seconds = ms * 1e-3;
        st->poisson_iterations = (int32_t)A.adj_iters;
        A.recorded = false;
        return TG_OK;
    });
}

}  // extern "C"
