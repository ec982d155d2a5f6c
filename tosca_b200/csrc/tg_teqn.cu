// Temperature transport (SolveTEqn, teqn.c:259-276) with the explicit RK4
// scheme (TeqnRK4, teqn_solvers.c:759-818): FormT (teqn_solvers.c:6-594)
// evaluates per face the WENO3 convective flux -V^q weno3(T) and the diffusive
// flux (g^{q1} dT/dcsi + g^{q2} dT/deta + g^{q3} dT/dzeta) ajc kappa_eff, the
// cell budget times aj forms the right-hand side. kappa_eff = nu/Pr without
// LES; with Smagorinsky the molecular part is dropped and kappa_eff = nu_t/Pr_t
// with the stability-corrected Pr_t = 1/(1 + 2 l/delta), delta = (1/ajc)^(1/3),
// l = min(delta, 7.6 nu_t/delta sqrt(tRef/|g dT/deta|)) in stable
// stratification (teqn_solvers.c:180-195). Boundary ghosts follow
// UpdateTemperatureBCs (boundary.c:2052-2616) for zeroGradient, fixedValue,
// fixedGradient, periodic and (zero-gradient) thetaWallFunction patches; the
// thetaWallFunction's heat flux (UpdateWallModelsT, boundary.c:3858-4178)
// replaces the diffusive flux of the jLeft wall faces. FP64 in every
// precision mode.
#include <cmath>

#include "tg_internal.cuh"
#include "tg_mo.cuh"

namespace tg {

namespace {

inline dim3 gint(const Grid &g) { return grid3(g.mx - 2, g.my - 2, g.mz - 2); }
inline int nblk(int64_t n) { int64_t b = (n + 255) / 256; return (int)(b < 148 * 16 ? b : 148 * 16); }

// weno3, inline.h:5147-5180, with the weights in one division:
// w0 = alpha0 / (alpha0 + alpha1) with alpha_q = d_q / (eps + beta_q)^2 is
// d0 s1^2 / (d0 s1^2 + d1 s0^2), s_q = eps + beta_q (same value up to
// rounding; a double division or library pow call costs tens of instructions)
__device__ __forceinline__ double weno3(double f0, double f1, double f2, double f3, double wavespeed)
{
    double fL, fC, fR;
    if (wavespeed > 0) { fL = f0; fC = f1; fR = f2; }
    else { fL = f3; fC = f2; fR = f1; }
    const double d0 = 2. / 3., d1 = 1. / 3., eps = 1.e-6;
    const double s0 = eps + (fC - fR) * (fC - fR), s1 = eps + (fL - fC) * (fL - fC);
    const double A = d0 * (s1 * s1), B = d1 * (s0 * s0);
    const double u0 = (fC * 0.5 + fR * 0.5), u1 = (-fL * 0.5 + fC * 1.5);
    return (A * u0 + B * u1) / (A + B);
}

// kappa_eff at a face (teqn_solvers.c:164-214); dtde: the face's eta
// derivative. With Smagorinsky, nu_t / Pr_t with Pr_t = 1 / (1 + 2 l/delta)
// and, in stable stratification, l/delta = min(1, 7.6 nu_t sqrt(tRef/|g
// dT/deta|) / delta^2), delta = (1/ajc)^(1/3): evaluated as nu_t (1 + 2
// l/delta) with 1/delta^2 = cbrt(ajc)^2, the same value up to rounding in
// one cube root, one division and one square root (the literal form takes
// five more divisions; the kernel issues about 1700 instructions per cell)
__device__ __forceinline__ double kappa_eff(const Params &p, double nut, double dtde, double ajc)
{
    if (!p.les) return p.nu / p.prandtl;
    const double gradTdotG = dtde * (-9.81);
    double ratio = 1.0;                                    // l / delta
    if (gradTdotG < 0.) {
        const double cr = cbrt(ajc);                       // 1 / delta
        ratio = fmin(1.0, 7.6 * nut * (cr * cr) * sqrt(p.t_ref / fabs(gradTdotG)));
    }
    return nut * (1.0 + 2.0 * ratio);
}

// 4-cell stencil ends of a face (getFace2Cell4Stencil*, inline.h:2190-2380)
__device__ __forceinline__ void stencil4(int i, int m, int per, int &L, int &R)
{
    if (i == 0 || i == m - 2) {
        if (per && i == m - 2) { R = m + 2; L = i - 1; }
        else if (per && i == 0) { L = -3; R = i + 2; }
        else if (i == 0) { L = i; R = i + 2; }
        else { L = i - 1; R = i + 1; }
    } else { L = i - 1; R = i + 2; }
}

// pass 1: convective and diffusive fluxes at the faces of the interior
// cells. One thread per interior cell (k, j, i) forms the i, j and k faces on
// the cell's + side, and a cell next to a non-periodic 0 boundary also the
// face on its - side (face 0; face 0 of a periodic direction is read from
// face m-2 by the budget and is not formed). T and nut are staged in a
// shared-memory tile of the block's cells with one cell below and two above
// in every direction (the DMDA wrap of periodic directions applied once, at
// staging), so every stencil read is a fixed tile offset; the WENO points of
// the boundary faces, which may lie outside the tile (periodic i = mx + 2 and
// i = -3), are read from global memory.
//
// AX: the mesh is axis-aligned (csi || y, eta || z, zet || x; tg_mesh_info):
// the metric tensor of a face is its normal component squared, g11 = csi.y^2
// at i faces, g21 = eta.z^2 at j faces, g31 = zet.x^2 at k faces, and the
// cross terms, zero up to the round-off of the metric evaluation, are left
// out with the derivatives they multiply; kappa_eff still reads the eta
// derivative of every face (the stability correction of Pr_t).
constexpr int TBX = 32, TBY = 4, TBZ = 2, TBN = TBX * TBY * TBZ;
constexpr int TTX = TBX + 3, TTY = TBY + 3, TTZ = TBZ + 3, TTN = TTX * TTY * TTZ;

template <bool AX>
__global__ void __launch_bounds__(TBN) k_t_face_fluxes(Grid g, Metrics m, State s, Params p, V3f<double> dv, V3f<double> vs)
{
    __shared__ double st[TTN];
    __shared__ double sn[TTN];
    const int mx = g.mx, my = g.my, mz = g.mz;
    const int i0 = 1 + blockIdx.x * TBX, j0 = 1 + blockIdx.y * TBY, k0 = 1 + blockIdx.z * TBZ;
    // staging: tile point (tx, ty, tz) <- DMDA (i0-1+tx, j0-1+ty, k0-1+tz),
    // wrapped; 0 outside a non-periodic extent
    auto stage = [&](int tx, int ty, int tz, int gi) {
        const int gj = g.wj(j0 - 1 + ty), gk = g.wk(k0 - 1 + tz), q = (tz * TTY + ty) * TTX + tx;
        double tv = 0.0, nv = 0.0;
        if (gi >= 0 && gi < mx && gj >= 0 && gj < my && gk >= 0 && gk < mz) {
            const int c = (gk * my + gj) * mx + gi;
            tv = s.tmprt[c];
            if (p.les) nv = s.nut[c];
        }
        st[q] = tv; sn[q] = nv;
    };
    {
        // each warp stages whole tile rows (lane = tx, warp-uniform row), then
        // every thread at most one point of the last three columns
        static_assert(TBX == 32 && TBN % 32 == 0 && 3 * TTY * TTZ <= TBN, "one warp per tile row, one pass for the last columns");
        const int lane = threadIdx.x, wid = threadIdx.z * TBY + threadIdx.y;
        const int gi = g.wi(i0 - 1 + lane);
        for (int r = wid; r < TTY * TTZ; r += TBN / 32) stage(lane, r % TTY, r / TTY, gi);
        const int q = wid * 32 + lane;
        if (q < 3 * TTY * TTZ) {
            const int r = q / 3, tx = TBX + (q - 3 * r);
            stage(tx, r % TTY, r / TTY, g.wi(i0 - 1 + tx));
        }
    }
    __syncthreads();
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y, k = k0 + threadIdx.z;
    if (i > mx - 2 || j > my - 2 || k > mz - 2) return;
    const bool npi = !g.pi, npj = !g.pj, npk = !g.pk;
    const int t0 = ((threadIdx.z + 1) * TTY + threadIdx.y + 1) * TTX + threadIdx.x + 1;
    auto T = [&](int dk, int dj, int di) { return st[t0 + (dk * TTY + dj) * TTX + di]; };
    auto NUT = [&](int dk, int dj, int di) { return sn[t0 + (dk * TTY + dj) * TTX + di]; };
    auto TG = [&](int kk, int jj, int ii) { return s.tmprt[g.id(kk, jj, ii)]; };

    // ---- i face fi = i + e (Compute_dscalar_i, inline.h:3210-3247)
    auto iface = [&](int fi, int e) {
        const int f = g.lin(k, j, fi);
        const bool edge = (fi == 0 || fi == mx - 2);
        const double dtdc = T(0, 0, e + 1) - T(0, 0, e);
        double dtde, dtdz = 0.0;
        if (j == my - 2 && edge && (npj || npi))      dtde = (T(0, 0, e + 1) + T(0, 0, e) - T(0, -1, e + 1) - T(0, -1, e)) * 0.5;
        else if (j == 1 && edge && (npj || npi))      dtde = (T(0, 1, e + 1) + T(0, 1, e) - T(0, 0, e + 1) - T(0, 0, e)) * 0.5;
        else                                          dtde = (T(0, 1, e + 1) + T(0, 1, e) - T(0, -1, e + 1) - T(0, -1, e)) * 0.25;
        if (!AX) {
            if (k == mz - 2 && edge && (npk || npi))  dtdz = (T(0, 0, e + 1) + T(0, 0, e) - T(-1, 0, e + 1) - T(-1, 0, e)) * 0.5;
            else if (k == 1 && edge && (npk || npi))  dtdz = (T(1, 0, e + 1) + T(1, 0, e) - T(0, 0, e + 1) - T(0, 0, e)) * 0.5;
            else                                      dtdz = (T(1, 0, e + 1) + T(1, 0, e) - T(-1, 0, e + 1) - T(-1, 0, e)) * 0.25;
        }
        const double uc = s.ucont.x[f];
        double w;
        if (edge) {
            int iL, iR;
            stencil4(fi, mx, g.pi, iL, iR);
            w = weno3(TG(k, j, iL), T(0, 0, e), T(0, 0, e + 1), TG(k, j, iR), uc);
        } else w = weno3(T(0, 0, e - 1), T(0, 0, e), T(0, 0, e + 1), T(0, 0, e + 2), uc);
        dv.x[f] = -uc * w;
        const double ajc = m.iaj[f];
        const double ke = kappa_eff(p, p.les ? 0.5 * (NUT(0, 0, e) + NUT(0, 0, e + 1)) : 0.0, dtde, ajc);
        if (AX) {
            const double cs = m.icsi.y[f];
            vs.x[f] = 0.0 + ((cs * cs) * dtdc) * ajc * ke;
        } else {
            const R3<double> cs = ld3(m.icsi, f), et = ld3(m.ieta, f), ze = ld3(m.izet, f);
            const double g11 = cs.x * cs.x + cs.y * cs.y + cs.z * cs.z, g21 = et.x * cs.x + et.y * cs.y + et.z * cs.z,
                         g31 = ze.x * cs.x + ze.y * cs.y + ze.z * cs.z;
            vs.x[f] = 0.0 + (g11 * dtdc + g21 * dtde + g31 * dtdz) * ajc * ke;
        }
    };
    // ---- j face fj = j + e (Compute_dscalar_j, inline.h:3252-3289)
    auto jface = [&](int fj, int e) {
        const int f = g.lin(k, fj, i);
        const bool edge = (fj == 0 || fj == my - 2);
        const double dtde = T(0, e + 1, 0) - T(0, e, 0);
        double dtdc = 0.0, dtdz = 0.0;
        if (!AX) {
            if (i == mx - 2 && edge && (npi || npj))  dtdc = (T(0, e + 1, 0) + T(0, e, 0) - T(0, e + 1, -1) - T(0, e, -1)) * 0.5;
            else if (i == 1 && edge && (npi || npj))  dtdc = (T(0, e + 1, 1) + T(0, e, 1) - T(0, e + 1, 0) - T(0, e, 0)) * 0.5;
            else                                      dtdc = (T(0, e + 1, 1) + T(0, e, 1) - T(0, e + 1, -1) - T(0, e, -1)) * 0.25;
            if (k == mz - 2 && edge && (npk || npj))  dtdz = (T(0, e + 1, 0) + T(0, e, 0) - T(-1, e + 1, 0) - T(-1, e, 0)) * 0.5;
            else if (k == 1 && edge && (npk || npj))  dtdz = (T(1, e + 1, 0) + T(1, e, 0) - T(0, e + 1, 0) - T(0, e, 0)) * 0.5;
            else                                      dtdz = (T(1, e + 1, 0) + T(1, e, 0) - T(-1, e + 1, 0) - T(-1, e, 0)) * 0.25;
        }
        const double uc = s.ucont.y[f];
        double w;
        if (edge) {
            int jL, jR;
            stencil4(fj, my, g.pj, jL, jR);
            w = weno3(TG(k, jL, i), T(0, e, 0), T(0, e + 1, 0), TG(k, jR, i), uc);
        } else w = weno3(T(0, e - 1, 0), T(0, e, 0), T(0, e + 1, 0), T(0, e + 2, 0), uc);
        dv.y[f] = -uc * w;
        const double ajc = m.jaj[f];
        double ke = kappa_eff(p, p.les ? 0.5 * (NUT(0, e, 0) + NUT(0, e + 1, 0)) : 0.0, dtde, ajc);
        double v0 = 0.0;
        if (p.t_wall && fj == 0) {
            // thetaWallFunction (teqn_solvers.c:337-352): the modelled flux
            // -qWall . jEta, qWall = (0, 0, q), replaces the diffusive one
            const R3<double> et = ld3(m.jeta, f);
            v0 = -1.0 * (0.0 * et.x + 0.0 * et.y + s.qwall[k * mx + i] * et.z);
            ke = 0.0;
        }
        if (AX) {
            const double et = m.jeta.z[f];
            vs.y[f] = v0 + ((et * et) * dtde) * ajc * ke;
        } else {
            const R3<double> cs = ld3(m.jcsi, f), et = ld3(m.jeta, f), ze = ld3(m.jzet, f);
            const double g11 = cs.x * et.x + cs.y * et.y + cs.z * et.z, g21 = et.x * et.x + et.y * et.y + et.z * et.z,
                         g31 = ze.x * et.x + ze.y * et.y + ze.z * et.z;
            vs.y[f] = v0 + (g11 * dtdc + g21 * dtde + g31 * dtdz) * ajc * ke;
        }
    };
    // ---- k face fk = k + e (Compute_dscalar_k, inline.h:3294-3331)
    auto kface = [&](int fk, int e) {
        const int f = g.lin(fk, j, i);
        const bool edge = (fk == 0 || fk == mz - 2);
        double dtdc = 0.0, dtde;
        if (!AX) {
            if (i == mx - 2 && edge && (npi || npk))  dtdc = (T(e + 1, 0, 0) + T(e, 0, 0) - T(e + 1, 0, -1) - T(e, 0, -1)) * 0.5;
            else if (i == 1 && edge && (npi || npk))  dtdc = (T(e + 1, 0, 1) + T(e, 0, 1) - T(e + 1, 0, 0) - T(e, 0, 0)) * 0.5;
            else                                      dtdc = (T(e + 1, 0, 1) + T(e, 0, 1) - T(e + 1, 0, -1) - T(e, 0, -1)) * 0.25;
        }
        if (j == my - 2 && edge && (npj || npk))      dtde = (T(e + 1, 0, 0) + T(e, 0, 0) - T(e + 1, -1, 0) - T(e, -1, 0)) * 0.5;
        else if (j == 1 && edge && (npj || npk))      dtde = (T(e + 1, 1, 0) + T(e, 1, 0) - T(e + 1, 0, 0) - T(e, 0, 0)) * 0.5;
        else                                          dtde = (T(e + 1, 1, 0) + T(e, 1, 0) - T(e + 1, -1, 0) - T(e, -1, 0)) * 0.25;
        const double dtdz = T(e + 1, 0, 0) - T(e, 0, 0);
        const double uc = s.ucont.z[f];
        double w;
        if (edge) {
            int kL, kR;
            stencil4(fk, mz, g.pk, kL, kR);
            w = weno3(TG(kL, j, i), T(e, 0, 0), T(e + 1, 0, 0), TG(kR, j, i), uc);
        } else w = weno3(T(e - 1, 0, 0), T(e, 0, 0), T(e + 1, 0, 0), T(e + 2, 0, 0), uc);
        dv.z[f] = -uc * w;
        const double ajc = m.kaj[f];
        const double ke = kappa_eff(p, p.les ? 0.5 * (NUT(e, 0, 0) + NUT(e + 1, 0, 0)) : 0.0, dtde, ajc);
        if (AX) {
            const double ze = m.kzet.x[f];
            vs.z[f] = 0.0 + ((ze * ze) * dtdz) * ajc * ke;
        } else {
            const R3<double> cs = ld3(m.kcsi, f), et = ld3(m.keta, f), ze = ld3(m.kzet, f);
            const double g11 = cs.x * ze.x + cs.y * ze.y + cs.z * ze.z, g21 = et.x * ze.x + et.y * ze.y + et.z * ze.z,
                         g31 = ze.x * ze.x + ze.y * ze.y + ze.z * ze.z;
            vs.z[f] = 0.0 + (g11 * dtdc + g21 * dtde + g31 * dtdz) * ajc * ke;
        }
    };
    const int ni = (i == 1 && npi) ? 2 : 1, nj = (j == 1 && npj) ? 2 : 1, nk = (k == 1 && npk) ? 2 : 1;
#pragma unroll 1
    for (int e = 0; e > -ni; e--) iface(i + e, e);
#pragma unroll 1
    for (int e = 0; e > -nj; e--) jface(j + e, e);
#pragma unroll 1
    for (int e = 0; e > -nk; e--) kface(k + e, e);
}

// FormT pass 1 on the context's stream
void t_face_fluxes(tg_ctx *C)
{
    const Grid g = C->g;
    const dim3 gr((g.mx - 2 + TBX - 1) / TBX, (g.my - 2 + TBY - 1) / TBY, (g.mz - 2 + TBZ - 1) / TBZ), bl(TBX, TBY, TBZ);
    State &s = C->s;
    if (C->axis_aligned)
        TG_PROF(C, "teqn_face_fluxes", k_t_face_fluxes<true><<<gr, bl, 0, C->stream>>>(g, C->m, s, C->prm, s.tdiv, s.tvisc));
    else
        TG_PROF(C, "teqn_face_fluxes", k_t_face_fluxes<false><<<gr, bl, 0, C->stream>>>(g, C->m, s, C->prm, s.tdiv, s.tvisc));
}

// pass 2 (teqn_solvers.c:520-566): rhs = (div budget + visc budget) aj at
// interior cells, face 0 of a periodic direction read from face m-2
// (resetFacePeriodicFluxesVector); formMode 1 keeps the convective budget
// only, 2 the diffusive one
__global__ void k_t_rhs(Grid g, Metrics m, V3f<double> dv, V3f<double> vs, double *rhs, int mode)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    const int c = g.lin(k, j, i), pl = g.mx * g.my;
    const int iw = (i == 1 && g.pi) ? c + g.mx - 3 : c - 1;
    const int js = (j == 1 && g.pj) ? c + (g.my - 3) * g.mx : c - g.mx;
    const int kb = (k == 1 && g.pk) ? c + (g.mz - 3) * pl : c - pl;
    const double divBudget = dv.x[c] - dv.x[iw] + dv.y[c] - dv.y[js] + dv.z[c] - dv.z[kb];
    const double viscBudget = vs.x[c] - vs.x[iw] + vs.y[c] - vs.y[js] + vs.z[c] - vs.z[kb];
    rhs[c] = 1.0 * ((mode != 2 ? divBudget : 0.0) + (mode != 1 ? viscBudget : 0.0)) * m.aj[c];
}

// TeqnABBE steps 3-5 (teqn_solvers.c:835-880): bT = 3/2 Conv - 1/2 Conv_o
// (Conv on the first step), b = dt bT (zero off the interior) + T_o, and the
// guess x = b
__global__ void k_t_abbe_b(int64_t n, double *b, double *x, const double *conv, const double *conv_o, const double *to,
                           double dt, int ab2)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        double bt = 0.0;
        if (ab2) { bt = bt + 1.5 * conv[q]; bt = bt + -0.5 * conv_o[q]; }
        else bt = bt + 1.0 * conv[q];
        const double v = bt * dt + 1.0 * to[q];
        b[q] = v;
        x[q] = v;
    }
}

// SNESFuncEvalT tail (teqn_solvers.c:688-711): F = dt FormT(T) (zero off the
// interior) - T + T_o, or with BDF2 - 3/2 T + 2 T_o - 1/2 T_oo
__global__ void k_t_snes_f(int64_t n, double *F, const double *rhs, const double *t, const double *to, const double *too,
                           double dt, int bdf2)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        double r = rhs[q] * dt;
        if (bdf2) { r = r + (-3.0 / 2.0) * t[q]; r = r + 2.0 * to[q]; r = r + (-1.0 / 2.0) * too[q]; }
        else { r = r + -1.0 * t[q]; r = r + 1.0 * to[q]; }
        F[q] = r;
    }
}

// ABBEMatVec tail (teqn_solvers.c:930-943): Av = v - dt D(v), D(v) zero off the interior
__global__ void k_t_abbe_av(int64_t n, double *Av, const double *v, const double *d, double dt)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        Av[q] = v[q] + -1.0 * (d[q] * dt);
}

// TeqnRK4 bookkeeping after stage st: Ttmp (+)= dt b Rhs, next stage T = T_o + a dt Rhs, last T = Ttmp
__global__ void k_t_rk(int64_t n, double *t, const double *to, double *ttmp, const double *rhs, double cb, double ca, int first, int last)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const double tt = (first ? to[q] : ttmp[q]) + cb * rhs[q];
        if (last) t[q] = tt;
        else { ttmp[q] = tt; t[q] = ca * rhs[q] + to[q]; }
    }
}

// UpdateTemperatureBCs (boundary.c:2052-2616) on the face ghosts of one patch
// pair (dir: 0 i, 1 j, 2 k), from the interior next to them
__global__ void k_t_bcs(Grid g, Metrics m, Params p, double *t, int dir, const double *series_st, const double *d_it, double it_start)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x + 1, b = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int na = dir == 0 ? g.my : g.mx, nb = dir == 2 ? g.my : g.mz;
    if (a > na - 2 || b > nb - 2) return;
    const int mdir = dir == 0 ? g.mx : (dir == 1 ? g.my : g.mz);
    auto at = [&](int l) { return dir == 0 ? g.lin(b, a, l) : (dir == 1 ? g.lin(b, l, a) : g.lin(l, b, a)); };
    const V3f<double> &S = dir == 0 ? m.csi : (dir == 1 ? m.eta : m.zet);
    for (int side = 0; side < 2; side++) {
        const int patch = 2 * dir + side;
        const int ci = side == 0 ? 1 : mdir - 2, gh = side == 0 ? 0 : mdir - 1;
        const int c = at(ci), q = at(gh);
        const int type = p.t_bc[patch];
        if (type == TG_TBC_WALL_FUNCTION && patch == TG_JLEFT && p.t_wall == TG_TWALL_SURFACE_SERIES && series_st &&
            d_it[0] != it_start)
            t[q] = 2.0 * series_st[0] - t[c];        // -4 after the first step, boundary.c:2392-2408
        else if (type == TG_TBC_ZERO_GRADIENT || type == TG_TBC_WALL_FUNCTION) t[q] = t[c];
        else if (type == TG_TBC_FIXED_VALUE) t[q] = p.t_bc_value[patch];
        else if (type == TG_TBC_FIXED_GRADIENT) {
            const double area = sqrt(S.x[c] * S.x[c] + S.y[c] * S.y[c] + S.z[c] * S.z[c]);
            const double d = (1.0 / m.aj[c]) / area;
            t[q] = d * p.t_bc_value[patch] + t[c];
        } else {
            t[q] = t[at(side == 0 ? mdir - 2 : 1)];   // periodic: the opposite interior cell
        }
    }
}

// ---- UpdateWallModelsT, jLeft thetaWallFunction (boundary.c:3858-4178) ----
// wall-parallel velocity magnitude and wall distance 0.5 / (aj |eta|) of the
// wall cell (k, 1, i)
__device__ __forceinline__ void twall_cell(Grid g, Metrics m, State s, int k, int i, double &upm, double &dist)
{
    const int c = g.lin(k, 1, i);
    R3<double> n;
    const R3<double> et = ld3(m.eta, c);
    calc_normal(ld3(m.csi, c), et, ld3(m.zet, c), 1, n);
    const R3<double> U = ld3(s.ucat, c);
    const R3<double> Up = U - dot3(U, n) * n;
    upm = sqrt(dot3(Up, Up));
    dist = 0.5 / m.aj[c] / sqrt(dot3(et, et));
}

// -4: the surface temperature at the clock time of the step, t_start + (it -
// it_start) dt + dt (clock.c:366), interpolated in the series as
// findInterpolationWeights does (inline.h:5873-5940: the two nearest points,
// points within a relative 1e-5 of the nearer one's distance skipped,
// extrapolating beyond the ends); one thread, out[0]
__global__ void k_twall_series(const double *tv, const double *vv, int n, const double *d_it, double it_start, double t_start,
                               double dt, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (n < 2 || !tv || !vv) { out[0] = 0.0; return; }     // no series: not launched by the host
    const double pval = t_start + (d_it[0] - it_start) * dt + dt;
    const double eqTol = 1e-5;
    int i1 = 0, i2 = 1;
    for (int q = 0; q < n; q++) {
        const double dq = fabs(tv[q] - pval);
        const double tol1 = fabs(dq - fabs(tv[i2] - pval)) / dq;
        if (dq < fabs(tv[i1] - pval) && tol1 > eqTol) { i2 = i1; i1 = q; }
        const double tol2 = fabs(dq - fabs(tv[i1] - pval)) / dq;
        if (dq < fabs(tv[i2] - pval) && q != i1 && tol2 > eqTol) i2 = q;
    }
    if (tv[i2] < tv[i1]) { const int t = i1; i1 = i2; i2 = t; }
    const double idx = (double)(i2 - i1) / (tv[i2] - tv[i1]) * (pval - tv[i1]) + (double)i1;
    const double w0 = ((double)i2 - idx) / (double)(i2 - i1), w1 = (idx - (double)i1) / (double)(i2 - i1);
    out[0] = w0 * vv[i1] + w1 * vv[i2];
}

// -3, first call: surfaceTheta = the wall value 0.5 (T(j=1) + T(j=0))
__global__ void k_twall_seed(Grid g, State s)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, k = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.mx - 2 || k > g.mz - 2) return;
    s.surf_theta[k * g.mx + i] = 0.5 * (s.tmprt[g.lin(k, 1, i)] + s.tmprt[g.lin(k, 0, i)]);
}

// -3 localized: surfaceTheta += heatingRate dt, then qWallShumann per cell
__global__ void k_twall_local(Grid g, Metrics m, State s, Params p, const double *sts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, k = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.mx - 2 || k > g.mz - 2) return;
    const int w = k * g.mx + i;
    double upm, dist;
    twall_cell(g, m, s, k, i, upm, dist);
    double st;
    if (sts) st = sts[0];
    else { st = s.surf_theta[w] + p.tw_heating * p.dt; s.surf_theta[w] = st; }
    s.qwall[w] = mo::qwall(upm, dist, p.tw_z0, p.tw_gamma_m, p.tw_gamma_h, p.tw_alpha_h, p.tw_theta_ref,
                           s.tmprt[g.lin(k, 1, i)] - st, p.tw_kappa);
}

// -3 averaged, pass 1: surfaceTheta += heatingRate dt and per-block partial
// sums of T(j=1) - surfaceTheta, |U_par| and the wall distance
__global__ void __launch_bounds__(256) k_twall_sums(Grid g, Metrics m, State s, Params p, double *part, const double *sts)
{
    const int nI = g.mx - 2, nK = g.mz - 2;
    double sT = 0.0, sU = 0.0, sD = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nI * nK; t += gridDim.x * blockDim.x) {
        const int i = t % nI + 1, k = t / nI + 1, w = k * g.mx + i;
        double upm, dist;
        twall_cell(g, m, s, k, i, upm, dist);
        double st;
        if (sts) st = sts[0];
        else { st = s.surf_theta[w] + p.tw_heating * p.dt; s.surf_theta[w] = st; }
        sT += (s.tmprt[g.lin(k, 1, i)] - st);
        sU += upm;
        sD += dist;
    }
    double v[3] = {sT, sU, sD};
    block_reduce<256>(v, RedSum{}, RedSum{}, RedSum{});
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++) part[3 * blockIdx.x + q] = v[q];
}

// -3 averaged, pass 2 (one block): the plane means in a fixed order,
// qWallShumann once, the result into every wall cell; -2 (fixed): the
// prescribed flux into every wall cell (nb = 0)
__global__ void k_twall_fill(Grid g, Params p, const double *part, int nb, double *sc, State s)
{
    __shared__ double q;
    if (threadIdx.x == 0) {
        if (nb > 0) {
            double sT = 0.0, sU = 0.0, sD = 0.0;
            for (int b = 0; b < nb; b++) { sT += part[3 * b]; sU += part[3 * b + 1]; sD += part[3 * b + 2]; }
            const double n = (double)(g.mx - 2) * (double)(g.mz - 2);
            sc[0] = sT / n; sc[1] = sU / n; sc[2] = sD / n;
            q = mo::qwall(sU / n, sD / n, p.tw_z0, p.tw_gamma_m, p.tw_gamma_h, p.tw_alpha_h, p.tw_theta_ref, sT / n, p.tw_kappa);
        } else q = p.tw_qwall;
        sc[3] = q;
    }
    __syncthreads();
    const int nI = g.mx - 2, nK = g.mz - 2;
    for (int t = threadIdx.x; t < nI * nK; t += blockDim.x) s.qwall[(t / nI + 1) * g.mx + t % nI + 1] = q;
}

}  // namespace

// SolveTEqn with TeqnABBE (teqn_solvers.c:821-945): AB2 convection,
// backward-Euler diffusion A T = b, A v = v - dt D(v) (ABBEMatVec: D is FormT
// with formMode 2 of v, periodic ghosts reset, zero off the interior; the
// boundary ghosts of v stay those of the Krylov vector, and kappa_eff follows
// v's vertical gradient, so A is not linear in v for LES, as in the reference)
// by GMRES (kspIMEX: PCNONE, restart -kspGMRESRestartT, relTolT / absTolT,
// 1000 iterations, the b as initial guess). Returns the GMRES status.
static int solve_t_abbe(tg_ctx *C)
{
    const Grid g = C->g;
    const int64_t G = g.size();
    State &s = C->s;
    const double dt = C->prm.dt;
    if (!C->tgm) C->tgm = gmres_alloc(C, G, C->cfg.t_gmres_restart > 0 ? C->cfg.t_gmres_restart : 30);
    // Steps 1-2: periodic ghosts, convective right-hand side at T^n
    reset_cell_periodic_s(C, s.tmprt);
    t_face_fluxes(C);
    TG_PROF(C, "teqn_rhs", k_t_rhs<<<gint(g), block3(), 0, C->stream>>>(g, C->m, s.tdiv, s.tvisc, C->tconv, 1));
    // Steps 3-4: b (in Ttmp) and the guess; as in the reference the solution
    // goes into RhsConv_o, whose AB2 history this kernel consumes first
    double *b = s.ttmp, *x = C->tconv_o;
    TG_PROF(C, "teqn_abbe_b", k_t_abbe_b<<<nblk(G), 256, 0, C->stream>>>(G, b, x, C->tconv, C->tconv_o, s.tmprt_o, dt,
                                                                         C->it > C->cfg.it_start ? 1 : 0));
    // Step 5: GMRES on ABBEMatVec
    auto A = [&](const double *v, double *Av) {
        TG_CUDA(cudaMemcpyAsync(s.tmprt, v, sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
        reset_cell_periodic_s(C, s.tmprt);
        t_face_fluxes(C);
        TG_PROF(C, "teqn_rhs", k_t_rhs<<<gint(g), block3(), 0, C->stream>>>(g, C->m, s.tdiv, s.tvisc, s.trhs, 2));
        TG_PROF(C, "teqn_abbe_av", k_t_abbe_av<<<nblk(G), 256, 0, C->stream>>>(G, Av, v, s.trhs, dt));
    };
    int its = 0;
    double res = 0.0;
    const int rc = gmres_solve(C, *C->tgm, A, b, x, C->cfg.t_rtol, C->cfg.t_atol, its, res);
    // Steps 6-7: T = solution, RhsConv_o = RhsConv
    TG_CUDA(cudaMemcpyAsync(s.tmprt, x, sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
    TG_CUDA(cudaMemcpyAsync(C->tconv_o, C->tconv, sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
    C->t_its = its;
    return rc;
}

// SolveTEqn with TeqnSNES (teqn_solvers.c:596-712; bT = 0 without
// hyperviscosity or controller): the root of SNESFuncEvalT from T_o by the
// Newton-Krylov solver of the Crank-Nicolson momentum step (jfnk_solve; the
// reference uses SNESNEWTONTR with MATMFFD products: converged tightly, the
// root does not depend on the path), -absTolT / -relTolT, 20 Newton steps
static int solve_t_snes(tg_ctx *C)
{
    const Grid g = C->g;
    const int64_t G = g.size();
    State &s = C->s;
    const double dt = C->prm.dt;
    const int bdf2 = (C->cfg.t_ddt_scheme == TG_TDDT_BDF2 && C->it > C->cfg.it_start) ? 1 : 0;
    if (!C->tsn) C->tsn = jfnk_alloc(C, G, C->cfg.t_gmres_restart > 0 ? C->cfg.t_gmres_restart : 30);
    double *T = jfnk_u(C->tsn);
    TG_CUDA(cudaMemcpyAsync(T, s.tmprt_o, sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
    auto Feval = [&](const double *t, double *F) {
        TG_CUDA(cudaMemcpyAsync(s.tmprt, t, sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
        reset_cell_periodic_s(C, s.tmprt);
        t_face_fluxes(C);
        TG_PROF(C, "teqn_rhs", k_t_rhs<<<gint(g), block3(), 0, C->stream>>>(g, C->m, s.tdiv, s.tvisc, s.trhs, 0));
        TG_PROF(C, "teqn_snes_f", k_t_snes_f<<<nblk(G), 256, 0, C->stream>>>(G, F, s.trhs, t, s.tmprt_o,
                                                                           bdf2 ? C->tmprt_oo : s.tmprt_o, dt, bdf2));
    };
    int newton = 0, linear = 0;
    double fn = 0.0;
    const int rc = jfnk_solve(C, *C->tsn, Feval, C->cfg.t_atol, C->cfg.t_rtol, 20, newton, linear, fn);
    TG_CUDA(cudaMemcpyAsync(s.tmprt, T, sizeof(double) * G, cudaMemcpyDeviceToDevice, C->stream));
    C->t_its = linear;
    return rc;
}

// SolveTEqn (teqn.c:259-276) with TeqnRK4 (teqn_solvers.c:714-818),
// TeqnABBE or TeqnSNES; returns the implicit solve's status (0 for RK4)
int solve_t(tg_ctx *C)
{
    const Grid g = C->g;
    const int64_t G = g.size();
    State &s = C->s;
    const double dt = C->prm.dt;
    if (C->cfg.t_ddt_scheme == TG_TDDT_BE || C->cfg.t_ddt_scheme == TG_TDDT_BDF2) {
        const int rc = solve_t_snes(C);
        reset_cell_periodic_s(C, s.tmprt);
        return rc;
    }
    if (C->cfg.t_ddt_scheme == TG_TDDT_ABBE) {
        const int rc = solve_t_abbe(C);
        reset_cell_periodic_s(C, s.tmprt);
        return rc;
    }
    const double b[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    const double a[4] = {0.0, 0.5, 0.5, 1.0};
    for (int st = 0; st < 4; st++) {
        // FormExplicitRhsT: periodic ghosts, FormT (Rhs zero off the interior)
        reset_cell_periodic_s(C, s.tmprt);
        t_face_fluxes(C);
        TG_PROF(C, "teqn_rhs", k_t_rhs<<<gint(g), block3(), 0, C->stream>>>(g, C->m, s.tdiv, s.tvisc, s.trhs, 0));
        TG_PROF(C, "teqn_rk_update", k_t_rk<<<nblk(G), 256, 0, C->stream>>>(G, s.tmprt, s.tmprt_o, s.ttmp, s.trhs,
                                                                          dt * b[st], st < 3 ? a[st + 1] * dt : 0.0, st == 0, st == 3));
    }
    reset_cell_periodic_s(C, s.tmprt);
    return 0;
}

// UpdateWallModelsT (boundary.c:3858-4178), jLeft thetaWallFunction: the
// wall heat flux qWall of the wall cells for the temperature step that
// follows and the velocity wall function of the next step. -2: the
// prescribed flux. -3: surfaceTheta is seeded from the wall value on the
// first call and rises by heatingRate * dt on every call; qWallShumann once
// from the plane means ("averaged", two launches) or per cell ("localized")
// -4: the surface temperature of the step into its device slot (nullptr
// when the series is not set yet: the steps refuse to run then, and the ghost
// update at initialisation, on the first step's clock, is zero-gradient)
static const double *series_surface(tg_ctx *C)
{
    if (C->prm.t_wall != TG_TWALL_SURFACE_SERIES || C->series_n < 2 || !C->series_t || !C->series_v) return nullptr;
    double *out = C->d_scal + SC_TWALL + 4;
    k_twall_series<<<1, 32, 0, C->stream>>>(C->series_t, C->series_v, C->series_n, C->d_scal + SC_IT, (double)C->cfg.it_start,
                                            C->cfg.t_start, C->prm.dt, out);
    TG_CUDA(cudaGetLastError());
    return out;
}

const char *theta_wall_missing(const tg_ctx *C)
{
    if (C->prm.t_wall == TG_TWALL_SURFACE_SERIES && C->series_n < 2)
        return "thetaWallFunction -4 needs its surface temperature series (tg_set_surface_temperature)";
    return nullptr;
}

void update_wall_models_t(tg_ctx *C)
{
    if (!C->prm.les || !C->prm.t_wall) return;
    const Grid g = C->g;
    const dim3 b2(32, 8), grid((g.mx - 2 + 31) / 32, (g.mz - 2 + 7) / 8);
    if (C->prm.t_wall == TG_TWALL_FIXED_FLUX) {
        TG_PROF(C, "twall_fill", k_twall_fill<<<1, 256, 0, C->stream>>>(g, C->prm, C->d_red, 0, C->d_scal + SC_TWALL, C->s));
        return;
    }
    const double *sts = series_surface(C);
    if (C->prm.t_wall == TG_TWALL_SURFACE_SERIES && !sts)     // the entry points refuse this case before any launch
        throw CudaError{cudaErrorInvalidValue, "thetaWallFunction -4 without its surface temperature series"};
    if (!sts && !C->surf_set) {
        k_twall_seed<<<grid, b2, 0, C->stream>>>(g, C->s);
        C->surf_set = true;
    }
    if (C->prm.t_wall_localized) {
        TG_PROF(C, "twall_local", k_twall_local<<<grid, b2, 0, C->stream>>>(g, C->m, C->s, C->prm, sts));
        return;
    }
    const int nb = 148;
    TG_PROF(C, "twall_sums", k_twall_sums<<<nb, 256, 0, C->stream>>>(g, C->m, C->s, C->prm, C->d_red, sts));
    TG_PROF(C, "twall_fill", k_twall_fill<<<1, 256, 0, C->stream>>>(g, C->prm, C->d_red, nb, C->d_scal + SC_TWALL, C->s));
}

void update_temperature_bcs(tg_ctx *C)
{
    const Grid g = C->g;
    const dim3 b2(32, 8);
    auto g2 = [](int na, int nb) { return dim3((na - 2 + 31) / 32, (nb - 2 + 7) / 8); };
    const double *sts = series_surface(C);
    const double *dit = C->d_scal + SC_IT, its = (double)C->cfg.it_start;
    TG_PROF(C, "teqn_bcs", k_t_bcs<<<g2(g.my, g.mz), b2, 0, C->stream>>>(g, C->m, C->prm, C->s.tmprt, 0, sts, dit, its));
    TG_PROF(C, "teqn_bcs", k_t_bcs<<<g2(g.mx, g.mz), b2, 0, C->stream>>>(g, C->m, C->prm, C->s.tmprt, 1, sts, dit, its));
    TG_PROF(C, "teqn_bcs", k_t_bcs<<<g2(g.mx, g.my), b2, 0, C->stream>>>(g, C->m, C->prm, C->s.tmprt, 2, sts, dit, its));
}

}  // namespace tg
