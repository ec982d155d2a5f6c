// ============================================================================
//  TEST INFRASTRUCTURE -- NOT PART OF THE PRODUCT.
//
//  CPU (FP64, C++17 + OpenMP) restatement of TOSCA's fractional time step for
//  one single-rank DMDA domain. It is the parity checker for the CUDA library
//  (tosca_b200/csrc) and the timed CPU baseline. Only tests/, the smoke check
//  and the CPU-baseline leg of bench.py load it.
//
//  TOSCA as a whole cannot be built in this environment (mpicxx, PETSc 3.15.5,
//  HYPRE 2.20.0 and HDF5 are absent), so every routine below is a restatement
//  of the cited reference source, written from reading it. Where the reference uses
//  HYPRE (BoomerAMG-preconditioned GMRES, peqn.c:357-429), this file assembles
//  the same 19-point matrix (peqn.c:703-1501) and solves it with its own
//  Krylov method to a tight tolerance: the pinned system has a unique solution,
//  so the solver choice does not change the answer beyond the tolerance.
//
//  PINNED to TOSCA's own code: oracle/refstub compiles the reference's stage
//  functions unmodified from their source files against single-rank
//  stand-ins of PETSc, HYPRE and MPI (oracle/_ref), and tests/test_ref_pin.py
//  compares this restatement with them stage by stage (metrics, the assembled
//  matrix, contravariantToCartesian, GradP, UpdateNut, the wall model, FormU,
//  ExplicitRhsU) and over whole FE / RK4 steps. The temperature equation,
//  buoyancy, Crank-Nicolson / IMEX, the turbines and the adjoint are checked
//  against derived known answers and finite differences only
//  (tests/test_oracle_*.py).
//
//  Single-rank PETSc semantics: a local (ghosted) vector equals the global one,
//  with out-of-range indices of a DM_BOUNDARY_PERIODIC direction wrapping
//  modulo the DMDA extent. Every "local" read below therefore goes through the
//  wrapping accessor; reads that the reference takes from a local copy while it
//  writes the global vector use an explicit snapshot.
// ============================================================================

#include "../include/tosca_gpu.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 { double x, y, z; };
inline V3 mk(double x, double y, double z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(double s, V3 a) { return mk(s * a.x, s * a.y, s * a.z); }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double mag(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

struct OracleError : std::runtime_error { using std::runtime_error::runtime_error; };

// CSR matrix of the assembled pressure operator
struct Csr {
    std::vector<int64_t> rowptr;
    std::vector<int64_t> col;
    std::vector<double>  val;
};

// one uniform actuator disk (tosca_oracle_farm.inc)
struct Turbine {
    tg_turbine d{};
    V3 rtrAxis{}, rotCenter{};
    std::vector<V3> points;
    std::vector<double> dA;
    std::vector<size_t> sphere;                 // controlledCells (interior, k-j-i order)
    std::vector<int> ci, cj, ck;                 // closestCells
    double Ct = 0.0, rtrAvgMagU = 0.0, rtrThrust = 0.0, aeroPwr = 0.0;
};

} // namespace

struct OracleMg;   // pressure-solve multigrid (tosca_oracle_mg.inc)

struct tg_ctx {
    tg_config c{};
    int mx = 0, my = 0, mz = 0;
    bool pi = false, pj = false, pk = false;   // periodic (type 2) in i, j, k
    size_t G = 0;
    std::string err;
    bool has_mesh = false;
    int it = 0;                                 // clock->it

    // metrics (global DMDA extent)
    std::vector<V3> coor, cent, csi, eta, zet, icsi, ieta, izet, jcsi, jeta, jzet, kcsi, keta, kzet;
    double grnd = 0.0;                          // mesh->grndLevel = bounds.zmin (mesh.c:2014-2063)
    std::vector<double> aj, iaj, jaj, kaj;
    std::vector<double> g11, g12, g13, g21, g22, g23, g31, g32, g33;  // SetCoeffMatrix tensors

    // state
    std::vector<V3> ucont, ucont_o, ucat, rhs, dp, btheta, btheta_o, gcont, utmp, fp, div1, div2, div3, visc1, visc2, visc3;
    std::vector<V3> source;                     // ueqn->sourceU (cell-centred Cartesian body force)
    // wind farm: turbines, lsourceFarmCat, sourceFarmCont
    std::vector<Turbine> farm;
    double farm_rho = 1.0, farm_power_sum = 0.0;
    bool farm_objective = false;
    std::vector<V3> farm_cat, farm_cont;
    std::vector<double> ct_grad;
    // adjoints (tosca_oracle_adjoint.inc)
    std::vector<V3> ucont_adj, ucat_adj, source_adj;
    std::vector<double> p_adj;
    std::vector<double> p, phi, nut, tmprt;
    std::vector<double> tmprt_o;                // teqn->Tmprt_o (tosca_oracle_teqn.inc)
    std::vector<V3> rhs_o;                      // ueqn->Rhs_o (tosca_oracle_cn.inc)
    std::vector<V3> conv_o;                     // ueqn->RhsConv_o (ABCN, tosca_oracle_imex.inc)
    std::vector<double> tconv_o;                // teqn->RhsConv_o (ABBE, tosca_oracle_teqn.inc)
    std::vector<double> tmprt_oo;               // teqn->Tmprt_oo (BDF2)
    // last implicit momentum solve: Newton steps or IMEX stages, Krylov
    // operator products, last Krylov residual estimate
    int mom_outer = 0, mom_inner = 0;
    double mom_res = 0.0;

    // jLeft wall model arrays, indexed k*mx + i (tauWall, uMeanMag, uFilt)
    std::vector<double> twx, twy, twz, umean, ufx, ufy, ufz;
    bool ufilt_set = false;
    // adjoints of the wall-model state (ufx, ufy, umean) and, within one
    // reversed step, of the wall stress (tosca_oracle_adjoint.inc)
    std::vector<double> wadj_x, wadj_y, wadj_m, twa_x, twa_y, twa_z;
    // jLeft thetaWallFunction: qWall.z and the -3 model's surfaceTheta
    // (planes k*mx + i), surfaceThetaSet (tosca_oracle_teqn.inc)
    std::vector<double> qwall, surf_theta;
    bool surf_set = false;
    std::vector<double> surf_series_t, surf_series_v;   // -4: surface temperature series

    // pressure system
    Csr A;
    std::vector<int64_t> gid;         // DMDA-indexed global cell ids (-1 at non-periodic ghosts)
    std::vector<double> phi1d;        // solution vector kept as the next initial guess
    int64_t N = 0;
    int64_t pinned_row = -1;
    bool symmetric = true;
    std::shared_ptr<OracleMg> mg;     // preconditioner hierarchy of A (built on first use)

    // ------------------------------------------------------------ indexing --
    inline int wi(int i) const { if (pi) { if (i < 0) i += mx; else if (i >= mx) i -= mx; } return i; }
    inline int wj(int j) const { if (pj) { if (j < 0) j += my; else if (j >= my) j -= my; } return j; }
    inline int wk(int k) const { if (pk) { if (k < 0) k += mz; else if (k >= mz) k -= mz; } return k; }
    // global index with DMDA periodic wrap (local-vector semantics)
    inline size_t I(int k, int j, int i) const {
        i = wi(i); j = wj(j); k = wk(k);
        if ((unsigned)i >= (unsigned)mx || (unsigned)j >= (unsigned)my || (unsigned)k >= (unsigned)mz)
            throw OracleError("index outside the DMDA extent in a non-periodic direction");
        return ((size_t)k * my + j) * mx + i;
    }
    inline size_t W(int k, int i) const { return (size_t)k * mx + i; }
    bool bc(int patch, int type) const { return c.bc[patch] == type; }
};

namespace {

template <class T> void zero(std::vector<T> &v, size_t n) { v.assign(n, T{}); }

// ---------------------------------------------------------------------------
// Mesh metrics: mesh.c:630-1976 (SetMeshMetrics), periodic type 2 only.
// ---------------------------------------------------------------------------
void setMeshMetrics(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const size_t G = C.G;
    auto &coor = C.coor;
    auto X = [&](int k, int j, int i) -> const V3 & { return coor[C.I(k, j, i)]; };

    zero(C.cent, G); zero(C.csi, G); zero(C.eta, G); zero(C.zet, G); zero(C.aj, G);

    // cell centres, mesh.c:713-743
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        V3 s = X(k, j, i) + X(k, j - 1, i) + X(k - 1, j, i) + X(k - 1, j - 1, i)
             + X(k, j, i - 1) + X(k, j - 1, i - 1) + X(k - 1, j, i - 1) + X(k - 1, j - 1, i - 1);
        // reference sums in the order written at mesh.c:720-741
        C.cent[C.I(k, j, i)] = 0.125 * s;
    }

    // face-centred dummy bases, mesh.c:773-945
    std::vector<V3> csit(G, V3{0, 0, 0}), etat(G, V3{0, 0, 0}), zett(G, V3{0, 0, 0});
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 0; i < mx - 1; i++) {
        double dxde = 0.5 * (X(k, j, i).x + X(k - 1, j, i).x - X(k, j - 1, i).x - X(k - 1, j - 1, i).x);
        double dyde = 0.5 * (X(k, j, i).y + X(k - 1, j, i).y - X(k, j - 1, i).y - X(k - 1, j - 1, i).y);
        double dzde = 0.5 * (X(k, j, i).z + X(k - 1, j, i).z - X(k, j - 1, i).z - X(k - 1, j - 1, i).z);
        double dxdz = 0.5 * (X(k, j - 1, i).x + X(k, j, i).x - X(k - 1, j - 1, i).x - X(k - 1, j, i).x);
        double dydz = 0.5 * (X(k, j - 1, i).y + X(k, j, i).y - X(k - 1, j - 1, i).y - X(k - 1, j, i).y);
        double dzdz = 0.5 * (X(k, j - 1, i).z + X(k, j, i).z - X(k - 1, j - 1, i).z - X(k - 1, j, i).z);
        csit[C.I(k, j, i)] = mk(dyde * dzdz - dzde * dydz, -dxde * dzdz + dzde * dxdz, dxde * dydz - dyde * dxdz);
    }
    for (int k = 1; k < mz - 1; k++)
    for (int j = 0; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        double dxdc = 0.5 * (X(k, j, i).x + X(k - 1, j, i).x - X(k, j, i - 1).x - X(k - 1, j, i - 1).x);
        double dydc = 0.5 * (X(k, j, i).y + X(k - 1, j, i).y - X(k, j, i - 1).y - X(k - 1, j, i - 1).y);
        double dzdc = 0.5 * (X(k, j, i).z + X(k - 1, j, i).z - X(k, j, i - 1).z - X(k - 1, j, i - 1).z);
        double dxdz = 0.5 * (X(k, j, i).x + X(k, j, i - 1).x - X(k - 1, j, i).x - X(k - 1, j, i - 1).x);
        double dydz = 0.5 * (X(k, j, i).y + X(k, j, i - 1).y - X(k - 1, j, i).y - X(k - 1, j, i - 1).y);
        double dzdz = 0.5 * (X(k, j, i).z + X(k, j, i - 1).z - X(k - 1, j, i).z - X(k - 1, j, i - 1).z);
        etat[C.I(k, j, i)] = mk(dydz * dzdc - dzdz * dydc, -dxdz * dzdc + dzdz * dxdc, dxdz * dydc - dydz * dxdc);
    }
    for (int k = 0; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        double dxdc = 0.5 * (X(k, j, i).x + X(k, j - 1, i).x - X(k, j, i - 1).x - X(k, j - 1, i - 1).x);
        double dydc = 0.5 * (X(k, j, i).y + X(k, j - 1, i).y - X(k, j, i - 1).y - X(k, j - 1, i - 1).y);
        double dzdc = 0.5 * (X(k, j, i).z + X(k, j - 1, i).z - X(k, j, i - 1).z - X(k, j - 1, i - 1).z);
        double dxde = 0.5 * (X(k, j, i).x + X(k, j, i - 1).x - X(k, j - 1, i).x - X(k, j - 1, i - 1).x);
        double dyde = 0.5 * (X(k, j, i).y + X(k, j, i - 1).y - X(k, j - 1, i).y - X(k, j - 1, i - 1).y);
        double dzde = 0.5 * (X(k, j, i).z + X(k, j, i - 1).z - X(k, j - 1, i).z - X(k, j - 1, i - 1).z);
        zett[C.I(k, j, i)] = mk(dydc * dzde - dzdc * dyde, -dxdc * dzde + dzdc * dxde, dxdc * dyde - dydc * dxde);
    }

    // cell-centred bases, mesh.c:970-1004
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        C.csi[c] = 0.5 * csit[c] + 0.5 * csit[C.I(k, j, i - 1)];
        C.eta[c] = 0.5 * etat[c] + 0.5 * etat[C.I(k, j - 1, i)];
        C.zet[c] = 0.5 * zett[c] + 0.5 * zett[C.I(k - 1, j, i)];
    }

    // Jacobian, mesh.c:1013-1098
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        auto P = [&](int dk, int dj, int di) -> const V3 & { return X(k - dk, j - dj, i - di); };
        double dxdc = 0.25 * (P(0,0,0).x + P(0,1,0).x + P(1,0,0).x + P(1,1,0).x - P(0,0,1).x - P(0,1,1).x - P(1,0,1).x - P(1,1,1).x);
        double dydc = 0.25 * (P(0,0,0).y + P(0,1,0).y + P(1,0,0).y + P(1,1,0).y - P(0,0,1).y - P(0,1,1).y - P(1,0,1).y - P(1,1,1).y);
        double dzdc = 0.25 * (P(0,0,0).z + P(0,1,0).z + P(1,0,0).z + P(1,1,0).z - P(0,0,1).z - P(0,1,1).z - P(1,0,1).z - P(1,1,1).z);
        double dxde = 0.25 * (P(0,0,0).x + P(0,0,1).x + P(1,0,0).x + P(1,0,1).x - P(0,1,0).x - P(0,1,1).x - P(1,1,0).x - P(1,1,1).x);
        double dyde = 0.25 * (P(0,0,0).y + P(0,0,1).y + P(1,0,0).y + P(1,0,1).y - P(0,1,0).y - P(0,1,1).y - P(1,1,0).y - P(1,1,1).y);
        double dzde = 0.25 * (P(0,0,0).z + P(0,0,1).z + P(1,0,0).z + P(1,0,1).z - P(0,1,0).z - P(0,1,1).z - P(1,1,0).z - P(1,1,1).z);
        double dxdz = 0.25 * (P(0,0,0).x + P(0,1,0).x + P(0,0,1).x + P(0,1,1).x - P(1,0,0).x - P(1,1,0).x - P(1,0,1).x - P(1,1,1).x);
        double dydz = 0.25 * (P(0,0,0).y + P(0,1,0).y + P(0,0,1).y + P(0,1,1).y - P(1,0,0).y - P(1,1,0).y - P(1,0,1).y - P(1,1,1).y);
        double dzdz = 0.25 * (P(0,0,0).z + P(0,1,0).z + P(0,0,1).z + P(0,1,1).z - P(1,0,0).z - P(1,1,0).z - P(1,0,1).z - P(1,1,1).z);
        double det = dxdc * (dyde * dzdz - dzde * dydz) - dydc * (dxde * dzdz - dzde * dxdz) + dzdc * (dxde * dydz - dyde * dxdz);
        C.aj[C.I(k, j, i)] = 1. / det;
    }

    // mirror the physical ghost layer, mesh.c:1100-1180 (i, then j, then k)
    auto copyc = [&](size_t d, size_t s) { C.csi[d] = C.csi[s]; C.eta[d] = C.eta[s]; C.zet[d] = C.zet[s]; C.aj[d] = C.aj[s]; };
    for (int k = 0; k < mz; k++) for (int j = 0; j < my; j++) {
        copyc(C.I(k, j, 0), C.I(k, j, 1));
        copyc(C.I(k, j, mx - 1), C.I(k, j, mx - 2));
    }
    for (int k = 0; k < mz; k++) for (int i = 0; i < mx; i++) {
        copyc(C.I(k, 0, i), C.I(k, 1, i));
        copyc(C.I(k, my - 1, i), C.I(k, my - 2, i));
    }
    for (int j = 0; j < my; j++) for (int i = 0; i < mx; i++) {
        copyc(C.I(0, j, i), C.I(1, j, i));
        copyc(C.I(mz - 1, j, i), C.I(mz - 2, j, i));
    }

    // periodic ghost cells from the opposite side, mesh.c:1190-1270 (reads the
    // pre-loop local copy: snapshot)
    {
        std::vector<V3> scsi = C.csi, seta = C.eta, szet = C.zet;
        std::vector<double> saj = C.aj;
        for (int k = 0; k < mz; k++)
        for (int j = 0; j < my; j++)
        for (int i = 0; i < mx; i++) {
            int a = i, b = j, cc = k, flag = 0;
            if (C.pi && i == 0) { a = -2; flag = 1; } else if (C.pi && i == mx - 1) { a = mx + 1; flag = 1; }
            if (C.pj && j == 0) { b = -2; flag = 1; } else if (C.pj && j == my - 1) { b = my + 1; flag = 1; }
            if (C.pk && k == 0) { cc = -2; flag = 1; } else if (C.pk && k == mz - 1) { cc = mz + 1; flag = 1; }
            if (flag) {
                size_t d = C.I(k, j, i), s = C.I(cc, b, a);
                C.csi[d] = scsi[s]; C.eta[d] = seta[s]; C.zet[d] = szet[s]; C.aj[d] = saj[s];
            }
        }
    }

    // i-face metrics, mesh.c:1354-1560
    zero(C.icsi, G); zero(C.ieta, G); zero(C.izet, G); zero(C.iaj, G);
    zero(C.jcsi, G); zero(C.jeta, G); zero(C.jzet, G); zero(C.jaj, G);
    zero(C.kcsi, G); zero(C.keta, G); zero(C.kzet, G); zero(C.kaj, G);
    auto facebasis = [](double dxdc, double dydc, double dzdc, double dxde, double dyde, double dzde,
                        double dxdz, double dydz, double dzdz, V3 &fc, V3 &fe, V3 &fz, double &faj) {
        fc = mk(dyde * dzdz - dzde * dydz, -dxde * dzdz + dzde * dxdz, dxde * dydz - dyde * dxdz);
        fe = mk(dydz * dzdc - dzdz * dydc, -dxdz * dzdc + dzdz * dxdc, dxdz * dydc - dydz * dxdc);
        fz = mk(dydc * dzde - dzdc * dyde, -dxdc * dzde + dzdc * dxde, dxdc * dyde - dydc * dxde);
        faj = dxdc * (dyde * dzdz - dzde * dydz) - dydc * (dxde * dzdz - dzde * dxdz) + dzdc * (dxde * dydz - dyde * dxdz);
        faj = 1. / faj;
    };
    {
        // face centres of i-faces: only their i-differences are used
        auto centx = [&](int k, int j, int i) {
            return 0.25 * (X(k, j, i) + X(k - 1, j, i) + X(k, j - 1, i) + X(k - 1, j - 1, i));
        };
        for (int k = 1; k < mz - 1; k++)
        for (int j = 1; j < my - 1; j++)
        for (int i = 0; i < mx - 1; i++) {
            V3 d;
            if (i == 0) d = centx(k, j, i + 1) - centx(k, j, i);
            else if (i == mx - 2) {
                if (C.pi) d = 0.5 * (centx(k, j, mx + 1) - centx(k, j, mx + 0) + centx(k, j, i) - centx(k, j, i - 1));
                else      d = centx(k, j, i) - centx(k, j, i - 1);
            } else d = 0.5 * (centx(k, j, i + 1) - centx(k, j, i - 1));
            // the reference writes each 0.5*(a-b+c-d) term by term; the sums above keep that order
            double dxde = 0.5 * (X(k, j, i).x + X(k - 1, j, i).x - X(k, j - 1, i).x - X(k - 1, j - 1, i).x);
            double dyde = 0.5 * (X(k, j, i).y + X(k - 1, j, i).y - X(k, j - 1, i).y - X(k - 1, j - 1, i).y);
            double dzde = 0.5 * (X(k, j, i).z + X(k - 1, j, i).z - X(k, j - 1, i).z - X(k - 1, j - 1, i).z);
            double dxdz = 0.5 * (X(k, j - 1, i).x + X(k, j, i).x - X(k - 1, j - 1, i).x - X(k - 1, j, i).x);
            double dydz = 0.5 * (X(k, j - 1, i).y + X(k, j, i).y - X(k - 1, j - 1, i).y - X(k - 1, j, i).y);
            double dzdz = 0.5 * (X(k, j - 1, i).z + X(k, j, i).z - X(k - 1, j - 1, i).z - X(k - 1, j, i).z);
            size_t f = C.I(k, j, i);
            facebasis(d.x, d.y, d.z, dxde, dyde, dzde, dxdz, dydz, dzdz, C.icsi[f], C.ieta[f], C.izet[f], C.iaj[f]);
        }
    }
    {
        auto centy = [&](int k, int j, int i) {
            return 0.25 * (X(k, j, i) + X(k - 1, j, i) + X(k, j, i - 1) + X(k - 1, j, i - 1));
        };
        for (int k = 1; k < mz - 1; k++)
        for (int j = 0; j < my - 1; j++)
        for (int i = 1; i < mx - 1; i++) {
            double dxdc = 0.5 * (X(k, j, i).x + X(k - 1, j, i).x - X(k, j, i - 1).x - X(k - 1, j, i - 1).x);
            double dydc = 0.5 * (X(k, j, i).y + X(k - 1, j, i).y - X(k, j, i - 1).y - X(k - 1, j, i - 1).y);
            double dzdc = 0.5 * (X(k, j, i).z + X(k - 1, j, i).z - X(k, j, i - 1).z - X(k - 1, j, i - 1).z);
            V3 d;
            if (j == 0) d = centy(k, j + 1, i) - centy(k, j, i);
            else if (j == my - 2) {
                if (C.pj) d = 0.5 * (centy(k, my + 1, i) - centy(k, my + 0, i) + centy(k, j, i) - centy(k, j - 1, i));
                else      d = centy(k, j, i) - centy(k, j - 1, i);
            } else d = 0.5 * (centy(k, j + 1, i) - centy(k, j - 1, i));
            double dxdz = 0.5 * (X(k, j, i).x + X(k, j, i - 1).x - X(k - 1, j, i).x - X(k - 1, j, i - 1).x);
            double dydz = 0.5 * (X(k, j, i).y + X(k, j, i - 1).y - X(k - 1, j, i).y - X(k - 1, j, i - 1).y);
            double dzdz = 0.5 * (X(k, j, i).z + X(k, j, i - 1).z - X(k - 1, j, i).z - X(k - 1, j, i - 1).z);
            size_t f = C.I(k, j, i);
            facebasis(dxdc, dydc, dzdc, d.x, d.y, d.z, dxdz, dydz, dzdz, C.jcsi[f], C.jeta[f], C.jzet[f], C.jaj[f]);
        }
    }
    {
        auto centz = [&](int k, int j, int i) {
            return 0.25 * (X(k, j, i) + X(k, j - 1, i) + X(k, j, i - 1) + X(k, j - 1, i - 1));
        };
        for (int k = 0; k < mz - 1; k++)
        for (int j = 1; j < my - 1; j++)
        for (int i = 1; i < mx - 1; i++) {
            double dxdc = 0.5 * (X(k, j, i).x + X(k, j - 1, i).x - X(k, j, i - 1).x - X(k, j - 1, i - 1).x);
            double dydc = 0.5 * (X(k, j, i).y + X(k, j - 1, i).y - X(k, j, i - 1).y - X(k, j - 1, i - 1).y);
            double dzdc = 0.5 * (X(k, j, i).z + X(k, j - 1, i).z - X(k, j, i - 1).z - X(k, j - 1, i - 1).z);
            double dxde = 0.5 * (X(k, j, i).x + X(k, j, i - 1).x - X(k, j - 1, i).x - X(k, j - 1, i - 1).x);
            double dyde = 0.5 * (X(k, j, i).y + X(k, j, i - 1).y - X(k, j - 1, i).y - X(k, j - 1, i - 1).y);
            double dzde = 0.5 * (X(k, j, i).z + X(k, j, i - 1).z - X(k, j - 1, i).z - X(k, j - 1, i - 1).z);
            V3 d;
            if (k == 0) d = centz(k + 1, j, i) - centz(k, j, i);
            else if (k == mz - 2) {
                if (C.pk) d = 0.5 * (centz(mz + 1, j, i) - centz(mz + 0, j, i) + centz(k, j, i) - centz(k - 1, j, i));
                else      d = centz(k, j, i) - centz(k - 1, j, i);
            } else d = 0.5 * (centz(k + 1, j, i) - centz(k - 1, j, i));
            size_t f = C.I(k, j, i);
            facebasis(dxdc, dydc, dzdc, dxde, dyde, dzde, d.x, d.y, d.z, C.kcsi[f], C.keta[f], C.kzet[f], C.kaj[f]);
        }
    }

    // face metric tensor of SetCoeffMatrix with boundary remapping, peqn.c:791-849
    for (auto *g : {&C.g11, &C.g12, &C.g13, &C.g21, &C.g22, &C.g23, &C.g31, &C.g32, &C.g33}) zero(*g, G);
    for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
        int a = i, b = j, cc = k;
        if (i == 0)      a = C.pi ? -2 : 1;
        if (i == mx - 1) a = C.pi ? mx + 1 : mx - 2;
        if (j == 0)      b = C.pj ? -2 : 1;
        if (j == my - 1) b = C.pj ? my + 1 : my - 2;
        if (k == 0)      cc = C.pk ? -2 : 1;
        if (k == mz - 1) cc = C.pk ? mz + 1 : mz - 2;
        size_t s = C.I(cc, b, a), d = C.I(k, j, i);
        C.g11[d] = dot(C.icsi[s], C.icsi[s]) * C.iaj[s];
        C.g12[d] = dot(C.ieta[s], C.icsi[s]) * C.iaj[s];
        C.g13[d] = dot(C.izet[s], C.icsi[s]) * C.iaj[s];
        C.g21[d] = dot(C.jcsi[s], C.jeta[s]) * C.jaj[s];
        C.g22[d] = dot(C.jeta[s], C.jeta[s]) * C.jaj[s];
        C.g23[d] = dot(C.jzet[s], C.jeta[s]) * C.jaj[s];
        C.g31[d] = dot(C.kcsi[s], C.kzet[s]) * C.kaj[s];
        C.g32[d] = dot(C.keta[s], C.kzet[s]) * C.kaj[s];
        C.g33[d] = dot(C.kzet[s], C.kzet[s]) * C.kaj[s];
    }
}

// ---------------------------------------------------------------------------
// Poisson connectivity and matrix: peqn.c:107-248 (SetPoissonConnectivity),
// peqn.c:703-1501 (SetCoeffMatrix) without IBM/overset cells.
// ---------------------------------------------------------------------------
enum { CP, EP, WP, NP, SP, TP, BP, NE, SE, NW, SW, TN, BN, TS, BS, TE, BE, TW, BW, NSTEN };

void setPoissonConnectivity(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    C.gid.assign(C.G, -1);
    int64_t n = 0;
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) C.gid[C.I(k, j, i)] = n++;
    C.N = n;
    // resetCellPeriodicFluxes(lGid, "scalar", "localToLocal"), inline.h:5453-5606
    std::vector<int64_t> s = C.gid;
    for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
        int a = i, b = j, cc = k, flag = 0;
        if (C.pi && i == 0) { a = -2; flag = 1; } else if (C.pi && i == mx - 1) { a = mx + 1; flag = 1; }
        if (C.pj && j == 0) { b = -2; flag = 1; } else if (C.pj && j == my - 1) { b = my + 1; flag = 1; }
        if (C.pk && k == 0) { cc = -2; flag = 1; } else if (C.pk && k == mz - 1) { cc = mz + 1; flag = 1; }
        if (flag) C.gid[C.I(k, j, i)] = s[C.I(cc, b, a)];
    }
}

void setCoeffMatrix(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    auto &g11 = C.g11, &g12 = C.g12, &g13 = C.g13, &g21 = C.g21, &g22 = C.g22, &g23 = C.g23,
         &g31 = C.g31, &g32 = C.g32, &g33 = C.g33;
    C.A.rowptr.assign(C.N + 1, 0);
    C.A.col.clear(); C.A.val.clear();
    C.mg.reset();
    C.A.col.reserve(C.N * 19); C.A.val.reserve(C.N * 19);
    const double r = 1.0;
    int64_t row = 0;
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++, row++) {
        auto G_ = [&](const std::vector<double> &g, int kk, int jj, int ii) { return g[C.I(kk, jj, ii)]; };
        if (i == 1 && j == 1 && k == 1) {
            // all-Neumann null space removed by pinning the first cell, peqn.c:883-887
            C.A.col.push_back(row); C.A.val.push_back(1.0);
            C.A.rowptr[row + 1] = (int64_t)C.A.col.size();
            C.pinned_row = row;
            continue;
        }
        double vol[NSTEN];
        for (int m = 0; m < NSTEN; m++) vol[m] = 0.0;

        // east face (i+1/2), peqn.c:897-965
        if (i != mx - 2 || C.pi) {
            double a = G_(g11, k, j, i), b = G_(g12, k, j, i), c = G_(g13, k, j, i);
            vol[CP] -= a / r; vol[EP] += a / r;
            if (j == my - 2)      { vol[CP] += b * 0.5 / r; vol[EP] += b * 0.5 / r; vol[SP] -= b * 0.5 / r; vol[SE] -= b * 0.5 / r; }
            else if (j == 1)      { vol[NP] += b * 0.5 / r; vol[NE] += b * 0.5 / r; vol[CP] -= b * 0.5 / r; vol[EP] -= b * 0.5 / r; }
            else                  { vol[NP] += b * 0.25 / r; vol[NE] += b * 0.25 / r; vol[SP] -= b * 0.25 / r; vol[SE] -= b * 0.25 / r; }
            if (k == mz - 2)      { vol[CP] += c * 0.5 / r; vol[EP] += c * 0.5 / r; vol[BP] -= c * 0.5 / r; vol[BE] -= c * 0.5 / r; }
            else if (k == 1)      { vol[TP] += c * 0.5 / r; vol[TE] += c * 0.5 / r; vol[CP] -= c * 0.5 / r; vol[EP] -= c * 0.5 / r; }
            else                  { vol[TP] += c * 0.25 / r; vol[TE] += c * 0.25 / r; vol[BP] -= c * 0.25 / r; vol[BE] -= c * 0.25 / r; }
        }
        // west face (i-1/2), peqn.c:977-1040
        if (i != 1 || C.pi) {
            double a = G_(g11, k, j, i - 1), b = G_(g12, k, j, i - 1), c = G_(g13, k, j, i - 1);
            vol[CP] -= a / r; vol[WP] += a / r;
            if (j == my - 2)      { vol[CP] -= b * 0.5 / r; vol[WP] -= b * 0.5 / r; vol[SP] += b * 0.5 / r; vol[SW] += b * 0.5 / r; }
            else if (j == 1)      { vol[NP] -= b * 0.5 / r; vol[NW] -= b * 0.5 / r; vol[CP] += b * 0.5 / r; vol[WP] += b * 0.5 / r; }
            else                  { vol[NP] -= b * 0.25 / r; vol[NW] -= b * 0.25 / r; vol[SP] += b * 0.25 / r; vol[SW] += b * 0.25 / r; }
            if (k == mz - 2)      { vol[CP] -= c * 0.5 / r; vol[WP] -= c * 0.5 / r; vol[BP] += c * 0.5 / r; vol[BW] += c * 0.5 / r; }
            else if (k == 1)      { vol[TP] -= c * 0.5 / r; vol[TW] -= c * 0.5 / r; vol[CP] += c * 0.5 / r; vol[WP] += c * 0.5 / r; }
            else                  { vol[TP] -= c * 0.25 / r; vol[TW] -= c * 0.25 / r; vol[BP] += c * 0.25 / r; vol[BW] += c * 0.25 / r; }
        }
        // north face (j+1/2), peqn.c:1052-1113
        if (j != my - 2 || C.pj) {
            double a = G_(g21, k, j, i), b = G_(g22, k, j, i), c = G_(g23, k, j, i);
            if (i == mx - 2)      { vol[CP] += a * 0.5 / r; vol[NP] += a * 0.5 / r; vol[WP] -= a * 0.5 / r; vol[NW] -= a * 0.5 / r; }
            else if (i == 1)      { vol[EP] += a * 0.5 / r; vol[NE] += a * 0.5 / r; vol[CP] -= a * 0.5 / r; vol[NP] -= a * 0.5 / r; }
            else                  { vol[EP] += a * 0.25 / r; vol[NE] += a * 0.25 / r; vol[WP] -= a * 0.25 / r; vol[NW] -= a * 0.25 / r; }
            vol[CP] -= b / r; vol[NP] += b / r;
            if (k == mz - 2)      { vol[CP] += c * 0.5 / r; vol[NP] += c * 0.5 / r; vol[BP] -= c * 0.5 / r; vol[BN] -= c * 0.5 / r; }
            else if (k == 1)      { vol[TP] += c * 0.5 / r; vol[TN] += c * 0.5 / r; vol[CP] -= c * 0.5 / r; vol[NP] -= c * 0.5 / r; }
            else                  { vol[TP] += c * 0.25 / r; vol[TN] += c * 0.25 / r; vol[BP] -= c * 0.25 / r; vol[BN] -= c * 0.25 / r; }
        }
        // south face (j-1/2), peqn.c:1128-1210
        if (j != 1 || C.pj) {
            double a = G_(g21, k, j - 1, i), b = G_(g22, k, j - 1, i), c = G_(g23, k, j - 1, i);
            if (i == mx - 2)      { vol[CP] -= a * 0.5 / r; vol[SP] -= a * 0.5 / r; vol[WP] += a * 0.5 / r; vol[SW] += a * 0.5 / r; }
            else if (i == 1)      { vol[EP] -= a * 0.5 / r; vol[SE] -= a * 0.5 / r; vol[CP] += a * 0.5 / r; vol[SP] += a * 0.5 / r; }
            else                  { vol[EP] -= a * 0.25 / r; vol[SE] -= a * 0.25 / r; vol[WP] += a * 0.25 / r; vol[SW] += a * 0.25 / r; }
            vol[CP] -= b / r; vol[SP] += b / r;
            if (k == mz - 2)      { vol[CP] -= c * 0.5 / r; vol[SP] -= c * 0.5 / r; vol[BP] += c * 0.5 / r; vol[BS] += c * 0.5 / r; }
            else if (k == 1)      { vol[TP] -= c * 0.5 / r; vol[TS] -= c * 0.5 / r; vol[CP] += c * 0.5 / r; vol[SP] += c * 0.5 / r; }
            else                  { vol[TP] -= c * 0.25 / r; vol[TS] -= c * 0.25 / r; vol[BP] += c * 0.25 / r; vol[BS] += c * 0.25 / r; }
        }
        // top face (k+1/2), peqn.c:1226-1290
        if (k != mz - 2 || C.pk) {
            double a = G_(g31, k, j, i), b = G_(g32, k, j, i), c = G_(g33, k, j, i);
            if (i == mx - 2)      { vol[CP] += a * 0.5 / r; vol[TP] += a * 0.5 / r; vol[WP] -= a * 0.5 / r; vol[TW] -= a * 0.5 / r; }
            else if (i == 1)      { vol[EP] += a * 0.5 / r; vol[TE] += a * 0.5 / r; vol[CP] -= a * 0.5 / r; vol[TP] -= a * 0.5 / r; }
            else                  { vol[EP] += a * 0.25 / r; vol[TE] += a * 0.25 / r; vol[WP] -= a * 0.25 / r; vol[TW] -= a * 0.25 / r; }
            if (j == my - 2)      { vol[CP] += b * 0.5 / r; vol[TP] += b * 0.5 / r; vol[SP] -= b * 0.5 / r; vol[TS] -= b * 0.5 / r; }
            else if (j == 1)      { vol[NP] += b * 0.5 / r; vol[TN] += b * 0.5 / r; vol[CP] -= b * 0.5 / r; vol[TP] -= b * 0.5 / r; }
            else                  { vol[NP] += b * 0.25 / r; vol[TN] += b * 0.25 / r; vol[SP] -= b * 0.25 / r; vol[TS] -= b * 0.25 / r; }
            vol[CP] -= c / r; vol[TP] += c / r;
        }
        // bottom face (k-1/2), peqn.c:1302-1373
        if (k != 1 || C.pk) {
            double a = G_(g31, k - 1, j, i), b = G_(g32, k - 1, j, i), c = G_(g33, k - 1, j, i);
            if (i == mx - 2)      { vol[CP] -= a * 0.5 / r; vol[BP] -= a * 0.5 / r; vol[WP] += a * 0.5 / r; vol[BW] += a * 0.5 / r; }
            else if (i == 1)      { vol[EP] -= a * 0.5 / r; vol[BE] -= a * 0.5 / r; vol[CP] += a * 0.5 / r; vol[BP] += a * 0.5 / r; }
            else                  { vol[EP] -= a * 0.25 / r; vol[BE] -= a * 0.25 / r; vol[WP] += a * 0.25 / r; vol[BW] += a * 0.25 / r; }
            if (j == my - 2)      { vol[CP] -= b * 0.5 / r; vol[BP] -= b * 0.5 / r; vol[SP] += b * 0.5 / r; vol[BS] += b * 0.5 / r; }
            else if (j == 1)      { vol[NP] -= b * 0.5 / r; vol[BN] -= b * 0.5 / r; vol[CP] += b * 0.5 / r; vol[BP] += b * 0.5 / r; }
            else                  { vol[NP] -= b * 0.25 / r; vol[BN] -= b * 0.25 / r; vol[SP] += b * 0.25 / r; vol[BS] += b * 0.25 / r; }
            vol[CP] -= c / r; vol[BP] += c / r;
        }

        // neighbour ids, peqn.c:1390-1408; insertion rule |v| > 1e-10, peqn.c:1410-1418
        const int off[NSTEN][3] = {
            {0,0,0},{0,0,1},{0,0,-1},{0,1,0},{0,-1,0},{1,0,0},{-1,0,0},
            {0,1,1},{0,-1,1},{0,1,-1},{0,-1,-1},
            {1,1,0},{-1,1,0},{1,-1,0},{-1,-1,0},
            {1,0,1},{-1,0,1},{1,0,-1},{-1,0,-1}};
        std::vector<std::pair<int64_t,double>> ent;
        for (int m = 0; m < NSTEN; m++) {
            int kk = k + off[m][0], jj = j + off[m][1], ii = i + off[m][2];
            int64_t id = C.gid[C.I(kk, jj, ii)];
            if ((std::fabs(vol[m]) > 1.e-10 && id >= 0) || m == CP) {
                // HYPRE_IJMatrixSetValues: a repeated column overwrites (grids here have >= 4 cells per axis)
                bool found = false;
                for (auto &e : ent) if (e.first == id) { e.second = vol[m]; found = true; }
                if (!found) ent.push_back({id, vol[m]});
            }
        }
        std::sort(ent.begin(), ent.end());
        for (auto &e : ent) { C.A.col.push_back(e.first); C.A.val.push_back(e.second); }
        C.A.rowptr[row + 1] = (int64_t)C.A.col.size();
    }

    // structural/numerical symmetry of the operator outside the pinned row
    C.symmetric = true;
    double amax = 0.0;
    for (double v : C.A.val) amax = std::max(amax, std::fabs(v));
    for (int64_t r2 = 0; r2 < C.N && C.symmetric; r2++) {
        if (r2 == C.pinned_row) continue;
        for (int64_t q = C.A.rowptr[r2]; q < C.A.rowptr[r2 + 1]; q++) {
            int64_t c2 = C.A.col[q];
            if (c2 == r2 || c2 == C.pinned_row) continue;
            double vt = 0.0; bool has = false;
            for (int64_t q2 = C.A.rowptr[c2]; q2 < C.A.rowptr[c2 + 1]; q2++)
                if (C.A.col[q2] == r2) { vt = C.A.val[q2]; has = true; break; }
            if (!has || std::fabs(vt - C.A.val[q]) > 1e-12 * amax) { C.symmetric = false; break; }
        }
    }
}

void spmv(const tg_ctx &C, const std::vector<double> &x, std::vector<double> &y)
{
    const Csr &A = C.A;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < C.N; r++) {
        double s = 0.0;
        for (int64_t q = A.rowptr[r]; q < A.rowptr[r + 1]; q++) s += A.val[q] * x[A.col[q]];
        y[r] = s;
    }
}

double dotv(const std::vector<double> &a, const std::vector<double> &b)
{
    double s = 0.0;
    int64_t n = (int64_t)a.size();
    #pragma omp parallel for reduction(+:s) schedule(static)
    for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

} // namespace
#include "tosca_oracle_mg.inc"
namespace {

// Pressure solve. The reference calls HYPRE GMRES/BoomerAMG (peqn.c:3856-3929);
// here: CG on the pinned system when the operator is symmetric (the pinned
// unknown is identically zero, so it is eliminated), otherwise BiCGStab, both
// preconditioned by one V-cycle of the aggregation multigrid
// (tosca_oracle_mg.inc), or by the diagonal where no hierarchy can be built.
int solvePoisson(tg_ctx &C, const std::vector<double> &b, std::vector<double> &x, tg_stats *st)
{
    const int64_t n = C.N;
    std::vector<double> dinv(n, 1.0);
    for (int64_t r = 0; r < n; r++)
        for (int64_t q = C.A.rowptr[r]; q < C.A.rowptr[r + 1]; q++)
            if (C.A.col[q] == r) dinv[r] = 1.0 / C.A.val[q];
    if (!C.mg) {
        auto M = std::make_shared<OracleMg>();
        try { mgBuild(C, *M); C.mg = M; }
        catch (const OracleError &) { C.mg.reset(); }
    }
    // z = M^-1 v
    auto precond = [&](const std::vector<double> &v, std::vector<double> &z) {
        if (C.mg) { mgApply(*C.mg, v, z); return; }
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) z[i] = dinv[i] * v[i];
    };
    const double bn = std::sqrt(dotv(b, b));
    std::vector<double> r(n), z(n), pv(n), Ap(n);
    const int maxit = C.c.poisson_maxit > 0 ? C.c.poisson_maxit : 10000;
    const double rtol = C.c.poisson_rtol > 0 ? C.c.poisson_rtol : 1e-14;
    const int64_t pin = C.pinned_row;
    if (pin >= 0) x[pin] = 0.0;   // b[pin] = 0 and row pin is the identity
    spmv(C, x, Ap);
    for (int64_t i = 0; i < n; i++) r[i] = b[i] - Ap[i];
    double rn0 = std::sqrt(dotv(r, r));
    if (st) st->poisson_initial_residual = bn > 0 ? rn0 / bn : rn0;
    if (bn == 0.0) { std::fill(x.begin(), x.end(), 0.0); if (st) { st->poisson_iterations = 0; st->poisson_final_residual = 0; } return 0; }
    int iters = 0;
    double rn = rn0;
    if (C.symmetric) {
        // CG on the reduced SPD system (negated operator is positive definite)
        if (pin >= 0) r[pin] = 0.0;
        precond(r, z);
        if (pin >= 0) z[pin] = 0.0;
        pv = z;
        double rz = dotv(r, z);
        while (rn / bn > rtol && iters < maxit) {
            spmv(C, pv, Ap);
            if (pin >= 0) Ap[pin] = 0.0;
            double alpha = rz / dotv(pv, Ap);
            #pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; i++) { x[i] += alpha * pv[i]; r[i] -= alpha * Ap[i]; }
            precond(r, z);
            if (pin >= 0) z[pin] = 0.0;
            double rz1 = dotv(r, z);
            double beta = rz1 / rz; rz = rz1;
            #pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; i++) pv[i] = z[i] + beta * pv[i];
            rn = std::sqrt(dotv(r, r));
            iters++;
        }
        // true residual
        spmv(C, x, Ap);
        for (int64_t i = 0; i < n; i++) r[i] = b[i] - Ap[i];
        rn = std::sqrt(dotv(r, r));
    } else {
        // Jacobi-preconditioned BiCGStab with restarts on breakdown
        std::vector<double> rhat = r, v(n, 0.0), s(n), t(n), phat(n), shat(n);
        double rho = 1.0, alpha = 1.0, omega = 1.0;
        pv.assign(n, 0.0);
        while (rn / bn > rtol && iters < maxit) {
            double rho1 = dotv(rhat, r);
            if (std::fabs(rho1) < 1e-300) { rhat = r; rho1 = dotv(rhat, r); pv.assign(n, 0.0); v.assign(n, 0.0); rho = alpha = omega = 1.0; }
            double beta = (rho1 / rho) * (alpha / omega);
            rho = rho1;
            for (int64_t i = 0; i < n; i++) pv[i] = r[i] + beta * (pv[i] - omega * v[i]);
            precond(pv, phat);
            spmv(C, phat, v);
            alpha = rho / dotv(rhat, v);
            for (int64_t i = 0; i < n; i++) s[i] = r[i] - alpha * v[i];
            precond(s, shat);
            spmv(C, shat, t);
            double tt = dotv(t, t);
            omega = tt > 0 ? dotv(t, s) / tt : 0.0;
            for (int64_t i = 0; i < n; i++) { x[i] += alpha * phat[i] + omega * shat[i]; r[i] = s[i] - omega * t[i]; }
            rn = std::sqrt(dotv(r, r));
            iters++;
            if ((iters % 50) == 0) {   // refresh the true residual
                spmv(C, x, Ap);
                for (int64_t i = 0; i < n; i++) r[i] = b[i] - Ap[i];
                rn = std::sqrt(dotv(r, r));
            }
        }
        spmv(C, x, Ap);
        for (int64_t i = 0; i < n; i++) r[i] = b[i] - Ap[i];
        rn = std::sqrt(dotv(r, r));
    }
    if (st) { st->poisson_iterations = iters; st->poisson_total_iterations += iters; st->poisson_final_residual = rn / bn; }
    return (rn / bn > rtol * 10 && iters >= maxit) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Ghost/periodic helpers, inline.h:5262-5606
// ---------------------------------------------------------------------------
// resetCellPeriodicFluxes (vector or scalar): periodic ghost cells take the
// first interior value of the opposite side (edges and corners included).
template <class T>
void resetCellPeriodic(tg_ctx &C, std::vector<T> &v)
{
    if (!(C.pi || C.pj || C.pk)) return;
    const int mx = C.mx, my = C.my, mz = C.mz;
    const std::vector<T> s = v;
    for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
        int a = i, b = j, cc = k, flag = 0;
        if (C.pi && i == 0) { a = -2; flag = 1; } else if (C.pi && i == mx - 1) { a = mx + 1; flag = 1; }
        if (C.pj && j == 0) { b = -2; flag = 1; } else if (C.pj && j == my - 1) { b = my + 1; flag = 1; }
        if (C.pk && k == 0) { cc = -2; flag = 1; } else if (C.pk && k == mz - 1) { cc = mz + 1; flag = 1; }
        if (flag) v[C.I(k, j, i)] = s[C.I(cc, b, a)];
    }
}

// resetFacePeriodicFluxesVector: left boundary faces copy the solved right ones
void resetFacePeriodic(tg_ctx &C, std::vector<V3> &v)
{
    if (!(C.pi || C.pj || C.pk)) return;
    const int mx = C.mx, my = C.my, mz = C.mz;
    const std::vector<V3> s = v;
    for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
        int a = i, b = j, cc = k, flag = 0;
        if (C.pi && i == 0) { a = -2; flag = 1; }
        if (C.pj && j == 0) { b = -2; flag = 1; }
        if (C.pk && k == 0) { cc = -2; flag = 1; }
        if (flag) v[C.I(k, j, i)] = s[C.I(cc, b, a)];
    }
}

bool isWall(int t) { return t == TG_BC_NOSLIP || t == TG_BC_SLIP || t == TG_BC_WALL_SHUMANN; }

// resetNoPenetrationFluxes, inline.h:5262-5355
void resetNoPenetration(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    for (int k = 0; k < mz - 1; k++)
    for (int j = 0; j < my - 1; j++)
    for (int i = 0; i < mx - 1; i++) {
        V3 &u = C.ucont[C.I(k, j, i)];
        if (i == 0 && isWall(C.c.bc[TG_ILEFT])) u.x = 0.0;
        if (i == mx - 2 && isWall(C.c.bc[TG_IRIGHT])) u.x = 0.0;
        if (j == 0 && isWall(C.c.bc[TG_JLEFT])) u.y = 0.0;
        if (j == my - 2 && isWall(C.c.bc[TG_JRIGHT])) u.y = 0.0;
        if (k == 0 && isWall(C.c.bc[TG_KLEFT])) u.z = 0.0;
        if (k == mz - 2 && isWall(C.c.bc[TG_KRIGHT])) u.z = 0.0;
    }
}

// ---------------------------------------------------------------------------
// contravariantToCartesian, ueqn.c:528-635 (interior cells only)
// ---------------------------------------------------------------------------
void contravariantToCartesian(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        const V3 &s = C.csi[c], &e = C.eta[c], &z = C.zet[c];
        double m00 = s.x, m01 = s.y, m02 = s.z, m10 = e.x, m11 = e.y, m12 = e.z, m20 = z.x, m21 = z.y, m22 = z.z;
        double q0 = 0.5 * (C.ucont[C.I(k, j, i - 1)].x + C.ucont[c].x);
        double q1 = 0.5 * (C.ucont[C.I(k, j - 1, i)].y + C.ucont[c].y);
        double q2 = 0.5 * (C.ucont[C.I(k - 1, j, i)].z + C.ucont[c].z);
        double det  =  m00 * (m11 * m22 - m12 * m21) - m01 * (m10 * m22 - m12 * m20) + m02 * (m10 * m21 - m11 * m20);
        double det0 =  q0 * (m11 * m22 - m12 * m21) - q1 * (m01 * m22 - m02 * m21) + q2 * (m01 * m12 - m02 * m11);
        double det1 = -q0 * (m10 * m22 - m12 * m20) + q1 * (m00 * m22 - m02 * m20) - q2 * (m00 * m12 - m02 * m10);
        double det2 =  q0 * (m10 * m21 - m11 * m20) - q1 * (m00 * m21 - m01 * m20) + q2 * (m00 * m11 - m01 * m10);
        C.ucat[c] = mk(det0 / det, det1 / det, det2 / det);
    }
}

// calculateNormal, inline.h:1210-1268: unit covariant directions of a cell
void calculateNormal(const V3 &csi, const V3 &eta, const V3 &zet, double ni[3], double nj[3], double nk[3])
{
    const double a11 = csi.x, a12 = csi.y, a13 = csi.z;
    const double a21 = eta.x, a22 = eta.y, a23 = eta.z;
    const double a31 = zet.x, a32 = zet.y, a33 = zet.z;
    double det = a11 * (a33 * a22 - a32 * a23) - a21 * (a33 * a12 - a32 * a13) + a31 * (a23 * a12 - a22 * a13);
    double G00 = (a33 * a22 - a32 * a23) / det, G01 = -(a33 * a12 - a32 * a13) / det, G02 = (a23 * a12 - a22 * a13) / det;
    double G10 = -(a33 * a21 - a31 * a23) / det, G11 = (a33 * a11 - a31 * a13) / det, G12 = -(a23 * a11 - a21 * a13) / det;
    double G20 = (a32 * a21 - a31 * a22) / det, G21 = -(a32 * a11 - a31 * a12) / det, G22 = (a22 * a11 - a21 * a12) / det;
    double nxi = G00, nyi = G10, nzi = G20;
    double nxj = G01, nyj = G11, nzj = G21;
    double nxk = G02, nyk = G12, nzk = G22;
    double si = std::sqrt(nxi * nxi + nyi * nyi + nzi * nzi);
    double sj = std::sqrt(nxj * nxj + nyj * nyj + nzj * nzj);
    double sk = std::sqrt(nxk * nxk + nyk * nyk + nzk * nzk);
    nxi /= si; nyi /= si; nzi /= si;
    nxj /= sj; nyj /= sj; nzj /= sj;
    nxk /= sk; nyk /= sk; nzk /= sk;
    ni[0] = nxi; ni[1] = nyi; ni[2] = nzi;
    nj[0] = nxj; nj[1] = nyj; nj[2] = nzj;
    nk[0] = nxk; nk[1] = nyk; nk[2] = nzk;
}

// ---------------------------------------------------------------------------
// UpdateCartesianBCs, boundary.c:824-2050 (periodic, slip, noSlip, wall
// function -3). Face-adjacent ghost cells only; reads the pre-call local copy.
// ---------------------------------------------------------------------------
void updateCartesianBCs(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const std::vector<V3> lu = C.ucat;
    auto L = [&](int k, int j, int i) -> const V3 & { return lu[C.I(k, j, i)]; };
    const int *bc = C.c.bc;
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        // wall function -3 on jLeft: slip preserving the normal gradient, boundary.c:1155-1226
        if (bc[TG_JLEFT] == TG_BC_WALL_SHUMANN && j == 1) {
            double area = mag(C.eta[c]);
            double sb = 0.5 / C.aj[c] / area;
            V3 Ub = L(k, j, i);
            V3 Uc = L(k, j + 1, i);
            double sc = 1.0 / C.aj[c] / area + 0.5 / C.aj[C.I(k, j + 1, i)] / area;
            (void)sc; (void)sb;
            double ni[3], nj[3], nk[3];
            calculateNormal(C.csi[c], C.eta[c], C.zet[c], ni, nj, nk);
            V3 n = mk(nj[0], nj[1], nj[2]);
            V3 UbN = dot(Ub, n) * n, UcN = dot(Uc, n) * n;
            V3 UbP = Ub - UbN, UcP = Uc - UcN;
            V3 Ug = mk(2. * UbP.x - UcP.x, 2. * UbP.y - UcP.y, 2. * UbP.z - UcP.z);
            Ug = Ug - UbN;
            C.ucat[C.I(k, j - 1, i)] = Ug;
        }
        // slip patches, boundary.c:1677-1853
        auto slip = [&](int patch, int dir, int gk, int gj, int gi) {
            if (bc[patch] != TG_BC_SLIP) return;
            double ni[3], nj[3], nk[3];
            calculateNormal(C.csi[c], C.eta[c], C.zet[c], ni, nj, nk);
            const double *nn = dir == 0 ? ni : (dir == 1 ? nj : nk);
            V3 n = mk(nn[0], nn[1], nn[2]);
            V3 U = L(k, j, i);
            V3 Un2 = (2.0 * dot(U, n)) * n;
            C.ucat[C.I(gk, gj, gi)] = U - Un2;
        };
        if (i == 1)      slip(TG_ILEFT, 0, k, j, i - 1);
        if (i == mx - 2) slip(TG_IRIGHT, 0, k, j, i + 1);
        if (j == 1)      slip(TG_JLEFT, 1, k, j - 1, i);
        if (j == my - 2) slip(TG_JRIGHT, 1, k, j + 1, i);
        if (k == 1)      slip(TG_KLEFT, 2, k - 1, j, i);
        if (k == mz - 2) slip(TG_KRIGHT, 2, k + 1, j, i);
        // no-slip, boundary.c:1855-1895
        if (i == 1 && bc[TG_ILEFT] == TG_BC_NOSLIP)       C.ucat[C.I(k, j, i - 1)] = -1.0 * L(k, j, i);
        if (i == mx - 2 && bc[TG_IRIGHT] == TG_BC_NOSLIP) C.ucat[C.I(k, j, i + 1)] = -1.0 * L(k, j, i);
        if (j == 1 && bc[TG_JLEFT] == TG_BC_NOSLIP)       C.ucat[C.I(k, j - 1, i)] = -1.0 * L(k, j, i);
        if (j == my - 2 && bc[TG_JRIGHT] == TG_BC_NOSLIP) C.ucat[C.I(k, j + 1, i)] = -1.0 * L(k, j, i);
        if (k == 1 && bc[TG_KLEFT] == TG_BC_NOSLIP)       C.ucat[C.I(k - 1, j, i)] = -1.0 * L(k, j, i);
        if (k == mz - 2 && bc[TG_KRIGHT] == TG_BC_NOSLIP) C.ucat[C.I(k + 1, j, i)] = -1.0 * L(k, j, i);
        // fixedValue, boundary.c:1632-1673: the ghost takes the patch value
        auto fixedv = [&](int patch, int gk, int gj, int gi) {
            if (bc[patch] == TG_BC_FIXED_VALUE)
                C.ucat[C.I(gk, gj, gi)] = mk(C.c.bc_value[3 * patch], C.c.bc_value[3 * patch + 1], C.c.bc_value[3 * patch + 2]);
        };
        if (i == 1)      fixedv(TG_ILEFT, k, j, i - 1);
        if (i == mx - 2) fixedv(TG_IRIGHT, k, j, i + 1);
        if (j == 1)      fixedv(TG_JLEFT, k, j - 1, i);
        if (j == my - 2) fixedv(TG_JRIGHT, k, j + 1, i);
        if (k == 1)      fixedv(TG_KLEFT, k - 1, j, i);
        if (k == mz - 2) fixedv(TG_KRIGHT, k + 1, j, i);
        // inletFunction type 2 on kLeft, boundary.c:1253-1283: the log law in
        // the height of the first cell's centre above the ground, clipped
        // below at 1e-5 and constant above hInv
        if (k == 1 && bc[TG_KLEFT] == TG_BC_INLET_LOG) {
            const double h = C.cent[c].z - C.grnd, kap = 0.4;
            const double um = h <= C.c.inlet_h_inv ? std::max((C.c.inlet_u_tau / kap) * std::log(h / C.c.inlet_z0), 1e-5)
                                                   : (C.c.inlet_u_tau / kap) * std::log(C.c.inlet_h_inv / C.c.inlet_z0);
            C.ucat[C.I(k - 1, j, i)] = mk(um * C.c.inlet_dir[0], um * C.c.inlet_dir[1], um * C.c.inlet_dir[2]);
        }
        // zeroGradient (outflow), boundary.c:1897-1970: linear extrapolation
        if (i == 1 && bc[TG_ILEFT] == TG_BC_ZERO_GRADIENT)       C.ucat[C.I(k, j, i - 1)] = 2.0 * L(k, j, i) - L(k, j, i + 1);
        if (i == mx - 2 && bc[TG_IRIGHT] == TG_BC_ZERO_GRADIENT) C.ucat[C.I(k, j, i + 1)] = 2.0 * L(k, j, i) - L(k, j, i - 1);
        if (j == 1 && bc[TG_JLEFT] == TG_BC_ZERO_GRADIENT)       C.ucat[C.I(k, j - 1, i)] = 2.0 * L(k, j, i) - L(k, j + 1, i);
        if (j == my - 2 && bc[TG_JRIGHT] == TG_BC_ZERO_GRADIENT) C.ucat[C.I(k, j + 1, i)] = 2.0 * L(k, j, i) - L(k, j - 1, i);
        if (k == 1 && bc[TG_KLEFT] == TG_BC_ZERO_GRADIENT)       C.ucat[C.I(k - 1, j, i)] = 2.0 * L(k, j, i) - L(k + 1, j, i);
        if (k == mz - 2 && bc[TG_KRIGHT] == TG_BC_ZERO_GRADIENT) C.ucat[C.I(k + 1, j, i)] = 2.0 * L(k, j, i) - L(k - 1, j, i);
        // periodic, boundary.c:1990-2018
        if (bc[TG_ILEFT] == TG_BC_PERIODIC && i == 1)       C.ucat[C.I(k, j, i - 1)] = L(k, j, -2);
        if (bc[TG_IRIGHT] == TG_BC_PERIODIC && i == mx - 2) C.ucat[C.I(k, j, i + 1)] = L(k, j, mx + 1);
        if (bc[TG_JLEFT] == TG_BC_PERIODIC && j == 1)       C.ucat[C.I(k, j - 1, i)] = L(k, -2, i);
        if (bc[TG_JRIGHT] == TG_BC_PERIODIC && j == my - 2) C.ucat[C.I(k, j + 1, i)] = L(k, my + 1, i);
        if (bc[TG_KLEFT] == TG_BC_PERIODIC && k == 1)       C.ucat[C.I(k - 1, j, i)] = L(-2, j, i);
        if (bc[TG_KRIGHT] == TG_BC_PERIODIC && k == mz - 2) C.ucat[C.I(k + 1, j, i)] = L(mz + 1, j, i);
    }
}

// UpdateContravariantBCs, boundary.c:614-822
void updateContravariantBCs(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const std::vector<V3> lc = C.ucont;
    const int *bc = C.c.bc;
    // patch type 0 = not a wall (periodic included), checkBCsAndSetPatchTypes boundary.c:321-350
    auto type0 = [&](int patch) { return !isWall(bc[patch]); };
    for (int k = 0; k < mz - 1; k++)
    for (int j = 0; j < my - 1; j++)
    for (int i = 0; i < mx - 1; i++) {
        size_t f = C.I(k, j, i);
        V3 &u = C.ucont[f];
        const V3 &uc = C.ucat[f];
        if ((type0(TG_KLEFT) && k == 0) || (type0(TG_KRIGHT) && k == mz - 2)) {
            const V3 &un = C.ucat[C.I(k + 1, j, i)]; const V3 &s = C.kzet[f];
            u.z = 0.5 * (un.x + uc.x) * s.x + 0.5 * (un.y + uc.y) * s.y + 0.5 * (un.z + uc.z) * s.z;
        }
        if ((type0(TG_JLEFT) && j == 0) || (type0(TG_JRIGHT) && j == my - 2)) {
            const V3 &un = C.ucat[C.I(k, j + 1, i)]; const V3 &s = C.jeta[f];
            u.y = 0.5 * (un.x + uc.x) * s.x + 0.5 * (un.y + uc.y) * s.y + 0.5 * (un.z + uc.z) * s.z;
        }
        if ((type0(TG_ILEFT) && i == 0) || (type0(TG_IRIGHT) && i == mx - 2)) {
            const V3 &un = C.ucat[C.I(k, j, i + 1)]; const V3 &s = C.icsi[f];
            u.x = 0.5 * (un.x + uc.x) * s.x + 0.5 * (un.y + uc.y) * s.y + 0.5 * (un.z + uc.z) * s.z;
        }
        if ((!type0(TG_ILEFT) && i == 0) || (!type0(TG_IRIGHT) && i == mx - 2)) u.x = 0.0;
        if ((!type0(TG_JLEFT) && j == 0) || (!type0(TG_JRIGHT) && j == my - 2)) u.y = 0.0;
        if ((!type0(TG_KLEFT) && k == 0) || (!type0(TG_KRIGHT) && k == mz - 2)) u.z = 0.0;
        // zeroGradient: no flow back in through the face, boundary.c:718-741
        const auto zg = [&](int patch) { return bc[patch] == TG_BC_ZERO_GRADIENT; };
        if (zg(TG_ILEFT) && i == 0 && u.x > 0.0) u.x = 0.0;
        if (zg(TG_IRIGHT) && i == mx - 2 && u.x < 0.0) u.x = 0.0;
        if (zg(TG_JLEFT) && j == 0 && u.y > 0.0) u.y = 0.0;
        if (zg(TG_JRIGHT) && j == my - 2 && u.y < 0.0) u.y = 0.0;
        if (zg(TG_KLEFT) && k == 0 && u.z > 0.0) u.z = 0.0;
        if (zg(TG_KRIGHT) && k == mz - 2 && u.z < 0.0) u.z = 0.0;
        if (bc[TG_ILEFT] == TG_BC_PERIODIC && i == 0) u.x = lc[C.I(k, j, -2)].x;
        if (bc[TG_JLEFT] == TG_BC_PERIODIC && j == 0) u.y = lc[C.I(k, -2, i)].y;
        if (bc[TG_KLEFT] == TG_BC_PERIODIC && k == 0) u.z = lc[C.I(-2, j, i)].z;
    }
}

// UpdatePhiBCs (boundary.c:3168-3255) / UpdatePressureBCs (boundary.c:3051-3166):
// zero-gradient or periodic ghost fill from the pre-call local copy
void updateScalarGhosts(tg_ctx &C, std::vector<double> &v)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const std::vector<double> s = v;
    for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
        int a = i, b = j, cc = k, flag = 0;
        if (i == 0)      { a = C.pi ? -2 : 1; flag = 1; }
        if (i == mx - 1) { a = C.pi ? mx + 1 : mx - 2; flag = 1; }
        if (j == 0)      { b = C.pj ? -2 : 1; flag = 1; }
        if (j == my - 1) { b = C.pj ? my + 1 : my - 2; flag = 1; }
        if (k == 0)      { cc = C.pk ? -2 : 1; flag = 1; }
        if (k == mz - 1) { cc = C.pk ? mz + 1 : mz - 2; flag = 1; }
        if (flag) v[C.I(k, j, i)] = s[C.I(cc, b, a)];
    }
}

// ---------------------------------------------------------------------------
// LES: UpdateCs (smagorinsky, les.c:172-178) + UpdateNut (les.c:2119-2578,
// formula les.c:2510-2514) + UpdateNutBCs (boundary.c:2630-2930)
// ---------------------------------------------------------------------------
void updateNut(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    std::fill(C.nut.begin(), C.nut.end(), 0.0);
    auto U = [&](int k, int j, int i) -> const V3 & { return C.ucat[C.I(k, j, i)]; };
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        double ajc = C.aj[c];
        const V3 &s = C.csi[c], &e = C.eta[c], &z = C.zet[c];
        // Compute_du_center, inline.h:3344-3418
        V3 dc, de, dz;
        if (!C.pi && i == mx - 2)  dc = U(k, j, i) - U(k, j, i - 1);
        else if (!C.pi && i == 1)  dc = U(k, j, i + 1) - U(k, j, i);
        else                       dc = 0.5 * (U(k, j, i + 1) - U(k, j, i - 1));
        if (!C.pj && j == my - 2)  de = U(k, j, i) - U(k, j - 1, i);
        else if (!C.pj && j == 1)  de = U(k, j + 1, i) - U(k, j, i);
        else                       de = 0.5 * (U(k, j + 1, i) - U(k, j - 1, i));
        if (!C.pk && k == mz - 2)  dz = U(k, j, i) - U(k - 1, j, i);
        else if (!C.pk && k == 1)  dz = U(k + 1, j, i) - U(k, j, i);
        else                       dz = 0.5 * (U(k + 1, j, i) - U(k - 1, j, i));
        // Compute_du_dxyz, inline.h:3635-3663
        double du_dx = (dc.x * s.x + de.x * e.x + dz.x * z.x) * ajc;
        double du_dy = (dc.x * s.y + de.x * e.y + dz.x * z.y) * ajc;
        double du_dz = (dc.x * s.z + de.x * e.z + dz.x * z.z) * ajc;
        double dv_dx = (dc.y * s.x + de.y * e.x + dz.y * z.x) * ajc;
        double dv_dy = (dc.y * s.y + de.y * e.y + dz.y * z.y) * ajc;
        double dv_dz = (dc.y * s.z + de.y * e.z + dz.y * z.z) * ajc;
        double dw_dx = (dc.z * s.x + de.z * e.x + dz.z * z.x) * ajc;
        double dw_dy = (dc.z * s.y + de.z * e.y + dz.z * z.y) * ajc;
        double dw_dz = (dc.z * s.z + de.z * e.z + dz.z * z.z) * ajc;
        double S00 = 0.5 * (du_dx + du_dx), S01 = 0.5 * (du_dy + dv_dx), S02 = 0.5 * (du_dz + dw_dx);
        double S10 = 0.5 * (dv_dx + du_dy), S11 = 0.5 * (dv_dy + dv_dy), S12 = 0.5 * (dv_dz + dw_dy);
        double S20 = 0.5 * (dw_dx + du_dz), S21 = 0.5 * (dw_dy + dv_dz), S22 = 0.5 * (dw_dz + dw_dz);
        double Sabs = std::sqrt(2.0 * (S00 * S00 + S01 * S01 + S02 * S02 + S10 * S10 + S11 * S11 + S12 * S12 + S20 * S20 + S21 * S21 + S22 * S22));
        double filter = std::pow(1. / ajc, 1. / 3.);
        C.nut[c] = C.c.cs * std::pow(filter, 2.0) * Sabs;
    }
    // UpdateNutBCs: face-adjacent ghosts
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        auto apply = [&](int patch, int gk, int gj, int gi, int sk, int sj, int si) {
            int t = C.c.nut_bc[patch];
            if (t == TG_NUTBC_ZEROGRADIENT) C.nut[C.I(gk, gj, gi)] = C.nut[C.I(k, j, i)];
            else if (t == TG_NUTBC_FIXEDVALUE) C.nut[C.I(gk, gj, gi)] = C.c.nut_bc_value[patch];
            else C.nut[C.I(gk, gj, gi)] = C.nut[C.I(sk, sj, si)];
        };
        if (i == 1)      apply(TG_ILEFT,  k, j, i - 1, k, j, -2);
        if (i == mx - 2) apply(TG_IRIGHT, k, j, i + 1, k, j, mx + 1);
        if (j == 1)      apply(TG_JLEFT,  k, j - 1, i, k, -2, i);
        if (j == my - 2) apply(TG_JRIGHT, k, j + 1, i, k, my + 1, i);
        if (k == 1)      apply(TG_KLEFT,  k - 1, j, i, -2, j, i);
        if (k == mz - 2) apply(TG_KRIGHT, k + 1, j, i, mz + 1, j, i);
    }
}

// ---------------------------------------------------------------------------
// Monin-Obukhov surface-layer relations of the Schumann-Grotzbach wall
// functions (wallfunctions.c:12-290). Both iterate the friction velocity (and
// the heat flux) with under-relaxation 0.5 to a change below 1e-5 or 500
// sweeps (then the neutral values), clamp |L| >= 1e-10, cap the unstable
// zeta at -1/15 + 1e-8 and use the Businger-Dyer psi functions; a stable
// result with u* < 1e-2 (no root) is replaced by the u* of the bisection on
// the slope of U_model(u*) (at most 50 halvings of [1e-6, u*_neutral]).
// The steps are those of the reference so that the stopping sweep, and with
// it the result, is the same.
// ---------------------------------------------------------------------------
constexpr double kMoG = 9.81, kMoTol = 1e-5, kMoOmega = 0.5;
constexpr int kMoIterMax = 500;

// Businger-Dyer stability functions at zeta = z/L (psiM, psiH, phiM, phiH)
void moStability(double zeta, bool stable, double gammaM, double gammaH, double alphaH,
                 double &psiM, double &psiH, double &phiM, double &phiH)
{
    if (stable) {
        psiM = -gammaM * zeta; psiH = -gammaH * zeta;
        phiM = 1.0 + gammaM * zeta; phiH = alphaH + gammaH * zeta;
    } else {
        if (zeta < -1.0 / 15.0) zeta = -1.0 / 15.0 + 1e-8;
        const double xi = std::pow(1.0 - 15.0 * zeta, 0.25);
        psiM = 2.0 * std::log((1.0 + xi) / 2.0) + std::log((1.0 + xi * xi) / 2.0) - 2.0 * std::atan(xi) + M_PI / 2.0;
        psiH = 2.0 * std::log((1.0 + xi * xi) / 2.0);
        phiM = std::pow(1.0 - 15.0 * zeta, -0.25);
        phiH = alphaH * std::pow(1.0 - 15.0 * zeta, -0.5);
    }
}

double moClampL(double L) { return (L > 0) ? std::max(1e-10, L) : std::min(-1e-10, L); }

// the slope proxy (U_model(u) - U) / u of the stable bisection, L from a fixed heat flux q
double moStableSlope(double u, double U, double wallDist, double z0, double gammaM, double kappa, double q, double thetaRef)
{
    const double Lq = std::max(1e-10, -std::pow(u, 3.0) / (kappa * (kMoG / thetaRef) * q));
    const double psiM = -gammaM * (wallDist / Lq);
    return ((u / kappa) * (std::log(wallDist / z0) - psiM) - U) / u;
}

// bisection for the extremum of U_model (wallfunctions.c:88-128, 240-286)
double moStableBisection(double U, double wallDist, double z0, double gammaM, double kappa, double q, double thetaRef,
                         double uNeutral)
{
    double uLow = 1e-6, uHigh = uNeutral, uMid = 0.0;
    for (int it = 0; it < 50; it++) {
        uMid = 0.5 * (uLow + uHigh);
        const double dfMid = moStableSlope(uMid, U, wallDist, z0, gammaM, kappa, q, thetaRef);
        if (std::fabs(uHigh - uLow) < 1e-6 || std::fabs(dfMid) < kMoTol) break;
        const double dfLow = moStableSlope(uLow, U, wallDist, z0, gammaM, kappa, q, thetaRef);
        if ((dfLow > 0 && dfMid > 0) || (dfLow < 0 && dfMid < 0)) uLow = uMid;
        else uHigh = uMid;
    }
    return uMid;
}

// uStarShumann, wallfunctions.c:12-130: friction velocity for a given wall heat flux
double uStarShumann(double U, double wallDist, double z0, double gammaM, double kappa, double qwall, double thetaRef)
{
    if (wallDist <= z0) throw OracleError("wall distance is smaller than the roughness length");
    const double logLaw = std::log(wallDist / z0);
    const double uN = std::max(0.0, (kappa * U) / logLaw);
    if (std::fabs(qwall) < 1e-6) return uN;
    double u0 = uN, diff = 1e30;
    int iter = 0;
    do {
        const double L0 = moClampL(-std::pow(u0, 3.0) / (kappa * (kMoG / thetaRef) * qwall));
        double psiM, psiH, phiM, phiH;
        moStability(wallDist / L0, L0 > 0, gammaM, 0.0, 0.0, psiM, psiH, phiM, phiH);
        const double uNew = std::max(0.0, (kappa * U) / (logLaw - psiM));
        u0 = kMoOmega * uNew + (1.0 - kMoOmega) * u0;
        diff = std::fabs(uNew - u0);
        iter++;
    } while (diff > kMoTol && iter < kMoIterMax);
    if (iter == kMoIterMax) return uN;
    const double L = moClampL(-std::pow(u0, 3.0) / (kappa * (kMoG / thetaRef) * qwall));
    if (L > 0 && u0 < 1e-2) return moStableBisection(U, wallDist, z0, gammaM, kappa, qwall, thetaRef, uN);
    return u0;
}

// qWallShumann, wallfunctions.c:133-290: wall heat flux (and u*) for a
// temperature difference deltaTheta between the first cell and the surface
double qWallShumann(double U, double wallDist, double z0, double gammaM, double gammaH, double alphaH, double thetaRef,
                    double deltaTheta, double kappa)
{
    if (wallDist <= z0) throw OracleError("wall distance is smaller than the roughness length");
    const double uN = std::max(0.0, (kappa * U) / std::log(wallDist / z0));
    double qN = (-deltaTheta * uN * kappa) / (alphaH * std::log(wallDist / z0));
    if (std::fabs(qN) < 1e-6) qN = (qN < 0 ? -1.0 : 1.0) * 1e-6;        // signNonZero, inline.h:335-341
    if (deltaTheta == 0.0) return qN;
    double u0 = uN, q0 = qN, du = 1e30, dq = 1e30;
    int iter = 0;
    do {
        const double L0 = moClampL(-std::pow(u0, 3.0) / (kappa * (kMoG / thetaRef) * q0));
        double psiM, psiH, phiM, phiH;
        moStability(wallDist / L0, L0 > 0, gammaM, gammaH, alphaH, psiM, psiH, phiM, phiH);
        const double uNew = std::max(0.0, (kappa * U) / (std::log(wallDist / z0) - psiM));
        u0 = kMoOmega * uNew + (1.0 - kMoOmega) * u0;
        const double qNew = (-deltaTheta * u0 * kappa) / (alphaH * std::log(wallDist / z0) - psiH);
        q0 = kMoOmega * qNew + (1.0 - kMoOmega) * q0;
        du = std::fabs(uNew - u0);
        dq = std::fabs(qNew - q0);
        iter++;
    } while ((du > kMoTol || dq > kMoTol) && iter < kMoIterMax);
    if (iter == kMoIterMax) return qN;
    const double L = moClampL(-std::pow(u0, 3.0) / (kappa * (kMoG / thetaRef) * q0));
    if (L > 0 && u0 < 1e-2) {
        // the bisection's L uses the neutral heat flux
        const double us = moStableBisection(U, wallDist, z0, gammaM, kappa, qN, thetaRef, uN);
        const double Lf = std::max(1e-10, -std::pow(us, 3.0) / (kappa * (kMoG / thetaRef) * qN));
        const double psiH = -gammaH * (wallDist / Lf);
        return (-deltaTheta * us * kappa) / (alphaH * std::log(wallDist / z0) - psiH);
    }
    return q0;
}

// the jLeft temperature patch carries a thetaWallFunction whose qWall enters
// the velocity wall function (boundary.c:3348-3356)
bool thetaWallCoupled(const tg_ctx &C)
{
    return C.c.teqn && C.c.t_bc[TG_JLEFT] == TG_TBC_WALL_FUNCTION;
}

// ---------------------------------------------------------------------------
// UpdateWallModelsU, boundary.c:3257-3600: jLeft wall function -3 (Schumann,
// plane-averaged friction velocity, wallfunctions.c:12-130; stratified by
// the plane mean of the last temperature wall heat flux when the temperature
// jLeft patch is a thetaWallFunction, neutral otherwise)
// ---------------------------------------------------------------------------
void updateWallModels(tg_ctx &C)
{
    if (!C.c.les) return;
    if (C.c.bc[TG_JLEFT] != TG_BC_WALL_SHUMANN) return;
    const int mx = C.mx, mz = C.mz;
    const int j = 1;
    double aN = (double)C.it;
    double m1 = aN / (aN + 1.0), m2 = 1.0 / (aN + 1.0);
    auto parallel = [&](int k, int i, V3 &Up, V3 &n) {
        size_t c = C.I(k, j, i);
        double ni[3], nj[3], nk[3];
        calculateNormal(C.csi[c], C.eta[c], C.zet[c], ni, nj, nk);
        n = mk(nj[0], nj[1], nj[2]);
        V3 U = C.ucat[c];
        Up = U - dot(U, n) * n;
    };
    // plane averages
    double sumU = 0.0, sumD = 0.0; long cnt = 0;
    for (int k = 1; k < mz - 1; k++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        double area = mag(C.eta[c]);
        double s = 0.5 / C.aj[c] / area;
        V3 Up, n; parallel(k, i, Up, n);
        sumU += mag(Up); sumD += s; cnt++;
    }
    double qWall = 0.0;
    if (thetaWallCoupled(C)) {
        for (int k = 1; k < mz - 1; k++)
        for (int i = 1; i < mx - 1; i++) qWall += C.qwall[C.W(k, i)];
        qWall = qWall / cnt;
    }
    double Umean = sumU / cnt, dist = sumD / cnt;
    double z0 = C.c.wall_roughness, kappa = C.c.wall_kappa;
    double uStar = uStarShumann(Umean, dist, z0, C.c.wall_gamma_m, kappa, qWall, C.c.wall_theta_ref);
    if (!C.ufilt_set) {
        for (int k = 1; k < mz - 1; k++)
        for (int i = 1; i < mx - 1; i++) {
            V3 Up, n; parallel(k, i, Up, n);
            size_t w = C.W(k, i);
            C.ufx[w] = Up.x; C.ufy[w] = Up.y; C.ufz[w] = Up.z;
        }
        C.ufilt_set = true;
    }
    for (int k = 1; k < mz - 1; k++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i), w = C.W(k, i);
        V3 Up, n; parallel(k, i, Up, n);
        double upm = mag(Up);
        // nUnit, inline.h:870-890
        V3 e1 = mk(Up.x / (upm + 1.e-12), Up.y / (upm + 1.e-12), Up.z / (upm + 1.e-12));
        V3 e3 = n;
        V3 e2 = mk(e3.y * e1.z - e3.z * e1.y, e3.z * e1.x - e3.x * e1.z, e3.x * e1.y - e3.y * e1.x);
        C.umean[w] = m1 * C.umean[w] + m2 * upm;
        double lx = 1.0 / C.aj[c] / mag(C.zet[c]), ly = 1.0 / C.aj[c] / mag(C.csi[c]);
        double T = std::max(std::sqrt(lx * lx + ly * ly) / C.umean[w], C.c.dt);
        C.ufx[w] = (1.0 - C.c.dt / T) * C.ufx[w] + (C.c.dt / T) * Up.x;
        C.ufy[w] = (1.0 - C.c.dt / T) * C.ufy[w] + (C.c.dt / T) * Up.y;
        const V3 &je = C.jeta[C.I(k, j - 1, i)];
        if (C.c.curvilinear) {
            double a11 = e1.x, a12 = e2.x, a13 = e3.x;
            double a21 = e1.y, a22 = e2.y, a23 = e3.y;
            double a31 = e1.z, a32 = e2.z, a33 = e3.z;
            double u2 = uStar * uStar;
            double t11 = -2.0 * a11 * a13 * u2, t12 = -(a13 * a21 + a11 * a23) * u2, t13 = -(a13 * a31 + a11 * a33) * u2;
            double t21 = -(a23 * a11 + a21 * a13) * u2, t22 = -2.0 * a23 * a21 * u2, t23 = -(a23 * a31 + a21 * a33) * u2;
            double t31 = -(a33 * a11 + a31 * a13) * u2, t32 = -(a33 * a21 + a31 * a23) * u2, t33 = -2.0 * a33 * a31 * u2;
            C.twx[w] = t11 * je.x + t12 * je.y + t13 * je.z;
            C.twy[w] = t21 * je.x + t22 * je.y + t23 * je.z;
            C.twz[w] = t31 * je.x + t32 * je.y + t33 * je.z;
        } else {
            double TauXZ = -uStar * uStar * (C.ufx[w] / std::max(Umean, 1e-5));
            double TauYZ = -uStar * uStar * (C.ufy[w] / std::max(Umean, 1e-5));
            C.twx[w] = je.z * TauXZ;
            C.twy[w] = je.z * TauYZ;
            C.twz[w] = je.x * TauXZ + je.y * TauYZ;
        }
    }
}

// ---------------------------------------------------------------------------
// GradP, peqn.c:3437-3773
// ---------------------------------------------------------------------------
// the GradP stencil applied to the scalar val(q) into outv
template <class Val>
void gradField(tg_ctx &C, Val val, std::vector<V3> &outv)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    std::fill(outv.begin(), outv.end(), V3{0, 0, 0});
    auto P = [&](int k, int j, int i) { return val(C.I(k, j, i)); };
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        const V3 &ic = C.icsi[c], &ie = C.ieta[c], &iz = C.izet[c];
        const V3 &jc = C.jcsi[c], &je = C.jeta[c], &jz = C.jzet[c];
        const V3 &kc = C.kcsi[c], &ke = C.keta[c], &kz = C.kzet[c];
        double g11 = dot(ic, ic), g12 = dot(ie, ic), g13 = dot(iz, ic);
        double g21 = dot(jc, je), g22 = dot(je, je), g23 = dot(jz, je);
        double g31 = dot(kc, kz), g32 = dot(ke, kz), g33 = dot(kz, kz);
        double dpdc, dpde, dpdz;
        V3 out;
        // i-direction
        dpdc = (i == mx - 2 && C.pi) ? P(k, j, mx + 1) - P(k, j, i) : P(k, j, i + 1) - P(k, j, i);
        if (j == my - 2 && i == mx - 2)  dpde = (P(k, j, i) - P(k, j - 1, i) + P(k, j, i + 1) - P(k, j - 1, i + 1)) * 0.5;
        else if (j == 1 && i == mx - 2)  dpde = (P(k, j + 1, i) - P(k, j, i) + P(k, j + 1, i + 1) - P(k, j, i + 1)) * 0.5;
        else                             dpde = (P(k, j + 1, i) - P(k, j - 1, i) + P(k, j + 1, i + 1) - P(k, j - 1, i + 1)) * 0.25;
        if (k == mz - 2 && i == mx - 2)  dpdz = (P(k, j, i) - P(k - 1, j, i) + P(k, j, i + 1) - P(k - 1, j, i + 1)) * 0.5;
        else if (k == 1 && i == mx - 2)  dpdz = (P(k + 1, j, i) - P(k, j, i) + P(k + 1, j, i + 1) - P(k, j, i + 1)) * 0.5;
        else                             dpdz = (P(k + 1, j, i) - P(k - 1, j, i) + P(k + 1, j, i + 1) - P(k - 1, j, i + 1)) * 0.25;
        out.x = (dpdc * g11 + dpde * g12 + dpdz * g13) * C.iaj[c];
        // j-direction
        if (i == mx - 2 && j == my - 2)  dpdc = (P(k, j, i) - P(k, j, i - 1) + P(k, j + 1, i) - P(k, j + 1, i - 1)) * 0.5;
        else if (i == 1 && j == my - 2)  dpdc = (P(k, j, i + 1) - P(k, j, i) + P(k, j + 1, i + 1) - P(k, j + 1, i)) * 0.5;
        else                             dpdc = (P(k, j, i + 1) - P(k, j, i - 1) + P(k, j + 1, i + 1) - P(k, j + 1, i - 1)) * 0.25;
        dpde = (j == my - 2 && C.pj) ? P(k, my + 1, i) - P(k, j, i) : P(k, j + 1, i) - P(k, j, i);
        if (k == mz - 2 && j == my - 2)  dpdz = (P(k, j, i) - P(k - 1, j, i) + P(k, j + 1, i) - P(k - 1, j + 1, i)) * 0.5;
        else if (k == 1 && j == my - 2)  dpdz = (P(k + 1, j, i) - P(k, j, i) + P(k + 1, j + 1, i) - P(k, j + 1, i)) * 0.5;
        else                             dpdz = (P(k + 1, j, i) - P(k - 1, j, i) + P(k + 1, j + 1, i) - P(k - 1, j + 1, i)) * 0.25;
        out.y = (dpdc * g21 + dpde * g22 + dpdz * g23) * C.jaj[c];
        // k-direction
        if (i == mx - 2 && k == mz - 2)  dpdc = (P(k, j, i) - P(k, j, i - 1) + P(k + 1, j, i) - P(k + 1, j, i - 1)) * 0.5;
        else if (i == 1 && k == mz - 2)  dpdc = (P(k, j, i + 1) - P(k, j, i) + P(k + 1, j, i + 1) - P(k + 1, j, i)) * 0.5;
        else                             dpdc = (P(k, j, i + 1) - P(k, j, i - 1) + P(k + 1, j, i + 1) - P(k + 1, j, i - 1)) * 0.25;
        if (j == my - 2 && k == mz - 2)  dpde = (P(k, j, i) - P(k, j - 1, i) + P(k + 1, j, i) - P(k + 1, j - 1, i)) * 0.5;
        else if (j == 1 && k == mz - 2)  dpde = (P(k, j + 1, i) - P(k, j, i) + P(k + 1, j + 1, i) - P(k + 1, j, i)) * 0.5;
        else                             dpde = (P(k, j + 1, i) - P(k, j - 1, i) + P(k + 1, j + 1, i) - P(k + 1, j - 1, i)) * 0.25;
        dpdz = (k == mz - 2 && C.pk) ? P(mz + 1, j, i) - P(k, j, i) : P(k + 1, j, i) - P(k, j, i);
        out.z = (dpdc * g31 + dpde * g32 + dpdz * g33) * C.kaj[c];
        // faces where the contravariant velocity is not solved
        if (!C.pi && i == mx - 2) out.x = 0;
        if (!C.pj && j == my - 2) out.y = 0;
        if (!C.pk && k == mz - 2) out.z = 0;
        outv[c] = out;
    }
}

void gradP(tg_ctx &C)
{
    gradField(C, [&](size_t q) { return C.p[q]; }, C.dp);
}

// ghGradRhoK, teqn.c:278-652 (-pTildeBuoyancy 1): the GradP stencil on
// rho_k = (tRef - T) / tRef scaled by g z of the cell's node, stored negated in
// bTheta so that the AB2 buoyancy sum of ExplicitRhsU (+3/2 b - 1/2 b_o) reads
// -3/2 ghGradRhok + 1/2 ghGradRhok_o (ueqn_solvers.c:1314-1324)
void ghGradRhoK(tg_ctx &C)
{
    const double tRef = C.c.t_ref;
    std::vector<V3> db(C.G);
    gradField(C, [&](size_t q) { return (tRef - C.tmprt[q]) / tRef; }, db);
    for (int k = 1; k < C.mz - 1; k++)
    for (int j = 1; j < C.my - 1; j++)
    for (int i = 1; i < C.mx - 1; i++) {
        const size_t c = C.I(k, j, i);
        const double gz = -9.81 * C.coor[c].z;
        C.btheta[c] = mk(-(gz * db[c].x), -(gz * db[c].y), -(gz * db[c].z));
    }
}

// Buoyancy, ueqn_sources.c:2726-2880 (frozen temperature)
void buoyancy(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const double gz = -9.81, tRef = C.c.t_ref;
    for (int k = 0; k < mz - 1; k++)
    for (int j = 0; j < my - 1; j++)
    for (int i = 0; i < mx - 1; i++) {
        size_t f = C.I(k, j, i);
        if (j > 0 && k > 0) C.gcont[f].x = 0 * C.icsi[f].x + 0 * C.icsi[f].y + gz * C.icsi[f].z;
        if (i > 0 && k > 0) C.gcont[f].y = 0 * C.jeta[f].x + 0 * C.jeta[f].y + gz * C.jeta[f].z;
        if (i > 0 && j > 0) C.gcont[f].z = 0 * C.kzet[f].x + 0 * C.kzet[f].y + gz * C.kzet[f].z;
    }
    std::fill(C.btheta.begin(), C.btheta.end(), V3{0, 0, 0});
    auto T = [&](int k, int j, int i) { return C.tmprt[C.I(k, j, i)]; };
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        double tI = 0.5 * (T(k, j, i) + T(k, j, i + 1));
        double tJ = 0.5 * (T(k, j, i) + T(k, j + 1, i));
        double tK = 0.5 * (T(k, j, i) + T(k + 1, j, i));
        C.btheta[c].x += 1.0 * (C.gcont[c].x * (tRef - tI) / tRef);
        C.btheta[c].y += 1.0 * (C.gcont[c].y * (tRef - tJ) / tRef);
        C.btheta[c].z += 1.0 * (C.gcont[c].z * (tRef - tK) / tRef);
    }
}

// ---------------------------------------------------------------------------
// FormU, ueqn_solvers.c:6-1083 (formMode 0, no IBM/overset, no damping)
// ---------------------------------------------------------------------------
inline V3 quick(const V3 &f0, const V3 &f1, const V3 &f2, const V3 &f3, double w)
{
    // quadraticUpwindVec, inline.h:5089-5109
    V3 fUU, fU, fD;
    if (w > 0) { fUU = f0; fU = f1; fD = f2; } else { fUU = f3; fU = f2; fD = f1; }
    return 0.5 * (fU + fD) + (1. / 8.) * (2.0 * fU - (fD + fUU));
}

// mode: formMode (ueqn_solvers.c:17, 105-106, 877-928): 0 convection +
// viscosity, 1 convection only, 2 viscosity (with the wall stress) only
void formU(tg_ctx &C, std::vector<V3> &R, double scale, int mode = 0)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const bool quickDiv = C.c.div_scheme == TG_DIV_QUICK;
    const bool les = C.c.les != 0;
    const double nu = C.c.nu;
    const int *bc = C.c.bc;
    auto U = [&](int k, int j, int i) -> const V3 & { return C.ucat[C.I(k, j, i)]; };
    auto NUT = [&](int k, int j, int i) { return C.nut[C.I(k, j, i)]; };
    std::fill(C.div1.begin(), C.div1.end(), V3{0, 0, 0});
    std::fill(C.div2.begin(), C.div2.end(), V3{0, 0, 0});
    std::fill(C.div3.begin(), C.div3.end(), V3{0, 0, 0});
    std::fill(C.visc1.begin(), C.visc1.end(), V3{0, 0, 0});
    std::fill(C.visc2.begin(), C.visc2.end(), V3{0, 0, 0});
    std::fill(C.visc3.begin(), C.visc3.end(), V3{0, 0, 0});
    std::fill(C.fp.begin(), C.fp.end(), V3{0, 0, 0});
    const bool npi = !C.pi, npj = !C.pj, npk = !C.pk;

    // viscous flux of one face: (g.grad u + R.S) * ajc * nuEff, ueqn_solvers.c:392-394
    auto viscFlux = [](V3 s0, V3 s1, V3 s2, int dir, V3 dc, V3 de, V3 dz, double ajc, double nuEff) {
        // s0,s1,s2 = face csi, eta, zet; dir selects the face normal (0 csi, 1 eta, 2 zet)
        double csi0 = s0.x, csi1 = s0.y, csi2 = s0.z;
        double eta0 = s1.x, eta1 = s1.y, eta2 = s1.z;
        double zet0 = s2.x, zet1 = s2.y, zet2 = s2.z;
        double g11, g21, g31;
        double n0, n1, n2;
        if (dir == 0) { g11 = csi0 * csi0 + csi1 * csi1 + csi2 * csi2; g21 = eta0 * csi0 + eta1 * csi1 + eta2 * csi2; g31 = zet0 * csi0 + zet1 * csi1 + zet2 * csi2; n0 = csi0; n1 = csi1; n2 = csi2; }
        else if (dir == 1) { g11 = csi0 * eta0 + csi1 * eta1 + csi2 * eta2; g21 = eta0 * eta0 + eta1 * eta1 + eta2 * eta2; g31 = zet0 * eta0 + zet1 * eta1 + zet2 * eta2; n0 = eta0; n1 = eta1; n2 = eta2; }
        else { g11 = csi0 * zet0 + csi1 * zet1 + csi2 * zet2; g21 = eta0 * zet0 + eta1 * zet1 + eta2 * zet2; g31 = zet0 * zet0 + zet1 * zet1 + zet2 * zet2; n0 = zet0; n1 = zet1; n2 = zet2; }
        double r11 = dc.x * csi0 + de.x * eta0 + dz.x * zet0;
        double r21 = dc.y * csi0 + de.y * eta0 + dz.y * zet0;
        double r31 = dc.z * csi0 + de.z * eta0 + dz.z * zet0;
        double r12 = dc.x * csi1 + de.x * eta1 + dz.x * zet1;
        double r22 = dc.y * csi1 + de.y * eta1 + dz.y * zet1;
        double r32 = dc.z * csi1 + de.z * eta1 + dz.z * zet1;
        double r13 = dc.x * csi2 + de.x * eta2 + dz.x * zet2;
        double r23 = dc.y * csi2 + de.y * eta2 + dz.y * zet2;
        double r33 = dc.z * csi2 + de.z * eta2 + dz.z * zet2;
        V3 v;
        v.x = (g11 * dc.x + g21 * de.x + g31 * dz.x + r11 * n0 + r21 * n1 + r31 * n2) * ajc * (nuEff);
        v.y = (g11 * dc.y + g21 * de.y + g31 * dz.y + r12 * n0 + r22 * n1 + r32 * n2) * ajc * (nuEff);
        v.z = (g11 * dc.z + g21 * de.z + g31 * dz.z + r13 * n0 + r23 * n1 + r33 * n2) * ajc * (nuEff);
        return v;
    };

    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < mz - 1; k++)
    for (int j = 0; j < my - 1; j++)
    for (int i = 0; i < mx - 1; i++) {
        size_t f = C.I(k, j, i);
        // ---------------- i faces, ueqn_solvers.c:173-395
        if (j != 0 && k != 0) {
            double ajc = C.iaj[f];
            // Compute_du_i, inline.h:2748-2807
            V3 dc = U(k, j, i + 1) - U(k, j, i), de, dz;
            bool iedge = (i == 0 || i == mx - 2);
            if (j == my - 2 && iedge && (npj || npi))      de = 0.5 * (U(k, j, i + 1) + U(k, j, i) - U(k, j - 1, i + 1) - U(k, j - 1, i));
            else if (j == 1 && iedge && (npj || npi))      de = 0.5 * (U(k, j + 1, i + 1) + U(k, j + 1, i) - U(k, j, i + 1) - U(k, j, i));
            else                                           de = 0.25 * (U(k, j + 1, i + 1) + U(k, j + 1, i) - U(k, j - 1, i + 1) - U(k, j - 1, i));
            if (k == mz - 2 && iedge && (npk || npi))      dz = 0.5 * (U(k, j, i + 1) + U(k, j, i) - U(k - 1, j, i + 1) - U(k - 1, j, i));
            else if (k == 1 && iedge && (npk || npi))      dz = 0.5 * (U(k + 1, j, i + 1) + U(k + 1, j, i) - U(k, j, i + 1) - U(k, j, i));
            else                                           dz = 0.25 * (U(k + 1, j, i + 1) + U(k + 1, j, i) - U(k - 1, j, i + 1) - U(k - 1, j, i));
            // convection
            double uc = C.ucont[f].x;
            if (quickDiv) {
                int iL, iR;
                if (i == 0 || i == mx - 2) {
                    if (C.pi && i == mx - 2) { iR = mx + 2; iL = i - 1; }
                    else if (C.pi && i == 0) { iL = -3; iR = i + 2; }
                    else if (i == 0) { iL = i; iR = i + 2; }
                    else { iL = i - 1; iR = i + 1; }
                } else { iL = i - 1; iR = i + 2; }
                C.div1[f] = (-uc) * quick(U(k, j, iL), U(k, j, i), U(k, j, i + 1), U(k, j, iR), uc);
            } else {
                C.div1[f] = (-uc) * (0.5 * (U(k, j, i) + U(k, j, i + 1)));
            }
            // viscous
            double nuEff;
            V3 base{0, 0, 0};
            if (les) {
                double nt = 0.5 * (NUT(k, j, i) + NUT(k, j, i + 1));
                if ((bc[TG_ILEFT] == TG_BC_SLIP && i == 0) || (bc[TG_IRIGHT] == TG_BC_SLIP && i == mx - 2)) nuEff = 0.0;
                else nuEff = nu + nt;
            } else nuEff = nu;
            V3 v = viscFlux(C.icsi[f], C.ieta[f], C.izet[f], 0, dc, de, dz, ajc, nuEff);
            C.visc1[f] = base + v;
        }
        // ---------------- j faces, ueqn_solvers.c:397-602
        if (i != 0 && k != 0) {
            double ajc = C.jaj[f];
            // Compute_du_j, inline.h:2809-2869
            V3 dc, de = U(k, j + 1, i) - U(k, j, i), dz;
            bool jedge = (j == 0 || j == my - 2);
            if (i == mx - 2 && jedge && (npi || npj))      dc = 0.5 * (U(k, j + 1, i) + U(k, j, i) - U(k, j + 1, i - 1) - U(k, j, i - 1));
            else if (i == 1 && jedge && (npi || npj))      dc = 0.5 * (U(k, j + 1, i + 1) + U(k, j, i + 1) - U(k, j + 1, i) - U(k, j, i));
            else                                           dc = 0.25 * (U(k, j + 1, i + 1) + U(k, j, i + 1) - U(k, j + 1, i - 1) - U(k, j, i - 1));
            if (k == mz - 2 && jedge && (npk || npj))      dz = 0.5 * (U(k, j + 1, i) + U(k, j, i) - U(k - 1, j + 1, i) - U(k - 1, j, i));
            else if (k == 1 && jedge && (npk || npj))      dz = 0.5 * (U(k + 1, j + 1, i) + U(k + 1, j, i) - U(k, j + 1, i) - U(k, j, i));
            else                                           dz = 0.25 * (U(k + 1, j + 1, i) + U(k + 1, j, i) - U(k - 1, j + 1, i) - U(k - 1, j, i));
            double uc = C.ucont[f].y;
            if (quickDiv) {
                int jL, jR;
                if (j == 0 || j == my - 2) {
                    if (C.pj && j == my - 2) { jR = my + 2; jL = j - 1; }
                    else if (C.pj && j == 0) { jL = -3; jR = j + 2; }
                    else if (j == 0) { jL = j; jR = j + 2; }
                    else { jL = j - 1; jR = j + 1; }
                } else { jL = j - 1; jR = j + 2; }
                C.div2[f] = (-uc) * quick(U(k, jL, i), U(k, j, i), U(k, j + 1, i), U(k, jR, i), uc);
            } else {
                C.div2[f] = (-uc) * (0.5 * (U(k, j, i) + U(k, j + 1, i)));
            }
            double nuEff;
            V3 base{0, 0, 0};
            if (les) {
                double nt = 0.5 * (NUT(k, j, i) + NUT(k, j + 1, i));
                // wall model on either j patch reads the jLeft stress, ueqn_solvers.c:548-558
                if ((bc[TG_JLEFT] == TG_BC_WALL_SHUMANN && j == 0) || (bc[TG_JRIGHT] == TG_BC_WALL_SHUMANN && j == my - 2)) {
                    size_t w = C.W(k, i);
                    base = mk(-C.twx[w], -C.twy[w], -C.twz[w]);
                    nuEff = nu;
                } else if ((bc[TG_JLEFT] == TG_BC_SLIP && j == 0) || (bc[TG_JRIGHT] == TG_BC_SLIP && j == my - 2)) nuEff = 0.0;
                else nuEff = nu + nt;
            } else nuEff = nu;
            V3 v = viscFlux(C.jcsi[f], C.jeta[f], C.jzet[f], 1, dc, de, dz, ajc, nuEff);
            C.visc2[f] = base + v;
        }
        // ---------------- k faces, ueqn_solvers.c:604-778
        if (i != 0 && j != 0) {
            double ajc = C.kaj[f];
            // Compute_du_k, inline.h:2871-2931
            V3 dc, de, dz = U(k + 1, j, i) - U(k, j, i);
            bool kedge = (k == 0 || k == mz - 2);
            if (i == mx - 2 && kedge && (npi || npk))      dc = 0.5 * (U(k + 1, j, i) + U(k, j, i) - U(k + 1, j, i - 1) - U(k, j, i - 1));
            else if (i == 1 && kedge && (npi || npk))      dc = 0.5 * (U(k + 1, j, i + 1) + U(k, j, i + 1) - U(k + 1, j, i) - U(k, j, i));
            else                                           dc = 0.25 * (U(k + 1, j, i + 1) + U(k, j, i + 1) - U(k + 1, j, i - 1) - U(k, j, i - 1));
            if (j == my - 2 && kedge && (npj || npk))      de = 0.5 * (U(k + 1, j, i) + U(k, j, i) - U(k + 1, j - 1, i) - U(k, j - 1, i));
            else if (j == 1 && kedge && (npj || npk))      de = 0.5 * (U(k + 1, j + 1, i) + U(k, j + 1, i) - U(k + 1, j, i) - U(k, j, i));
            else                                           de = 0.25 * (U(k + 1, j + 1, i) + U(k, j + 1, i) - U(k + 1, j - 1, i) - U(k, j - 1, i));
            double uc = C.ucont[f].z;
            if (quickDiv) {
                int kL, kR;
                if (k == 0 || k == mz - 2) {
                    if (C.pk && k == mz - 2) { kR = mz + 2; kL = k - 1; }
                    else if (C.pk && k == 0) { kL = -3; kR = k + 2; }
                    else if (k == 0) { kL = k; kR = k + 2; }
                    else { kL = k - 1; kR = k + 1; }
                } else { kL = k - 1; kR = k + 2; }
                C.div3[f] = (-uc) * quick(U(kL, j, i), U(k, j, i), U(k + 1, j, i), U(kR, j, i), uc);
            } else {
                C.div3[f] = (-uc) * (0.5 * (U(k, j, i) + U(k + 1, j, i)));
            }
            double nuEff;
            if (les) {
                double nt = 0.5 * (NUT(k, j, i) + NUT(k + 1, j, i));
                if ((bc[TG_KLEFT] == TG_BC_SLIP && k == 0) || (bc[TG_KRIGHT] == TG_BC_SLIP && k == mz - 2)) nuEff = 0.0;
                else nuEff = nu + nt;
            } else nuEff = nu;
            C.visc3[f] = viscFlux(C.kcsi[f], C.keta[f], C.kzet[f], 2, dc, de, dz, ajc, nuEff);
        }
    }

    // periodic face copies, ueqn_solvers.c:807-812
    resetFacePeriodic(C, C.div1); resetFacePeriodic(C, C.div2); resetFacePeriodic(C, C.div3);
    resetFacePeriodic(C, C.visc1); resetFacePeriodic(C, C.visc2); resetFacePeriodic(C, C.visc3);

    // cell sums, ueqn_solvers.c:825-990
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        size_t iw = C.I(k, j, i - 1), js = C.I(k, j - 1, i), kb = C.I(k - 1, j, i);
        V3 &F = C.fp[c];
        if (mode != 2) {
            F.x += (C.div1[c].x - C.div1[iw].x + C.div2[c].x - C.div2[js].x + C.div3[c].x - C.div3[kb].x);
            F.y += (C.div1[c].y - C.div1[iw].y + C.div2[c].y - C.div2[js].y + C.div3[c].y - C.div3[kb].y);
            F.z += (C.div1[c].z - C.div1[iw].z + C.div2[c].z - C.div2[js].z + C.div3[c].z - C.div3[kb].z);
        }
        if (mode != 1) {
            F.x += (C.visc1[c].x - C.visc1[iw].x + C.visc2[c].x - C.visc2[js].x + C.visc3[c].x - C.visc3[kb].x);
            F.y += (C.visc1[c].y - C.visc1[iw].y + C.visc2[c].y - C.visc2[js].y + C.visc3[c].y - C.visc3[kb].y);
            F.z += (C.visc1[c].z - C.visc1[iw].z + C.visc2[c].z - C.visc2[js].z + C.visc3[c].z - C.visc3[kb].z);
        }
        if (i == 1 && npi)      C.fp[C.I(k, j, i - 1)] = F;
        if (j == 1 && npj)      C.fp[C.I(k, j - 1, i)] = F;
        if (k == 1 && npk)      C.fp[C.I(k - 1, j, i)] = F;
        if (i == mx - 2 && npi) C.fp[C.I(k, j, i + 1)] = F;
        if (j == my - 2 && npj) C.fp[C.I(k, j + 1, i)] = F;
        if (k == mz - 2 && npk) C.fp[C.I(k + 1, j, i)] = F;
    }
    resetCellPeriodic(C, C.fp);

    // face interpolation dotted with area vectors, ueqn_solvers.c:1008-1035
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        size_t ie = C.I(k, j, i + 1), jn = C.I(k, j + 1, i), kt = C.I(k + 1, j, i);
        double v1, v2;
        v1 = C.csi[c].x * C.fp[c].x + C.csi[c].y * C.fp[c].y + C.csi[c].z * C.fp[c].z;
        v2 = C.csi[ie].x * C.fp[ie].x + C.csi[ie].y * C.fp[ie].y + C.csi[ie].z * C.fp[ie].z;
        R[c].x += scale * C.iaj[c] * (0.5 * (v1 + v2));
        v1 = C.eta[c].x * C.fp[c].x + C.eta[c].y * C.fp[c].y + C.eta[c].z * C.fp[c].z;
        v2 = C.eta[jn].x * C.fp[jn].x + C.eta[jn].y * C.fp[jn].y + C.eta[jn].z * C.fp[jn].z;
        R[c].y += scale * C.jaj[c] * (0.5 * (v1 + v2));
        v1 = C.zet[c].x * C.fp[c].x + C.zet[c].y * C.fp[c].y + C.zet[c].z * C.fp[c].z;
        v2 = C.zet[kt].x * C.fp[kt].x + C.zet[kt].y * C.fp[kt].y + C.zet[kt].z * C.fp[kt].z;
        R[c].z += scale * C.kaj[c] * (0.5 * (v1 + v2));
    }
}

// meanGradPForcing, ueqn_sources.c:3735-3822
void meanGradPForcing(tg_ctx &C, std::vector<V3> &R)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const double *g = C.c.mean_grad_p_value;
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        R[c].x += 1.0 * (g[0] * C.icsi[c].x + g[1] * C.icsi[c].y + g[2] * C.icsi[c].z);
        R[c].y += 1.0 * (g[0] * C.jeta[c].x + g[1] * C.jeta[c].y + g[2] * C.jeta[c].z);
        R[c].z += 1.0 * (g[0] * C.kzet[c].x + g[1] * C.kzet[c].y + g[2] * C.kzet[c].z);
    }
}

// sourceU, ueqn_sources.c:2884-2980: central face value of the body force
// dotted with the face area vector, faces of interior cells
void sourceU(tg_ctx &C, std::vector<V3> &R)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const std::vector<V3> &f = C.source;
    auto lin = [&](int k, int j, int i) { return ((size_t)k * my + j) * mx + i; };   // global Vec: no wrap
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = lin(k, j, i), ie = lin(k, j, i + 1), jn = lin(k, j + 1, i), kt = lin(k + 1, j, i);
        R[c].x += 1.0 * (0.5 * (f[c].x + f[ie].x) * C.icsi[c].x + 0.5 * (f[c].y + f[ie].y) * C.icsi[c].y + 0.5 * (f[c].z + f[ie].z) * C.icsi[c].z);
        R[c].y += 1.0 * (0.5 * (f[c].x + f[jn].x) * C.jeta[c].x + 0.5 * (f[c].y + f[jn].y) * C.jeta[c].y + 0.5 * (f[c].z + f[jn].z) * C.jeta[c].z);
        R[c].z += 1.0 * (0.5 * (f[c].x + f[kt].x) * C.kzet[c].x + 0.5 * (f[c].y + f[kt].y) * C.kzet[c].y + 0.5 * (f[c].z + f[kt].z) * C.kzet[c].z);
    }
}

// resetNonResolvedCellFaces, inline.h:1674-1835
void resetNonResolvedCellFaces(tg_ctx &C, std::vector<V3> &V)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
        size_t c = C.I(k, j, i);
        V3 &v = V[c];
        const V3 &uo = C.ucont_o[c];
        // a boundary face keeps its value on a zeroGradient patch or where
        // the flow left the domain at the step start
        auto zg = [&](int patch) { return C.c.bc[patch] == TG_BC_ZERO_GRADIENT; };
        if (i == 0) { if (!(zg(TG_ILEFT) || uo.x < 0)) v.x = 0.0; }
        else if (i == mx - 1) v.x = 0.0;
        else if (i == mx - 2 && !C.pi) { if (!(zg(TG_IRIGHT) || uo.x > 0)) v.x = 0.0; }
        if (j == 0) { if (!(zg(TG_JLEFT) || uo.y < 0)) v.y = 0.0; }
        else if (j == my - 1) v.y = 0.0;
        else if (j == my - 2 && !C.pj) { if (!(zg(TG_JRIGHT) || uo.y > 0)) v.y = 0.0; }
        if (k == 0) { if (!(zg(TG_KLEFT) || uo.z < 0)) v.z = 0.0; }
        else if (k == mz - 1) v.z = 0.0;
        else if (k == mz - 2 && !C.pk) { if (!(zg(TG_KRIGHT) || uo.z > 0)) v.z = 0.0; }
    }
}

#include "tosca_oracle_farm.inc"
#include "tosca_oracle_cn.inc"
#include "tosca_oracle_teqn.inc"

// ExplicitRhsU, ueqn_solvers.c:1276-1407 (mode: formMode of its FormU)
void explicitRhsU(tg_ctx &C, int mode = 0)
{
    resetNoPenetration(C);
    resetFacePeriodic(C, C.ucont);
    contravariantToCartesian(C);
    resetCellPeriodic(C, C.ucat);
    const size_t G = C.G;
    for (size_t q = 0; q < G; q++) C.rhs[q] = V3{0, 0, 0} - C.dp[q];
    if (C.c.buoyancy) {
        if (C.it > C.c.it_start) {
            for (size_t q = 0; q < G; q++) {
                C.rhs[q] = C.rhs[q] + (3.0 / 2.0) * C.btheta[q];
                C.rhs[q] = C.rhs[q] + (-1.0 / 2.0) * C.btheta_o[q];
            }
        } else {
            for (size_t q = 0; q < G; q++) C.rhs[q] = C.rhs[q] + 1.0 * C.btheta[q];
        }
    }
    if (!C.farm.empty())                                // ueqn_solvers.c:1340-1344
        for (size_t q = 0; q < G; q++) C.rhs[q] = C.rhs[q] + 1.0 * C.farm_cont[q];
    formU(C, C.rhs, 1.0, mode);
    if (C.c.source) sourceU(C, C.rhs);                 // ueqn_solvers.c:1365-1370
    if (C.c.mean_grad_p) meanGradPForcing(C, C.rhs);
    resetNonResolvedCellFaces(C, C.rhs);
}

#include "tosca_oracle_imex.inc"

// adjustFluxesLocal, ueqn.c:748-1135. The faces of the non-periodic, non-wall
// patches (patch type 0) are split by the sign of their flux into inflow (into
// the domain) and outflow; the outflow faces then take the imbalance
// FluxOut - FluxIn in proportion to their own flux, so that the boundary
// fluxes sum to zero. A face with zero (or non-finite) flux is set to zero.
// Patches are visited in the reference's order (k, j, i; left, right) and
// their faces in its loop order.
void adjustFluxesLocal(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const int *bc = C.c.bc;
    auto type0 = [&](int patch) { return bc[patch] != TG_BC_PERIODIC && !isWall(bc[patch]); };
    auto faces = [&](int patch, auto &&fn) {
        const int dir = patch >> 1, right = patch & 1;
        if (dir == 2) {
            const int k = right ? mz - 2 : 0;
            for (int j = 1; j < my - 1; j++) for (int i = 1; i < mx - 1; i++) fn(C.ucont[C.I(k, j, i)].z);
        } else if (dir == 1) {
            const int j = right ? my - 2 : 0;
            for (int k = 1; k < mz - 1; k++) for (int i = 1; i < mx - 1; i++) fn(C.ucont[C.I(k, j, i)].y);
        } else {
            const int i = right ? mx - 2 : 0;
            for (int k = 1; k < mz - 1; k++) for (int j = 1; j < my - 1; j++) fn(C.ucont[C.I(k, j, i)].x);
        }
    };
    const int order[6] = {TG_KLEFT, TG_KRIGHT, TG_JLEFT, TG_JRIGHT, TG_ILEFT, TG_IRIGHT};
    double in = 0.0, out = 0.0;
    for (int patch : order) {
        if (!type0(patch)) continue;
        const bool right = patch & 1;
        faces(patch, [&](double &u) {
            if (u > 0.0) { if (right) out += u; else in += u; }
            else if (u < 0.0) { if (right) in += std::fabs(u); else out += std::fabs(u); }
            else u = 0.0;
        });
    }
    const double gf = out - in;
    for (int patch : order) {
        if (!type0(patch)) continue;
        const bool right = patch & 1;
        faces(patch, [&](double &u) {
            if (!right && u < 0.0) u += gf * (std::fabs(u) / out);
            if (right && u > 0.0) u -= gf * (u / out);
        });
    }
}

// SolveUEqn with UeqnFE / UeqnRK4, ueqn.c:397-440, ueqn_solvers.c:1411-1504
// (UeqnSNES and the IMEX schemes in their own files)
int solveUEqn(tg_ctx &C)
{
    const size_t G = C.G;
    const double dt = C.c.dt;
    int rc = 0;
    if (C.c.ddt_scheme == TG_DDT_CN) {
        rc = ueqnSNES(C);
    } else if (C.c.ddt_scheme >= TG_DDT_ABCN) {
        rc = ueqnIMEX(C);
    } else if (C.c.ddt_scheme == TG_DDT_FE) {
        explicitRhsU(C);
        // VecScale(Rhs,dt) then VecAXPY(Rhs,1,Ucont_o): dt*rhs + ucont_o
        for (size_t q = 0; q < G; q++) C.ucont[q] = mk(C.rhs[q].x * dt + C.ucont_o[q].x, C.rhs[q].y * dt + C.ucont_o[q].y, C.rhs[q].z * dt + C.ucont_o[q].z);
    } else {
        const double b[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
        const double a[4] = {0.0, 0.5, 0.5, 1.0};
        C.utmp = C.ucont_o;
        for (int s = 0; s < 4; s++) {
            if (s != 0)
                for (size_t q = 0; q < G; q++) C.ucont[q] = mk(a[s] * dt * C.rhs[q].x + C.ucont_o[q].x, a[s] * dt * C.rhs[q].y + C.ucont_o[q].y, a[s] * dt * C.rhs[q].z + C.ucont_o[q].z);
            explicitRhsU(C);
            for (size_t q = 0; q < G; q++) C.utmp[q] = C.utmp[q] + (dt * b[s]) * C.rhs[q];
        }
        C.ucont = C.utmp;
    }
    resetNoPenetration(C);
    resetFacePeriodic(C, C.ucont);
    contravariantToCartesian(C);
    resetCellPeriodic(C, C.ucat);
    adjustFluxesLocal(C);
    return rc;
}

// SetRHS, peqn.c:1942-2063
void setRHS(tg_ctx &C, std::vector<double> &b)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const double dt = C.c.dt;
    int64_t row = 0;
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++, row++) {
        if (i == 1 && j == 1 && k == 1) { b[row] = 0; continue; }
        size_t c = C.I(k, j, i);
        double val = 0;
        val += C.ucont[c].x;
        val -= C.ucont[C.I(k, j, i - 1)].x;
        val += C.ucont[c].y;
        val -= C.ucont[C.I(k, j - 1, i)].y;
        val += C.ucont[c].z;
        val -= C.ucont[C.I(k - 1, j, i)].z;
        val *= 1.0 / dt;
        b[row] = val;
    }
}

// ProjectVelocity, peqn.c:2495-2905
void projectVelocity(tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const double dt = C.c.dt;
    auto F = [&](int k, int j, int i) { return C.phi[C.I(k, j, i)]; };
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < mz - 1; k++)
    for (int j = 0; j < my - 1; j++)
    for (int i = 0; i < mx - 1; i++) {
        size_t f = C.I(k, j, i);
        if (j > 0 && k > 0 && ((i > 0 && i < mx - 2) || C.pi)) {
            double dpdc = F(k, j, i + 1) - F(k, j, i), dpde, dpdz;
            if (j == my - 2)      dpde = (F(k, j, i) + F(k, j, i + 1) - F(k, j - 1, i) - F(k, j - 1, i + 1)) * 0.5;
            else if (j == 1)      dpde = (F(k, j + 1, i) + F(k, j + 1, i + 1) - F(k, j, i) - F(k, j, i + 1)) * 0.5;
            else                  dpde = (F(k, j + 1, i) + F(k, j + 1, i + 1) - F(k, j - 1, i) - F(k, j - 1, i + 1)) * 0.25;
            if (k == mz - 2)      dpdz = (F(k, j, i) + F(k, j, i + 1) - F(k - 1, j, i) - F(k - 1, j, i + 1)) * 0.5;
            else if (k == 1)      dpdz = (F(k + 1, j, i) + F(k + 1, j, i + 1) - F(k, j, i) - F(k, j, i + 1)) * 0.5;
            else                  dpdz = (F(k + 1, j, i) + F(k + 1, j, i + 1) - F(k - 1, j, i) - F(k - 1, j, i + 1)) * 0.25;
            const V3 &c1 = C.icsi[f], &e1 = C.ieta[f], &z1 = C.izet[f];
            double a = C.iaj[f];
            C.ucont[f].x -= (dpdc * (c1.x * c1.x + c1.y * c1.y + c1.z * c1.z) * a
                           + dpde * (e1.x * c1.x + e1.y * c1.y + e1.z * c1.z) * a
                           + dpdz * (z1.x * c1.x + z1.y * c1.y + z1.z * c1.z) * a) * dt;
        }
        if (i > 0 && k > 0 && ((j > 0 && j < my - 2) || C.pj)) {
            double dpdc, dpde = F(k, j + 1, i) - F(k, j, i), dpdz;
            if (i == mx - 2)      dpdc = (F(k, j, i) + F(k, j + 1, i) - F(k, j, i - 1) - F(k, j + 1, i - 1)) * 0.5;
            else if (i == 1)      dpdc = (F(k, j, i + 1) + F(k, j + 1, i + 1) - F(k, j, i) - F(k, j + 1, i)) * 0.5;
            else                  dpdc = (F(k, j, i + 1) + F(k, j + 1, i + 1) - F(k, j, i - 1) - F(k, j + 1, i - 1)) * 0.25;
            if (k == mz - 2)      dpdz = (F(k, j, i) + F(k, j + 1, i) - F(k - 1, j, i) - F(k - 1, j + 1, i)) * 0.5;
            else if (k == 1)      dpdz = (F(k + 1, j, i) + F(k + 1, j + 1, i) - F(k, j, i) - F(k, j + 1, i)) * 0.5;
            else                  dpdz = (F(k + 1, j, i) + F(k + 1, j + 1, i) - F(k - 1, j, i) - F(k - 1, j + 1, i)) * 0.25;
            const V3 &c2 = C.jcsi[f], &e2 = C.jeta[f], &z2 = C.jzet[f];
            double a = C.jaj[f];
            C.ucont[f].y -= (dpdc * (c2.x * e2.x + c2.y * e2.y + c2.z * e2.z) * a
                           + dpde * (e2.x * e2.x + e2.y * e2.y + e2.z * e2.z) * a
                           + dpdz * (z2.x * e2.x + z2.y * e2.y + z2.z * e2.z) * a) * dt;
        }
        if (i > 0 && j > 0 && ((k > 0 && k < mz - 2) || C.pk)) {
            double dpdc, dpde, dpdz = F(k + 1, j, i) - F(k, j, i);
            if (i == mx - 2)      dpdc = (F(k, j, i) + F(k + 1, j, i) - F(k, j, i - 1) - F(k + 1, j, i - 1)) * 0.5;
            else if (i == 1)      dpdc = (F(k, j, i + 1) + F(k + 1, j, i + 1) - F(k, j, i) - F(k + 1, j, i)) * 0.5;
            else                  dpdc = (F(k, j, i + 1) + F(k + 1, j, i + 1) - F(k, j, i - 1) - F(k + 1, j, i - 1)) * 0.25;
            if (j == my - 2)      dpde = (F(k, j, i) + F(k + 1, j, i) - F(k, j - 1, i) - F(k + 1, j - 1, i)) * 0.5;
            else if (j == 1)      dpde = (F(k, j + 1, i) + F(k + 1, j + 1, i) - F(k, j, i) - F(k + 1, j, i)) * 0.5;
            else                  dpde = (F(k, j + 1, i) + F(k + 1, j + 1, i) - F(k, j - 1, i) - F(k + 1, j - 1, i)) * 0.25;
            const V3 &c3 = C.kcsi[f], &e3 = C.keta[f], &z3 = C.kzet[f];
            double a = C.kaj[f];
            C.ucont[f].z -= (dpdc * (c3.x * z3.x + c3.y * z3.y + c3.z * z3.z) * a
                           + dpde * (e3.x * z3.x + e3.y * z3.y + e3.z * z3.z) * a
                           + dpdz * (z3.x * z3.x + z3.y * z3.y + z3.z * z3.z) * a) * dt;
        }
    }
}

// SolvePEqn, peqn.c:3777-3971 (SetRHS, solve, phiToPhi, UpdatePhiBCs,
// UpdatePressure, UpdatePressureBCs, ProjectVelocity)
int solvePEqn(tg_ctx &C, tg_stats *st)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    std::vector<double> b(C.N);
    setRHS(C, b);
    // initial guess: previous solution with the mean removed (SubtractAverageHypre, peqn.c:1768-1853)
    double mean = 0.0;
    for (double v : C.phi1d) mean += v;
    mean /= (double)C.N;
    for (double &v : C.phi1d) v -= mean;
    int rc = solvePoisson(C, b, C.phi1d, st);
    // phiToPhi, peqn.c:1579-1636
    std::fill(C.phi.begin(), C.phi.end(), 0.0);
    int64_t pos = 0;
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) C.phi[C.I(k, j, i)] = C.phi1d[pos++];
    updateScalarGhosts(C, C.phi);
    // UpdatePressure, peqn.c:2909-2962
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) C.p[C.I(k, j, i)] += C.phi[C.I(k, j, i)];
    updateScalarGhosts(C, C.p);
    projectVelocity(C);
    return rc;
}

// ContinuityErrorsOptimized, peqn.c:4114-4181
double continuityError(const tg_ctx &C)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    double m = 0.0;
    #pragma omp parallel for collapse(2) reduction(max:m) schedule(static)
    for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
    for (int i = 1; i < mx - 1; i++) {
        size_t c = C.I(k, j, i);
        double d = std::fabs((C.ucont[c].x - C.ucont[C.I(k, j, i - 1)].x + C.ucont[c].y - C.ucont[C.I(k, j - 1, i)].y
                             + C.ucont[c].z - C.ucont[C.I(k - 1, j, i)].z) * C.aj[c]);
        if (d > m) m = d;
    }
    return m;
}

// SyncPressureAcrossDomains (single domain), overset.c:263-315
void syncPressure(tg_ctx &C)
{
    double ref = C.p[C.I(1, 1, 1)];
    for (double &v : C.p) v -= ref;
}

// one time step in main.c order (main.c:54-327)
int step(tg_ctx &C, tg_stats *st)
{
    C.ucont_o = C.ucont;                                 // main.c:81
    if (C.c.teqn) {                                      // main.c:83-99
        if (C.c.t_ddt_scheme == TG_TDDT_BDF2) C.tmprt_oo = C.tmprt_o.empty() ? std::vector<double>(C.G, 0.0) : C.tmprt_o;
        C.tmprt_o = C.tmprt;
    }
    if (C.c.les) { updateNut(C); updateWallModels(C); }  // main.c:112-117
    if (!C.farm.empty()) updateWindTurbines(C);          // main.c:144-147
    gradP(C);                                            // main.c:160-167
    if (C.c.buoyancy) {                                  // main.c:175-192
        if (C.it > C.c.it_start) C.btheta_o = C.btheta;
        if (C.c.p_tilde) ghGradRhoK(C); else buoyancy(C);   // main.c:176-181
    }
    const int urc = solveUEqn(C);                        // main.c:195
    int rc = solvePEqn(C, st);                           // main.c:198
    if (urc == 2) rc = 2;
    else if (rc != 2) rc |= urc;
    contravariantToCartesian(C);                         // main.c:201
    if (C.c.teqn) {                                      // main.c:194-205
        updateWallModelsT(C);                            // main.c:201
        const int trc = solveTEqn(C);
        if (trc == 2) rc = 2;
        else if (rc != 2) rc |= trc;
    }
    double md = continuityError(C);                      // main.c:227
    if (st) st->max_divergence = md;
    if (C.c.ddt_scheme == TG_DDT_CN) {                   // main.c:214-272: Rhs_o of the next step
        std::fill(C.rhs_o.begin(), C.rhs_o.end(), V3{0, 0, 0});
        formU(C, C.rhs_o, 1.0);
    }
    if (C.c.teqn) updateTemperatureBCs(C);               // main.c:274-278
    updateCartesianBCs(C);                               // main.c:281
    updateContravariantBCs(C);                           // main.c:284
    syncPressure(C);                                     // main.c:313
    C.it++;
    return rc;
}

void allocState(tg_ctx &C)
{
    const size_t G = C.G;
    for (auto *v : {&C.ucont, &C.ucont_o, &C.ucat, &C.rhs, &C.dp, &C.btheta, &C.btheta_o, &C.gcont, &C.utmp, &C.fp, &C.source, &C.ucont_adj, &C.ucat_adj, &C.source_adj,
                    &C.div1, &C.div2, &C.div3, &C.visc1, &C.visc2, &C.visc3}) zero(*v, G);
    for (auto *v : {&C.p, &C.phi, &C.nut, &C.tmprt, &C.p_adj, &C.tmprt_o}) zero(*v, G);
    zero(C.rhs_o, G);
    const size_t P = (size_t)C.mx * C.mz;
    for (auto *v : {&C.twx, &C.twy, &C.twz, &C.umean, &C.ufx, &C.ufy, &C.ufz, &C.wadj_x, &C.wadj_y, &C.wadj_m,
                    &C.twa_x, &C.twa_y, &C.twa_z, &C.qwall, &C.surf_theta}) zero(*v, P);
}

std::vector<V3> *vecField(tg_ctx &C, int w)
{
    switch (w) {
    case TG_F_CENT: return &C.cent;   case TG_F_CSI: return &C.csi;   case TG_F_ETA: return &C.eta;
    case TG_F_ZET: return &C.zet;     case TG_F_ICSI: return &C.icsi; case TG_F_IETA: return &C.ieta;
    case TG_F_IZET: return &C.izet;   case TG_F_JCSI: return &C.jcsi; case TG_F_JETA: return &C.jeta;
    case TG_F_JZET: return &C.jzet;   case TG_F_KCSI: return &C.kcsi; case TG_F_KETA: return &C.keta;
    case TG_F_KZET: return &C.kzet;   case TG_F_UCONT: return &C.ucont; case TG_F_UCAT: return &C.ucat;
    case TG_F_UCONT_O: return &C.ucont_o; case TG_F_RHS: return &C.rhs; case TG_F_DP: return &C.dp;
    case TG_F_BTHETA: return &C.btheta; case TG_F_SOURCE: return &C.source;
    case TG_F_UCONT_ADJ: return &C.ucont_adj; case TG_F_UCAT_ADJ: return &C.ucat_adj; case TG_F_SOURCE_ADJ: return &C.source_adj;
    case TG_F_FARM_FORCE: return C.farm.empty() ? nullptr : &C.farm_cat;
    case TG_F_FARM_CONT: return C.farm.empty() ? nullptr : &C.farm_cont;
    default: return nullptr;
    }
}
std::vector<double> *scalField(tg_ctx &C, int w)
{
    switch (w) {
    case TG_F_AJ: return &C.aj; case TG_F_IAJ: return &C.iaj; case TG_F_JAJ: return &C.jaj; case TG_F_KAJ: return &C.kaj;
    case TG_F_P: return &C.p; case TG_F_PHI: return &C.phi; case TG_F_NUT: return &C.nut; case TG_F_TMPRT: return &C.tmprt;
    case TG_F_P_ADJ: return &C.p_adj;
    default: return nullptr;
    }
}

tg_status fail(tg_ctx *C, tg_status s, const std::string &m) { if (C) C->err = m; return s; }

template <class F>
tg_status guarded(tg_ctx *C, F &&f)
{
    if (!C) return TG_ERR_BAD_ARG;
    try { return f(); }
    catch (const OracleError &e) { return fail(C, TG_ERR_STATE, e.what()); }
    catch (const std::bad_alloc &) { return fail(C, TG_ERR_ALLOC, "host allocation failed"); }
    catch (const std::exception &e) { return fail(C, TG_ERR_STATE, e.what()); }
}

// copy between a global-extent array and a caller array of extent +2*halo
template <int NC>
void copyIn(const tg_ctx &C, double *dst, const double *src, int halo)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const int lx = mx + 2 * halo, ly = my + 2 * halo;
    for (int k = 0; k < mz; k++) for (int j = 0; j < my; j++)
        std::memcpy(dst + (((size_t)k * my + j) * mx) * NC,
                    src + ((((size_t)(k + halo)) * ly + (j + halo)) * lx + halo) * NC, sizeof(double) * NC * mx);
}
template <int NC>
void copyOut(const tg_ctx &C, double *dst, const double *src, int halo)
{
    const int mx = C.mx, my = C.my, mz = C.mz;
    const int lx = mx + 2 * halo, ly = my + 2 * halo;
    for (int k = 0; k < mz; k++) for (int j = 0; j < my; j++)
        std::memcpy(dst + ((((size_t)(k + halo)) * ly + (j + halo)) * lx + halo) * NC,
                    src + (((size_t)k * my + j) * mx) * NC, sizeof(double) * NC * mx);
}

} // namespace

// ============================================================================
//  C-ABI (prefix tor_), same semantics as the tg_ entry points
// ============================================================================
#include "tosca_oracle_adjoint.inc"

extern "C" {

const char *tor_status_string(tg_status s)
{
    switch (s) {
    case TG_OK: return "ok"; case TG_ERR_CUDA: return "CUDA error"; case TG_ERR_BAD_ARG: return "bad argument";
    case TG_ERR_NOT_CONVERGED: return "pressure solve did not converge"; case TG_ERR_NAN: return "non-finite value";
    case TG_ERR_ALLOC: return "allocation failed"; case TG_ERR_STATE: return "invalid state";
    }
    return "unknown status";
}

const char *tor_last_error(const tg_ctx *C) { return C ? C->err.c_str() : "null context"; }

// a thetaWallFunction needs LES (UpdateWallModelsT returns without it and
// FormT applies qWall only with LES), one of the two types, and with -3 the
// positive constants its logarithms and divisions use; with the velocity
// wall function it also needs that one's thetaRef
static bool theta_wall_config_ok(const tg_config *cfg)
{
    if (!cfg->les) return false;
    if (cfg->t_wall_type == TG_TWALL_SHUMANN || cfg->t_wall_type == TG_TWALL_SURFACE_SERIES) {
        if (!(cfg->t_wall_kappa > 0) || !(cfg->t_wall_theta_ref > 0) || !(cfg->t_wall_roughness > 0) || !(cfg->t_wall_alpha_h > 0))
            return false;
        if (cfg->t_wall_localized != 0 && cfg->t_wall_localized != 1) return false;
    } else if (cfg->t_wall_type != TG_TWALL_FIXED_FLUX) return false;
    if (cfg->bc[TG_JLEFT] == TG_BC_WALL_SHUMANN && !(cfg->wall_theta_ref > 0)) return false;
    return true;
}

// inletFunction type 2 (inflow.c:65-72): a positive roughness and friction
// velocity, hInv above the roughness, a unit direction (the reference scales
// directionU to unit length as it reads it)
static bool inlet_log_config_ok(const tg_config *cfg)
{
    const double *d = cfg->inlet_dir;
    const double n = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    return cfg->inlet_z0 > 0 && cfg->inlet_u_tau >= 0 && cfg->inlet_h_inv > cfg->inlet_z0 && std::fabs(n - 1.0) < 1e-12;
}

tg_status tor_create(const tg_config *cfg, tg_ctx **out)
{
    if (!cfg || !out) return TG_ERR_BAD_ARG;
    *out = nullptr;
    if (cfg->mx < 6 || cfg->my < 6 || cfg->mz < 6) return TG_ERR_BAD_ARG;
    for (int p = 0; p < 6; p++) if (cfg->bc[p] < 0 || cfg->bc[p] > TG_BC_INLET_LOG) return TG_ERR_BAD_ARG;
    for (int p = 0; p < 6; p++)
        if (cfg->bc[p] >= TG_BC_FIXED_VALUE && cfg->ddt_scheme != TG_DDT_FE && cfg->ddt_scheme != TG_DDT_RK4) return TG_ERR_BAD_ARG;
    for (int p = 0; p < 6; p++)
        if (cfg->bc[p] == TG_BC_INLET_LOG && (p != TG_KLEFT || !inlet_log_config_ok(cfg))) return TG_ERR_BAD_ARG;
    for (int d = 0; d < 3; d++)
        if ((cfg->bc[2 * d] == TG_BC_PERIODIC) != (cfg->bc[2 * d + 1] == TG_BC_PERIODIC)) return TG_ERR_BAD_ARG;
    if (cfg->bc[TG_IRIGHT] == TG_BC_WALL_SHUMANN || cfg->bc[TG_ILEFT] == TG_BC_WALL_SHUMANN ||
        cfg->bc[TG_KRIGHT] == TG_BC_WALL_SHUMANN || cfg->bc[TG_KLEFT] == TG_BC_WALL_SHUMANN ||
        cfg->bc[TG_JRIGHT] == TG_BC_WALL_SHUMANN) return TG_ERR_BAD_ARG;
    if (cfg->dt <= 0 || cfg->ddt_scheme < 0 || cfg->ddt_scheme > TG_DDT_RK3SOCN) return TG_ERR_BAD_ARG;
    if (cfg->gmres_restart < 0 || cfg->gmres_restart > 60) return TG_ERR_BAD_ARG;
    if (cfg->p_tilde && !cfg->buoyancy) return TG_ERR_BAD_ARG;
    if (cfg->poisson_guess > 2 || cfg->poisson_guess < -1) return TG_ERR_BAD_ARG;   // the CUDA solver's initial guess; the oracle starts from 0
    if (cfg->teqn) {
        if (!(cfg->prandtl > 0) || (cfg->les && !(cfg->t_ref > 0))) return TG_ERR_BAD_ARG;
        if (cfg->t_ddt_scheme < TG_TDDT_RK4 || cfg->t_ddt_scheme > TG_TDDT_BDF2) return TG_ERR_BAD_ARG;
        if (cfg->t_gmres_restart < 0 || cfg->t_gmres_restart > 60) return TG_ERR_BAD_ARG;
        for (int p = 0; p < 6; p++) {
            if (cfg->t_bc[p] < 0 || cfg->t_bc[p] > TG_TBC_WALL_FUNCTION) return TG_ERR_BAD_ARG;
            if (cfg->t_bc[p] == TG_TBC_WALL_FUNCTION && p != TG_JLEFT) return TG_ERR_BAD_ARG;
            if ((cfg->t_bc[p] == TG_TBC_PERIODIC) != (cfg->bc[p] == TG_BC_PERIODIC)) return TG_ERR_BAD_ARG;
        }
        if (cfg->t_bc[TG_JLEFT] == TG_TBC_WALL_FUNCTION && !theta_wall_config_ok(cfg)) return TG_ERR_BAD_ARG;
    }
    tg_ctx *C = new (std::nothrow) tg_ctx();
    if (!C) return TG_ERR_ALLOC;
    C->c = *cfg;
    C->mx = cfg->mx; C->my = cfg->my; C->mz = cfg->mz;
    C->pi = cfg->bc[TG_ILEFT] == TG_BC_PERIODIC;
    C->pj = cfg->bc[TG_JLEFT] == TG_BC_PERIODIC;
    C->pk = cfg->bc[TG_KLEFT] == TG_BC_PERIODIC;
    C->G = (size_t)cfg->mx * cfg->my * cfg->mz;
    C->it = cfg->it_start;
    try { allocState(*C); zero(C->coor, C->G); }
    catch (...) { delete C; return TG_ERR_ALLOC; }
    *out = C;
    return TG_OK;
}

tg_status tor_destroy(tg_ctx *C) { delete C; return TG_OK; }

tg_status tor_set_mesh_nodes(tg_ctx *C, const double *nodes)
{
    return guarded(C, [&]() -> tg_status {
        if (!nodes) return fail(C, TG_ERR_BAD_ARG, "null nodes");
        std::memcpy(C->coor.data(), nodes, sizeof(V3) * C->G);
        // the last DMDA point of each direction carries no node (mesh.c:92-94)
        for (int k = 0; k < C->mz; k++) for (int j = 0; j < C->my; j++) for (int i = 0; i < C->mx; i++)
            if (i == C->mx - 1 || j == C->my - 1 || k == C->mz - 1) C->coor[((size_t)k * C->my + j) * C->mx + i] = V3{0, 0, 0};
        setMeshMetrics(*C);
        // mesh->grndLevel: the lowest node (mesh.c:2014-2063)
        C->grnd = 1e30;
        for (int k = 0; k < C->mz - 1; k++) for (int j = 0; j < C->my - 1; j++) for (int i = 0; i < C->mx - 1; i++)
            C->grnd = std::min(C->grnd, C->coor[((size_t)k * C->my + j) * C->mx + i].z);
        setPoissonConnectivity(*C);
        setCoeffMatrix(*C);
        C->phi1d.assign(C->N, 0.0);
        C->has_mesh = true;
        return TG_OK;
    });
}

tg_status tor_set_field(tg_ctx *C, int32_t w, const double *host, int32_t halo)
{
    return guarded(C, [&]() -> tg_status {
        if (!host || halo < 0) return fail(C, TG_ERR_BAD_ARG, "bad field argument");
        if (w == TG_F_WALL_ADJ) {
            for (size_t q = 0; q < (size_t)C->mx * C->mz; q++) { C->wadj_x[q] = host[3 * q]; C->wadj_y[q] = host[3 * q + 1]; C->wadj_m[q] = host[3 * q + 2]; }
            return TG_OK;
        }
        if (w == TG_F_QWALL || w == TG_F_SURF_THETA) {
            std::vector<double> &d = w == TG_F_QWALL ? C->qwall : C->surf_theta;
            std::memcpy(d.data(), host, sizeof(double) * d.size());
            if (w == TG_F_SURF_THETA) C->surf_set = true;
            return TG_OK;
        }
        if (auto *v = vecField(*C, w)) { copyIn<3>(*C, (double *)v->data(), host, halo); return TG_OK; }
        if (auto *s = scalField(*C, w)) { copyIn<1>(*C, s->data(), host, halo); return TG_OK; }
        return fail(C, TG_ERR_BAD_ARG, "field not settable");
    });
}

tg_status tor_get_field(tg_ctx *C, int32_t w, double *host, int32_t halo)
{
    return guarded(C, [&]() -> tg_status {
        if (!host || halo < 0) return fail(C, TG_ERR_BAD_ARG, "bad field argument");
        if (w == TG_F_TAUWALL) {
            // plane (mz x mx) of the j-left wall stress
            for (size_t q = 0; q < (size_t)C->mx * C->mz; q++) { host[3 * q] = C->twx[q]; host[3 * q + 1] = C->twy[q]; host[3 * q + 2] = C->twz[q]; }
            return TG_OK;
        }
        if (w == TG_F_WALL_ADJ) {
            for (size_t q = 0; q < (size_t)C->mx * C->mz; q++) { host[3 * q] = C->wadj_x[q]; host[3 * q + 1] = C->wadj_y[q]; host[3 * q + 2] = C->wadj_m[q]; }
            return TG_OK;
        }
        if (w == TG_F_QWALL || w == TG_F_SURF_THETA) {
            const std::vector<double> &d = w == TG_F_QWALL ? C->qwall : C->surf_theta;
            std::memcpy(host, d.data(), sizeof(double) * d.size());
            return TG_OK;
        }
        if (auto *v = vecField(*C, w)) { copyOut<3>(*C, host, (const double *)v->data(), halo); return TG_OK; }
        if (auto *s = scalField(*C, w)) { copyOut<1>(*C, host, s->data(), halo); return TG_OK; }
        return fail(C, TG_ERR_BAD_ARG, "unknown field");
    });
}

// PETSc binary VecView / VecLoad of a DMDA vector (readFields / writeFields,
// io.c:247-420, 2261): big-endian class id 1211214 and entry count (64-bit,
// or 32-bit when reading), then big-endian doubles in natural order
tg_status tor_write_field_petsc(tg_ctx *C, int32_t w, const char *path)
{
    return guarded(C, [&]() -> tg_status {
        size_t dof = vecField(*C, w) ? 3 : (scalField(*C, w) ? 1 : 0);
        if (!path || !dof || w == TG_F_TAUWALL) return fail(C, TG_ERR_BAD_ARG, "bad field or path");
        std::vector<double> h(C->G * dof);
        tg_status s = tor_get_field(C, w, h.data(), 0);
        if (s != TG_OK) return s;
        std::vector<unsigned char> out(16 + 8 * h.size());
        auto put = [&](size_t at, uint64_t v) { for (int b = 0; b < 8; b++) out[at + b] = (unsigned char)(v >> (56 - 8 * b)); };
        put(0, 1211214);
        put(8, (uint64_t)h.size());
        for (size_t q = 0; q < h.size(); q++) { uint64_t u; std::memcpy(&u, &h[q], 8); put(16 + 8 * q, u); }
        FILE *f = std::fopen(path, "wb");
        if (!f) return fail(C, TG_ERR_BAD_ARG, "cannot open file");
        bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
        ok = std::fclose(f) == 0 && ok;
        return ok ? TG_OK : fail(C, TG_ERR_BAD_ARG, "write failed");
    });
}
tg_status tor_read_field_petsc(tg_ctx *C, int32_t w, const char *path)
{
    return guarded(C, [&]() -> tg_status {
        size_t dof = vecField(*C, w) ? 3 : (scalField(*C, w) ? 1 : 0);
        if (!path || !dof || w == TG_F_TAUWALL) return fail(C, TG_ERR_BAD_ARG, "bad field or path");
        FILE *f = std::fopen(path, "rb");
        if (!f) return fail(C, TG_ERR_BAD_ARG, "cannot open file");
        std::vector<unsigned char> buf;
        unsigned char tmp[65536];
        size_t got;
        while ((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
        std::fclose(f);
        auto get = [&](size_t at, int nb) { uint64_t v = 0; for (int b = 0; b < nb; b++) v = (v << 8) | buf[at + b]; return v; };
        const size_t n = C->G * dof;
        size_t off;
        if (buf.size() >= 8 && get(0, 4) == 1211214) off = 8;                   // 32-bit integers
        else if (buf.size() >= 16 && get(0, 8) == 1211214) off = 16;            // 64-bit integers
        else return fail(C, TG_ERR_BAD_ARG, "not a PETSc vector file");
        if ((off == 8 ? get(4, 4) : get(8, 8)) != n || buf.size() != off + 8 * n) return fail(C, TG_ERR_BAD_ARG, "entry count mismatch");
        std::vector<double> h(n);
        for (size_t q = 0; q < n; q++) { uint64_t u = get(off + 8 * q, 8); std::memcpy(&h[q], &u, 8); }
        return tor_set_field(C, w, h.data(), 0);
    });
}

tg_status tor_init_from_cartesian(tg_ctx *C, const double *ucat, int32_t halo)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        std::vector<V3> in(C->G);
        copyIn<3>(*C, (double *)in.data(), ucat, halo);
        const int mx = C->mx, my = C->my, mz = C->mz;
        // SetTaylorGreenFieldU tail, initialField.c:1100-1204
        for (int k = 1; k < mz - 1; k++) for (int j = 1; j < my - 1; j++) for (int i = 1; i < mx - 1; i++)
            C->ucat[C->I(k, j, i)] = in[C->I(k, j, i)];
        if (C->c.teqn) updateTemperatureBCs(*C);
        updateCartesianBCs(*C);
        auto &U = C->ucat;
        for (int k = 1; k < mz - 1; k++) for (int j = 1; j < my - 1; j++) for (int i = 0; i < mx - 1; i++) {
            size_t f = C->I(k, j, i); const V3 &a = U[f], &b = U[C->I(k, j, i + 1)]; const V3 &s = C->icsi[f];
            V3 uf = mk(0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z));
            C->ucont[f].x = uf.x * s.x + uf.y * s.y + uf.z * s.z;
        }
        for (int k = 1; k < mz - 1; k++) for (int j = 0; j < my - 1; j++) for (int i = 1; i < mx - 1; i++) {
            size_t f = C->I(k, j, i); const V3 &a = U[f], &b = U[C->I(k, j + 1, i)]; const V3 &s = C->jeta[f];
            V3 uf = mk(0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z));
            C->ucont[f].y = uf.x * s.x + uf.y * s.y + uf.z * s.z;
        }
        for (int k = 0; k < mz - 1; k++) for (int j = 1; j < my - 1; j++) for (int i = 1; i < mx - 1; i++) {
            size_t f = C->I(k, j, i); const V3 &a = U[f], &b = U[C->I(k + 1, j, i)]; const V3 &s = C->kzet[f];
            V3 uf = mk(0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z));
            C->ucont[f].z = uf.x * s.x + uf.y * s.y + uf.z * s.z;
        }
        updateContravariantBCs(*C);
        return TG_OK;
    });
}

#define TOR_STAGE(name, body) \
    tg_status name(tg_ctx *C) { return guarded(C, [&]() -> tg_status { if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set"); body; return TG_OK; }); }

TOR_STAGE(tor_contravariant_to_cartesian, contravariantToCartesian(*C); resetCellPeriodic(*C, C->ucat))
TOR_STAGE(tor_update_nut, updateNut(*C))
TOR_STAGE(tor_update_wall_models, updateWallModels(*C))
TOR_STAGE(tor_grad_p, gradP(*C))
TOR_STAGE(tor_buoyancy, (C->c.p_tilde ? ghGradRhoK(*C) : buoyancy(*C)))
TOR_STAGE(tor_explicit_rhs, explicitRhsU(*C))
TOR_STAGE(tor_solve_u, solveUEqn(*C))
TOR_STAGE(tor_update_cartesian_bcs, updateCartesianBCs(*C))
TOR_STAGE(tor_update_contravariant_bcs, updateContravariantBCs(*C))
TOR_STAGE(tor_sync_pressure, syncPressure(*C))
TOR_STAGE(tor_update_wall_models_t,
          if (!C->c.teqn) return fail(C, TG_ERR_STATE, "temperature equation off"); updateWallModelsT(*C))
TOR_STAGE(tor_update_temperature_bcs,
          if (!C->c.teqn) return fail(C, TG_ERR_STATE, "temperature equation off"); updateTemperatureBCs(*C))

tg_status tor_set_surface_temperature(tg_ctx *C, int32_t n, const double *time, const double *temp)
{
    return guarded(C, [&]() -> tg_status {
        if (n < 2 || !time || !temp) return fail(C, TG_ERR_BAD_ARG, "a surface temperature series needs n >= 2 points");
        C->surf_series_t.assign(time, time + n);
        C->surf_series_v.assign(temp, temp + n);
        return TG_OK;
    });
}

// the Monin-Obukhov functions of the restatement, for comparison with the reference's
double tor_mo_ustar(double U, double dist, double z0, double gammaM, double kappa, double qwall, double thetaRef)
{
    try { return uStarShumann(U, dist, z0, gammaM, kappa, qwall, thetaRef); }
    catch (...) { return std::nan(""); }
}
double tor_mo_qwall(double U, double dist, double z0, double gammaM, double gammaH, double alphaH, double thetaRef,
                    double deltaTheta, double kappa)
{
    try { return qWallShumann(U, dist, z0, gammaM, gammaH, alphaH, thetaRef, deltaTheta, kappa); }
    catch (...) { return std::nan(""); }
}

tg_status tor_form_u(tg_ctx *C, double scale, int32_t zero_rhs)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        if (zero_rhs) std::fill(C->rhs.begin(), C->rhs.end(), V3{0, 0, 0});
        formU(*C, C->rhs, scale);
        return TG_OK;
    });
}

tg_status tor_solve_p(tg_ctx *C, tg_stats *st)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        tg_stats local{};
        int rc = solvePEqn(*C, st ? st : &local);
        return rc ? fail(C, TG_ERR_NOT_CONVERGED, "pressure solve reached its iteration cap") : TG_OK;
    });
}

tg_status tor_continuity_error(tg_ctx *C, double *md)
{
    return guarded(C, [&]() -> tg_status {
        if (!md) return fail(C, TG_ERR_BAD_ARG, "null output");
        *md = continuityError(*C);
        return TG_OK;
    });
}

tg_status tor_step(tg_ctx *C, int32_t nsteps, tg_stats *st)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        tg_stats local{};
        tg_stats *s = st ? st : &local;
        *s = tg_stats{};
        auto t0 = std::chrono::steady_clock::now();
        int rc = 0;
        for (int n = 0; n < nsteps; n++) { rc |= step(*C, s); s->steps++; }
        s->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        for (const V3 &v : C->ucont) if (!std::isfinite(v.x) || !std::isfinite(v.y) || !std::isfinite(v.z))
            return fail(C, TG_ERR_NAN, "non-finite contravariant flux");
        return rc ? fail(C, TG_ERR_NOT_CONVERGED, "pressure solve reached its iteration cap") : TG_OK;
    });
}

tg_status tor_momentum_info(tg_ctx *C, int32_t *outer, int32_t *inner, double *residual)
{
    if (!C || !outer || !inner || !residual) return TG_ERR_BAD_ARG;
    *outer = C->mom_outer;
    *inner = C->mom_inner;
    *residual = C->mom_res;
    return TG_OK;
}

tg_status tor_step_host(tg_ctx *C, double *ucont, double *ucat, double *p, double *nut, int32_t halo, tg_stats *st)
{
    return guarded(C, [&]() -> tg_status {
        if (!ucont || !ucat || !p) return fail(C, TG_ERR_BAD_ARG, "null state");
        copyIn<3>(*C, (double *)C->ucont.data(), ucont, halo);
        copyIn<3>(*C, (double *)C->ucat.data(), ucat, halo);
        copyIn<1>(*C, C->p.data(), p, halo);
        // nut is recomputed from Ucat before any read (updateNut): output only
        tg_status s = tor_step(C, 1, st);
        copyOut<3>(*C, ucont, (const double *)C->ucont.data(), halo);
        copyOut<3>(*C, ucat, (const double *)C->ucat.data(), halo);
        copyOut<1>(*C, p, C->p.data(), halo);
        if (nut && C->c.les) copyOut<1>(*C, nut, C->nut.data(), halo);
        return s;
    });
}

// number of unknowns and the assembled matrix, for tests
int64_t tor_poisson_size(tg_ctx *C) { return C ? C->N : -1; }
int64_t tor_poisson_nnz(tg_ctx *C) { return C ? (int64_t)C->A.val.size() : -1; }
tg_status tor_poisson_matrix(tg_ctx *C, int64_t *rowptr, int64_t *col, double *val)
{
    if (!C) return TG_ERR_BAD_ARG;
    std::memcpy(rowptr, C->A.rowptr.data(), sizeof(int64_t) * (C->N + 1));
    std::memcpy(col, C->A.col.data(), sizeof(int64_t) * C->A.col.size());
    std::memcpy(val, C->A.val.data(), sizeof(double) * C->A.val.size());
    return TG_OK;
}
int32_t tor_poisson_symmetric(tg_ctx *C) { return C ? (C->symmetric ? 1 : 0) : -1; }
int32_t tor_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// wind farm (tosca_oracle_farm.inc)
tg_status tor_set_turbines(tg_ctx *C, int32_t n, const tg_turbine *tb, double rho)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        if (n < 0 || (n > 0 && !tb) || !(rho > 0)) return fail(C, TG_ERR_BAD_ARG, "bad turbine arguments");
        for (int t = 0; t < n; t++)
            if (tb[t].n_radial < 2 || tb[t].n_azimuth < 1 || !(tb[t].r_tip > tb[t].r_hub) || !(tb[t].r_hub > 0) || !(tb[t].epsilon > 0))
                return fail(C, TG_ERR_BAD_ARG, "bad turbine description");
        setTurbines(*C, n, tb, rho);
        return TG_OK;
    });
}
tg_status tor_set_turbine_ct(tg_ctx *C, const double *ct)
{
    return guarded(C, [&]() -> tg_status {
        if (C->farm.empty()) return fail(C, TG_ERR_STATE, "no turbines");
        for (size_t t = 0; t < C->farm.size(); t++) C->farm[t].Ct = ct[t];
        return TG_OK;
    });
}
tg_status tor_turbine_state(tg_ctx *C, double *uref, double *thrust, double *power, double *power_sum, int32_t reset)
{
    return guarded(C, [&]() -> tg_status {
        if (C->farm.empty()) return fail(C, TG_ERR_STATE, "no turbines");
        for (size_t t = 0; t < C->farm.size(); t++) {
            if (uref) uref[t] = C->farm[t].rtrAvgMagU;
            if (thrust) thrust[t] = C->farm[t].rtrThrust;
            if (power) power[t] = C->farm[t].aeroPwr;
        }
        if (power_sum) *power_sum = C->farm_power_sum;
        if (reset) C->farm_power_sum = 0.0;
        return TG_OK;
    });
}
tg_status tor_set_farm_objective(tg_ctx *C, int32_t on)
{
    return guarded(C, [&]() -> tg_status {
        if (C->farm.empty()) return fail(C, TG_ERR_STATE, "no turbines");
        C->farm_objective = on != 0;
        return TG_OK;
    });
}
tg_status tor_ct_gradient(tg_ctx *C, double *grad, int32_t reset)
{
    return guarded(C, [&]() -> tg_status {
        if (C->farm.empty()) return fail(C, TG_ERR_STATE, "no turbines");
        for (size_t t = 0; t < C->farm.size(); t++) {
            if (grad) grad[t] = C->ct_grad[t];
            if (reset) C->ct_grad[t] = 0.0;
        }
        return TG_OK;
    });
}

// Discrete adjoint of one step (test infrastructure, see tosca_oracle_adjoint.inc).
// The context holds the state at the start of the step and the adjoint fields
// the adjoints of the state after it; on return the adjoint fields hold the
// adjoints of the state before the step, TG_F_SOURCE_ADJ has the step's
// contribution added, and the state is again the one at the start of the step.
tg_status tor_adjoint_step(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        if (C->c.teqn) return fail(C, TG_ERR_BAD_ARG, "the adjoint of the temperature equation is not implemented");
        if (C->c.ddt_scheme == TG_DDT_CN) return fail(C, TG_ERR_BAD_ARG, "the adjoint of the Crank-Nicolson scheme is not implemented");
        if (C->c.ddt_scheme >= TG_DDT_ABCN) return fail(C, TG_ERR_BAD_ARG, "the adjoint of the IMEX schemes is not implemented");
        for (int q = 0; q < 6; q++)
            if (C->c.bc[q] >= TG_BC_FIXED_VALUE)
                return fail(C, TG_ERR_BAD_ARG, "the adjoint of the inflow/outflow patches is not implemented");
        // state saved around the taped forward step
        auto ucont = C->ucont, ucat = C->ucat, btheta = C->btheta, btheta_o = C->btheta_o;
        auto p = C->p, phi = C->phi, phi1d = C->phi1d, nut = C->nut;
        auto umean = C->umean, ufx = C->ufx, ufy = C->ufy, ufz = C->ufz, twx = C->twx, twy = C->twy, twz = C->twz;
        const bool ufilt_set = C->ufilt_set;
        int it = C->it;
        AdjTape T;
        tg_stats st{};
        stepTaped(*C, &st, T);
        C->ucont = ucont; C->ucat = ucat; C->btheta = btheta; C->btheta_o = btheta_o;
        C->p = p; C->phi = phi; C->phi1d = phi1d; C->nut = nut; C->it = it;
        C->umean = umean; C->ufx = ufx; C->ufy = ufy; C->ufz = ufz; C->twx = twx; C->twy = twy; C->twz = twz;
        C->ufilt_set = ufilt_set;
        adjointStep(*C, T);
        return TG_OK;
    });
}

} // extern "C"
