// TEST INFRASTRUCTURE ONLY: the reference's own stage functions (TOSCA's
// ueqn.c, solvers/ueqn_solvers.c, sources/ueqn_sources.c, peqn.c, les.c,
// boundary.c, wallfunctions.c, mesh.c, overset.c, compiled unmodified from
// their source files against the single-rank stand-ins of petsc_stub.h),
// driven through the C-ABI of include/tosca_gpu.h with the prefix "ref_" so
// that the parity tests can compare the oracle restatement with them stage by
// stage and step by step.
//
// The harness builds TOSCA's structures the way its set-up code would for one
// rank (SetDistributedArrays, mesh.c:34-447; InitializeUEqn, ueqn.c:27-393;
// InitializePEqn, peqn.c:35-103; InitializeLES, les.c:20-150; InitializeTEqn,
// teqn.c:19-257; SetWallModels, boundary.c:4640-5200), with the values a
// control.dat and boundary/ files would hold, and then calls the reference's
// functions. Supported: periodic, slip, noSlip, fixedValue, zeroGradient, the kLeft
// log-law inletFunction (type 2) and the Schumann velocity wall
// function (-3, averaged u*) on jLeft; central and QUICK convection; FE and
// RK4; no LES or Smagorinsky (TOSCA's hard-coded Cs^2 = 0.0289,
// les.c:10,175); the mean pressure gradient; the potential temperature
// (teqn.c, solvers/teqn_solvers.c) with RK4, Boussinesq buoyancy or the
// p-tilde form, zeroGradient / fixedValue / fixedGradient / periodic
// patches and the jLeft thetaWallFunction (-2, -3). The HYPRE solve inside
// SolvePEqn is replaced by a tight solve of the captured matrix
// (petsc_stub.cpp).
#include "include/base.h"
#include "include/domain.h"
#include "include/io.h"
#include "include/inline.h"
#include "include/wallfunctions.h"

#include <memory>
#include <stdexcept>

#include "tgref_capture.h"
#include "tosca_gpu.h"

// SyncPressureAcrossDomains is defined in overset.c (overset.c:263-315)
PetscErrorCode SyncPressureAcrossDomains(domain_ *domain);

namespace {

const double TOSCA_STD_CS = 0.0289;   // les.c:10, used by UpdateCs for Smagorinsky (les.c:171-176)

_p_DM make_dm(const tg_config &c, PetscInt dof)
{
    _p_DM d;
    d.M = c.mx; d.N = c.my; d.P = c.mz;
    d.dof = dof;
    d.s = 3;                                                         // stencil width (mesh.c:42)
    // DM_BOUNDARY_GHOSTED unless periodic (mesh.c:136-142)
    d.bx = c.bc[0] == TG_BC_PERIODIC ? DM_BOUNDARY_PERIODIC : DM_BOUNDARY_GHOSTED;
    d.by = c.bc[2] == TG_BC_PERIODIC ? DM_BOUNDARY_PERIODIC : DM_BOUNDARY_GHOSTED;
    d.bz = c.bc[4] == TG_BC_PERIODIC ? DM_BOUNDARY_PERIODIC : DM_BOUNDARY_GHOSTED;
    return d;
}

const char *u_bc_name(int t)
{
    switch (t) {
    case TG_BC_PERIODIC: return "periodic";
    case TG_BC_NOSLIP: return "noSlip";
    case TG_BC_SLIP: return "slip";
    case TG_BC_WALL_SHUMANN: return "velocityWallFunction";
    case TG_BC_FIXED_VALUE: return "fixedValue";
    case TG_BC_ZERO_GRADIENT: return "zeroGradient";
    case TG_BC_INLET_LOG: return "inletFunction";
    default: return "";
    }
}
const char *nut_bc_name(int t)
{
    switch (t) {
    case TG_NUTBC_PERIODIC: return "periodic";
    case TG_NUTBC_ZEROGRADIENT: return "zeroGradient";
    case TG_NUTBC_FIXEDVALUE: return "fixedValue";
    default: return "";
    }
}

// the wall-model patch arrays of SetWallModels (boundary.c:4832-4870), mz x mx
wallModel *make_shumann(const tg_config &c)
{
    wallModel *w = new wallModel();
    w->uFiltSet = 0;
    PetscReal **arrs[7];
    const PetscInt mz = c.mz, mx = c.mx;
    for (PetscReal **&a : arrs) {
        a = new PetscReal *[mz];
        for (PetscInt k = 0; k < mz; k++) a[k] = new PetscReal[mx]();
    }
    w->tauWall.x = arrs[0]; w->tauWall.y = arrs[1]; w->tauWall.z = arrs[2];
    w->uMeanMag = arrs[3];
    w->uFilt.x = arrs[4]; w->uFilt.y = arrs[5]; w->uFilt.z = arrs[6];
    Shumann *s = new Shumann();
    s->wfEvalType = "averaged";                 // plane-averaged friction velocity
    s->kappa = c.wall_kappa;
    s->thetaRef = c.wall_theta_ref;             // these two enter only stratified (qWall != 0) evaluations
    s->roughness = c.wall_roughness;
    s->gammaM = c.wall_gamma_m;
    w->wmShumann = s;
    return w;
}

const char *t_bc_name(int t)
{
    switch (t) {
    case TG_TBC_ZERO_GRADIENT: return "zeroGradient";
    case TG_TBC_FIXED_VALUE: return "fixedValue";
    case TG_TBC_FIXED_GRADIENT: return "fixedGradient";
    case TG_TBC_PERIODIC: return "periodic";
    case TG_TBC_WALL_FUNCTION: return "thetaWallFunction";
    default: return "";
    }
}

// the jLeft thetaWallFunction of SetWallModels (boundary.c:5110-5160): the
// qWall patch field (zero), the Shumann constants, tLast = -1, surfaceTheta unset
wallModel *make_theta_wall(const tg_config &c)
{
    wallModel *w = new wallModel();
    const PetscInt mz = c.mz, mx = c.mx;
    PetscReal **q[3];
    for (PetscReal **&a : q) {
        a = new PetscReal *[mz];
        for (PetscInt k = 0; k < mz; k++) a[k] = new PetscReal[mx]();
    }
    w->qWall.x = q[0]; w->qWall.y = q[1]; w->qWall.z = q[2];
    Shumann *s = new Shumann();
    if (c.t_wall_type == TG_TWALL_SHUMANN || c.t_wall_type == TG_TWALL_SURFACE_SERIES) {
        s->wfEvalType = c.t_wall_localized ? "localized" : "averaged";
        s->kappa = c.t_wall_kappa;
        s->thetaRef = c.t_wall_theta_ref;
        s->roughness = c.t_wall_roughness;
        s->gammaM = c.t_wall_gamma_m;
        s->gammaH = c.t_wall_gamma_h;
        s->alphaH = c.t_wall_alpha_h;
        s->heatingRate = c.t_wall_heating_rate;
        s->tLast = -1.0;
        s->surfaceThetaSet = 0;
        s->numT = 0;                 // -4: the series comes from ref_set_surface_temperature
    } else {
        s->qWall = c.t_wall_qwall;
    }
    w->wmShumann = s;
    return w;
}

}  // namespace

struct tg_ctx {
    tg_config cfg{};
    std::string err;
    bool has_mesh = false;
    _p_DM da{}, fda{}, sda{}, tda{};
    PetscInt domainID = 0;
    std::unique_ptr<domain_> dom;
    clock_ clock{};
    io_ *io = nullptr;
    std::unique_ptr<inletFunctionTypes> inlet;
    mesh_ mesh{};
    ueqn_ ueqn{};
    peqn_ peqn{};
    les_ les{};
    teqn_ teqn{};
    double last_div = 0.0;
};

namespace {

tg_status fail(tg_ctx *C, tg_status s, const std::string &m)
{
    if (C) C->err = m;
    return s;
}

template <class F>
tg_status guarded(tg_ctx *C, F &&f)
{
    if (!C) return TG_ERR_BAD_ARG;
    try { return f(); }
    catch (const std::exception &e) { return fail(C, TG_ERR_STATE, e.what()); }
}

void build(tg_ctx &X)
{
    const tg_config &c = X.cfg;
    X.da = make_dm(c, 1);
    X.fda = make_dm(c, 3);
    X.sda = make_dm(c, 6);
    X.tda = make_dm(c, 9);
    X.da.cdm = &X.fda;

    X.dom.reset(new domain_());
    domain_ &d = *X.dom;
    d.info.nDomains = 1;
    d.info.periodic = 0;
    d.constants.nu = c.nu;
    d.constants.rho = 1.0;
    d.constants.tRef = c.t_ref;
    d.constants.Pr = c.prandtl;
    d.domainID = 0;
    d.clock = &X.clock;
    d.mesh = &X.mesh;
    X.io = new io_();
    d.io = X.io;
    d.ueqn = &X.ueqn;
    d.peqn = &X.peqn;
    d.les = &X.les;
    d.teqn = nullptr;

    flags_ &f = d.flags;
    f = flags_{};
    f.isLesActive = c.les ? 1 : 0;
    f.isMeanGradPForcingActive = c.mean_grad_p ? 1 : 0;

    access_ &a = d.access;
    a.clock = &X.clock;
    a.info = &d.info;
    a.constants = &d.constants;
    a.flags = &d.flags;
    a.mesh = &X.mesh;
    a.io = X.io;
    a.ueqn = &X.ueqn;
    a.peqn = &X.peqn;
    a.teqn = nullptr;
    a.les = &X.les;
    a.domainID = &X.domainID;

    X.clock.dt = c.dt;
    X.clock.startDt = c.dt;
    X.clock.dtOld = c.dt;
    X.clock.itStart = c.it_start;
    X.clock.it = c.it_start;
    X.clock.startTime = c.t_start;
    X.clock.time = c.t_start;

    // ---- mesh (SetDistributedArrays, mesh.c:34-447)
    mesh_ &m = X.mesh;
    m.meshName = ".";
    m.meshFileType = c.curvilinear ? "curvilinear" : "cartesian";
    m.IM = c.mx - 1; m.JM = c.my - 1; m.KM = c.mz - 1;
    m.da = &X.da; m.fda = &X.fda; m.sda = &X.sda; m.tda = &X.tda;
    DMDAGetLocalInfo(m.da, &m.info);
    // periodic type 2 (ghosted periodicity, the DM_BOUNDARY_PERIODIC of mesh.c:139-141)
    m.ii_periodic = c.bc[0] == TG_BC_PERIODIC; m.i_periodic = 0;
    m.jj_periodic = c.bc[2] == TG_BC_PERIODIC; m.j_periodic = 0;
    m.kk_periodic = c.bc[4] == TG_BC_PERIODIC; m.k_periodic = 0;
    // the count of periodic directions (SetPeriodicConnectivity, boundary.c:604-607)
    d.info.periodic = m.kk_periodic + m.k_periodic + m.jj_periodic + m.j_periodic + m.ii_periodic + m.i_periodic;
    m.MESH_COMM = PETSC_COMM_WORLD;
    m.access = &a;
    DMCreateGlobalVector(m.fda, &m.Cent);
    DMCreateLocalVector(m.fda, &m.lCent);
    for (Vec *v : {&m.lCsi, &m.lEta, &m.lZet, &m.lICsi, &m.lIEta, &m.lIZet, &m.lJCsi, &m.lJEta, &m.lJZet,
                   &m.lKCsi, &m.lKEta, &m.lKZet})
        VecDuplicate(m.lCent, v);
    VecDuplicate(m.Cent, &m.fluxLimiter);
    DMCreateGlobalVector(m.da, &m.Nvert);
    DMCreateLocalVector(m.da, &m.lAj);
    for (Vec *v : {&m.lIAj, &m.lJAj, &m.lKAj, &m.lNvert, &m.lNvert_o}) VecDuplicate(m.lAj, v);
    VecDuplicate(m.Nvert, &m.Nvert_o);
    VecDuplicate(m.Nvert, &m.meshTag);
    VecDuplicate(m.lNvert, &m.lmeshTag);

    // boundary conditions (SetBoundaryConditions / readVectorBC / readScalarBC)
    auto setU = [&](word &w, int t) { w = u_bc_name(t); };
    setU(m.boundaryU.iLeft, c.bc[0]); setU(m.boundaryU.iRight, c.bc[1]);
    setU(m.boundaryU.jLeft, c.bc[2]); setU(m.boundaryU.jRight, c.bc[3]);
    setU(m.boundaryU.kLeft, c.bc[4]); setU(m.boundaryU.kRight, c.bc[5]);
    {
        Cmpnts *vals[6] = {&m.boundaryU.iLval, &m.boundaryU.iRval, &m.boundaryU.jLval, &m.boundaryU.jRval,
                           &m.boundaryU.kLval, &m.boundaryU.kRval};
        for (int q = 0; q < 6; q++) {
            vals[q]->x = c.bc_value[3 * q]; vals[q]->y = c.bc_value[3 * q + 1]; vals[q]->z = c.bc_value[3 * q + 2];
        }
    }
    // inletFunction type 2 on kLeft (boundary/U inletFunction dictionary, inflow.c:65-72)
    if (c.bc[4] == TG_BC_INLET_LOG) {
        X.inlet.reset(new inletFunctionTypes());
        inletFunctionTypes &f = *X.inlet;
        f.typeU = 2;
        f.Udir.x = c.inlet_dir[0]; f.Udir.y = c.inlet_dir[1]; f.Udir.z = c.inlet_dir[2];
        f.hInv = c.inlet_h_inv; f.uTau = c.inlet_u_tau; f.roughness = c.inlet_z0;
        m.inletF.kLeft = X.inlet.get();
    }
    m.boundaryU.jLWF = c.bc[2] == TG_BC_WALL_SHUMANN ? -3 : 0;
    m.boundaryU.jRWF = c.bc[3] == TG_BC_WALL_SHUMANN ? -3 : 0;
    auto setS = [&](word &w, PetscReal &val, int t, double v) { w = nut_bc_name(t); val = v; };
    setS(m.boundaryNut.iLeft, m.boundaryNut.iLval, c.nut_bc[0], c.nut_bc_value[0]);
    setS(m.boundaryNut.iRight, m.boundaryNut.iRval, c.nut_bc[1], c.nut_bc_value[1]);
    setS(m.boundaryNut.jLeft, m.boundaryNut.jLval, c.nut_bc[2], c.nut_bc_value[2]);
    setS(m.boundaryNut.jRight, m.boundaryNut.jRval, c.nut_bc[3], c.nut_bc_value[3]);
    setS(m.boundaryNut.kLeft, m.boundaryNut.kLval, c.nut_bc[4], c.nut_bc_value[4]);
    setS(m.boundaryNut.kRight, m.boundaryNut.kRval, c.nut_bc[5], c.nut_bc_value[5]);
    checkBCsAndSetPatchTypes(&m);

    // ---- momentum (InitializeUEqn, ueqn.c:27-120)
    ueqn_ &u = X.ueqn;
    u.access = &a;
    for (Vec *v : {&u.Utmp, &u.Rhs, &u.Rhs_o, &u.Ucont, &u.Ucont_o, &u.Ucat, &u.dP, &u.gCont}) VecDuplicate(m.Cent, v);
    for (Vec *v : {&u.lUcont, &u.lUcat, &u.lFp, &u.lDiv1, &u.lDiv2, &u.lDiv3, &u.lVisc1, &u.lVisc2, &u.lVisc3, &u.sourceU})
        VecDuplicate(m.lCent, v);
    VecDuplicate(m.lAj, &u.lUstar);
    u.inviscid = 0;
    u.divScheme = c.div_scheme == TG_DIV_QUICK ? "quickDiv" : "central";
    u.centralDiv = c.div_scheme == TG_DIV_CENTRAL;
    u.quickDiv = c.div_scheme == TG_DIV_QUICK;
    u.ddtScheme = c.ddt_scheme == TG_DDT_RK4 ? "RK4" : "FE";
    u.hyperVisc = 0.0;
    u.hyperVisc4i = u.hyperVisc4j = u.hyperVisc4k = 0.0;
    u.meanGradP.x = c.mean_grad_p_value[0];
    u.meanGradP.y = c.mean_grad_p_value[1];
    u.meanGradP.z = c.mean_grad_p_value[2];
    if (c.bc[2] == TG_BC_WALL_SHUMANN) u.jLWM = make_shumann(c);

    // ---- pressure (InitializePEqn, peqn.c:35-103)
    peqn_ &p = X.peqn;
    p.access = &a;
    VecDuplicate(m.Nvert, &p.P);
    VecDuplicate(m.Nvert, &p.Phi);
    VecDuplicate(m.lNvert, &p.lP);
    VecDuplicate(m.lNvert, &p.lPhi);
    VecDuplicate(m.lNvert, &p.lGid);
    VecDuplicate(m.lNvert, &p.lLid);
    p.poissonIt = 8;
    p.poissonTol = 1e-8;
    p.solverType = "HYPRE";
    p.hypreSolverType = 1;

    // ---- LES (InitializeLES, les.c:60-90)
    les_ &l = X.les;
    l.access = &a;
    l.model = SMAGORINSKY;
    VecDuplicate(m.lAj, &l.lCs);
    VecDuplicate(m.lAj, &l.lNu_t);
    VecDuplicate(m.lAj, &l.lKsgs);
    VecDuplicate(m.lCsi, &l.lSx);
    VecDuplicate(m.lCsi, &l.lSy);
    VecDuplicate(m.lCsi, &l.lSz);
    VecDuplicate(m.lAj, &l.lS);

    // ---- temperature (InitializeTEqn, teqn.c:19-257, RK4; bTheta, ueqn.c:56-60;
    // the boundary/T patches and the thetaWallFunction of SetWallModels)
    if (c.teqn) {
        f.isTeqnActive = 1;
        teqn_ &t = X.teqn;
        t.access = &a;
        a.teqn = &t;
        d.teqn = &t;
        t.pTildeFormulation = c.p_tilde ? 1 : 0;
        for (Vec *v : {&t.TmprtTmp, &t.Tmprt, &t.Tmprt_o, &t.bT, &t.Rhs, &t.sourceT}) VecDuplicate(m.Nvert, v);
        for (Vec *v : {&t.lTmprt, &t.lTmprt_o}) VecDuplicate(m.lAj, v);
        for (Vec *v : {&t.lDivT, &t.lViscT}) VecDuplicate(m.lCent, v);
        if (t.pTildeFormulation) {
            VecDuplicate(m.lAj, &t.lRhoK);
            VecDuplicate(m.Cent, &t.ghGradRhok);
            VecDuplicate(m.Cent, &t.ghGradRhok_o);
        }
        t.ddtScheme = "RK4";
        t.solverType = "EXP";
        t.hyperVisc4i = t.hyperVisc4j = t.hyperVisc4k = 0.0;
        VecDuplicate(m.Cent, &u.bTheta);
        VecDuplicate(m.Cent, &u.bTheta_o);
        scalarBC &bt = m.boundaryT;
        word *names[6] = {&bt.iLeft, &bt.iRight, &bt.jLeft, &bt.jRight, &bt.kLeft, &bt.kRight};
        PetscReal *vals[6] = {&bt.iLval, &bt.iRval, &bt.jLval, &bt.jRval, &bt.kLval, &bt.kRval};
        for (int q = 0; q < 6; q++) { *names[q] = t_bc_name(c.t_bc[q]); *vals[q] = c.t_bc_value[q]; }
        bt.iLWF = bt.iRWF = bt.jRWF = bt.kLWF = bt.kRWF = 0;
        bt.jLWF = 0;
        if (c.t_bc[2] == TG_TBC_WALL_FUNCTION) {
            bt.jLWF = c.t_wall_type;
            t.jLWM = make_theta_wall(c);
        }
    }
}

// ------------------------------------------------------------ field access
enum Where { GLOBAL, LOCAL };
struct FieldRef {
    DM dm = nullptr;
    Vec global = nullptr;     // the global Vec, if the reference keeps one
    Vec local = nullptr;      // the local Vec, if the reference keeps one
};

FieldRef field(tg_ctx &X, int w)
{
    mesh_ &m = X.mesh;
    ueqn_ &u = X.ueqn;
    peqn_ &p = X.peqn;
    FieldRef r;
    switch (w) {
    case TG_F_CENT: r = {m.fda, m.Cent, m.lCent}; break;
    case TG_F_CSI: r = {m.fda, nullptr, m.lCsi}; break;
    case TG_F_ETA: r = {m.fda, nullptr, m.lEta}; break;
    case TG_F_ZET: r = {m.fda, nullptr, m.lZet}; break;
    case TG_F_ICSI: r = {m.fda, nullptr, m.lICsi}; break;
    case TG_F_IETA: r = {m.fda, nullptr, m.lIEta}; break;
    case TG_F_IZET: r = {m.fda, nullptr, m.lIZet}; break;
    case TG_F_JCSI: r = {m.fda, nullptr, m.lJCsi}; break;
    case TG_F_JETA: r = {m.fda, nullptr, m.lJEta}; break;
    case TG_F_JZET: r = {m.fda, nullptr, m.lJZet}; break;
    case TG_F_KCSI: r = {m.fda, nullptr, m.lKCsi}; break;
    case TG_F_KETA: r = {m.fda, nullptr, m.lKEta}; break;
    case TG_F_KZET: r = {m.fda, nullptr, m.lKZet}; break;
    case TG_F_AJ: r = {m.da, nullptr, m.lAj}; break;
    case TG_F_IAJ: r = {m.da, nullptr, m.lIAj}; break;
    case TG_F_JAJ: r = {m.da, nullptr, m.lJAj}; break;
    case TG_F_KAJ: r = {m.da, nullptr, m.lKAj}; break;
    case TG_F_UCONT: r = {m.fda, u.Ucont, u.lUcont}; break;
    case TG_F_UCAT: r = {m.fda, u.Ucat, u.lUcat}; break;
    case TG_F_UCONT_O: r = {m.fda, u.Ucont_o, nullptr}; break;
    case TG_F_RHS: r = {m.fda, u.Rhs, nullptr}; break;
    case TG_F_DP: r = {m.fda, u.dP, nullptr}; break;
    case TG_F_P: r = {m.da, p.P, p.lP}; break;
    case TG_F_PHI: r = {m.da, p.Phi, p.lPhi}; break;
    case TG_F_NUT: r = {m.da, nullptr, X.cfg.les ? X.les.lNu_t : nullptr}; break;
    case TG_F_TMPRT: if (X.cfg.teqn) r = {m.da, X.teqn.Tmprt, X.teqn.lTmprt}; break;
    case TG_F_BTHETA:
        if (X.cfg.teqn) r = {m.fda, X.cfg.p_tilde ? X.teqn.ghGradRhok : u.bTheta, nullptr};
        break;
    default: break;
    }
    return r;
}

// copy between the owned points of a Vec and a caller array of extent +2*halo
void copy_owned(tg_ctx &X, Vec v, DM dm, double *host, int halo, bool to_host)
{
    const PetscInt mx = X.cfg.mx, my = X.cfg.my, mz = X.cfg.mz, dof = dm->dof;
    const PetscInt lx = mx + 2 * halo, ly = my + 2 * halo;
    const PetscInt gx = v->local ? tgref_gsize(dm->bx, mx, dm->s) : mx;
    const PetscInt gy = v->local ? tgref_gsize(dm->by, my, dm->s) : my;
    const PetscInt ox = v->local ? -tgref_gstart(dm->bx, dm->s) : 0;
    const PetscInt oy = v->local ? -tgref_gstart(dm->by, dm->s) : 0;
    const PetscInt oz = v->local ? -tgref_gstart(dm->bz, dm->s) : 0;
    for (PetscInt k = 0; k < mz; k++)
        for (PetscInt j = 0; j < my; j++)
            for (PetscInt i = 0; i < mx; i++) {
                double *h = host + (((size_t)(k + halo) * ly + (j + halo)) * lx + (i + halo)) * dof;
                double *a = v->a.data() + (((size_t)(k + oz) * gy + (j + oy)) * gx + (i + ox)) * dof;
                for (PetscInt q = 0; q < dof; q++) {
                    if (to_host) h[q] = a[q];
                    else a[q] = h[q];
                }
            }
}

}  // namespace

// ====================================================================== C-ABI
extern "C" {

tg_status ref_create(const tg_config *cfg, tg_ctx **out)
{
    if (!cfg || !out) return TG_ERR_BAD_ARG;
    *out = nullptr;
    const tg_config &c = *cfg;
    if (c.mx < 6 || c.my < 6 || c.mz < 6) return TG_ERR_BAD_ARG;
    for (int q = 0; q < 6; q++) {
        if (c.bc[q] < 0 || c.bc[q] > TG_BC_INLET_LOG || (c.bc[q] == TG_BC_INLET_LOG && q != 4)) return TG_ERR_BAD_ARG;
        if (c.bc[q] == TG_BC_WALL_SHUMANN && q != 2) return TG_ERR_BAD_ARG;
    }
    // supported subset of the workloads (see the file header)
    if (c.ddt_scheme != TG_DDT_FE && c.ddt_scheme != TG_DDT_RK4) return TG_ERR_BAD_ARG;
    // the reference applies buoyancy exactly when the temperature equation is on
    if (c.source || (c.buoyancy != 0) != (c.teqn != 0)) return TG_ERR_BAD_ARG;
    if (c.teqn && c.t_ddt_scheme != TG_TDDT_RK4) return TG_ERR_BAD_ARG;
    for (int q = 0; q < 6; q++) {
        if (c.teqn && (c.t_bc[q] < 0 || c.t_bc[q] > TG_TBC_WALL_FUNCTION)) return TG_ERR_BAD_ARG;
        if (c.teqn && c.t_bc[q] == TG_TBC_WALL_FUNCTION && q != 2) return TG_ERR_BAD_ARG;
    }
    if (c.teqn && c.t_bc[2] == TG_TBC_WALL_FUNCTION &&
        (!c.les || (c.t_wall_type != TG_TWALL_SHUMANN && c.t_wall_type != TG_TWALL_FIXED_FLUX &&
                    c.t_wall_type != TG_TWALL_SURFACE_SERIES))) return TG_ERR_BAD_ARG;
    if (c.les && std::fabs(c.cs - TOSCA_STD_CS) > 1e-15) return TG_ERR_BAD_ARG;
    tg_ctx *C = new tg_ctx();
    C->cfg = c;
    tgref_set_quiet(true);
    tg_status s = guarded(C, [&]() -> tg_status { build(*C); return TG_OK; });
    if (s != TG_OK) { delete C; return s; }
    *out = C;
    return TG_OK;
}

tg_status ref_destroy(tg_ctx *C)
{
    // the stand-in Vecs and DMs are released with the process (test use only)
    delete C;
    return TG_OK;
}

const char *ref_last_error(tg_ctx *C) { return C ? C->err.c_str() : "null context"; }
const char *ref_status_string(tg_status s)
{
    switch (s) {
    case TG_OK: return "ok";
    case TG_ERR_BAD_ARG: return "bad argument or configuration outside the reference harness";
    case TG_ERR_STATE: return "reference code failed";
    default: return "error";
    }
}

tg_status ref_set_mesh_nodes(tg_ctx *C, const double *nodes)
{
    return guarded(C, [&]() -> tg_status {
        if (!nodes) return fail(C, TG_ERR_BAD_ARG, "null nodes");
        mesh_ &m = C->mesh;
        Vec g;
        DMCreateGlobalVector(m.fda, &g);
        const PetscInt mx = C->cfg.mx, my = C->cfg.my, mz = C->cfg.mz;
        // the last DMDA point of each direction carries no node (mesh.c:92-94, 190-290)
        for (PetscInt k = 0; k < mz; k++)
            for (PetscInt j = 0; j < my; j++)
                for (PetscInt i = 0; i < mx; i++) {
                    const size_t q = ((size_t)k * my + j) * mx + i;
                    const bool node = i < mx - 1 && j < my - 1 && k < mz - 1;
                    for (int c = 0; c < 3; c++) g->a[3 * q + c] = node ? nodes[3 * q + c] : 0.0;
                }
        // DMSetCoordinates: the local coordinates follow by the DM's scatter
        m.da->coords_global = g;
        DMCreateLocalVector(m.fda, &m.da->coords_local);
        DMGlobalToLocalEnd(m.fda, g, INSERT_VALUES, m.da->coords_local);
        SetBoundingBox(&m);
        SetMeshMetrics(&m);
        // Poisson connectivity and matrix (InitializePEqn, peqn.c:60-90)
        peqn_ &p = C->peqn;
        SetPoissonConnectivity(&p);
        CreateHypreMatrix(&p);
        CreateHypreVector(&p);
        tgref_matrix_clear();
        SetCoeffMatrix(&p);
        C->has_mesh = true;
        return TG_OK;
    });
}

tg_status ref_set_field(tg_ctx *C, int32_t w, const double *host, int32_t halo)
{
    return guarded(C, [&]() -> tg_status {
        if (!host || halo < 0) return fail(C, TG_ERR_BAD_ARG, "bad field argument");
        FieldRef r = field(*C, w);
        if (!r.dm) return fail(C, TG_ERR_BAD_ARG, "field not available in the reference harness");
        if (r.global) {
            copy_owned(*C, r.global, r.dm, (double *)host, halo, false);
            if (r.local) DMGlobalToLocalEnd(r.dm, r.global, INSERT_VALUES, r.local);
        } else {
            copy_owned(*C, r.local, r.dm, (double *)host, halo, false);
            DMLocalToLocalEnd(r.dm, r.local, INSERT_VALUES, r.local);
        }
        return TG_OK;
    });
}

tg_status ref_get_field(tg_ctx *C, int32_t w, double *host, int32_t halo)
{
    return guarded(C, [&]() -> tg_status {
        if (!host || halo < 0) return fail(C, TG_ERR_BAD_ARG, "bad field argument");
        if (w == TG_F_TAUWALL) {
            if (!C->ueqn.jLWM) return fail(C, TG_ERR_BAD_ARG, "no wall model");
            const PetscInt mx = C->cfg.mx, mz = C->cfg.mz;
            for (PetscInt k = 0; k < mz; k++)
                for (PetscInt i = 0; i < mx; i++) {
                    double *h = host + 3 * ((size_t)k * mx + i);
                    h[0] = C->ueqn.jLWM->tauWall.x[k][i];
                    h[1] = C->ueqn.jLWM->tauWall.y[k][i];
                    h[2] = C->ueqn.jLWM->tauWall.z[k][i];
                }
            return TG_OK;
        }
        if (w == TG_F_QWALL || w == TG_F_SURF_THETA) {
            wallModel *wm = C->cfg.teqn ? C->teqn.jLWM : nullptr;
            if (!wm) return fail(C, TG_ERR_BAD_ARG, "no thetaWallFunction");
            const Shumann *sh = wm->wmShumann;
            const PetscInt mx = C->cfg.mx, mz = C->cfg.mz;
            for (PetscInt k = 0; k < mz; k++)
                for (PetscInt i = 0; i < mx; i++) {
                    double v = 0.0;
                    if (w == TG_F_QWALL) v = wm->qWall.z[k][i];
                    else if (C->cfg.t_wall_type == TG_TWALL_SHUMANN && sh->surfaceThetaSet && k >= 1 && k <= mz - 2 && i >= 1 && i <= mx - 2)
                        v = sh->surfaceTheta[k][i];
                    host[(size_t)k * mx + i] = v;
                }
            return TG_OK;
        }
        FieldRef r = field(*C, w);
        if (!r.dm) return fail(C, TG_ERR_BAD_ARG, "field not available in the reference harness");
        copy_owned(*C, r.global ? r.global : r.local, r.dm, host, halo, true);
        return TG_OK;
    });
}

tg_status ref_contravariant_to_cartesian(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status { contravariantToCartesian(&C->ueqn); return TG_OK; });
}

tg_status ref_update_nut(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->cfg.les) return fail(C, TG_ERR_STATE, "LES is off");
        UpdateCs(&C->les);
        UpdateNut(&C->les);
        return TG_OK;
    });
}

tg_status ref_update_wall_models(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status { UpdateWallModelsU(&C->ueqn); return TG_OK; });
}

tg_status ref_grad_p(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status { GradP(&C->peqn); return TG_OK; });
}

tg_status ref_form_u(tg_ctx *C, double scale, int32_t zero_rhs)
{
    return guarded(C, [&]() -> tg_status {
        if (zero_rhs) VecSet(C->ueqn.Rhs, 0.0);
        FormU(&C->ueqn, C->ueqn.Rhs, scale, 0);
        return TG_OK;
    });
}

tg_status ref_explicit_rhs(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status { ExplicitRhsU(&C->ueqn, 0); return TG_OK; });
}

tg_status ref_solve_u(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status { SolveUEqn(&C->ueqn); return TG_OK; });
}

tg_status ref_solve_p(tg_ctx *C, tg_stats *st)
{
    return guarded(C, [&]() -> tg_status {
        SolvePEqn(&C->peqn);
        if (st) {
            st->poisson_iterations = (int32_t)C->peqn.poissonIterations;
            st->poisson_final_residual = C->peqn.finalPoissonRes;
        }
        return TG_OK;
    });
}

tg_status ref_continuity_error(tg_ctx *C, double *max_div)
{
    return guarded(C, [&]() -> tg_status {
        ContinuityErrorsOptimized(&C->peqn);
        // the value the reference prints (peqn.c:4169-4170)
        if (!tgref_printed_value("Time step continuity error:", &C->last_div))
            return fail(C, TG_ERR_STATE, "continuity error not reported");
        if (max_div) *max_div = C->last_div;
        return TG_OK;
    });
}

tg_status ref_update_cartesian_bcs(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status { UpdateCartesianBCs(&C->ueqn); return TG_OK; });
}

tg_status ref_update_contravariant_bcs(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status { UpdateContravariantBCs(&C->ueqn); return TG_OK; });
}

tg_status ref_sync_pressure(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status { SyncPressureAcrossDomains(C->dom.get()); return TG_OK; });
}

// one time step in the order of TOSCA's time loop (main.c:54-327) for the
// supported workloads: no IBM, overset, turbines, damping, controllers or
// temperature
tg_status ref_step(tg_ctx *C, int32_t nsteps, tg_stats *st)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        ueqn_ &u = C->ueqn;
        peqn_ &p = C->peqn;
        tg_stats local{};
        teqn_ *t = C->cfg.teqn ? &C->teqn : nullptr;
        for (int32_t s = 0; s < nsteps; s++) {
            // adjustTimeStep with a fixed time step (clock.c:347-367): the
            // clock time of the step, it counted from itStart
            C->clock.time = C->clock.startTime + (C->clock.it - C->clock.itStart) * C->clock.dt + C->clock.dt;
            VecCopy(u.Ucont, u.Ucont_o);                            // main.c:81
            if (t) VecCopy(t->Tmprt, t->Tmprt_o);                   // main.c:83-99 (RK4)
            if (C->cfg.les) {                                       // main.c:108-113
                UpdateCs(&C->les);
                UpdateNut(&C->les);
                UpdateWallModelsU(&u);
            }
            GradP(&p);                                              // main.c:146-153
            if (t) {                                                // main.c:166-182
                if (C->clock.it > C->clock.itStart) {
                    if (t->pTildeFormulation) VecCopy(t->ghGradRhok, t->ghGradRhok_o);
                    else VecCopy(u.bTheta, u.bTheta_o);
                }
                if (t->pTildeFormulation) ghGradRhoK(t);
                else Buoyancy(&u, 1.0);
            }
            SolveUEqn(&u);                                          // main.c:185
            SolvePEqn(&p);                                          // main.c:188
            contravariantToCartesian(&u);                           // main.c:191
            if (t) {                                                // main.c:194-205
                // UpdateCsk / UpdatekT (lesScalar.c, not compiled here) set the
                // scalar SGS fields of the dynamic models, which FormT reads
                // only for those models, not for Smagorinsky
                UpdateWallModelsT(t);
                SolveTEqn(t);
            }
            ContinuityErrorsOptimized(&p);                          // main.c:211
            tgref_printed_value("Time step continuity error:", &C->last_div);
            if (t) UpdateTemperatureBCs(t);                         // main.c:274-278
            UpdateCartesianBCs(&u);                                 // main.c:284
            UpdateContravariantBCs(&u);                             // main.c:287
            SyncPressureAcrossDomains(C->dom.get());                // main.c:318
            C->clock.it++;                                          // main.c:319
            local.steps++;
            local.poisson_iterations = (int32_t)p.poissonIterations;
            local.poisson_total_iterations += (int32_t)p.poissonIterations;
            local.poisson_final_residual = p.finalPoissonRes;
            local.max_divergence = C->last_div;
        }
        if (st) *st = local;
        return TG_OK;
    });
}

// the matrix SetCoeffMatrix assembled (captured from HYPRE_IJMatrixSetValues)
int64_t ref_poisson_size(tg_ctx *) { return tgref_matrix_rows(); }
int64_t ref_poisson_nnz(tg_ctx *) { return tgref_matrix_nnz(); }
tg_status ref_poisson_matrix(tg_ctx *, int64_t *rowptr, int64_t *col, double *val)
{
    tgref_matrix_csr((long *)rowptr, (long *)col, val);
    return TG_OK;
}

// Buoyancy (ueqn_sources.c:2726-2820) or, with -pTildeBuoyancy, ghGradRhoK (teqn.c:278-652)
tg_status ref_buoyancy(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->cfg.teqn) return fail(C, TG_ERR_STATE, "the reference applies buoyancy only with its temperature equation");
        if (C->teqn.pTildeFormulation) ghGradRhoK(&C->teqn);
        else Buoyancy(&C->ueqn, 1.0);
        return TG_OK;
    });
}

// UpdateWallModelsT (boundary.c:3858-4520) and UpdateTemperatureBCs (boundary.c:2052-2616)
tg_status ref_update_wall_models_t(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->cfg.teqn) return fail(C, TG_ERR_STATE, "no temperature equation");
        UpdateWallModelsT(&C->teqn);
        return TG_OK;
    });
}
tg_status ref_update_temperature_bcs(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->cfg.teqn) return fail(C, TG_ERR_STATE, "no temperature equation");
        UpdateTemperatureBCs(&C->teqn);
        return TG_OK;
    });
}

// the series readSurfaceTempData (boundary.c:5269-5400) would read from
// inflowDatabase/mesoscaleData: timeVec, surfTemp and numT of the jLeft Shumann model
tg_status ref_set_surface_temperature(tg_ctx *C, int32_t n, const double *time, const double *temp)
{
    return guarded(C, [&]() -> tg_status {
        if (n < 2 || !time || !temp) return fail(C, TG_ERR_BAD_ARG, "a surface temperature series needs n >= 2 points");
        if (!C->cfg.teqn || !C->teqn.jLWM) return fail(C, TG_ERR_STATE, "no thetaWallFunction");
        Shumann *wm = C->teqn.jLWM->wmShumann;
        wm->timeVec = new PetscReal[n];
        wm->surfTemp = new PetscReal[n];
        for (int32_t q = 0; q < n; q++) { wm->timeVec[q] = time[q]; wm->surfTemp[q] = temp[q]; }
        wm->numT = n;
        return TG_OK;
    });
}

// the Monin-Obukhov functions themselves (wallfunctions.c:12-290)
double ref_mo_ustar(double U, double dist, double z0, double gammaM, double kappa, double qwall, double thetaRef)
{
    double us = 0.0, phiM = 0.0, L = 0.0;
    uStarShumann(U, dist, z0, gammaM, kappa, qwall, thetaRef, us, phiM, L, 0, 0, 0);
    return us;
}
double ref_mo_qwall(double U, double dist, double z0, double gammaM, double gammaH, double alphaH, double thetaRef,
                    double deltaTheta, double kappa)
{
    double q = 0.0, us = 0.0, phiM = 0.0, phiH = 0.0, L = 0.0;
    qWallShumann(U, dist, z0, gammaM, gammaH, alphaH, thetaRef, deltaTheta, kappa, q, us, phiM, phiH, L, 0, 0, 0);
    return q;
}

// entry points of the C-ABI the harness does not provide
#define REF_UNSUPPORTED(name, ...) \
    tg_status ref_##name(tg_ctx *C, __VA_ARGS__) { return fail(C, TG_ERR_BAD_ARG, "not provided by the reference harness"); }
REF_UNSUPPORTED(init_from_cartesian, const double *, int32_t)
REF_UNSUPPORTED(step_host, double *, double *, double *, double *, int32_t, tg_stats *)
REF_UNSUPPORTED(write_field_petsc, int32_t, const char *)
REF_UNSUPPORTED(read_field_petsc, int32_t, const char *)
REF_UNSUPPORTED(set_turbines, int32_t, const tg_turbine *, double)
REF_UNSUPPORTED(set_turbine_ct, const double *)
REF_UNSUPPORTED(turbine_state, double *, double *, double *, double *, int32_t)
REF_UNSUPPORTED(set_farm_objective, int32_t)
REF_UNSUPPORTED(ct_gradient, double *, int32_t)
REF_UNSUPPORTED(momentum_info, int32_t *, int32_t *, double *)

}  // extern "C"
