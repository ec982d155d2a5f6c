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
// InitializePEqn, peqn.c:35-103; InitializeLES, les.c:20-150; SetWallModels,
// boundary.c:4640-4990), with the values a control.dat and boundary/ files
// would hold, and then calls the reference's functions. Supported: periodic,
// slip, noSlip and the Schumann velocity wall function (-3, averaged u*) on
// jLeft; central and QUICK convection; FE and RK4; no LES or Smagorinsky
// (TOSCA's hard-coded Cs^2 = 0.0289, les.c:10,175); the mean pressure
// gradient. The HYPRE solve inside SolvePEqn is replaced by a tight solve of
// the captured matrix (petsc_stub.cpp).
#include "include/base.h"
#include "include/domain.h"
#include "include/io.h"
#include "include/inline.h"

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
    s->thetaRef = c.t_ref;
    s->roughness = c.wall_roughness;
    s->gammaM = 4.8;                            // enters only stratified (qWall != 0) evaluations
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
    mesh_ mesh{};
    ueqn_ ueqn{};
    peqn_ peqn{};
    les_ les{};
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
    X.clock.time = 0.0;

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
        if (c.bc[q] < 0 || c.bc[q] > TG_BC_WALL_SHUMANN) return TG_ERR_BAD_ARG;
        if (c.bc[q] == TG_BC_WALL_SHUMANN && q != 2) return TG_ERR_BAD_ARG;
    }
    // supported subset of the workloads (see the file header)
    if (c.ddt_scheme != TG_DDT_FE && c.ddt_scheme != TG_DDT_RK4) return TG_ERR_BAD_ARG;
    if (c.buoyancy || c.teqn || c.source || c.p_tilde) return TG_ERR_BAD_ARG;
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
        for (int32_t s = 0; s < nsteps; s++) {
            VecCopy(u.Ucont, u.Ucont_o);                            // main.c:77
            if (C->cfg.les) {                                       // main.c:104-117
                UpdateCs(&C->les);
                UpdateNut(&C->les);
                UpdateWallModelsU(&u);
            }
            GradP(&p);                                              // main.c:146-153
            SolveUEqn(&u);                                          // main.c:183
            SolvePEqn(&p);                                          // main.c:186
            contravariantToCartesian(&u);                           // main.c:189
            ContinuityErrorsOptimized(&p);                          // main.c:211
            tgref_printed_value("Time step continuity error:", &C->last_div);
            UpdateCartesianBCs(&u);                                 // main.c:284
            UpdateContravariantBCs(&u);                             // main.c:287
            SyncPressureAcrossDomains(C->dom.get());                // main.c:318
            C->clock.it++;                                          // main.c:321
            C->clock.time += C->clock.dt;
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

tg_status ref_buoyancy(tg_ctx *C) { return fail(C, TG_ERR_BAD_ARG, "not provided by the reference harness"); }

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
