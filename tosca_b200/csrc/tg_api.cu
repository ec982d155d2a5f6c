// C-ABI of include/tosca_gpu.h: context lifetime, host<->device transfers in
// TOSCA's AoS DMDA layout, and the stage entry points. Every entry point
// returns a tg_status and never exits or traps.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "tg_internal.cuh"
#include "../../include/tosca_gpu_prof.h"

namespace tg {

void *dalloc(tg_ctx *C, size_t bytes)
{
    void *p = nullptr;
    if (bytes == 0) bytes = 8;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) throw CudaError{e, "cudaMalloc"};
    C->allocs.push_back(p);
    e = cudaMemsetAsync(p, 0, bytes, C->stream);
    if (e != cudaSuccess) throw CudaError{e, "cudaMemsetAsync"};
    return p;
}

V3f<double> dalloc3(tg_ctx *C, size_t n)
{
    double *b = (double *)dalloc(C, 3 * n * sizeof(double));
    return V3f<double>{b, b + n, b + 2 * n};
}

namespace {

struct ApiError { tg_status s; std::string msg; };

tg_status fail(tg_ctx *C, tg_status s, const std::string &m)
{
    if (C) C->err = m;
    return s;
}

template <class F>
tg_status guarded(tg_ctx *C, F &&f)
{
    if (!C) return TG_ERR_BAD_ARG;
    try {
        cudaError_t e = cudaSetDevice(C->cfg.device);
        if (e != cudaSuccess) return fail(C, TG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        tg_status s = f();
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) return fail(C, TG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(le));
        return s;
    } catch (const CudaError &e) {
        tg_status s = (e.e == cudaErrorMemoryAllocation) ? TG_ERR_ALLOC : TG_ERR_CUDA;
        if (e.e == cudaErrorInvalidValue && std::string(e.what).find("grid") != std::string::npos) s = TG_ERR_BAD_ARG;
        return fail(C, s, std::string(e.what) + ": " + cudaGetErrorString(e.e));
    } catch (const ApiError &e) {
        return fail(C, e.s, e.msg);
    } catch (const std::bad_alloc &) {
        return fail(C, TG_ERR_ALLOC, "host allocation failed");
    }
}

// field lookup: vector (3 planes) or scalar
bool vec_field(tg_ctx *C, int w, V3f<double> &out)
{
    Metrics &m = C->m; State &s = C->s;
    switch (w) {
    case TG_F_CENT: out = m.cent; return true;   case TG_F_CSI: out = m.csi; return true;
    case TG_F_ETA: out = m.eta; return true;     case TG_F_ZET: out = m.zet; return true;
    case TG_F_ICSI: out = m.icsi; return true;   case TG_F_IETA: out = m.ieta; return true;
    case TG_F_IZET: out = m.izet; return true;   case TG_F_JCSI: out = m.jcsi; return true;
    case TG_F_JETA: out = m.jeta; return true;   case TG_F_JZET: out = m.jzet; return true;
    case TG_F_KCSI: out = m.kcsi; return true;   case TG_F_KETA: out = m.keta; return true;
    case TG_F_KZET: out = m.kzet; return true;   case TG_F_UCONT: out = s.ucont; return true;
    case TG_F_UCAT: out = s.ucat; return true;   case TG_F_UCONT_O: out = s.ucont_o; return true;
    case TG_F_RHS: out = s.rhs; return true;     case TG_F_DP: out = s.dp; return true;
    case TG_F_BTHETA: out = s.btheta; return true;
    case TG_F_SOURCE: out = s.source; return true;
    case TG_F_FARM_FORCE: return farm_field(C, w, out);
    case TG_F_FARM_CONT: return farm_field(C, w, out);
    default: return false;
    }
}
double *scal_field(tg_ctx *C, int w)
{
    switch (w) {
    case TG_F_AJ: return C->m.aj; case TG_F_IAJ: return C->m.iaj; case TG_F_JAJ: return C->m.jaj; case TG_F_KAJ: return C->m.kaj;
    case TG_F_P: return C->s.p; case TG_F_PHI: return C->s.phi; case TG_F_NUT: return C->s.nut; case TG_F_TMPRT: return C->s.tmprt;
    default: return nullptr;
    }
}

// AoS (host, extent +2 halo) <-> SoA (device, global extent)
__global__ void k_aos_to_soa(Grid g, const double *src, int halo, double *x, double *y, double *z)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    int lx = g.mx + 2 * halo, ly = g.my + 2 * halo;
    int64_t s = ((int64_t)(k + halo) * ly + (j + halo)) * lx + (i + halo);
    int q = g.lin(k, j, i);
    if (y) { x[q] = src[3 * s]; y[q] = src[3 * s + 1]; z[q] = src[3 * s + 2]; }
    else x[q] = src[s];
}
__global__ void k_soa_to_aos(Grid g, double *dst, int halo, const double *x, const double *y, const double *z)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    int lx = g.mx + 2 * halo, ly = g.my + 2 * halo;
    int64_t d = ((int64_t)(k + halo) * ly + (j + halo)) * lx + (i + halo);
    int q = g.lin(k, j, i);
    if (y) { dst[3 * d] = x[q]; dst[3 * d + 1] = y[q]; dst[3 * d + 2] = z[q]; }
    else dst[d] = x[q];
}

// staging buffer for AoS host arrays, owned by the context (grows on demand)
double *staging(tg_ctx *C, size_t bytes)
{
    if (C->stage_bytes < bytes) { C->stage = (double *)dalloc(C, bytes); C->stage_bytes = bytes; }
    return C->stage;
}

// interior cells of a vector field: dst <- src
__global__ void k_copy_interior3(Grid g, V3f<double> src, V3f<double> dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int q = g.lin(k, j, i);
    dst.x[q] = src.x[q]; dst.y[q] = src.y[q]; dst.z[q] = src.z[q];
}

// the last DMDA point of each direction carries no node (mesh.c:92-94)
__global__ void k_zero_last_nodes(Grid g, double *nodes)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    if (i == g.mx - 1 || j == g.my - 1 || k == g.mz - 1) {
        int q = 3 * g.lin(k, j, i);
        nodes[q] = 0.0; nodes[q + 1] = 0.0; nodes[q + 2] = 0.0;
    }
}

void upload(tg_ctx *C, const double *host, int halo, double *x, double *y, double *z)
{
    const Grid g = C->g;
    size_t n = (size_t)(g.mx + 2 * halo) * (g.my + 2 * halo) * (g.mz + 2 * halo) * (y ? 3 : 1);
    double *st = staging(C, n * sizeof(double));
    TG_CUDA(cudaMemcpyAsync(st, host, n * sizeof(double), cudaMemcpyHostToDevice, C->stream));
    k_aos_to_soa<<<grid3(g.mx, g.my, g.mz), block3(), 0, C->stream>>>(g, st, halo, x, y, z);
    TG_CUDA(cudaGetLastError());
}

void download(tg_ctx *C, double *host, int halo, const double *x, const double *y, const double *z)
{
    const Grid g = C->g;
    size_t n = (size_t)(g.mx + 2 * halo) * (g.my + 2 * halo) * (g.mz + 2 * halo) * (y ? 3 : 1);
    double *st = staging(C, n * sizeof(double));
    if (halo > 0) {
        // keep the caller's halo entries: start from the caller's array
        TG_CUDA(cudaMemcpyAsync(st, host, n * sizeof(double), cudaMemcpyHostToDevice, C->stream));
    }
    k_soa_to_aos<<<grid3(g.mx, g.my, g.mz), block3(), 0, C->stream>>>(g, st, halo, x, y, z);
    TG_CUDA(cudaGetLastError());
    TG_CUDA(cudaMemcpyAsync(host, st, n * sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaStreamSynchronize(C->stream));
}

void check_nan(tg_ctx *C)
{
    // max |div| is NaN-propagating through fmax only partially; test a few
    // scalars of the state instead: the last divergence and the first face flux
    double h[2];
    TG_CUDA(cudaMemcpyAsync(&h[0], C->d_scal + 16, sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaMemcpyAsync(&h[1], C->s.ucont.x + C->g.lin(1, 1, 1), sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaStreamSynchronize(C->stream));
    if (!std::isfinite(h[0]) || !std::isfinite(h[1])) throw ApiError{TG_ERR_NAN, "non-finite value in the state"};
}

}  // namespace
}  // namespace tg

using namespace tg;

extern "C" {

const char *tg_status_string(tg_status s)
{
    switch (s) {
    case TG_OK: return "ok"; case TG_ERR_CUDA: return "CUDA error"; case TG_ERR_BAD_ARG: return "bad argument";
    case TG_ERR_NOT_CONVERGED: return "pressure solve did not converge"; case TG_ERR_NAN: return "non-finite value";
    case TG_ERR_ALLOC: return "allocation failed"; case TG_ERR_STATE: return "invalid state";
    }
    return "unknown status";
}

const char *tg_last_error(const tg_ctx *C) { return C ? C->err.c_str() : "null context"; }

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

tg_status tg_create(const tg_config *cfg, tg_ctx **out)
{
    if (!cfg || !out) return TG_ERR_BAD_ARG;
    *out = nullptr;
    if (cfg->mx < 6 || cfg->my < 6 || cfg->mz < 6) return TG_ERR_BAD_ARG;
    if ((int64_t)cfg->mx * cfg->my * cfg->mz > (int64_t)INT32_MAX / 4) return TG_ERR_BAD_ARG;
    for (int p = 0; p < 6; p++) if (cfg->bc[p] < 0 || cfg->bc[p] > TG_BC_INLET_LOG) return TG_ERR_BAD_ARG;
    // the inflow/outflow patches with the explicit schemes only
    for (int p = 0; p < 6; p++)
        if (cfg->bc[p] >= TG_BC_FIXED_VALUE && cfg->ddt_scheme != TG_DDT_FE && cfg->ddt_scheme != TG_DDT_RK4) return TG_ERR_BAD_ARG;
    // the log-law inletFunction (type 2) on kLeft: positive roughness, hInv
    // above it, a unit direction (TOSCA normalises directionU, inflow.c:71)
    for (int p = 0; p < 6; p++)
        if (cfg->bc[p] == TG_BC_INLET_LOG) {
            const double *d = cfg->inlet_dir;
            const double n = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (p != TG_KLEFT || !(cfg->inlet_z0 > 0) || !(cfg->inlet_u_tau >= 0) || !(cfg->inlet_h_inv > cfg->inlet_z0) ||
                !(std::fabs(n - 1.0) < 1e-12)) return TG_ERR_BAD_ARG;
        }
    for (int d = 0; d < 3; d++)
        if ((cfg->bc[2 * d] == TG_BC_PERIODIC) != (cfg->bc[2 * d + 1] == TG_BC_PERIODIC)) return TG_ERR_BAD_ARG;
    for (int p = 0; p < 6; p++) if (cfg->bc[p] == TG_BC_WALL_SHUMANN && p != TG_JLEFT) return TG_ERR_BAD_ARG;
    if (cfg->dt <= 0 || cfg->div_scheme < 0 || cfg->div_scheme > 1 || cfg->ddt_scheme < 0 || cfg->ddt_scheme > TG_DDT_RK3SOCN) return TG_ERR_BAD_ARG;
    if (cfg->gmres_restart < 0 || cfg->gmres_restart > 60) return TG_ERR_BAD_ARG;
    if (cfg->p_tilde && !cfg->buoyancy) return TG_ERR_BAD_ARG;
    if (cfg->poisson_guess > 2 || cfg->poisson_guess < -1) return TG_ERR_BAD_ARG;
    if (cfg->precision != TG_PREC_FP64 && cfg->precision != TG_PREC_MIXED) return TG_ERR_BAD_ARG;
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
    C->cfg = *cfg;
    tg_status s = guarded(C, [&]() -> tg_status {
        TG_CUDA(cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking));
        TG_CUDA(cudaEventCreate(&C->ev0));
        TG_CUDA(cudaEventCreate(&C->ev1));
        // before any step graph is captured, so that every captured step records it
        if (cfg->les) TG_CUDA(cudaEventCreateWithFlags(&C->ev_nut, cudaEventDisableTiming));
        Grid &g = C->g;
        g.mx = cfg->mx; g.my = cfg->my; g.mz = cfg->mz;
        g.pi = cfg->bc[TG_ILEFT] == TG_BC_PERIODIC;
        g.pj = cfg->bc[TG_JLEFT] == TG_BC_PERIODIC;
        g.pk = cfg->bc[TG_KLEFT] == TG_BC_PERIODIC;
        Params &p = C->prm;
        for (int q = 0; q < 6; q++) { p.bc[q] = cfg->bc[q]; p.nut_bc[q] = cfg->nut_bc[q]; p.nut_bc_value[q] = cfg->nut_bc_value[q]; }
        for (int q = 0; q < 18; q++) p.bc_value[q] = cfg->bc_value[q];
        p.inlet_u_tau = cfg->inlet_u_tau; p.inlet_z0 = cfg->inlet_z0; p.inlet_h_inv = cfg->inlet_h_inv;
        for (int q = 0; q < 3; q++) p.inlet_dir[q] = cfg->inlet_dir[q];
        p.grnd = 0.0;
        p.curvilinear = cfg->curvilinear; p.les = cfg->les; p.div_scheme = cfg->div_scheme;
        p.buoyancy = cfg->buoyancy; p.mean_grad_p = cfg->mean_grad_p; p.source = cfg->source;
        p.cs = cfg->cs; p.nu = cfg->nu; p.dt = cfg->dt; p.t_ref = cfg->t_ref;
        for (int q = 0; q < 3; q++) p.mgp[q] = cfg->mean_grad_p_value[q];
        p.z0 = cfg->wall_roughness; p.kappa = cfg->wall_kappa;
        p.teqn = cfg->teqn; p.prandtl = cfg->prandtl;
        for (int q = 0; q < 6; q++) { p.t_bc[q] = cfg->t_bc[q]; p.t_bc_value[q] = cfg->t_bc_value[q]; }
        p.t_wall = (cfg->teqn && cfg->t_bc[TG_JLEFT] == TG_TBC_WALL_FUNCTION) ? cfg->t_wall_type : 0;
        p.wall_coupled = p.t_wall != 0;
        p.t_wall_localized = cfg->t_wall_localized;
        p.tw_qwall = cfg->t_wall_qwall; p.tw_heating = cfg->t_wall_heating_rate; p.tw_kappa = cfg->t_wall_kappa;
        p.tw_theta_ref = cfg->t_wall_theta_ref; p.tw_z0 = cfg->t_wall_roughness; p.tw_gamma_m = cfg->t_wall_gamma_m;
        p.tw_gamma_h = cfg->t_wall_gamma_h; p.tw_alpha_h = cfg->t_wall_alpha_h;
        p.wall_gamma_m = cfg->wall_gamma_m; p.wall_theta_ref = cfg->wall_theta_ref;
        C->it = cfg->it_start;
        const size_t G = (size_t)g.size();
        Metrics &m = C->m;
        V3f<double> *mv[] = {&m.cent, &m.csi, &m.eta, &m.zet, &m.icsi, &m.ieta, &m.izet, &m.jcsi, &m.jeta, &m.jzet, &m.kcsi, &m.keta, &m.kzet};
        for (auto *v : mv) *v = dalloc3(C, G);
        double **ms[] = {&m.aj, &m.iaj, &m.jaj, &m.kaj, &m.g11, &m.g12, &m.g13, &m.g21, &m.g22, &m.g23, &m.g31, &m.g32, &m.g33};
        for (auto **v : ms) *v = dallocd(C, G);
        State &st = C->s;
        V3f<double> *sv[] = {&st.ucont, &st.ucont_o, &st.ucat, &st.rhs, &st.dp, &st.btheta, &st.btheta_o, &st.gcont, &st.utmp, &st.snap, &st.source};
        for (auto *v : sv) *v = dalloc3(C, G);
        C->mixed = cfg->precision == TG_PREC_MIXED;
        alloc_precision_work(C);
        double **ss[] = {&st.p, &st.phi, &st.nut, &st.tmprt, &st.ssnap};
        for (auto **v : ss) *v = dallocd(C, G);
        if (cfg->ddt_scheme == TG_DDT_CN) st.rhs_o = dalloc3(C, G);
        if (cfg->teqn) {
            st.tdiv = dalloc3(C, G); st.tvisc = dalloc3(C, G);
            st.trhs = dallocd(C, G); st.tmprt_o = dallocd(C, G); st.ttmp = dallocd(C, G);
            if (cfg->t_ddt_scheme == TG_TDDT_ABBE) { C->tconv = dallocd(C, G); C->tconv_o = dallocd(C, G); }
            if (cfg->t_ddt_scheme == TG_TDDT_BDF2) C->tmprt_oo = dallocd(C, G);
        }
        const size_t P = (size_t)g.mx * g.mz;
        double **ws[] = {&st.twx, &st.twy, &st.twz, &st.umean, &st.ufx, &st.ufy, &st.ufz, &st.qwall, &st.surf_theta};
        for (auto **v : ws) *v = dallocd(C, P);
        C->red_blocks = 148 * 4;
        C->d_red = dallocd(C, 4 * (size_t)C->red_blocks + 64);
        C->d_scal = dallocd(C, 128);
        set_device_step(C);
        TG_CUDA(cudaMallocHost((void **)&C->h_scal, 128 * sizeof(double)));
        std::memset(C->h_scal, 0, 128 * sizeof(double));
        TG_CUDA(cudaStreamSynchronize(C->stream));
        return TG_OK;
    });
    if (s != TG_OK) {
        std::string e = C->err;
        tg_destroy(C);
        (void)e;
        return s;
    }
    *out = C;
    return TG_OK;
}

tg_status tg_destroy(tg_ctx *C)
{
    if (!C) return TG_OK;
    cudaSetDevice(C->cfg.device);
    if (C->stream) cudaStreamSynchronize(C->stream);
    graph_destroy(C);
    for (cudaStream_t a : C->aux) if (a) cudaStreamDestroy(a);
    try { farm_destroy(C); } catch (...) {}
    cn_destroy(C);
    imex_destroy(C);
    gmres_free(C->tgm);
    C->tgm = nullptr;
    jfnk_free(C->tsn);
    C->tsn = nullptr;
    poisson_destroy(C);
    adj_destroy(C);
    for (void *p : C->allocs) cudaFree(p);
    for (cudaEvent_t e : C->prof.pool) cudaEventDestroy(e);
    if (C->h_scal) cudaFreeHost(C->h_scal);
    if (C->ev0) cudaEventDestroy(C->ev0);
    if (C->ev1) cudaEventDestroy(C->ev1);
    if (C->copy_stream) { cudaStreamSynchronize(C->copy_stream); cudaStreamDestroy(C->copy_stream); }
    if (C->ev_nut) cudaEventDestroy(C->ev_nut);
    if (C->stream) cudaStreamDestroy(C->stream);
    delete C;
    return TG_OK;
}

tg_status tg_set_mesh_nodes(tg_ctx *C, const double *nodes)
{
    return guarded(C, [&]() -> tg_status {
        if (!nodes) return fail(C, TG_ERR_BAD_ARG, "null nodes");
        const Grid g = C->g;
        const size_t G = (size_t)g.size();
        double *dn = (double *)dalloc(C, 3 * G * sizeof(double));
        TG_CUDA(cudaMemcpyAsync(dn, nodes, 3 * G * sizeof(double), cudaMemcpyHostToDevice, C->stream));
        k_zero_last_nodes<<<grid3(g.mx, g.my, g.mz), block3(), 0, C->stream>>>(g, dn);
        // mesh->grndLevel (SetBoundingBox, mesh.c:2014-2063): the lowest node
        double grnd = 1e30;
        for (int k = 0; k < g.mz - 1; k++) for (int j = 0; j < g.my - 1; j++) for (int i = 0; i < g.mx - 1; i++)
            grnd = std::min(grnd, nodes[3 * (size_t)g.lin(k, j, i) + 2]);
        C->prm.grnd = grnd;
        TG_CUDA(cudaStreamSynchronize(C->stream));
        metrics_from_nodes(C, dn);
        refresh_filter(C);
        if (C->cfg.p_tilde) {
            if (!C->node_z) C->node_z = dallocd(C, G);
            TG_CUDA(cudaMemcpy2DAsync(C->node_z, sizeof(double), dn + 2, 3 * sizeof(double), sizeof(double), G,
                                      cudaMemcpyDeviceToDevice, C->stream));
        }
        C->met32_stale = true;
        // orthogonality: every cross term of the face metric tensor vanishes
        std::vector<double> h(G);
        double mx = 0.0;
        for (double *a : {C->m.g12, C->m.g13, C->m.g21, C->m.g23, C->m.g31, C->m.g32}) {
            TG_CUDA(cudaMemcpy(h.data(), a, G * sizeof(double), cudaMemcpyDeviceToHost));
            for (double v : h) mx = std::max(mx, std::fabs(v));
        }
        C->orthogonal = (mx == 0.0);
        // axis alignment: in every cell-face (csi, eta, zet) and face (icsi ..
        // kzet) metric only csi.y, eta.z, zet.x differ from zero by more than
        // the round-off of the metric evaluation (1e-12 of the array's largest
        // component; the face averages of a mesh of planes leave ~1e-16)
        const Metrics &M = C->m;
        auto amax = [&](const double *a) {
            TG_CUDA(cudaMemcpy(h.data(), a, G * sizeof(double), cudaMemcpyDeviceToHost));
            double r = 0.0;
            for (double v : h) r = std::max(r, std::fabs(v));
            return r;
        };
        bool ax = true;
        auto along = [&](const V3f<double> &v, int keep) {
            const double *c[3] = {v.x, v.y, v.z};
            const double d = amax(c[keep]);
            for (int q = 0; q < 3 && ax; q++)
                if (q != keep && !(amax(c[q]) <= 1e-12 * d)) ax = false;
        };
        for (const V3f<double> &v : {M.csi, M.icsi, M.jcsi, M.kcsi}) along(v, 1);
        for (const V3f<double> &v : {M.eta, M.ieta, M.jeta, M.keta}) along(v, 2);
        for (const V3f<double> &v : {M.zet, M.izet, M.jzet, M.kzet}) along(v, 0);
        C->axis_aligned = ax;
        graph_destroy(C);          // the captured step refers to the old solver buffers
        C->graph_failed = false;
        farm_destroy(C);           // turbine stencils refer to the old cell centres
        poisson_setup(C);
        C->has_mesh = true;
        return TG_OK;
    });
}

tg_status tg_set_field(tg_ctx *C, int32_t w, const double *host, int32_t halo)
{
    return guarded(C, [&]() -> tg_status {
        if (!host || halo < 0) return fail(C, TG_ERR_BAD_ARG, "bad field argument");
        if (w == TG_F_WALL_ADJ) {
            double *x, *y, *m;
            adj_wall_field(C, x, y, m);
            const size_t P = (size_t)C->g.mx * C->g.mz;
            std::vector<double> a(P), b(P), c(P);
            for (size_t q = 0; q < P; q++) { a[q] = host[3 * q]; b[q] = host[3 * q + 1]; c[q] = host[3 * q + 2]; }
            TG_CUDA(cudaMemcpy(x, a.data(), P * sizeof(double), cudaMemcpyHostToDevice));
            TG_CUDA(cudaMemcpy(y, b.data(), P * sizeof(double), cudaMemcpyHostToDevice));
            TG_CUDA(cudaMemcpy(m, c.data(), P * sizeof(double), cudaMemcpyHostToDevice));
            return TG_OK;
        }
        if (w == TG_F_QWALL || w == TG_F_SURF_THETA) {
            const size_t P = (size_t)C->g.mx * C->g.mz;
            TG_CUDA(cudaMemcpy(w == TG_F_QWALL ? C->s.qwall : C->s.surf_theta, host, P * sizeof(double), cudaMemcpyHostToDevice));
            if (w == TG_F_SURF_THETA) C->surf_set = true;
            return TG_OK;
        }
        V3f<double> v;
        double *sp = nullptr;
        if (adj_field(C, w, v, sp)) {
            if (sp) upload(C, host, halo, sp, nullptr, nullptr);
            else upload(C, host, halo, v.x, v.y, v.z);
            TG_CUDA(cudaStreamSynchronize(C->stream));
            return TG_OK;
        }
        if (vec_field(C, w, v)) upload(C, host, halo, v.x, v.y, v.z);
        else if ((sp = scal_field(C, w)) != nullptr) upload(C, host, halo, sp, nullptr, nullptr);
        else return fail(C, TG_ERR_BAD_ARG, "field not settable");
        TG_CUDA(cudaStreamSynchronize(C->stream));
        if (w == TG_F_RHS) C->clear_rhs = true;
        if (w == TG_F_DP) C->clear_dp = true;
        if ((w >= TG_F_CSI && w <= TG_F_KZET) || (w >= TG_F_AJ && w <= TG_F_KAJ)) C->met32_stale = true;
        return TG_OK;
    });
}

tg_status tg_get_field(tg_ctx *C, int32_t w, double *host, int32_t halo)
{
    return guarded(C, [&]() -> tg_status {
        if (!host || halo < 0) return fail(C, TG_ERR_BAD_ARG, "bad field argument");
        if (w == TG_F_TAUWALL) {
            const size_t P = (size_t)C->g.mx * C->g.mz;
            std::vector<double> a(P), b(P), c(P);
            TG_CUDA(cudaMemcpy(a.data(), C->s.twx, P * sizeof(double), cudaMemcpyDeviceToHost));
            TG_CUDA(cudaMemcpy(b.data(), C->s.twy, P * sizeof(double), cudaMemcpyDeviceToHost));
            TG_CUDA(cudaMemcpy(c.data(), C->s.twz, P * sizeof(double), cudaMemcpyDeviceToHost));
            for (size_t q = 0; q < P; q++) { host[3 * q] = a[q]; host[3 * q + 1] = b[q]; host[3 * q + 2] = c[q]; }
            return TG_OK;
        }
        if (w == TG_F_WALL_ADJ) {
            double *x, *y, *m;
            adj_wall_field(C, x, y, m);
            TG_CUDA(cudaStreamSynchronize(C->stream));
            const size_t P = (size_t)C->g.mx * C->g.mz;
            std::vector<double> a(P), b(P), c(P);
            TG_CUDA(cudaMemcpy(a.data(), x, P * sizeof(double), cudaMemcpyDeviceToHost));
            TG_CUDA(cudaMemcpy(b.data(), y, P * sizeof(double), cudaMemcpyDeviceToHost));
            TG_CUDA(cudaMemcpy(c.data(), m, P * sizeof(double), cudaMemcpyDeviceToHost));
            for (size_t q = 0; q < P; q++) { host[3 * q] = a[q]; host[3 * q + 1] = b[q]; host[3 * q + 2] = c[q]; }
            return TG_OK;
        }
        if (w == TG_F_QWALL || w == TG_F_SURF_THETA) {
            TG_CUDA(cudaStreamSynchronize(C->stream));
            const size_t P = (size_t)C->g.mx * C->g.mz;
            TG_CUDA(cudaMemcpy(host, w == TG_F_QWALL ? C->s.qwall : C->s.surf_theta, P * sizeof(double), cudaMemcpyDeviceToHost));
            return TG_OK;
        }
        V3f<double> v;
        double *sp = nullptr;
        if (adj_field(C, w, v, sp)) {
            if (sp) download(C, host, halo, sp, nullptr, nullptr);
            else download(C, host, halo, v.x, v.y, v.z);
            return TG_OK;
        }
        if (vec_field(C, w, v)) { download(C, host, halo, v.x, v.y, v.z); return TG_OK; }
        if (double *s = scal_field(C, w)) { download(C, host, halo, s, nullptr, nullptr); return TG_OK; }
        return fail(C, TG_ERR_BAD_ARG, "unknown field");
    });
}

}  // extern "C"

namespace {

constexpr int64_t kPetscVecClassId = 1211214;     // VEC_FILE_CLASSID

// entries per point of a field in the file (0: not a grid field)
int field_dof(tg_ctx *C, int w)
{
    if (w == TG_F_TAUWALL || w == TG_F_WALL_ADJ || w == TG_F_QWALL || w == TG_F_SURF_THETA || w < 0 || w >= TG_F_COUNT) return 0;
    if (w == TG_F_P_ADJ || scal_field(C, w)) return 1;
    return 3;
}

template <class T>
T byteswap(T v)
{
    unsigned char b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));
    for (size_t q = 0; q < sizeof(T) / 2; q++) std::swap(b[q], b[sizeof(T) - 1 - q]);
    std::memcpy(&v, b, sizeof(T));
    return v;
}

}  // namespace

extern "C" {

tg_status tg_write_field_petsc(tg_ctx *C, int32_t w, const char *path)
{
    return guarded(C, [&]() -> tg_status {
        const int dof = field_dof(C, w);
        if (!path || !dof) return fail(C, TG_ERR_BAD_ARG, "bad field or path");
        const size_t n = (size_t)C->g.size() * dof;
        std::vector<double> h(n);
        tg_status s = tg_get_field(C, w, h.data(), 0);
        if (s != TG_OK) return s;
        for (double &v : h) v = byteswap(v);
        FILE *f = std::fopen(path, "wb");
        if (!f) return fail(C, TG_ERR_BAD_ARG, std::string("cannot open ") + path);
        const int64_t hdr[2] = {byteswap(kPetscVecClassId), byteswap((int64_t)n)};
        bool ok = std::fwrite(hdr, sizeof(hdr), 1, f) == 1 && std::fwrite(h.data(), sizeof(double), n, f) == n;
        ok = (std::fclose(f) == 0) && ok;
        return ok ? TG_OK : fail(C, TG_ERR_BAD_ARG, std::string("write failed: ") + path);
    });
}

tg_status tg_read_field_petsc(tg_ctx *C, int32_t w, const char *path)
{
    return guarded(C, [&]() -> tg_status {
        const int dof = field_dof(C, w);
        if (!path || !dof) return fail(C, TG_ERR_BAD_ARG, "bad field or path");
        const size_t n = (size_t)C->g.size() * dof;
        FILE *f = std::fopen(path, "rb");
        if (!f) return fail(C, TG_ERR_BAD_ARG, std::string("cannot open ") + path);
        std::vector<double> h(n);
        unsigned char hb[16];
        bool ok = std::fread(hb, 1, 8, f) == 8;
        int64_t cls = 0, cnt = -1;
        if (ok) {
            int32_t c32, n32;
            std::memcpy(&c32, hb, 4);
            if (byteswap(c32) == (int32_t)kPetscVecClassId) {          // 32-bit header
                std::memcpy(&n32, hb + 4, 4);
                cls = kPetscVecClassId; cnt = byteswap(n32);
            } else {                                                  // 64-bit header
                std::memcpy(&cls, hb, 8);
                cls = byteswap(cls);
                int64_t n64;
                ok = std::fread(&n64, 8, 1, f) == 1;
                cnt = byteswap(n64);
            }
        }
        ok = ok && cls == kPetscVecClassId && cnt == (int64_t)n && std::fread(h.data(), sizeof(double), n, f) == n;
        std::fclose(f);
        if (!ok) return fail(C, TG_ERR_BAD_ARG, std::string("not a PETSc vector of ") + std::to_string(n) + " entries: " + path);
        for (double &v : h) v = byteswap(v);
        return tg_set_field(C, w, h.data(), 0);
    });
}

tg_status tg_init_from_cartesian(tg_ctx *C, const double *ucat, int32_t halo)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        if (!ucat) return fail(C, TG_ERR_BAD_ARG, "null ucat");
        // interior cells only: ghost cells are produced by the boundary conditions
        upload(C, ucat, halo, C->s.snap.x, C->s.snap.y, C->s.snap.z);
        const Grid g = C->g;
        k_copy_interior3<<<grid3(g.mx - 2, g.my - 2, g.mz - 2), block3(), 0, C->stream>>>(g, C->s.snap, C->s.ucat);
        init_from_cartesian(C);
        TG_CUDA(cudaStreamSynchronize(C->stream));
        return TG_OK;
    });
}

#define TG_STAGE(name, body)                                                                     \
    tg_status name(tg_ctx *C)                                                                    \
    {                                                                                            \
        return guarded(C, [&]() -> tg_status {                                                   \
            if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");                      \
            body;                                                                                \
            TG_CUDA(cudaStreamSynchronize(C->stream));                                           \
            return TG_OK;                                                                        \
        });                                                                                      \
    }

TG_STAGE(tg_contravariant_to_cartesian, contra_to_cart(C))
TG_STAGE(tg_update_nut, update_nut(C))
TG_STAGE(tg_update_wall_models, update_wall_models(C))
TG_STAGE(tg_grad_p, grad_p(C))
TG_STAGE(tg_buoyancy, buoyancy(C))
TG_STAGE(tg_explicit_rhs, explicit_rhs(C))
TG_STAGE(tg_solve_u, solve_u(C))
TG_STAGE(tg_update_cartesian_bcs, update_cartesian_bcs(C))
TG_STAGE(tg_update_contravariant_bcs, update_contravariant_bcs(C))
TG_STAGE(tg_sync_pressure, sync_pressure(C))
TG_STAGE(tg_update_wall_models_t,
         if (!C->prm.teqn) return fail(C, TG_ERR_STATE, "temperature equation off");
         if (const char *why = theta_wall_missing(C)) return fail(C, TG_ERR_STATE, why); update_wall_models_t(C))
TG_STAGE(tg_update_temperature_bcs,
         if (!C->prm.teqn) return fail(C, TG_ERR_STATE, "temperature equation off");
         if (const char *why = theta_wall_missing(C)) return fail(C, TG_ERR_STATE, why); update_temperature_bcs(C))

tg_status tg_set_surface_temperature(tg_ctx *C, int32_t n, const double *time, const double *temp)
{
    return guarded(C, [&]() -> tg_status {
        if (n < 2 || !time || !temp) return fail(C, TG_ERR_BAD_ARG, "a surface temperature series needs n >= 2 points");
        if (n > C->series_n) {
            // captured step graphs hold the old arrays: rebuild them
            graph_destroy(C);
            C->series_t = dallocd(C, (size_t)n);
            C->series_v = dallocd(C, (size_t)n);
        }
        TG_CUDA(cudaMemcpyAsync(C->series_t, time, sizeof(double) * n, cudaMemcpyHostToDevice, C->stream));
        TG_CUDA(cudaMemcpyAsync(C->series_v, temp, sizeof(double) * n, cudaMemcpyHostToDevice, C->stream));
        TG_CUDA(cudaStreamSynchronize(C->stream));
        if (n != C->series_n) graph_destroy(C);     // the count is a launch argument of the captured steps
        C->series_n = n;
        return TG_OK;
    });
}

tg_status tg_form_u(tg_ctx *C, double scale, int32_t zero_rhs)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        if (zero_rhs) TG_CUDA(cudaMemsetAsync(C->s.rhs.x, 0, 3 * sizeof(double) * C->g.size(), C->stream));
        form_u(C, C->s.rhs, scale);
        TG_CUDA(cudaStreamSynchronize(C->stream));
        return TG_OK;
    });
}

tg_status tg_solve_p(tg_ctx *C, tg_stats *st)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        tg_stats local{};
        int rc = solve_p(C, st ? st : &local);
        TG_CUDA(cudaStreamSynchronize(C->stream));
        if (rc == 2) return fail(C, TG_ERR_NAN, "non-finite residual in the pressure solve");
        return rc ? fail(C, TG_ERR_NOT_CONVERGED, "pressure solve reached its iteration cap") : TG_OK;
    });
}

tg_status tg_continuity_error(tg_ctx *C, double *md)
{
    return guarded(C, [&]() -> tg_status {
        if (!md) return fail(C, TG_ERR_BAD_ARG, "null output");
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        *md = continuity_error(C);
        return TG_OK;
    });
}

tg_status tg_step(tg_ctx *C, int32_t nsteps, tg_stats *st)
{
    return guarded(C, [&]() -> tg_status {
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        if (nsteps < 0) return fail(C, TG_ERR_BAD_ARG, "negative step count");
        if (const char *why = theta_wall_missing(C)) return fail(C, TG_ERR_STATE, why);
        tg_stats local{};
        tg_stats *s = st ? st : &local;
        *s = tg_stats{};
        step_stats_reset(C);
        TG_CUDA(cudaEventRecord(C->ev0, C->stream));
        int rc = 0;
        bool any = false, last = false;
        for (int n = 0; n < nsteps; n++) {
            int r = step(C, s, &last);
            any |= last;
            s->steps++;
            if (r == 2) { rc = 2; break; }
            rc |= r;
        }
        TG_CUDA(cudaEventRecord(C->ev1, C->stream));
        const int gr = step_stats_read(C, s, any, last);
        if (gr == 2) rc = 2;
        else if (rc != 2) rc |= gr;
        float ms = 0.f;
        TG_CUDA(cudaEventElapsedTime(&ms, C->ev0, C->ev1));
        s->seconds = ms * 1e-3;
        s->max_divergence = C->h_scal[16];
        check_nan(C);
        if (rc == 2) return fail(C, TG_ERR_NAN, "non-finite residual in the pressure solve");
        return rc ? fail(C, TG_ERR_NOT_CONVERGED, "pressure solve reached its iteration cap") : TG_OK;
    });
}

tg_status tg_set_graphs(tg_ctx *C, int32_t on)
{
    return guarded(C, [&]() -> tg_status {
        C->graphs = on != 0;
        if (!C->graphs) graph_destroy(C);
        C->graph_failed = false;
        return TG_OK;
    });
}

tg_status tg_graph_info(tg_ctx *C, int64_t *replays, int32_t *capture_failed)
{
    return guarded(C, [&]() -> tg_status {
        if (!replays || !capture_failed) return fail(C, TG_ERR_BAD_ARG, "null output");
        *replays = C->replays;
        *capture_failed = C->graph_failed ? 1 : 0;
        return TG_OK;
    });
}

tg_status tg_mesh_info(tg_ctx *C, int32_t *orthogonal, int32_t *axis_aligned)
{
    return guarded(C, [&]() -> tg_status {
        if (!orthogonal || !axis_aligned) return fail(C, TG_ERR_BAD_ARG, "null output");
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        *orthogonal = C->orthogonal ? 1 : 0;
        *axis_aligned = C->axis_aligned ? 1 : 0;
        return TG_OK;
    });
}

tg_status tg_momentum_info(tg_ctx *C, int32_t *outer, int32_t *inner, double *residual)
{
    return guarded(C, [&]() -> tg_status {
        if (!outer || !inner || !residual) return fail(C, TG_ERR_BAD_ARG, "null output");
        *outer = C->mom_outer;
        *inner = C->mom_inner;
        *residual = C->mom_res;
        return TG_OK;
    });
}

tg_status tg_step_host(tg_ctx *C, double *ucont, double *ucat, double *p, double *nut, int32_t halo, tg_stats *st)
{
    return guarded(C, [&]() -> tg_status {
        if (!ucont || !ucat || !p || halo < 0) return fail(C, TG_ERR_BAD_ARG, "null state");
        if (!C->has_mesh) return fail(C, TG_ERR_STATE, "mesh not set");
        if (const char *why = theta_wall_missing(C)) return fail(C, TG_ERR_STATE, why);
        upload(C, ucont, halo, C->s.ucont.x, C->s.ucont.y, C->s.ucont.z);
        upload(C, ucat, halo, C->s.ucat.x, C->s.ucat.y, C->s.ucat.z);
        upload(C, p, halo, C->s.p, nullptr, nullptr);
        // nut is recomputed from Ucat before any read: output only. It is
        // final after UpdateNut (the only writer), so it is copied out on the
        // copy stream from that point while the rest of the step runs.
        const bool nut_out = nut && C->prm.les && C->ev_nut;
        const Grid g = C->g;
        const size_t nn = (size_t)(g.mx + 2 * halo) * (g.my + 2 * halo) * (g.mz + 2 * halo);
        if (nut_out) {
            if (!C->copy_stream) TG_CUDA(cudaStreamCreateWithFlags(&C->copy_stream, cudaStreamNonBlocking));
            if (C->stage_nut_bytes < nn * sizeof(double)) {
                TG_CUDA(cudaStreamSynchronize(C->copy_stream));
                C->stage_nut = (double *)dalloc(C, nn * sizeof(double));
                C->stage_nut_bytes = nn * sizeof(double);
            }
            // keep the caller's halo entries: start from the caller's array
            if (halo > 0)
                TG_CUDA(cudaMemcpyAsync(C->stage_nut, nut, nn * sizeof(double), cudaMemcpyHostToDevice, C->copy_stream));
        }
        tg_stats local{};
        tg_stats *s = st ? st : &local;
        *s = tg_stats{};
        step_stats_reset(C);
        bool rep = false;
        int rc = step(C, s, &rep);
        s->steps = 1;
        if (nut_out) {
            TG_CUDA(cudaStreamWaitEvent(C->copy_stream, C->ev_nut, 0));
            k_soa_to_aos<<<grid3(g.mx, g.my, g.mz), block3(), 0, C->copy_stream>>>(g, C->stage_nut, halo, C->s.nut, nullptr, nullptr);
            TG_CUDA(cudaGetLastError());
            TG_CUDA(cudaMemcpyAsync(nut, C->stage_nut, nn * sizeof(double), cudaMemcpyDeviceToHost, C->copy_stream));
        }
        download(C, ucont, halo, C->s.ucont.x, C->s.ucont.y, C->s.ucont.z);
        download(C, ucat, halo, C->s.ucat.x, C->s.ucat.y, C->s.ucat.z);
        download(C, p, halo, C->s.p, nullptr, nullptr);
        if (nut_out) TG_CUDA(cudaStreamSynchronize(C->copy_stream));
        const int gr = step_stats_read(C, s, rep, rep);
        if (rep) rc = gr;
        s->max_divergence = C->h_scal[16];
        if (rc == 2) return fail(C, TG_ERR_NAN, "non-finite residual in the pressure solve");
        return rc ? fail(C, TG_ERR_NOT_CONVERGED, "pressure solve reached its iteration cap") : TG_OK;
    });
}

}  // extern "C"

// ============================================================== profiling
namespace tg {

int Profiler::slot(const char *name)
{
    for (size_t q = 0; q < acc.size(); q++) if (acc[q].name == name) return (int)q;
    acc.push_back(ProfAcc{name, 0, 0.0});
    return (int)acc.size() - 1;
}

void prof_begin(tg_ctx *C, const char *name, cudaEvent_t *a, cudaEvent_t *b, int *slot)
{
    Profiler &P = C->prof;
    if (P.next + 2 > P.pool.size()) {
        // pool exhausted: resolve what is pending and reuse the events
        prof_flush(C);
        if (P.next + 2 > P.pool.size()) {
            for (int q = 0; q < 256; q++) { cudaEvent_t e; TG_CUDA(cudaEventCreate(&e)); P.pool.push_back(e); }
        }
    }
    *a = P.pool[P.next++];
    *b = P.pool[P.next++];
    *slot = P.slot(name);
    TG_CUDA(cudaEventRecord(*a, C->stream));
}

void prof_end(tg_ctx *C, cudaEvent_t a, cudaEvent_t b, int slot)
{
    TG_CUDA(cudaEventRecord(b, C->stream));
    C->prof.pending.push_back(ProfPending{slot, a, b});
}

void prof_flush(tg_ctx *C)
{
    Profiler &P = C->prof;
    if (P.pending.empty()) { P.next = 0; return; }
    TG_CUDA(cudaStreamSynchronize(C->stream));
    for (auto &r : P.pending) {
        float ms = 0.f;
        TG_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        P.acc[r.slot].launches++;
        P.acc[r.slot].ms += ms;
    }
    P.pending.clear();
    P.next = 0;
}

}  // namespace tg

extern "C" {

tg_status tg_prof_enable(tg_ctx *C, int32_t on)
{
    return guarded(C, [&]() -> tg_status { prof_flush(C); C->prof.on = on != 0; return TG_OK; });
}

tg_status tg_prof_reset(tg_ctx *C)
{
    return guarded(C, [&]() -> tg_status { prof_flush(C); C->prof.acc.clear(); return TG_OK; });
}

int32_t tg_prof_count(tg_ctx *C)
{
    if (!C) return -1;
    try { prof_flush(C); } catch (...) { return -1; }
    return (int32_t)C->prof.acc.size();
}

tg_status tg_prof_get(tg_ctx *C, int32_t index, char *name, int64_t *launches, double *ms)
{
    return guarded(C, [&]() -> tg_status {
        prof_flush(C);
        if (index < 0 || index >= (int32_t)C->prof.acc.size() || !name || !launches || !ms) return fail(C, TG_ERR_BAD_ARG, "bad profile index");
        const ProfAcc &a = C->prof.acc[index];
        std::snprintf(name, 64, "%s", a.name.c_str());
        *launches = a.launches;
        *ms = a.ms;
        return TG_OK;
    });
}

}  // extern "C"
