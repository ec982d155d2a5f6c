// Internal declarations of the B200 TOSCA time-step library.
//
// Device layout: every field lives on the global DMDA extent (mx, my, mz),
// [k][j][i] with i fastest, as structure-of-arrays (one contiguous plane per
// vector component) so that a warp reading 32 consecutive i issues one
// 256-byte coalesced transaction per component. Out-of-range indices of a
// periodic direction wrap modulo the extent, which is exactly what a
// single-rank PETSc local vector returns for DM_BOUNDARY_PERIODIC.
#pragma once

#include <functional>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/tosca_gpu.h"

namespace tg {

// ------------------------------------------------------------------- grid --
struct Grid {
    int mx, my, mz;
    int pi, pj, pk;   // periodic (type 2) per direction

    __host__ __device__ __forceinline__ int wi(int i) const { if (pi) { if (i < 0) i += mx; else if (i >= mx) i -= mx; } return i; }
    __host__ __device__ __forceinline__ int wj(int j) const { if (pj) { if (j < 0) j += my; else if (j >= my) j -= my; } return j; }
    __host__ __device__ __forceinline__ int wk(int k) const { if (pk) { if (k < 0) k += mz; else if (k >= mz) k -= mz; } return k; }
    // wrapped linear index (callers guarantee in-range indices in non-periodic directions)
    __host__ __device__ __forceinline__ int id(int k, int j, int i) const { return (wk(k) * my + wj(j)) * mx + wi(i); }
    // unwrapped linear index
    __host__ __device__ __forceinline__ int lin(int k, int j, int i) const { return (k * my + j) * mx + i; }
    __host__ __device__ __forceinline__ int64_t size() const { return (int64_t)mx * my * mz; }
};

// SoA vector field (three planes of the same extent)
template <class T>
struct V3f {
    T *x, *y, *z;
};

template <class T>
struct R3 { T x, y, z; };

template <class T>
__device__ __forceinline__ R3<T> ld3(const V3f<T> &f, int q) { return R3<T>{f.x[q], f.y[q], f.z[q]}; }
template <class T>
__device__ __forceinline__ void st3(const V3f<T> &f, int q, R3<T> v) { f.x[q] = v.x; f.y[q] = v.y; f.z[q] = v.z; }
template <class T>
__device__ __forceinline__ R3<T> operator+(R3<T> a, R3<T> b) { return R3<T>{a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
__device__ __forceinline__ R3<T> operator-(R3<T> a, R3<T> b) { return R3<T>{a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T>
__device__ __forceinline__ R3<T> operator*(T s, R3<T> a) { return R3<T>{s * a.x, s * a.y, s * a.z}; }
template <class T>
__device__ __forceinline__ T dot3(R3<T> a, R3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// metric fields (mesh.c:630-1976) on the device
struct Metrics {
    V3f<double> cent, csi, eta, zet, icsi, ieta, izet, jcsi, jeta, jzet, kcsi, keta, kzet;
    double *aj, *iaj, *jaj, *kaj;
    // face metric tensor g_qr * face-aj with boundary remapping (peqn.c:791-849)
    double *g11, *g12, *g13, *g21, *g22, *g23, *g31, *g32, *g33;
};

// the metric fields read by the momentum stencils at storage precision T:
// views of Metrics for FP64, converted copies for the mixed-precision mode
template <class T>
struct FaceMet {
    V3f<T> csi, eta, zet, icsi, ieta, izet, jcsi, jeta, jzet, kcsi, keta, kzet;
    T *aj, *iaj, *jaj, *kaj;
    T *flt2;      // Smagorinsky filter width squared, ((1/aj)^(1/3))^2 (les.c:2204-2514)
};

// FormU work planes at storage precision T: face fluxes per direction and
// their cell divergence
template <class T>
struct FluxWork {
    V3f<T> f1, f2, f3, fp;
};

// physical state and work arrays
struct State {
    V3f<double> ucont, ucont_o, ucat, rhs, dp, btheta, btheta_o, gcont, utmp, snap;
    V3f<double> source;          // ueqn->sourceU, cell-centred Cartesian body force
    V3f<double> farmcont;        // farm->sourceFarmCont, contravariant turbine body force (tg_farm.cu)
    // temperature transport (tg_teqn.cu): lDivT, lViscT face fluxes, Rhs, Tmprt_o, TmprtTmp
    V3f<double> tdiv, tvisc;
    double *trhs, *tmprt_o, *ttmp;
    V3f<double> rhs_o;           // ueqn->Rhs_o: FormU of the last step's final state (CN)
    double *p, *phi, *nut, *tmprt, *ssnap;
    // jLeft wall model (plane mz x mx)
    double *twx, *twy, *twz, *umean, *ufx, *ufy, *ufz;
    // jLeft thetaWallFunction (plane mz x mx): qWall.z and surfaceTheta
    double *qwall, *surf_theta;
};

struct Params {
    int bc[6];
    double bc_value[18];           // TG_BC_FIXED_VALUE: Cartesian velocity of patch p at [3p, 3p+2]
    // TG_BC_INLET_LOG on kLeft: uTau, roughness, hInv, unit direction, and
    // the ground level (the lowest mesh node, set with the mesh)
    double inlet_u_tau, inlet_z0, inlet_h_inv, inlet_dir[3], grnd;
    int nut_bc[6];
    double nut_bc_value[6];
    int curvilinear, les, div_scheme, buoyancy, mean_grad_p, source, farm;
    double cs, nu, dt, t_ref, mgp[3], z0, kappa;
    int teqn, t_bc[6];
    double prandtl, t_bc_value[6];
    // jLeft thetaWallFunction (0: none, else TG_TWALL_*), its constants, and
    // whether its qWall corrects the velocity wall function (wall_coupled)
    int t_wall, t_wall_localized, wall_coupled;
    double tw_qwall, tw_heating, tw_kappa, tw_theta_ref, tw_z0, tw_gamma_m, tw_gamma_h, tw_alpha_h;
    double wall_gamma_m, wall_theta_ref;
};

// ------------------------------------------------------------------------
// calculateNormal (inline.h:1210-1268): unit covariant direction of a cell
// ------------------------------------------------------------------------
__device__ __forceinline__ void calc_normal(R3<double> csi, R3<double> eta, R3<double> zet, int dir, R3<double> &n)
{
    const double a11 = csi.x, a12 = csi.y, a13 = csi.z;
    const double a21 = eta.x, a22 = eta.y, a23 = eta.z;
    const double a31 = zet.x, a32 = zet.y, a33 = zet.z;
    double det = a11 * (a33 * a22 - a32 * a23) - a21 * (a33 * a12 - a32 * a13) + a31 * (a23 * a12 - a22 * a13);
    double x, y, z;
    if (dir == 0) {        // G[:,0]
        x = (a33 * a22 - a32 * a23) / det; y = -(a33 * a21 - a31 * a23) / det; z = (a32 * a21 - a31 * a22) / det;
    } else if (dir == 1) { // G[:,1]
        x = -(a33 * a12 - a32 * a13) / det; y = (a33 * a11 - a31 * a13) / det; z = -(a32 * a11 - a31 * a12) / det;
    } else {               // G[:,2]
        x = (a23 * a12 - a22 * a13) / det; y = -(a23 * a11 - a21 * a13) / det; z = (a22 * a11 - a21 * a12) / det;
    }
    double sm = sqrt(x * x + y * y + z * z);
    n = R3<double>{x / sm, y / sm, z / sm};
}

struct PoissonCtx;   // tg_poisson.cu
struct AdjState;     // tg_adjoint.cu
struct Farm;         // tg_farm.cu
struct CnWork;       // tg_cn.cu
struct ImexWork;     // tg_imex.cu
struct GmresWork;    // tg_imex.cu
struct JfnkWork;     // tg_cn.cu

// per-kernel event timing (tosca_gpu_prof.h)
struct ProfPending { int slot; cudaEvent_t a, b; };
struct ProfAcc { std::string name; int64_t launches = 0; double ms = 0.0; };
struct Profiler {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    size_t next = 0;
    std::vector<ProfPending> pending;
    std::vector<ProfAcc> acc;
    int slot(const char *name);
};

}  // namespace tg

struct tg_ctx {
    tg_config cfg{};
    tg::Grid g{};
    tg::Params prm{};
    tg::Metrics m{};
    tg::State s{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<void *> allocs;          // every device allocation of this context
    double *d_red = nullptr;             // reduction scratch (partials)
    double *d_scal = nullptr;            // device scalars
    double *h_scal = nullptr;            // pinned host mirror of scalars
    double *stage = nullptr;             // staging buffer for AoS host transfers
    size_t stage_bytes = 0;
    // tg_step_host's early nut download: nut is final once UpdateNut has run,
    // so its copy overlaps the rest of the step on its own stream and buffer
    cudaEvent_t ev_nut = nullptr;        // recorded after UpdateNut (an external event node in the step graph)
    cudaStream_t copy_stream = nullptr;
    double *stage_nut = nullptr;
    size_t stage_nut_bytes = 0;
    int red_blocks = 0;
    bool has_mesh = false;
    bool orthogonal = true;              // all cross metric-tensor terms vanish
    // csi || y, eta || z, zet || x at every point of every cell and face
    // metric up to round-off (the reference's i -> y, j -> z, k -> x axes on
    // a mesh of planes): FormU reads only those components
    bool axis_aligned = false;
    bool ufilt_set = false;
    bool surf_set = false;               // thetaWallFunction -3 surfaceTheta seeded
    double *series_t = nullptr, *series_v = nullptr;   // thetaWallFunction -4 surface temperature series
    int series_n = 0;
    int it = 0;
    // mixed precision: FP32 copies of the stencil metrics (and FP32 FormU
    // planes when the policy stores the face fluxes in FP32)
    bool mixed = false;
    // which momentum stages read the FP32 metric copies (and compute in FP32)
    struct {
        bool contra_m32 = false;     // contravariantToCartesian: FP32 metrics
        bool contra_a32 = false;     //   ... and FP32 arithmetic
        bool visc32 = false;         // FormU viscous fluxes
        bool flux32 = false;         // FormU face-flux planes stored in FP32
        bool rhs32 = false;          // FormU face assembly metrics
        bool smag32 = false;         // Smagorinsky eddy viscosity
        bool gradp32 = false;        // GradP
        bool proj32 = false;         // ProjectVelocity (FP64 arithmetic)
    } pol;
    bool met32_stale = true;             // metrics changed since the FP32 copies were made
    tg::FaceMet<double> fm64{};
    tg::FaceMet<float> fm32{};
    tg::FluxWork<double> fw64{};
    tg::FluxWork<float> fw32{};
    // a caller wrote Rhs / dP through tg_set_field: the next evaluation clears
    // the points outside the ones it writes
    bool clear_rhs = false, clear_dp = false;
    std::string err;
    tg::PoissonCtx *pois = nullptr;
    tg::AdjState *adj = nullptr;         // adjoint fields, tape and checkpoints (tg_adjoint.cu)
    tg::Farm *farm = nullptr;            // actuator-disk turbines (tg_farm.cu)
    tg::CnWork *cn = nullptr;            // Crank-Nicolson Newton-Krylov work (tg_cn.cu)
    tg::ImexWork *imex = nullptr;        // IMEX GMRES work (tg_imex.cu)
    tg::GmresWork *tgm = nullptr;        // GMRES work of the ABBE temperature solve (tg_teqn.cu)
    double *tconv = nullptr, *tconv_o = nullptr;   // teqn->RhsConv, RhsConv_o (ABBE)
    int t_its = 0;                       // GMRES iterations of the last ABBE temperature solve
    tg::JfnkWork *tsn = nullptr;         // Newton-Krylov work of the BE/BDF2 temperature solve (tg_teqn.cu)
    double *tmprt_oo = nullptr;          // teqn->Tmprt_oo (BDF2)
    double *node_z = nullptr;            // z of node (k, j, i) (ghGradRhoK, p_tilde)
    // last implicit momentum solve: Newton steps or IMEX stages, Krylov
    // operator products, last Krylov residual estimate
    int mom_outer = 0, mom_inner = 0;
    double mom_res = 0.0;
    bool taping = false;                 // the running step records its stage states
    // CUDA graph of a whole step (tg_step.cu): built on the first step that can
    // be captured, replayed afterwards
    cudaGraphExec_t step_exec = nullptr;
    cudaGraphExec_t step_exec_taped = nullptr;   // the same step recording its stages
    bool graphs = true;                  // tg_set_graphs
    int64_t replays = 0;
    bool graph_failed = false;
    cudaStream_t aux[2] = {nullptr, nullptr};   // capture streams of conditional bodies
    tg::Profiler prof;
};

namespace tg {

// error helpers ----------------------------------------------------------------
struct CudaError {
    cudaError_t e;
    const char *what;
};
#define TG_CUDA(call)                                                            \
    do {                                                                         \
        cudaError_t _e = (call);                                                 \
        if (_e != cudaSuccess) throw ::tg::CudaError{_e, #call};                 \
    } while (0)

void *dalloc(tg_ctx *C, size_t bytes);        // zeroed device allocation owned by C
inline double *dallocd(tg_ctx *C, size_t n) { return (double *)dalloc(C, n * sizeof(double)); }
V3f<double> dalloc3(tg_ctx *C, size_t n);

// NaN-propagating maximum (fmax ignores NaN operands)
__device__ __forceinline__ double nanmax(double a, double b) { return (a != a || b != b) ? (a + b) : fmax(a, b); }

// per-slot combiners of block_reduce
struct RedSum { __device__ __forceinline__ double operator()(double a, double b) const { return a + b; } };
struct RedMax { __device__ __forceinline__ double operator()(double a, double b) const { return fmax(a, b); } };
struct RedNanMax { __device__ __forceinline__ double operator()(double a, double b) const { return nanmax(a, b); } };

// Block-wide reduction of NV per-thread values for a block of NT threads (NT
// a power of two, 64..1024): a shuffle tree inside each warp, the warp
// results through shared memory, a second shuffle tree in warp 0. The
// combination order is fixed, so the result is deterministic; it is valid in
// thread 0 only. Every thread of the block must call it.
template <int NT, int NV, class... Ops>
__device__ __forceinline__ void block_reduce(double (&v)[NV], Ops... ops)
{
    static_assert(NT >= 64 && NT <= 1024 && (NT & (NT - 1)) == 0, "block size");
    static_assert(sizeof...(Ops) == NV, "one combiner per slot");
    constexpr int NW = NT / 32;
    __shared__ double ws[NV][NW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        int q = 0;
        ((v[q] = ops(v[q], __shfl_down_sync(0xffffffffu, v[q], o)), q++), ...);
    }
    if (lane == 0) {
        #pragma unroll
        for (int q = 0; q < NV; q++) ws[q][w] = v[q];
    }
    __syncthreads();
    if (w == 0) {
        #pragma unroll
        for (int q = 0; q < NV; q++) v[q] = ws[q][lane < NW ? lane : 0];
        #pragma unroll
        for (int o = NW / 2; o > 0; o >>= 1) {
            int q = 0;
            ((v[q] = ops(v[q], __shfl_down_sync(0xffffffffu, v[q], o)), q++), ...);
        }
    }
}

// block_reduce of one sum, returned to every thread of the block
template <int NT>
__device__ __forceinline__ double block_sum_all(double x)
{
    __shared__ double out;
    double v[1] = {x};
    block_reduce<NT>(v, RedSum{});
    if (threadIdx.x == 0) out = v[0];
    __syncthreads();
    const double r = out;
    __syncthreads();
    return r;
}

// profiling brackets around one kernel launch on C->stream
void prof_begin(tg_ctx *C, const char *name, cudaEvent_t *a, cudaEvent_t *b, int *slot);
void prof_end(tg_ctx *C, cudaEvent_t a, cudaEvent_t b, int slot);
void prof_flush(tg_ctx *C);
#define TG_PROF(C, name, ...)                                                       \
    do {                                                                               \
        if ((C)->prof.on) {                                                            \
            cudaEvent_t _a, _b; int _s;                                                \
            ::tg::prof_begin((C), (name), &_a, &_b, &_s);                              \
            __VA_ARGS__;                                                               \
            ::tg::prof_end((C), _a, _b, _s);                                           \
        } else {                                                                       \
            __VA_ARGS__;                                                                    \
        }                                                                              \
    } while (0)

// launch helpers: 3-D blocks with i fastest
constexpr int BX = 32, BY = 4, BZ = 2;
inline dim3 grid3(int ni, int nj, int nk) { return dim3((ni + BX - 1) / BX, (nj + BY - 1) / BY, (nk + BZ - 1) / BZ); }
inline dim3 block3() { return dim3(BX, BY, BZ); }

// stage entry points (tg_step.cu)
void metrics_from_nodes(tg_ctx *C, const double *d_nodes);
void alloc_precision_work(tg_ctx *C);         // FP64 views, FP32 copies (mixed mode)
void refresh_met32(tg_ctx *C);
void refresh_filter(tg_ctx *C);          // FP64 Smagorinsky filter widths after a mesh change                // FP32 metric copies from the FP64 fields
void contra_to_cart(tg_ctx *C);
void reset_cell_periodic(tg_ctx *C, V3f<double> v);
void reset_cell_periodic_s(tg_ctx *C, double *v);
void reset_face_periodic(tg_ctx *C, V3f<double> v);
void reset_no_penetration(tg_ctx *C);
void update_cartesian_bcs(tg_ctx *C);
void update_contravariant_bcs(tg_ctx *C);
void adjust_fluxes(tg_ctx *C);               // adjustFluxesLocal (inflow/outflow patches only)
void update_scalar_ghosts(tg_ctx *C, double *v);
void update_nut(tg_ctx *C);
void update_wall_models(tg_ctx *C);
void grad_p(tg_ctx *C);
void buoyancy(tg_ctx *C);
// formMode (ueqn_solvers.c:17): 0 convection + viscosity, 1 convection, 2 viscosity
void form_u(tg_ctx *C, V3f<double> rhs, double scale, int mode = 0);
void form_u_again(tg_ctx *C, V3f<double> rhs, double scale);
void explicit_rhs(tg_ctx *C, int mode = 0);
void solve_u(tg_ctx *C);
int solve_p(tg_ctx *C, tg_stats *st);
double continuity_error(tg_ctx *C);
void sync_pressure(tg_ctx *C);
void init_from_cartesian(tg_ctx *C);
int step(tg_ctx *C, tg_stats *st, bool *replayed = nullptr);
void step_stats_reset(tg_ctx *C);            // zero the SC_G and SC_ADJ slots before a run of steps
// after a run of steps: copy d_scal[16..SC_IT) to h_scal, merge the statistics of
// replayed steps into s (last: the final step was replayed); returns 0, 1
// (iteration cap) or 2 (non-finite residual) for the replayed steps
int step_stats_read(tg_ctx *C, tg_stats *s, bool any, bool last);

// device reductions (tg_reduce.cu): result written to d_out[0]
void reduce_max_abs_div(tg_ctx *C, double *d_out);

// Poisson (tg_poisson.cu)
void poisson_setup(tg_ctx *C);
void poisson_destroy(tg_ctx *C);
int poisson_solve(tg_ctx *C, tg_stats *st);
void poisson_solve_capture(tg_ctx *C);       // the same solve with device-side loop control
// device scalar slots (C->d_scal): statistics of captured solves, as offsets
// from a base (SC_G: forward step, SC_ADJ: transposed solve), and the step counter
constexpr int ST_IT = 0, ST_RES0 = 1, ST_RES = 2, ST_TOT = 3, ST_NOCONV = 4, ST_NAN = 5, ST_COUNT = 6;
constexpr int SC_G = 60, SC_ADJ = 70, SC_IT = 80;
// solutions in the Poisson guess history (0, 1, 2 or more: order of the extrapolation)
constexpr int SC_PHIST = 96;
// thetaWallFunction averaged model: plane means and the resulting qWall
constexpr int SC_TWALL = 24;       // 24..26 plane means, 27 qWall, 28 surface temperature (-4)
// number of transposed-solve solutions in the adjoint guess history
constexpr int SC_LHIST = 76;
// adjustFluxesLocal: total inflow and outflow through the inflow/outflow patches
constexpr int SC_FLUX = 100;
constexpr int SC_GIT = SC_G + ST_IT, SC_GRES0 = SC_G + ST_RES0, SC_GRES = SC_G + ST_RES, SC_GTOT = SC_G + ST_TOT,
              SC_GNOCONV = SC_G + ST_NOCONV, SC_GNAN = SC_G + ST_NAN;
void poisson_solve_adjoint_capture(tg_ctx *C, const double *rhs, double *lam, double rtol);
// initial guess of a transposed pressure solve: lam extrapolated from the
// solutions of the previously reversed steps (lam, lp, lp2; hist counts them),
// of the order the forward solve uses; the history shifts
void adjoint_guess(tg_ctx *C, double *lam, double *lp, double *lp2, double *hist);
// capture body() (launches on C->stream) into an instantiated graph; false when
// capture or instantiation fails (nothing is left capturing)
bool capture_graph(tg_ctx *C, cudaGraphExec_t *out, const std::function<void()> &body);
void adj_graph_destroy(tg_ctx *C);
// temperature transport (tg_teqn.cu)
// Crank-Nicolson momentum step (tg_cn.cu)
int solve_u_cn(tg_ctx *C, tg_stats *st);
// Jacobian-free Newton-Krylov root of F, Feval(U, F) (tg_cn.cu): the guess and
// the root in the work's U
JfnkWork *jfnk_alloc(tg_ctx *C, int64_t n, int m);
void jfnk_free(JfnkWork *W);
double *jfnk_u(JfnkWork *W);
int jfnk_solve(tg_ctx *C, JfnkWork &W, const std::function<void(const double *, double *)> &Feval, double atol, double rtol,
               int maxit, int &newton, int &linear, double &fn_out);
void cn_destroy(tg_ctx *C);
bool imex_scheme(int ddt);                                         // tg_imex.cu
// restarted GMRES as PETSc's KSPGMRES (tg_imex.cu): A(v, Av) writes A v
GmresWork *gmres_alloc(tg_ctx *C, int64_t n, int m);
void gmres_free(GmresWork *W);
int gmres_solve(tg_ctx *C, GmresWork &W, const std::function<void(const double *, double *)> &A, const double *b, double *x,
                double rtol, double atol, int &its, double &res);
int solve_u_imex(tg_ctx *C);
void imex_destroy(tg_ctx *C);
void cn_build_bu(tg_ctx *C, V3f<double> bu, bool half_rhs_o);   // tg_step.cu
void mask_non_resolved(tg_ctx *C, V3f<double> v);               // resetNonResolvedCellFaces on v
void contra_to_cart_stage(tg_ctx *C);
int solve_t(tg_ctx *C);      // 0, or the ABBE GMRES status (1 iteration cap, 2 breakdown)
void update_temperature_bcs(tg_ctx *C);
void update_wall_models_t(tg_ctx *C);   // UpdateWallModelsT: jLeft thetaWallFunction qWall
// thetaWallFunction -4 without its surface temperature series: the error text, else nullptr
const char *theta_wall_missing(const tg_ctx *C);
// wind farm (tg_farm.cu)
void farm_update(tg_ctx *C);                 // sampling, forces, projection, face body force
void farm_destroy(tg_ctx *C);
bool farm_field(tg_ctx *C, int w, V3f<double> &out);   // TG_F_FARM_FORCE / TG_F_FARM_CONT
// reversed step: adjoint of the face body force of one stage accumulates
// from the stage's Rhs adjoint; farm_adj_finish turns the step's sum into the
// C_T' gradient and the adjoint of the sampled Ucat (ucat_n: the taped Ucat
// at the step's start; ca: its adjoint)
void farm_adj_begin(tg_ctx *C);
void farm_adj_stage(tg_ctx *C, V3f<double> ra);
void farm_adj_finish(tg_ctx *C, V3f<double> ucat_n, V3f<double> ca);
bool tape_in_work(const tg_ctx *C);          // the step tapes into the fixed work tape
void set_device_step(tg_ctx *C);             // C->d_scal[SC_IT] <- C->it
void graph_destroy(tg_ctx *C);

// adjoint (tg_adjoint.cu)
void tape_step_start(tg_ctx *C);
void tape_nut(tg_ctx *C);
void tape_stage(tg_ctx *C);
bool adj_field(tg_ctx *C, int w, V3f<double> &v, double *&s);   // adjoint fields (allocated on first use)
bool adj_wall_field(tg_ctx *C, double *&x, double *&y, double *&m);   // TG_F_WALL_ADJ planes
void adj_destroy(tg_ctx *C);
int poisson_solve_adjoint(tg_ctx *C, const double *rhs, double *lam, double rtol, tg_stats *st);
double *poisson_x(tg_ctx *C);
double *poisson_xprev(tg_ctx *C);
double *poisson_xprev2(tg_ctx *C);
int64_t poisson_n(tg_ctx *C);

}  // namespace tg
