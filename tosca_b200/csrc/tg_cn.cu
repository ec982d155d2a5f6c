// Crank-Nicolson momentum step (ddtScheme CN: UeqnSNES and SNESFuncEval,
// ueqn_solvers.c:1087-1272). The implicit equation
//   F(U) = dt [bU + s FormU(U)] (zero at non-resolved faces) - U + U_o = 0,
// s = 1/2 (1 on the first step), with the constant part
//   bU = -dP + buoyancy (AB2) + 1/2 Rhs_o + turbine force + sourceU + meanGradP,
// Rhs_o = FormU of the previous step's final state (main.c:214-272), is solved
// by a Jacobian-free Newton-Krylov iteration from U = U_o: restarted GMRES on
// J d = -F with the products J v = (F(U + h v) - F(U)) / h, h = sqrt(eps)
// sqrt(1 + |U|) / |v| (PETSc's MATMFFD_WP differencing), full Newton steps
// halved while they do not decrease |F|. Stopping: |F| <= max(snes_atol,
// snes_rtol |F_0|) (SNESSetTolerances) or snes_maxit Newton steps.
//
// The reference adds meanGradPForcing to ueqn->Rhs instead of the function
// argument in SNESFuncEval (ueqn_solvers.c:1258), which leaves the term out of
// F and corrupts the residual stored for the matrix-free products; here the
// term is part of bU, as in the explicit schemes.
//
// The Newton-Krylov iteration (jfnk_solve) takes F as a callback and also
// solves the BE/BDF2 temperature step (SNESFuncEvalT, tg_teqn.cu).
#include <cmath>
#include <vector>

#include "tg_internal.cuh"

namespace tg {

// Jacobian-free Newton-Krylov work on n unknowns (jfnk_solve)
struct JfnkWork {
    int m = 30;                       // GMRES restart
    int64_t n = 0;
    double *U = nullptr, *F = nullptr, *W = nullptr, *FW = nullptr;   // iterate, F(U), correction, F(probe)
    double *V = nullptr;              // (m + 1) Krylov vectors of n
    double *part = nullptr;           // dot-product partials
    int nb = 0;
};

struct CnWork {
    JfnkWork j;                       // n = 3 G
    V3f<double> bu{};
};

namespace {

constexpr int DB = 256;

__global__ void __launch_bounds__(DB) k_dot_part(int64_t n, const double *a, const double *b, double *part)
{
    double v[1] = {0.0};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) v[0] += a[t] * b[t];
    block_reduce<DB>(v, RedSum{});
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}
__global__ void __launch_bounds__(DB) k_dot_sum(const double *part, int nb, double *out)
{
    double v[1] = {0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v[0] += part[b];
    block_reduce<DB>(v, RedSum{});
    if (threadIdx.x == 0) out[0] = v[0];
}
// y = a x + b y
__global__ void k_axpby(int64_t n, double a, const double *x, double b, double *y)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) y[t] = a * x[t] + b * y[t];
}
// w = x + a y
__global__ void k_waxpy(int64_t n, double *w, const double *x, double a, const double *y)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) w[t] = x[t] + a * y[t];
}
// dt-scaling before the non-resolved mask (VecScale then resetNonResolvedCellFaces)
__global__ void k_scale(int64_t n, double a, double *x)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) x[t] *= a;
}
// F = F - U + U_o
__global__ void k_cn_time(int64_t n, double *F, const double *U, const double *Uo)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        double f = F[t] + -1.0 * U[t];
        F[t] = f + 1.0 * Uo[t];
    }
}

inline int nblk(int64_t n) { int64_t b = (n + DB - 1) / DB; return (int)(b < 148 * 8 ? b : 148 * 8); }

double dot(tg_ctx *C, JfnkWork &W, const double *a, const double *b, int64_t n)
{
    k_dot_part<<<W.nb, DB, 0, C->stream>>>(n, a, b, W.part);
    k_dot_sum<<<1, DB, 0, C->stream>>>(W.part, W.nb, C->d_scal + 90);
    TG_CUDA(cudaMemcpyAsync(C->h_scal + 90, C->d_scal + 90, sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaStreamSynchronize(C->stream));
    return C->h_scal[90];
}

void jfnk_init(tg_ctx *C, JfnkWork &W, int64_t n, int m)
{
    W.m = m;
    W.n = n;
    W.U = dallocd(C, n); W.F = dallocd(C, n); W.W = dallocd(C, n); W.FW = dallocd(C, n);
    W.V = dallocd(C, (size_t)(m + 1) * n);
    W.nb = nblk(n);
    W.part = dallocd(C, W.nb);
}

CnWork &work(tg_ctx *C)
{
    if (!C->cn) {
        CnWork *W = new CnWork();
        const size_t G = (size_t)C->g.size();
        W->bu = dalloc3(C, G);
        C->cn = W;
        jfnk_init(C, W->j, 3 * (int64_t)G, C->cfg.gmres_restart > 0 ? C->cfg.gmres_restart : 30);
    }
    return *C->cn;
}

}  // namespace

void cn_destroy(tg_ctx *C)
{
    delete C->cn;        // device buffers are owned by the context allocation list
    C->cn = nullptr;
}

// SNESFuncEval (ueqn_solvers.c:1203-1272): F(U) into Fout; leaves Ucont = U
// and the Ucat of U in the state, as the reference does
static void cn_eval(tg_ctx *C, CnWork &W, const double *U, double *F, double scale)
{
    const int64_t G = C->g.size(), n = 3 * G;
    V3f<double> Fout{F, F + G, F + 2 * G};
    TG_CUDA(cudaMemcpyAsync(C->s.ucont.x, U, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
    reset_no_penetration(C);
    reset_face_periodic(C, C->s.ucont);
    contra_to_cart_stage(C);
    reset_cell_periodic(C, C->s.ucat);
    TG_CUDA(cudaMemcpyAsync(Fout.x, W.bu.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
    form_u(C, Fout, scale);
    k_scale<<<nblk(n), DB, 0, C->stream>>>(n, C->prm.dt, Fout.x);
    mask_non_resolved(C, Fout);
    k_cn_time<<<nblk(n), DB, 0, C->stream>>>(n, Fout.x, U, C->s.ucont_o.x);
}

// Jacobian-free Newton-Krylov root of F (Feval(U, F) writes F(U)) from the
// guess in W.U, left in W.U: restarted GMRES on J d = -F to 1e-3 relative
// residual per Newton step, J v = (F(U + h v) - F(U)) / h with PETSc's
// MATMFFD_WP h = sqrt(eps) sqrt(1 + |U|) / |v|, Newton steps halved while |F|
// does not fall; stop at |F| <= max(atol, rtol |F_0|) or maxit Newton steps.
// Returns 0 converged, 1 not converged, 2 not finite.
int jfnk_solve(tg_ctx *C, JfnkWork &W, const std::function<void(const double *, double *)> &Feval, double atol, double rtol,
               int maxit, int &newton, int &linear, double &fn_out)
{
    const int64_t n = W.n;
    Feval(W.U, W.F);
    double fn = std::sqrt(dot(C, W, W.F, W.F, n));
    const double f0 = fn;
    const double erel = std::sqrt(2.220446049250313e-16);
    const int m = W.m;
    auto Vk = [&](int k) { return W.V + (size_t)k * n; };
    newton = 0;
    linear = 0;
    int rc = 0;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    while (!(fn <= std::max(atol, rtol * f0)) && newton < maxit) {
        if (!std::isfinite(fn)) { rc = 2; break; }
        // GMRES(m) on J d = -F from d = 0, to 1e-3 relative residual (inexact Newton)
        const double unorm = std::sqrt(dot(C, W, W.U, W.U, n));
        double *d = W.W;                                    // accumulated correction
        TG_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n, C->stream));
        const double beta0 = fn, tol = 1e-3 * fn;
        double res = beta0;
        for (int cycle = 0; cycle < 20 && res > tol; cycle++) {
            // r = -F - J d (J d = 0 on the first cycle)
            double *v0 = Vk(0);
            if (cycle == 0) {
                k_axpby<<<nblk(n), DB, 0, C->stream>>>(n, -1.0, W.F, 0.0, v0);
            } else {
                // J d by differencing
                const double dn = std::sqrt(dot(C, W, d, d, n));
                const double h = erel * std::sqrt(1.0 + unorm) / dn;
                double *UP = Vk(m);
                k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, UP, W.U, h, d);
                Feval(UP, W.FW);
                linear++;
                // v0 = -F - (FW - F) / h
                k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, v0, W.FW, -1.0, W.F);
                k_axpby<<<nblk(n), DB, 0, C->stream>>>(n, -1.0, W.F, -1.0 / h, v0);
            }
            double beta = std::sqrt(dot(C, W, v0, v0, n));
            if (!(beta > 0)) break;
            k_axpby<<<nblk(n), DB, 0, C->stream>>>(n, 0.0, v0, 1.0 / beta, v0);
            std::fill(g.begin(), g.end(), 0.0);
            g[0] = beta;
            int kk = 0;
            for (; kk < m; kk++) {
                // w = J v_k
                double *w = Vk(kk + 1);
                const double h = erel * std::sqrt(1.0 + unorm);        // |v_k| = 1
                k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, w, W.U, h, Vk(kk));
                Feval(w, W.FW);
                linear++;
                k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, w, W.FW, -1.0, W.F);
                k_axpby<<<nblk(n), DB, 0, C->stream>>>(n, 0.0, w, 1.0 / h, w);
                // modified Gram-Schmidt
                for (int q = 0; q <= kk; q++) {
                    const double hq = dot(C, W, w, Vk(q), n);
                    H[(size_t)q * m + kk] = hq;
                    k_axpby<<<nblk(n), DB, 0, C->stream>>>(n, -hq, Vk(q), 1.0, w);
                }
                const double hn = std::sqrt(dot(C, W, w, w, n));
                H[(size_t)(kk + 1) * m + kk] = hn;
                if (hn > 0) k_axpby<<<nblk(n), DB, 0, C->stream>>>(n, 0.0, w, 1.0 / hn, w);
                // Givens rotations
                for (int q = 0; q < kk; q++) {
                    const double a = H[(size_t)q * m + kk], b = H[(size_t)(q + 1) * m + kk];
                    H[(size_t)q * m + kk] = cs[q] * a + sn[q] * b;
                    H[(size_t)(q + 1) * m + kk] = -sn[q] * a + cs[q] * b;
                }
                const double a = H[(size_t)kk * m + kk], b = H[(size_t)(kk + 1) * m + kk];
                const double r = std::sqrt(a * a + b * b);
                cs[kk] = r > 0 ? a / r : 1.0; sn[kk] = r > 0 ? b / r : 0.0;
                H[(size_t)kk * m + kk] = r; H[(size_t)(kk + 1) * m + kk] = 0.0;
                g[kk + 1] = -sn[kk] * g[kk]; g[kk] = cs[kk] * g[kk];
                res = std::fabs(g[kk + 1]);
                if (res <= tol || !(hn > 0)) { kk++; break; }
            }
            // y = R^-1 g, d += V y
            for (int q = kk - 1; q >= 0; q--) {
                double s = g[q];
                for (int r2 = q + 1; r2 < kk; r2++) s -= H[(size_t)q * m + r2] * y[r2];
                y[q] = s / H[(size_t)q * m + q];
            }
            for (int q = 0; q < kk; q++) k_axpby<<<nblk(n), DB, 0, C->stream>>>(n, y[q], Vk(q), 1.0, d);
        }
        // Newton step, halved while |F| does not decrease
        double lam = 1.0, fnew = 0.0;
        double *UT = Vk(m);
        for (int ls = 0; ls < 8; ls++) {
            k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, UT, W.U, lam, d);
            Feval(UT, W.FW);
            fnew = std::sqrt(dot(C, W, W.FW, W.FW, n));
            if (fnew < fn || !std::isfinite(fnew)) break;
            lam *= 0.5;
        }
        TG_CUDA(cudaMemcpyAsync(W.U, UT, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
        TG_CUDA(cudaMemcpyAsync(W.F, W.FW, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
        fn = fnew;
        newton++;
    }
    if (!std::isfinite(fn)) rc = 2;
    else if (rc == 0 && !(fn <= std::max(atol, rtol * f0))) rc = 1;
    fn_out = fn;
    return rc;
}

JfnkWork *jfnk_alloc(tg_ctx *C, int64_t n, int m)
{
    JfnkWork *W = new JfnkWork();
    jfnk_init(C, *W, n, m);
    return W;
}

void jfnk_free(JfnkWork *W) { delete W; }   // device buffers are owned by the context allocation list

double *jfnk_u(JfnkWork *W) { return W->U; }

// UeqnSNES (ueqn_solvers.c:1087-1199): Ucont <- the root of F from Ucont_o
int solve_u_cn(tg_ctx *C, tg_stats *st)
{
    CnWork &W = work(C);
    const int64_t n = 3 * C->g.size();
    const double scale = C->it > C->cfg.it_start ? 0.5 : 1.0;
    cn_build_bu(C, W.bu, C->it > C->cfg.it_start);
    TG_CUDA(cudaMemcpyAsync(W.j.U, C->s.ucont_o.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
    const int maxit = C->cfg.snes_maxit > 0 ? C->cfg.snes_maxit : 20;
    int newton = 0, linear = 0;
    double fn = 0.0;
    // F is evaluated in FP64 in every precision mode: the differenced
    // Jacobian-vector products divide F's change over h ~ 1e-8 |U|, below
    // the rounding of an FP32 residual
    const auto pol = C->pol;
    C->pol = decltype(C->pol){};
    const int rc = jfnk_solve(C, W.j, [&](const double *U, double *F) { cn_eval(C, W, U, F, scale); }, C->cfg.snes_atol,
                              C->cfg.snes_rtol, maxit, newton, linear, fn);
    C->pol = pol;
    // Ucont <- U (SNESFuncEval left the last evaluated point in the state)
    TG_CUDA(cudaMemcpyAsync(C->s.ucont.x, W.j.U, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
    C->mom_outer = newton;
    C->mom_inner = linear;
    C->mom_res = fn;
    (void)st;
    return rc;
}

}  // namespace tg
