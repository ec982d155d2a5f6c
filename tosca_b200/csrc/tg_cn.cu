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
#include <cmath>
#include <vector>

#include "tg_internal.cuh"

namespace tg {

struct CnWork {
    int m = 30;                       // GMRES restart (-kspGMRESRestartU)
    V3f<double> bu{}, U{}, F{}, W{}, FW{};
    double *V = nullptr;              // (m + 1) Krylov vectors of 3 G
    double *part = nullptr;           // dot-product partials
    int nb = 0;
};

namespace {

constexpr int DB = 256;

__global__ void k_dot_part(int64_t n, const double *a, const double *b, double *part)
{
    __shared__ double sh[DB];
    double s = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) s += a[t] * b[t];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) { if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w]; __syncthreads(); }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_dot_sum(const double *part, int nb, double *out)
{
    __shared__ double sh[DB];
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += part[b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) { if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w]; __syncthreads(); }
    if (threadIdx.x == 0) out[0] = sh[0];
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

double dot(tg_ctx *C, CnWork &W, const double *a, const double *b, int64_t n)
{
    k_dot_part<<<W.nb, DB, 0, C->stream>>>(n, a, b, W.part);
    k_dot_sum<<<1, DB, 0, C->stream>>>(W.part, W.nb, C->d_scal + 90);
    TG_CUDA(cudaMemcpyAsync(C->h_scal + 90, C->d_scal + 90, sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaStreamSynchronize(C->stream));
    return C->h_scal[90];
}

CnWork &work(tg_ctx *C)
{
    if (!C->cn) {
        CnWork *W = new CnWork();
        const size_t G = (size_t)C->g.size();
        W->m = C->cfg.gmres_restart > 0 ? C->cfg.gmres_restart : 30;
        W->bu = dalloc3(C, G); W->U = dalloc3(C, G); W->F = dalloc3(C, G); W->W = dalloc3(C, G); W->FW = dalloc3(C, G);
        W->V = dallocd(C, (size_t)(W->m + 1) * 3 * G);
        W->nb = nblk(3 * (int64_t)G);
        W->part = dallocd(C, W->nb);
        C->cn = W;
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
static void cn_eval(tg_ctx *C, CnWork &W, V3f<double> U, V3f<double> Fout, double scale)
{
    const int64_t n = 3 * C->g.size();
    TG_CUDA(cudaMemcpyAsync(C->s.ucont.x, U.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
    reset_no_penetration(C);
    reset_face_periodic(C, C->s.ucont);
    contra_to_cart_stage(C);
    reset_cell_periodic(C, C->s.ucat);
    TG_CUDA(cudaMemcpyAsync(Fout.x, W.bu.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
    form_u(C, Fout, scale);
    k_scale<<<nblk(n), DB, 0, C->stream>>>(n, C->prm.dt, Fout.x);
    mask_non_resolved(C, Fout);
    k_cn_time<<<nblk(n), DB, 0, C->stream>>>(n, Fout.x, U.x, C->s.ucont_o.x);
}

// UeqnSNES (ueqn_solvers.c:1087-1199): Ucont <- the root of F from Ucont_o
int solve_u_cn(tg_ctx *C, tg_stats *st)
{
    CnWork &W = work(C);
    const int64_t n = 3 * C->g.size();
    const double scale = C->it > C->cfg.it_start ? 0.5 : 1.0;
    cn_build_bu(C, W.bu, C->it > C->cfg.it_start);
    TG_CUDA(cudaMemcpyAsync(W.U.x, C->s.ucont_o.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
    cn_eval(C, W, W.U, W.F, scale);
    double fn = std::sqrt(dot(C, W, W.F.x, W.F.x, n));
    const double f0 = fn;
    const double atol = C->cfg.snes_atol, rtol = C->cfg.snes_rtol;
    const int maxit = C->cfg.snes_maxit > 0 ? C->cfg.snes_maxit : 20;
    const double erel = std::sqrt(2.220446049250313e-16);
    const int m = W.m;
    auto Vk = [&](int k) { return W.V + (size_t)k * n; };
    int newton = 0, linear = 0, rc = 0;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    while (!(fn <= std::max(atol, rtol * f0)) && newton < maxit) {
        if (!std::isfinite(fn)) { rc = 2; break; }
        // GMRES(m) on J d = -F from d = 0, to 1e-3 relative residual (inexact Newton)
        const double unorm = std::sqrt(dot(C, W, W.U.x, W.U.x, n));
        double *d = W.W.x;                                  // accumulated correction (reuse of W)
        TG_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n, C->stream));
        const double beta0 = fn, tol = 1e-3 * fn;
        double res = beta0;
        for (int cycle = 0; cycle < 20 && res > tol; cycle++) {
            // r = -F - J d (J d = 0 on the first cycle)
            double *v0 = Vk(0);
            if (cycle == 0) {
                k_axpby<<<nblk(n), DB, 0, C->stream>>>(n, -1.0, W.F.x, 0.0, v0);
            } else {
                // J d by differencing
                const double dn = std::sqrt(dot(C, W, d, d, n));
                const double h = erel * std::sqrt(1.0 + unorm) / dn;
                V3f<double> UP{Vk(m), Vk(m) + n / 3, Vk(m) + 2 * (n / 3)};
                k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, UP.x, W.U.x, h, d);
                cn_eval(C, W, UP, W.FW, scale);
                linear++;
                // v0 = -F - (FW - F) / h
                k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, v0, W.FW.x, -1.0, W.F.x);
                k_axpby<<<nblk(n), DB, 0, C->stream>>>(n, -1.0, W.F.x, -1.0 / h, v0);
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
                V3f<double> UP{w, w + n / 3, w + 2 * (n / 3)};
                k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, w, W.U.x, h, Vk(kk));
                cn_eval(C, W, UP, W.FW, scale);
                linear++;
                k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, w, W.FW.x, -1.0, W.F.x);
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
        V3f<double> UT{Vk(m), Vk(m) + n / 3, Vk(m) + 2 * (n / 3)};
        for (int ls = 0; ls < 8; ls++) {
            k_waxpy<<<nblk(n), DB, 0, C->stream>>>(n, UT.x, W.U.x, lam, d);
            cn_eval(C, W, UT, W.FW, scale);
            fnew = std::sqrt(dot(C, W, W.FW.x, W.FW.x, n));
            if (fnew < fn || !std::isfinite(fnew)) break;
            lam *= 0.5;
        }
        TG_CUDA(cudaMemcpyAsync(W.U.x, UT.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
        TG_CUDA(cudaMemcpyAsync(W.F.x, W.FW.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
        fn = fnew;
        newton++;
    }
    if (!std::isfinite(fn)) rc = 2;
    else if (rc == 0 && !(fn <= std::max(atol, rtol * f0))) rc = 1;
    // Ucont <- U (SNESFuncEval left the last evaluated point in the state)
    TG_CUDA(cudaMemcpyAsync(C->s.ucont.x, W.U.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
    C->mom_outer = newton;
    C->mom_inner = linear;
    C->mom_res = fn;
    (void)st;
    return rc;
}

}  // namespace tg
