// Implicit-explicit momentum steps with a Crank-Nicolson viscous part
// (ueqn_solvers.c:1508-1799): ABCN (UeqnABCN), RK3WCN (UeqnRK3CN_W) and
// RK3SOCN (UeqnRK3CN_SO). Each stage forms the convective right-hand side
// explicitly (ExplicitRhsU with formMode 1) and the viscous one of the stage
// state (FormU formMode 2), builds bU, and solves
//   A U = bU,   A v = v - dt' s Visc(v)   (IMEXMatVec, ueqn_solvers.c:1739-1799)
// with restarted GMRES from the explicit-Euler guess. Visc(v) is FormU with
// formMode 2 of the Ucat of v after the no-penetration and periodic resets,
// zeroed at non-resolved faces; the eddy viscosity and the wall stress stay
// those of the step start, so with a wall model A is affine and GMRES treats
// it as linear, as PETSc's KSP does. s = 1/2 for ABCN after the first step,
// else 1; the RK3 schemes fold their stage weight into dt' = gamma dt.
//
// The Krylov solver restates PETSc's KSPGMRES as configured by ueqn.c:261-282
// (PCNONE, nonzero initial guess, classical Gram-Schmidt without refinement,
// Givens rotations, restart -kspGMRESRestartU, tolerances relTolU / absTolU
// against |b|, 1000 iterations): every cycle starts from the true residual
// b - A x, stops on the rotated residual estimate and adds V y to x.
// The dot products return to the host (one synchronisation per Arnoldi step
// for the Hessenberg column, one for its norm); every vector operation runs
// on the device. gmres_solve takes the operator as a callback and serves the
// ABBE temperature solve too (tg_teqn.cu, n = G instead of 3 G).
#include <cmath>
#include <vector>

#include "tg_internal.cuh"

namespace tg {

// restarted GMRES on n unknowns (gmres_solve)
struct GmresWork {
    int m = 30;                       // restart
    int64_t n = 0;                    // unknowns
    double *V = nullptr;              // (m + 1) Krylov vectors of n
    double *part = nullptr;           // block partials: (m + 1) x nb
    double *d_out = nullptr;          // reduced dot products (m + 2)
    double *h_out = nullptr;          // pinned host copy
    int nb = 0;                       // blocks of the chunked kernels
};

struct ImexWork {
    GmresWork k;                      // n = 3 G
    V3f<double> bu{}, visc{}, conv{}, conv_o{}, x{}, rhs_o{};
};

namespace {

constexpr int TB = 256;               // threads per block
constexpr int PT = 8;                 // elements per thread of a chunked kernel
constexpr int CH = TB * PT;           // elements per block
constexpr int MAXV = 64;              // coefficient slots of one kernel argument

struct Coef { double a[MAXV]; };

__device__ __forceinline__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) {
        s = threadIdx.x < (TB >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;   // valid in thread 0
}

// part[q * nb + b] = sum over block b's chunk of w . V_q, q < nv (VecMDot):
// the chunk of w stays in registers while the nv basis vectors stream past
__global__ void __launch_bounds__(TB) k_mdot(int64_t n, const double *__restrict__ w, const double *__restrict__ V, int nv, double *part)
{
    __shared__ double sh[TB / 32];
    const int64_t base = (int64_t)blockIdx.x * CH + threadIdx.x;
    double r[PT];
#pragma unroll
    for (int e = 0; e < PT; e++) { const int64_t t = base + (int64_t)e * TB; r[e] = t < n ? w[t] : 0.0; }
    for (int q = 0; q < nv; q++) {
        const double *v = V + (int64_t)q * n;
        double s = 0.0;
#pragma unroll
        for (int e = 0; e < PT; e++) { const int64_t t = base + (int64_t)e * TB; if (t < n) s += r[e] * v[t]; }
        s = block_sum(s, sh);
        if (threadIdx.x == 0) part[(int64_t)q * gridDim.x + blockIdx.x] = s;
    }
}

// out[q] = sum of the nb partials of row q (one block per row)
__global__ void __launch_bounds__(TB) k_rows_sum(const double *part, int nb, double *out)
{
    __shared__ double sh[TB / 32];
    const double *p = part + (int64_t)blockIdx.x * nb;
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += TB) s += p[b];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// w += sum_q c_q V_q (VecMAXPY) and part[b] = |w|^2 over the block's chunk
__global__ void __launch_bounds__(TB) k_maxpy_norm(int64_t n, double *__restrict__ w, const double *__restrict__ V, int nv, Coef c, double *part)
{
    __shared__ double sh[TB / 32];
    const int64_t base = (int64_t)blockIdx.x * CH + threadIdx.x;
    double r[PT];
#pragma unroll
    for (int e = 0; e < PT; e++) { const int64_t t = base + (int64_t)e * TB; r[e] = t < n ? w[t] : 0.0; }
    for (int q = 0; q < nv; q++) {
        const double *v = V + (int64_t)q * n;
        const double a = c.a[q];
#pragma unroll
        for (int e = 0; e < PT; e++) { const int64_t t = base + (int64_t)e * TB; if (t < n) r[e] += a * v[t]; }
    }
    double s = 0.0;
#pragma unroll
    for (int e = 0; e < PT; e++) { const int64_t t = base + (int64_t)e * TB; if (t < n) { w[t] = r[e]; s += r[e] * r[e]; } }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// x = x + sum_q c_q V_q with the sum formed first (KSPGMRESBuildSoln: VecMAXPY
// into a zeroed temporary, then VecAXPY)
__global__ void __launch_bounds__(TB) k_update_x(int64_t n, double *__restrict__ x, const double *__restrict__ V, int nv, Coef c)
{
    for (int64_t t = blockIdx.x * (int64_t)TB + threadIdx.x; t < n; t += (int64_t)gridDim.x * TB) {
        double s = 0.0;
        for (int q = 0; q < nv; q++) s += c.a[q] * V[(int64_t)q * n + t];
        x[t] = x[t] + 1.0 * s;
    }
}

// part[b] = |a|^2 over the block's chunk
__global__ void __launch_bounds__(TB) k_norm2(int64_t n, const double *__restrict__ a, double *part)
{
    __shared__ double sh[TB / 32];
    const int64_t base = (int64_t)blockIdx.x * CH + threadIdx.x;
    double s = 0.0;
#pragma unroll
    for (int e = 0; e < PT; e++) { const int64_t t = base + (int64_t)e * TB; if (t < n) s += a[t] * a[t]; }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// y = a x + b y
__global__ void k_axpby(int64_t n, double a, const double *x, double b, double *y)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) y[t] = a * x[t] + b * y[t];
}

// Av = Av + v (IMEXMatVec's VecAXPY(Av, 1, v))
__global__ void k_add(int64_t n, double *Av, const double *v)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) Av[t] = Av[t] + 1.0 * v[t];
}

// ABCN right-hand side and guess (ueqn_solvers.c:1685-1715), in VecAXPY order:
// bU = Rhs + 1/2 RhsConv - 1/2 RhsConv_o + 1/2 RhsVisc (later steps) or
// Rhs + Rhs (first step), bU = dt bU + Ucont_o; Utmp = gv RhsVisc + bU
__global__ void k_abcn_bu(int64_t n, double *bu, double *x, const double *rhs, const double *conv, const double *conv_o,
                          const double *visc, const double *uo, double dt, double gv, int ab2)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        double b = rhs[t];
        if (ab2) {
            b = b + 0.5 * conv[t];
            b = b + -0.5 * conv_o[t];
            b = b + 0.5 * visc[t];
        } else {
            b = b + 1.0 * rhs[t];
        }
        b = b * dt;
        b = b + 1.0 * uo[t];
        bu[t] = b;
        x[t] = (0.0 + gv * visc[t]) + 1.0 * b;
    }
}

// RK3WCN stage right-hand side and guess (ueqn_solvers.c:1536-1546):
// bU = Ucont + dt beta Rhs - dt delta Rhs_o + dt gamma RhsVisc; Utmp = bU + dt gamma RhsVisc
__global__ void k_rk3w_bu(int64_t n, double *bu, double *x, const double *u, const double *rhs, const double *rhs_o,
                          const double *visc, double ab, double ad, double ag)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        double b = u[t];
        b = b + ab * rhs[t];
        b = b + ad * rhs_o[t];
        b = b + ag * visc[t];
        bu[t] = b;
        x[t] = b + ag * visc[t];
    }
}

// RK3SOCN stage right-hand side and guess (ueqn_solvers.c:1612-1628):
// bU = alpha Ucont_o (+ (1 - alpha) Ucont) + dt beta Rhs + dt gamma RhsVisc; Utmp = bU + dt gamma RhsVisc
__global__ void k_rk3so_bu(int64_t n, double *bu, double *x, const double *uo, const double *u, const double *rhs,
                           const double *visc, double alpha, double om, int with_u, double ab, double ag)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        double b = uo[t] * alpha;
        if (with_u) b = b + om * u[t];
        b = b + ab * rhs[t];
        b = b + ag * visc[t];
        bu[t] = b;
        x[t] = b + ag * visc[t];
    }
}

inline int nblk(int64_t n) { int64_t b = (n + TB - 1) / TB; return (int)(b < 148 * 8 ? b : 148 * 8); }

void gmres_init(tg_ctx *C, GmresWork &W, int64_t n, int m)
{
    W.m = m;
    W.n = n;
    W.V = dallocd(C, (size_t)(W.m + 1) * W.n);
    W.nb = (int)((W.n + CH - 1) / CH);
    W.part = dallocd(C, (size_t)(W.m + 1) * W.nb);
    W.d_out = dallocd(C, MAXV + 2);
    TG_CUDA(cudaMallocHost((void **)&W.h_out, (MAXV + 2) * sizeof(double)));
}

ImexWork &work(tg_ctx *C)
{
    if (!C->imex) {
        ImexWork *W = new ImexWork();
        const size_t G = (size_t)C->g.size();
        W->bu = dalloc3(C, G); W->visc = dalloc3(C, G); W->x = dalloc3(C, G);
        if (C->cfg.ddt_scheme == TG_DDT_ABCN) { W->conv = dalloc3(C, G); W->conv_o = dalloc3(C, G); }
        if (C->cfg.ddt_scheme == TG_DDT_RK3WCN) W->rhs_o = dalloc3(C, G);
        C->imex = W;
        gmres_init(C, W->k, 3 * (int64_t)G, C->cfg.gmres_restart > 0 ? C->cfg.gmres_restart : 30);
    }
    return *C->imex;
}

// |a| (VecNorm NORM_2)
double norm(tg_ctx *C, GmresWork &W, const double *a)
{
    k_norm2<<<W.nb, TB, 0, C->stream>>>(W.n, a, W.part);
    k_rows_sum<<<1, TB, 0, C->stream>>>(W.part, W.nb, W.d_out);
    TG_CUDA(cudaMemcpyAsync(W.h_out, W.d_out, sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaStreamSynchronize(C->stream));
    return std::sqrt(W.h_out[0]);
}

// Av = A v = v - dtp s Visc(v) (IMEXMatVec): leaves Ucont = v and its Ucat in
// the state, as the reference does
void apply(tg_ctx *C, const double *v, double *Av, double dtp, double s)
{
    const int64_t G = C->g.size(), n = 3 * G;
    TG_CUDA(cudaMemcpyAsync(C->s.ucont.x, v, sizeof(double) * n, cudaMemcpyDeviceToDevice, C->stream));
    reset_no_penetration(C);
    reset_face_periodic(C, C->s.ucont);
    contra_to_cart_stage(C);
    reset_cell_periodic(C, C->s.ucat);
    V3f<double> out{Av, Av + G, Av + 2 * G};
    TG_CUDA(cudaMemsetAsync(Av, 0, sizeof(double) * n, C->stream));
    form_u(C, out, -1.0 * s * dtp, 2);
    mask_non_resolved(C, out);
    k_add<<<nblk(n), TB, 0, C->stream>>>(n, Av, v);
}

}  // namespace

// KSPSolve with KSPGMRES on the operator A (A(v, Av) writes A v): 0
// converged, 1 iteration limit, 2 not a number or breakdown
int gmres_solve(tg_ctx *C, GmresWork &W, const std::function<void(const double *, double *)> &A, const double *b, double *x,
                double rtol, double atol, int &its, double &res)
{
    const int64_t n = W.n;
    const int m = W.m, maxit = 1000;
    const double haptol = 1e-30;
    auto Vk = [&](int k) { return W.V + (int64_t)k * n; };
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    auto Hq = [&](int r, int c) -> double & { return H[(size_t)r * m + c]; };
    its = 0;
    res = 0.0;
    double ttol = 0.0;
    bool first = true;
    int reason = 0;   // 1 converged, -1 iteration limit, -2 nan / breakdown
    while (!reason) {
        // KSPInitialResidual: V0 = b - A x
        A(x, Vk(0));
        k_axpby<<<nblk(n), TB, 0, C->stream>>>(n, 1.0, b, -1.0, Vk(0));
        const double beta = norm(C, W, Vk(0));
        if (first) {
            // KSPConvergedDefault at iteration 0 with a nonzero guess: |b|
            double snorm = norm(C, W, b);
            if (snorm == 0.0) snorm = beta;
            ttol = std::max(rtol * snorm, atol);
            first = false;
        }
        res = beta;
        if (!std::isfinite(beta)) { reason = -2; break; }
        if (beta == 0.0 || beta <= ttol) { reason = 1; break; }
        k_axpby<<<nblk(n), TB, 0, C->stream>>>(n, 0.0, Vk(0), 1.0 / beta, Vk(0));
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        while (!reason && k < m && its < maxit) {
            double *w = Vk(k + 1);
            A(Vk(k), w);
            // classical Gram-Schmidt: h = V^T w, w -= V h, |w|
            k_mdot<<<W.nb, TB, 0, C->stream>>>(n, w, W.V, k + 1, W.part);
            k_rows_sum<<<k + 1, TB, 0, C->stream>>>(W.part, W.nb, W.d_out);
            TG_CUDA(cudaMemcpyAsync(W.h_out, W.d_out, sizeof(double) * (k + 1), cudaMemcpyDeviceToHost, C->stream));
            TG_CUDA(cudaStreamSynchronize(C->stream));
            Coef c{};
            for (int q = 0; q <= k; q++) { Hq(q, k) = W.h_out[q]; c.a[q] = -W.h_out[q]; }
            k_maxpy_norm<<<W.nb, TB, 0, C->stream>>>(n, w, W.V, k + 1, c, W.part);
            k_rows_sum<<<1, TB, 0, C->stream>>>(W.part, W.nb, W.d_out);
            TG_CUDA(cudaMemcpyAsync(W.h_out, W.d_out, sizeof(double), cudaMemcpyDeviceToHost, C->stream));
            TG_CUDA(cudaStreamSynchronize(C->stream));
            const double tt = std::sqrt(W.h_out[0]);
            if (tt != 0.0) k_axpby<<<nblk(n), TB, 0, C->stream>>>(n, 0.0, w, 1.0 / tt, w);
            Hq(k + 1, k) = tt;
            double hapbnd = std::fabs(tt / g[k]);
            if (hapbnd > haptol) hapbnd = haptol;
            const bool hap = tt < hapbnd;
            // KSPGMRESUpdateHessenberg: old rotations, then the new one
            for (int q = 0; q < k; q++) {
                const double a = Hq(q, k), bq = Hq(q + 1, k);
                Hq(q, k) = cs[q] * a + sn[q] * bq;
                Hq(q + 1, k) = cs[q] * bq - sn[q] * a;
            }
            if (!hap) {
                const double a = Hq(k, k), bq = Hq(k + 1, k);
                const double r = std::sqrt(a * a + bq * bq);
                if (r == 0.0) { reason = -2; break; }
                cs[k] = a / r; sn[k] = bq / r;
                g[k + 1] = -(sn[k] * g[k]);
                g[k] = cs[k] * g[k];
                Hq(k, k) = cs[k] * a + sn[k] * bq;
                res = std::fabs(g[k + 1]);
            } else {
                res = 0.0;
            }
            k++;
            its++;
            if (!std::isfinite(res)) reason = -2;
            else if (res <= ttol) reason = 1;
            if (hap && !reason) reason = -2;
        }
        // KSPGMRESBuildSoln: y = R^-1 g over the k columns, x += V y
        if (k > 0 && reason != -2) {
            for (int q = k - 1; q >= 0; q--) {
                double t = g[q];
                for (int r = q + 1; r < k; r++) t -= Hq(q, r) * y[r];
                y[q] = t / Hq(q, q);
            }
            Coef c{};
            for (int q = 0; q < k; q++) c.a[q] = y[q];
            k_update_x<<<nblk(n), TB, 0, C->stream>>>(n, x, W.V, k, c);
        }
        if (!reason && its >= maxit) reason = -1;
    }
    return reason == 1 ? 0 : reason == -1 ? 1 : 2;
}

GmresWork *gmres_alloc(tg_ctx *C, int64_t n, int m)
{
    GmresWork *W = new GmresWork();
    gmres_init(C, *W, n, m);
    return W;
}

void gmres_free(GmresWork *W)
{
    if (W && W->h_out) cudaFreeHost(W->h_out);
    delete W;            // device buffers are owned by the context allocation list
}

void imex_destroy(tg_ctx *C)
{
    if (C->imex && C->imex->k.h_out) cudaFreeHost(C->imex->k.h_out);
    delete C->imex;      // device buffers are owned by the context allocation list
    C->imex = nullptr;
}

bool imex_scheme(int ddt) { return ddt == TG_DDT_ABCN || ddt == TG_DDT_RK3WCN || ddt == TG_DDT_RK3SOCN; }

// SolveUEqn with UeqnABCN / UeqnRK3CN_W / UeqnRK3CN_SO: Ucont <- U^{n+1}
int solve_u_imex(tg_ctx *C)
{
    ImexWork &W = work(C);
    const int64_t n = W.k.n;
    const double dt = C->prm.dt;
    const size_t bytes = sizeof(double) * n;
    int rc = 0, stages = 0, inner = 0;
    double res = 0.0;
    // RhsVisc = FormU(formMode 2) of the current state, zero at non-resolved faces
    auto visc = [&]() {
        TG_CUDA(cudaMemsetAsync(W.visc.x, 0, bytes, C->stream));
        form_u(C, W.visc, 1.0, 2);
        mask_non_resolved(C, W.visc);
    };
    auto solve = [&](double dtp, double s) {
        int its = 0;
        const int r = gmres_solve(C, W.k, [&](const double *v, double *Av) { apply(C, v, Av, dtp, s); }, W.bu.x, W.x.x,
                                  C->cfg.snes_rtol, C->cfg.snes_atol, its, res);
        inner += its;
        stages++;
        if (r == 2) rc = 2;
        else if (rc != 2) rc |= r;
        TG_CUDA(cudaMemcpyAsync(C->s.ucont.x, W.x.x, bytes, cudaMemcpyDeviceToDevice, C->stream));
    };
    if (C->cfg.ddt_scheme == TG_DDT_ABCN) {
        // UeqnABCN, ueqn_solvers.c:1665-1735. The convective FormU reuses the
        // cell sums of ExplicitRhsU's (same state, formMode 1)
        const bool ab2 = C->it > C->cfg.it_start;
        explicit_rhs(C, 1);
        TG_CUDA(cudaMemsetAsync(W.conv.x, 0, bytes, C->stream));
        form_u_again(C, W.conv, 1.0);
        mask_non_resolved(C, W.conv);
        visc();
        k_abcn_bu<<<nblk(n), TB, 0, C->stream>>>(n, W.bu.x, W.x.x, C->s.rhs.x, W.conv.x, W.conv_o.x, W.visc.x, C->s.ucont_o.x,
                                                 dt, ab2 ? 0.5 * dt : dt, ab2 ? 1 : 0);
        solve(dt, ab2 ? 0.5 : 1.0);
        TG_CUDA(cudaMemcpyAsync(W.conv_o.x, W.conv.x, bytes, cudaMemcpyDeviceToDevice, C->stream));
    } else if (C->cfg.ddt_scheme == TG_DDT_RK3WCN) {
        // UeqnRK3CN_W, ueqn_solvers.c:1508-1565
        const double beta[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
        const double gamma[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
        const double delta[3] = {0.0, 17.0 / 60.0, 5.0 / 12.0};
        TG_CUDA(cudaMemsetAsync(W.rhs_o.x, 0, bytes, C->stream));
        for (int i = 0; i < 3; i++) {
            explicit_rhs(C, 1);
            visc();
            k_rk3w_bu<<<nblk(n), TB, 0, C->stream>>>(n, W.bu.x, W.x.x, C->s.ucont.x, C->s.rhs.x, W.rhs_o.x, W.visc.x,
                                                     dt * beta[i], -1.0 * dt * delta[i], dt * gamma[i]);
            solve(dt * gamma[i], 1.0);
            TG_CUDA(cudaMemcpyAsync(W.rhs_o.x, C->s.rhs.x, bytes, cudaMemcpyDeviceToDevice, C->stream));
        }
    } else {
        // UeqnRK3CN_SO, ueqn_solvers.c:1586-1643
        const double alpha[3] = {1.0, 3.0 / 4.0, 1.0 / 3.0};
        const double beta[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
        const double gamma[3] = {1.0 / 2.0, 1.0 / 8.0, 1.0 / 3.0};
        for (int i = 0; i < 3; i++) {
            explicit_rhs(C, 1);
            visc();
            k_rk3so_bu<<<nblk(n), TB, 0, C->stream>>>(n, W.bu.x, W.x.x, C->s.ucont_o.x, C->s.ucont.x, C->s.rhs.x, W.visc.x,
                                                      alpha[i], 1.0 - alpha[i], i > 0 ? 1 : 0, dt * beta[i], dt * gamma[i]);
            solve(dt * gamma[i], 1.0);
        }
    }
    C->mom_outer = stages;
    C->mom_inner = inner;
    C->mom_res = res;
    return rc;
}

}  // namespace tg
