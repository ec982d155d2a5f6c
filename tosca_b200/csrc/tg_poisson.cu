// Pressure Poisson solve for TOSCA's pinned 19-point operator (peqn.c:703-1501)
// replacing the HYPRE BoomerAMG-GMRES solve (peqn.c:3856-3929).
//
// Unknowns live in a compact interior layout c = (kc*ny + jc)*nx + ic
// (ic = i-1, ...). The operator is applied matrix-free from the nine face
// metric-tensor arrays g11..g33 at the east/north/top face of each cell; the
// 19 coefficients of a row are rebuilt in registers with the reference's
// one-sided rules and its |v| > 1e-10 insertion filter, so the product equals
// the assembled matrix. On orthogonal grids (all cross terms zero) a 7-point
// kernel reads three coefficient arrays only.
//
// Solved system: L phi = -b with L = -A (positive semidefinite away from the
// pinned row), row (1,1,1) the identity (peqn.c:883-887). Symmetric operators
// use preconditioned CG on the reduced system (the pinned unknown stays zero);
// others use right-preconditioned BiCGStab.
//
// Preconditioner: the geometric multigrid V-cycle of tg_mg.cu on the 7-point
// part of the operator, applied in the grounded form z = P M P^T r (P shifts
// so that z at the pinned cell is zero), which is the inverse structure of the
// pinned operator. In the mixed-precision mode the multigrid stores and
// computes in FP32; residuals, inner products and the solution stay FP64.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "tg_internal.cuh"
#include "tg_mg.cuh"

namespace tg {

struct PoissonCtx {
    int nx, ny, nz, pi, pj, pk;
    int64_t n;
    int pin;                     // compact index of the pinned cell (0)
    bool ortho;
    double *gE1, *gE2, *gE3, *gN1, *gN2, *gN3, *gT1, *gT2, *gT3;  // fine face tensors (compact)
    double *x, *b, *r, *z, *p, *q, *rhat, *v, *s, *t, *aj;
    double *xprev, *xprev2;      // the two previous steps' solutions (extrapolated initial guess)
    double *part;                // reduction partials (4 per block)
    int nblocks;
    MG *mg;                      // multigrid preconditioner (host object)
};

namespace {

constexpr int RB = 256;   // reduction block size

struct Cg {   // compact grid indexing with periodic wrap
    int nx, ny, nz, pi, pj, pk;
    __device__ __forceinline__ int wi(int i) const { if (i < 0) i += nx; else if (i >= nx) i -= nx; return i; }
    __device__ __forceinline__ int wj(int j) const { if (j < 0) j += ny; else if (j >= ny) j -= ny; return j; }
    __device__ __forceinline__ int wk(int k) const { if (k < 0) k += nz; else if (k >= nz) k -= nz; return k; }
    __device__ __forceinline__ int id(int k, int j, int i) const { return (wk(k) * ny + wj(j)) * nx + wi(i); }
    __device__ __forceinline__ bool in(int k, int j, int i) const {
        return (pi || (i >= 0 && i < nx)) && (pj || (j >= 0 && j < ny)) && (pk || (k >= 0 && k < nz));
    }
};

// ------------------------------------------------------------ setup kernels
__global__ void k_gather_g(Grid g, Metrics m, PoissonCtx P)
{
    int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y * blockDim.y + threadIdx.y, kc = blockIdx.z * blockDim.z + threadIdx.z;
    if (ic >= P.nx || jc >= P.ny || kc >= P.nz) return;
    int c = (kc * P.ny + jc) * P.nx + ic;
    int d = g.lin(kc + 1, jc + 1, ic + 1);
    P.gE1[c] = m.g11[d]; P.gE2[c] = m.g12[d]; P.gE3[c] = m.g13[d];
    P.gN1[c] = m.g21[d]; P.gN2[c] = m.g22[d]; P.gN3[c] = m.g23[d];
    P.gT1[c] = m.g31[d]; P.gT2[c] = m.g32[d]; P.gT3[c] = m.g33[d];
    P.aj[c] = m.aj[d];
}

// --------------------------------------------------------- fine operators
// 7-point: (L x)_c = sum_f a_f (x_c - x_nb); pinned row = identity
__global__ void k_apply7(PoissonCtx P, const double *__restrict__ x, double *__restrict__ y)
{
    int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y * blockDim.y + threadIdx.y, kc = blockIdx.z * blockDim.z + threadIdx.z;
    if (ic >= P.nx || jc >= P.ny || kc >= P.nz) return;
    const int nx = P.nx, pl = P.nx * P.ny;
    int c = (kc * P.ny + jc) * nx + ic;
    if (c == P.pin) { y[c] = x[c]; return; }
    // neighbours by offset; a periodic seam wraps to the opposite end
    const int e = ic < nx - 1 ? c + 1 : c + 1 - nx, w = ic > 0 ? c - 1 : c - 1 + nx;
    const int n = jc < P.ny - 1 ? c + nx : c + nx - pl, s = jc > 0 ? c - nx : c - nx + pl;
    const int t = kc < P.nz - 1 ? c + pl : c + pl - pl * P.nz, b = kc > 0 ? c - pl : c - pl + pl * P.nz;
    double xc = x[c], acc = 0.0;
    if (ic < nx - 1 || P.pi)   acc += P.gE1[c] * (xc - x[e]);
    if (ic > 0 || P.pi)        acc += P.gE1[w] * (xc - x[w]);
    if (jc < P.ny - 1 || P.pj) acc += P.gN2[c] * (xc - x[n]);
    if (jc > 0 || P.pj)        acc += P.gN2[s] * (xc - x[s]);
    if (kc < P.nz - 1 || P.pk) acc += P.gT3[c] * (xc - x[t]);
    if (kc > 0 || P.pk)        acc += P.gT3[b] * (xc - x[b]);
    y[c] = acc;
}

enum { CP, EP, WP, NP, SP, TP, BP, NE, SE, NW, SW, TN, BN, TS, BS, TE, BE, TW, BW, NST };

// 19 coefficients of one row of SetCoeffMatrix (peqn.c:889-1388)
__device__ void row19(const PoissonCtx &P, const Cg &q, int ic, int jc, int kc, double vol[NST])
{
    for (int m = 0; m < NST; m++) vol[m] = 0.0;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const bool jr = jc == ny - 1, jl = jc == 0, kr = kc == nz - 1, kl = kc == 0, ir = ic == nx - 1, il = ic == 0;
    int c = (kc * ny + jc) * nx + ic;
    if (!ir || P.pi) {   // east
        double a = P.gE1[c], b = P.gE2[c], cc = P.gE3[c];
        vol[CP] -= a; vol[EP] += a;
        if (jr)      { vol[CP] += b * 0.5; vol[EP] += b * 0.5; vol[SP] -= b * 0.5; vol[SE] -= b * 0.5; }
        else if (jl) { vol[NP] += b * 0.5; vol[NE] += b * 0.5; vol[CP] -= b * 0.5; vol[EP] -= b * 0.5; }
        else         { vol[NP] += b * 0.25; vol[NE] += b * 0.25; vol[SP] -= b * 0.25; vol[SE] -= b * 0.25; }
        if (kr)      { vol[CP] += cc * 0.5; vol[EP] += cc * 0.5; vol[BP] -= cc * 0.5; vol[BE] -= cc * 0.5; }
        else if (kl) { vol[TP] += cc * 0.5; vol[TE] += cc * 0.5; vol[CP] -= cc * 0.5; vol[EP] -= cc * 0.5; }
        else         { vol[TP] += cc * 0.25; vol[TE] += cc * 0.25; vol[BP] -= cc * 0.25; vol[BE] -= cc * 0.25; }
    }
    if (!il || P.pi) {   // west
        int w = q.id(kc, jc, ic - 1);
        double a = P.gE1[w], b = P.gE2[w], cc = P.gE3[w];
        vol[CP] -= a; vol[WP] += a;
        if (jr)      { vol[CP] -= b * 0.5; vol[WP] -= b * 0.5; vol[SP] += b * 0.5; vol[SW] += b * 0.5; }
        else if (jl) { vol[NP] -= b * 0.5; vol[NW] -= b * 0.5; vol[CP] += b * 0.5; vol[WP] += b * 0.5; }
        else         { vol[NP] -= b * 0.25; vol[NW] -= b * 0.25; vol[SP] += b * 0.25; vol[SW] += b * 0.25; }
        if (kr)      { vol[CP] -= cc * 0.5; vol[WP] -= cc * 0.5; vol[BP] += cc * 0.5; vol[BW] += cc * 0.5; }
        else if (kl) { vol[TP] -= cc * 0.5; vol[TW] -= cc * 0.5; vol[CP] += cc * 0.5; vol[WP] += cc * 0.5; }
        else         { vol[TP] -= cc * 0.25; vol[TW] -= cc * 0.25; vol[BP] += cc * 0.25; vol[BW] += cc * 0.25; }
    }
    if (!jr || P.pj) {   // north
        double a = P.gN1[c], b = P.gN2[c], cc = P.gN3[c];
        if (ir)      { vol[CP] += a * 0.5; vol[NP] += a * 0.5; vol[WP] -= a * 0.5; vol[NW] -= a * 0.5; }
        else if (il) { vol[EP] += a * 0.5; vol[NE] += a * 0.5; vol[CP] -= a * 0.5; vol[NP] -= a * 0.5; }
        else         { vol[EP] += a * 0.25; vol[NE] += a * 0.25; vol[WP] -= a * 0.25; vol[NW] -= a * 0.25; }
        vol[CP] -= b; vol[NP] += b;
        if (kr)      { vol[CP] += cc * 0.5; vol[NP] += cc * 0.5; vol[BP] -= cc * 0.5; vol[BN] -= cc * 0.5; }
        else if (kl) { vol[TP] += cc * 0.5; vol[TN] += cc * 0.5; vol[CP] -= cc * 0.5; vol[NP] -= cc * 0.5; }
        else         { vol[TP] += cc * 0.25; vol[TN] += cc * 0.25; vol[BP] -= cc * 0.25; vol[BN] -= cc * 0.25; }
    }
    if (!jl || P.pj) {   // south
        int s = q.id(kc, jc - 1, ic);
        double a = P.gN1[s], b = P.gN2[s], cc = P.gN3[s];
        if (ir)      { vol[CP] -= a * 0.5; vol[SP] -= a * 0.5; vol[WP] += a * 0.5; vol[SW] += a * 0.5; }
        else if (il) { vol[EP] -= a * 0.5; vol[SE] -= a * 0.5; vol[CP] += a * 0.5; vol[SP] += a * 0.5; }
        else         { vol[EP] -= a * 0.25; vol[SE] -= a * 0.25; vol[WP] += a * 0.25; vol[SW] += a * 0.25; }
        vol[CP] -= b; vol[SP] += b;
        if (kr)      { vol[CP] -= cc * 0.5; vol[SP] -= cc * 0.5; vol[BP] += cc * 0.5; vol[BS] += cc * 0.5; }
        else if (kl) { vol[TP] -= cc * 0.5; vol[TS] -= cc * 0.5; vol[CP] += cc * 0.5; vol[SP] += cc * 0.5; }
        else         { vol[TP] -= cc * 0.25; vol[TS] -= cc * 0.25; vol[BP] += cc * 0.25; vol[BS] += cc * 0.25; }
    }
    if (!kr || P.pk) {   // top
        double a = P.gT1[c], b = P.gT2[c], cc = P.gT3[c];
        if (ir)      { vol[CP] += a * 0.5; vol[TP] += a * 0.5; vol[WP] -= a * 0.5; vol[TW] -= a * 0.5; }
        else if (il) { vol[EP] += a * 0.5; vol[TE] += a * 0.5; vol[CP] -= a * 0.5; vol[TP] -= a * 0.5; }
        else         { vol[EP] += a * 0.25; vol[TE] += a * 0.25; vol[WP] -= a * 0.25; vol[TW] -= a * 0.25; }
        if (jr)      { vol[CP] += b * 0.5; vol[TP] += b * 0.5; vol[SP] -= b * 0.5; vol[TS] -= b * 0.5; }
        else if (jl) { vol[NP] += b * 0.5; vol[TN] += b * 0.5; vol[CP] -= b * 0.5; vol[TP] -= b * 0.5; }
        else         { vol[NP] += b * 0.25; vol[TN] += b * 0.25; vol[SP] -= b * 0.25; vol[TS] -= b * 0.25; }
        vol[CP] -= cc; vol[TP] += cc;
    }
    if (!kl || P.pk) {   // bottom
        int bb = q.id(kc - 1, jc, ic);
        double a = P.gT1[bb], b = P.gT2[bb], cc = P.gT3[bb];
        if (ir)      { vol[CP] -= a * 0.5; vol[BP] -= a * 0.5; vol[WP] += a * 0.5; vol[BW] += a * 0.5; }
        else if (il) { vol[EP] -= a * 0.5; vol[BE] -= a * 0.5; vol[CP] += a * 0.5; vol[BP] += a * 0.5; }
        else         { vol[EP] -= a * 0.25; vol[BE] -= a * 0.25; vol[WP] += a * 0.25; vol[BW] += a * 0.25; }
        if (jr)      { vol[CP] -= b * 0.5; vol[BP] -= b * 0.5; vol[SP] += b * 0.5; vol[BS] += b * 0.5; }
        else if (jl) { vol[NP] -= b * 0.5; vol[BN] -= b * 0.5; vol[CP] += b * 0.5; vol[BP] += b * 0.5; }
        else         { vol[NP] -= b * 0.25; vol[BN] -= b * 0.25; vol[SP] += b * 0.25; vol[BS] += b * 0.25; }
        vol[CP] -= cc; vol[BP] += cc;
    }
}

__constant__ int c_off[NST][3] = {   // (dk, dj, di) of each stencil point
    {0,0,0},{0,0,1},{0,0,-1},{0,1,0},{0,-1,0},{1,0,0},{-1,0,0},
    {0,1,1},{0,-1,1},{0,1,-1},{0,-1,-1},
    {1,1,0},{-1,1,0},{1,-1,0},{-1,-1,0},
    {1,0,1},{-1,0,1},{1,0,-1},{-1,0,-1}};

// 19-point: y = -(A x) on non-pinned rows (entries |v| <= 1e-10 dropped as
// at peqn.c:1410-1418), y = x on the pinned row
__global__ void k_apply19(PoissonCtx P, const double *__restrict__ x, double *__restrict__ y)
{
    int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y * blockDim.y + threadIdx.y, kc = blockIdx.z * blockDim.z + threadIdx.z;
    if (ic >= P.nx || jc >= P.ny || kc >= P.nz) return;
    Cg q{P.nx, P.ny, P.nz, P.pi, P.pj, P.pk};
    int c = (kc * P.ny + jc) * P.nx + ic;
    if (c == P.pin) { y[c] = x[c]; return; }
    double vol[NST];
    row19(P, q, ic, jc, kc, vol);
    double acc = 0.0;
    #pragma unroll
    for (int m = 0; m < NST; m++) {
        int kk = kc + c_off[m][0], jj = jc + c_off[m][1], ii = ic + c_off[m][2];
        if (m != CP && (!(fabs(vol[m]) > 1.e-10) || !q.in(kk, jj, ii))) continue;
        acc += vol[m] * x[q.id(kk, jj, ii)];
    }
    y[c] = -acc;
}

// ------------------------------------------------------ vector kernels
// The vectors are separate cudaMalloc allocations (256-byte aligned), so the
// grid-stride loops below move two doubles per access (double2, 16-byte
// loads and stores); an odd last element is taken by thread 0 of block 0
// after its loop.
__device__ __forceinline__ const double2 *v2(const double *a) { return reinterpret_cast<const double2 *>(a); }
__device__ __forceinline__ double2 *v2(double *a) { return reinterpret_cast<double2 *>(a); }
__device__ __forceinline__ bool odd_tail(int64_t n) { return (n & 1) && blockIdx.x == 0 && threadIdx.x == 0; }
#define TG_PAIRS(t, n2) for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (n2); t += (int64_t)gridDim.x * blockDim.x)

// partial sums: slot 0 = a.b, slot 1 = sum(a), slot 2 = max |a * w|
__device__ __forceinline__ void dot_acc(double av, double bv, double wv, double (&v)[3])
{
    v[0] += av * bv;
    v[1] += av;
    v[2] = fmax(v[2], fabs(av * wv));
}
__device__ __forceinline__ void dot_store(double (&v)[3], double *part)
{
    block_reduce<RB>(v, RedSum{}, RedSum{}, RedMax{});
    if (threadIdx.x == 0) { part[3 * blockIdx.x] = v[0]; part[3 * blockIdx.x + 1] = v[1]; part[3 * blockIdx.x + 2] = v[2]; }
}
__global__ void __launch_bounds__(RB) k_dot_partial(int64_t n, const double *a, const double *b, const double *w, double *part)
{
    double v[3] = {0.0, 0.0, 0.0};
    const int64_t n2 = n >> 1;
    TG_PAIRS(t, n2) {
        const double2 av = v2(a)[t], bv = v2(b)[t];
        const double2 wv = w ? v2(w)[t] : double2{0.0, 0.0};
        dot_acc(av.x, bv.x, wv.x, v);
        dot_acc(av.y, bv.y, wv.y, v);
    }
    if (odd_tail(n)) dot_acc(a[n - 1], b[n - 1], w ? w[n - 1] : 0.0, v);
    dot_store(v, part);
}
// final: out[0..2] = totals
__global__ void __launch_bounds__(RB) k_dot_final(const double *part, int nb, double *out)
{
    double v[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) { v[0] += part[3 * b]; v[1] += part[3 * b + 1]; v[2] = fmax(v[2], part[3 * b + 2]); }
    block_reduce<RB>(v, RedSum{}, RedSum{}, RedMax{});
    if (threadIdx.x == 0) { out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; }
}

// y = b - y (residual from y = L x)
__global__ void k_resid(int64_t n, const double *b, double *y)
{
    const int64_t n2 = n >> 1;
    TG_PAIRS(t, n2) { const double2 bv = v2(b)[t], yv = v2(y)[t]; v2(y)[t] = double2{bv.x - yv.x, bv.y - yv.y}; }
    if (odd_tail(n)) y[n - 1] = b[n - 1] - y[n - 1];
}
__global__ void k_copy(int64_t n, const double *a, double *b)
{
    const int64_t n2 = n >> 1;
    TG_PAIRS(t, n2) v2(b)[t] = v2(a)[t];
    if (odd_tail(n)) b[n - 1] = a[n - 1];
}
__global__ void k_zero_at(double *z, int pin) { z[pin] = 0.0; }
// initial guess of the step's solve from the last three solutions (the
// reference starts from x_n): 3 x_n - 3 x_{n-1} + x_{n-2} (quadratic
// extrapolation), 2 x_n - x_{n-1} while only two are known, x_n with one;
// the history shifts (xprev2 <- xprev <- x_n). hist: device count of the
// solutions in the history, read here and advanced by k_hist_next
__global__ void k_extrapolate(int64_t n, double *x, double *xprev, double *xprev2, const double *hist, int order)
{
    const double h = fmin(hist[0], (double)order);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const double xn = x[t], xp = xprev[t];
        if (h >= 2.0) x[t] = 3.0 * xn - 3.0 * xp + xprev2[t];
        else if (h >= 1.0) x[t] = 2.0 * xn - xp;
        xprev2[t] = xp;
        xprev[t] = xn;
    }
}
__global__ void k_hist_next(double *hist) { hist[0] = hist[0] + 1.0; }
inline int guess_order(const tg_ctx *C) { return C->cfg.poisson_guess < 0 ? 2 : C->cfg.poisson_guess; }
__global__ void k_negcopy(int64_t n, const double *a, double *b)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) b[t] = -a[t];
}

// CG: alpha = rz / pq ; x += alpha p ; r -= alpha q, with the partials of
// k_dot_partial(r, r, w) formed in the same grid-stride order (same grid), so
// the totals equal those of a separate update and dot product
__global__ void __launch_bounds__(RB, 4) k_cg_update_rr(int64_t n, const double *rz, const double *pq, double *x, const double *p,
                                                     double *r, const double *q, const double *w, double *part)
{
    const double alpha = rz[0] / pq[0];
    double v[3] = {0.0, 0.0, 0.0};
    const int64_t n2 = n >> 1;
    TG_PAIRS(t, n2) {
        const double2 xv = v2(x)[t], pv = v2(p)[t], rv = v2(r)[t], qv = v2(q)[t];
        const double2 xn{xv.x + alpha * pv.x, xv.y + alpha * pv.y}, rn{rv.x - alpha * qv.x, rv.y - alpha * qv.y};
        v2(x)[t] = xn;
        v2(r)[t] = rn;
        const double2 wv = w ? v2(w)[t] : double2{0.0, 0.0};
        dot_acc(rn.x, rn.x, wv.x, v);
        dot_acc(rn.y, rn.y, wv.y, v);
    }
    if (odd_tail(n)) {
        x[n - 1] += alpha * p[n - 1];
        r[n - 1] -= alpha * q[n - 1];
        const double rv = r[n - 1];
        dot_acc(rv, rv, w ? w[n - 1] : 0.0, v);
    }
    dot_store(v, part);
}
// CG: beta = rz_new / rz_old ; p = z + beta p
__global__ void k_cg_dir(int64_t n, const double *rznew, const double *rzold, const double *z, double *p)
{
    const double beta = rznew[0] / rzold[0];
    const int64_t n2 = n >> 1;
    TG_PAIRS(t, n2) { const double2 zv = v2(z)[t], pv = v2(p)[t]; v2(p)[t] = double2{zv.x + beta * pv.x, zv.y + beta * pv.y}; }
    if (odd_tail(n)) p[n - 1] = z[n - 1] + beta * p[n - 1];
}
__global__ void k_scalar_copy(const double *a, double *b, int n) { for (int t = 0; t < n; t++) b[t] = a[t]; }

// BiCGStab pieces (device scalars in sc: rho, alpha, omega, rho_old)
__global__ void k_bicg_p(int64_t n, const double *sc, double *p, const double *r, const double *v)
{
    // beta = (rho/rho_old) * (alpha/omega)
    double beta = (sc[0] / sc[3]) * (sc[1] / sc[2]);
    double omega = sc[2];
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        p[t] = r[t] + beta * (p[t] - omega * v[t]);
}
__global__ void k_bicg_s(int64_t n, const double *rho, const double *rhv, double *alpha_out, double *s, const double *r, const double *v)
{
    double alpha = rho[0] / rhv[0];
    if (blockIdx.x == 0 && threadIdx.x == 0) alpha_out[0] = alpha;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) s[t] = r[t] - alpha * v[t];
}
__global__ void k_bicg_x(int64_t n, const double *alpha, const double *ts, const double *tt, double *omega_out,
                         double *x, const double *phat, const double *shat, double *r, const double *s, const double *t_)
{
    double om = tt[0] > 0 ? ts[0] / tt[0] : 0.0;
    double al = alpha[0];
    if (blockIdx.x == 0 && threadIdx.x == 0) omega_out[0] = om;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        x[t] += al * phat[t] + om * shat[t];
        r[t] = s[t] - om * t_[t];
    }
}

// ---- loop control of the captured CG solve (device scalars: sc[50] iteration
// count, sc[51] first-direction flag, sc[52] converged flag, sc[53] BiCGStab
// restart after a failed true-residual check). The tests are
// those of krylov_solve; a non-finite residual also ends the loop.
__device__ inline bool cg_converged(const double *sc, double rtol, double divtol, double dt)
{
    const double bn = sqrt(sc[0]), rn = sqrt(sc[3]), rmax = sc[5] * dt;
    return bn == 0.0 || rn / bn <= rtol || (divtol > 0 && rmax <= divtol);
}
__global__ void k_cg_start(double *sc, double rtol, double divtol, double dt, int maxit, cudaGraphConditionalHandle h, int base)
{
    const double bn = sqrt(sc[0]), rn = sqrt(sc[3]);
    const bool conv = cg_converged(sc, rtol, divtol, dt);
    sc[base + ST_RES0] = bn > 0 ? rn / bn : rn;
    sc[50] = 0.0; sc[51] = 1.0; sc[52] = conv ? 1.0 : 0.0; sc[53] = 0.0;
    cudaGraphSetConditional(h, (!conv && maxit > 0 && isfinite(rn)) ? 1u : 0u);
}
__global__ void k_cg_next(double *sc, double rtol, double divtol, double dt, int maxit, cudaGraphConditionalHandle h)
{
    const double rn = sqrt(sc[3]);
    const int it = (int)sc[50] + 1;
    const bool conv = cg_converged(sc, rtol, divtol, dt);
    sc[50] = it; sc[51] = 0.0; sc[52] = conv ? 1.0 : 0.0;
    cudaGraphSetConditional(h, (!conv && it < maxit && isfinite(rn)) ? 1u : 0u);
}
// statistics of the solve, accumulated over the replayed solves in the
// ST_* slots from base
__global__ void k_cg_finish(double *sc, int base)
{
    const double bn = sqrt(sc[0]), rn = sqrt(sc[3]);
    sc[base + ST_IT] = sc[50];
    sc[base + ST_TOT] += sc[50];
    sc[base + ST_RES] = bn > 0 ? rn / bn : rn;
    if (!isfinite(rn)) sc[base + ST_NAN] = 1.0;
    else if (sc[52] == 0.0) sc[base + ST_NOCONV] += 1.0;
}
// p = z on the first pass through the loop body, else p = z + (rz_new / rz_old) p
__global__ void k_cg_dir_loop(int64_t n, const double *sc, const double *z, double *p)
{
    const bool first = sc[51] != 0.0;
    const double beta = first ? 0.0 : sc[6] / sc[14];
    const int64_t n2 = n >> 1;
    TG_PAIRS(t, n2) {
        const double2 zv = v2(z)[t];
        if (first) v2(p)[t] = zv;
        else { const double2 pv = v2(p)[t]; v2(p)[t] = double2{zv.x + beta * pv.x, zv.y + beta * pv.y}; }
    }
    if (odd_tail(n)) p[n - 1] = first ? z[n - 1] : z[n - 1] + beta * p[n - 1];
}

inline dim3 cgrid(int nx, int ny, int nz) { return grid3(nx, ny, nz); }
inline int vblocks(int64_t n) { int64_t b = (n + RB - 1) / RB; return (int)std::min<int64_t>(b, 148 * 8); }

}  // namespace

// ============================================================== host side
static void apply_op(tg_ctx *C, const double *x, double *y)
{
    PoissonCtx &P = *C->pois;
    if (P.ortho) TG_PROF(C, "pois_apply7", k_apply7<<<cgrid(P.nx, P.ny, P.nz), block3(), 0, C->stream>>>(P, x, y));
    else TG_PROF(C, "pois_apply19", k_apply19<<<cgrid(P.nx, P.ny, P.nz), block3(), 0, C->stream>>>(P, x, y));
}

// totals of (a.b, sum a, max|a w|) into out[0..2] (device)
static void dot3v(tg_ctx *C, const double *a, const double *b, const double *w, double *out)
{
    PoissonCtx &P = *C->pois;
    TG_PROF(C, "pois_dot", k_dot_partial<<<P.nblocks, RB, 0, C->stream>>>(P.n, a, b, w, P.part));
    k_dot_final<<<1, RB, 0, C->stream>>>(P.part, P.nblocks, out);
}

// z = P M P^T r (grounded multigrid); needs sum(r) at d_sum
static void precondition(tg_ctx *C, const double *r, double *z, const double *d_sum)
{
    mg_apply(C, C->pois->mg, r, d_sum, z);
}

// SetRHS (peqn.c:1942-2063) into the compact vector, negated (L = -A)
__global__ void k_set_rhs(Grid g, State s, PoissonCtx P, double dt)
{
    int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y * blockDim.y + threadIdx.y, kc = blockIdx.z * blockDim.z + threadIdx.z;
    if (ic >= P.nx || jc >= P.ny || kc >= P.nz) return;
    int c = (kc * P.ny + jc) * P.nx + ic;
    if (c == P.pin) { P.b[c] = 0.0; return; }
    int d = g.lin(kc + 1, jc + 1, ic + 1);
    double val = 0;
    val += s.ucont.x[d];
    val -= s.ucont.x[d - 1];
    val += s.ucont.y[d];
    val -= s.ucont.y[d - g.mx];
    val += s.ucont.z[d];
    val -= s.ucont.z[d - g.mx * g.my];
    val *= 1.0 / dt;
    P.b[c] = -val;
}

// phiToPhi (peqn.c:1579-1636): compact solution into the DMDA interior
__global__ void k_phi_to_dmda(Grid g, State s, PoissonCtx P)
{
    int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y * blockDim.y + threadIdx.y, kc = blockIdx.z * blockDim.z + threadIdx.z;
    if (ic >= P.nx || jc >= P.ny || kc >= P.nz) return;
    s.phi[g.lin(kc + 1, jc + 1, ic + 1)] = P.x[(kc * P.ny + jc) * P.nx + ic];
}

void poisson_setup(tg_ctx *C)
{
    if (C->pois) poisson_destroy(C);
    PoissonCtx *P = new PoissonCtx();
    C->pois = P;
    const Grid g = C->g;
    P->nx = g.mx - 2; P->ny = g.my - 2; P->nz = g.mz - 2;
    P->pi = g.pi; P->pj = g.pj; P->pk = g.pk;
    P->n = (int64_t)P->nx * P->ny * P->nz;
    P->pin = 0;
    P->ortho = C->orthogonal;
    const int64_t n = P->n;
    double **fine[] = {&P->gE1, &P->gE2, &P->gE3, &P->gN1, &P->gN2, &P->gN3, &P->gT1, &P->gT2, &P->gT3,
                       &P->x, &P->b, &P->r, &P->z, &P->p, &P->q, &P->rhat, &P->v, &P->s, &P->t, &P->aj, &P->xprev, &P->xprev2};
    for (double **f : fine) *f = dallocd(C, n);
    TG_CUDA(cudaMemsetAsync(C->d_scal + SC_PHIST, 0, sizeof(double), C->stream));   // empty guess history
    P->nblocks = vblocks(n);
    P->part = dallocd(C, 3 * (size_t)P->nblocks);
    k_gather_g<<<cgrid(P->nx, P->ny, P->nz), block3(), 0, C->stream>>>(g, C->m, *P);

    P->mg = mg_create(C, C->cfg.precision == TG_PREC_MIXED, P->gE1, P->gN2, P->gT3,
                      P->nx, P->ny, P->nz, P->pi, P->pj, P->pk);
    TG_CUDA(cudaGetLastError());
}

void poisson_destroy(tg_ctx *C)
{
    if (C->pois && C->pois->mg) mg_destroy(C->pois->mg);
    delete C->pois;   // device buffers are owned by the context allocation list
    C->pois = nullptr;
}

// host read of device scalars [off, off+cnt)
static void read_scal(tg_ctx *C, int off, int cnt)
{
    TG_CUDA(cudaMemcpyAsync(C->h_scal + off, C->d_scal + off, sizeof(double) * cnt, cudaMemcpyDeviceToHost, C->stream));
    TG_CUDA(cudaStreamSynchronize(C->stream));
}

// Krylov solve of L x = b from the current P.x (P.b set by the caller):
// preconditioned CG on orthogonal grids, BiCGStab otherwise. Stops at the
// relative residual rtol or, when divtol > 0, at dt * max|r aj| <= divtol.
static int krylov_solve(tg_ctx *C, tg_stats *st, double rtol, double divtol, int maxit)
{
    PoissonCtx &P = *C->pois;
    const int64_t n = P.n;
    cudaStream_t s = C->stream;
    const double dt = C->prm.dt;
    double *sc = C->d_scal;          // device scalar slots 0..7 used below
    double *hs = C->h_scal;

    dot3v(C, P.b, P.b, nullptr, sc + 0);
    apply_op(C, P.x, P.r);
    k_resid<<<vblocks(n), RB, 0, s>>>(n, P.b, P.r);   // r = b - L x
    dot3v(C, P.r, P.r, divtol > 0 ? P.aj : nullptr, sc + 3);
    read_scal(C, 0, 6);
    const double bn = std::sqrt(hs[0]);
    double rn = std::sqrt(hs[3]);
    double rmax = hs[5] * dt;
    if (st) st->poisson_initial_residual = bn > 0 ? rn / bn : rn;
    int it = 0;
    auto converged = [&]() {
        if (bn == 0.0) return true;
        if (rn / bn <= rtol) return true;
        if (divtol > 0 && rmax <= divtol) return true;
        return false;
    };
    bool ok = converged();
    if (P.ortho) {
        // preconditioned CG on the reduced SPD system (r[pin] = 0, x[pin] = 0)
        precondition(C, P.r, P.z, sc + 4);
        dot3v(C, P.r, P.z, nullptr, sc + 6);                 // rz at sc[6]
        TG_PROF(C, "pois_copy", k_copy<<<vblocks(n), RB, 0, s>>>(n, P.z, P.p));
        while (!converged() && it < maxit) {
            apply_op(C, P.p, P.q);
            k_zero_at<<<1, 1, 0, s>>>(P.q, P.pin);
            dot3v(C, P.p, P.q, nullptr, sc + 9);             // pq at sc[9]
            // x += alpha p, r -= alpha q; rr, sum r, max|r aj|
            TG_PROF(C, "pois_cg_update", k_cg_update_rr<<<P.nblocks, RB, 0, s>>>(n, sc + 6, sc + 9, P.x, P.p, P.r, P.q, divtol > 0 ? P.aj : nullptr, P.part));
            k_dot_final<<<1, RB, 0, s>>>(P.part, P.nblocks, sc + 3);
            read_scal(C, 3, 3);
            rn = std::sqrt(hs[3]); rmax = hs[5] * dt;
            it++;
            if (converged()) { ok = true; break; }
            precondition(C, P.r, P.z, sc + 4);
            k_scalar_copy<<<1, 1, 0, s>>>(sc + 6, sc + 14, 1);   // rz_old
            dot3v(C, P.r, P.z, nullptr, sc + 6);                 // rz_new
            TG_PROF(C, "pois_cg_dir", k_cg_dir<<<vblocks(n), RB, 0, s>>>(n, sc + 6, sc + 14, P.z, P.p));
        }
    } else {
        // right-preconditioned BiCGStab on the full pinned system
        // scalars: sc[20]=rho sc[21]=alpha sc[22]=omega sc[23]=rho_old
        TG_PROF(C, "pois_copy", k_copy<<<vblocks(n), RB, 0, s>>>(n, P.r, P.rhat));
        double one[4] = {1.0, 1.0, 1.0, 1.0};
        TG_CUDA(cudaMemcpyAsync(sc + 20, one, sizeof(one), cudaMemcpyHostToDevice, s));
        TG_CUDA(cudaMemsetAsync(P.p, 0, sizeof(double) * n, s));
        TG_CUDA(cudaMemsetAsync(P.v, 0, sizeof(double) * n, s));
        double *phat = P.z, *shat = P.q;
        bool restart_pending = false;
        while (!converged() && it < maxit) {
            if ((it > 0 && (it % 50) == 0) || restart_pending) {
                // restart from the true residual (limits recursive drift)
                restart_pending = false;
                apply_op(C, P.x, P.r);
                TG_PROF(C, "pois_resid", k_resid<<<vblocks(n), RB, 0, s>>>(n, P.b, P.r));
                k_copy<<<vblocks(n), RB, 0, s>>>(n, P.r, P.rhat);
                TG_CUDA(cudaMemcpyAsync(sc + 20, one, sizeof(one), cudaMemcpyHostToDevice, s));
                TG_CUDA(cudaMemsetAsync(P.p, 0, sizeof(double) * n, s));
                TG_CUDA(cudaMemsetAsync(P.v, 0, sizeof(double) * n, s));
            }
            dot3v(C, P.rhat, P.r, nullptr, sc + 24);            // rho_new at sc[24]
            k_scalar_copy<<<1, 1, 0, s>>>(sc + 20, sc + 23, 1); // rho_old
            k_scalar_copy<<<1, 1, 0, s>>>(sc + 24, sc + 20, 1); // rho
            TG_PROF(C, "pois_bicg_p", k_bicg_p<<<vblocks(n), RB, 0, s>>>(n, sc + 20, P.p, P.r, P.v));
            dot3v(C, P.p, P.p, nullptr, sc + 27);               // sum(p) at sc[28]
            precondition(C, P.p, phat, sc + 28);
            apply_op(C, phat, P.v);
            dot3v(C, P.rhat, P.v, nullptr, sc + 30);            // rhat.v at sc[30]
            TG_PROF(C, "pois_bicg_s", k_bicg_s<<<vblocks(n), RB, 0, s>>>(n, sc + 20, sc + 30, sc + 21, P.s, P.r, P.v));
            dot3v(C, P.s, P.s, nullptr, sc + 33);               // sum(s) at sc[34]
            precondition(C, P.s, shat, sc + 34);
            apply_op(C, shat, P.t);
            dot3v(C, P.t, P.s, nullptr, sc + 36);               // t.s
            dot3v(C, P.t, P.t, nullptr, sc + 39);               // t.t
            TG_PROF(C, "pois_bicg_x", k_bicg_x<<<vblocks(n), RB, 0, s>>>(n, sc + 21, sc + 36, sc + 39, sc + 22, P.x, phat, shat, P.r, P.s, P.t));
            dot3v(C, P.r, P.r, divtol > 0 ? P.aj : nullptr, sc + 3);
            read_scal(C, 3, 3);
            rn = std::sqrt(hs[3]); rmax = hs[5] * dt;
            it++;
            if (!std::isfinite(rn)) break;
            if (converged()) {
                // the recursive residual drifts from b - L x: stop only when
                // the true residual meets the test, else restart from it
                apply_op(C, P.x, P.r);
                TG_PROF(C, "pois_resid", k_resid<<<vblocks(n), RB, 0, s>>>(n, P.b, P.r));
                dot3v(C, P.r, P.r, divtol > 0 ? P.aj : nullptr, sc + 3);
                read_scal(C, 3, 3);
                rn = std::sqrt(hs[3]); rmax = hs[5] * dt;
                if (!converged()) restart_pending = true;
            }
        }
        ok = converged();
        // true residual (reported; it may sit slightly above the recursive one at round-off level)
        apply_op(C, P.x, P.r);
        TG_PROF(C, "pois_resid", k_resid<<<vblocks(n), RB, 0, s>>>(n, P.b, P.r));
        dot3v(C, P.r, P.r, divtol > 0 ? P.aj : nullptr, sc + 3);
        read_scal(C, 3, 3);
        rn = std::sqrt(hs[3]); rmax = hs[5] * dt;
    }
    k_zero_at<<<1, 1, 0, s>>>(P.x, P.pin);
    TG_CUDA(cudaGetLastError());
    if (st) {
        st->poisson_iterations = it;
        st->poisson_total_iterations += it;
        st->poisson_final_residual = bn > 0 ? rn / bn : rn;
    }
    if (!std::isfinite(rn)) return 2;
    return ok ? 0 : 1;
}

int poisson_solve(tg_ctx *C, tg_stats *st)
{
    PoissonCtx &P = *C->pois;
    const Grid g = C->g;
    cudaStream_t s = C->stream;
    const double rtol = C->cfg.poisson_rtol > 0 ? C->cfg.poisson_rtol : 1e-14;
    const int maxit = C->cfg.poisson_maxit > 0 ? C->cfg.poisson_maxit : 500;
    const dim3 cg3 = cgrid(P.nx, P.ny, P.nz);
    TG_PROF(C, "pois_set_rhs", k_set_rhs<<<cg3, block3(), 0, s>>>(g, C->s, P, C->prm.dt));
    k_extrapolate<<<vblocks(P.n), RB, 0, s>>>(P.n, P.x, P.xprev, P.xprev2, C->d_scal + SC_PHIST, guess_order(C));
    k_hist_next<<<1, 1, 0, s>>>(C->d_scal + SC_PHIST);
    k_zero_at<<<1, 1, 0, s>>>(P.x, P.pin);            // warm start from the previous solutions
    int rc = krylov_solve(C, st, rtol, C->cfg.poisson_div_tol, maxit);
    TG_PROF(C, "pois_phi_to_dmda", k_phi_to_dmda<<<cg3, block3(), 0, s>>>(g, C->s, P));
    TG_CUDA(cudaGetLastError());
    return rc;
}

// ---------------------------------------------------- captured solves
// Conditional node of `type` appended to the graph being captured on
// C->stream; body() is captured into the node's body graph on the auxiliary
// stream `aux` (C->stream points there while body() runs).
template <class F>
static void capture_conditional(tg_ctx *C, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                                cudaStream_t aux, F &&body)
{
    cudaStream_t s = C->stream;
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    TG_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &nd));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    TG_CUDA(cudaGraphAddNode(&node, graph, deps, nd, &cp));
    cudaGraph_t bg = cp.conditional.phGraph_out[0];
    TG_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    TG_CUDA(cudaStreamBeginCaptureToGraph(aux, bg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    {
        struct Swap { tg_ctx *C; cudaStream_t keep; ~Swap() { C->stream = keep; } } sw{C, s};
        C->stream = aux;
        body();
    }
    cudaGraph_t done;
    TG_CUDA(cudaStreamEndCapture(aux, &done));
}

// conditional handle of the graph being captured on C->stream (no default
// value: a kernel sets it before the node runs)
static cudaGraphConditionalHandle capture_handle(tg_ctx *C)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph;
    TG_CUDA(cudaStreamGetCaptureInfo(C->stream, &cs, nullptr, &graph, nullptr, nullptr));
    if (cs != cudaStreamCaptureStatusActive) throw CudaError{cudaErrorStreamCaptureInvalidated, "capture_handle: stream not capturing"};
    cudaGraphConditionalHandle h;
    TG_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 0, 0));
    return h;
}

__global__ void k_fill(int64_t n, double *a, double v)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) a[t] = v;
}
// BiCGStab restarts from the true residual every 50 iterations, and after a
// true residual that missed the stopping test (sc[53] set); clears sc[53]
__global__ void k_bicg_restart_flag(double *sc, cudaGraphConditionalHandle h)
{
    const int it = (int)sc[50];
    const bool pending = sc[53] != 0.0;
    sc[53] = 0.0;
    cudaGraphSetConditional(h, ((it > 0 && (it % 50) == 0) || pending) ? 1u : 0u);
}
// the recursive residual met the stopping test: verify it on b - L x
__global__ void k_bicg_verify_flag(const double *sc, double rtol, double divtol, double dt, cudaGraphConditionalHandle h)
{
    cudaGraphSetConditional(h, cg_converged(sc, rtol, divtol, dt) ? 1u : 0u);
}
// after the verification: restart on the next pass if the true residual missed
__global__ void k_bicg_mark_restart(double *sc, double rtol, double divtol, double dt)
{
    sc[53] = cg_converged(sc, rtol, divtol, dt) ? 0.0 : 1.0;
}

// krylov_solve for a step being captured into a CUDA graph: the iterations
// form a conditional WHILE node whose condition a one-thread kernel sets from
// the device residuals, so the solve needs no host round trip per iteration.
// The CG body is krylov_solve's iteration rotated to start with the direction
// update (p = z on the first pass), the BiCGStab body is krylov_solve's with
// its restarts and its true-residual check as conditional IF nodes; both perform the same
// arithmetic in the same order. Statistics go to the ST_* slots from base.
static void krylov_capture(tg_ctx *C, double rtol, double divtol, int maxit, int base)
{
    PoissonCtx &P = *C->pois;
    const int64_t n = P.n;
    cudaStream_t s = C->stream;
    const double dt = C->prm.dt;
    double *sc = C->d_scal;
    const int vb = vblocks(n);
    dot3v(C, P.b, P.b, nullptr, sc + 0);
    apply_op(C, P.x, P.r);
    k_resid<<<vb, RB, 0, s>>>(n, P.b, P.r);
    dot3v(C, P.r, P.r, divtol > 0 ? P.aj : nullptr, sc + 3);
    if (P.ortho) {
        cudaGraphConditionalHandle h = capture_handle(C);
        k_cg_start<<<1, 1, 0, s>>>(sc, rtol, divtol, dt, maxit, h, base);
        capture_conditional(C, h, cudaGraphCondTypeWhile, C->aux[0], [&]() {
            cudaStream_t a = C->stream;
            precondition(C, P.r, P.z, sc + 4);
            k_scalar_copy<<<1, 1, 0, a>>>(sc + 6, sc + 14, 1);           // rz_old
            dot3v(C, P.r, P.z, nullptr, sc + 6);                          // rz
            k_cg_dir_loop<<<vb, RB, 0, a>>>(n, sc, P.z, P.p);
            apply_op(C, P.p, P.q);
            k_zero_at<<<1, 1, 0, a>>>(P.q, P.pin);
            dot3v(C, P.p, P.q, nullptr, sc + 9);                          // pq
            k_cg_update_rr<<<P.nblocks, RB, 0, a>>>(n, sc + 6, sc + 9, P.x, P.p, P.r, P.q, divtol > 0 ? P.aj : nullptr, P.part);
            k_dot_final<<<1, RB, 0, a>>>(P.part, P.nblocks, sc + 3);      // rr, sum r, max|r aj|
            k_cg_next<<<1, 1, 0, a>>>(sc, rtol, divtol, dt, maxit, h);
        });
    } else {
        k_copy<<<vb, RB, 0, s>>>(n, P.r, P.rhat);
        k_fill<<<1, 32, 0, s>>>(4, sc + 20, 1.0);
        k_fill<<<vb, RB, 0, s>>>(n, P.p, 0.0);
        k_fill<<<vb, RB, 0, s>>>(n, P.v, 0.0);
        double *phat = P.z, *shat = P.q;
        cudaGraphConditionalHandle h = capture_handle(C);
        k_cg_start<<<1, 1, 0, s>>>(sc, rtol, divtol, dt, maxit, h, base);
        capture_conditional(C, h, cudaGraphCondTypeWhile, C->aux[0], [&]() {
            cudaStream_t a = C->stream;
            cudaGraphConditionalHandle hr = capture_handle(C);
            k_bicg_restart_flag<<<1, 1, 0, a>>>(sc, hr);
            capture_conditional(C, hr, cudaGraphCondTypeIf, C->aux[1], [&]() {
                cudaStream_t b = C->stream;
                apply_op(C, P.x, P.r);
                k_resid<<<vb, RB, 0, b>>>(n, P.b, P.r);
                k_copy<<<vb, RB, 0, b>>>(n, P.r, P.rhat);
                k_fill<<<1, 32, 0, b>>>(4, sc + 20, 1.0);
                k_fill<<<vb, RB, 0, b>>>(n, P.p, 0.0);
                k_fill<<<vb, RB, 0, b>>>(n, P.v, 0.0);
            });
            dot3v(C, P.rhat, P.r, nullptr, sc + 24);
            k_scalar_copy<<<1, 1, 0, a>>>(sc + 20, sc + 23, 1);
            k_scalar_copy<<<1, 1, 0, a>>>(sc + 24, sc + 20, 1);
            k_bicg_p<<<vb, RB, 0, a>>>(n, sc + 20, P.p, P.r, P.v);
            dot3v(C, P.p, P.p, nullptr, sc + 27);
            precondition(C, P.p, phat, sc + 28);
            apply_op(C, phat, P.v);
            dot3v(C, P.rhat, P.v, nullptr, sc + 30);
            k_bicg_s<<<vb, RB, 0, a>>>(n, sc + 20, sc + 30, sc + 21, P.s, P.r, P.v);
            dot3v(C, P.s, P.s, nullptr, sc + 33);
            precondition(C, P.s, shat, sc + 34);
            apply_op(C, shat, P.t);
            dot3v(C, P.t, P.s, nullptr, sc + 36);
            dot3v(C, P.t, P.t, nullptr, sc + 39);
            k_bicg_x<<<vb, RB, 0, a>>>(n, sc + 21, sc + 36, sc + 39, sc + 22, P.x, phat, shat, P.r, P.s, P.t);
            dot3v(C, P.r, P.r, divtol > 0 ? P.aj : nullptr, sc + 3);
            cudaGraphConditionalHandle hv = capture_handle(C);
            k_bicg_verify_flag<<<1, 1, 0, a>>>(sc, rtol, divtol, dt, hv);
            capture_conditional(C, hv, cudaGraphCondTypeIf, C->aux[1], [&]() {
                cudaStream_t b = C->stream;
                apply_op(C, P.x, P.r);
                k_resid<<<vb, RB, 0, b>>>(n, P.b, P.r);
                dot3v(C, P.r, P.r, divtol > 0 ? P.aj : nullptr, sc + 3);
                k_bicg_mark_restart<<<1, 1, 0, b>>>(sc, rtol, divtol, dt);
            });
            k_cg_next<<<1, 1, 0, a>>>(sc, rtol, divtol, dt, maxit, h);
        });
        // true residual (reported)
        apply_op(C, P.x, P.r);
        k_resid<<<vb, RB, 0, s>>>(n, P.b, P.r);
        dot3v(C, P.r, P.r, divtol > 0 ? P.aj : nullptr, sc + 3);
    }
    k_zero_at<<<1, 1, 0, s>>>(P.x, P.pin);
    k_cg_finish<<<1, 1, 0, s>>>(sc, base);
}

// poisson_solve for a step being captured into a CUDA graph
void poisson_solve_capture(tg_ctx *C)
{
    PoissonCtx &P = *C->pois;
    const Grid g = C->g;
    cudaStream_t s = C->stream;
    const double rtol = C->cfg.poisson_rtol > 0 ? C->cfg.poisson_rtol : 1e-14;
    const int maxit = C->cfg.poisson_maxit > 0 ? C->cfg.poisson_maxit : 500;
    const dim3 cg3 = cgrid(P.nx, P.ny, P.nz);
    k_set_rhs<<<cg3, block3(), 0, s>>>(g, C->s, P, C->prm.dt);
    k_extrapolate<<<vblocks(P.n), RB, 0, s>>>(P.n, P.x, P.xprev, P.xprev2, C->d_scal + SC_PHIST, guess_order(C));
    k_hist_next<<<1, 1, 0, s>>>(C->d_scal + SC_PHIST);
    k_zero_at<<<1, 1, 0, s>>>(P.x, P.pin);
    krylov_capture(C, rtol, C->cfg.poisson_div_tol, maxit, SC_G);
    k_phi_to_dmda<<<cg3, block3(), 0, s>>>(g, C->s, P);
    TG_CUDA(cudaGetLastError());
}

// poisson_solve_adjoint for a reversed step being captured into a CUDA graph
// (statistics in the SC_ADJ slots)
void poisson_solve_adjoint_capture(tg_ctx *C, const double *rhs, double *lam, double rtol)
{
    PoissonCtx &P = *C->pois;
    cudaStream_t s = C->stream;
    const int64_t n = P.n;
    TG_CUDA(cudaMemcpyAsync(P.v, P.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_negcopy<<<vblocks(n), RB, 0, s>>>(n, rhs, P.b);
    k_zero_at<<<1, 1, 0, s>>>(P.b, P.pin);
    TG_CUDA(cudaMemcpyAsync(P.x, lam, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    krylov_capture(C, rtol, 0.0, C->cfg.poisson_maxit > 0 ? C->cfg.poisson_maxit : 500, SC_ADJ);
    TG_CUDA(cudaMemcpyAsync(lam, P.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    TG_CUDA(cudaMemcpyAsync(P.x, P.v, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    TG_CUDA(cudaGetLastError());
}

// Adjoint pressure solve: lam = A^-T rhs for the pinned operator A of
// SetCoeffMatrix (rhs and lam compact, pinned entry of rhs ignored,
// lam[pin] = 0). On orthogonal grids the operator without the pinned row and
// column is symmetric, so this is the forward Krylov solve started from the
// value lam holds on entry (the caller's guess, adjoint_guess); the
// forward warm start P.x is kept. Returns 3 for the non-symmetric curvilinear
// operator.
int poisson_solve_adjoint(tg_ctx *C, const double *rhs, double *lam, double rtol, tg_stats *st)
{
    PoissonCtx &P = *C->pois;
    if (!P.ortho) return 3;
    cudaStream_t s = C->stream;
    const int64_t n = P.n;
    TG_CUDA(cudaMemcpyAsync(P.v, P.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_negcopy<<<vblocks(n), RB, 0, s>>>(n, rhs, P.b);       // the solver's operator is L = -A
    k_zero_at<<<1, 1, 0, s>>>(P.b, P.pin);
    TG_CUDA(cudaMemcpyAsync(P.x, lam, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    int rc = krylov_solve(C, st, rtol, 0.0, C->cfg.poisson_maxit > 0 ? C->cfg.poisson_maxit : 500);
    TG_CUDA(cudaMemcpyAsync(lam, P.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    TG_CUDA(cudaMemcpyAsync(P.x, P.v, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    return rc;
}

void adjoint_guess(tg_ctx *C, double *lam, double *lp, double *lp2, double *hist)
{
    PoissonCtx &P = *C->pois;
    cudaStream_t s = C->stream;
    k_extrapolate<<<vblocks(P.n), RB, 0, s>>>(P.n, lam, lp, lp2, hist, guess_order(C));
    k_hist_next<<<1, 1, 0, s>>>(hist);
    k_zero_at<<<1, 1, 0, s>>>(lam, P.pin);
    TG_CUDA(cudaGetLastError());
}

// compact Poisson solution vectors (the next solve extrapolates x, xprev, xprev2): snapshots
double *poisson_x(tg_ctx *C) { return C->pois->x; }
double *poisson_xprev(tg_ctx *C) { return C->pois->xprev; }
double *poisson_xprev2(tg_ctx *C) { return C->pois->xprev2; }
int64_t poisson_n(tg_ctx *C) { return C->pois->n; }

}  // namespace tg
