// Geometric multigrid V-cycle for the 7-point part of TOSCA's pressure
// operator, used as the preconditioner of the Krylov pressure solve.
//
//  * coarsening: every direction with >= 3 cells is halved (n -> ceil(n/2):
//    fine cells 2I and 2I+1 form coarse cell I; the last coarse cell of an
//    odd direction holds one fine cell) until a level has <= 1024 cells, so
//    every grid size coarsens; coarse face coefficients are face sums of the
//    fine ones, halved when the face-normal direction is coarsened
//  * transfers: summed residual restriction, piecewise-constant prolongation
//  * smoothing: zebra j-line Gauss-Seidel when j (the wall-normal direction)
//    is non-periodic, red-black point Gauss-Seidel otherwise; 2 pre + 2 post
//    sweeps in reversed colour order, so the cycle is a symmetric operator
//  * coarsest level (<= 1024 cells): the pseudo-inverse on mean-free vectors,
//    (I - 11^T/n) (A + 11^T/n)^-1 (I - 11^T/n), formed densely at set-up and
//    applied as one matrix-vector product (a warp per row)
//
// Layout: on every level the cells of an (k, j) row are stored with even i
// first and odd i second. The cells of one zebra colour in a k-row then form
// one contiguous half-row, so a warp of same-colour lines reads 32 adjacent
// doubles (or floats): full coalescing, no idle half-warps.
//
// The tridiagonal line matrices never change, so their LU factors (c' and
// 1/m of the Thomas algorithm) are computed once at setup and a line solve is
// a chain of FMAs. On the large levels a block solves 32 same-colour lines at
// once: each of its warps takes one chunk of j, runs the forward and backward
// recurrences of its chunk as affine maps (coalesced loads, all warps in
// flight), and the chunk ends are combined by shuffle scans. The small levels
// use one warp segment per line (k_line_warp). An earlier design ran the
// levels of <= 1024 cells, smoothing included, in one single-block kernel:
// 71-73 us per V-cycle at 128 x 64 x 64, one SM's latency chain; the dense
// solve at the first level of <= 1024 cells replaces it.
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <vector>

#include "tg_mg.cuh"

namespace tg {

template <class T>
struct Lvl {
    int nx, ny, nz, pi, pj, pk;
    int h0;                  // number of even i in a row (first half of the row)
    int cx, cy, cz;          // coarsening factors to the next level
    int64_t n;
    T *aE, *aN, *aT, *diag;  // east/north/top face coefficients, diagonal
    T *cp, *minv;            // Thomas factors of the j-lines
    T *x, *r, *tmp;          // unknown, right-hand side, line scratch
};

constexpr int MAXL = 16;
constexpr int COARSEST_CELLS = 1024;   // coarsening stops at the first level this small
constexpr int LINE_NW = 32;         // warps per block of the chunked line solver (one line chunk each)

struct MG {
    bool fp32;
    int nlev, line, nu;
    Lvl<double> Ld[MAXL];
    Lvl<float> Lf[MAXL];
    double *Bd;              // projected dense pseudo-inverse of the coarsest level (FP64 multigrid)
    float *Bf;               // the same in FP32 (mixed-precision multigrid)
    int nc;
};

template <class T> inline const T *mg_dense(const MG *mg);
template <> inline const double *mg_dense<double>(const MG *mg) { return mg->Bd; }
template <> inline const float *mg_dense<float>(const MG *mg) { return mg->Bf; }

int mg_levels(const MG *mg) { return mg->nlev; }

namespace {

__device__ __forceinline__ int spos(int i, int h0) { return (i & 1) ? (h0 + (i >> 1)) : (i >> 1); }
template <class T>
__device__ __forceinline__ int sidx(const Lvl<T> &L, int k, int j, int i) { return (k * L.ny + j) * L.nx + spos(i, L.h0); }

// sum of a_f x_nb over the i and k neighbours (and j when with_j)
template <class T>
__device__ __forceinline__ T nb_sum(const Lvl<T> &L, int k, int j, int i, int c, bool with_j)
{
    T s = T(0);
    if (i + 1 < L.nx)  s += L.aE[c] * L.x[sidx(L, k, j, i + 1)];
    else if (L.pi)     s += L.aE[c] * L.x[sidx(L, k, j, 0)];
    if (i > 0)         { int w = sidx(L, k, j, i - 1); s += L.aE[w] * L.x[w]; }
    else if (L.pi)     { int w = sidx(L, k, j, L.nx - 1); s += L.aE[w] * L.x[w]; }
    if (k + 1 < L.nz)  s += L.aT[c] * L.x[sidx(L, k + 1, j, i)];
    else if (L.pk)     s += L.aT[c] * L.x[sidx(L, 0, j, i)];
    if (k > 0)         { int b = sidx(L, k - 1, j, i); s += L.aT[b] * L.x[b]; }
    else if (L.pk)     { int b = sidx(L, L.nz - 1, j, i); s += L.aT[b] * L.x[b]; }
    if (with_j) {
        if (j + 1 < L.ny)  s += L.aN[c] * L.x[c + L.nx];
        else if (L.pj)     s += L.aN[c] * L.x[sidx(L, k, 0, i)];
        if (j > 0)         s += L.aN[c - L.nx] * L.x[c - L.nx];
        else if (L.pj)     { int q = sidx(L, k, L.ny - 1, i); s += L.aN[q] * L.x[q]; }
    }
    return s;
}

// ------------------------------------------------------------------- setup
template <class T>
__global__ void k_l0_coeffs(const double *aE, const double *aN, const double *aT, Lvl<T> L)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= L.nx || j >= L.ny || k >= L.nz) return;
    int q = (k * L.ny + j) * L.nx + i, c = sidx(L, k, j, i);
    L.aE[c] = (T)((i < L.nx - 1 || L.pi) ? aE[q] : 0.0);
    L.aN[c] = (T)((j < L.ny - 1 || L.pj) ? aN[q] : 0.0);
    L.aT[c] = (T)((k < L.nz - 1 || L.pk) ? aT[q] : 0.0);
}

template <class T>
__global__ void k_coarsen(Lvl<T> F, Lvl<T> Cc)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y, K = blockIdx.z * blockDim.z + threadIdx.z;
    if (I >= Cc.nx || J >= Cc.ny || K >= Cc.nz) return;
    // fine cells of the aggregate (the last one of an odd direction has one)
    const int i0 = F.cx * I, i1 = min(i0 + F.cx, F.nx), j0 = F.cy * J, j1 = min(j0 + F.cy, F.ny);
    const int k0 = F.cz * K, k1 = min(k0 + F.cz, F.nz);
    double sE = 0.0, sN = 0.0, sT = 0.0;
    for (int k = k0; k < k1; k++) for (int j = j0; j < j1; j++) sE += (double)F.aE[sidx(F, k, j, i1 - 1)];
    for (int k = k0; k < k1; k++) for (int i = i0; i < i1; i++) sN += (double)F.aN[sidx(F, k, j1 - 1, i)];
    for (int j = j0; j < j1; j++) for (int i = i0; i < i1; i++) sT += (double)F.aT[sidx(F, k1 - 1, j, i)];
    int c = sidx(Cc, K, J, I);
    Cc.aE[c] = (T)(sE * (F.cx == 2 ? 0.5 : 1.0));
    Cc.aN[c] = (T)(sN * (F.cy == 2 ? 0.5 : 1.0));
    Cc.aT[c] = (T)(sT * (F.cz == 2 ? 0.5 : 1.0));
}

template <class T>
__global__ void k_diag(Lvl<T> L)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= L.nx || j >= L.ny || k >= L.nz) return;
    int c = sidx(L, k, j, i);
    double aW = i > 0 ? (double)L.aE[sidx(L, k, j, i - 1)] : (L.pi ? (double)L.aE[sidx(L, k, j, L.nx - 1)] : 0.0);
    double aS = j > 0 ? (double)L.aN[sidx(L, k, j - 1, i)] : (L.pj ? (double)L.aN[sidx(L, k, L.ny - 1, i)] : 0.0);
    double aB = k > 0 ? (double)L.aT[sidx(L, k - 1, j, i)] : (L.pk ? (double)L.aT[sidx(L, L.nz - 1, j, i)] : 0.0);
    L.diag[c] = (T)((double)L.aE[c] + aW + (double)L.aN[c] + aS + (double)L.aT[c] + aB);
}

// Thomas factors of every j-line: m_j = diag_j + aS_j c'_{j-1}, c'_j = -aN_j/m_j
template <class T>
__global__ void k_line_factors(Lvl<T> L)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= L.nx || k >= L.nz) return;
    double cprev = 0.0;
    for (int j = 0; j < L.ny; j++) {
        int c = sidx(L, k, j, i);
        double aS = j > 0 ? (double)L.aN[c - L.nx] : 0.0;
        double aN = j < L.ny - 1 ? (double)L.aN[c] : 0.0;
        double m = (double)L.diag[c] + aS * cprev;
        double cp = -aN / m;
        L.cp[c] = (T)cp;
        L.minv[c] = (T)(1.0 / m);
        cprev = cp;
    }
}

// ---------------------------------------------------------------- smoothing
// one j-line of colour `color` (zebra Gauss-Seidel): forward substitution with
// the stored factors, then back substitution
template <class T>
__device__ __forceinline__ void line_solve(const Lvl<T> &L, int k, int i, bool zx)
{
    T dprev = T(0);
    const int nx = L.nx;
    int c = sidx(L, k, 0, i);
    for (int j = 0; j < L.ny; j++, c += nx) {
        T rhs = zx ? L.r[c] : L.r[c] + nb_sum(L, k, j, i, c, false);
        T aS = j > 0 ? L.aN[c - nx] : T(0);
        T dp = (rhs + aS * dprev) * L.minv[c];
        L.tmp[c] = dp;
        dprev = dp;
    }
    T xn = T(0);
    c -= nx;
    for (int j = L.ny - 1; j >= 0; j--, c -= nx) {
        T xv = L.tmp[c] - L.cp[c] * xn;
        L.x[c] = xv;
        xn = xv;
    }
}

// Chunked zebra line solve (nx even): lane -> one of 32 consecutive
// same-colour lines (flattened over (k, t)), warp w -> j in [w*CJ, (w+1)*CJ).
// dp_j = (rhs_j + aS_j dp_{j-1}) / m_j and x_j = dp_j - c'_j x_{j+1} are first
// order affine recurrences: each warp composes its chunk into (offset,
// multiplier) pairs, the chunk ends of a line are chained by a shuffle scan of
// those affine maps (warp w scans line w over the 32 chunks, one per lane),
// and each warp finishes its chunk. The chunk-end arrays are padded to a row
// stride of 33 so that both the per-chunk writes and the per-line scan reads
// are free of bank conflicts.
// The loads of a chunk do not depend on each other, so they are issued in an
// unrolled pass of compile-time length CJ before the recurrence runs on
// shared memory.
template <class T, int CJ, bool ZX>
__global__ void __launch_bounds__(LINE_NW * 32) k_line_chunked(Lvl<T> L, int color)
{
    extern __shared__ unsigned char smraw[];
    T *D = reinterpret_cast<T *>(smraw);            // [NW*CJ][32] offsets
    T *Mu = D + LINE_NW * CJ * 32;                  // [NW*CJ][32] multipliers
    T *SD = Mu + LINE_NW * CJ * 32;                 // [NW][33] chunk offsets
    T *SM = SD + LINE_NW * 33;                      // [NW][33] chunk multipliers
    T *ST = SM + LINE_NW * 33;                      // [NW][33] chunk boundary values
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int half = L.nx >> 1;
    const int lid = blockIdx.x * 32 + lane;
    const bool active = lid < half * L.nz;
    const int k = active ? lid / half : 0, t = active ? lid % half : 0;
    const int i = 2 * t + ((color ^ k) & 1);
    const int nx = L.nx, ny = L.ny;
    const int j0 = w * CJ;
    // (1a) independent loads: D = rhs * minv, Mu = aS * minv
    if (active) {
        const int c0 = sidx(L, k, j0, i);
        #pragma unroll
        for (int u = 0; u < CJ; u++) {
            const int j = j0 + u;
            if (j < ny) {
                const int c = c0 + u * nx;
                T rhs = ZX ? L.r[c] : L.r[c] + nb_sum(L, k, j, i, c, false);
                T mi = L.minv[c];
                T aS = j > 0 ? L.aN[c - nx] : T(0);
                D[(w * CJ + u) * 32 + lane] = rhs * mi;
                Mu[(w * CJ + u) * 32 + lane] = aS * mi;
            }
        }
    }
    // (1b) local forward recurrence of the chunk
    T dl = T(0), ml = T(1);
    #pragma unroll
    for (int u = 0; u < CJ; u++) {
        if (active && j0 + u < ny) {
            const int q = (w * CJ + u) * 32 + lane;
            const T f = Mu[q];
            dl = D[q] + f * dl;
            ml = f * ml;
            D[q] = dl;
            Mu[q] = ml;
        }
    }
    static_assert(LINE_NW == 32, "one lane per chunk in the chunk-end scans");
    SD[w * 33 + lane] = dl;
    SM[w * 33 + lane] = ml;
    __syncthreads();
    {
        // warp w, lane q: chunk q of line w; inclusive scan of s -> B + A s
        // over the chunks, then shifted by one (the value entering chunk q)
        T A = SM[lane * 33 + w], B = SD[lane * 33 + w];
        #pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T Ap = __shfl_up_sync(0xffffffffu, A, d), Bp = __shfl_up_sync(0xffffffffu, B, d);
            if (lane >= d) { B = A * Bp + B; A = A * Ap; }
        }
        const T in = __shfl_up_sync(0xffffffffu, B, 1);
        ST[lane * 33 + w] = lane == 0 ? T(0) : in;
    }
    __syncthreads();
    const T st = ST[w * 33 + lane];
    // (3) backward recurrence of the chunk; c' loaded before the chain
    T cpv[CJ];
    if (active) {
        const int c0 = sidx(L, k, j0, i);
        #pragma unroll
        for (int u = 0; u < CJ; u++) cpv[u] = (j0 + u < ny) ? L.cp[c0 + u * nx] : T(0);
    }
    T xl = T(0), nl = T(1);
    #pragma unroll
    for (int u = CJ - 1; u >= 0; u--) {
        if (active && j0 + u < ny) {
            const int q = (w * CJ + u) * 32 + lane;
            const T dp = D[q] + Mu[q] * st;
            xl = dp - cpv[u] * xl;
            nl = -cpv[u] * nl;
            D[q] = xl;
            Mu[q] = nl;
        }
    }
    SD[w * 33 + lane] = xl;
    SM[w * 33 + lane] = nl;
    __syncthreads();
    {
        // backward: inclusive scan from the last chunk down, shifted by one
        T C = SM[lane * 33 + w], E = SD[lane * 33 + w];
        #pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T Cn = __shfl_down_sync(0xffffffffu, C, d), En = __shfl_down_sync(0xffffffffu, E, d);
            if (lane + d < 32) { E = C * En + E; C = C * Cn; }
        }
        const T in = __shfl_down_sync(0xffffffffu, E, 1);
        ST[lane * 33 + w] = lane == 31 ? T(0) : in;
    }
    __syncthreads();
    const T xnext = ST[w * 33 + lane];
    if (active) {
        const int c0 = sidx(L, k, j0, i);
        #pragma unroll
        for (int u = 0; u < CJ; u++)
            if (j0 + u < ny) {
                const int q = (w * CJ + u) * 32 + lane;
                L.x[c0 + u * nx] = D[q] + Mu[q] * xnext;
            }
    }
}

template <class T>
size_t line_chunk_smem_cj(int cj) { return sizeof(T) * (2 * (size_t)LINE_NW * cj * 32 + 3 * LINE_NW * 33); }

// chunk length (power of two >= ceil(ny / NW)) of the line solver; 0 if the
// lines are too long for its shared memory
template <class T>
int line_cj(int ny)
{
    int need = (ny + LINE_NW - 1) / LINE_NW;
    int cj = 1;
    while (cj < need) cj <<= 1;
    return (cj <= 32 && line_chunk_smem_cj<T>(cj) <= 200 * 1024) ? cj : 0;
}

template <class T, bool ZX>
void launch_line_chunked_zx(Lvl<T> &F, int color, int cj, int nb, size_t shm, cudaStream_t st)
{
    switch (cj) {
    case 1: k_line_chunked<T, 1, ZX><<<nb, LINE_NW * 32, shm, st>>>(F, color); break;
    case 2: k_line_chunked<T, 2, ZX><<<nb, LINE_NW * 32, shm, st>>>(F, color); break;
    case 4: k_line_chunked<T, 4, ZX><<<nb, LINE_NW * 32, shm, st>>>(F, color); break;
    case 8: k_line_chunked<T, 8, ZX><<<nb, LINE_NW * 32, shm, st>>>(F, color); break;
    case 16: k_line_chunked<T, 16, ZX><<<nb, LINE_NW * 32, shm, st>>>(F, color); break;
    default: k_line_chunked<T, 32, ZX><<<nb, LINE_NW * 32, shm, st>>>(F, color); break;
    }
}

// zx: the unknown is zero on the level (the first sweep after k_in or the
// restriction), so the off-line neighbour terms are skipped
template <class T>
void launch_line_chunked(Lvl<T> &F, int color, bool zx, cudaStream_t st)
{
    const int lines = (F.nx >> 1) * F.nz;
    const int nb = (lines + 31) / 32;
    const int cj = line_cj<T>(F.ny);
    const size_t shm = line_chunk_smem_cj<T>(cj);
    if (zx) launch_line_chunked_zx<T, true>(F, color, cj, nb, shm, st);
    else launch_line_chunked_zx<T, false>(F, color, cj, nb, shm, st);
}

// Warp-segmented zebra line solve for the coarse levels (nx even, ny <= 32 CJ):
// a line is a segment of P lanes (P a power of two, P CJ >= ny), each lane
// CJ consecutive cells held in registers; the forward and backward Thomas
// recurrences are composed per lane into affine maps and chained across the
// segment by shuffle scans. No block barrier and
// no scratch array: on the small levels a launch costs about one round of
// loads plus the two scans.
template <class T, int CJ, bool ZX>
__global__ void __launch_bounds__(256) k_line_warp(Lvl<T> L, int color, int P)
{
    const int lane = threadIdx.x & 31, sl = lane & (P - 1);
    const int half = L.nx >> 1, nlines = half * L.nz;
    const int line = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (32 / P) + (lane / P);
    const bool on = line < nlines;
    const int k = on ? line / half : 0, t = on ? line - k * half : 0;
    const int i = 2 * t + ((color ^ k) & 1);
    const int nx = L.nx, ny = L.ny, j0 = sl * CJ;
    const int c0 = on ? sidx(L, k, j0, i) : 0;
    T a[CJ], b[CJ], cp[CJ];
    T A = T(1), B = T(0);
    #pragma unroll
    for (int u = 0; u < CJ; u++) {
        const int j = j0 + u;
        a[u] = T(0); b[u] = T(0); cp[u] = T(0);
        if (on && j < ny) {
            const int c = c0 + u * nx;
            const T mi = L.minv[c];
            a[u] = j > 0 ? mi * L.aN[c - nx] : T(0);
            b[u] = mi * (ZX ? L.r[c] : L.r[c] + nb_sum(L, k, j, i, c, false));
            cp[u] = L.cp[c];
            B = a[u] * B + b[u];
            A = a[u] * A;
        }
    }
    for (int d = 1; d < P; d <<= 1) {
        const T Ap = __shfl_up_sync(0xffffffffu, A, d, P), Bp = __shfl_up_sync(0xffffffffu, B, d, P);
        if (sl >= d) { B = A * Bp + B; A = A * Ap; }
    }
    T dp = __shfl_up_sync(0xffffffffu, B, 1, P);
    if (sl == 0) dp = T(0);
    T C = T(1), D = T(0);
    #pragma unroll
    for (int u = 0; u < CJ; u++) {
        dp = a[u] * dp + b[u];
        b[u] = dp;                       // b now holds dp_j
    }
    #pragma unroll
    for (int u = CJ - 1; u >= 0; u--) {
        if (on && j0 + u < ny) { D = -cp[u] * D + b[u]; C = -cp[u] * C; }
    }
    for (int d = 1; d < P; d <<= 1) {
        const T Cn = __shfl_down_sync(0xffffffffu, C, d, P), Dn = __shfl_down_sync(0xffffffffu, D, d, P);
        if (sl + d < P) { D = C * Dn + D; C = C * Cn; }
    }
    T xv = __shfl_down_sync(0xffffffffu, D, 1, P);
    if (sl == P - 1) xv = T(0);
    #pragma unroll
    for (int u = CJ - 1; u >= 0; u--) {
        if (on && j0 + u < ny) {
            xv = b[u] - cp[u] * xv;
            L.x[c0 + u * nx] = xv;
        }
    }
}

// levels of at most this many cells use k_line_warp; larger ones the chunked
// solver, whose coalesced loads win there. ABL 256 x 256 x 128, coarse-level
// smoothing per step: 0.632 ms chunked on every level, 0.589 ms warp-segmented
// on the levels of <= 16,384 cells, 0.621 ms on those of <= 131,072, 0.927 ms
// on all
constexpr int64_t LINE_WARP_CELLS = 65536;

// cells per lane of k_line_warp (0: lines longer than 32 x 4 cells)
inline int line_warp_cj(int ny) { return ny <= 32 ? 1 : ny <= 64 ? 2 : ny <= 128 ? 4 : 0; }

template <class T>
void launch_line_warp(Lvl<T> &F, int color, bool zx, cudaStream_t st)
{
    const int cj = line_warp_cj(F.ny);
    int P = 1;
    while (P * cj < F.ny) P <<= 1;
    const int lines = (F.nx >> 1) * F.nz, per_warp = 32 / P;
    const int warps = (lines + per_warp - 1) / per_warp;
    const int nb = (warps * 32 + 255) / 256;
    auto go = [&](auto zxc) {
        constexpr bool Z = decltype(zxc)::value;
        switch (cj) {
        case 1: k_line_warp<T, 1, Z><<<nb, 256, 0, st>>>(F, color, P); break;
        case 2: k_line_warp<T, 2, Z><<<nb, 256, 0, st>>>(F, color, P); break;
        default: k_line_warp<T, 4, Z><<<nb, 256, 0, st>>>(F, color, P); break;
        }
    };
    if (zx) go(std::true_type{});
    else go(std::false_type{});
}

template <class T>
void set_line_smem_attrs()
{
    auto set = [](const void *f, int cj) {
        const size_t b = line_chunk_smem_cj<T>(cj);
        if (b <= 200 * 1024) TG_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b));
    };
    set((const void *)k_line_chunked<T, 1, false>, 1);
    set((const void *)k_line_chunked<T, 2, false>, 2);
    set((const void *)k_line_chunked<T, 4, false>, 4);
    set((const void *)k_line_chunked<T, 8, false>, 8);
    set((const void *)k_line_chunked<T, 16, false>, 16);
    set((const void *)k_line_chunked<T, 32, false>, 32);
    set((const void *)k_line_chunked<T, 1, true>, 1);
    set((const void *)k_line_chunked<T, 2, true>, 2);
    set((const void *)k_line_chunked<T, 4, true>, 4);
    set((const void *)k_line_chunked<T, 8, true>, 8);
    set((const void *)k_line_chunked<T, 16, true>, 16);
    set((const void *)k_line_chunked<T, 32, true>, 32);
}


// lines of one colour: (i + k) & 1 == color, i.e. i of parity (color ^ k) & 1
template <class T>
__global__ void k_smooth_line(Lvl<T> L, int color, int zx)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (k >= L.nz) return;
    int q = (color ^ k) & 1;
    int cnt = q ? (L.nx >> 1) : ((L.nx + 1) >> 1);
    if (t >= cnt) return;
    line_solve(L, k, 2 * t + q, zx != 0);
}

template <class T>
__device__ __forceinline__ void point_update(const Lvl<T> &L, int k, int j, int i, bool zx)
{
    int c = sidx(L, k, j, i);
    L.x[c] = (zx ? L.r[c] : L.r[c] + nb_sum(L, k, j, i, c, true)) / L.diag[c];
}

template <class T>
__global__ void k_smooth_rb(Lvl<T> L, int color, int zx)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= L.nx || j >= L.ny || k >= L.nz) return;
    if (((i + j + k) & 1) != color) return;
    point_update(L, k, j, i, zx != 0);
}

// ------------------------------------------------------------------ transfers
// Grid restriction: a block takes 32 consecutive coarse cells of one coarse
// row (J, K) and one thread per fine cell under them (up to 64 x 2 x 2), so
// the loads of all fine residuals issue at once; the residuals meet in shared
// memory and thread I of the block sums its coarse cell's fine residuals
// r - diag x + (off-diagonal terms) in k, j, i order.
constexpr int RS_I = 32;    // coarse cells per block
template <class T>
__global__ void __launch_bounds__(8 * RS_I) k_restrict(Lvl<T> F, Lvl<T> Cc)
{
    __shared__ T res[2][2][2 * RS_I];
    const int t = threadIdx.x, fo = t & (2 * RS_I - 1), dj = (t >> 6) & 1, dk = t >> 7;
    const int I0 = blockIdx.x * RS_I, J = blockIdx.y, K = blockIdx.z;
    const int i = F.cx * I0 + fo, j = F.cy * J + dj, k = F.cz * K + dk;
    T v = T(0);
    if (fo < F.cx * RS_I && dj < F.cy && dk < F.cz && i < F.nx && j < F.ny && k < F.nz) {
        const int c = sidx(F, k, j, i);
        v = F.r[c] - F.diag[c] * F.x[c] + nb_sum(F, k, j, i, c, true);
    }
    res[dk][dj][fo] = v;
    __syncthreads();
    const int I = I0 + t;
    if (t < RS_I && I < Cc.nx) {
        T sum = T(0);
        const int i1 = min(F.cx * I + F.cx, F.nx) - F.cx * I0, j1 = min(F.cy * J + F.cy, F.ny) - F.cy * J,
                  k1 = min(F.cz * K + F.cz, F.nz) - F.cz * K;
        for (int a = 0; a < k1; a++) for (int b = 0; b < j1; b++) for (int q = F.cx * t; q < i1; q++) sum += res[a][b][q];
        const int cc = sidx(Cc, K, J, I);
        Cc.r[cc] = sum;
        Cc.x[cc] = T(0);
    }
}

template <class T>
__global__ void k_prolong(Lvl<T> F, Lvl<T> Cc)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= F.nx || j >= F.ny || k >= F.nz) return;
    F.x[sidx(F, k, j, i)] += Cc.x[sidx(Cc, k / F.cz, j / F.cy, i / F.cx)];
}

// ------------------------------------------------------- coarsest level
// x = Bp r with Bp = (I - 11^T/n) (A + 11^T/n)^-1 (I - 11^T/n): the
// pseudo-inverse of the singular coarsest operator applied to the mean-free
// part of r, returned mean-free (the two projections are folded into Bp at
// set-up). One warp per row, FP64 accumulation; Bp is symmetric.
template <class T>
__global__ void __launch_bounds__(256) k_coarse_dense(const T *Bp, Lvl<T> L)
{
    const int n = (int)L.n, row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (row >= n) return;   // row is uniform over the warp
    const T *b = Bp + (size_t)row * n;
    double acc = 0.0;
    for (int u = lane; u < n; u += 32) acc += (double)b[u] * (double)L.r[u];
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) L.x[row] = (T)acc;
}

template <class T>
__global__ void k_in(const double *r, const double *d_sum, Lvl<T> L)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= L.nx || j >= L.ny || k >= L.nz) return;
    int q = (k * L.ny + j) * L.nx + i, c = sidx(L, k, j, i);
    double v = q == 0 ? -d_sum[0] : r[q];
    L.r[c] = (T)v;
    L.x[c] = T(0);
}
// z <- L0.x - L0.x[pinned] (natural order, FP64)
template <class T>
__global__ void k_out(Lvl<T> L, double *z)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= L.nx || j >= L.ny || k >= L.nz) return;
    int q = (k * L.ny + j) * L.nx + i, c = sidx(L, k, j, i);
    z[q] = (double)L.x[c] - (double)L.x[0];
}

inline dim3 g3(int a, int b, int c) { return grid3(a, b, c); }

template <class T>
void vcycle(tg_ctx *C, MG *mg, Lvl<T> *L, int l)
{
    cudaStream_t st = C->stream;
    if (l == mg->nlev - 1) {
        TG_PROF(C, "mg_coarse_dense", k_coarse_dense<T><<<(int)((L[l].n * 32 + 255) / 256), 256, 0, st>>>(mg_dense<T>(mg), L[l]));
        return;
    }
    Lvl<T> &F = L[l];
    const bool fine = l == 0;
    // zx: the level's unknown is still the zero written by k_in or the
    // restriction (the first sweep of the pre-smoothing), so the sweep skips
    // the off-line (off-point) neighbour terms, which are zero
    auto smooth = [&](int color, bool zx) {
        if (mg->line && !fine && F.n <= LINE_WARP_CELLS && (F.nx % 2) == 0 && line_warp_cj(F.ny) > 0) {
            TG_PROF(C, "mg_smooth_line_coarse", launch_line_warp<T>(F, color, zx, st));
        } else if (mg->line && (F.nx % 2) == 0 && line_cj<T>(F.ny) > 0) {
            TG_PROF(C, fine ? "mg_smooth_line_L0" : "mg_smooth_line_coarse", launch_line_chunked<T>(F, color, zx, st));
        } else if (mg->line) {
            int half = (F.nx + 1) >> 1;
            TG_PROF(C, fine ? "mg_smooth_line_L0" : "mg_smooth_line_coarse",
                    k_smooth_line<T><<<dim3((half + 31) / 32, (F.nz + 7) / 8), dim3(32, 8), 0, st>>>(F, color, zx ? 1 : 0));
        } else {
            TG_PROF(C, fine ? "mg_smooth_rb_L0" : "mg_smooth_rb_coarse",
                    k_smooth_rb<T><<<g3(F.nx, F.ny, F.nz), block3(), 0, st>>>(F, color, zx ? 1 : 0));
        }
    };
    for (int s = 0; s < mg->nu; s++) { smooth(0, s == 0); smooth(1, false); }
    Lvl<T> &Cc = L[l + 1];
    TG_PROF(C, fine ? "mg_restrict_L0" : "mg_restrict_coarse", k_restrict<T><<<dim3((Cc.nx + RS_I - 1) / RS_I, Cc.ny, Cc.nz), 8 * RS_I, 0, st>>>(F, Cc));
    vcycle(C, mg, L, l + 1);
    TG_PROF(C, fine ? "mg_prolong_L0" : "mg_prolong_coarse", k_prolong<T><<<g3(F.nx, F.ny, F.nz), block3(), 0, st>>>(F, Cc));
    for (int s = 0; s < mg->nu; s++) { smooth(1, false); smooth(0, false); }
}

// split-layout index on the host
inline int hsidx(int nx, int ny, int h0, int k, int j, int i) { return (k * ny + j) * nx + ((i & 1) ? (h0 + (i >> 1)) : (i >> 1)); }

// inverse of the symmetric positive definite n x n matrix A (row-major):
// Cholesky factor A = L L^T (lower, row-oriented), X = L^-1 by columns (kept
// transposed, Xt[c][q] = X(q, c), so every inner loop runs over contiguous
// memory), A^-1 = X^T X. About n^3 / 2 multiply-adds; false if A is not
// positive definite to working precision. A is overwritten.
bool spd_inverse(std::vector<double> &A, int n, std::vector<double> &inv)
{
    auto a = [&](int r, int c) -> double & { return A[(size_t)r * n + c]; };
    for (int i = 0; i < n; i++)
        for (int k = 0; k <= i; k++) {
            double v = a(i, k);
            const double *li = &a(i, 0), *lk = &a(k, 0);
            for (int q = 0; q < k; q++) v -= li[q] * lk[q];
            if (i == k) {
                if (!(v > 0.0)) return false;
                a(i, i) = std::sqrt(v);
            } else {
                a(i, k) = v / a(k, k);
            }
        }
    std::vector<double> Xt((size_t)n * n, 0.0);
    for (int c = 0; c < n; c++) {
        double *x = &Xt[(size_t)c * n];
        x[c] = 1.0 / a(c, c);
        for (int r = c + 1; r < n; r++) {
            const double *lr = &a(r, 0);
            double v = 0.0;
            for (int q = c; q < r; q++) v += lr[q] * x[q];
            x[r] = -v / lr[r];
        }
    }
    inv.assign((size_t)n * n, 0.0);
    for (int r = 0; r < n; r++)
        for (int c = r; c < n; c++) {
            const double *xr = &Xt[(size_t)r * n], *xc = &Xt[(size_t)c * n];
            double v = 0.0;
            for (int q = c; q < n; q++) v += xr[q] * xc[q];
            inv[(size_t)r * n + c] = v;
            inv[(size_t)c * n + r] = v;
        }
    return true;
}

template <class T>
void setup_levels(tg_ctx *C, MG *mg, Lvl<T> *L, const double *aE, const double *aN, const double *aT,
                  int nx, int ny, int nz, int pi, int pj, int pk)
{
    cudaStream_t st = C->stream;
    mg->nlev = 1;
    L[0] = Lvl<T>{};
    L[0].nx = nx; L[0].ny = ny; L[0].nz = nz; L[0].pi = pi; L[0].pj = pj; L[0].pk = pk;
    for (;;) {
        Lvl<T> &F = L[mg->nlev - 1];
        F.n = (int64_t)F.nx * F.ny * F.nz;
        F.h0 = (F.nx + 1) >> 1;
        auto can = [](int m) { return m >= 3; };
        F.cx = can(F.nx) ? 2 : 1; F.cy = can(F.ny) ? 2 : 1; F.cz = can(F.nz) ? 2 : 1;
        bool coarsen = F.n > COARSEST_CELLS && (F.cx * F.cy * F.cz) > 1 && mg->nlev < MAXL;
        if (!coarsen) { F.cx = F.cy = F.cz = 1; break; }
        Lvl<T> &Cn = L[mg->nlev++];
        Cn = Lvl<T>{};
        Cn.nx = (F.nx + F.cx - 1) / F.cx; Cn.ny = (F.ny + F.cy - 1) / F.cy; Cn.nz = (F.nz + F.cz - 1) / F.cz;
        Cn.pi = F.pi; Cn.pj = F.pj; Cn.pk = F.pk;
    }
    for (int l = 0; l < mg->nlev; l++) {
        Lvl<T> &V = L[l];
        T **arrs[] = {&V.aE, &V.aN, &V.aT, &V.diag, &V.cp, &V.minv, &V.x, &V.r, &V.tmp};
        for (T **a : arrs) *a = (T *)dalloc(C, sizeof(T) * (size_t)V.n);
    }
    k_l0_coeffs<T><<<g3(nx, ny, nz), block3(), 0, st>>>(aE, aN, aT, L[0]);
    for (int l = 0; l + 1 < mg->nlev; l++)
        k_coarsen<T><<<g3(L[l + 1].nx, L[l + 1].ny, L[l + 1].nz), block3(), 0, st>>>(L[l], L[l + 1]);
    for (int l = 0; l < mg->nlev; l++) {
        k_diag<T><<<g3(L[l].nx, L[l].ny, L[l].nz), block3(), 0, st>>>(L[l]);
        if (mg->line) k_line_factors<T><<<dim3((L[l].nx + 31) / 32, (L[l].nz + 7) / 8), dim3(32, 8), 0, st>>>(L[l]);
    }
    if (mg->line) set_line_smem_attrs<T>();
    // dense pseudo-inverse of the coarsest level in its own (split) order
    Lvl<T> &Lc = L[mg->nlev - 1];
    if (Lc.n > COARSEST_CELLS) throw CudaError{cudaErrorInvalidValue, "grid does not coarsen to <= 1024 cells"};
    const int nc = (int)Lc.n;
    std::vector<T> hE(nc), hN(nc), hT(nc);
    TG_CUDA(cudaMemcpyAsync(hE.data(), Lc.aE, sizeof(T) * nc, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaMemcpyAsync(hN.data(), Lc.aN, sizeof(T) * nc, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaMemcpyAsync(hT.data(), Lc.aT, sizeof(T) * nc, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    std::vector<double> A((size_t)nc * nc, 1.0 / nc);
    auto id = [&](int k, int j, int i) {
        i = (i + Lc.nx) % Lc.nx; j = (j + Lc.ny) % Lc.ny; k = (k + Lc.nz) % Lc.nz;
        return hsidx(Lc.nx, Lc.ny, Lc.h0, k, j, i);
    };
    for (int k = 0; k < Lc.nz; k++) for (int j = 0; j < Lc.ny; j++) for (int i = 0; i < Lc.nx; i++) {
        int c = id(k, j, i);
        auto add = [&](int nb, double a) { A[(size_t)c * nc + c] += a; A[(size_t)c * nc + nb] -= a; };
        if (i < Lc.nx - 1 || Lc.pi) add(id(k, j, i + 1), hE[c]);
        if (i > 0 || Lc.pi)         { int w = id(k, j, i - 1); add(w, hE[w]); }
        if (j < Lc.ny - 1 || Lc.pj) add(id(k, j + 1, i), hN[c]);
        if (j > 0 || Lc.pj)         { int s = id(k, j - 1, i); add(s, hN[s]); }
        if (k < Lc.nz - 1 || Lc.pk) add(id(k + 1, j, i), hT[c]);
        if (k > 0 || Lc.pk)         { int b = id(k - 1, j, i); add(b, hT[b]); }
    }
    std::vector<double> inv;
    if (!spd_inverse(A, nc, inv)) throw CudaError{cudaErrorInvalidValue, "singular coarsest multigrid operator"};
    // Bp = (I - J/n) inv (I - J/n): subtract row and column means, add the grand mean
    std::vector<double> rm(nc, 0.0);
    double gm = 0.0;
    for (int r = 0; r < nc; r++) {
        for (int c = 0; c < nc; c++) rm[r] += inv[(size_t)r * nc + c];
        rm[r] /= nc;
        gm += rm[r];
    }
    gm /= nc;
    std::vector<T> Bp((size_t)nc * nc);
    for (int r = 0; r < nc; r++)
        for (int c = 0; c < nc; c++) Bp[(size_t)r * nc + c] = (T)(inv[(size_t)r * nc + c] - rm[r] - rm[c] + gm);
    T *dB = (T *)dalloc(C, sizeof(T) * (size_t)nc * nc);
    if (sizeof(T) == sizeof(double)) mg->Bd = (double *)dB;
    else mg->Bf = (float *)dB;
    mg->nc = nc;
    TG_CUDA(cudaMemcpyAsync(dB, Bp.data(), sizeof(T) * (size_t)nc * nc, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaStreamSynchronize(st));
    TG_CUDA(cudaGetLastError());
}

}  // namespace

MG *mg_create(tg_ctx *C, bool fp32, const double *aE, const double *aN, const double *aT,
              int nx, int ny, int nz, int pi, int pj, int pk)
{
    MG *mg = new MG();
    mg->fp32 = fp32;
    mg->line = !pj && ny >= 2;
    mg->nu = 2;
    if (fp32) setup_levels<float>(C, mg, mg->Lf, aE, aN, aT, nx, ny, nz, pi, pj, pk);
    else setup_levels<double>(C, mg, mg->Ld, aE, aN, aT, nx, ny, nz, pi, pj, pk);
    return mg;
}

void mg_destroy(MG *mg) { delete mg; }

template <class T>
static void apply_t(tg_ctx *C, MG *mg, Lvl<T> *L, const double *r, const double *d_sum, double *z)
{
    cudaStream_t st = C->stream;
    TG_PROF(C, "mg_in", k_in<T><<<g3(L[0].nx, L[0].ny, L[0].nz), block3(), 0, st>>>(r, d_sum, L[0]));
    vcycle<T>(C, mg, L, 0);
    TG_PROF(C, "mg_out", k_out<T><<<g3(L[0].nx, L[0].ny, L[0].nz), block3(), 0, st>>>(L[0], z));
}

void mg_apply(tg_ctx *C, MG *mg, const double *r, const double *d_sum, double *z)
{
    if (mg->fp32) apply_t<float>(C, mg, mg->Lf, r, d_sum, z);
    else apply_t<double>(C, mg, mg->Ld, r, d_sum, z);
}

}  // namespace tg
