// Allocation-free divergence check: the same maximum as
// tg_continuity_error (max over interior cells of |div(Ucont)| * aj), on
// caller-owned device arrays, with its per-plane partial maxima kept in a
// file-scope device array instead of memory obtained from cudaMalloc.
//
// Callers that cannot allocate: code running while a CUDA stream is being
// captured into a graph (cudaMalloc is not allowed there), hosts whose device
// memory is owned by a fixed pool or a framework allocator that must stay the
// only allocator, and real-time loops that cannot absorb the implicit device
// synchronisation of cudaMalloc/cudaFree. This entry point calls neither.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "tg_internal.cuh"

namespace {

// one partial maximum per (interior k-plane, chunk of that plane); a call
// accepts at most this many interior k-planes
constexpr int TG_NOALLOC_MAX_PLANES = 16384;
constexpr int TG_NOALLOC_SLOTS = TG_NOALLOC_MAX_PLANES;
// cells of a plane per block before the plane is split over more blocks
constexpr int TG_NOALLOC_CHUNK_CELLS = 2048;

// Scratch of the entry point: every GPU that loads this library holds one copy
// (128 KiB) until the process exits. Every call shares it and it keeps the
// last call's contents; each call writes every entry it reads before reading
// it, so nothing has to start at zero. Calls that overlap on the same GPU
// (e.g. on two streams) race on it and must be serialised by the caller.
static __device__ __align__(256) double g_div_planes[TG_NOALLOC_SLOTS];

// device address of g_div_planes per device ordinal, found once per device
constexpr int TG_NOALLOC_MAX_DEVICES = 64;
double *g_plane_addr[TG_NOALLOC_MAX_DEVICES] = {nullptr};
std::mutex g_addr_mutex;

// maximum over a 256-thread block: warp shuffles, then one value per warp
__device__ __forceinline__ double block_nanmax(double m)
{
    __shared__ double warp_max[8];
    for (int o = 16; o > 0; o >>= 1) m = tg::nanmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? warp_max[threadIdx.x] : 0.0;
        for (int o = 4; o > 0; o >>= 1) m = tg::nanmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    return m;
}

// block (x, y) = (interior k-plane k = x + 1, chunk y of its cells); the
// plane's cells t = y, y + chunks, ... are strided over the chunks so that
// every chunk reads whole rows of consecutive i
__global__ void __launch_bounds__(256) k_div_planes_noalloc(const double *ucont, const double *aj, int mx, int my,
                                                            double *planes)
{
    const int k = blockIdx.x + 1;
    const int ni = mx - 2, n = (mx - 2) * (my - 2);
    const int chunks = gridDim.y;
    double m = 0.0;
    for (int t = blockIdx.y * blockDim.x + threadIdx.x; t < n; t += chunks * blockDim.x) {
        int i = t % ni + 1, j = t / ni + 1;
        int c = (k * my + j) * mx + i;
        int w = c - 1, s = c - mx, b = c - mx * my;
        double d = fabs((ucont[3 * c] - ucont[3 * w] + ucont[3 * c + 1] - ucont[3 * s + 1]
                        + ucont[3 * c + 2] - ucont[3 * b + 2]) * aj[c]);
        m = tg::nanmax(m, d);
    }
    m = block_nanmax(m);
    if (threadIdx.x == 0) planes[blockIdx.x * chunks + blockIdx.y] = m;
}

__global__ void __launch_bounds__(256) k_div_final_noalloc(const double *planes, int nslots, double *out)
{
    double m = 0.0;
    for (int t = threadIdx.x; t < nslots; t += blockDim.x) m = tg::nanmax(m, planes[t]);
    m = block_nanmax(m);
    if (threadIdx.x == 0) out[0] = m;
}

}  // namespace

extern "C" tg_status tg_continuity_error_noalloc(const double *ucont, const double *aj, int32_t mx, int32_t my,
                                                 int32_t mz, double *max_div, void *stream)
{
    if (!ucont || !aj || !max_div) return TG_ERR_BAD_ARG;
    if (mx < 3 || my < 3 || mz < 3) return TG_ERR_BAD_ARG;
    if (mz - 2 > TG_NOALLOC_MAX_PLANES) return TG_ERR_BAD_ARG;              // beyond the scratch array
    if ((int64_t)mx * my * mz * 3 > (int64_t)INT32_MAX) return TG_ERR_BAD_ARG;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return TG_ERR_CUDA;
    if (dev < 0 || dev >= TG_NOALLOC_MAX_DEVICES) return TG_ERR_BAD_ARG;
    double *planes = nullptr;
    {
        // set-up, once per device, with that device current: the host-side name
        // g_div_planes is not a device address, so look the address up
        std::lock_guard<std::mutex> lock(g_addr_mutex);
        if (!g_plane_addr[dev]) {
            double *p = nullptr;
            if (cudaGetSymbolAddress((void **)&p, g_div_planes) != cudaSuccess || !p) return TG_ERR_CUDA;
            g_plane_addr[dev] = p;
        }
        planes = g_plane_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int nplanes = mz - 2;
    // split large planes over several blocks while the slots last
    const int64_t plane_cells = (int64_t)(mx - 2) * (my - 2);
    int chunks = (int)std::min<int64_t>((plane_cells + TG_NOALLOC_CHUNK_CELLS - 1) / TG_NOALLOC_CHUNK_CELLS,
                                        TG_NOALLOC_SLOTS / nplanes);
    chunks = std::max(1, std::min(chunks, 65535));
    k_div_planes_noalloc<<<dim3(nplanes, chunks), 256, 0, st>>>(ucont, aj, mx, my, planes);
    k_div_final_noalloc<<<1, 256, 0, st>>>(planes, nplanes * chunks, max_div);
    return cudaGetLastError() == cudaSuccess ? TG_OK : TG_ERR_CUDA;
}
