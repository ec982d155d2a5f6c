// Uniform actuator-disk wind farm (TOSCA "uniformADM", sampleType rotorDisk,
// CtType constant) and its adjoint with respect to the turbines' C_T'.
//
// Geometry is fixed (no yaw or tilt motion), so everything that depends only
// on the mesh and the disks is built once on the host in tg_set_turbines:
//  * disk points and areas (turbines_io.c:1925-2000),
//  * projection cells: interior cells within r_tip + eps * sqrt(ln 1000) of
//    the rotor centre (turbines_parallel.c:40-135),
//  * per point the closest projection cell, searched from the point shifted by
//    1e-10 in x, y, z as on a single rank (turbines_parallel.c:772-840), and
//    the eight cells and clamped local coordinates of its trilinear
//    interpolation (inline.h:6904-7265),
//  * per (turbine, projection cell) the Gaussian weight
//    g = sum_p exp(-(r/eps)^2) / (eps^3 pi^1.5) dA_p over the points within
//    eps * sqrt(ln 1000) (turbines_force.c:858-910), computed on the device.
// Per step (main.c:146, before GradP): one block per turbine samples Ucat at
// its points, U = sum_p |u_p without its radial part| dA_p / sum dA
// (turbines_sampling.c:174-262), s = 0.5 U^2 C_T' (point force s dA_p along
// the axis, turbines_force.c:345-362), thrust = rho s (axis . axis) sum dA and
// power = thrust U; the projected Cartesian force sum_t s_t g_t axis_t is
// written at the covered cells, and its central face values dotted with the
// face areas (turbines_force.c:1741-1835) into State::farmcont, which the
// fused right-hand-side kernel adds after the buoyancy term
// (ueqn_solvers.c:1340-1344).
#include <algorithm>
#include <cmath>
#include <set>
#include <vector>

#include "tg_internal.cuh"

namespace tg {

struct Farm {
    int nt = 0, np = 0, ne = 0, nc = 0, nf = 0;
    double rho = 1.0;
    bool objective = false;
    std::vector<double> ct;               // host copy of C_T'
    std::vector<void *> mem;              // device allocations of the farm
    // points
    int *pt_off = nullptr;                // nt + 1
    int *pt_cells = nullptr;              // 8 per point: v000 v100 v010 v001 v110 v011 v101 v111
    double *pt_del = nullptr;             // 3 per point: clamped local coordinates (csi, eta, zet)
    double *pt_xb = nullptr, *pt_yb = nullptr;   // 3 per point: in-plane basis (xb = -axis, yb = zb x xb)
    double *pt_da = nullptr;              // area per point
    double *pt_xyz = nullptr;             // 3 per point
    // turbines
    double *t_ct = nullptr, *t_area = nullptr, *t_axd = nullptr, *t_axis = nullptr, *t_eps = nullptr;
    // projection entries (per turbine) and covered cells
    int *te_off = nullptr, *te_cell = nullptr, *te_t = nullptr, *te_cov = nullptr;
    double *te_g = nullptr;
    int *cov_cell = nullptr, *cov_off = nullptr, *cov_ent = nullptr;
    int *face_cell = nullptr;
    V3f<double> cat{};                    // projected Cartesian body force
    double *state = nullptr;              // per turbine U, s, thrust, power; [4 nt] = power sum
    // adjoint
    double *fsa = nullptr;                // 3 per covered cell: adjoint of the projected force
    double *astate = nullptr;             // per turbine U, U_bar (reversed step)
    double *ct_grad = nullptr;
};

namespace {

constexpr int FB = 256;

template <class T>
T *falloc(tg_ctx *C, Farm &F, size_t n)
{
    T *p = (T *)dalloc(C, n * sizeof(T));
    F.mem.push_back(p);
    return p;
}

template <class T>
void upload(tg_ctx *C, T *dst, const std::vector<T> &src)
{
    if (!src.empty()) TG_CUDA(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, C->stream));
}

// trilinear interpolation in TOSCA's form c0 + c1 dC + c2 dE + c3 dZ + c4 dC dE
// + c5 dE dZ + c6 dZ dC + c7 dC dE dZ (inline.h:7203-7263)
__device__ __forceinline__ double tri(const double *v, const double d[3], const int *cl)
{
    const double v000 = v[cl[0]], v100 = v[cl[1]], v010 = v[cl[2]], v001 = v[cl[3]];
    const double v110 = v[cl[4]], v011 = v[cl[5]], v101 = v[cl[6]], v111 = v[cl[7]];
    const double c0 = v000, c1 = v100 - v000, c2 = v010 - v000, c3 = v001 - v000;
    const double c4 = v110 - v010 - v100 + v000, c5 = v011 - v001 - v010 + v000, c6 = v101 - v001 - v100 + v000;
    const double c7 = v111 - v011 - v101 - v110 + v100 + v001 + v010 - v000;
    return c0 + c1 * d[0] + c2 * d[1] + c3 * d[2] + c4 * d[0] * d[1] + c5 * d[1] * d[2] + c6 * d[2] * d[0] +
           c7 * d[0] * d[1] * d[2];
}

// point velocity and its in-plane speed
__device__ __forceinline__ void point_speed(const Farm &F, V3f<double> u, int p, double &ubx, double &uby, double &m)
{
    const int *cl = F.pt_cells + 8 * p;
    const double d[3] = {F.pt_del[3 * p], F.pt_del[3 * p + 1], F.pt_del[3 * p + 2]};
    const double ux = tri(u.x, d, cl), uy = tri(u.y, d, cl), uz = tri(u.z, d, cl);
    const double *xb = F.pt_xb + 3 * p, *yb = F.pt_yb + 3 * p;
    ubx = ux * xb[0] + uy * xb[1] + uz * xb[2];
    uby = ux * yb[0] + uy * yb[1] + uz * yb[2];
    m = sqrt(ubx * ubx + uby * uby);
}

// one block per turbine: disk speed, force scale, thrust and power
__global__ void __launch_bounds__(FB) k_farm_sample(Farm F, V3f<double> u, double *out, int stride)
{
    const int t = blockIdx.x;
    double s = 0.0;
    for (int p = F.pt_off[t] + threadIdx.x; p < F.pt_off[t + 1]; p += blockDim.x) {
        double ubx, uby, m;
        point_speed(F, u, p, ubx, uby, m);
        s += m * F.pt_da[p];
    }
    s = block_sum_all<FB>(s);
    if (threadIdx.x == 0) {
        const double U = s / F.t_area[t];
        const double sc = 0.5 * U * U * F.t_ct[t];
        out[stride * t] = U;
        if (stride == 4) {
            const double thrust = F.rho * sc * F.t_axd[t] * F.t_area[t];
            out[4 * t + 1] = sc;
            out[4 * t + 2] = thrust;
            out[4 * t + 3] = thrust * U;
        }
    }
}

__global__ void k_farm_power_sum(Farm F)
{
    double s = 0.0;
    for (int t = 0; t < F.nt; t++) s += F.state[4 * t + 3];
    F.state[4 * F.nt] += s;
}

// projected Cartesian force at the covered cells
__global__ void k_farm_force(Farm F)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= F.nc) return;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int e = F.cov_off[q]; e < F.cov_off[q + 1]; e++) {
        const int en = F.cov_ent[e], t = F.te_t[en];
        const double w = F.state[4 * t + 1] * F.te_g[en];
        fx += w * F.t_axis[3 * t]; fy += w * F.t_axis[3 * t + 1]; fz += w * F.t_axis[3 * t + 2];
    }
    const int c = F.cov_cell[q];
    F.cat.x[c] = fx; F.cat.y[c] = fy; F.cat.z[c] = fz;
}

// bodyForceCartesian2Contravariant at the faces that read a covered cell
__global__ void k_farm_cont(Farm F, Grid g, Metrics m, V3f<double> fc)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= F.nf) return;
    const int c = F.face_cell[q], ie = c + 1, jn = c + g.mx, kt = c + g.mx * g.my;
    const V3f<double> s = F.cat;
    fc.x[c] = 0.5 * (s.x[c] + s.x[ie]) * m.icsi.x[c] + 0.5 * (s.y[c] + s.y[ie]) * m.icsi.y[c] + 0.5 * (s.z[c] + s.z[ie]) * m.icsi.z[c];
    fc.y[c] = 0.5 * (s.x[c] + s.x[jn]) * m.jeta.x[c] + 0.5 * (s.y[c] + s.y[jn]) * m.jeta.y[c] + 0.5 * (s.z[c] + s.z[jn]) * m.jeta.z[c];
    fc.z[c] = 0.5 * (s.x[c] + s.x[kt]) * m.kzet.x[c] + 0.5 * (s.y[c] + s.y[kt]) * m.kzet.y[c] + 0.5 * (s.z[c] + s.z[kt]) * m.kzet.z[c];
}

// Gaussian projection weight of every (turbine, covered cell) entry
__global__ void k_farm_weights(Farm F, V3f<double> cent)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= F.ne) return;
    const int t = F.te_t[e], c = F.te_cell[e];
    const double eps = F.t_eps[t], rprj = eps * sqrt(log(1.0 / 0.001));
    const double cx = cent.x[c], cy = cent.y[c], cz = cent.z[c];
    double g = 0.0;
    for (int p = F.pt_off[t]; p < F.pt_off[t + 1]; p++) {
        const double dx = F.pt_xyz[3 * p] - cx, dy = F.pt_xyz[3 * p + 1] - cy, dz = F.pt_xyz[3 * p + 2] - cz;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        if (r < rprj) g += exp(-(r / eps) * (r / eps)) / (pow(eps, 3.0) * pow(M_PI, 1.5)) * F.pt_da[p];
    }
    F.te_g[e] = g;
}

// ---------------------------------------------------------------- adjoint
// adjoint of the projected force at the covered cells from one stage's Rhs
// adjoint: the transpose of the central face values (faces of interior
// cells: the cell's own faces and the +faces of its -i/-j/-k neighbours)
__global__ void k_farm_adj_stage(Farm F, Grid g, Metrics m, V3f<double> ra)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= F.nc) return;
    const int c = F.cov_cell[q], pl = g.mx * g.my;
    const int k = c / pl, j = (c - k * pl) / g.mx, i = c - k * pl - j * g.mx;
    double ax = 0.5 * ra.x[c] * m.icsi.x[c] + 0.5 * ra.y[c] * m.jeta.x[c] + 0.5 * ra.z[c] * m.kzet.x[c];
    double ay = 0.5 * ra.x[c] * m.icsi.y[c] + 0.5 * ra.y[c] * m.jeta.y[c] + 0.5 * ra.z[c] * m.kzet.y[c];
    double az = 0.5 * ra.x[c] * m.icsi.z[c] + 0.5 * ra.y[c] * m.jeta.z[c] + 0.5 * ra.z[c] * m.kzet.z[c];
    if (i > 1) { const int w = c - 1; ax += 0.5 * ra.x[w] * m.icsi.x[w]; ay += 0.5 * ra.x[w] * m.icsi.y[w]; az += 0.5 * ra.x[w] * m.icsi.z[w]; }
    if (j > 1) { const int s = c - g.mx; ax += 0.5 * ra.y[s] * m.jeta.x[s]; ay += 0.5 * ra.y[s] * m.jeta.y[s]; az += 0.5 * ra.y[s] * m.jeta.z[s]; }
    if (k > 1) { const int b = c - pl; ax += 0.5 * ra.z[b] * m.kzet.x[b]; ay += 0.5 * ra.z[b] * m.kzet.y[b]; az += 0.5 * ra.z[b] * m.kzet.z[b]; }
    F.fsa[3 * q] += ax; F.fsa[3 * q + 1] += ay; F.fsa[3 * q + 2] += az;
}

// one block per turbine: D = sum_e g_e axis . fsa, then the C_T' gradient and
// the adjoint of the disk speed (with the power objective, + dP/dC_T', dP/dU)
__global__ void __launch_bounds__(FB) k_farm_adj_turbine(Farm F, int objective)
{
    const int t = blockIdx.x;
    const double ax = F.t_axis[3 * t], ay = F.t_axis[3 * t + 1], az = F.t_axis[3 * t + 2];
    double d = 0.0;
    for (int e = F.te_off[t] + threadIdx.x; e < F.te_off[t + 1]; e += blockDim.x) {
        const int q = F.te_cov[e];
        d += F.te_g[e] * (ax * F.fsa[3 * q] + ay * F.fsa[3 * q + 1] + az * F.fsa[3 * q + 2]);
    }
    d = block_sum_all<FB>(d);
    if (threadIdx.x == 0) {
        const double U = F.astate[2 * t], ct = F.t_ct[t];
        double gct = 0.5 * U * U * d, ub = ct * U * d;
        if (objective) {
            const double k = F.rho * F.t_axd[t] * F.t_area[t];
            gct += k * 0.5 * U * U * U;
            ub += k * 1.5 * ct * U * U;
        }
        F.ct_grad[t] += gct;
        F.astate[2 * t + 1] = ub;
    }
}

// adjoint of the sampling: Ucat_adj of the eight interpolation cells of every
// point += U_bar dA_p / A (u_perp / |u_perp|) w_q
__global__ void __launch_bounds__(FB) k_farm_adj_sample(Farm F, V3f<double> u, V3f<double> ca)
{
    const int t = blockIdx.x;
    const double ub = F.astate[2 * t + 1], area = F.t_area[t];
    for (int p = F.pt_off[t] + threadIdx.x; p < F.pt_off[t + 1]; p += blockDim.x) {
        double ubx, uby, m;
        point_speed(F, u, p, ubx, uby, m);
        if (!(m > 0.0)) continue;
        const double coef = ub * F.pt_da[p] / area / m;
        const double *xb = F.pt_xb + 3 * p, *yb = F.pt_yb + 3 * p;
        const double gx = coef * (ubx * xb[0] + uby * yb[0]);
        const double gy = coef * (ubx * xb[1] + uby * yb[1]);
        const double gz = coef * (ubx * xb[2] + uby * yb[2]);
        const double dC = F.pt_del[3 * p], dE = F.pt_del[3 * p + 1], dZ = F.pt_del[3 * p + 2];
        const double w[8] = {(1 - dC) * (1 - dE) * (1 - dZ), dC * (1 - dE) * (1 - dZ), (1 - dC) * dE * (1 - dZ),
                             (1 - dC) * (1 - dE) * dZ, dC * dE * (1 - dZ), (1 - dC) * dE * dZ, dC * (1 - dE) * dZ, dC * dE * dZ};
        const int *cl = F.pt_cells + 8 * p;
        for (int q = 0; q < 8; q++) {
            atomicAdd(ca.x + cl[q], w[q] * gx);
            atomicAdd(ca.y + cl[q], w[q] * gy);
            atomicAdd(ca.z + cl[q], w[q] * gz);
        }
    }
}

inline int nb(int n) { return std::max(1, (n + FB - 1) / FB); }

struct H3 { double x, y, z; };
inline H3 operator-(H3 a, H3 b) { return H3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline H3 operator+(H3 a, H3 b) { return H3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline H3 operator*(double s, H3 a) { return H3{s * a.x, s * a.y, s * a.z}; }
inline double dot(H3 a, H3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double mag(H3 a) { return std::sqrt(dot(a, a)); }
// nUnit (inline.h:870-889): v / (|v| + 1e-12)
inline H3 unit(H3 a) { double m = mag(a) + 1e-12; return H3{a.x / m, a.y / m, a.z / m}; }
inline H3 cross(H3 a, H3 b) { return H3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
// rotation of v about axis by theta, right hand (mRot, inline.h:1048-1094)
inline H3 rotate(H3 axis, H3 v, double th)
{
    const double am = mag(axis);
    H3 a{axis.x / am, axis.y / am, axis.z / am};
    const double c = std::cos(th), s = std::sin(th);
    H3 r{0, 0, 0};
    r.x += (c + (1 - c) * a.x * a.x) * v.x; r.x += ((1 - c) * a.x * a.y - a.z * s) * v.y; r.x += ((1 - c) * a.x * a.z + a.y * s) * v.z;
    r.y += ((1 - c) * a.x * a.y + a.z * s) * v.x; r.y += (c + (1 - c) * a.y * a.y) * v.y; r.y += ((1 - c) * a.y * a.z - a.x * s) * v.z;
    r.z += ((1 - c) * a.x * a.z - a.y * s) * v.x; r.z += ((1 - c) * a.y * a.z + a.x * s) * v.y; r.z += (c + (1 - c) * a.z * a.z) * v.z;
    return r;
}

void free_farm(tg_ctx *C, Farm *F)
{
    if (!F) return;
    TG_CUDA(cudaStreamSynchronize(C->stream));
    for (void *p : F->mem) {
        auto it = std::find(C->allocs.begin(), C->allocs.end(), p);
        if (it != C->allocs.end()) C->allocs.erase(it);
        cudaFree(p);
    }
    delete F;
}

}  // namespace

void farm_destroy(tg_ctx *C)
{
    Farm *F = C->farm;
    C->farm = nullptr;
    C->prm.farm = 0;
    free_farm(C, F);
}

bool farm_field(tg_ctx *C, int w, V3f<double> &out)
{
    if (!C->farm) return false;
    out = w == TG_F_FARM_FORCE ? C->farm->cat : C->s.farmcont;
    return true;
}

void farm_update(tg_ctx *C)
{
    Farm &F = *C->farm;
    TG_PROF(C, "farm_sample", k_farm_sample<<<F.nt, FB, 0, C->stream>>>(F, C->s.ucat, F.state, 4));
    k_farm_power_sum<<<1, 1, 0, C->stream>>>(F);
    TG_PROF(C, "farm_force", k_farm_force<<<nb(F.nc), FB, 0, C->stream>>>(F));
    TG_PROF(C, "farm_cont", k_farm_cont<<<nb(F.nf), FB, 0, C->stream>>>(F, C->g, C->m, C->s.farmcont));
}

void farm_adj_begin(tg_ctx *C)
{
    Farm &F = *C->farm;
    TG_CUDA(cudaMemsetAsync(F.fsa, 0, sizeof(double) * 3 * (size_t)F.nc, C->stream));
}

void farm_adj_stage(tg_ctx *C, V3f<double> ra)
{
    Farm &F = *C->farm;
    TG_PROF(C, "adj_farm", k_farm_adj_stage<<<nb(F.nc), FB, 0, C->stream>>>(F, C->g, C->m, ra));
}

void farm_adj_finish(tg_ctx *C, V3f<double> ucat_n, V3f<double> ca)
{
    Farm &F = *C->farm;
    k_farm_sample<<<F.nt, FB, 0, C->stream>>>(F, ucat_n, F.astate, 2);
    k_farm_adj_turbine<<<F.nt, FB, 0, C->stream>>>(F, F.objective ? 1 : 0);
    TG_PROF(C, "adj_farm", k_farm_adj_sample<<<F.nt, FB, 0, C->stream>>>(F, ucat_n, ca));
}

}  // namespace tg

using namespace tg;

namespace {

template <class F>
tg_status farm_guard(tg_ctx *C, F &&f)
{
    if (!C) return TG_ERR_BAD_ARG;
    try {
        cudaError_t e = cudaSetDevice(C->cfg.device);
        if (e != cudaSuccess) { C->err = std::string("cudaSetDevice: ") + cudaGetErrorString(e); return TG_ERR_CUDA; }
        tg_status s = f();
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) { C->err = std::string("kernel launch: ") + cudaGetErrorString(le); return TG_ERR_CUDA; }
        return s;
    } catch (const CudaError &e) {
        C->err = std::string(e.what) + ": " + cudaGetErrorString(e.e);
        return e.e == cudaErrorMemoryAllocation ? TG_ERR_ALLOC : TG_ERR_CUDA;
    } catch (const std::bad_alloc &) {
        C->err = "host allocation failed";
        return TG_ERR_ALLOC;
    }
}

tg_status bad(tg_ctx *C, tg_status s, const char *m)
{
    C->err = m;
    return s;
}

}  // namespace

extern "C" {

tg_status tg_set_turbines(tg_ctx *C, int32_t n, const tg_turbine *tb, double rho)
{
    return farm_guard(C, [&]() -> tg_status {
        if (!C->has_mesh) return bad(C, TG_ERR_STATE, "mesh not set");
        if (n < 0 || (n > 0 && !tb) || !(rho > 0)) return bad(C, TG_ERR_BAD_ARG, "bad turbine arguments");
        for (int t = 0; t < n; t++) {
            const tg_turbine &d = tb[t];
            H3 ax{d.axis[0], d.axis[1], d.axis[2]}, up{d.up[0], d.up[1], d.up[2]};
            if (d.n_radial < 2 || d.n_azimuth < 1 || !(d.r_tip > d.r_hub) || !(d.r_hub > 0) || !(d.epsilon > 0) ||
                !(mag(ax) > 0) || !(mag(up) > 0) || !(mag(cross(ax, up)) > 1e-12 * mag(ax) * mag(up)))
                return bad(C, TG_ERR_BAD_ARG, "bad turbine description");
        }
        graph_destroy(C);                 // captured steps refer to the old farm
        farm_destroy(C);
        if (n == 0) return TG_OK;
        const Grid g = C->g;
        const size_t G = (size_t)g.size();
        std::vector<double> cx(G), cy(G), cz(G);
        TG_CUDA(cudaMemcpy(cx.data(), C->m.cent.x, G * sizeof(double), cudaMemcpyDeviceToHost));
        TG_CUDA(cudaMemcpy(cy.data(), C->m.cent.y, G * sizeof(double), cudaMemcpyDeviceToHost));
        TG_CUDA(cudaMemcpy(cz.data(), C->m.cent.z, G * sizeof(double), cudaMemcpyDeviceToHost));
        auto cent = [&](int k, int j, int i) { size_t q = g.lin(k, j, i); return H3{cx[q], cy[q], cz[q]}; };

        Farm *F = new Farm();
        F->nt = n;
        F->rho = rho;
        const double nsig = std::sqrt(std::log(1.0 / 0.001));
        std::vector<int> pt_off{0}, pt_cells, te_off{0}, te_cell, te_t;
        std::vector<double> pt_del, pt_xb, pt_yb, pt_da, pt_xyz, t_ct, t_area, t_axd, t_axis, t_eps;
        for (int t = 0; t < n; t++) {
            const tg_turbine &d = tb[t];
            const H3 ctr{d.center[0], d.center[1], d.center[2]};
            const H3 axis = unit(H3{d.axis[0], d.axis[1], d.axis[2]});
            const H3 rh = unit(H3{d.up[0], d.up[1], d.up[2]});
            // disk points (turbines_io.c:1925-2000, no uptilt or precone)
            const double drval = (d.r_tip - d.r_hub) / (d.n_radial - 1), daval = 2 * M_PI / d.n_azimuth;
            const double hCoeff = (M_PI * d.r_hub * d.r_hub) / (M_PI * (d.r_tip * d.r_tip - d.r_hub * d.r_hub));
            std::vector<H3> pts;
            std::vector<double> da;
            double r = d.r_hub, area = 0.0;
            for (int ri = 0; ri < d.n_radial; ri++) {
                const double dr = (ri == 0 || ri == d.n_radial - 1) ? drval / 2 : drval;
                const double crown = M_PI * ((r + dr) * (r + dr) - r * r);
                const H3 rvec = (drval * ri) * rh + d.r_hub * rh;
                for (int ai = 0; ai < d.n_azimuth; ai++) {
                    da.push_back((1.0 + hCoeff) * crown / d.n_azimuth);
                    area += da.back();
                    pts.push_back(rotate(axis, rvec, daval * ai) + ctr);
                }
                r += dr;
            }
            // projection (controlled) cells
            const double radius = d.r_tip + d.epsilon * nsig;
            std::vector<int> sphere;
            for (int k = 1; k < g.mz - 1; k++)
            for (int j = 1; j < g.my - 1; j++)
            for (int i = 1; i < g.mx - 1; i++)
                if (mag(cent(k, j, i) - ctr) <= radius) sphere.push_back(g.lin(k, j, i));
            if (sphere.empty()) { delete F; return bad(C, TG_ERR_BAD_ARG, "a turbine has no cells within its projection radius"); }
            // closest cell and trilinear stencil per point
            for (size_t p = 0; p < pts.size(); p++) {
                const H3 pp = pts[p] + H3{1e-10, 1e-10, 1e-10};
                double best = 1e20;
                int bc = -1;
                for (int q : sphere) {
                    const double dm = mag(pp - H3{cx[q], cy[q], cz[q]});
                    if (dm < best) { best = dm; bc = q; }
                }
                const int pl = g.mx * g.my, kc = bc / pl, jc = (bc - kc * pl) / g.mx, ic = bc - kc * pl - jc * g.mx;
                const H3 P = pts[p];
                auto pick = [&](int c, int m, H3 right, H3 left, int &L, int &R) {
                    if (c > 1 && c < m - 2) {
                        const H3 dr = right - P, dl = P - left;
                        if (dot(dr, dr) <= dot(dl, dl)) { L = c; R = c + 1; } else { L = c - 1; R = c; }
                    } else if (c == 1) { L = c; R = c + 1; }
                    else { L = c - 1; R = c; }
                };
                int iL, iR, jL, jR, kL, kR;
                pick(ic, g.mx, ic + 1 < g.mx ? cent(kc, jc, ic + 1) : P, ic > 0 ? cent(kc, jc, ic - 1) : P, iL, iR);
                pick(jc, g.my, jc + 1 < g.my ? cent(kc, jc + 1, ic) : P, jc > 0 ? cent(kc, jc - 1, ic) : P, jL, jR);
                pick(kc, g.mz, kc + 1 < g.mz ? cent(kc + 1, jc, ic) : P, kc > 0 ? cent(kc - 1, jc, ic) : P, kL, kR);
                const H3 c000 = cent(kL, jL, iL);
                const H3 ch = cent(kL, jL, iR) - c000, eh = cent(kL, jR, iL) - c000, zh = cent(kR, jL, iL) - c000;
                const double cn = mag(ch), en = mag(eh), zn = mag(zh);
                auto clamp01 = [](double v) { return std::max(std::min(v, 1.0), 0.0); };
                const H3 rel = P - c000;
                pt_del.push_back(clamp01(dot((1.0 / cn) * ch, rel) / cn));
                pt_del.push_back(clamp01(dot((1.0 / en) * eh, rel) / en));
                pt_del.push_back(clamp01(dot((1.0 / zn) * zh, rel) / zn));
                const int cells[8] = {g.lin(kL, jL, iL), g.lin(kL, jL, iR), g.lin(kL, jR, iL), g.lin(kR, jL, iL),
                                      g.lin(kL, jR, iR), g.lin(kR, jR, iL), g.lin(kR, jL, iR), g.lin(kR, jR, iR)};
                pt_cells.insert(pt_cells.end(), cells, cells + 8);
                // in-plane basis (turbines_sampling.c:230-250): xb = -axis, yb = zb x xb
                const H3 zb = unit(P - ctr), xb = -1.0 * axis, yb = cross(zb, xb);
                pt_xb.insert(pt_xb.end(), {xb.x, xb.y, xb.z});
                pt_yb.insert(pt_yb.end(), {yb.x, yb.y, yb.z});
                pt_da.push_back(da[p]);
                pt_xyz.insert(pt_xyz.end(), {P.x, P.y, P.z});
            }
            pt_off.push_back((int)pt_da.size());
            for (int q : sphere) { te_cell.push_back(q); te_t.push_back(t); }
            te_off.push_back((int)te_cell.size());
            t_ct.push_back(d.ct);
            t_area.push_back(area);
            t_axd.push_back(dot(axis, axis));
            t_axis.insert(t_axis.end(), {axis.x, axis.y, axis.z});
            t_eps.push_back(d.epsilon);
        }
        // covered cells (deterministic per-cell entry order: by turbine)
        std::vector<int> order(te_cell.size());
        for (size_t e = 0; e < order.size(); e++) order[e] = (int)e;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return te_cell[a] < te_cell[b]; });
        std::vector<int> cov_cell, cov_off{0}, cov_ent, te_cov(te_cell.size());
        for (size_t o = 0; o < order.size(); o++) {
            const int e = order[o];
            if (cov_cell.empty() || cov_cell.back() != te_cell[e]) {
                if (!cov_cell.empty()) cov_off.push_back((int)cov_ent.size());
                cov_cell.push_back(te_cell[e]);
            }
            te_cov[e] = (int)cov_cell.size() - 1;
            cov_ent.push_back(e);
        }
        cov_off.push_back((int)cov_ent.size());
        // faces that read a covered cell (faces of interior cells only)
        std::set<int> faces;
        const int pl = g.mx * g.my;
        for (int c : cov_cell) {
            const int k = c / pl, j = (c - k * pl) / g.mx, i = c - k * pl - j * g.mx;
            faces.insert(c);
            if (i > 1) faces.insert(c - 1);
            if (j > 1) faces.insert(c - g.mx);
            if (k > 1) faces.insert(c - pl);
        }
        std::vector<int> face_cell(faces.begin(), faces.end());

        F->np = (int)pt_da.size(); F->ne = (int)te_cell.size(); F->nc = (int)cov_cell.size(); F->nf = (int)face_cell.size();
        F->ct = t_ct;
        C->farm = F;
        F->pt_off = falloc<int>(C, *F, pt_off.size()); upload(C, F->pt_off, pt_off);
        F->pt_cells = falloc<int>(C, *F, pt_cells.size()); upload(C, F->pt_cells, pt_cells);
        F->pt_del = falloc<double>(C, *F, pt_del.size()); upload(C, F->pt_del, pt_del);
        F->pt_xb = falloc<double>(C, *F, pt_xb.size()); upload(C, F->pt_xb, pt_xb);
        F->pt_yb = falloc<double>(C, *F, pt_yb.size()); upload(C, F->pt_yb, pt_yb);
        F->pt_da = falloc<double>(C, *F, pt_da.size()); upload(C, F->pt_da, pt_da);
        F->pt_xyz = falloc<double>(C, *F, pt_xyz.size()); upload(C, F->pt_xyz, pt_xyz);
        F->t_ct = falloc<double>(C, *F, n); upload(C, F->t_ct, t_ct);
        F->t_area = falloc<double>(C, *F, n); upload(C, F->t_area, t_area);
        F->t_axd = falloc<double>(C, *F, n); upload(C, F->t_axd, t_axd);
        F->t_axis = falloc<double>(C, *F, 3 * (size_t)n); upload(C, F->t_axis, t_axis);
        F->t_eps = falloc<double>(C, *F, n); upload(C, F->t_eps, t_eps);
        F->te_off = falloc<int>(C, *F, te_off.size()); upload(C, F->te_off, te_off);
        F->te_cell = falloc<int>(C, *F, te_cell.size()); upload(C, F->te_cell, te_cell);
        F->te_t = falloc<int>(C, *F, te_t.size()); upload(C, F->te_t, te_t);
        F->te_cov = falloc<int>(C, *F, te_cov.size()); upload(C, F->te_cov, te_cov);
        F->te_g = falloc<double>(C, *F, te_cell.size());
        F->cov_cell = falloc<int>(C, *F, cov_cell.size()); upload(C, F->cov_cell, cov_cell);
        F->cov_off = falloc<int>(C, *F, cov_off.size()); upload(C, F->cov_off, cov_off);
        F->cov_ent = falloc<int>(C, *F, cov_ent.size()); upload(C, F->cov_ent, cov_ent);
        F->face_cell = falloc<int>(C, *F, face_cell.size()); upload(C, F->face_cell, face_cell);
        double *cat = falloc<double>(C, *F, 3 * G);
        F->cat = V3f<double>{cat, cat + G, cat + 2 * G};
        F->state = falloc<double>(C, *F, 4 * (size_t)n + 1);
        F->fsa = falloc<double>(C, *F, 3 * (size_t)F->nc);
        F->astate = falloc<double>(C, *F, 2 * (size_t)n);
        F->ct_grad = falloc<double>(C, *F, n);
        if (!C->s.farmcont.x) C->s.farmcont = dalloc3(C, G);
        else TG_CUDA(cudaMemsetAsync(C->s.farmcont.x, 0, 3 * G * sizeof(double), C->stream));
        k_farm_weights<<<nb(F->ne), FB, 0, C->stream>>>(*F, C->m.cent);
        TG_CUDA(cudaGetLastError());
        TG_CUDA(cudaStreamSynchronize(C->stream));
        C->prm.farm = 1;
        return TG_OK;
    });
}

tg_status tg_set_turbine_ct(tg_ctx *C, const double *ct)
{
    return farm_guard(C, [&]() -> tg_status {
        if (!C->farm) return bad(C, TG_ERR_STATE, "no turbines");
        if (!ct) return bad(C, TG_ERR_BAD_ARG, "null C_T'");
        Farm &F = *C->farm;
        F.ct.assign(ct, ct + F.nt);
        TG_CUDA(cudaMemcpy(F.t_ct, ct, sizeof(double) * F.nt, cudaMemcpyHostToDevice));
        return TG_OK;
    });
}

tg_status tg_turbine_state(tg_ctx *C, double *uref, double *thrust, double *power, double *power_sum, int32_t reset)
{
    return farm_guard(C, [&]() -> tg_status {
        if (!C->farm) return bad(C, TG_ERR_STATE, "no turbines");
        Farm &F = *C->farm;
        std::vector<double> h(4 * (size_t)F.nt + 1);
        TG_CUDA(cudaStreamSynchronize(C->stream));
        TG_CUDA(cudaMemcpy(h.data(), F.state, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int t = 0; t < F.nt; t++) {
            if (uref) uref[t] = h[4 * t];
            if (thrust) thrust[t] = h[4 * t + 2];
            if (power) power[t] = h[4 * t + 3];
        }
        if (power_sum) *power_sum = h[4 * F.nt];
        if (reset) TG_CUDA(cudaMemset(F.state + 4 * F.nt, 0, sizeof(double)));
        return TG_OK;
    });
}

tg_status tg_set_farm_objective(tg_ctx *C, int32_t on)
{
    return farm_guard(C, [&]() -> tg_status {
        if (!C->farm) return bad(C, TG_ERR_STATE, "no turbines");
        if (C->farm->objective != (on != 0)) adj_graph_destroy(C);   // the flag is a kernel argument
        C->farm->objective = on != 0;
        return TG_OK;
    });
}

tg_status tg_ct_gradient(tg_ctx *C, double *grad, int32_t reset)
{
    return farm_guard(C, [&]() -> tg_status {
        if (!C->farm) return bad(C, TG_ERR_STATE, "no turbines");
        Farm &F = *C->farm;
        TG_CUDA(cudaStreamSynchronize(C->stream));
        if (grad) TG_CUDA(cudaMemcpy(grad, F.ct_grad, sizeof(double) * F.nt, cudaMemcpyDeviceToHost));
        if (reset) TG_CUDA(cudaMemset(F.ct_grad, 0, sizeof(double) * F.nt));
        return TG_OK;
    });
}

}  // extern "C"
