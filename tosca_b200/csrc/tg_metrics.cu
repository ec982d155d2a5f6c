// Mesh metrics on the device: restatement of SetMeshMetrics (mesh.c:630-1976)
// and of the metric tensor built by SetCoeffMatrix (peqn.c:791-849).
// Setup-only kernels: one thread per DMDA point, SoA output planes.
#include "tg_internal.cuh"

namespace tg {
namespace {

struct Nodes {
    const double *c;   // AoS xyz nodes, global extent
    Grid g;
    __device__ __forceinline__ R3<double> operator()(int k, int j, int i) const {
        int q = g.id(k, j, i) * 3;
        return R3<double>{c[q], c[q + 1], c[q + 2]};
    }
};

__device__ __forceinline__ void face_basis(double dxdc, double dydc, double dzdc, double dxde, double dyde, double dzde,
                                           double dxdz, double dydz, double dzdz,
                                           R3<double> &fc, R3<double> &fe, R3<double> &fz, double &faj)
{
    fc = R3<double>{dyde * dzdz - dzde * dydz, -dxde * dzdz + dzde * dxdz, dxde * dydz - dyde * dxdz};
    fe = R3<double>{dydz * dzdc - dzdz * dydc, -dxdz * dzdc + dzdz * dxdc, dxdz * dydc - dydz * dxdc};
    fz = R3<double>{dydc * dzde - dzdc * dyde, -dxdc * dzde + dzdc * dxde, dxdc * dyde - dydc * dxde};
    faj = dxdc * (dyde * dzdz - dzde * dydz) - dydc * (dxde * dzdz - dzde * dxdz) + dzdc * (dxde * dydz - dyde * dxdz);
    faj = 1. / faj;
}

// cell centres (mesh.c:713-743), face-centred dummy bases (mesh.c:773-945) and
// the cell Jacobian (mesh.c:1013-1098)
__global__ void k_cell_pass1(Nodes X, Metrics m, V3f<double> csit, V3f<double> etat, V3f<double> zett)
{
    const Grid g = X.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    int q = g.lin(k, j, i);
    bool ii = i >= 1 && i <= g.mx - 2, jj = j >= 1 && j <= g.my - 2, kk = k >= 1 && k <= g.mz - 2;
    if (ii && jj && kk) {
        R3<double> s = X(k, j, i) + X(k, j - 1, i) + X(k - 1, j, i) + X(k - 1, j - 1, i)
                     + X(k, j, i - 1) + X(k, j - 1, i - 1) + X(k - 1, j, i - 1) + X(k - 1, j - 1, i - 1);
        st3(m.cent, q, 0.125 * s);
        auto P = [&](int dk, int dj, int di) { return X(k - dk, j - dj, i - di); };
        R3<double> a = P(0,0,0), b = P(0,1,0), c = P(1,0,0), d = P(1,1,0), e = P(0,0,1), f = P(0,1,1), h = P(1,0,1), l = P(1,1,1);
        double dxdc = 0.25 * (a.x + b.x + c.x + d.x - e.x - f.x - h.x - l.x);
        double dydc = 0.25 * (a.y + b.y + c.y + d.y - e.y - f.y - h.y - l.y);
        double dzdc = 0.25 * (a.z + b.z + c.z + d.z - e.z - f.z - h.z - l.z);
        double dxde = 0.25 * (a.x + e.x + c.x + h.x - b.x - f.x - d.x - l.x);
        double dyde = 0.25 * (a.y + e.y + c.y + h.y - b.y - f.y - d.y - l.y);
        double dzde = 0.25 * (a.z + e.z + c.z + h.z - b.z - f.z - d.z - l.z);
        double dxdz = 0.25 * (a.x + b.x + e.x + f.x - c.x - d.x - h.x - l.x);
        double dydz = 0.25 * (a.y + b.y + e.y + f.y - c.y - d.y - h.y - l.y);
        double dzdz = 0.25 * (a.z + b.z + e.z + f.z - c.z - d.z - h.z - l.z);
        double det = dxdc * (dyde * dzdz - dzde * dydz) - dydc * (dxde * dzdz - dzde * dxdz) + dzdc * (dxde * dydz - dyde * dxdz);
        m.aj[q] = 1. / det;
    }
    if (kk && jj && i <= g.mx - 2) {
        R3<double> A = X(k, j, i), B = X(k - 1, j, i), Cc = X(k, j - 1, i), D = X(k - 1, j - 1, i);
        double dxde = 0.5 * (A.x + B.x - Cc.x - D.x), dyde = 0.5 * (A.y + B.y - Cc.y - D.y), dzde = 0.5 * (A.z + B.z - Cc.z - D.z);
        double dxdz = 0.5 * (Cc.x + A.x - D.x - B.x), dydz = 0.5 * (Cc.y + A.y - D.y - B.y), dzdz = 0.5 * (Cc.z + A.z - D.z - B.z);
        st3(csit, q, R3<double>{dyde * dzdz - dzde * dydz, -dxde * dzdz + dzde * dxdz, dxde * dydz - dyde * dxdz});
    }
    if (kk && ii && j <= g.my - 2) {
        R3<double> A = X(k, j, i), B = X(k - 1, j, i), Cc = X(k, j, i - 1), D = X(k - 1, j, i - 1);
        double dxdc = 0.5 * (A.x + B.x - Cc.x - D.x), dydc = 0.5 * (A.y + B.y - Cc.y - D.y), dzdc = 0.5 * (A.z + B.z - Cc.z - D.z);
        double dxdz = 0.5 * (A.x + Cc.x - B.x - D.x), dydz = 0.5 * (A.y + Cc.y - B.y - D.y), dzdz = 0.5 * (A.z + Cc.z - B.z - D.z);
        st3(etat, q, R3<double>{dydz * dzdc - dzdz * dydc, -dxdz * dzdc + dzdz * dxdc, dxdz * dydc - dydz * dxdc});
    }
    if (jj && ii && k <= g.mz - 2) {
        R3<double> A = X(k, j, i), B = X(k, j - 1, i), Cc = X(k, j, i - 1), D = X(k, j - 1, i - 1);
        double dxdc = 0.5 * (A.x + B.x - Cc.x - D.x), dydc = 0.5 * (A.y + B.y - Cc.y - D.y), dzdc = 0.5 * (A.z + B.z - Cc.z - D.z);
        double dxde = 0.5 * (A.x + Cc.x - B.x - D.x), dyde = 0.5 * (A.y + Cc.y - B.y - D.y), dzde = 0.5 * (A.z + Cc.z - B.z - D.z);
        st3(zett, q, R3<double>{dydc * dzde - dzdc * dyde, -dxdc * dzde + dzdc * dxde, dxdc * dyde - dydc * dxde});
    }
}

// cell-centred contravariant bases (mesh.c:970-1004)
__global__ void k_cell_pass2(Grid g, Metrics m, V3f<double> csit, V3f<double> etat, V3f<double> zett)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1, k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
    int q = g.lin(k, j, i);
    st3(m.csi, q, 0.5 * ld3(csit, q) + 0.5 * ld3(csit, g.lin(k, j, i - 1)));
    st3(m.eta, q, 0.5 * ld3(etat, q) + 0.5 * ld3(etat, g.lin(k, j - 1, i)));
    st3(m.zet, q, 0.5 * ld3(zett, q) + 0.5 * ld3(zett, g.lin(k - 1, j, i)));
}

// physical ghost layer mirrored from the first interior layer (mesh.c:1100-1180).
// dir 0: i planes over (k, j); dir 1: j planes over (k, i); dir 2: k planes over (j, i)
__global__ void k_mirror(Grid g, Metrics m, int dir)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = dir == 0 ? g.my : g.mx, nb = dir == 2 ? g.my : g.mz;
    if (a >= na || b >= nb) return;
    for (int side = 0; side < 2; side++) {
        int d, s;
        if (dir == 0) { int i = side ? g.mx - 1 : 0, is = side ? g.mx - 2 : 1; d = g.lin(b, a, i); s = g.lin(b, a, is); }
        else if (dir == 1) { int j = side ? g.my - 1 : 0, js = side ? g.my - 2 : 1; d = g.lin(b, j, a); s = g.lin(b, js, a); }
        else { int k = side ? g.mz - 1 : 0, ks = side ? g.mz - 2 : 1; d = g.lin(k, b, a); s = g.lin(ks, b, a); }
        st3(m.csi, d, ld3(m.csi, s)); st3(m.eta, d, ld3(m.eta, s)); st3(m.zet, d, ld3(m.zet, s)); m.aj[d] = m.aj[s];
    }
}

// periodic ghost cells of the cell metrics (mesh.c:1190-1270), one direction per launch
__global__ void k_periodic_cell_metrics(Grid g, Metrics m, int dir)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
    int na = dir == 0 ? g.my : g.mx, nb = dir == 2 ? g.my : g.mz;
    if (a >= na || b >= nb) return;
    for (int side = 0; side < 2; side++) {
        int d, s;
        if (dir == 0) { d = g.lin(b, a, side ? g.mx - 1 : 0); s = g.lin(b, a, side ? 1 : g.mx - 2); }
        else if (dir == 1) { d = g.lin(b, side ? g.my - 1 : 0, a); s = g.lin(b, side ? 1 : g.my - 2, a); }
        else { d = g.lin(side ? g.mz - 1 : 0, b, a); s = g.lin(side ? 1 : g.mz - 2, b, a); }
        st3(m.csi, d, ld3(m.csi, s)); st3(m.eta, d, ld3(m.eta, s)); st3(m.zet, d, ld3(m.zet, s)); m.aj[d] = m.aj[s];
    }
}

// face metrics: i faces (mesh.c:1354-1560), j faces (mesh.c:1562-1760),
// k faces (mesh.c:1762-1930)
__global__ void k_face_metrics(Nodes X, Metrics m)
{
    const Grid g = X.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    int q = g.lin(k, j, i);
    bool ii = i >= 1 && i <= g.mx - 2, jj = j >= 1 && j <= g.my - 2, kk = k >= 1 && k <= g.mz - 2;
    if (kk && jj && i <= g.mx - 2) {
        auto cx = [&](int ia) { return 0.25 * (X(k, j, ia) + X(k - 1, j, ia) + X(k, j - 1, ia) + X(k - 1, j - 1, ia)); };
        R3<double> d;
        if (i == 0) d = cx(i + 1) - cx(i);
        else if (i == g.mx - 2) {
            if (g.pi) { R3<double> t = cx(g.mx + 1) - cx(g.mx + 0) + cx(i) - cx(i - 1); d = 0.5 * t; }
            else d = cx(i) - cx(i - 1);
        } else d = 0.5 * (cx(i + 1) - cx(i - 1));
        R3<double> A = X(k, j, i), B = X(k - 1, j, i), Cc = X(k, j - 1, i), D = X(k - 1, j - 1, i);
        double dxde = 0.5 * (A.x + B.x - Cc.x - D.x), dyde = 0.5 * (A.y + B.y - Cc.y - D.y), dzde = 0.5 * (A.z + B.z - Cc.z - D.z);
        double dxdz = 0.5 * (Cc.x + A.x - D.x - B.x), dydz = 0.5 * (Cc.y + A.y - D.y - B.y), dzdz = 0.5 * (Cc.z + A.z - D.z - B.z);
        R3<double> fc, fe, fz; double faj;
        face_basis(d.x, d.y, d.z, dxde, dyde, dzde, dxdz, dydz, dzdz, fc, fe, fz, faj);
        st3(m.icsi, q, fc); st3(m.ieta, q, fe); st3(m.izet, q, fz); m.iaj[q] = faj;
    }
    if (kk && ii && j <= g.my - 2) {
        auto cy = [&](int ja) { return 0.25 * (X(k, ja, i) + X(k - 1, ja, i) + X(k, ja, i - 1) + X(k - 1, ja, i - 1)); };
        R3<double> A = X(k, j, i), B = X(k - 1, j, i), Cc = X(k, j, i - 1), D = X(k - 1, j, i - 1);
        double dxdc = 0.5 * (A.x + B.x - Cc.x - D.x), dydc = 0.5 * (A.y + B.y - Cc.y - D.y), dzdc = 0.5 * (A.z + B.z - Cc.z - D.z);
        R3<double> d;
        if (j == 0) d = cy(j + 1) - cy(j);
        else if (j == g.my - 2) {
            if (g.pj) { R3<double> t = cy(g.my + 1) - cy(g.my + 0) + cy(j) - cy(j - 1); d = 0.5 * t; }
            else d = cy(j) - cy(j - 1);
        } else d = 0.5 * (cy(j + 1) - cy(j - 1));
        double dxdz = 0.5 * (A.x + Cc.x - B.x - D.x), dydz = 0.5 * (A.y + Cc.y - B.y - D.y), dzdz = 0.5 * (A.z + Cc.z - B.z - D.z);
        R3<double> fc, fe, fz; double faj;
        face_basis(dxdc, dydc, dzdc, d.x, d.y, d.z, dxdz, dydz, dzdz, fc, fe, fz, faj);
        st3(m.jcsi, q, fc); st3(m.jeta, q, fe); st3(m.jzet, q, fz); m.jaj[q] = faj;
    }
    if (jj && ii && k <= g.mz - 2) {
        auto cz = [&](int ka) { return 0.25 * (X(ka, j, i) + X(ka, j - 1, i) + X(ka, j, i - 1) + X(ka, j - 1, i - 1)); };
        R3<double> A = X(k, j, i), B = X(k, j - 1, i), Cc = X(k, j, i - 1), D = X(k, j - 1, i - 1);
        double dxdc = 0.5 * (A.x + B.x - Cc.x - D.x), dydc = 0.5 * (A.y + B.y - Cc.y - D.y), dzdc = 0.5 * (A.z + B.z - Cc.z - D.z);
        double dxde = 0.5 * (A.x + Cc.x - B.x - D.x), dyde = 0.5 * (A.y + Cc.y - B.y - D.y), dzde = 0.5 * (A.z + Cc.z - B.z - D.z);
        R3<double> d;
        if (k == 0) d = cz(k + 1) - cz(k);
        else if (k == g.mz - 2) {
            if (g.pk) { R3<double> t = cz(g.mz + 1) - cz(g.mz + 0) + cz(k) - cz(k - 1); d = 0.5 * t; }
            else d = cz(k) - cz(k - 1);
        } else d = 0.5 * (cz(k + 1) - cz(k - 1));
        R3<double> fc, fe, fz; double faj;
        face_basis(dxdc, dydc, dzdc, dxde, dyde, dzde, d.x, d.y, d.z, fc, fe, fz, faj);
        st3(m.kcsi, q, fc); st3(m.keta, q, fe); st3(m.kzet, q, fz); m.kaj[q] = faj;
    }
}

// metric tensor at faces with boundary remapping (peqn.c:791-849)
__global__ void k_gtensor(Grid g, Metrics m)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.mx || j >= g.my || k >= g.mz) return;
    int a = i, b = j, c = k;
    if (i == 0)        a = g.pi ? -2 : 1;
    if (i == g.mx - 1) a = g.pi ? g.mx + 1 : g.mx - 2;
    if (j == 0)        b = g.pj ? -2 : 1;
    if (j == g.my - 1) b = g.pj ? g.my + 1 : g.my - 2;
    if (k == 0)        c = g.pk ? -2 : 1;
    if (k == g.mz - 1) c = g.pk ? g.mz + 1 : g.mz - 2;
    int s = g.id(c, b, a), d = g.lin(k, j, i);
    R3<double> ic = ld3(m.icsi, s), ie = ld3(m.ieta, s), iz = ld3(m.izet, s);
    R3<double> jc = ld3(m.jcsi, s), je = ld3(m.jeta, s), jz = ld3(m.jzet, s);
    R3<double> kc = ld3(m.kcsi, s), ke = ld3(m.keta, s), kz = ld3(m.kzet, s);
    m.g11[d] = dot3(ic, ic) * m.iaj[s];
    m.g12[d] = dot3(ie, ic) * m.iaj[s];
    m.g13[d] = dot3(iz, ic) * m.iaj[s];
    m.g21[d] = dot3(jc, je) * m.jaj[s];
    m.g22[d] = dot3(je, je) * m.jaj[s];
    m.g23[d] = dot3(jz, je) * m.jaj[s];
    m.g31[d] = dot3(kc, kz) * m.kaj[s];
    m.g32[d] = dot3(ke, kz) * m.kaj[s];
    m.g33[d] = dot3(kz, kz) * m.kaj[s];
}

}  // namespace

void metrics_from_nodes(tg_ctx *C, const double *d_nodes)
{
    const Grid g = C->g;
    const size_t G = (size_t)g.size();
    cudaStream_t st = C->stream;
    V3f<double> csit = dalloc3(C, G), etat = dalloc3(C, G), zett = dalloc3(C, G);
    Nodes X{d_nodes, g};
    k_cell_pass1<<<grid3(g.mx, g.my, g.mz), block3(), 0, st>>>(X, C->m, csit, etat, zett);
    k_cell_pass2<<<grid3(g.mx - 2, g.my - 2, g.mz - 2), block3(), 0, st>>>(g, C->m, csit, etat, zett);
    dim3 b2(32, 8);
    auto g2 = [&](int na, int nb) { return dim3((na + 31) / 32, (nb + 7) / 8); };
    k_mirror<<<g2(g.my, g.mz), b2, 0, st>>>(g, C->m, 0);
    k_mirror<<<g2(g.mx, g.mz), b2, 0, st>>>(g, C->m, 1);
    k_mirror<<<g2(g.mx, g.my), b2, 0, st>>>(g, C->m, 2);
    if (g.pi) k_periodic_cell_metrics<<<g2(g.my, g.mz), b2, 0, st>>>(g, C->m, 0);
    if (g.pj) k_periodic_cell_metrics<<<g2(g.mx, g.mz), b2, 0, st>>>(g, C->m, 1);
    if (g.pk) k_periodic_cell_metrics<<<g2(g.mx, g.my), b2, 0, st>>>(g, C->m, 2);
    k_face_metrics<<<grid3(g.mx, g.my, g.mz), block3(), 0, st>>>(X, C->m);
    k_gtensor<<<grid3(g.mx, g.my, g.mz), block3(), 0, st>>>(g, C->m);
    TG_CUDA(cudaGetLastError());
    TG_CUDA(cudaStreamSynchronize(st));
}

}  // namespace tg
