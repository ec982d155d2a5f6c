// TEST INFRASTRUCTURE ONLY: implementations of the single-rank PETSc / HYPRE /
// MPI stand-ins declared in petsc_stub.h (see there for the semantics kept).
#include "petsc_stub.h"

#include <map>
#include <stdexcept>
#include <string>

#include "tgref_capture.h"

[[noreturn]] void tgref_unexpected(const char *what)
{
    throw std::runtime_error(std::string("reference code called an unsupported PETSc/HYPRE/MPI function: ") + what);
}

// ------------------------------------------------------------------ layout
namespace {

struct Box {
    PetscInt xs, ys, zs, xm, ym, zm;
};

Box box_of(DM dm, bool local)
{
    Box b;
    if (local) {
        b.xs = tgref_gstart(dm->bx, dm->s); b.xm = tgref_gsize(dm->bx, dm->M, dm->s);
        b.ys = tgref_gstart(dm->by, dm->s); b.ym = tgref_gsize(dm->by, dm->N, dm->s);
        b.zs = tgref_gstart(dm->bz, dm->s); b.zm = tgref_gsize(dm->bz, dm->P, dm->s);
    } else {
        b.xs = b.ys = b.zs = 0;
        b.xm = dm->M; b.ym = dm->N; b.zm = dm->P;
    }
    return b;
}

size_t npoints(DM dm, bool local)
{
    Box b = box_of(dm, local);
    return (size_t)b.xm * b.ym * b.zm;
}

// global index of a (possibly ghost) index along a direction: wrapped for a
// periodic direction, -1 where a non-periodic direction has no point
inline PetscInt wrap(PetscInt q, PetscInt m, DMBoundaryType b)
{
    if (q >= 0 && q < m) return q;
    if (b == DM_BOUNDARY_PERIODIC) return ((q % m) + m) % m;
    return -1;
}

inline size_t offset(const Box &b, PetscInt k, PetscInt j, PetscInt i)
{
    return ((size_t)(k - b.zs) * b.ym + (j - b.ys)) * b.xm + (i - b.xs);
}

Vec new_vec(DM dm, bool local)
{
    Vec v = new _p_Vec();
    v->dm = dm;
    v->local = local;
    v->a.assign(npoints(dm, local) * dm->dof, 0.0);
    return v;
}

// dst (local) <- src (global or local): every point of dst whose global image
// exists takes the value src holds there; other ghost points keep theirs
void fill_local(DM dm, Vec src, Vec dst)
{
    const Box bs = box_of(dm, src->local), bd = box_of(dm, dst->local);
    const PetscInt dof = dm->dof;
    std::vector<double> out(dst->a);
    for (PetscInt k = bd.zs; k < bd.zs + bd.zm; k++) {
        const PetscInt kg = wrap(k, dm->P, dm->bz);
        if (kg < 0) continue;
        for (PetscInt j = bd.ys; j < bd.ys + bd.ym; j++) {
            const PetscInt jg = wrap(j, dm->N, dm->by);
            if (jg < 0) continue;
            for (PetscInt i = bd.xs; i < bd.xs + bd.xm; i++) {
                const PetscInt ig = wrap(i, dm->M, dm->bx);
                if (ig < 0) continue;
                const size_t d = offset(bd, k, j, i) * dof, s = offset(bs, kg, jg, ig) * dof;
                for (PetscInt c = 0; c < dof; c++) out[d + c] = src->a[s + c];
            }
        }
    }
    dst->a.swap(out);
}

}  // namespace

void *tgref_view(DM dm, Vec v, size_t elem_bytes)
{
    if (!dm || !v) tgref_unexpected("DMDAVecGetArray on a null DM or Vec");
    if (elem_bytes != sizeof(double) * (size_t)dm->dof)
        tgref_unexpected("DMDAVecGetArray: element size does not match the DM's dof");
    const Box b = box_of(dm, v->local);
    // pointer tables: [k] -> row tables, [k][j] -> element rows, offset so
    // that global (ghost) indices address them directly
    char **rows = new char *[(size_t)b.zm * b.ym];
    char ***planes = new char **[(size_t)b.zm];
    char *base = (char *)v->a.data();
    for (PetscInt k = 0; k < b.zm; k++) {
        for (PetscInt j = 0; j < b.ym; j++)
            rows[(size_t)k * b.ym + j] = base + (((size_t)k * b.ym + j) * b.xm) * elem_bytes - (ptrdiff_t)b.xs * (ptrdiff_t)elem_bytes;
        planes[k] = rows + (size_t)k * b.ym - b.ys;
    }
    v->views.push_back(rows);
    v->views.push_back(planes);
    return (void *)(planes - b.zs);
}

// ---------------------------------------------------------------------- DM
PetscErrorCode DMDAGetLocalInfo(DM dm, DMDALocalInfo *info)
{
    const Box g = box_of(dm, true);
    *info = DMDALocalInfo{};
    info->dim = 3; info->dof = dm->dof; info->sw = dm->s;
    info->mx = dm->M; info->my = dm->N; info->mz = dm->P;
    info->xs = info->ys = info->zs = 0;
    info->xm = dm->M; info->ym = dm->N; info->zm = dm->P;
    info->gxs = g.xs; info->gys = g.ys; info->gzs = g.zs;
    info->gxm = g.xm; info->gym = g.ym; info->gzm = g.zm;
    info->bx = dm->bx; info->by = dm->by; info->bz = dm->bz;
    info->st = DMDA_STENCIL_BOX;
    info->da = dm;
    return 0;
}
PetscErrorCode DMCreateGlobalVector(DM dm, Vec *v) { *v = new_vec(dm, false); return 0; }
PetscErrorCode DMCreateLocalVector(DM dm, Vec *v) { *v = new_vec(dm, true); return 0; }
PetscErrorCode DMGetLocalVector(DM dm, Vec *v) { *v = new_vec(dm, true); return 0; }
PetscErrorCode DMRestoreLocalVector(DM, Vec *v) { VecDestroy(v); return 0; }
PetscErrorCode DMGetGlobalVector(DM dm, Vec *v) { *v = new_vec(dm, false); return 0; }
PetscErrorCode DMRestoreGlobalVector(DM, Vec *v) { VecDestroy(v); return 0; }

PetscErrorCode DMGlobalToLocalBegin(DM, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode DMGlobalToLocalEnd(DM dm, Vec g, InsertMode mode, Vec l)
{
    if (mode != INSERT_VALUES) tgref_unexpected("DMGlobalToLocal with a mode other than INSERT_VALUES");
    fill_local(dm, g, l);
    return 0;
}
PetscErrorCode DMLocalToLocalBegin(DM, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode DMLocalToLocalEnd(DM dm, Vec a, InsertMode mode, Vec b)
{
    if (mode != INSERT_VALUES) tgref_unexpected("DMLocalToLocal with a mode other than INSERT_VALUES");
    fill_local(dm, a, b);
    return 0;
}
PetscErrorCode DMLocalToGlobalBegin(DM, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode DMLocalToGlobalEnd(DM dm, Vec l, InsertMode mode, Vec g)
{
    const Box bl = box_of(dm, true), bg = box_of(dm, false);
    const PetscInt dof = dm->dof;
    if (mode == INSERT_VALUES) {
        for (PetscInt k = 0; k < dm->P; k++)
            for (PetscInt j = 0; j < dm->N; j++)
                for (PetscInt i = 0; i < dm->M; i++)
                    for (PetscInt c = 0; c < dof; c++)
                        g->a[offset(bg, k, j, i) * dof + c] = l->a[offset(bl, k, j, i) * dof + c];
        return 0;
    }
    if (mode == ADD_VALUES) {
        for (PetscInt k = bl.zs; k < bl.zs + bl.zm; k++) {
            const PetscInt kg = wrap(k, dm->P, dm->bz);
            if (kg < 0) continue;
            for (PetscInt j = bl.ys; j < bl.ys + bl.ym; j++) {
                const PetscInt jg = wrap(j, dm->N, dm->by);
                if (jg < 0) continue;
                for (PetscInt i = bl.xs; i < bl.xs + bl.xm; i++) {
                    const PetscInt ig = wrap(i, dm->M, dm->bx);
                    if (ig < 0) continue;
                    for (PetscInt c = 0; c < dof; c++)
                        g->a[offset(bg, kg, jg, ig) * dof + c] += l->a[offset(bl, k, j, i) * dof + c];
                }
            }
        }
        return 0;
    }
    tgref_unexpected("DMLocalToGlobal with MAX_VALUES");
}
PetscErrorCode DMGetCoordinatesLocal(DM dm, Vec *c)
{
    if (!dm->coords_local) tgref_unexpected("DMGetCoordinatesLocal before coordinates were set");
    *c = dm->coords_local;
    return 0;
}
PetscErrorCode DMGetCoordinates(DM dm, Vec *c)
{
    if (!dm->coords_global) tgref_unexpected("DMGetCoordinates before coordinates were set");
    *c = dm->coords_global;
    return 0;
}
PetscErrorCode DMGetCoordinateDM(DM dm, DM *cdm)
{
    if (!dm->cdm) tgref_unexpected("DMGetCoordinateDM without a coordinate DM");
    *cdm = dm->cdm;
    return 0;
}

// --------------------------------------------------------------------- Vec
PetscErrorCode VecDuplicate(Vec a, Vec *b)
{
    *b = new _p_Vec();
    (*b)->dm = a->dm;
    (*b)->local = a->local;
    (*b)->a.assign(a->a.size(), 0.0);
    return 0;
}
PetscErrorCode VecDestroy(Vec *v)
{
    if (v && *v) {
        // the pointer tables of views handed out stay valid until here
        for (size_t q = 0; q < (*v)->views.size(); q += 2) {
            delete[] (char **)(*v)->views[q];
            delete[] (char ***)(*v)->views[q + 1];
        }
        delete *v;
        *v = nullptr;
    }
    return 0;
}
PetscErrorCode VecSet(Vec v, PetscScalar x) { for (double &e : v->a) e = x; return 0; }
PetscErrorCode VecCopy(Vec a, Vec b)
{
    if (a->a.size() != b->a.size()) tgref_unexpected("VecCopy between Vecs of different sizes");
    b->a = a->a;
    return 0;
}
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x)
{
    for (size_t q = 0; q < y->a.size(); q++) y->a[q] += a * x->a[q];
    return 0;
}
PetscErrorCode VecAYPX(Vec y, PetscScalar a, Vec x)
{
    for (size_t q = 0; q < y->a.size(); q++) y->a[q] = x->a[q] + a * y->a[q];
    return 0;
}
PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y)
{
    for (size_t q = 0; q < w->a.size(); q++) w->a[q] = a * x->a[q] + y->a[q];
    return 0;
}
PetscErrorCode VecScale(Vec v, PetscScalar a) { for (double &e : v->a) e *= a; return 0; }
PetscErrorCode VecNorm(Vec v, NormType t, PetscReal *r)
{
    double s = 0.0;
    if (t == NORM_2) { for (double e : v->a) s += e * e; *r = std::sqrt(s); return 0; }
    if (t == NORM_1) { for (double e : v->a) s += std::fabs(e); *r = s; return 0; }
    if (t == NORM_INFINITY) { for (double e : v->a) s = std::fmax(s, std::fabs(e)); *r = s; return 0; }
    tgref_unexpected("VecNorm type");
}
PetscErrorCode VecMax(Vec v, PetscInt *p, PetscReal *r)
{
    PetscInt arg = 0;
    for (size_t q = 1; q < v->a.size(); q++) if (v->a[q] > v->a[arg]) arg = (PetscInt)q;
    if (p) *p = arg;
    *r = v->a.empty() ? 0.0 : v->a[arg];
    return 0;
}
PetscErrorCode VecMin(Vec v, PetscInt *p, PetscReal *r)
{
    PetscInt arg = 0;
    for (size_t q = 1; q < v->a.size(); q++) if (v->a[q] < v->a[arg]) arg = (PetscInt)q;
    if (p) *p = arg;
    *r = v->a.empty() ? 0.0 : v->a[arg];
    return 0;
}
PetscErrorCode VecSum(Vec v, PetscScalar *s) { double t = 0.0; for (double e : v->a) t += e; *s = t; return 0; }
PetscErrorCode VecDot(Vec a, Vec b, PetscScalar *r)
{
    double t = 0.0;
    for (size_t q = 0; q < a->a.size(); q++) t += a->a[q] * b->a[q];
    *r = t;
    return 0;
}
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) { *a = v->a.data(); return 0; }
PetscErrorCode VecRestoreArray(Vec, PetscScalar **a) { *a = nullptr; return 0; }
PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n) { *n = (PetscInt)v->a.size(); return 0; }
PetscErrorCode VecGetSize(Vec v, PetscInt *n) { *n = (PetscInt)v->a.size(); return 0; }
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }

// ------------------------------------------------------------------- misc
static bool g_quiet = true;
static std::vector<std::string> g_printed;     // the last messages of PetscPrintf
void tgref_set_quiet(bool q) { g_quiet = q; }

PetscErrorCode PetscPrintf(MPI_Comm, const char *fmt, ...)
{
    char buf[2048];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (g_printed.size() >= 256) g_printed.erase(g_printed.begin(), g_printed.begin() + 128);
    g_printed.emplace_back(buf);
    if (!g_quiet) std::fputs(buf, stdout);
    return 0;
}

bool tgref_printed_value(const char *prefix, double *value)
{
    const size_t n = std::strlen(prefix);
    for (size_t q = g_printed.size(); q-- > 0;) {
        const std::string &m = g_printed[q];
        if (m.compare(0, n, prefix) == 0) {
            *value = std::strtod(m.c_str() + n, nullptr);
            return true;
        }
    }
    return false;
}
PetscErrorCode PetscFPrintf(MPI_Comm, FILE *f, const char *fmt, ...)
{
    if (g_quiet) return 0;
    va_list ap;
    va_start(ap, fmt);
    vfprintf(f, fmt, ap);
    va_end(ap);
    return 0;
}
PetscErrorCode PetscTime(PetscLogDouble *t) { *t = 0.0; return 0; }
PetscErrorCode PetscBarrier(void *) { return 0; }
PetscErrorCode MatMFFDComputeJacobian(SNES, Vec, Mat, Mat, void *) { tgref_unexpected("MatMFFDComputeJacobian"); }
HYPRE_Int HYPRE_BoomerAMGSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { tgref_unexpected("HYPRE_BoomerAMGSolve"); }
HYPRE_Int HYPRE_BoomerAMGSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { tgref_unexpected("HYPRE_BoomerAMGSetup"); }

// --------------------------------------------------------------------- MPI
static size_t type_bytes(MPI_Datatype t)
{
    switch (t) {
    case MPI_DOUBLE: return sizeof(double);
    case MPI_INT: return sizeof(int);
    case MPI_LONG: return sizeof(long);
    case MPI_CHAR: return 1;
    case MPI_FLOAT: return sizeof(float);
    case MPI_UNSIGNED_LONG: return sizeof(unsigned long);
    default: tgref_unexpected("MPI datatype");
    }
}
int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm)
{
    if (send != MPI_IN_PLACE) std::memcpy(recv, send, (size_t)count * type_bytes(type));
    return 0;
}
int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm)
{
    if (send != MPI_IN_PLACE) std::memcpy(recv, send, (size_t)count * type_bytes(type));
    return 0;
}
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
int MPI_Ibcast(void *, int, MPI_Datatype, int, MPI_Comm, MPI_Request *r) { if (r) *r = 0; return 0; }
int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
int MPI_Barrier(MPI_Comm) { return 0; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }

// ------------------------------------------------------------------- HYPRE
// the matrix of SetCoeffMatrix, captured row by row (see tgref_capture.h)
static std::map<long, std::map<long, double>> g_rows;

HYPRE_Int HYPRE_IJMatrixSetValues(HYPRE_IJMatrix, HYPRE_Int nrows, HYPRE_Int *ncols, const HYPRE_BigInt *rows,
                                  const HYPRE_BigInt *cols, const HYPRE_Complex *values)
{
    size_t q = 0;
    for (HYPRE_Int r = 0; r < nrows; r++) {
        auto &row = g_rows[rows[r]];
        for (HYPRE_Int c = 0; c < ncols[r]; c++, q++) row[cols[q]] = values[q];
    }
    return 0;
}
HYPRE_Int HYPRE_IJMatrixCreate(MPI_Comm, HYPRE_BigInt, HYPRE_BigInt, HYPRE_BigInt, HYPRE_BigInt, HYPRE_IJMatrix *A)
{
    *A = (HYPRE_IJMatrix)&g_rows;
    return 0;
}
HYPRE_Int HYPRE_IJMatrixInitialize(HYPRE_IJMatrix) { return 0; }
HYPRE_Int HYPRE_IJMatrixAssemble(HYPRE_IJMatrix) { return 0; }
HYPRE_Int HYPRE_IJMatrixSetObjectType(HYPRE_IJMatrix, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_IJMatrixSetRowSizes(HYPRE_IJMatrix, const HYPRE_Int *) { return 0; }
HYPRE_Int HYPRE_IJMatrixSetMaxOffProcElmts(HYPRE_IJMatrix, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_IJMatrixDestroy(HYPRE_IJMatrix) { return 0; }
HYPRE_Int HYPRE_IJMatrixGetObject(HYPRE_IJMatrix, void **obj) { *obj = nullptr; return 0; }

void tgref_matrix_clear() { g_rows.clear(); }
long tgref_matrix_nnz()
{
    long n = 0;
    for (auto &r : g_rows) n += (long)r.second.size();
    return n;
}
long tgref_matrix_rows() { return g_rows.empty() ? 0 : g_rows.rbegin()->first + 1; }
void tgref_matrix_csr(long *rowptr, long *col, double *val)
{
    const long n = tgref_matrix_rows();
    long q = 0, r = 0;
    for (auto &row : g_rows) {
        while (r <= row.first) rowptr[r++] = q;
        for (auto &e : row.second) { col[q] = e.first; val[q] = e.second; q++; }
    }
    while (r <= n) rowptr[r++] = q;
}

// -------------------------------------------------------- HYPRE vectors
struct hypre_IJVector_struct {
    HYPRE_BigInt lo = 0;
    std::vector<double> v;
};

HYPRE_Int HYPRE_IJMatrixGetValues(HYPRE_IJMatrix, HYPRE_Int nrows, HYPRE_Int *ncols, HYPRE_BigInt *rows,
                                  HYPRE_BigInt *cols, HYPRE_Complex *values)
{
    size_t q = 0;
    for (HYPRE_Int r = 0; r < nrows; r++) {
        auto it = g_rows.find((long)rows[r]);
        for (HYPRE_Int c = 0; c < ncols[r]; c++, q++) {
            double val = 0.0;
            if (it != g_rows.end()) {
                auto e = it->second.find((long)cols[q]);
                if (e != it->second.end()) val = e->second;
            }
            values[q] = val;
        }
    }
    return 0;
}
HYPRE_Int HYPRE_IJVectorCreate(MPI_Comm, HYPRE_BigInt jl, HYPRE_BigInt ju, HYPRE_IJVector *v)
{
    *v = new hypre_IJVector_struct();
    (*v)->lo = jl;
    (*v)->v.assign((size_t)(ju - jl + 1), 0.0);
    return 0;
}
HYPRE_Int HYPRE_IJVectorSetObjectType(HYPRE_IJVector, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_IJVectorInitialize(HYPRE_IJVector) { return 0; }
HYPRE_Int HYPRE_IJVectorSetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt *idx, const HYPRE_Complex *val)
{
    for (HYPRE_Int q = 0; q < n; q++) v->v.at((size_t)(idx[q] - v->lo)) = val[q];
    return 0;
}
HYPRE_Int HYPRE_IJVectorAddToValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt *idx, const HYPRE_Complex *val)
{
    for (HYPRE_Int q = 0; q < n; q++) v->v.at((size_t)(idx[q] - v->lo)) += val[q];
    return 0;
}
HYPRE_Int HYPRE_IJVectorGetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt *idx, HYPRE_Complex *val)
{
    for (HYPRE_Int q = 0; q < n; q++) val[q] = v->v.at((size_t)(idx[q] - v->lo));
    return 0;
}
HYPRE_Int HYPRE_IJVectorAssemble(HYPRE_IJVector) { return 0; }
HYPRE_Int HYPRE_IJVectorGetObject(HYPRE_IJVector v, void **obj) { *obj = (void *)v; return 0; }
HYPRE_Int HYPRE_IJVectorDestroy(HYPRE_IJVector v) { delete v; return 0; }

PetscErrorCode VecCreateMPI(MPI_Comm, PetscInt n, PetscInt, Vec *v)
{
    *v = new _p_Vec();
    (*v)->a.assign((size_t)n, 0.0);
    return 0;
}

// ------------------------------------------------------ HYPRE solve stand-in
// The pinned pressure system has a unique solution, so the reference's
// BoomerAMG-preconditioned GMRES / PCG to its tolerance is replaced by a
// Jacobi-preconditioned BiCGStab on the captured matrix, run until the true
// relative residual is below TGREF_SOLVE_RTOL. With inflow and outflow
// patches the attainable residual lies a few times above 1e-14 (a direct
// solve of the 20 x 12 x 10 channel leaves 2.7e-14), so a solve that ends
// below TGREF_SOLVE_ACCEPT still counts as converged.
namespace {
constexpr double TGREF_SOLVE_RTOL = 1e-14;
constexpr double TGREF_SOLVE_ACCEPT = 1e-13;
long g_last_iterations = 0;
double g_last_residual = 0.0;

struct Csr {
    std::vector<long> rp, col;
    std::vector<double> val, dinv;
};

Csr captured_csr(size_t n)
{
    Csr A;
    A.rp.assign(n + 1, 0);
    A.dinv.assign(n, 1.0);
    for (auto &row : g_rows) {
        if ((size_t)row.first >= n) tgref_unexpected("captured matrix row beyond the vector size");
        A.rp[row.first + 1] = (long)row.second.size();
    }
    for (size_t r = 0; r < n; r++) A.rp[r + 1] += A.rp[r];
    A.col.resize(A.rp[n]);
    A.val.resize(A.rp[n]);
    for (auto &row : g_rows) {
        long q = A.rp[row.first];
        for (auto &e : row.second) {
            A.col[q] = e.first; A.val[q] = e.second; q++;
            if (e.first == row.first && e.second != 0.0) A.dinv[row.first] = 1.0 / e.second;
        }
    }
    return A;
}

void matvec(const Csr &A, const std::vector<double> &x, std::vector<double> &y)
{
    const size_t n = x.size();
    for (size_t r = 0; r < n; r++) {
        double s = 0.0;
        for (long q = A.rp[r]; q < A.rp[r + 1]; q++) s += A.val[q] * x[A.col[q]];
        y[r] = s;
    }
}

double dot(const std::vector<double> &a, const std::vector<double> &b)
{
    double s = 0.0;
    for (size_t q = 0; q < a.size(); q++) s += a[q] * b[q];
    return s;
}

HYPRE_Int tight_solve(HYPRE_ParVector bv, HYPRE_ParVector xv)
{
    auto *b = (hypre_IJVector_struct *)bv, *xs = (hypre_IJVector_struct *)xv;
    const size_t n = b->v.size();
    const Csr A = captured_csr(n);
    std::vector<double> x = xs->v, r(n), rh(n), p(n, 0.0), v(n, 0.0), ph(n), s(n), sh(n), t(n);
    const double bn = std::sqrt(dot(b->v, b->v));
    long it = 0;
    double rn = 0.0;
    for (int restart = 0; restart < 200; restart++) {
        matvec(A, x, r);
        for (size_t q = 0; q < n; q++) r[q] = b->v[q] - r[q];
        rn = std::sqrt(dot(r, r));
        if (bn == 0.0 || rn <= TGREF_SOLVE_RTOL * bn) break;
        rh = r;
        std::fill(p.begin(), p.end(), 0.0);
        std::fill(v.begin(), v.end(), 0.0);
        double rho = 1.0, alpha = 1.0, omega = 1.0;
        for (int k = 0; k < 2000; k++, it++) {
            const double rho1 = dot(rh, r);
            if (rho1 == 0.0) break;
            const double beta = (rho1 / rho) * (alpha / omega);
            rho = rho1;
            for (size_t q = 0; q < n; q++) p[q] = r[q] + beta * (p[q] - omega * v[q]);
            for (size_t q = 0; q < n; q++) ph[q] = A.dinv[q] * p[q];
            matvec(A, ph, v);
            alpha = rho / dot(rh, v);
            for (size_t q = 0; q < n; q++) s[q] = r[q] - alpha * v[q];
            for (size_t q = 0; q < n; q++) sh[q] = A.dinv[q] * s[q];
            matvec(A, sh, t);
            const double tt = dot(t, t);
            omega = tt > 0.0 ? dot(t, s) / tt : 0.0;
            for (size_t q = 0; q < n; q++) { x[q] += alpha * ph[q] + omega * sh[q]; r[q] = s[q] - omega * t[q]; }
            if (std::sqrt(dot(r, r)) <= 0.1 * TGREF_SOLVE_RTOL * bn || omega == 0.0) { it++; break; }
        }
    }
    xs->v = x;
    g_last_iterations = it;
    g_last_residual = bn > 0.0 ? rn / bn : rn;
    if (bn > 0.0 && rn > TGREF_SOLVE_ACCEPT * bn) tgref_unexpected("stand-in pressure solve did not converge");
    return 0;
}
}  // namespace

HYPRE_Int HYPRE_ParCSRGMRESSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { return 0; }
HYPRE_Int HYPRE_ParCSRGMRESSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector b, HYPRE_ParVector x) { return tight_solve(b, x); }
HYPRE_Int HYPRE_GMRESGetNumIterations(HYPRE_Solver, HYPRE_Int *it) { *it = g_last_iterations; return 0; }
HYPRE_Int HYPRE_ParCSRGMRESGetFinalRelativeResidualNorm(HYPRE_Solver, HYPRE_Real *r) { *r = g_last_residual; return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { return 0; }
HYPRE_Int HYPRE_ParCSRPCGSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector b, HYPRE_ParVector x) { return tight_solve(b, x); }
HYPRE_Int HYPRE_PCGGetNumIterations(HYPRE_Solver, HYPRE_Int *it) { *it = g_last_iterations; return 0; }
HYPRE_Int HYPRE_PCGGetFinalRelativeResidualNorm(HYPRE_Solver, HYPRE_Real *r) { *r = g_last_residual; return 0; }
