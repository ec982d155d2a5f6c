/*
 * TEST INFRASTRUCTURE ONLY. A single-rank stand-in for the parts of the PETSc
 * 3.15, HYPRE 2.20 and MPI interfaces that TOSCA's sources name, so that the
 * reference's own stage functions (FormU, GradP, UpdateNut, SetCoeffMatrix,
 * ProjectVelocity, ...) compile unchanged from their source files and can be
 * run on the CPU as the checker of the oracle restatement.
 *
 * Semantics kept (one MPI rank, one DMDA block per grid):
 *   - Vec: a contiguous array of doubles; global Vecs span the DMDA extent,
 *     local Vecs the ghosted extent (extent + 2 s in every direction for the
 *     GHOSTED and PERIODIC boundary types TOSCA uses, mesh.c:136-142);
 *   - DMDAVecGetArray: a [k][j][i] view indexed by global indices (ghost
 *     indices negative or >= m on a local Vec), elements of dof doubles;
 *   - DMGlobalToLocal / DMLocalToLocal: copy owned points and fill ghosts of
 *     periodic directions by wrap; ghosts of non-periodic directions keep
 *     their values (DM_BOUNDARY_GHOSTED);
 *   - DMLocalToGlobal: owned points (INSERT_VALUES) or summed images (ADD_VALUES);
 *   - MPI collectives: identities on one rank;
 *   - HYPRE_IJMatrixSetValues: rows captured into a sparse map.
 * Everything else that TOSCA's set-up code calls is declared as a catch-all
 * that reports an unexpected call: the harness builds TOSCA's structures
 * itself and never runs that code.
 */
#ifndef TGREF_PETSC_STUB_H
#define TGREF_PETSC_STUB_H

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

// ------------------------------------------------------------------ scalars
typedef int64_t PetscInt;          // the 64-bit-index build TOSCA recommends
typedef double PetscReal;
typedef double PetscScalar;
typedef int PetscErrorCode;
typedef int PetscMPIInt;
typedef double PetscLogDouble;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef int PetscEnum;

#define PETSC_NULL 0
#define PETSC_DEFAULT (-2)
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE (-1)
#define PETSC_MAX_PATH_LEN 4096

#define PetscMax(a, b) (((a) < (b)) ? (b) : (a))
#define PetscMin(a, b) (((a) < (b)) ? (a) : (b))
#define PetscSign(a) (((a) >= 0) ? ((a) == 0 ? 0 : 1) : -1)
#define PetscSqrtReal(a) std::sqrt(a)
#define PetscPowReal(a, b) std::pow(a, b)
#define PetscAbsReal(a) std::fabs(a)
#define PetscAbsScalar(a) std::fabs(a)
#define PetscExpReal(a) std::exp(a)
#define PetscLogReal(a) std::log(a)
#define PetscSinReal(a) std::sin(a)
#define PetscCosReal(a) std::cos(a)
#define PetscTanhReal(a) std::tanh(a)
#define PetscAtanReal(a) std::atan(a)
#define PetscAtan2Real(a, b) std::atan2(a, b)
#define PetscFloorReal(a) std::floor(a)
#define PetscCeilReal(a) std::ceil(a)
#define PetscRealPart(a) (a)
#define PetscSqr(a) ((a) * (a))
#define PetscSqrReal(a) ((a) * (a))

// ---------------------------------------------------------------------- MPI
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define PETSC_COMM_WORLD 1
#define PETSC_COMM_SELF 2
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_LONG 3
#define MPI_CHAR 4
#define MPI_FLOAT 5
#define MPI_UNSIGNED_LONG 6
#define MPIU_REAL 1
#define MPIU_SCALAR 1
#define MPIU_INT 3
#define MPIU_BOOL 2
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPIU_SUM 1
#define MPIU_MAX 2
#define MPIU_MIN 3
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

typedef long MPI_Aint;
#define MPI_BYTE 7
#define MPI_REPLACE 4
#define PETSC_COPY_VALUES 0
typedef struct { PetscMPIInt rank; PetscInt index; } PetscSFNode;

int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Ibcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *st);
int MPI_Barrier(MPI_Comm comm);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);

// ------------------------------------------------------------ PETSc objects
struct _p_Vec;
struct _p_DM;
typedef _p_Vec *Vec;
typedef _p_DM *DM;
typedef struct _p_Mat *Mat;
typedef struct _p_KSP *KSP;
typedef struct _p_SNES *SNES;
typedef struct _p_PC *PC;
typedef struct _p_IS *IS;
typedef struct _p_PetscSF *PetscSF;
typedef struct _p_MatNullSpace *MatNullSpace;
typedef struct _p_PetscViewer *PetscViewer;
typedef struct _p_PetscSubcomm *PetscSubcomm;
typedef struct _p_PetscRandom *PetscRandom;
typedef struct _p_VecScatter *VecScatter;
typedef struct _p_PetscViewerAndFormat PetscViewerAndFormat;
typedef const char *KSPType;
typedef const char *PCType;
typedef const char *SNESType;
typedef const char *MatType;
typedef const char *MatMFFDType;
typedef enum { INSERT_VALUES, ADD_VALUES, MAX_VALUES } InsertMode;
typedef enum { NORM_1, NORM_2, NORM_FROBENIUS, NORM_INFINITY, NORM_1_AND_2 } NormType;
typedef enum { SCATTER_FORWARD, SCATTER_REVERSE } ScatterMode;
typedef enum { DM_BOUNDARY_NONE, DM_BOUNDARY_GHOSTED, DM_BOUNDARY_MIRROR, DM_BOUNDARY_PERIODIC, DM_BOUNDARY_TWIST } DMBoundaryType;
typedef enum { DMDA_STENCIL_STAR, DMDA_STENCIL_BOX } DMDAStencilType;
typedef enum { PC_LEFT, PC_RIGHT, PC_SYMMETRIC } PCSide;
typedef enum { PC_MG_MULTIPLICATIVE, PC_MG_ADDITIVE, PC_MG_FULL, PC_MG_KASKADE } PCMGType;
typedef enum { MAT_FINAL_ASSEMBLY, MAT_FLUSH_ASSEMBLY } MatAssemblyType;
typedef enum { MATOP_MULT } MatOperation;
typedef enum { MAT_NEW_NONZERO_ALLOCATION_ERR, MAT_NEW_NONZERO_LOCATION_ERR, MAT_IGNORE_ZERO_ENTRIES } MatOption;
typedef enum { PETSC_VIEWER_DEFAULT } PetscViewerFormat;
#define PETSC_VIEWER_STDOUT_WORLD ((PetscViewer)0)

#define KSPGMRES "gmres"
#define KSPFGMRES "fgmres"
#define KSPBCGS "bcgs"
#define KSPBCGSL "bcgsl"
#define KSPCG "cg"
#define PCNONE "none"
#define PCGAMG "gamg"
#define PCMG "mg"
#define PCSOR "sor"
#define PCJACOBI "jacobi"
#define PCILU "ilu"
#define SNESNEWTONTR "newtontr"
#define SNESNEWTONLS "newtonls"
#define MATMFFD "mffd"
#define MATMFFD_WP "wp"
#define MATMFFD_DS "ds"
#define MATSHELL "shell"
#define MATMPIAIJ "mpiaij"

struct DMDALocalInfo {
    PetscInt dim, dof, sw;
    PetscInt mx, my, mz;
    PetscInt xs, ys, zs;
    PetscInt xm, ym, zm;
    PetscInt gxs, gys, gzs;
    PetscInt gxm, gym, gzm;
    DMBoundaryType bx, by, bz;
    DMDAStencilType st;
    DM da;
};

// the stand-ins' own structures
struct _p_DM {
    PetscInt M, N, P;              // global points in x (i), y (j), z (k)
    PetscInt dof, s;
    DMBoundaryType bx, by, bz;
    Vec coords_local = nullptr;    // node coordinates (local, ghosted), dof 3
    Vec coords_global = nullptr;
    DM cdm = nullptr;              // coordinate DM (dof 3)
};
struct _p_Vec {
    DM dm = nullptr;
    bool local = false;
    std::vector<double> a;
    std::vector<void *> views;     // pointer tables of DMDAVecGetArray
};

// ghosted start of a direction of a DMDA (one rank)
inline PetscInt tgref_gstart(DMBoundaryType b, PetscInt s) { return b == DM_BOUNDARY_NONE ? 0 : -s; }
inline PetscInt tgref_gsize(DMBoundaryType b, PetscInt m, PetscInt s) { return b == DM_BOUNDARY_NONE ? m : m + 2 * s; }

[[noreturn]] void tgref_unexpected(const char *what);
void *tgref_view(DM dm, Vec v, size_t elem_bytes);

template <class T>
inline PetscErrorCode DMDAVecGetArray(DM dm, Vec v, T *array)
{
    typedef typename std::remove_pointer<typename std::remove_pointer<typename std::remove_pointer<T>::type>::type>::type E;
    *array = (T)tgref_view(dm, v, sizeof(E));
    return 0;
}
template <class T>
inline PetscErrorCode DMDAVecGetArrayRead(DM dm, Vec v, T *array) { return DMDAVecGetArray(dm, v, array); }
template <class T>
inline PetscErrorCode DMDAVecRestoreArray(DM, Vec, T *array) { *array = nullptr; return 0; }
template <class T>
inline PetscErrorCode DMDAVecRestoreArrayRead(DM, Vec, T *array) { *array = nullptr; return 0; }

PetscErrorCode DMDAGetLocalInfo(DM dm, DMDALocalInfo *info);
PetscErrorCode DMCreateGlobalVector(DM dm, Vec *v);
PetscErrorCode DMCreateLocalVector(DM dm, Vec *v);
PetscErrorCode DMGetLocalVector(DM dm, Vec *v);
PetscErrorCode DMRestoreLocalVector(DM dm, Vec *v);
PetscErrorCode DMGetGlobalVector(DM dm, Vec *v);
PetscErrorCode DMRestoreGlobalVector(DM dm, Vec *v);
PetscErrorCode DMGlobalToLocalBegin(DM dm, Vec g, InsertMode mode, Vec l);
PetscErrorCode DMGlobalToLocalEnd(DM dm, Vec g, InsertMode mode, Vec l);
PetscErrorCode DMLocalToLocalBegin(DM dm, Vec a, InsertMode mode, Vec b);
PetscErrorCode DMLocalToLocalEnd(DM dm, Vec a, InsertMode mode, Vec b);
PetscErrorCode DMLocalToGlobalBegin(DM dm, Vec l, InsertMode mode, Vec g);
PetscErrorCode DMLocalToGlobalEnd(DM dm, Vec l, InsertMode mode, Vec g);
PetscErrorCode DMGetCoordinatesLocal(DM dm, Vec *c);
PetscErrorCode DMGetCoordinates(DM dm, Vec *c);
PetscErrorCode DMGetCoordinateDM(DM dm, DM *cdm);

PetscErrorCode VecDuplicate(Vec a, Vec *b);
PetscErrorCode VecDestroy(Vec *v);
PetscErrorCode VecSet(Vec v, PetscScalar x);
PetscErrorCode VecCopy(Vec a, Vec b);
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x);
PetscErrorCode VecAYPX(Vec y, PetscScalar a, Vec x);
PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y);
PetscErrorCode VecScale(Vec v, PetscScalar a);
PetscErrorCode VecNorm(Vec v, NormType t, PetscReal *r);
PetscErrorCode VecMax(Vec v, PetscInt *p, PetscReal *r);
PetscErrorCode VecMin(Vec v, PetscInt *p, PetscReal *r);
PetscErrorCode VecSum(Vec v, PetscScalar *s);
PetscErrorCode VecDot(Vec a, Vec b, PetscScalar *r);
PetscErrorCode VecGetArray(Vec v, PetscScalar **a);
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a);
PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n);
PetscErrorCode VecGetSize(Vec v, PetscInt *n);
PetscErrorCode VecAssemblyBegin(Vec v);
PetscErrorCode VecAssemblyEnd(Vec v);

PetscErrorCode PetscPrintf(MPI_Comm comm, const char *fmt, ...);
PetscErrorCode PetscFPrintf(MPI_Comm comm, FILE *f, const char *fmt, ...);
PetscErrorCode PetscTime(PetscLogDouble *t);
PetscErrorCode PetscBarrier(void *);
// PetscMalloc writes the new block's address through a void** view of its
// second argument, whatever that argument's declared type
template <class T>
inline PetscErrorCode PetscMalloc(size_t n, T *p) { *(void **)p = std::calloc(1, n ? n : 1); return 0; }
template <class T>
inline PetscErrorCode PetscFree(T *&p) { std::free((void *)p); p = nullptr; return 0; }

// ------------------------------------------------------------------- HYPRE
// PETSc built with 64-bit indices builds HYPRE with big integers too
typedef long long HYPRE_Int;
typedef long long HYPRE_BigInt;
typedef double HYPRE_Real;
typedef double HYPRE_Complex;
typedef struct hypre_IJMatrix_struct *HYPRE_IJMatrix;
typedef struct hypre_IJVector_struct *HYPRE_IJVector;
typedef struct hypre_ParCSRMatrix_struct *HYPRE_ParCSRMatrix;
typedef struct hypre_ParVector_struct *HYPRE_ParVector;
typedef struct hypre_Solver_struct *HYPRE_Solver;
typedef struct hypre_Matrix_struct *HYPRE_Matrix;
typedef struct hypre_Vector_struct *HYPRE_Vector;
typedef HYPRE_Int (*HYPRE_PtrToSolverFcn)(HYPRE_Solver, HYPRE_Matrix, HYPRE_Vector, HYPRE_Vector);
#define HYPRE_PARCSR 5555

HYPRE_Int HYPRE_IJMatrixSetValues(HYPRE_IJMatrix A, HYPRE_Int nrows, HYPRE_Int *ncols, const HYPRE_BigInt *rows,
                                  const HYPRE_BigInt *cols, const HYPRE_Complex *values);
HYPRE_Int HYPRE_IJMatrixCreate(MPI_Comm comm, HYPRE_BigInt il, HYPRE_BigInt iu, HYPRE_BigInt jl, HYPRE_BigInt ju,
                               HYPRE_IJMatrix *A);
HYPRE_Int HYPRE_IJMatrixInitialize(HYPRE_IJMatrix A);
HYPRE_Int HYPRE_IJMatrixAssemble(HYPRE_IJMatrix A);
HYPRE_Int HYPRE_IJMatrixSetObjectType(HYPRE_IJMatrix A, HYPRE_Int type);
HYPRE_Int HYPRE_IJMatrixSetRowSizes(HYPRE_IJMatrix A, const HYPRE_Int *sizes);
HYPRE_Int HYPRE_IJMatrixSetMaxOffProcElmts(HYPRE_IJMatrix A, HYPRE_Int n);
HYPRE_Int HYPRE_IJMatrixDestroy(HYPRE_IJMatrix A);
HYPRE_Int HYPRE_IJMatrixGetObject(HYPRE_IJMatrix A, void **obj);
HYPRE_Int HYPRE_IJMatrixGetValues(HYPRE_IJMatrix A, HYPRE_Int nrows, HYPRE_Int *ncols, HYPRE_BigInt *rows,
                                  HYPRE_BigInt *cols, HYPRE_Complex *values);
HYPRE_Int HYPRE_IJVectorCreate(MPI_Comm comm, HYPRE_BigInt jl, HYPRE_BigInt ju, HYPRE_IJVector *v);
HYPRE_Int HYPRE_IJVectorSetObjectType(HYPRE_IJVector v, HYPRE_Int type);
HYPRE_Int HYPRE_IJVectorInitialize(HYPRE_IJVector v);
HYPRE_Int HYPRE_IJVectorSetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt *idx, const HYPRE_Complex *val);
HYPRE_Int HYPRE_IJVectorAddToValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt *idx, const HYPRE_Complex *val);
HYPRE_Int HYPRE_IJVectorGetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt *idx, HYPRE_Complex *val);
HYPRE_Int HYPRE_IJVectorAssemble(HYPRE_IJVector v);
HYPRE_Int HYPRE_IJVectorGetObject(HYPRE_IJVector v, void **obj);
HYPRE_Int HYPRE_IJVectorDestroy(HYPRE_IJVector v);
// the Krylov solves of SolvePEqn: a tight solve of the captured matrix
HYPRE_Int HYPRE_ParCSRGMRESSetup(HYPRE_Solver s, HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x);
HYPRE_Int HYPRE_ParCSRGMRESSolve(HYPRE_Solver s, HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x);
HYPRE_Int HYPRE_GMRESGetNumIterations(HYPRE_Solver s, HYPRE_Int *it);
HYPRE_Int HYPRE_ParCSRGMRESGetFinalRelativeResidualNorm(HYPRE_Solver s, HYPRE_Real *r);
HYPRE_Int HYPRE_ParCSRPCGSetup(HYPRE_Solver s, HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x);
HYPRE_Int HYPRE_ParCSRPCGSolve(HYPRE_Solver s, HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x);
HYPRE_Int HYPRE_PCGGetNumIterations(HYPRE_Solver s, HYPRE_Int *it);
HYPRE_Int HYPRE_PCGGetFinalRelativeResidualNorm(HYPRE_Solver s, HYPRE_Real *r);
PetscErrorCode VecCreateMPI(MPI_Comm comm, PetscInt n, PetscInt N, Vec *v);

// passed by name as callbacks, so declared with their signatures
PetscErrorCode MatMFFDComputeJacobian(SNES snes, Vec x, Mat J, Mat B, void *ctx);
HYPRE_Int HYPRE_BoomerAMGSolve(HYPRE_Solver s, HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x);
HYPRE_Int HYPRE_BoomerAMGSetup(HYPRE_Solver s, HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x);

// ---------------------------------------------------- catch-all declarations
// Named by TOSCA's set-up and solver code that the harness never runs: a call
// reports itself as unexpected.
#define TGREF_UNEXPECTED(name) \
    template <class... A> inline int name(A...) { tgref_unexpected(#name); }

TGREF_UNEXPECTED(PetscOptionsGetReal)
TGREF_UNEXPECTED(PetscOptionsGetInt)
TGREF_UNEXPECTED(PetscOptionsGetString)
TGREF_UNEXPECTED(PetscOptionsGetEnum)
TGREF_UNEXPECTED(PetscOptionsInsertFile)
TGREF_UNEXPECTED(PetscOptionsSetValue)
TGREF_UNEXPECTED(PetscOptionsHasName)
TGREF_UNEXPECTED(PetscViewerAndFormatCreate)
TGREF_UNEXPECTED(PetscViewerAndFormatDestroy)
TGREF_UNEXPECTED(PetscSubcommCreate)
TGREF_UNEXPECTED(PetscSubcommSetTypeGeneral)
TGREF_UNEXPECTED(PetscSubcommChild)
TGREF_UNEXPECTED(DMDACreate3d)
TGREF_UNEXPECTED(DMSetUp)
TGREF_UNEXPECTED(DMDASetUniformCoordinates)
TGREF_UNEXPECTED(DMSetCoordinates)
TGREF_UNEXPECTED(DMSetCoordinatesLocal)
TGREF_UNEXPECTED(DMDAGetCoordinates)
TGREF_UNEXPECTED(DMDestroy)
TGREF_UNEXPECTED(DMDAGetInfo)
TGREF_UNEXPECTED(DMDAGetCorners)
TGREF_UNEXPECTED(DMDAGetGhostCorners)
TGREF_UNEXPECTED(DMDAGetOwnershipRanges)
TGREF_UNEXPECTED(VecCreateSeq)
TGREF_UNEXPECTED(VecSetValues)
TGREF_UNEXPECTED(VecGetValues)
TGREF_UNEXPECTED(VecView)
TGREF_UNEXPECTED(VecLoad)
TGREF_UNEXPECTED(VecPointwiseMult)
TGREF_UNEXPECTED(VecMAXPY)
TGREF_UNEXPECTED(VecSetSizes)
TGREF_UNEXPECTED(VecSetFromOptions)
TGREF_UNEXPECTED(MatCreate)
TGREF_UNEXPECTED(MatSetSizes)
TGREF_UNEXPECTED(MatSetType)
TGREF_UNEXPECTED(MatSetFromOptions)
TGREF_UNEXPECTED(MatSetValues)
TGREF_UNEXPECTED(MatSetOption)
TGREF_UNEXPECTED(MatAssemblyBegin)
TGREF_UNEXPECTED(MatAssemblyEnd)
TGREF_UNEXPECTED(MatZeroEntries)
TGREF_UNEXPECTED(MatMPIAIJSetPreallocation)
TGREF_UNEXPECTED(MatSetNullSpace)
TGREF_UNEXPECTED(MatNullSpaceCreate)
TGREF_UNEXPECTED(MatCreateShell)
TGREF_UNEXPECTED(MatShellSetOperation)
TGREF_UNEXPECTED(MatShellGetContext)
TGREF_UNEXPECTED(MatCreateSNESMF)
TGREF_UNEXPECTED(MatMFFDSetType)
TGREF_UNEXPECTED(MatDestroy)
TGREF_UNEXPECTED(KSPCreate)
TGREF_UNEXPECTED(KSPSetType)
TGREF_UNEXPECTED(KSPSetOperators)
TGREF_UNEXPECTED(KSPSetTolerances)
TGREF_UNEXPECTED(KSPGetPC)
TGREF_UNEXPECTED(KSPSetPCSide)
TGREF_UNEXPECTED(KSPSetFromOptions)
TGREF_UNEXPECTED(KSPSetUp)
TGREF_UNEXPECTED(KSPSolve)
TGREF_UNEXPECTED(KSPDestroy)
TGREF_UNEXPECTED(KSPGMRESSetRestart)
TGREF_UNEXPECTED(KSPBCGSLSetEll)
TGREF_UNEXPECTED(KSPGetResidualNorm)
TGREF_UNEXPECTED(KSPGetIterationNumber)
TGREF_UNEXPECTED(KSPSetInitialGuessNonzero)
TGREF_UNEXPECTED(KSPMonitorSet)
TGREF_UNEXPECTED(KSPMonitorTrueResidualNorm)
TGREF_UNEXPECTED(PCSetType)
TGREF_UNEXPECTED(PCMGSetType)
TGREF_UNEXPECTED(PCGAMGSetNSmooths)
TGREF_UNEXPECTED(SNESCreate)
TGREF_UNEXPECTED(SNESSetType)
TGREF_UNEXPECTED(SNESSetFunction)
TGREF_UNEXPECTED(SNESSetJacobian)
TGREF_UNEXPECTED(SNESSetTolerances)
TGREF_UNEXPECTED(SNESSetMaxNonlinearStepFailures)
TGREF_UNEXPECTED(SNESSetMaxLinearSolveFailures)
TGREF_UNEXPECTED(SNESMonitorSet)
TGREF_UNEXPECTED(SNESKSPSetUseEW)
TGREF_UNEXPECTED(SNESKSPSetParametersEW)
TGREF_UNEXPECTED(SNESGetLinearSolveIterations)
TGREF_UNEXPECTED(SNESGetKSP)
TGREF_UNEXPECTED(SNESGetIterationNumber)
TGREF_UNEXPECTED(SNESGetFunctionNorm)
TGREF_UNEXPECTED(SNESSolve)
TGREF_UNEXPECTED(SNESSetFromOptions)
TGREF_UNEXPECTED(SNESDestroy)
TGREF_UNEXPECTED(PetscSFCreate)
TGREF_UNEXPECTED(PetscSFSetGraph)
TGREF_UNEXPECTED(PetscSFBcastBegin)
TGREF_UNEXPECTED(PetscSFBcastEnd)
TGREF_UNEXPECTED(PetscSFDestroy)
TGREF_UNEXPECTED(PetscSFSetUp)
TGREF_UNEXPECTED(MPI_Type_contiguous)
TGREF_UNEXPECTED(MPI_Type_commit)
TGREF_UNEXPECTED(MPI_Type_free)
TGREF_UNEXPECTED(MPI_Type_create_struct)
TGREF_UNEXPECTED(MPI_Get_address)
TGREF_UNEXPECTED(MPI_Allgather)
TGREF_UNEXPECTED(MPI_Alltoall)
TGREF_UNEXPECTED(MPI_Alltoallv)
TGREF_UNEXPECTED(HYPRE_BoomerAMGCreate)
TGREF_UNEXPECTED(HYPRE_BoomerAMGDestroy)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetTol)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetStrongThreshold)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetSmoothType)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetSmoothNumSweeps)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetRelaxWt)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetRelaxType)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetPrintLevel)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetMaxIter)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetLevelOuterWt)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetInterpType)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetCycleType)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetCycleNumSweeps)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetCoarsenType)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetAggNumLevels)
TGREF_UNEXPECTED(HYPRE_BoomerAMGSetNumSweeps)
TGREF_UNEXPECTED(HYPRE_ParCSRGMRESCreate)
TGREF_UNEXPECTED(HYPRE_ParCSRGMRESDestroy)
TGREF_UNEXPECTED(HYPRE_ParCSRGMRESSetKDim)
TGREF_UNEXPECTED(HYPRE_ParCSRPCGCreate)
TGREF_UNEXPECTED(HYPRE_ParCSRPCGDestroy)
TGREF_UNEXPECTED(HYPRE_PCGSetTwoNorm)
TGREF_UNEXPECTED(HYPRE_PCGSetTol)
TGREF_UNEXPECTED(HYPRE_PCGSetPrintLevel)
TGREF_UNEXPECTED(HYPRE_PCGSetPrecond)
TGREF_UNEXPECTED(HYPRE_PCGSetMaxIter)
TGREF_UNEXPECTED(HYPRE_PCGSetLogging)
TGREF_UNEXPECTED(HYPRE_GMRESSetTol)
TGREF_UNEXPECTED(HYPRE_GMRESSetPrintLevel)
TGREF_UNEXPECTED(HYPRE_GMRESSetPrecond)
TGREF_UNEXPECTED(HYPRE_GMRESSetMaxIter)
TGREF_UNEXPECTED(HYPRE_GMRESSetLogging)

#endif
