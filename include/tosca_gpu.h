/*
 * tosca_gpu.h -- C-ABI of the B200 fractional-step time step for TOSCA.
 *
 * One context owns one single-domain DMDA-shaped grid on one GPU. Every array
 * that crosses this boundary is a caller-owned HOST array laid out exactly like
 * TOSCA's PETSc DMDA arrays: [k][j][i] with i fastest, vectors as interleaved
 * Cmpnts {x,y,z} triples (base.h:80-84), scalars as PetscReal (double). The
 * extent is either the global DMDA extent (mx,my,mz) -- halo = 0 -- or the
 * single-rank local ghosted extent (mx+2h, my+2h, mz+2h) that DMDAVecGetArray
 * on a local Vec exposes -- halo = h (TOSCA uses h = 3, mesh.c:42).
 *
 * The entry points replace the stage functions that TOSCA's time loop calls
 * (src/main.c:54-327). Each declaration names the reference function it
 * stands in for. All calls return a tg_status (0 = success) and never exit,
 * abort or trap; the text of the last error is available from
 * tg_last_error(). A context is used by one host thread at a time.
 *
 * The same declarations, with the prefix "tor_" instead of "tg_", are exported
 * by the CPU restatement used as the parity checker (oracle/); both libraries
 * consume the tg_config structure below.
 */
#ifndef TOSCA_GPU_H
#define TOSCA_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status -- */
typedef enum tg_status {
    TG_OK                = 0,
    TG_ERR_CUDA          = 1,  /* a CUDA runtime call failed                      */
    TG_ERR_BAD_ARG       = 2,  /* invalid argument or unsupported configuration   */
    TG_ERR_NOT_CONVERGED = 3,  /* Poisson solve hit its iteration cap             */
    TG_ERR_NAN           = 4,  /* non-finite value detected in the state          */
    TG_ERR_ALLOC         = 5,  /* device or host allocation failed                */
    TG_ERR_STATE         = 6   /* call out of order (e.g. step before mesh)       */
} tg_status;

/* ---------------------------------------------------- boundary patch types -- */
/* Velocity patch types (boundary/U). Periodic means TOSCA's periodic type 2
 * (DM_BOUNDARY_PERIODIC, ghost cells at -2 / m+1: mesh.c:129-136). */
enum {
    TG_BC_PERIODIC        = 0,
    TG_BC_NOSLIP          = 1,  /* "noSlip"                                        */
    TG_BC_SLIP            = 2,  /* "slip"                                          */
    TG_BC_WALL_SHUMANN    = 3,  /* "velocityWallFunction" type -3 (jLeft only)     */
    /* patch type 0 (not a wall, checkBCsAndSetPatchTypes boundary.c:321-350):
     * the boundary face flux is interpolated from the ghost and first cells
     * (UpdateContravariantBCs boundary.c:651-689), and the outflow faces of
     * all such patches take the mass imbalance (adjustFluxesLocal,
     * ueqn.c:748-1135, at the end of the momentum solve); explicit schemes
     * (TG_DDT_FE, TG_DDT_RK4) only, no adjoint                                  */
    TG_BC_FIXED_VALUE     = 4,  /* "fixedValue": ghost cell = bc_value of the      */
                                /* patch (boundary.c:1632-1673), an inflow          */
    TG_BC_ZERO_GRADIENT   = 5,  /* "zeroGradient": ghost 2 U(1) - U(2)             */
                                /* (boundary.c:1897-1970), reverse flow through the */
                                /* face set to zero (boundary.c:718-741), an outflow */
    TG_BC_INLET_LOG       = 6   /* "inletFunction" type 2 on kLeft only: log-law    */
                                /* ghost (uTau/0.4) ln(h/z0) Udir, h the first      */
                                /* cell's height above the ground, constant above   */
                                /* hInv (boundary.c:1253-1283), an inflow           */
};
/* eddy-viscosity patch types (boundary/nut) */
enum {
    TG_NUTBC_PERIODIC     = 0,
    TG_NUTBC_ZEROGRADIENT = 1,
    TG_NUTBC_FIXEDVALUE   = 2
};
/* -divScheme (ueqn.c:82-110) */
enum { TG_DIV_CENTRAL = 0, TG_DIV_QUICK = 1 };
/* -dUdtScheme (ueqn.c:123-323): explicit (FE, RK4), Crank-Nicolson (CN,
 * UeqnSNES) and the implicit-explicit schemes with a Crank-Nicolson viscous
 * part solved by GMRES on the shell operator IMEXMatVec
 * (ueqn_solvers.c:1508-1799): ABCN (Adams-Bashforth 2 convection), RK3WCN
 * (Wray low-storage RK3) and RK3SOCN (Shu-Osher TVD RK3) */
enum { TG_DDT_FE = 0, TG_DDT_RK4 = 1, TG_DDT_CN = 2, TG_DDT_ABCN = 3, TG_DDT_RK3WCN = 4, TG_DDT_RK3SOCN = 5 };
/* arithmetic of the step */
enum {
    TG_PREC_FP64  = 0,   /* every stage in FP64                                   */
    TG_PREC_MIXED = 1    /* FP32 stencils/RHS/multigrid inside an FP64 outer loop */
};

/* patch order used by every 6-entry array below */
enum { TG_ILEFT = 0, TG_IRIGHT = 1, TG_JLEFT = 2, TG_JRIGHT = 3, TG_KLEFT = 4, TG_KRIGHT = 5 };

/* ------------------------------------------------------------ configuration -- */
/* temperature patch types (boundary/T, UpdateTemperatureBCs boundary.c:2052-2616);
 * TG_TBC_WALL_FUNCTION is thetaWallFunction, jLeft only (see t_wall_type) */
enum { TG_TBC_ZERO_GRADIENT = 0, TG_TBC_FIXED_VALUE = 1, TG_TBC_FIXED_GRADIENT = 2, TG_TBC_PERIODIC = 3,
       TG_TBC_WALL_FUNCTION = 4 };
/* thetaWallFunction types (boundary/T "type", boundary.c:5110-5180) */
enum { TG_TWALL_FIXED_FLUX = -2, TG_TWALL_SHUMANN = -3, TG_TWALL_SURFACE_SERIES = -4 };
/* -dTdtScheme (teqn.c:66-230): explicit RK4; ABBE (Adams-Bashforth 2
 * convection, backward-Euler diffusion solved by GMRES on ABBEMatVec,
 * teqn_solvers.c:821-945); BE and BDF2 (implicit, Newton-Krylov on
 * SNESFuncEvalT, teqn_solvers.c:596-712) */
enum { TG_TDDT_RK4 = 0, TG_TDDT_ABBE = 1, TG_TDDT_BE = 2, TG_TDDT_BDF2 = 3 };

typedef struct tg_config {
    int32_t mx, my, mz;            /* DMDA extent incl. the one-cell physical ghost layer  */
    int32_t bc[6];                 /* velocity patch types, TG_ILEFT..TG_KRIGHT order       */
    int32_t nut_bc[6];             /* eddy-viscosity patch types                            */
    double  nut_bc_value[6];       /* value for TG_NUTBC_FIXEDVALUE patches                 */
    int32_t curvilinear;           /* -meshFileType curvilinear (wall-stress branch)        */
    int32_t les;                   /* -les 1: Smagorinsky eddy viscosity                    */
    double  cs;                    /* Smagorinsky constant as applied to (vol^(1/3))^2|S|;  */
                                   /* the reference hard-codes 0.0289 (les.c:10,175)        */
    double  nu;                    /* -nu                                                   */
    int32_t div_scheme;            /* TG_DIV_*                                              */
    int32_t ddt_scheme;            /* TG_DDT_*                                              */
    double  dt;                    /* -timeStep (fixed)                                     */
    int32_t buoyancy;              /* -potentialT 1 with a frozen temperature field         */
    double  t_ref;                 /* -tRef                                                 */
    int32_t mean_grad_p;           /* -meanGradPForce 1                                     */
    double  mean_grad_p_value[3];  /* -dpdx_mean, -dpdy_mean, -dpdz_mean                    */
    double  wall_roughness;        /* velocityWallFunction kRough                           */
    double  wall_kappa;            /* velocityWallFunction kappa                            */
    double  poisson_rtol;          /* relative residual tolerance of the pressure solve     */
    double  poisson_div_tol;       /* >0: also stop once dt*max|r*aj| <= this (div bound)   */
    int32_t poisson_maxit;         /* iteration cap of the pressure solve                   */
    int32_t precision;             /* TG_PREC_*                                             */
    int32_t it_start;              /* clock->itStart                                        */
    int32_t device;                /* CUDA device ordinal (ignored by the CPU restatement)  */
    int32_t source;                /* body force TG_F_SOURCE added by sourceU               */
                                   /* (ueqn_sources.c:2884-2980, ueqn_solvers.c:1369)       */
    /* temperature transport (SolveTEqn, teqn.c:259; scheme t_ddt_scheme,
     * independent of ddt_scheme): with teqn = 1 the temperature TG_F_TMPRT is
     * advanced after the projection and the buoyancy of the next step reads it */
    int32_t teqn;
    int32_t t_bc[6];               /* TG_TBC_* per patch (periodic where bc is periodic)    */
    double  prandtl;               /* -Pr: molecular Prandtl number (no LES)                */
    double  t_bc_value[6];         /* fixedValue: ghost value; fixedGradient: gradient      */
    /* Crank-Nicolson momentum solve (TG_DDT_CN; -absTolU, -relTolU, -snesMaxItersU,
     * ueqn.c:128-138): stop at |F| <= max(snes_atol, snes_rtol |F_0|). The
     * IMEX schemes stop their GMRES at |r| <= max(snes_atol, snes_rtol |b|)
     * (KSPSetTolerances(kspIMEX, relTolU, absTolU, 1e30, 1000), ueqn.c:282) */
    double  snes_atol;
    double  snes_rtol;
    int32_t snes_maxit;
    int32_t gmres_restart;         /* -kspGMRESRestartU (ueqn.c:233), 0 = 30                */
    /* temperature scheme (teqn = 1): TG_TDDT_*; ABBE's GMRES stops at
     * |r| <= max(t_rtol |b|, t_atol) (-relTolT, -absTolT, defaults 1e-30, 1e-5)
     * or 1000 iterations, restart -kspGMRESRestartT (0 = 30); BE/BDF2 stop
     * their Newton iteration at |F| <= max(t_atol, t_rtol |F_0|) or 20 steps */
    int32_t t_ddt_scheme;
    int32_t t_gmres_restart;
    double  t_atol;
    double  t_rtol;
    /* -pTildeBuoyancy 1 (teqn.c:38-57): the buoyancy term is ghGradRhoK,
     * g z grad((tRef - T)/tRef) at the faces (teqn.c:278-652), in place of
     * Buoyancy; needs buoyancy = 1 */
    int32_t p_tilde;
    /* initial guess of each pressure solve: 0 the previous solution (the
     * reference's, peqn.c:3885), 1 its linear, 2 (default) its quadratic
     * extrapolation from the previous two or three solutions; -1 = 2 */
    int32_t poisson_guess;
    /* thetaWallFunction on the jLeft temperature patch (t_bc[TG_JLEFT] =
     * TG_TBC_WALL_FUNCTION; needs teqn = 1 and les = 1). UpdateWallModelsT
     * (boundary.c:3858-4178) sets the wall heat flux qWall of the j = 0
     * faces, which FormT applies in place of the diffusive flux
     * (teqn_solvers.c:337-352); the ghost temperature is zero-gradient.
     * t_wall_type TG_TWALL_SHUMANN (-3): Schumann-Grotzbach with Monin-Obukhov
     * stability (qWallShumann, wallfunctions.c:133-290) from the difference
     * between the first-cell temperature and a surface temperature that starts
     * at the wall value and rises by t_wall_heating_rate * dt every step;
     * t_wall_localized 0 ("averaged") evaluates it once from plane means,
     * 1 ("localized") per wall cell. TG_TWALL_FIXED_FLUX (-2): qWall =
     * t_wall_qwall everywhere. TG_TWALL_SURFACE_SERIES (-4): as -3, with the
     * surface temperature interpolated in time from the series given by
     * tg_set_surface_temperature (findInterpolationWeights,
     * inline.h:5873-5940) at the clock time of the step, t_start +
     * (it - it_start + 1) dt (fixed time step, clock.c:347-367), and from
     * the second step on the ghost temperature 2 T_s - T(j=1) on the ground
     * (boundary.c:2390-2411). */
    int32_t t_wall_type;
    int32_t t_wall_localized;
    double  t_wall_qwall;          /* -2: heat flux (K m/s)                                  */
    double  t_wall_heating_rate;   /* -3: heatingRate (K/s)                                  */
    double  t_wall_kappa;          /* -3: kappa                                              */
    double  t_wall_theta_ref;      /* -3: thetaRef (K)                                       */
    double  t_wall_roughness;      /* -3: kRough (m)                                         */
    double  t_wall_gamma_m;        /* -3: gammaM                                             */
    double  t_wall_gamma_h;        /* -3: gammaH                                             */
    double  t_wall_alpha_h;        /* -3: alphaH                                             */
    /* stability correction of the velocity wall function -3 (uStarShumann,
     * wallfunctions.c:12-130, boundary.c:3336-3420): with a thetaWallFunction
     * on the temperature jLeft patch, the plane mean of its qWall enters the
     * friction velocity; gammaM and thetaRef of velocityWallFunction */
    double  wall_gamma_m;
    double  wall_theta_ref;
    double  t_start;               /* -startTime: clock time at it_start (thetaWallFunction -4) */
    double  bc_value[18];          /* TG_BC_FIXED_VALUE: Cartesian velocity (x, y, z) of  */
                                   /* patch p at [3p, 3p+2] (boundaryU *val, boundary.c)  */
    /* TG_BC_INLET_LOG (inletFunction type 2, boundary/U): uTau, roughness,
     * hInv (the profile is constant above it) and the unit direction Udir */
    double  inlet_u_tau;
    double  inlet_z0;
    double  inlet_h_inv;
    double  inlet_dir[3];
} tg_config;

/* per-call statistics */
typedef struct tg_stats {
    int64_t steps;                 /* steps completed by this call                          */
    int32_t poisson_iterations;    /* Krylov iterations of the last pressure solve          */
    int32_t poisson_total_iterations; /* summed over the steps of this call                 */
    double  poisson_initial_residual;
    double  poisson_final_residual;/* relative L2 residual of the last solve                */
    double  max_divergence;        /* ContinuityErrorsOptimized value after the last step   */
    double  seconds;               /* device (or CPU) time of this call                     */
} tg_stats;

typedef struct tg_ctx tg_ctx;

/* metric / field selectors for tg_get_field / tg_set_field */
enum {
    TG_F_CENT = 0, TG_F_CSI, TG_F_ETA, TG_F_ZET,
    TG_F_ICSI, TG_F_IETA, TG_F_IZET, TG_F_JCSI, TG_F_JETA, TG_F_JZET,
    TG_F_KCSI, TG_F_KETA, TG_F_KZET,                                    /* vectors (3 doubles) */
    TG_F_AJ, TG_F_IAJ, TG_F_JAJ, TG_F_KAJ,                              /* scalars             */
    TG_F_UCONT, TG_F_UCAT, TG_F_UCONT_O, TG_F_RHS, TG_F_DP, TG_F_BTHETA,/* vectors             */
    TG_F_P, TG_F_PHI, TG_F_NUT, TG_F_TMPRT,                             /* scalars             */
    TG_F_TAUWALL,                                                       /* vector, j=0 plane   */
    TG_F_SOURCE,                  /* vector: cell-centred Cartesian body force (ueqn->sourceU) */
    /* adjoint fields of tg_adjoint_*: adjoints of Ucont, Ucat, P and the
     * gradient of the objective with respect to TG_F_SOURCE */
    TG_F_UCONT_ADJ, TG_F_UCAT_ADJ, TG_F_P_ADJ, TG_F_SOURCE_ADJ,
    /* turbine body force of the last step (read only, with turbines set):
     * projected Cartesian force (lsourceFarmCat) and its face values
     * (sourceFarmCont) */
    TG_F_FARM_FORCE, TG_F_FARM_CONT,
    /* adjoint of the state of the Schumann wall model (the time-filtered
     * wall-parallel velocity and the running mean of its magnitude,
     * boundary.c:3490-3520), a plane of (mz x mx) triples (filtered x, filtered
     * y, running mean); carried from one reversed step to the one before */
    TG_F_WALL_ADJ,
    /* thetaWallFunction state, planes of (mz x mx) scalars: the wall heat
     * flux qWall of the last UpdateWallModelsT and the surface temperature of
     * the -3 model (set by the first step from the wall value unless written) */
    TG_F_QWALL, TG_F_SURF_THETA,
    TG_F_COUNT
};

/* ----------------------------------------------------------------- lifecycle -- */
/* Replaces simulationInitialize's per-domain allocation (initialization.h:39 /
 * initialization.c:63) and the solver set-up of InitializeUEqn / InitializePEqn
 * (ueqn.h:92, peqn.h:58). */
tg_status tg_create(const tg_config *cfg, tg_ctx **out);
tg_status tg_destroy(tg_ctx *ctx);
const char *tg_last_error(const tg_ctx *ctx);
const char *tg_status_string(tg_status s);

/* Grid nodes (AoS xyz, global extent, node (k,j,i) at DMDA point (k,j,i) for
 * k<mz-1, j<my-1, i<mx-1; mesh.c:34-447). Computes all cell and face metrics on
 * the device: replaces SetMeshMetrics (mesh.h:94 / mesh.c:630-1976) and the
 * connectivity and matrix of SetPoissonConnectivity / SetCoeffMatrix
 * (peqn.h:115,118 / peqn.c:107-248, 703-1501), which become a matrix-free
 * operator and its multigrid hierarchy. */
tg_status tg_set_mesh_nodes(tg_ctx *ctx, const double *nodes);

/* Generic field transfer (global extent if halo = 0, local ghosted if halo > 0).
 * Vectors are AoS triples. Used to hand over TOSCA's own metrics and state
 * (DMDAVecGetArray pointers) and to read results back. */
tg_status tg_set_field(tg_ctx *ctx, int32_t which, const double *host, int32_t halo);
tg_status tg_get_field(tg_ctx *ctx, int32_t which, double *host, int32_t halo);
/* A field in TOSCA's field-file format (readFields / writeFields, io.c:247-420,
 * 2261): PETSc binary VecView of the DMDA vector, big-endian, header of two
 * 64-bit integers (class id 1211214, entry count) then the entries in natural
 * order over the whole DMDA extent (components interleaved for vectors). The
 * reader also accepts the 32-bit-integer header of a PETSc build without
 * 64-bit indices; a wrong class id or entry count returns TG_ERR_BAD_ARG. */
tg_status tg_write_field_petsc(tg_ctx *ctx, int32_t which, const char *path);
tg_status tg_read_field_petsc(tg_ctx *ctx, int32_t which, const char *path);

/* Cartesian cell velocity -> ghost cells -> face fluxes. Replaces the common
 * tail of SetTaylorGreenFieldU / SetABLInitialFlowU (initialField.c:1100-1204):
 * Ucat interior, UpdateCartesianBCs, face interpolation, UpdateContravariantBCs. */
tg_status tg_init_from_cartesian(tg_ctx *ctx, const double *ucat, int32_t halo);

/* ------------------------------------------------------------------ stages -- */
/* Each replaces one reference function: declaration (header) / definition. */
tg_status tg_contravariant_to_cartesian(tg_ctx *ctx);  /* ueqn.h:98 / ueqn.c:528-635              */
tg_status tg_update_nut(tg_ctx *ctx);                  /* les.h:73,76 / les.c:165-180,2119-2578    */
tg_status tg_update_wall_models(tg_ctx *ctx);          /* boundary.h:188 / boundary.c:3257-3600    */
tg_status tg_grad_p(tg_ctx *ctx);                      /* peqn.h:109 / peqn.c:3437-3773            */
tg_status tg_buoyancy(tg_ctx *ctx);                    /* ueqn_sources.h:23 / ueqn_sources.c:2726  */
/* with teqn = 1 (TG_ERR_STATE otherwise): the jLeft thetaWallFunction's
 * qWall (TG_F_QWALL, TG_F_SURF_THETA) and the temperature ghost cells */
tg_status tg_update_wall_models_t(tg_ctx *ctx);        /* boundary.h:191 / boundary.c:3858-4520    */
tg_status tg_update_temperature_bcs(tg_ctx *ctx);      /* boundary.h:170 / boundary.c:2052-2616    */
/* the surface temperature series of thetaWallFunction -4: n >= 2 times and
 * temperatures (the reference reads them from inflowDatabase/mesoscaleData,
 * readSurfaceTempData boundary.c:5269-5400); copied, kept until replaced */
tg_status tg_set_surface_temperature(tg_ctx *ctx, int32_t n, const double *time, const double *temp);
/* Rhs (TG_F_RHS) += scale * FormU on the current lUcont/lUcat/nut:
 * ueqn_solvers.h:15 / ueqn_solvers.c:6-1083 with formMode 0. Rhs is
 * zeroed first when zero_rhs. */
tg_status tg_form_u(tg_ctx *ctx, double scale, int32_t zero_rhs);
tg_status tg_explicit_rhs(tg_ctx *ctx);                /* ueqn_solvers.h:24 / ueqn_solvers.c:1276  */
tg_status tg_solve_u(tg_ctx *ctx);                     /* ueqn.h:107 / ueqn.c:397-440 (FE, RK4)    */
tg_status tg_solve_p(tg_ctx *ctx, tg_stats *stats);    /* peqn.h:142 / peqn.c:3777-3971            */
tg_status tg_continuity_error(tg_ctx *ctx, double *max_div); /* peqn.h:148 / peqn.c:4114-4181      */
/* Allocation-free form of the divergence check; no counterpart in the
 * reference. For callers that cannot allocate device memory: code running
 * while a stream is captured into a CUDA graph (cudaMalloc is not allowed
 * there), hosts whose device memory belongs to a fixed pool or framework
 * allocator that must stay the only allocator, and loops that cannot absorb
 * the device synchronisation of cudaMalloc/cudaFree. Computes the same value
 * as tg_continuity_error, max over interior cells of |div(Ucont)| * aj, from
 * caller-owned DEVICE arrays of the global extent (ucont AoS triples, aj
 * scalars) on the caller's current device, and writes it to the device
 * scalar *max_div on `stream` (a cudaStream_t; NULL = default stream). No
 * context is needed and nothing is allocated: the per-plane partial maxima
 * live in a file-scope device array of 16384 doubles (128 KiB) that every GPU
 * loading the library holds until exit, so mz - 2 <= 16384 interior planes;
 * larger grids return TG_ERR_BAD_ARG. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and should come before any
 * stream capture. All calls share the array: calls that overlap on one GPU
 * race and must be serialised by the caller. */
tg_status tg_continuity_error_noalloc(const double *ucont, const double *aj, int32_t mx, int32_t my,
                                      int32_t mz, double *max_div, void *stream);
tg_status tg_update_cartesian_bcs(tg_ctx *ctx);        /* boundary.h:167 / boundary.c:824-2050     */
tg_status tg_update_contravariant_bcs(tg_ctx *ctx);    /* boundary.h:164 / boundary.c:614-822      */
tg_status tg_sync_pressure(tg_ctx *ctx);               /* overset.h:107 / overset.c:263-315        */

/* nsteps full time steps in the order of main.c:54-327 (fixed dt). */
tg_status tg_step(tg_ctx *ctx, int32_t nsteps, tg_stats *stats);

/* Step replay (default on; no reference counterpart): from the second step on,
 * a step is captured once into a CUDA graph whose pressure-solver loop runs
 * under device-side control, and replayed after that, with the same
 * arithmetic as the step launched kernel by kernel. With
 * it on, tg_step runs every requested step (a non-finite residual is reported
 * at the end of the call rather than stopping it). on = 0 launches every step
 * kernel by kernel, as profiling and taping do. */
tg_status tg_set_graphs(tg_ctx *ctx, int32_t on);
/* Steps replayed from the captured graph since the context was created, and
 * whether capture failed for this configuration (steps then run kernel by
 * kernel). */
tg_status tg_graph_info(tg_ctx *ctx, int64_t *replays, int32_t *capture_failed);
/* Iterations of the last implicit momentum solve (CN, ABCN, RK3WCN, RK3SOCN):
 * outer = Newton steps (CN) or Runge-Kutta stages solved (IMEX); inner =
 * operator products of the Krylov solver (the KSPGetIterationNumber values,
 * summed); residual = the last Krylov residual estimate (KSPGetResidualNorm,
 * ueqn_solvers.c:1560-1561). Zeros after an explicit step. */
tg_status tg_momentum_info(tg_ctx *ctx, int32_t *outer, int32_t *inner, double *residual);
/* How the kernels classified the mesh set by tg_set_mesh_nodes: orthogonal
 * (every cross term of the face metric tensor is zero: 7-point pressure
 * operator, conjugate gradients) and axis-aligned (csi || y, eta || z,
 * zet || x up to round-off: the stencil kernels read one component of each
 * metric vector). */
tg_status tg_mesh_info(tg_ctx *ctx, int32_t *orthogonal, int32_t *axis_aligned);

/* --------------------------------------------------------------- wind farm -- */
/* Uniform actuator-disk turbines: TOSCA's "uniformADM" with sampleType
 * rotorDisk and CtType constant (a disk-based thrust coefficient C_T', axial
 * induction 0). Per step, after the eddy viscosity (main.c:146,
 * UpdateWindTurbines turbines.c:39-170): the velocity is sampled at the disk
 * points by trilinear interpolation (turbines_sampling.c:174-262,
 * inline.h:6904-7265), the disk-averaged in-plane speed U gives the point
 * forces 0.5 U^2 dA C_T' along the axis (turbines_force.c:219-383), a
 * Gaussian projection spreads them to the cells (turbines_force.c:858-910)
 * and their central face values times the face areas
 * (bodyForceCartesian2Contravariant, turbines_force.c:1741-1835) are added to
 * the momentum right-hand side of every stage (ueqn_solvers.c:1340-1344).
 * Disk points follow turbines_io.c:1925-2000 with zero tilt and precone;
 * projection cells are the interior cells within r_tip + 2.628 epsilon of the
 * centre (turbines_parallel.c:40-135). */
typedef struct tg_turbine {
    double center[3];        /* rotor centre (x, y, z), mesh coordinates              */
    double axis[3];          /* rotor axis, pointing upstream (rtrDir)                */
    double up[3];            /* azimuth-zero direction of the disk points (twrDir)    */
    double r_tip, r_hub;     /* tip and hub radius (r_hub > 0)                        */
    double epsilon;          /* width of the Gaussian projection                      */
    double ct;               /* C_T'                                                  */
    int32_t n_radial, n_azimuth;
} tg_turbine;

/* Define the farm (after tg_set_mesh_nodes); n = 0 removes it. rho: air
 * density of thrust and power (the body force is per unit density). */
tg_status tg_set_turbines(tg_ctx *ctx, int32_t n, const tg_turbine *turbines, double rho);
/* Change the C_T' of every turbine (n values) without rebuilding the geometry. */
tg_status tg_set_turbine_ct(tg_ctx *ctx, const double *ct);
/* Values of the last step per turbine (n each; any pointer may be NULL): disk
 * speed U, thrust rho sum(B . axis), power thrust U; power_sum: the farm power
 * summed over the steps since the last reset (reset != 0 zeroes it after the
 * read). */
tg_status tg_turbine_state(tg_ctx *ctx, double *uref, double *thrust, double *power,
                           double *power_sum, int32_t reset);

/* ----------------------------------------------------------------- adjoint -- */
/* Discrete adjoint of tg_step. No counterpart in the reference: TOSCA has no
 * adjoint. Adjoint fields are exchanged with tg_set_field / tg_get_field
 * (TG_F_UCONT_ADJ, TG_F_UCAT_ADJ, TG_F_P_ADJ: adjoints of Ucont, of the full
 * Ucat array and of P; TG_F_SOURCE_ADJ: gradient with respect to the body
 * force TG_F_SOURCE, accumulated). Supported: orthogonal grids, FE and RK4,
 * central and QUICK convection, constant or Smagorinsky viscosity, noSlip /
 * slip / periodic patches; anything else returns TG_ERR_BAD_ARG. */
typedef struct tg_adjoint_stats {
    int64_t steps;                 /* steps reversed                                        */
    int64_t forward_steps;         /* forward steps run by the reversal (recomputation)     */
    int32_t snapshots;             /* device snapshots of the checkpoint schedule           */
    int32_t poisson_iterations;    /* Krylov iterations of the transposed pressure solves   */
    double  seconds;               /* device time of the call                               */
} tg_adjoint_stats;

/* Farm adjoint: the gradient of a functional with respect to the C_T' of the
 * turbines accumulates in every reversed step (the farm forces enter each
 * step). With the power objective on, each reversed step also adds the
 * derivatives of the farm power at the step's start state, so that a
 * reversal seeded with zero adjoint fields yields the gradient of the farm
 * power summed over the steps (tg_turbine_state's power_sum). */
tg_status tg_set_farm_objective(tg_ctx *ctx, int32_t on);
/* d(functional)/dC_T' per turbine (n values); reset != 0 zeroes it after the read. */
tg_status tg_ct_gradient(tg_ctx *ctx, double *grad, int32_t reset);

/* Vector-Jacobian product of one step: the context holds the state at the
 * start of a step and the adjoint fields hold the adjoints of the state after
 * it; on return they hold the adjoints of the state before it, the body-force
 * gradient has the step's contribution added, and the state is again the one
 * at the start of the step (the step is re-run once to record its stages). */
tg_status tg_adjoint_step(tg_ctx *ctx);
/* nsteps forward steps from the current state with checkpointing in at most
 * nsnap device snapshots; leaves the final state in the context (to seed the
 * adjoint fields from it). The reversal re-runs forward steps from the
 * snapshots to record their stages (tapes). With nsnap >= nsteps and room in
 * device memory every step's tape is kept and nothing is re-run. Otherwise,
 * when tapes of k >= 2 steps fit (see tg_adjoint_set_tapes) and ceil(nsteps/k)
 * snapshots suffice, snapshots are kept every k steps and the reversal re-runs
 * each segment once, taped, before reversing it (every step runs forward once
 * in the reversal); else a binomial (revolve) schedule over the snapshots. */
tg_status tg_adjoint_forward(tg_ctx *ctx, int32_t nsteps, int32_t nsnap, tg_stats *stats);
/* Cap on the step tapes the segment schedule of tg_adjoint_forward may hold:
 * -1 (default) as many as 60 % of the free device memory holds, 0 none (the
 * binomial schedule over the snapshots only), n > 0 at most n. No counterpart
 * in the reference (it has no adjoint). */
tg_status tg_adjoint_set_tapes(tg_ctx *ctx, int32_t max_tapes);
/* Reverse sweep over the steps of the last tg_adjoint_forward, from the adjoint
 * fields of the final state to those of the initial state; the context returns
 * to the initial state. */
tg_status tg_adjoint_reverse(tg_ctx *ctx, tg_adjoint_stats *stats);

/* One drop-in step with host state: Ucont, Ucat and P are uploaded from the
 * caller's arrays, one step runs, and the same arrays are overwritten with the
 * new state; nut (LES on) is only written, since the step recomputes it from
 * Ucat before any use (UpdateNut at the start of the step, main.c:54-99). This
 * is the call a host time loop makes when the state lives in its own (PETSc)
 * vectors. With teqn = 1 the temperature stays in the context between calls;
 * a host that keeps it in its own vector moves it with tg_set_field /
 * tg_get_field (TG_F_TMPRT) around the call. */
tg_status tg_step_host(tg_ctx *ctx, double *ucont, double *ucat, double *p,
                       double *nut, int32_t halo, tg_stats *stats);

#ifdef __cplusplus
}
#endif

#endif /* TOSCA_GPU_H */
