/*
 * flite_gpu.h -- C ABI of the B200 (sm_100a) flow-solver hot path.
 *
 * The Fortran solver host (SolverSource/mgnsg3d_mg_par.F90) drives the grid
 * solver module GridSolver (SolverSource/mgnsg3d_def_par.F90) through a small
 * set of module calls.  Each entry point below replaces one of those calls one
 * for one; the reference routine it replaces is cited beside it.  All arrays
 * cross the boundary as plain host pointers in the reference's own layout
 * (Fortran column-major, 1-based node indices), so a Fortran host can bind them
 * with ISO_C_BINDING without copies or reshapes (the interface module
 * include/flite_gpu_mod.f90 declares them for Fortran).
 *
 * Every function returns an int status (FLITE_OK on success).  The reference
 * STOPs on errors; this library returns a code and keeps a message that
 * flite_last_error() retrieves; with a NULL context it returns the message of
 * the calling thread's last failed flite_create or flite_batch_create.
 */
#ifndef FLITE_GPU_H
#define FLITE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define FLITE_OK            0
#define FLITE_EINVAL        1   /* bad argument, inconsistent mesh arrays   */
#define FLITE_EUNSUPPORTED  2   /* control value outside the supported path */
#define FLITE_ENAN          3   /* non-finite residual (mg_par:1464-1470)   */
#define FLITE_ETIMEOUT      4   /* a bounded device wait expired            */
#define FLITE_ECUDA         5   /* CUDA runtime error                       */
#define FLITE_ENOMEM        6   /* device allocation failed                 */
#define FLITE_EIO           7   /* file format / record error               */

/* ---- precision modes --------------------------------------------------- */
#define FLITE_FP64   0   /* every kernel in double precision                  */
#define FLITE_MIXED  1   /* FP32 fluxes/gradients/stages, FP64 accumulation   */

/*
 * Controls: a POD mirror of the InputVariablesData fields the hot path reads
 * (SolverSource/mgnsg3d_def_par.F90:64-196).  flite_controls_default() sets the
 * reference defaults (def_par:217-378); flite_controls_derive() applies the
 * post-read overrides and the freestream state (def_par:387-415).  Logical
 * fields are ints (0 = .false.).
 */
typedef struct flite_controls {
    /* freestream and physics */
    double MachNumber, alpha, beta, ReynoldsNumber, PrandtlNumber, gamma;
    double inflowTemperature, wallTemperature;
    int    wallsAreIsentropic;
    int    fluxType;            /* 1 central, 2 LLF, 3 Roe, 4 HLLC            */
    int    HLLCFluxOrder;
    double HLLCClipping;
    int    Automaticlipping;
    int    GradientMethod;      /* 1 Galerkin, else least squares            */
    int    dissipationScheme, coarseGridDissipationScheme;
    double secondOrderDissipationFactor, fourthOrderDissipationFactor;
    double coarseGridDissipationFactor;
    int    useMatrixDissipation;
    double HartensCorrectionFactor;
    int    useDissipationWeighting;
    int    viscosityScheme;
    int    boundaryTerm;
    /* time stepping and multigrid */
    double CFLNumber, turbulentCFLNumber, turbK, maxIncrementFactor, minimumDensity;
    int    multigridScheme, numberOfRelaxationSteps, numberOfGridsToUse;
    double multigridBCRelaxation, prolongationRelaxation, turbProlongationRelaxation;
    int    prolongationMappingScheme;
    int    numberOfMGIterations, maximumnumberofcycles, writeToFileInterval;
    double initialResidual;
    int    numberOfCFLIncrements;
    /* turbulence and bookkeeping */
    int    turbulenceModel, numberOfTurbulenceGrids, numberOfTurbulenceSteps;
    double tripFactor, triggerRadius, turbulenceTriggerValue;
    int    numberOfTriggerSteps;
    double maxTurbulenceValue, turbulentPrandtlNumber;
    double referenceArea, datum[3], groundplane;
    int    forceCalcType, restartNumber, numberOfProcesses;
    /* controls the path rejects unless they hold their steady default (SAS
     * and patchInitialization change nothing on this path, as in the
     * reference's solver; flowType and explicit_ are taken)                 */
    int    flowType, explicit_, SAS, GUSTMODEL, movingwall, patchInitialization, nspan;
    int    timeScheme, numberOfRSSteps, numberOfPSSteps;
    double residualSmoothingFactor, prolongationSmoothingFactor, physicalTimeStep;
    double engineBCRelaxation;
    /* engine boundary conditions (def_par:114-117, 182): the inlet mass flow
     * target of engines 1 and 2, the exhaust state (rho, rho u, rho v, rho w,
     * rho E, p, nu~) of each engine as enginesRearParameters(7,2) stored
     * column-major, and the cycles over which the exhaust state is ramped in
     * from the freestream                                                    */
    int    engineFlowType;      /* 1 mass flow, 2 mass flow function          */
    int    numberOfEORelaxationSteps;
    double enginesFrontMassFlow[2];
    double enginesRearParameters[14];
    /* derived: inflowField(1:6, 1:2) stored column-major as in def_par:88 */
    double inflowField[12];
    /* extension controls (no reference counterpart) */
    int    precision;           /* FLITE_FP64 | FLITE_MIXED                   */
    int    reconstruction;      /* FLITE_RECON_NONE | FLITE_RECON_VAN_ALBADA  */
    int    rungeKuttaStages;    /* 3 (the reference's 0.6, 0.6, 1) or 5       */
} flite_controls;

/*
 * The upwind extension (no reference counterpart).  FLITE_RECON_VAN_ALBADA
 * makes the Roe flux (fluxType 3) upwind on every level (the reference's
 * interior branch, def_par:1725-1792, subtracts its dissipation; the
 * extension adds it) and second order on level 1: the states of an
 * edge i1 -> i2 are reconstructed in (rho, u, v, w, rho E) from the Galerkin
 * node gradients (computeGradient, def_par:2923-3245) with the Van Albada
 * limiter,
 *     q_L = q1 + va(2 g1.d - dq, dq) / 2,   q_R = q2 - va(2 g2.d - dq, dq) / 2,
 *     va(a, b) = ab (a + b) / (a^2 + b^2) if ab > 0, else 0,
 * d = x2 - x1, dq = q2 - q1; an edge whose reconstructed density or pressure
 * is not positive keeps its first-order states.  Coarse levels stay first
 * order.  rungeKuttaStages 5 runs the stages with the coefficients
 * 1/4, 1/6, 3/8, 1/2, 1 in place of the reference's three.
 */
#define FLITE_RECON_NONE        0
#define FLITE_RECON_VAN_ALBADA  1

/*
 * One grid level as read from a gen3d .sol file (readGridComputationData,
 * def_par:13812-14074).  Pointers are host memory owned by the caller; the
 * library copies what it needs.  Index arrays are 1-based as in the file.
 */
typedef struct flite_level_desc {
    int32_t n_nodes;            /* N                                          */
    int32_t n_sides;            /* E interior edges                           */
    int32_t n_bsides;           /* B boundary edges                           */
    int32_t n_bnodes;           /* boundary nodes (numbered 1..n_bnodes)      */
    int32_t n_normals;          /* length of node_ind                         */
    const int32_t *side_idx;    /* [2][E] sideIndexArray(E,2)                 */
    const double  *side_w;      /* [3][E] sideWeightsArray(E,3)               */
    const double  *side_len;    /* [E]    sideLengthArray                     */
    const int32_t *bnd_idx;     /* [3][B] brp%sideIndexArray(B,3)             */
    const double  *bnd_w;       /* [3][B] brp%sideWeightsArray(B,3)           */
    const int32_t *node_reg;    /* [21]   nodeIndicatorRegister(-20:0)        */
    const int32_t *node_ind;    /* [n_normals] nodeIndicatorArray             */
    const double  *volume;      /* [N]    nodeVolume                          */
    const double  *wall_dist;   /* [N]    wallDistance (may be NULL)          */
    const double  *coords;      /* [3][N] coordinates (level 1; NULL coarse)  */
    const double  *coord_move;  /* [3][N] coordinateMovement (NULL = zero)    */
    const int32_t *parent;      /* [N_finer] prolongationArray (levels >= 2)  */
    const double  *rweight;     /* [N_finer] restrictionArray  (levels >= 2)  */
    /* moving meshes (flowType 2; NULL = static mesh): the records of the
     * step's .sol (def_par:800-818, 13855-13899)                             */
    const double  *side_gcl;    /* [2][E] GCLWeightsArray, the previous step's */
    const double  *bnd_gcl;     /* [4][B] brp%GCLWeightsArray(B,1:2), previous */
    const double  *volume_prev; /* [N]    nodeVolumeP  (level 1)              */
    const double  *volume_prev2;/* [N]    nodeVolumeP2 (level 1)              */
    /* engine inlet sides (def_par:852-864; 0 = none): per side its two nodes
     * and inlet number 1|2 as engineInletSideIndexes(n,3), its coefficient
     * vector as engineInletSideCoefficients(n,3)                              */
    int32_t n_engine_sides;
    const int32_t *engine_idx;  /* [3][n_engine_sides]                        */
    const double  *engine_w;    /* [3][n_engine_sides]                        */
} flite_level_desc;

typedef struct flite_ctx flite_ctx;

/* ---- controls --------------------------------------------------------- */
/* defaults of readInputVariables (def_par:217-378)                        */
int flite_controls_default(flite_controls *c);
/* post-read overrides + freestream (def_par:387-415)                      */
int flite_controls_derive(flite_controls *c);

/* ---- lifecycle -------------------------------------------------------- */
/* Replaces readComputationData (mg_par:1198-1268) + the allocations of
 * readGridComputationData and the geometry set-up it performs
 * (makeBoundaryNormals def_par:15394, makeSurfaceArea :15523, connectivity
 * count :14262-14275).  Copies every level to the current CUDA device.    */
int flite_create(const flite_controls *c, int nlevels,
                 const flite_level_desc *levels, flite_ctx **out);
int flite_destroy(flite_ctx *ctx);
int flite_last_error(const flite_ctx *ctx, char *buf, size_t len);

/* ---- state ------------------------------------------------------------ */
/* u is [nvar][N] column-major conserved variables (grp%u(N,nvar)),        */
/* nvar = 5 (+1 with Spalart-Allmaras).                                    */
int flite_set_state(flite_ctx *ctx, int level, const double *u);
int flite_get_state(flite_ctx *ctx, int level, double *u);
int flite_get_pressure(flite_ctx *ctx, int level, double *p);
/* Freestream start-up: setUpInitialField2 freestream branch (def_par:
 * 3878-3996) on level 1.  The restart branch (:3740-3873) is the host
 * reading .rst, converting to conserved and calling flite_set_state, then
 * flite_start.                                                             */
int flite_init_freestream(flite_ctx *ctx);
/* The start-up tail shared by both branches: makePressureField +
 * setBCsOnSolutionField on level 1 (def_par:3992-3994), laminar viscosity
 * and restriction of u to every coarse level (mg_par:586-602).             */
int flite_start(flite_ctx *ctx);

/* ---- solver steps (one per replaced Fortran call) --------------------- */
/* doTimeIterations (def_par:966-1000)                                     */
/* Unsteady runs (flowType 1 on a static mesh, 2 on a moving one; dual
 * time): between physical
 * time steps of multiGridCycles (mg_par:483-890), uold2 = uold and uold = u
 * on level 1, then the head of the next step: laminar viscosity 1/Re on
 * every level, u and uold restricted to every coarse level (mg_par:586-602).
 * flite_start sets uold = uold2 = u and performs the first step's head.
 * Each RK stage adds the time differences of addTimeDifferences
 * (def_par:1184-1241: second-order backward on level 1 with timeScheme 2,
 * first order elsewhere; for nu~ before its convection) and solveSystem
 * divides the local step by 1 + 1.5 dt / physicalTimeStep (def_par:
 * 1427-1442; solveTurbulenceSystem does not).  On a static mesh the
 * previous volumes are the volumes.                                         */
/* Explicit time stepping (explicit = 1 with flowType 1 or 2, def_par:386-394,
 * 1427-1517, 13598-13607): no time differences, and every node's solve takes
 * ivd%physicalTimeStep, which each makeTimeSteps sets to the smallest local
 * time step of its level.  The value after the last cycle (the step the host
 * adds to its current time, mg_par:711-713):                               */
int flite_explicit_time_step(flite_ctx *ctx, double *dt);
int flite_next_physical_step(flite_ctx *ctx);
/* Moving meshes (flowType 2, ALE): the geometry of the next physical step,
 * read from that step's .sol (mg_par:525-545, readComputationData with the
 * arrays already allocated).  Called after flite_next_physical_step; the
 * levels must have the topology given to flite_create (sizes, side and
 * boundary-side indices, indicators, transfer operators' parents); their
 * coefficients, GCL weights, volumes (current and the two previous), wall
 * distances, coordinates, coordinate movements and restriction weights are
 * taken.  On level 1 with timeScheme 2 the GCL weights are combined as
 * 1.5 GCL - 0.5 GCLprev (def_par:816-818, 13858-13860).  The head of the
 * step (laminar viscosity, u and uold restricted to the coarse levels) is
 * redone with the new restriction weights.  The GCL terms enter every
 * interior-edge flux as -(q1 + q2) GCL/physicalTimeStep (the HLLC flux:
 * -q* GCL/physicalTimeStep with the state of its wave region, def_par:
 * 2046-2085) and every boundary edge as -(3 q1 + q2) GCL1/physicalTimeStep
 * and -(q1 + 3 q2) GCL2/physicalTimeStep (boundaryTerm 2: -4 q GCL/
 * physicalTimeStep; def_par:2124-2177), and the time differences use the
 * current and previous volumes (def_par:1184-1241).                         */
int flite_update_geometry(flite_ctx *ctx, int nlevels, const flite_level_desc *levels);
int flite_do_time_iterations(flite_ctx *ctx, int level, int nsteps,
                             int calc_diss, int calc_turb, int cycle_no);
/* restrictGrid (def_par:12141-12430)                                      */
int flite_restrict(flite_ctx *ctx, int fine_level, int calc_turb);
/* prolongateGrid (def_par:12432-12570)                                    */
int flite_prolong(flite_ctx *ctx, int coarse_level);
/* mapFineToCoarse of the solution (def_par:12572-12679)                   */
int flite_map_fine_to_coarse(flite_ctx *ctx, int fine_level);
/* oneCycle (mg_par:907-1196), every kernel on the device                  */
int flite_cycle(flite_ctx *ctx, int cycle_no);
/* residual norms of writeResiduals (mg_par:1271-1516): res_k = sqrt(sum
 * (u-uprev)^2) on level 1, max |u-uprev| and its 1-based node.  Returns
 * FLITE_ENAN when any res_k is not finite (the reference STOPs).          */
int flite_residuals(flite_ctx *ctx, double res[7], double maxres[7],
                    int32_t maxind[7]);
/* the forces of writeResiduals (mg_par:1359-1367): calculateLiftAndDrag
 * (def_par:14710-14870) gives out[0..5] = {lift, drag, latF, frictionDrag,
 * latM, longM}, the first four as coefficients; with forceCalcType 3,
 * calculateLiftAndDrag3 (def_par:15129-15313) replaces lift, drag, latF and
 * latM and fills out[6..8] = {longMl, longMd, rollM} (else 0).  These are
 * the force columns of the .rsd file (mg_par:1481-1507).                   */
int flite_forces(flite_ctx *ctx, double out[9]);

/* ---- one residual evaluation (adjoint primal / parity probe) ----------- */
/* rhs = makeRHS(u) on a level (def_par:1525-2590) with the level's current
 * pressure recomputed from u; r is [5][N].                                 */
int flite_residual_fwd(flite_ctx *ctx, int level, const double *u, double *r);

/* ---- discrete adjoint of the edge residual ------------------------------
 * ubar = (dR/du)^T rbar for R = flite_residual_fwd on a level (central flux,
 * fluxType 1, FP64; wall, symmetry and far-field boundary fluxes), the
 * backward half of the forward/backward pair.  u, rbar, ubar are [5][N].
 * Like flite_residual_fwd it replaces the level's state by u.  No reference
 * counterpart: the reference has no adjoint.  Moving meshes (flowType 2):
 * FLITE_EUNSUPPORTED.                                                      */
int flite_residual_vjp(flite_ctx *ctx, int level, const double *u, const double *rbar,
                       double *ubar);
/* average device ms of one forward residual evaluation and of one adjoint
 * product on a level (the adjoint cost ratio is vjp/fwd)                  */
int flite_profile_adjoint(flite_ctx *ctx, int level, int reps, double *fwd_ms, double *vjp_ms);

/* ---- steady adjoint: force sensitivities to the level-1 geometry ---------
 * For the central flux with scalar JST dissipation, inviscid or laminar
 * (no turbulence model), FP64 (other controls: FLITE_EUNSUPPORTED).  G is
 * one smoother iteration of level 1 (doTimeIterations with calcDiss,
 * def_par:966-1181: time steps, dissipation, the viscous term, three RK
 * stages with their boundary conditions); in a laminar run its state is the
 * conserved variables and the laminar viscosity [N] that the time step reads
 * (makeTimeSteps runs before makeViscosityTerm recomputes it).  The
 * geometry g is the level-1 side_w [3][E], bnd_w [3][B] and volume [N] of
 * the level descriptor
 * (the node normals and wall areas follow from bnd_w as in
 * makeBoundaryNormals def_par:15394 and makeSurfaceArea :15523).
 * flite_iteration_vjp: ubar = (dG/du)^T lam at the state u [5][N] and, for
 * the geometry pointers that are not NULL, (dG/dg)^T lam; laminar runs pass
 * the viscosity mu [N] the step reads and the adjoint lam_mu [N] of the
 * viscosity the iteration computes (NULL: zero), and get mu_bar [N].
 * flite_adjoint_solve: at the context's level-1 state, which must be a
 * converged solution u* = G(u*), the objective J (FLITE_OBJ_CL or
 * FLITE_OBJ_CD of calculateLiftAndDrag def_par:14710-14870 with the
 * pressure and, in laminar runs, the wall stress of the state) and dJ/dg =
 * J_g + lam^T (dG/dg), where lam = P((dG/du)^T lam + (dJ/du)^T) is solved
 * to the relative residual tol or max_iter products
 * with (dG/du)^T (P keeps the energy of subsonic inflow nodes, which the
 * boundary condition never updates, out of the adjoint).  Sensitivities to
 * node coordinates follow with fp_geometry_vjp of the preprocessor, which
 * owns the elements.  No reference counterpart: the reference has no
 * adjoint.                                                                  */
#define FLITE_OBJ_CL 0
#define FLITE_OBJ_CD 1
/* How flite_adjoint_solve iterates: FLITE_ADJ_FIXED_POINT (lam <- P(G_u^T
 * lam + J_u^T)) or FLITE_ADJ_GMRES (restarted GMRES with the given restart
 * length on the same equation; the default, restart 50).  The stopping test
 * is the same: |P J_u^T - (I - P G_u^T) lam| <= tol |P J_u^T|.               */
#define FLITE_ADJ_FIXED_POINT 0
#define FLITE_ADJ_GMRES 1
int flite_set_adjoint_method(flite_ctx *ctx, int method, int restart);
/* the objective J of flite_adjoint_solve at the context's level-1 state    */
int flite_objective(flite_ctx *ctx, int objective, double *J);
int flite_iteration_vjp(flite_ctx *ctx, const double *u, const double *lam, double *ubar,
                        double *side_w_bar, double *bnd_w_bar, double *volume_bar,
                        const double *mu, const double *lam_mu, double *mu_bar);
int flite_adjoint_solve(flite_ctx *ctx, int objective, double tol, int max_iter, double *J,
                        double *side_w_bar, double *bnd_w_bar, double *volume_bar, int *iterations,
                        double *residual);

/* ---- batched solves (no reference counterpart: the reference runs one
 * condition per job) --------------------------------------------------------
 * ncases solves, case i on mesh mesh_of_case[i] (levels[m] points to the
 * nlevels[m] level descriptors of mesh m) with its own controls[i].  Cases on
 * one mesh share its device copy.  flite_batch_cycle advances every case by
 * one oneCycle with a single CUDA-graph launch; flite_batch_context returns
 * a case's context for flite_set_state/flite_start/flite_residuals/...      */
typedef struct flite_batch flite_batch;
int flite_batch_create(int ncases, const flite_controls *controls, const int32_t *mesh_of_case,
                       int nmeshes, const int32_t *nlevels, const flite_level_desc *const *levels,
                       flite_batch **out);
int flite_batch_destroy(flite_batch *b);
int flite_batch_context(flite_batch *b, int case_index, flite_ctx **ctx);
int flite_batch_cycle(flite_batch *b, int cycle_no);
/* multiGridCycles over the batch: batch cycles first_cycle, first_cycle+1, ...
 * until every case has res1 <= 10^-orders times its res1 after the first
 * cycle (checked after the first cycle and then every check_every cycles),
 * or max_cycles.  A converged case leaves the batch graph.  cycles[i] is the
 * number of cycles case i ran, log10_reduction[i] its log10(res1/res1(1));
 * FLITE_ENAN when a residual is not finite.                                */
int flite_batch_run(flite_batch *b, int first_cycle, int max_cycles, double orders, int check_every,
                    int32_t *cycles, double *log10_reduction);
/* device time of ncycles batch cycles, as one graph launch each
 * (sequential = 0) or as the cases' own graphs launched one after another
 * (sequential = 1); also the kernel launches one batch cycle holds          */
int flite_batch_time_cycles(flite_batch *b, int cycle_no, int ncycles, int sequential, double *ms,
                            int64_t *launches_per_cycle);
/* time reps batch cycles for each edge/node block size in {64,128,256} and
 * keep the fastest pair (advances every case by 9*(reps+1) cycles)       */
int flite_batch_autotune(flite_batch *b, int cycle_no, int reps, int32_t *edge_block,
                         int32_t *node_block, double *best_ms);
/* Case groups (on by default): the cases on one mesh whose controls take
 * the same kernels advance together, every kernel of the cycle launched once
 * for the group with the case in its grid's y index; 0 turns them off (each
 * case its own cycle graph inside the batch graph).  Results are the same
 * either way.  flite_batch_groups gives the groups of the last batch graph;
 * flite_batch_autotune keeps groups on or off, whichever it times faster.  */
int flite_batch_set_grouping(flite_batch *b, int on);
/* The gather tile of each level (lanes per node: 1, 4, 8, 16 or 32) picked
 * by timing batch cycles, coarsest level first, and set on every case;
 * lanes[l] receives level l+1's choice.  Results do not depend on it.     */
int flite_batch_autotune_lanes(flite_batch *b, int cycle_no, int reps, int32_t nlevels, int32_t *lanes,
                               double *best_ms);
int flite_batch_groups(const flite_batch *b, int32_t *ngroups);
int flite_batch_grouping(const flite_batch *b, int32_t *on);
int flite_batch_set_blocks(flite_batch *b, int32_t edge_block, int32_t node_block);

/* ---- residual evaluation that allocates nothing ------------------------
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc (device memory owned by another allocator or by the host
 * program, or code where allocation is not allowed).  Computes the residual
 * of flite_residual_fwd for the central flux (fluxType 1) with its boundary
 * faces, from caller-owned DEVICE arrays in the reference layout: side_idx
 * [2][E] and bnd_idx [3][B] 1-based, side_w [3][E], bnd_w [3][B], u [5][N];
 * writes rhs [5][N].  Scratch lives in one static device array of the
 * library (24,380,160 bytes on every GPU that loads it); limits N <= 65536,
 * E <= 262144, B <= 65536, larger sizes return FLITE_EINVAL, as do an
 * index outside 1..N and a boundary code outside 1..9 (engine faces, codes
 * 5..8, take their flux as in flite_residual_fwd).  The first call on
 * a device looks the scratch up for that device.  The call runs on `stream`
 * (a cudaStream_t, NULL for the default stream), copies its status to host
 * memory and synchronises the stream, so it must not be made while any
 * stream is being captured.  Calls share the scratch: calls that overlap on
 * the GPU race.                                                            */
int flite_residual_noalloc(const flite_controls *c, int32_t n_nodes, int32_t n_sides,
                           int32_t n_bsides, const int32_t *d_side_idx, const double *d_side_w,
                           const int32_t *d_bnd_idx, const double *d_bnd_w, const double *d_u,
                           double *d_rhs, void *stream);

/* ---- timing ----------------------------------------------------------- */
/* Capture one oneCycle as a CUDA graph and replay it `ncycles` times;
 * returns the device time (ms) measured with CUDA events on the context's
 * stream.  cycle numbers only affect numberOfCFLIncrements ramps and are
 * frozen at cycle_no inside the graph.                                     */
int flite_time_cycles(flite_ctx *ctx, int cycle_no, int ncycles, double *ms);
/* Number of kernel launches one oneCycle issues (for launch accounting).  */
int flite_cycle_launches(flite_ctx *ctx, int64_t *n);
/* Kernel-level timing of the dominant kernel (edge flux + gather) over one
 * relaxation of level 1: average ms per launch of the edge-flux kernel and
 * of the node gather/update kernel.                                        */
int flite_profile_level(flite_ctx *ctx, int level, int reps, double *edge_ms,
                        double *node_ms);
/* Launch options of a context (no effect on any result): threads per block
 * of the edge kernels and of the node kernels (32..256, multiples of 32) and
 * the incidences whose loads the fused central gather issues together (1 or
 * 2).  Drops the captured cycle graph.                                     */
int flite_set_kernel_options(flite_ctx *ctx, int32_t edge_block, int32_t node_block, int32_t gather_unroll);
/* Node numbering of the contexts created after this call (no effect on any
 * result; no reference counterpart): 1 renumbers the nodes of every level
 * for locality -- boundary nodes stay first, level 1 in Morton order of the
 * coordinates, coarse levels by their children -- and 0 (the default) keeps
 * the caller's numbering, which a structured mesh generated line by line
 * already orders well.  Node arrays always cross this ABI in the caller's
 * numbering; edges keep their numbers.                                      */
int flite_set_node_order(int32_t order);
/* Lanes per node of the node gathers of a level (no effect on any result):
 * 1 (a thread per node), 4, 8, 16 or 32, or 0 for the default (32 below 8192
 * nodes, else 1).  Drops the captured cycle graph.                         */
int flite_set_gather_lanes(flite_ctx *ctx, int32_t level, int32_t lanes);
/* How a level's fused central gather with a thread per node (fluxType 1,
 * FP64) reads its incidences: 0 (the default) through the node's incidence
 * list; 1..4 through incidence rows of blocks of 256 nodes (row k holds
 * incidence k of every node of the block with its edge coefficients, read
 * with coalesced loads a step ahead), with the block's nodes and the other
 * nodes its edges reach staged in shared memory (1: compiled for two blocks
 * per SM, 2: three) or read from global memory (3: two, 4: three).  No
 * effect on any result.  Drops the captured cycle graph.                   */
int flite_set_tiled_gather(flite_ctx *ctx, int32_t level, int32_t on);
/* Whether a level's node gathers that walk the same incidence list share one
 * walk where a thread serves a node and the list form is used: the time step
 * with the JST Laplacian, and the JST flux with the viscous gradients.  1 (the
 * default) shares, 0 runs them as separate kernels.  No effect on any result.
 * Drops the captured cycle graph.                                           */
int flite_set_gather_fusion(flite_ctx *ctx, int32_t level, int32_t on);
/* Average device ms of the kernel groups of one relaxation step of a level,
 * in order: pressure, time steps, dissipation, viscous primitives, viscous
 * gradients, viscous fluxes, flux terms (edge or boundary kernels), node
 * update (restrictGrid's fine-increment mode: the stage's read set), the
 * shared walk of time step and Laplacian, the shared walk of JST flux and
 * viscous gradients (where the walks are shared, the separate groups hold
 * what is left of them); *n is the number written (at most nmax).  The
 * level's rhs and dissipation are overwritten.                              */
int flite_profile_kernels(flite_ctx *ctx, int level, int reps, double *ms, int32_t nmax, int32_t *n);

#ifdef __cplusplus
}
#endif
#endif /* FLITE_GPU_H */
