/* kofm.h - C ABI of the B200 D2Q9 + k-omega time step.
 *
 * This is the drop-in boundary for the reference's LB/k-omega hot path.  The
 * reference dispatches that path through positional OpenCL kernel objects
 * (Kernel / DualKernel, source/Kernels.h:29-727) whose arguments are set in
 * clVariablesLB::setKernelArgs (clVariablesLB.cpp:790-856),
 * kOmega::setKernelArgs (kOmega.cpp:573-650) and GMRESSolver::createKernels
 * (GMRESSolver.cpp:930-1210), and enqueues them from Solve_no_TR
 * (LBLS.cpp:185-205), clVariablesLB::Solve (clVariablesLB.h:375-441) and
 * kOmega::Solve (kOmega.cpp:31-73).  Each entry point below replaces one of
 * those dispatch sites; the citation is beside it.
 *
 * Conventions
 *  - Plain C types only.  Host arrays use the reference's padded FP64 layout
 *    (Array.h:2377-2383): node (i, j) at i + nx_full*j, population q at
 *    node + q*nx_full*ny, direction order C,E,W,N,S,NE,SW,SE,NW
 *    (Kernels/Heading.cl:197-205).  Populations exchanged through
 *    kofm_set_state / kofm_get_state are the reference's FA buffer
 *    (pre-collision, post-stream; the content of its lbf.bin checkpoint).
 *  - The context owns all device memory.  Host pointers are only read or
 *    written during the call.  The device layout and storage precision are
 *    private to the library.
 *  - Every call returns an int status: 0 = ok, negative = error.  Codes
 *    -100..-123 reuse the reference's error numbers (ConstDef.h:588-611)
 *    where the meaning maps; -200 and below are new.  No call exits the
 *    process.
 *  - One context = one CUDA stream (the reference's LBQUEUE).  Calls on one
 *    context are not thread-safe; several contexts may coexist.  Work is
 *    asynchronous until kofm_sync, a kofm_get_* call or kofm_reduce.
 */
#ifndef KOFM_H
#define KOFM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KOFM_ABI_VERSION 3

/* ---- status codes ------------------------------------------------------ */
#define KOFM_OK 0
#define KOFM_ERR_BUFFER_ALLOCATION -101   /* ERROR_BUFFER_ALLOCATION */
#define KOFM_ERR_MEMORY_COPY -103         /* ERROR_MEMORY_COPY */
#define KOFM_ERR_CALLING_KERNEL -107      /* ERROR_CALLING_KERNEL */
#define KOFM_ERR_LOADING_PARAMS -110      /* ERROR_LOADING_PARAMS: bad descriptor */
#define KOFM_ERR_INITIALIZING_KOMEGA -111 /* ERROR_INITIALIZING_KOMEGA */
#define KOFM_ERR_INITIALIZING_VLS -112    /* ERROR_INITIALIZING_VLS: bad geometry */
#define KOFM_ERR_INITIALIZING_VLB -120    /* ERROR_INITIALIZING_VLB */
#define KOFM_ERR_INVALID_ARG -200         /* NULL pointer / out-of-range value */
#define KOFM_ERR_NO_DEVICE -201           /* no usable sm_100 device */
#define KOFM_ERR_NOT_CONVERGED -202       /* k-omega solve hit its iteration cap */
#define KOFM_ERR_NAN -203                 /* NaN residual; dt halving engaged */
#define KOFM_ERR_TIMEOUT -204             /* a bounded device wait expired */
#define KOFM_ERR_STATE -205               /* call order: geometry/state not set */
#define KOFM_ERR_TOO_LARGE -206           /* input beyond a fixed scratch limit */

/* ---- options (Kernels/Heading.cl:309-311) -------------------------------- */
#define KOFM_OPTION_SAVE_MACRO_FIELDS 0x2 /* write rho, ux, uy this step */

/* ---- storage forms of the populations ------------------------------------ */
#define KOFM_STORE_FP32 0     /* f_i - w_i in FP32, FP64 collide arithmetic */
#define KOFM_STORE_FP16_DEV 1 /* f_i - w_i in FP16, FP32 collide arithmetic */
#define KOFM_STORE_BF16_DEV 2 /* f_i - w_i in BF16, FP32 collide arithmetic */
#define KOFM_STORE_FP16_NEQ 3 /* f_i - feq_i(rho_r, u_r) in FP16 (scaled by 2^12),
                                 with the writer's FP32 rho, u as reference;
                                 FP64 collide arithmetic.  No counterpart in
                                 the reference (its arrays are FP64). */
#define KOFM_STORE_FP16_NEQ32 5 /* as KOFM_STORE_FP16_NEQ with FP32 collide
                                   arithmetic; the reference moments of a stored
                                   value are the writer's unforced rho, u, and the
                                   value carries the force increment.  No
                                   counterpart in the reference. */
#define KOFM_STORE_FP64 4     /* f_i - w_i in FP64 and every node field (k,
                                 omega, nu_t, strain rates, wall distance,
                                 moments) in FP64, FP64 arithmetic throughout:
                                 the reference's precision (Heading.cl:7,
                                 FTYPE double), the truth of the precision
                                 study.  Not with the thermal update, the
                                 device geometry builder or the adjoint. */
#define KOFM_STORE_FP16_ROW 6 /* f_i - feq_i(rho_R(y), u_R(y)) in FP16 (scaled
                                 by 2^12) with ONE reference per row: the mean
                                 density and velocity of the row's fluid nodes
                                 at kofm_set_state, re-centred on the row means
                                 of the moments every 32 collides that save
                                 them (the stored values re-encoded).  FP32
                                 collide arithmetic, u from FP64 sums of the
                                 deviations.  Suited to flows close to
                                 their row profile (straight channels); not in
                                 kofm_batch.  No counterpart in the reference. */

/* ---- fields for kofm_reduce ---------------------------------------------- */
#define KOFM_FIELD_RHO 0   /* Ro_array   (clVariablesLB.cpp:343-345 sumRo) */
#define KOFM_FIELD_UX 1    /* Ux_array   (sumUx) */
#define KOFM_FIELD_UY 2    /* Uy_array   (sumUy) */
#define KOFM_FIELD_K 3     /* Kappa_array (kOmega.cpp:315-318 sumKappa/minKappa) */
#define KOFM_FIELD_OMEGA 4 /* Omega_array (sumOmega/minOmega) */
#define KOFM_FIELD_NUT 5   /* Nut_array */
#define KOFM_FIELD_WALL_SHEAR 6 /* wall-shear integral (see kofm_reduce) */
#define KOFM_FIELD_TEMP 7  /* tempArray (clVariablesFD.cpp:266 sumTemp) */
#define KOFM_OP_SUM 0
#define KOFM_OP_MIN 1
#define KOFM_OP_MAX 2

typedef struct kofm_ctx kofm_ctx;

/* Run parameters.  Replaces the program-build-time defines that
 * clVariablesLB::setSourceDefines / kOmega::setSourceDefines /
 * clProblem::setSourceDefines inject (clVariablesLB.cpp:860-877,
 * kOmega.cpp:660-680) and the solver settings of
 * GMRESSolver::CreateSolverWithVarTime (GMRESSolver.cpp:1304-1418). */
typedef struct kofm_desc {
    int32_t nx;          /* CHANNEL_LENGTH (nX) */
    int32_t nx_full;     /* XsizeFull: row pitch of host arrays, >= nx */
    int32_t ny;          /* CHANNEL_HEIGHT (nY); rows 0 and ny-1 must be solid */
    int32_t use_komega;  /* kOmegaSolverFlag */
    double tau;          /* relaxation RATE 1/tau (the reference's "Tau" / tau0) */
    double fterm;        /* FTERM_VAL: EDM velocity increment per step */
    double mu;           /* MU_NUMBER: laminar kinematic viscosity */
    double max_turb_visc;/* MAX_TURB_VISC (ConstDef.h:195, 10.0) */
    int32_t storage;     /* KOFM_STORE_* */
    int32_t device;      /* CUDA device ordinal */
    int32_t komega_max_iters; /* KOMEGA_MAX_ITERS (1000) */
    int32_t krylov_dim;       /* GMRES_KRYLOV_DIM_SIZE (10); 1..10 */
    double komega_rel_tol;    /* KOMEGA_MAX_REL_TOL (1e-4) */
    double komega_abs_tol;    /* KOMEGA_MAX_ABS_TOL (1e-7) */
    double komega_dt;         /* initial k-omega time step (p.dTlb = 1) */
    int32_t komega_full_cycle;/* 1: always build all krylov_dim vectors of a
                                 restart cycle, as GMRESSolver::solve does;
                                 0 (default): end the cycle as soon as its
                                 truncation tests fire (see kofm_komega_solve) */
    int32_t solver_max_blocks;/* cap on the k-omega solver's grid (0: two
                                 blocks per SM, fewer on small lattices);
                                 lattices advanced together (kofm_batch_*)
                                 may share the GPU better with a cap */
    /* thermal implicit FD (clVariablesFD::loadParams, clVariablesFD.cpp:444-493) */
    int32_t use_thermal;      /* thermalSolverFlag (USE_THERMAL_SOLVER) */
    int32_t thermal_every;    /* tfdSteps: LB steps per thermal update
                                 (LB_STEPS_PER_FD = 1, LBLS.cpp:197) */
    double pr_number;         /* Pr (PR_NUMBER 0.708): alpha_fluid = mu / Pr */
    double pr_turb_number;    /* Pr_t (PR_TURB_NUMBER 0.9) */
    double alpha_foul;        /* LB_ALPHA_FOUL: diffusivity of fouling-layer
                                 nodes (M0_FLUID | M_SOLID) */
    double t_in;              /* TFD_X_IN_VAL (TFD_X_IN 2.0): inlet temperature
                                 and upper clamp of T in the source term */
    int32_t thermal_max_iters;/* THERMAL_MAX_ITERS (1000) */
    int32_t komega_classic;   /* k-omega solver form: 0 (default) builds all
                                 Krylov directions of a cycle in one sweep
                                 (powers of the off-diagonal operator, Gram
                                 matrix, the simpler-GMRES steps in that
                                 basis), each sweep its own kernel launch and
                                 the host enqueueing one round at a time;
                                 2 is the same solve in one cooperative
                                 launch (the form kofm_batch graphs capture);
                                 3 is form 0 with the host enqueueing each
                                 round and synchronising per solve (status
                                 codes at once, no update graph);
                                 1 builds one vector per sweep as
                                 GMRESSolver::solve does.  komega_full_cycle = 1
                                 implies 1.  All follow the reference's
                                 restart loop and truncation tests. */
    double thermal_rel_tol;   /* THERMAL_MAX_REL_TOL (1e-4) */
    double thermal_abs_tol;   /* THERMAL_MAX_ABS_TOL (1e-7) */
    double thermal_dt;        /* dTtfd (= tfdSteps, 1); sub-steps per update
                                 start at (int)(1 / thermal_dt) */
} kofm_desc;

/* Per-context counters of the last k-omega update (kOmega::Solve). */
typedef struct kofm_stats {
    int32_t omega_iters, k_iters;       /* GMRESSolver::iterCount */
    int32_t omega_restarts, k_restarts; /* restart-loop iterations entered */
    int32_t omega_cycles, k_cycles;     /* Krylov cycles run */
    int32_t omega_vectors, k_vectors;   /* Krylov vectors built (device passes) */
    int32_t omega_vec_index_sum, k_vec_index_sum; /* sum of in-cycle indices */
    int32_t omega_update_terms, k_update_terms;   /* sum of update lengths kk */
    int32_t omega_nan, k_nan;           /* NaN residual seen */
    int32_t steps_per_lb;               /* kOmega::stepsPerLB */
    int32_t time_since_change;          /* kOmega::timeSinceTimeStepChange */
    double dt;                          /* kOmega::timeStep */
    double omega_rel_res, k_rel_res;    /* rho_0 / norm_rhs at exit */
    int64_t steps;                      /* LB steps taken */
    int32_t solver_passes;              /* grid sweeps of the last solve */
    int32_t phase;                      /* 0: populations pre-collision, 1: post */
    /* last thermal update (clVariablesFD::Solve) */
    int32_t thermal_iters;              /* BiCGStabSolver::iterCount, last solve */
    int32_t thermal_checks;             /* residual checks of the last solve */
    int32_t thermal_solves;             /* solves run by the update */
    int32_t thermal_resets;             /* dt halvings in the update */
    int32_t thermal_steps_per_lb;       /* clVariablesFD::stepsPerLB */
    int32_t thermal_time_since_change;  /* clVariablesFD::timeSinceTimeStepChange */
    double thermal_dt;                  /* clVariablesFD::timeStep */
    double thermal_residual;            /* last ||r||_1 / ||b||_1 */
    double solver_bytes_per_node;       /* algorithmic HBM bytes per lattice node of the
                                           last k-omega solve (both systems): every
                                           array its sweeps stream, counted once per sweep */
    int32_t omega_powers, k_powers;     /* one-sweep cycles: powers computed (all rounds) */
    int32_t solver_launches;            /* kernel launches of the last k-omega solve */
    int32_t solver_rounds;              /* rounds of the last solve (phase launches:
                                           powers + Gram + update sweeps; 1 otherwise) */
    int64_t solver_launches_total;      /* kernel launches of all k-omega updates
                                           since the state was loaded */
} kofm_stats;

int kofm_abi_version(void);
const char* kofm_error_string(int status);

/* Fills *d with the reference defaults (ConstDef.h: KOMEGA_* tolerances,
 * GMRES_KRYLOV_DIM_SIZE, MAX_TURB_VISC, dTlb = 1, FP32 storage, device 0). */
int kofm_desc_default(kofm_desc* d);

/* Allocates device memory for the descriptor's lattice and its solver.
 * Replaces clVariablesLB::allocateBuffers / kOmega::allocateBuffers /
 * GMRESSolver::ini + CreateSolver (clVariablesLB.cpp:56-75,
 * kOmega.cpp:99-108, GMRESSolver.cpp:1225-1259, 1314-1418). */
int kofm_create(const kofm_desc* d, kofm_ctx** out);
int kofm_destroy(kofm_ctx* ctx);

/* Geometry: nType flags (Heading.cl:223-251 bits), wall distance WallD
 * (kOmega.cpp:330-349), link fractions dXArr [4 planes E,W,N,S]
 * (clVariablesLS.cpp:650-684) and the interpolated bounce-back link list
 * ibbArr/ibbDistArr (population index + wall fraction q) consumed by lbIBB
 * (lbKernels.cl:640-668; set at clVariablesLB.cpp:841-852).  wallD and dX4
 * may be NULL when use_komega = 0; n_ibb may be 0.
 * Rejects fluid nodes in rows 0 / ny-1 (clVariablesLS.cpp:935-937). */
int kofm_set_geometry(kofm_ctx* ctx, const int16_t* ntype, const double* wallD,
                      const double* dX4, const int32_t* ibb_idx,
                      const double* ibb_q, int32_t n_ibb);

/* Geometry built on the device from the wall heights at every column: node
 * (x, y) is fluid iff y_bot[x] < y < y_top[x] (rows 0 and ny-1 never), the
 * walls being polylines through (x, y_w[x]), periodic in x.  Builds what
 * kofm_set_geometry takes -- the nType flags, the E/W/N/S link fractions, the
 * interpolated bounce-back links (wall fraction q = first crossing of the link
 * with a wall; links with q = 1/2 left out unless KOFM_WALLS_IBB_ALL; none on
 * columns 0 and nx-1, as updateIBBOnly, lsKernels.cl:455-466, unless
 * KOFM_WALLS_SEAM_IBB) and, with k-omega, the wall distance of the
 * reference's updateWallD (kOmegaKernels.cl:751-840) over the segments within
 * wall_radius ("Wall D Search Rad", default WALLD_SEARCH_RADIUS = 50) of the
 * node's column, the walls taken through x = -1 .. nx -- plus, with the
 * thermal update, what kofm_set_thermal_geometry takes (fractions of the
 * unfouled walls y_bot0 / y_top0, NULL = the fouled ones).  Replaces the
 * host set-up of clVariablesLS::ini (clVariablesLS.cpp:650-1000) and
 * kOmega::iniWallD (kOmega.cpp:136-193, 330-349) for such walls, and can be
 * called again on a live context when the walls move (clVariablesLS::update,
 * clVariablesLS.cpp:1020-1033); on a stepped context the nodes that turn
 * from fluid to solid get k, omega, nu_t, the strain rates and the moments
 * set to 0, as updateNType (lsKernels.cl:47-163) does for a growing deposit
 * (populations and temperature stay).  min_dx is the smallest E/W/N/S link
 * fraction ("Min dX Dist", reference default MINIMUM_DX_DIST = 0.001,
 * bcSetdXArr, clVariablesLS.cpp:248-286), in [0, 1]; the interpolated list
 * keeps the unclamped fraction.  Requires y_bot0 <= y_bot and
 * y_top0 >= y_top, all finite. */
#define KOFM_WALLS_IBB_ALL 1
#define KOFM_WALLS_SEAM_IBB 2   /* interpolated links on columns 0 and nx-1 too */
int kofm_set_walls(kofm_ctx* ctx, const double* y_bot, const double* y_top,
                   const double* y_bot0, const double* y_top0, double min_dx,
                   int32_t wall_radius, int32_t flags);

/* The context's geometry in the layouts kofm_set_geometry / _thermal_geometry
 * take (any output may be NULL): ntype [nx_full*ny], wallD (k-omega
 * contexts), dX4 and dX04 [4][nx_full*ny] (dX4: k-omega or thermal contexts,
 * or any geometry from kofm_set_walls; dX04: thermal contexts), and the
 * interpolated links ordered by (direction, node) with their q (*n_ibb gets
 * the count; cap = room in ibb_idx / ibb_q).  KOFM_ERR_STATE for an output
 * the context does not hold.  No counterpart in the reference. */
int kofm_get_geometry(kofm_ctx* ctx, int16_t* ntype, double* wallD, double* dX4,
                      double* dX04, int32_t* ibb_idx, double* ibb_q, int32_t cap,
                      int32_t* n_ibb);

/* State upload: f = FA (9 planes), k, omega, nut (1 plane each), sxy (3
 * planes Sxx,Sxy,Syy).  The k-omega arrays may be NULL when use_komega = 0;
 * nut may be NULL (it is recomputed by the next step).  Replaces the
 * allocate_buffer_w_copy uploads of ini() and the lbf/lbkappa/lbomega bin
 * loads (clVariablesLB.cpp:883-902, kOmega.cpp:685-710); as there, the
 * k-omega sub-stepping starts again from the descriptor's komega_dt. */
int kofm_set_state(kofm_ctx* ctx, const double* f, const double* k,
                   const double* omega, const double* nut, const double* sxy);

/* State download in the same layout (FA = what saveRestartFiles writes,
 * clVariablesLB.cpp:752-765).  Any pointer may be NULL. */
int kofm_get_state(kofm_ctx* ctx, double* f, double* k, double* omega,
                   double* nut, double* sxy);

/* Macroscopic fields written by the last step with
 * KOFM_OPTION_SAVE_MACRO_FIELDS (Ro_array, Ux_array, Uy_array).  Any pointer
 * may be NULL. */
int kofm_get_macro(kofm_ctx* ctx, double* rho, double* ux, double* uy);

/* One collide + stream + interpolated bounce-back pass:
 * vlb.collisionKernel.call_kernel + vlb.ibbKernel.call_kernel
 * (LBLS.cpp:188-190; LB_collision_SRT_Fluid[_w_kOmega], lbIBB). */
int kofm_lb_step(kofm_ctx* ctx, int32_t options);

/* Builds both implicit k/omega systems for time step dt:
 * kOmegaUpdateDiffCoeffs + kOmegaUpdateCoeffs (kOmega.cpp:43-44;
 * Update_kOmega_Diffusivities, Update_kOmega_Coeffs_Implicit). */
int kofm_komega_assemble(kofm_ctx* ctx, double dt);

/* Solves the assembled systems and updates omega and k:
 * OmegaGMRES.solve(); KappaGMRES.solve() (kOmega.cpp:68-70;
 * GMRESSolver::solve, GMRESSolver.cpp:227-355).  Both run in one
 * device-resident launch.  The reference builds all krylov_dim vectors of a
 * cycle and only then applies its truncation tests (diag(R) against
 * relTol * R(0,0), then |xi_i| >= rho); the default here applies the same
 * tests as each vector is made and stops at the first that fires, which gives
 * the reference's update unless a diag(R) cut would fall after the xi cut
 * (the reference then indexes its back-substitution with that later cut).
 * komega_full_cycle = 1 keeps the reference's full cycle.  iters/rel_res receive (omega, k) pairs; either
 * may be NULL.  Returns KOFM_ERR_NAN if a residual was NaN (the caller's
 * kOmega::Solve halves dt), KOFM_ERR_NOT_CONVERGED at the iteration cap. */
int kofm_komega_solve(kofm_ctx* ctx, int32_t* iters, double* rel_res);

/* kOmega::Solve (kOmega.cpp:31-73): adaptive sub-stepping (halve dt on a
 * NaN residual, double it after 20 calm steps; kOmega.cpp:387-414) around
 * assemble + solve.  A field whose solve met a NaN keeps its value from
 * before that solve.  Where the reference would halve for ever (a NaN that
 * no smaller dt removes), this returns KOFM_ERR_NAN once more than 2^20
 * sub-steps per LB step would be needed; kofm_get_stats then shows the
 * halved dt, and kofm_set_state (a repaired state) starts the sub-stepping
 * again. */
int kofm_komega_update(kofm_ctx* ctx);

/* nsteps x Solve_no_TR (LBLS.cpp:185-205): kofm_lb_step with
 * options | KOFM_OPTION_SAVE_MACRO_FIELDS when k-omega is on, then
 * kofm_komega_update. */
int kofm_step(kofm_ctx* ctx, int32_t nsteps, int32_t options);

/* Reducer<double>::reduceSingle (Reducer.h:240-278) over the full padded
 * array of a field (FP64 accumulation, deterministic order).  For
 * KOFM_FIELD_WALL_SHEAR and op SUM: sum over fluid nodes with an N or S wall
 * link of rho*(mu + nu_t)*2*|S_xy| (a diagnostic of this library; the
 * reference's per-link shear coefficients, trKernelsShear.cl, are not part
 * of this path). */
int kofm_reduce(kofm_ctx* ctx, int32_t field, int32_t op, double* out);

/* Wall shear set-up: the shear nodes (node indices i + nx_full*j of the
 * padded host layout; clVariablesLS::fillShearArray, clVariablesLS.cpp:288-320),
 * their two coefficient rows of 8 (x then y; TR_Find_Shear_Coeffs1,
 * Kernels/trKernelsShear.cl:333-375), and per boundary link the list indices
 * of its four nearest shear nodes (-1: none) with their weights
 * (TR_Find_Shear_Coeffs2, trKernelsShear.cl:414-505).  n_bl may be 0.
 * komegafoulingmodel_b200/shear.py builds all of them from the walls. */
int kofm_set_shear(kofm_ctx* ctx, const int32_t* nodes, int32_t n_nodes, const double* cfss,
                   const int32_t* bl_nodes, const double* bl_weights, int32_t n_bl);

/* Wall shear of the current state at the shear nodes (TR_shear_1,
 * trKernelsShear.cl:131-222: non-equilibrium part of the node's post-stream
 * populations against the moments of the last step, (nu + nu_t)-scaled) and
 * at the boundary links (TR_shear_2, trKernelsShear.cl:300-316).  Either
 * output may be NULL; synchronises. */
int kofm_wall_shear(kofm_ctx* ctx, double* node_tau, double* bl_tau);

/* ---- thermal implicit finite differences ----------------------------------
 * The temperature update of Solve_no_TR (LBLS.cpp:197-200 -> vfd.Solve,
 * clVariablesFD.h:343-358): Update_T_Coeffs_Implicit (tfdKernels.cl:122-279)
 * and BiCGStabSolver::solve (BiCGStabSolver.cpp:628-723) with the dt halving
 * and doubling of clVariablesFD.cpp:202-228.  Needs desc.use_thermal; kofm_step
 * runs it after the k-omega update every thermal_every steps.  T lives on the
 * device in FP64. */

/* tempArray in (host layout, FP64): clVariablesFD::ini fills ROE0 (Tinitial,
 * 0.5) on M0_FLUID nodes and 0 elsewhere (clVariablesFD.cpp:236-239);
 * restart files load it instead. */
int kofm_set_temperature(kofm_ctx* ctx, const double* T);
int kofm_get_temperature(kofm_ctx* ctx, double* T);
/* Link fractions of the unfouled walls, vls.dXArr0 (E, W, N, S planes of
 * nx_full*ny each) that the thermal rows use; without this call the dX4 of
 * kofm_set_geometry serves (no fouling layer). */
int kofm_set_thermal_geometry(kofm_ctx* ctx, const double* dX0);
/* One clVariablesFD::Solve; synchronises once per solve (reads the solver's
 * exit state for the dt halving). */
int kofm_thermal_update(kofm_ctx* ctx);

int kofm_sync(kofm_ctx* ctx);
int kofm_get_stats(kofm_ctx* ctx, kofm_stats* out);

/* Diagnostic for the bounded device waits: runs the k-omega solver with a
 * grid barrier that can never complete and the given spin bound (polls of
 * about 100 ns).  Returns KOFM_ERR_TIMEOUT with the context still usable and
 * the fields unchanged.  No counterpart in the reference. */
int kofm_debug_barrier_timeout(kofm_ctx* ctx, int64_t spin_limit);

/* Test hook for the k-omega sub-stepping (kOmega::halveTimeStep,
 * kOmega.cpp:387-399): the next n k-omega solves report a NaN residual for
 * the systems in mask (1: omega, 2: k) at their first convergence check and
 * leave those fields as they were -- what a solve whose right-hand side holds
 * a NaN does -- so that kofm_komega_update halves dt.  The failure is made on
 * the host side of the call; nothing faults on the device.  No counterpart in
 * the reference. */
int kofm_debug_fail_solves(kofm_ctx* ctx, int32_t n, int32_t mask);

/* Diagnostic: device times (ns after the launch started) at which the last
 * k-omega solve's grid barriers released -- the ends of its sweeps -- into
 * ns[0 .. min(*n, cap) - 1]; *n gets the number of barriers (at most 32 are
 * timed).  Synchronises.  No counterpart in the reference. */
int kofm_debug_solver_trace(kofm_ctx* ctx, int64_t* ns, int32_t cap, int32_t* n);

/* Diagnostic: the rows of one k-omega system (0: omega, 1: k) as the last
 * assembly (kofm_komega_assemble, or the assembly of the last update) left
 * them.  coef: [4][ny][nx_full] off-diagonals E, W, N, S of each row
 * normalised by its diagonal (the values Update_kOmega_Coeffs_Implicit,
 * kOmegaKernels.cl:187-480, scatters into the CSR row); rhs: [ny][nx_full]
 * b - A x0 with b the normalised right-hand side and x0 the field the
 * assembly read.  Columns x >= nx are left untouched; either pointer may be
 * NULL.  Synchronises.  No counterpart in the reference. */
int kofm_debug_komega_rows(kofm_ctx* ctx, int32_t system, double* coef, double* rhs);

/* ---- discrete adjoint of the laminar step -----------------------------------
 * No counterpart in the reference.  From the current state (a stepped FP32
 * laminar context without thermal update), takes T steps and returns
 *   J = sum over the T steps of j(FA), FA the populations a step gathers,
 *   j = (mean rho of the fluid nodes of column 0 - that of column nx-1) / 3
 *       + sum of the wall shear of TR_shear_1 (trKernelsShear.cl:175-222) at
 *         the shear nodes of kofm_set_shear (none: the pressure term only),
 *       computed from FA and its own moments,
 * and dJ/dq for every interpolated bounce-back link given to
 * kofm_set_geometry (its wall fraction q; dJdq may be NULL), by the hand-written
 * adjoint of the gather + collide.  The forward's states are kept on the
 * device as far as the cap of kofm_set_adjoint_memory allows; the rest are
 * recomputed from checkpoints (one per segment of s steps, s >= ceil(sqrt(T))).
 * The work buffers stay with the context for the next call.  The lattice ends
 * T steps ahead. */
int kofm_adjoint(kofm_ctx* ctx, int32_t T, double* J, double* dJdq);

/* Device memory kofm_adjoint may hold for stored states: bytes < 0 (the
 * default) = half of the free device memory at the call; 0 = only the
 * checkpoints and one segment of ceil(sqrt(T)) steps; otherwise that many
 * bytes (never fewer than the sqrt(T) minimum).  Results do not depend on it.
 * No counterpart in the reference. */
int kofm_set_adjoint_memory(kofm_ctx* ctx, int64_t bytes);

/* ---- reduction without device allocation ---------------------------------
 * No counterpart in the reference.  For callers that must not let the library
 * allocate device memory (an application that owns a fixed device-memory
 * budget and serves every buffer from its own pool, or a latency-critical
 * caller that cannot accept an allocation's implicit device synchronisation).
 * Reduces (KOFM_OP_SUM / MIN / MAX, FP64 accumulation, deterministic order) a
 * device FP32 field of ny rows of `pitch` floats, counting the first `ncols`
 * columns of each row, into *out (one double in device memory), on `stream`.
 * Both buffers belong to the caller.  The only scratch is a fixed array of
 * KOFM_NOALLOC_MAX_PARTIALS doubles (32 KiB) inside the library, kept by every
 * device that loads it until the process exits: one partial per
 * KOFM_NOALLOC_CHUNK nodes, so pitch*ny may not exceed KOFM_NOALLOC_MAX_NODES
 * (KOFM_ERR_TOO_LARGE otherwise).  All calls share that array: calls that
 * overlap on the GPU race.  Each call overwrites the partials it uses.  A
 * call made outside stream capture looks the array's address up
 * (cudaGetSymbolAddress) in the calling thread's current CUDA context and
 * remembers it for that context; a call made while `stream` is being captured
 * uses the remembered address, so make the first call in each context before
 * any capture (KOFM_ERR_STATE otherwise). */
#define KOFM_NOALLOC_MAX_PARTIALS 4096
#define KOFM_NOALLOC_CHUNK 65536
#define KOFM_NOALLOC_MAX_NODES (4096LL * 65536LL)
int kofm_reduce_field_noalloc(const float* field, int32_t ncols, int32_t pitch, int32_t ny,
                              int32_t op, double* out, void* stream);

/* The CUDA stream the context enqueues on (cudaStream_t as void*), for
 * callers that order their own work against it. */
void* kofm_stream(kofm_ctx* ctx);

/* ---- batched lattices ------------------------------------------------------
 * No counterpart in the reference, which runs one channel per process.
 * Advances n independent lattices together: two time steps of every lattice
 * are captured once into one CUDA graph, and kofm_batch_step replays it (one
 * graph launch per two steps).  Per step the collide of all lattices runs as
 * one persistent launch per group of lattices with the same storage form and
 * model, its blocks walking a table of tiles (tile_rows block rows of 4
 * lattice rows x 128 columns of one lattice; kofm_batch_create_tiled chooses
 * tile_rows, 0 or kofm_batch_create: 2; -1 keeps one collide launch per
 * lattice in the lattice's own branch); then every k-omega lattice's
 * assembly and solve run as concurrent graph branches (the one-sweep-per-
 * cycle solver in its one-launch form, komega_classic 2, for contexts of the
 * phase-launch forms).  Requirements checked by kofm_batch_create: all
 * contexts on one device, each past its first step (kofm_step /
 * kofm_lb_step called at least once), and for k-omega lattices
 * steps_per_lb == 1 (no dt halving in progress).  The captured solves
 * cannot run the dt halving: a NaN residual in any of them stops
 * kofm_batch_step with KOFM_ERR_NAN, after which the contexts are used on
 * their own (kofm_step).  While the batch exists the contexts may be read
 * (kofm_get_*, kofm_reduce, kofm_get_stats) but not stepped on their own. */
typedef struct kofm_batch kofm_batch;
int kofm_batch_create(kofm_ctx* const* ctxs, int32_t n, kofm_batch** out);
int kofm_batch_create_tiled(kofm_ctx* const* ctxs, int32_t n, int32_t tile_rows, kofm_batch** out);
/* nsteps must be a multiple of 2; returns after the steps completed. */
int kofm_batch_step(kofm_batch* b, int32_t nsteps);
int kofm_batch_destroy(kofm_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* KOFM_H */
