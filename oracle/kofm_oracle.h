/* kofm_oracle.h - CPU restatement (FP64) of the reference's D2Q9 + k-omega
 * time step.  TEST INFRASTRUCTURE ONLY: the tests, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg use it as the checker.  The product path
 * (komegafoulingmodel_b200) never links or calls it.
 *
 * Parity pinning: every LB and k-omega kernel restated here is compared
 * against the reference's own kernel sources compiled for the CPU
 * (oracle/_ref, built by oracle/Makefile) and against committed fixtures
 * generated from them (tests/golden/).  The GMRES restatement follows the
 * reference host loop GMRESSolver::solve (GMRESSolver.cpp:227-355) and the
 * kernels of gmresKernels.cl; it is cross-checked against a direct sparse
 * solve (scipy) because the reference ships no solver fixtures.
 *
 * Layout (the reference's): node (i, j) -> gi = i + nxf*j, nxf = XsizeFull;
 * population q of node gi -> gi + q*nxf*ny (Array.h:2377-2383).
 * Direction order C,E,W,N,S,NE,SW,SE,NW (Heading.cl:197-205).
 */
#ifndef KOFM_ORACLE_H
#define KOFM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_cfg {
    int nx;               /* CHANNEL_LENGTH (nX) */
    int nxf;              /* CHANNEL_LENGTH_FULL (XsizeFull) */
    int ny;               /* CHANNEL_HEIGHT (nY) */
    double tau0;          /* relaxation RATE 1/tau (the reference's "tau0") */
    double fterm;         /* FTERM_VAL: velocity increment per step (EDM) */
    double mu;            /* MU_NUMBER: laminar kinematic viscosity */
    double max_turb_visc; /* MAX_TURB_VISC */
} orc_cfg;

/* nType bits (Heading.cl:223-251). */
enum {
    ORC_M_SOLID = 0x0001, ORC_M_FLUID = 0x0002, ORC_M0_SOLID = 0x0004,
    ORC_M0_FLUID = 0x0008, ORC_SOLID_BOUNDARY = 0x0010,
    ORC_SOLID_BOUNDARY0 = 0x0020, ORC_NESW_BOUNDARY0 = 0x0040,
    ORC_BOUNDARY0 = 0x0080, ORC_E_BOUND = 0x0100, ORC_W_BOUND = 0x0200,
    ORC_N_BOUND = 0x0400, ORC_S_BOUND = 0x0800, ORC_NE_BOUND = 0x1000,
    ORC_SW_BOUND = 0x2000, ORC_SE_BOUND = 0x4000, ORC_NW_BOUND = 0x8000,
    ORC_NESW_BOUNDARY = 0x0F00, ORC_BOUNDARY = 0xFF00
};
#define ORC_OPTION_SAVE_MACRO_FIELDS 0x2

/* ---- LB ---------------------------------------------------------------- */
void orc_feq(double rho, double ux, double uy, double* feq9);
void orc_collide_push(const orc_cfg* c, const double* FA, double* FB,
                      const int16_t* map, double* rho, double* ux, double* uy,
                      double* K, double* O, const double* wallD, double* nut,
                      double* Sxy, int options, int komega);
void orc_ibb(const orc_cfg* c, const int32_t* ibb, const double* q, double* FB,
             int n);
void orc_macro(const orc_cfg* c, const double* F, const int16_t* map,
               double* rho, double* ux, double* uy);

/* ---- k-omega assembly --------------------------------------------------- */
void orc_komega_diffusivities(const orc_cfg* c, const int16_t* map,
                              const double* K, const double* O,
                              const double* nut, const double* wallD,
                              double* Dk, double* Do, double* F1,
                              double* dkdxy, const double* rho,
                              const double* dX);
void orc_komega_coeffs(const orc_cfg* c, const int32_t* ind, const double* K,
                       const double* O, const double* nut, const double* Dk,
                       const double* Do, const double* F1, const double* dkdo,
                       const double* Sxy, const double* rho, const double* ux,
                       const double* uy, double* kA, double* oA, double* kb,
                       double* ob, const double* dX, const double* wallD,
                       const int16_t* map, double dt);

/* ---- CSR pattern + GMRES ------------------------------------------------ */
/* Returns nnz.  IA has nxf*ny+1 entries, ind has 5*nxf*ny (C,E,W,N,S planes);
 * JA must hold nnz entries (call once with JA = NULL to size it). */
int orc_csr_build(const orc_cfg* c, const int16_t* map, int32_t* IA,
                  int32_t* JA, int32_t* ind);
/* Fills the diagonal of solid-boundary rows with 1 (GMRESSolver.cpp:1421-1433). */
void orc_csr_fill_solid_boundary(const orc_cfg* c, const int16_t* map,
                                 const int32_t* ind, double* A);

typedef struct orc_gmres_stats {
    int iters;        /* accumulated iteration counter (iterCount) */
    int restarts;     /* restart cycles entered */
    int nan;          /* 1 when the residual became NaN (resetTimeFunc path) */
    double rho0;      /* last residual norm */
    double norm_rhs;  /* ||b - A x0|| */
    double prev_err;  /* prevErr estimate */
} orc_gmres_stats;

/* GMRESSolver::solve.  b is overwritten with b - A x0 (updateRHS); x holds
 * the initial guess on entry and the solution on exit. */
void orc_gmres_solve(int n, const int32_t* IA, const int32_t* JA,
                     const double* A, double* b, double* x, int krylov,
                     int max_iters, double rel_tol, double abs_tol,
                     orc_gmres_stats* st);

/* ---- k-omega solve driver (kOmega::Solve) ------------------------------ */
typedef struct orc_komega_state {
    int steps_per_lb;          /* stepsPerLB */
    int time_since_change;     /* timeSinceTimeStepChange */
    double dt;                 /* timeStep */
    int max_iters;
    double rel_tol, abs_tol;
    orc_gmres_stats last_k, last_o;
    /* test hook (no counterpart in the reference): the next fail_solves
     * solves of the systems in fail_mask (1: omega, 2: k) report a NaN
     * residual at their first convergence check and leave their field as it
     * was, which is what a solve whose right-hand side holds a NaN does */
    int fail_solves, fail_mask;
} orc_komega_state;

/* Runs kOmega::Solve on the given fields.  Work buffers: Dk, Do, F1 [n],
 * dkdo [2n], kA, oA [nnz], kb, ob [n].  CSR arrays from orc_csr_build. */
void orc_komega_solve(const orc_cfg* c, orc_komega_state* s,
                      const int16_t* map, const int32_t* IA, const int32_t* JA,
                      const int32_t* ind, double* K, double* O,
                      const double* nut, const double* wallD, const double* rho,
                      const double* ux, const double* uy, const double* Sxy,
                      const double* dX, double* Dk, double* Do, double* F1,
                      double* dkdo, double* kA, double* oA, double* kb,
                      double* ob);

/* ---- geometry ----------------------------------------------------------- */
/* Straight channel: rows 0 and ny-1 solid, half-way walls at y = 0.5 and
 * y = ny - 1.5.  Fills nType (with boundary bits), dX [4n] (E,W,N,S link
 * fractions) and wall distance. */
void orc_geom_straight(const orc_cfg* c, int16_t* map, double* dX,
                       double* wallD);

/* ---- reductions ---------------------------------------------------------- */
/* ---- wall shear (TR_shear_1 / TR_shear_2, Kernels/trKernelsShear.cl:131-222,
 * 300-316) ------------------------------------------------------------------
 * tau at every shear node from the post-stream populations FA and the
 * moments rho, ux, uy of the last collision; nut may be NULL (laminar). */
void orc_wall_shear_nodes(const orc_cfg* c, const double* FA, const double* rho,
                          const double* ux, const double* uy, const double* nut,
                          const int32_t* nodes, int n, const double* cfss, double* tau);
/* weighted mean of the four nearest shear nodes per boundary link (-1: none) */
void orc_wall_shear_links(const double* tau_nodes, const int32_t* sind, const double* w,
                          int nbl, double* out);

/* ---- thermal implicit FD (clVariablesFD::Solve, clVariablesFD.h:343-358) -- */
typedef struct orc_thermal_cfg {
    double alpha_fluid;   /* LB_ALPHA_FLUID = MU / Pr (clVariablesFD.cpp:457) */
    double alpha_foul;    /* LB_ALPHA_FOUL, fouling-layer diffusivity */
    double pr_turb_inv;   /* PR_TURB_NUMBER_INV = 1 / Pr_t */
    double t_in;          /* TFD_X_IN_VAL: inlet temperature, upper clamp of T */
} orc_thermal_cfg;

typedef struct orc_bicgstab_stats {
    int iters;        /* iterCount at exit */
    int checks;       /* convergence checks run */
    int conv;         /* converged (or b == 0) */
    int reset;        /* resetTimeFunc path taken */
    double residual;  /* last checked ||r||_1 / ||b||_1 */
    double initial_residual;
} orc_bicgstab_stats;

typedef struct orc_thermal_state {
    int steps_per_lb;          /* stepsPerLB */
    int time_since_change;     /* timeSinceTimeStepChange */
    double dt;                 /* timeStep */
    int max_iters;
    double rel_tol, abs_tol;
    int solves, resets;        /* of the last orc_thermal_solve */
    orc_bicgstab_stats last;
} orc_thermal_state;

/* CSR_Inds (non-periodic) with the thermal flags; same conventions as
 * orc_csr_build. */
int orc_csr_build_thermal(const orc_cfg* c, const int16_t* map, int32_t* IA,
                          int32_t* JA, int32_t* ind);
void orc_csr_fill_solid_boundary_thermal(const orc_cfg* c, const int16_t* map,
                                         const int32_t* ind, double* A);
/* Update_T_Coeffs_Implicit; nut may be NULL (no eddy diffusivity). */
void orc_thermal_coeffs(const orc_cfg* c, const orc_thermal_cfg* th, const int32_t* ind,
                        const int16_t* map, const double* dX0, double* A, double* b,
                        const double* T, const double* ux, const double* uy,
                        const double* nut, double dt);
void orc_bicgstab_solve(int n, const int32_t* IA, const int32_t* JA, const double* A,
                        double* b, double* x, int max_iters, double rel_tol, double abs_tol,
                        int reset_flag, orc_bicgstab_stats* st);
void orc_thermal_solve(const orc_cfg* c, const orc_thermal_cfg* th, orc_thermal_state* s,
                       const int16_t* map, const int32_t* IA, const int32_t* JA,
                       const int32_t* ind, const double* dX0, double* T, double* Tprev,
                       const double* ux, const double* uy, const double* nut, double* A,
                       double* b);

/* ---- discrete adjoint of the laminar step (kofm_adjoint.c) --------------- */
void orc_adj_collide(const orc_cfg* c, const int16_t* map, const double* FA, double* fstar);
void orc_adj_stream(const orc_cfg* c, const int16_t* map, const int32_t* ibb, const double* q,
                    int nibb, const double* fstar, double* FA);
void orc_adj_stream_T(const orc_cfg* c, const int16_t* map, const int32_t* ibb, const double* q,
                      int nibb, const double* lam, const double* fstar, double* nu, double* dq);
double orc_adj_j(const orc_cfg* c, const int16_t* map, const double* FA, const int32_t* snodes,
                 const double* cfss, int nshear, double* grad);
double orc_adj_run(const orc_cfg* c, const int16_t* map, const int32_t* ibb, const double* q,
                   int nibb, const double* FA0, int T, const int32_t* snodes, const double* cfss,
                   int nshear, double* dq, double* dF0);

double orc_sum(const double* a, int64_t n);
double orc_min(const double* a, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
