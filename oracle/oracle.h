/*
 * oracle.h -- CPU restatement of the reference flow solver (test
 * infrastructure only).
 *
 * This is the checker the GPU library is compared against.  It is a plain
 * FP64 C++ restatement of the Fortran routines of SolverSource/
 * mgnsg3d_def_par.F90 and mgnsg3d_mg_par.F90 on the hot path, in the
 * reference's own operation order (edge-order scatter, left-to-right
 * evaluation, no FMA contraction).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it.  Parity is pinned by the reference's
 * own invariants and analytic known answers (the reference ships no tests,
 * fixtures or outputs and cannot be compiled here: there is no Fortran
 * compiler), see tests/golden/.
 */
#ifndef FLITE_ORACLE_H
#define FLITE_ORACLE_H
#include "flite_gpu.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct oracle_ctx oracle_ctx;
int oracle_create(const flite_controls *c, int nlevels, const flite_level_desc *lv,
                  oracle_ctx **out);
int oracle_destroy(oracle_ctx *o);
int oracle_set_state(oracle_ctx *o, int level, const double *u);
int oracle_get_state(oracle_ctx *o, int level, double *u);
int oracle_explicit_time_step(oracle_ctx *o, double *dt);
int oracle_get_pressure(oracle_ctx *o, int level, double *p);
/* named per-level arrays: "dt", "diss", "rhs", "uprev", "src", "normal",
 * "wallArea", "conn", "mu", "grad" (15 columns of nodeHelpArray)          */
int oracle_get_array(oracle_ctx *o, int level, const char *name, double *out);
int oracle_init_freestream(oracle_ctx *o);
int oracle_start(oracle_ctx *o);
int oracle_do_time_iterations(oracle_ctx *o, int level, int nsteps, int calc_diss,
                              int calc_turb, int cycle_no);
int oracle_restrict(oracle_ctx *o, int fine_level, int calc_turb);
int oracle_prolong(oracle_ctx *o, int coarse_level);
int oracle_map_fine_to_coarse(oracle_ctx *o, int fine_level);
int oracle_cycle(oracle_ctx *o, int cycle_no);
/* unsteady runs: close the physical time step, open the next one          */
int oracle_next_physical_step(oracle_ctx *o);
int oracle_update_geometry(oracle_ctx *o, int nlevels, const flite_level_desc *levels);
int oracle_residuals(oracle_ctx *o, double res[7], double maxres[7], int maxind[7]);
int oracle_forces(oracle_ctx *o, double out[9]);
int oracle_residual_fwd(oracle_ctx *o, int level, const double *u, double *r);
/* the artificial dissipation (time steps, then the run's scheme) at the state u */
int oracle_dissipation(oracle_ctx *o, int level, const double *u, double *diss);
/* makeViscosityTerm alone at the state u: diss [5][N] (subtracted from
 * zero), the laminar viscosity mu [N] and the wall stress [3][N] (level 1) */
int oracle_viscous_term(oracle_ctx *o, int level, const double *u, double *diss, double *mu,
                        double *wall_stress);
/* nodeHelpArray(:, col + 1) of level 1 after the last evaluation */
int oracle_help_column(oracle_ctx *o, int col, double *out);
/* pinned exp (which 0) / log (which 1) of the SA source term            */
int oracle_pinned_math(int which, const double *x, double *y, int n);
/* threads of the timing mode (default 1 = the reference's loop order)  */
int oracle_set_threads(int n);
/* tangent (forward-mode) of the residual: jv = (dR/du) du               */
int oracle_residual_jvp(oracle_ctx *o, int level, const double *u, const double *du, double *jv);
/* tangent of one smoother iteration on level 1 (central flux, scalar JST,
 * inviscid or laminar): v = G(u, mu), dv = G_u du + G_mu dmu + G_g dg with
 * dg = (dsw [3][E], dbw [3][B], dvol [N]) a direction in the level-1
 * geometry (NULL = zero); in a laminar run mu [N] is the viscosity the time
 * step reads, and mu_out = the viscosity of u with its tangent dmu_out      */
int oracle_iteration_jvp(oracle_ctx *o, const double *u, const double *du, const double *dsw,
                         const double *dbw, const double *dvol, double *v, double *dv,
                         const double *mu, const double *dmu, double *mu_out, double *dmu_out);
/* lift (which 0) or drag (1) coefficient of u (pressure and, in laminar
 * runs, wall stress) and its tangent along (du, dsw, dbw, dvol)            */
int oracle_objective_jvp(oracle_ctx *o, int which, const double *u, const double *du,
                         const double *dsw, const double *dbw, const double *dvol, double *J, double *dJ);
#ifdef __cplusplus
}
#endif
#endif
