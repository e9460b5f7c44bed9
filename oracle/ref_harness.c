/*
 * ref_harness.c -- driver around a build of the reference's own C sources.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/build.py compiles this file together with
 * NRPyElliptic_Ccodes/*.c (all but main.c) from the reference checkout into
 * oracle/_ref/libnrpyell_ref_*.so.  The tests use it to generate golden
 * vectors, and bench.py's reference arm uses it to time the reference CPU
 * implementation.  It only sequences reference functions the way
 * NRPyElliptic_Ccodes/main.c:14-187 does, with run-time parameters instead
 * of free_parameters.h.
 */
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "nrpyell_abi.h"

/* Reference prototypes, NRPyElliptic_Ccodes/NRPy_function_prototypes.h. */
void set_Cparameters_to_default(paramstruct *params);
void set_Nxx_dxx_invdx_params__and__xx(const int EigenCoord, const int Nxx[3], paramstruct *params, REAL *NRPYELL_RESTRICT xx[3]);
void bcstruct_set_up(const paramstruct *params, REAL *NRPYELL_RESTRICT xx[3], bc_struct *bcstruct);
REAL find_timestep(const paramstruct *params, REAL *NRPYELL_RESTRICT xx[3], const REAL CFL_FACTOR);
void MoL_malloc_y_n_gfs(const paramstruct *params, MoL_gridfunctions_struct *gridfuncs);
void MoL_malloc_non_y_n_gfs(const paramstruct *params, MoL_gridfunctions_struct *gridfuncs);
void MoL_free_memory_y_n_gfs(const paramstruct *params, MoL_gridfunctions_struct *gridfuncs);
void MoL_free_memory_non_y_n_gfs(const paramstruct *params, MoL_gridfunctions_struct *gridfuncs);
void rfm_precompute_rfmstruct_malloc(const paramstruct *params, rfm_struct *rfmstruct);
void rfm_precompute_rfmstruct_define(const paramstruct *params, REAL *NRPYELL_RESTRICT xx[3], rfm_struct *rfmstruct);
void rfm_precompute_rfmstruct_freemem(const paramstruct *params, rfm_struct *rfmstruct);
void initial_guess_all_points(const paramstruct *params, REAL *NRPYELL_RESTRICT xx[3], REAL *in_gfs);
void auxevol_gfs_all_points(const paramstruct *params, REAL *NRPYELL_RESTRICT xx[3], REAL *auxevol_gfs);
void wavespeed_gf_all_points(const paramstruct *params, const REAL CFL_FACTOR, const REAL dt, REAL *NRPYELL_RESTRICT xx[3],
                             REAL *auxevol_gfs);
REAL compute_wavespeed_at_OB(const paramstruct *params, REAL *auxevol_gfs);
void residual_all_points(const paramstruct *params, const rfm_struct *rfmstruct, const REAL *auxevol_gfs,
                         const REAL *in_gfs, REAL *residual_gf);
REAL L2_norm_of_gf(const paramstruct *params, const int gf_index, const REAL integration_radius, REAL *NRPYELL_RESTRICT xx[3],
                   const REAL *in_gf);
void MoL_step_forward_in_time(griddata_struct *griddata, const REAL dt);

/* main.c:14-105 with the physical parameters taken from *phys (only the
 * puncture, metric and damping fields are read). */
double refh_setup(griddata_struct *g, const int Nxx[3], const paramstruct *phys, double CFL_FACTOR) {
  memset(g, 0, sizeof(*g));
  set_Cparameters_to_default(&g->params);
  g->params.outer_bc_type = RADIATION_OUTER_BCS;
  g->params.time = 0.0;
  g->params.AMAX = phys->AMAX;
  g->params.SINHWAA = phys->SINHWAA;
  g->params.bScale = phys->bScale;
  g->params.eta_damping = phys->eta_damping;
  g->params.bare_mass_0 = phys->bare_mass_0;
  g->params.bare_mass_1 = phys->bare_mass_1;
  g->params.puncture_0_x = phys->puncture_0_x;
  g->params.puncture_0_y = phys->puncture_0_y;
  g->params.puncture_0_z = phys->puncture_0_z;
  g->params.puncture_1_x = phys->puncture_1_x;
  g->params.puncture_1_y = phys->puncture_1_y;
  g->params.puncture_1_z = phys->puncture_1_z;
  g->params.P0_x = phys->P0_x; g->params.P0_y = phys->P0_y; g->params.P0_z = phys->P0_z;
  g->params.P1_x = phys->P1_x; g->params.P1_y = phys->P1_y; g->params.P1_z = phys->P1_z;
  g->params.S0_x = phys->S0_x; g->params.S0_y = phys->S0_y; g->params.S0_z = phys->S0_z;
  g->params.S1_x = phys->S1_x; g->params.S1_y = phys->S1_y; g->params.S1_z = phys->S1_z;
  set_Nxx_dxx_invdx_params__and__xx(1, Nxx, &g->params, g->xx);
  bcstruct_set_up(&g->params, g->xx, &g->bcstruct);
  for (int i = 0; i < 3; i++) free(g->xx[i]);
  set_Nxx_dxx_invdx_params__and__xx(0, Nxx, &g->params, g->xx);
  const double dt = find_timestep(&g->params, g->xx, CFL_FACTOR);
  MoL_malloc_y_n_gfs(&g->params, &g->gridfuncs);
  rfm_precompute_rfmstruct_malloc(&g->params, &g->rfmstruct);
  rfm_precompute_rfmstruct_define(&g->params, g->xx, &g->rfmstruct);
  initial_guess_all_points(&g->params, g->xx, g->gridfuncs.y_n_gfs);
  MoL_malloc_non_y_n_gfs(&g->params, &g->gridfuncs);
  auxevol_gfs_all_points(&g->params, g->xx, g->gridfuncs.auxevol_gfs);
  wavespeed_gf_all_points(&g->params, CFL_FACTOR, dt, g->xx, g->gridfuncs.auxevol_gfs);
  const double c = compute_wavespeed_at_OB(&g->params, g->gridfuncs.auxevol_gfs);
  g->params.uu_wavespeed_at_OB = c;
  g->params.vv_wavespeed_at_OB = c;
  return dt;
}

void refh_free(griddata_struct *g) {
  rfm_precompute_rfmstruct_freemem(&g->params, &g->rfmstruct);
  free(g->bcstruct.inner_bc_array);
  for (int i = 0; i < NGHOSTS * 3; i++) free(g->bcstruct.pure_outer_bc_array[i]);
  MoL_free_memory_y_n_gfs(&g->params, &g->gridfuncs);
  MoL_free_memory_non_y_n_gfs(&g->params, &g->gridfuncs);
  for (int i = 0; i < 3; i++) free(g->xx[i]);
}

/* main.c:138-187 plus a stop test: residual + L2 of y_n, then one RK4 step. */
int refh_relax(griddata_struct *g, double dt, double log10_tol, int max_steps, double R, double *history,
               int *steps_taken) {
  int n, converged = 0;
  for (n = 0; n <= max_steps; n++) {
    g->params.time = ((REAL)n) * dt;
    residual_all_points(&g->params, &g->rfmstruct, g->gridfuncs.auxevol_gfs, g->gridfuncs.y_n_gfs,
                        g->gridfuncs.diagnostic_output_gfs);
    const double l2 = L2_norm_of_gf(&g->params, UUGF, R, g->xx, g->gridfuncs.diagnostic_output_gfs);
    if (history) history[n] = l2;
    if (l2 <= log10_tol) {
      converged = 1;
      break;
    }
    if (n == max_steps) break;
    MoL_step_forward_in_time(g, dt);
  }
  if (steps_taken) *steps_taken = n;
  return converged ? 0 : 1;
}

/* Wall time of n_iter iterations of the main.c loop body (residual, L2, RK4
 * step), no file output. */
double refh_time_iterations(griddata_struct *g, double dt, int n_iter, double R) {
  const double t0 = omp_get_wtime();
  for (int n = 0; n < n_iter; n++) {
    residual_all_points(&g->params, &g->rfmstruct, g->gridfuncs.auxevol_gfs, g->gridfuncs.y_n_gfs,
                        g->gridfuncs.diagnostic_output_gfs);
    volatile double l2 = L2_norm_of_gf(&g->params, UUGF, R, g->xx, g->gridfuncs.diagnostic_output_gfs);
    (void)l2;
    MoL_step_forward_in_time(g, dt);
  }
  return omp_get_wtime() - t0;
}

int refh_max_threads(void) { return omp_get_max_threads(); }
void refh_set_threads(int n) { omp_set_num_threads(n); }
