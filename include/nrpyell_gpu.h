/*
 * nrpyell_gpu.h -- C ABI of the B200 (sm_100a) hyperbolic-relaxation library.
 *
 * Part 1 keeps the reference prototypes of NRPyElliptic's hot path, so the
 * reference main.c links against libnrpyell_gpu.so unchanged.  Part 2 adds
 * set-up helpers, a stop-on-tolerance relaxation driver and the mixed
 * precision / batched drivers.  All gridfunction pointers handed to Part 1
 * and to the device drivers must be device-accessible (memory from the
 * allocators below, cudaMalloc or cudaMallocManaged); plain host memory is
 * rejected with an error, never dereferenced on the GPU.
 *
 * Errors: every CUDA call is checked.  By default an error prints
 * "file:line message" to stderr and calls exit(1), the reference's
 * convention for set-up failures; nrpyell_set_exit_on_error(0) turns that
 * into a recorded status (nrpyell_last_status / nrpyell_last_error).
 *
 * Threading: one host thread, one CUDA stream per process; calls run in
 * program order on that stream and, by default, return when their GPU work
 * is done (see nrpyell_set_async).
 */
#ifndef NRPYELL_GPU_H
#define NRPYELL_GPU_H

#include <stddef.h>
#include "nrpyell_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- Part 1: reference prototypes ---------------- */

/* Replaces MoL_malloc_y_n_gfs.c:7-14 (NRPy_function_prototypes.h:1): y_n_gfs in
 * CUDA managed memory, so host set-up code can still write it. */
void MoL_malloc_y_n_gfs(const paramstruct *NRPYELL_RESTRICT params, MoL_gridfunctions_struct *NRPYELL_RESTRICT gridfuncs);
/* Replaces MoL_free_memory_y_n_gfs.c:7-11. */
void MoL_free_memory_y_n_gfs(const paramstruct *NRPYELL_RESTRICT params, MoL_gridfunctions_struct *NRPYELL_RESTRICT gridfuncs);
/* Replaces MoL_malloc_non_y_n_gfs.c:7-17; diagnostic_output_gfs aliases
 * y_nplus1_running_total_gfs exactly as in the reference. */
void MoL_malloc_non_y_n_gfs(const paramstruct *NRPYELL_RESTRICT params, MoL_gridfunctions_struct *NRPYELL_RESTRICT gridfuncs);
/* Replaces MoL_free_memory_non_y_n_gfs.c:7-14. */
void MoL_free_memory_non_y_n_gfs(const paramstruct *NRPYELL_RESTRICT params, MoL_gridfunctions_struct *NRPYELL_RESTRICT gridfuncs);

/* Replaces MoL_step_forward_in_time.c:7-178: one RK4 step of (uu,vv). */
void MoL_step_forward_in_time(griddata_struct *NRPYELL_RESTRICT griddata, const REAL dt);

/* Replaces rhs_eval.c:7-117: interior RHS of (uu,vv); bitwise the reference's
 * operation order (every FMA, product and quotient as in rhs_eval.c:86-112). */
void rhs_eval(const paramstruct *NRPYELL_RESTRICT params, const rfm_struct *NRPYELL_RESTRICT rfmstruct,
              const REAL *NRPYELL_RESTRICT auxevol_gfs, const REAL *NRPYELL_RESTRICT in_gfs, REAL *NRPYELL_RESTRICT rhs_gfs);

/* Replaces apply_bcs_outerradiation_and_inner.c:410-469: radiation BC on the
 * RHS at pure outer points, layer by layer, then the inner parity copy. */
void apply_bcs_outerradiation_and_inner(const paramstruct *NRPYELL_RESTRICT params, const bc_struct *NRPYELL_RESTRICT bcstruct,
                                        REAL *NRPYELL_RESTRICT xx[3], const REAL custom_wavespeed[NUM_EVOL_GFS],
                                        const REAL custom_f_infinity[NUM_EVOL_GFS], REAL *NRPYELL_RESTRICT gfs,
                                        REAL *NRPYELL_RESTRICT rhs_gfs);

/* Replaces apply_bcs_inner_only.c:11-27. */
void apply_bcs_inner_only(const paramstruct *NRPYELL_RESTRICT params, const bc_struct *NRPYELL_RESTRICT bcstruct, REAL *NRPYELL_RESTRICT gfs);

/* Replaces apply_bcs_outerextrap_and_inner.c:15-75 (quadratic extrapolation). */
void apply_bcs_outerextrap_and_inner(const paramstruct *NRPYELL_RESTRICT params, const bc_struct *NRPYELL_RESTRICT bcstruct, REAL *NRPYELL_RESTRICT gfs);

/* Replaces residual_all_points.c:7-112 (bitwise reference operation order). */
void residual_all_points(const paramstruct *NRPYELL_RESTRICT params, const rfm_struct *NRPYELL_RESTRICT rfmstruct,
                         const REAL *NRPYELL_RESTRICT auxevol_gfs, const REAL *NRPYELL_RESTRICT in_gfs,
                         REAL *NRPYELL_RESTRICT residual_gf);

/* Replaces L2_norm_of_gf.c:6-43: log10(1e-16 + sqrt(sum g^2 dV / sum dV)) over
 * interior points with r < integration_radius.  Deterministic two-pass FP64
 * reduction (the result does not depend on thread counts). */
REAL L2_norm_of_gf(const paramstruct *NRPYELL_RESTRICT params, const int gf_index, const REAL integration_radius,
                   REAL *NRPYELL_RESTRICT xx[3], const REAL *NRPYELL_RESTRICT in_gf);

/* Same result as L2_norm_of_gf, for callers that may not allocate device
 * memory (no counterpart in the reference): all working memory is one
 * fixed-size array in the library (37.5 KB per GPU, held until exit), so no
 * cudaMalloc/cudaFree is ever called.  Grids are limited to 2048 x 2048
 * points in xx0 x xx1 (ghosts included), and Nxx_plus_2NGHOSTSi must equal
 * Nxxi + 2 NGHOSTS; other grids are rejected with an error and NaN before
 * any GPU work.  Calls share the array: calls that overlap on the GPU race.
 * Every call copies xx0/xx1 from pageable host memory and waits for its
 * result, so it must not be called while the library's stream (or the legacy
 * default stream) is being captured.  The first call on a device looks the
 * array up (cudaGetSymbolAddress); with CUDA's lazy module loading (the
 * default) that first lookup also loads the library's GPU code, which makes
 * the driver's own allocations for code and globals -- make the first call
 * at start-up, before a fixed arena or quota is in force, or run with
 * CUDA_MODULE_LOADING=EAGER for a strict guarantee. */
REAL L2_norm_of_gf_noalloc(const paramstruct *NRPYELL_RESTRICT params, const int gf_index,
                           const REAL integration_radius, REAL *NRPYELL_RESTRICT xx[3],
                           const REAL *NRPYELL_RESTRICT in_gf);

/* ---------------- Part 2: library extensions ---------------- */

/* Status and error policy. */
int nrpyell_last_status(void);          /* 0 = ok */
int nrpyell_gpu_last_status(void);      /* the same status under the harness name a drop-in shim exports */
const char *nrpyell_last_error(void);
void nrpyell_clear_status(void);
void nrpyell_set_exit_on_error(int enable);
/* Layout self-description for binding checks: writes up to n ints
 * {sizeof(paramstruct), sizeof(rfm_struct), sizeof(innerpt_bc_struct),
 *  sizeof(outerpt_bc_struct), sizeof(bc_info_struct), sizeof(bc_struct),
 *  sizeof(MoL_gridfunctions_struct), sizeof(griddata_struct),
 *  offsetof(paramstruct,Nxx0), offsetof(paramstruct,outer_bc_type),
 *  offsetof(griddata_struct,xx), offsetof(griddata_struct,bcstruct),
 *  offsetof(griddata_struct,rfmstruct), offsetof(griddata_struct,gridfuncs),
 *  NGHOSTS}; returns how many it wrote. */
int nrpyell_abi_layout(int *out, int n);
/* Number of kernel launches issued by this process so far. */
long long nrpyell_launch_count(void);
/* Number of device (cudaMalloc) and managed allocations the library has
 * made so far in this process. */
long long nrpyell_device_alloc_count(void);

/* How MoL_step_forward_in_time runs.
 *  NRPYELL_STEP_FUSED (default): per RK4 substep one fused RHS + update
 *    kernel over the interior, a radiation-BC column kernel for the outer
 *    face and an inner-ghost copy.  Inner ghost zones of y_n are treated as
 *    images of their source points (what apply_bcs_inner_only enforces).
 *  NRPYELL_STEP_REFERENCE_ORDER: rhs_eval, BCs and the all-points update in
 *    the reference's order and arithmetic, for arbitrary ghost contents. */
#define NRPYELL_STEP_FUSED 0
#define NRPYELL_STEP_REFERENCE_ORDER 1
void nrpyell_set_step_mode(int mode);
int nrpyell_get_step_mode(void);

/* Part-1 calls return after their GPU work has finished (default), like the
 * reference's functions, so the host may read managed gridfunctions right
 * away.  nrpyell_set_async(1) lets them return after enqueueing; the caller
 * then orders host access with nrpyell_synchronize(). */
void nrpyell_set_async(int enable);
/* Tile shape of the fused RK4 substep kernel.  By default the library times
 * every shape on the caller's grid the first time a grid size is stepped
 * and keeps the fastest.  nrpyell_set_tile(t) forces shape t (-1: autotune);
 * nrpyell_get_tile reports the shape in use for a grid (block 32 x by threads,
 * `planes` consecutive i2 planes per thread), -1 if not tuned yet; its fp32
 * argument selects FP64 (0), FP32 (1) or the FP32 correction form of
 * nrpyell_relax_mixed (2: marching shapes and the 8-warp direct shapes).
 * nrpyell_num_tiles gives the number of shapes; nrpyell_tile_info describes
 * shape t and returns -1 for an index out of range.  kind: 0 one thread per
 * (i0,i1) column of `planes` points reading its stencil through L1; 2 the
 * same with the pointwise inputs loaded before the first store; 4 the
 * block's uu planes staged in shared memory; 5 the block marches through `planes` i2 planes, each plane
 * and its pointwise inputs copied into shared memory ahead of use by
 * asynchronous copies. */
void nrpyell_set_tile(int tile);
/* Programmatic dependent launch of the fused substep kernels (default on):
 * each substep kernel may be scheduled while the previous one drains and
 * waits on the device (griddepcontrol.wait) before reading its results, so
 * the launch gap between the four substeps of an RK4 step is hidden.  Results
 * are identical either way; 0 turns it off (cached relaxation graphs are
 * dropped and captured again). */
void nrpyell_set_programmatic_launch(int on);
int nrpyell_get_programmatic_launch(void);
int nrpyell_get_tile(const paramstruct *params, int fp32, int *bx, int *by, int *planes);
int nrpyell_num_tiles(void);
int nrpyell_tile_info(int tile, int *by, int *planes, int *kind);
/* Selects the CUDA device used by every later call (default: device 0).
 * Call before any other GPU work in the process. */
int nrpyell_set_device(int device);
/* Waits for all queued GPU work of the library. */
void nrpyell_synchronize(void);
/* Drops every cached device table (rfm, BC maps, L2 weights, scratch). */
void nrpyell_release_tables(void);

/* Device / pinned memory for callers that keep gridfunctions resident. */
void *nrpyell_device_malloc(size_t bytes);
void nrpyell_device_free(void *ptr);
void *nrpyell_host_pinned_malloc(size_t bytes);
void nrpyell_host_pinned_free(void *ptr);
/* kind: 0 host->device, 1 device->host, 2 device->device, 3 default. */
int nrpyell_memcpy(void *dst, const void *src, size_t bytes, int kind);
int nrpyell_memset(void *dst, int value, size_t bytes);

/* Set-up, restated from the reference's generated set-up code (host). */
void nrpyell_set_Cparameters_to_default(paramstruct *params);                 /* set_Cparameters_to_default.c:5-86 */
void nrpyell_set_Nxx_dxx_invdx_params__and__xx(const int EigenCoord, const int Nxx[3], paramstruct *params,
                                               REAL *xx[3]);                  /* set_Nxx_dxx_invdx_params__and__xx.c:5-54 */
void nrpyell_free_xx(REAL *xx[3]);
void nrpyell_bcstruct_set_up(const paramstruct *params, bc_struct *bcstruct);   /* bcstruct_set_up.c:350-521 */
void nrpyell_bcstruct_free(bc_struct *bcstruct);
void nrpyell_rfm_precompute_rfmstruct_malloc(const paramstruct *params, rfm_struct *rfmstruct);
void nrpyell_rfm_precompute_rfmstruct_define(const paramstruct *params, REAL *xx[3], rfm_struct *rfmstruct); /* rfm_precompute_rfmstruct_define.c */
void nrpyell_rfm_precompute_rfmstruct_freemem(const paramstruct *params, rfm_struct *rfmstruct);
REAL nrpyell_find_timestep(const paramstruct *params, REAL *xx[3], const REAL CFL_FACTOR);               /* find_timestep.c:5-46 */
void nrpyell_auxevol_gfs_all_points(const paramstruct *params, REAL *xx[3], REAL *auxevol_gfs);         /* auxevol_gfs_all_points.c */
void nrpyell_wavespeed_gf_all_points(const paramstruct *params, const REAL CFL_FACTOR, const REAL dt, REAL *xx[3],
                                     REAL *auxevol_gfs);                                                /* wavespeed_gf_all_points.c */
REAL nrpyell_compute_wavespeed_at_OB(const paramstruct *params, const REAL *auxevol_gfs);               /* compute_wavespeed_at_OB.c */
/* The three auxevol gridfunctions computed on the GPU straight into device
 * memory (auxevol_gfs: 3 Ntot doubles): psi_background and ADD_times_AUU at
 * all points, the wavespeed CFL_FACTOR * min(ds) / dt on the interior and 0
 * in the ghost zones -- the nrpyell_auxevol_gfs_all_points and
 * nrpyell_wavespeed_gf_all_points results without host arrays or copies. */
int nrpyell_auxevol_device(const paramstruct *params, REAL *xx[3], const REAL CFL_FACTOR, const REAL dt,
                           REAL *auxevol_gfs);

/* Stop-on-tolerance relaxation on device-resident gridfunctions.
 * For n = 0, 1, ..., max_steps: evaluate the residual of y_n and its L2 norm
 * (integration_radius as in L2_norm_of_gf); stop when log10 L2 <= log10_tol,
 * otherwise take one RK4 step (main.c:138-187 order, plus the stop test of the
 * Einstein Toolkit driver).  griddata->params must already carry the
 * wavespeeds at the outer boundary.  history (nullable) receives log10 L2 of
 * every evaluated n (max_steps+1 entries).  Returns 0 when converged, 1 when
 * max_steps was reached, negative on error. */
int nrpyell_relax(griddata_struct *griddata, const REAL dt, const REAL log10_tol, const int max_steps,
                  const REAL integration_radius, int *steps_taken, REAL *final_log10_l2, REAL *history);

/* Mixed-precision relaxation to log10 L2 <= log10_tol, main.c's stop test
 * (residual before each step).  The state y_n stays FP64; the FP32 phase
 * relaxes a correction to it (defect correction):
 *   1. from the FP64 state U: its RHS with the radiation BC, its residual
 *      bracket (residual_all_points) and log10 L2, all in FP64, and the
 *      stop test on that norm;
 *   2. an FP32 correction d starts at zero and takes up to fold_every RK4
 *      steps of the same equations written for U + d, with U's FP64 RHS as a
 *      fixed input, so FP32 rounding scales with d, not with U; its own
 *      (FP32-evaluated) residual is tested against log10_switch each step;
 *   3. U += d in FP64, and back to 1.
 * Once the FP64 residual of U is <= log10_switch, or an FP32 stretch met
 * log10_switch by its own evaluation or made no progress, FP64 RK4 steps
 * (the plain fused kernels) continue from U to log10_tol.  log10_switch =
 * log10_tol keeps every step in FP32, with the FP64 norm as the judge.
 * steps_fp32 / steps_fp64 receive the RK4 steps of each phase; history
 * (nullable) log10 L2 per step (FP64 values at the fold steps, the FP32
 * evaluation in between).  1 <= fold_every <= 4096; grids with
 * 3 Ntot >= 2^32 are rejected.  Returns as nrpyell_relax. */
int nrpyell_relax_mixed(griddata_struct *griddata, const REAL dt, const REAL log10_tol, const REAL log10_switch,
                        const int fold_every, const int max_steps, const REAL integration_radius, int *steps_fp32,
                        int *steps_fp64, REAL *final_log10_l2, REAL *history);

/* The same relaxation with the stopping rule of the Einstein Toolkit thorn
 * (NRPyEllipticET_conformally_flat_BBH_Hyperbolic_Relaxation.c:185-217):
 * its loop n = 0..max_iterations takes one RK4 step, then, when n is a
 * multiple of check_every or n == max_iterations, evaluates the residual of
 * the new state and stops once log10 L2 < log_target_residual (strictly).
 * *iterations = the n of the last test; returns 0 when the target was met, 1
 * when it was not (the thorn errors out there), < 0 on error. */
int nrpyell_relax_et(griddata_struct *griddata, const REAL dt, const REAL log_target_residual, const int max_iterations,
                     const int check_every, const REAL integration_radius, int *iterations, REAL *final_log10_l2);
/* Damping parameter of arXiv:2111.02424 (the thorn's
 * conformally_flat_BBH_set_optimum_eta_damping.c:3-27): TRC from Eq. (B6),
 * eta = 6.9 TRC^-0.79 - 0.7 from Eq. (36), fitted for AMAX = 1e6,
 * SINHWAA = 0.07 and bScale = 5; writes params->eta_damping. */
REAL nrpyell_compute_TRC(const REAL A, const REAL b, const REAL C_0, const REAL dt, const REAL dxx1, const REAL dxx2);
void nrpyell_set_optimum_eta_damping(const REAL dt, const REAL CFL_FACTOR, paramstruct *params);
/* Device tables of a grid built on the GPU (the batch set-up path): the
 * reference-metric arrays and folded RHS weights, the inner-boundary map
 * (SymTP images, parity +1) and the pure outer points of the x0max face with
 * their radiation geometry -- the roles of rfm_precompute_rfmstruct_define.c:5-93
 * and bcstruct_set_up.c:350-521 -- from params and xx alone.  rfm and bc
 * are the structs the caller will pass to the drivers (griddata->rfmstruct,
 * ->bcstruct); they are not read, only used as cache keys, and may be left
 * zeroed (no host arrays).  Call after the grid is set up and before any
 * driver, with the same params and xx.  Requires Nxx2 even and >= NGHOSTS,
 * Nxx0 >= 12, radiation outer BCs.  Returns 0 or -1. */
int nrpyell_setup_tables_device(const paramstruct *params, REAL *xx[3], const rfm_struct *rfm, const bc_struct *bc);
/* Copies one device table of a grid to host memory (built from the host
 * structs first if it does not exist): what = 0 inner map (dst, src) int32
 * pairs, 1 inner parity int8, 2 pure outer points as 8 int32 (which_gz, dirn,
 * i0, i1, i2, FACEX0, FACEX1, FACEX2, in the reference's list order), 3 their
 * geometry as 6 doubles (r, dxx0/dr, dxx1/dr at the point and at its interior
 * neighbour), 4 column geometry [3][6][N1], 5..13 f0, f0', f0'', f3, f3', f1,
 * f1', f2, d f2/d xx0, 14 folded RHS weights [6][N0 N1].  capacity in
 * elements; returns the number of elements written, -1 on error. */
long long nrpyell_device_tables_read(const paramstruct *params, REAL *xx[3], const rfm_struct *rfm,
                                     const bc_struct *bc, int what, void *host_out, long long capacity);
/* Solution export (the Einstein Toolkit thorn's Initialize_ADMBase role,
 * without Cactus): for npts Cartesian points xyz (host, x y z per point, in
 * this code's frame), uu by Lagrange interpolation of the given order (1..8;
 * the thorn's default is 4) on the (xx0,xx1,xx2) grid including ghost zones
 * from uu (device: the uu gridfunction of a y_n whose ghost zones are
 * filled, as the relaxation drivers leave it), and the ADM quantities of the
 * conformally flat data: psi = psi_background + uu, gamma_ij = psi^4
 * delta_ij, K_ij = psi^-2 Abar_ij (Bowen-York; beta = 0).  Outputs (host,
 * each optional): uu_out, psi_out [npts]; gamma_out, K_out [6 npts] in the
 * order xx xy xz yy yz zz. */
int nrpyell_interpolate_solution(const paramstruct *params, REAL *xx[3], const REAL *uu, int npts, const REAL *xyz,
                                 int order, REAL *uu_out, REAL *psi_out, REAL *gamma_out, REAL *K_out);
/* Initial lapse at npts Cartesian points (host arrays), the thorn's
 * initial_lapse options (conformally_flat_BBH_compute_ADM_Cartesian_quantities_from_uu.c:25-29):
 *  NRPYELL_LAPSE_PSI_POWER ("NRPyEllipticET-psi^n",
 *    conformally_flat_BBH_lapse_power_of_psi_initial_data.c):
 *    alpha = (1 + m0/(2 r0) + m1/(2 r1) + uu)^lapse_exponent, uu_at_points
 *    from nrpyell_interpolate_solution (the thorn's default exponent is -2);
 *  NRPYELL_LAPSE_AVERAGED ("NRPyEllipticET-averaged",
 *    conformally_flat_BBH_lapse_averaged_initial_data.c):
 *    alpha = (1 - s)/(2 (1 + s)) + 1/2 with s = m0/(2 r0) + m1/(2 r1);
 *    uu_at_points and lapse_exponent are not used (may be NULL / 0).
 * r_i is the distance to puncture i.  Returns 0, or -1 on bad arguments. */
#define NRPYELL_LAPSE_PSI_POWER 0
#define NRPYELL_LAPSE_AVERAGED 1
int nrpyell_initial_lapse(const paramstruct *params, int npts, const REAL *xyz, const REAL *uu_at_points, int mode,
                          REAL lapse_exponent, REAL *alpha_out);
/* Batched relaxation: n configurations, each a griddata_struct set up as for
 * nrpyell_relax (its own grid size, parameters, bc_struct, rfm_struct and
 * device gridfunctions; dt[c] its time step), relaxed together from their
 * y_n_gfs to log10 L2 <= log10_tol or max_steps.  Every RK4 substep of all
 * configurations is one kernel launch (a shared-memory planes or marching
 * shape, autotuned on the batch or forced by nrpyell_set_tile); each
 * configuration stops on its own.
 * steps_taken[c] and final_log10_l2[c] as in nrpyell_relax.  Returns the
 * number of configurations that did not converge (0: all did), < 0 on
 * error. */
int nrpyell_relax_batch(int n, griddata_struct *grids, const REAL *dt, REAL log10_tol, int max_steps,
                        REAL integration_radius, int *steps_taken, REAL *final_log10_l2);
/* nrpyell_relax_mixed on a batch: each configuration follows the
 * single-grid schedule (FP64 evaluation and stop test of its base state, an
 * FP32 correction stretch of up to fold_every steps or to log10_switch, the
 * fold; FP64 steps from the switch on), and the stretches of all
 * configurations still in the FP32 phase, then their FP64 phases, run as
 * batches (marching shapes for the FP32 stretches).  With the same tile
 * shapes each configuration's result is bitwise that of nrpyell_relax_mixed.
 * steps_fp32[c], steps_fp64[c], final_log10_l2[c] as there (each array may
 * be NULL); the FP32 buffers (13 Ntot floats per configuration) stay
 * allocated for later calls until nrpyell_release_tables.  Returns the number
 * of configurations that did not converge, < 0 on error. */
int nrpyell_relax_batch_mixed(int n, griddata_struct *grids, const REAL *dt, REAL log10_tol, REAL log10_switch,
                              int fold_every, int max_steps, REAL integration_radius, int *steps_fp32,
                              int *steps_fp64, REAL *final_log10_l2);
/* Learned initial guess (BF16 tensor-core MLP, FP32 master weights, Adam).
 * The network maps n_in inputs through `depth` tanh layers of `width` to
 * n_out linear outputs.  All arrays are device pointers unless named host.
 * Parameters are stored layer by layer: W [in x out] row-major, then b. */
void *nrpyell_mlp_create(int n_in, int width, int depth, int n_out, int batch_max, unsigned seed);
void nrpyell_mlp_destroy(void *mlp);
long long nrpyell_mlp_num_params(void *mlp);
int nrpyell_mlp_get_params(void *mlp, float *host);
int nrpyell_mlp_set_params(void *mlp, const float *host);
/* y [n x n_out] = network(x [n x n_in]). */
int nrpyell_mlp_predict(void *mlp, const float *x, int n, float *y);
/* Mean squared error of one batch and its parameter gradient (copied to
 * grad_host when non-NULL); 0 < rows <= batch_max. */
double nrpyell_mlp_loss_grad(void *mlp, const float *x, const float *t, int rows, float *grad_host);
/* Adam over `epochs` passes of seeded, shuffled minibatches (cosine decay of
 * the learning rate to lr/100); returns the last epoch's mean loss and
 * writes every epoch's to loss_history (host, optional). */
double nrpyell_mlp_train(void *mlp, const float *x, const float *t, int n, int batch, int epochs, float lr,
                         unsigned seed, double *loss_history);
/* y_n of one configuration from K <= 4096 POD coefficients c: uu = mean +
 * sum_k c_k basis_k (mean [Ntot], basis [K x Ntot], FP32), vv = eta uu. */
int nrpyell_pod_guess(const float *mean, const float *basis, int K, long long ntot, const float *c, double eta,
                      double *y_n);
/* The same solve with host buffers: copies auxevol_host (3 gfs) and
 * y_n_host (2 gfs, the initial guess) to the device, relaxes, copies the
 * solution back into y_n_host.  The library keeps one set of device
 * gridfunction buffers between calls, reallocated when the point count
 * changes.  Its device tables are cached by the addresses of the caller's
 * bc_struct / rfm_struct arrays and xx plus the grid parameters: a caller
 * that frees those arrays and reallocates them at the same addresses for a
 * different grid must call nrpyell_release_tables() before the next call. */
int nrpyell_relax_host(const paramstruct *params, REAL *xx[3], const bc_struct *bcstruct, const rfm_struct *rfmstruct,
                       const REAL *auxevol_host, REAL *y_n_host, const REAL dt, const REAL log10_tol, const int max_steps,
                       const REAL integration_radius, int *steps_taken, REAL *final_log10_l2);

/* Timing on the library's stream.  nrpyell_event_record(slot) records CUDA
 * event `slot` (0..15); nrpyell_event_elapsed_ms(a, b) waits for event b and
 * returns the device time from a to b in milliseconds. */
int nrpyell_event_record(int slot);
float nrpyell_event_elapsed_ms(int a, int b);
/* Writes a 256 MiB device buffer, evicting the 126 MB L2 (benchmark hygiene). */
void nrpyell_flush_l2(void);
/* Copy bandwidth of the GPU in GB/s (bytes read + written per second): a
 * 16-byte-vector copy kernel between two buffers of bytes/2 each, repeated
 * within one launch until about 1 GiB has moved, best of `iters` timed
 * launches after a warm-up.  A footprint below the L2 size measures L2
 * bandwidth, a larger one HBM bandwidth.  Allocates and frees its buffers. */
double nrpyell_copy_bandwidth(size_t bytes, int iters);
/* Device time of the fused RK4 pieces on griddata's buffers, averaged over
 * n_iter launches replayed from a CUDA graph (the buffers are modified):
 *   ms_interior: one fused interior kernel of RK4 stage `stage` (1..4)
 *   ms_step:     one whole RK4 step (4 stages x interior/outer-BC/ghost kernels) */
int nrpyell_time_fused(griddata_struct *griddata, const REAL dt, const int stage, const int n_iter, double *ms_interior,
                       double *ms_step);

#ifdef __cplusplus
}
#endif

#endif /* NRPYELL_GPU_H */
