/*
 * nrpyell_abi.h -- data types shared with NRPyElliptic's generated C code.
 *
 * Every struct here has the same members, types and order as the
 * reference's NRPyElliptic_Ccodes/NRPy_basic_defines.h, so that a caller
 * compiled against the reference header (for example the reference main.c
 * and its set-up objects) can hand its griddata_struct straight to the GPU
 * library.  Sizes and offsets are checked by the test suite through
 * nrpyell_abi_layout().
 *
 *   paramstruct              NRPy_basic_defines.h:40-120  (72 REAL, 8 int)
 *   rfm_struct               NRPy_basic_defines.h:135-151
 *   innerpt/outerpt/bc_*     NRPy_basic_defines.h:164-195
 *   MoL_gridfunctions_struct NRPy_basic_defines.h:206-213
 *   griddata_struct          NRPy_basic_defines.h:263-269
 *   NGHOSTS, gf indices      NRPy_basic_defines.h:129,161-162,222-235
 */
#ifndef NRPYELL_ABI_H
#define NRPYELL_ABI_H

#include <stdint.h>

#ifdef __cplusplus
#define NRPYELL_RESTRICT __restrict__
extern "C" {
#else
#define NRPYELL_RESTRICT restrict
#endif

#ifndef REAL
#define REAL double
#endif

/* Ghost-zone width of the 10th-order centred stencil (radius 5). */
#ifndef NGHOSTS
#define NGHOSTS 5
#endif

#define EXTRAPOLATION_OUTER_BCS 0
#define RADIATION_OUTER_BCS 1

#define NUM_EVOL_GFS 2
#define UUGF 0
#define VVGF 1
#define NUM_AUX_GFS 0
#define NUM_AUXEVOL_GFS 3
#define ADD_TIMES_AUUGF 0
#define PSI_BACKGROUNDGF 1
#define WAVESPEEDGF 2

typedef struct __paramstruct__ {
  REAL AMAX;
  REAL Cart_CoM_offsetx, Cart_CoM_offsety, Cart_CoM_offsetz;
  REAL Cart_originx, Cart_originy, Cart_originz;
  REAL P0_x, P0_y, P0_z;
  REAL P1_x, P1_y, P1_z;
  REAL S0_x, S0_y, S0_z;
  REAL S1_x, S1_y, S1_z;
  REAL SINHWAA;
  REAL bScale;
  REAL bare_mass_0, bare_mass_1;
  REAL dxx0, dxx1, dxx2;
  REAL eta_damping;
  REAL f0_of_xx0, f0_of_xx0__D0, f0_of_xx0__DD00, f0_of_xx0__DDD000;
  REAL f1_of_xx1, f1_of_xx1__D1, f1_of_xx1__DD11, f1_of_xx1__DDD111;
  REAL f2_of_xx0_xx1, f2_of_xx0_xx1__D0, f2_of_xx0_xx1__D1, f2_of_xx0_xx1__DD00, f2_of_xx0_xx1__DD11;
  REAL f2_of_xx1, f2_of_xx1__D1, f2_of_xx1__DD11, f2_of_xx1__DDD111;
  REAL f3_of_xx0, f3_of_xx0__D0, f3_of_xx0__DD00;
  REAL f4_of_xx2, f4_of_xx2__D2, f4_of_xx2__DD22;
  REAL invdx0, invdx1, invdx2;
  REAL puncture_0_x, puncture_0_y, puncture_0_z;
  REAL puncture_1_x, puncture_1_y, puncture_1_z;
  REAL time;
  REAL uu_wavespeed_at_OB, vv_wavespeed_at_OB;
  REAL xx0, xx1, xx2;
  REAL xxmax0, xxmax1, xxmax2;
  REAL xxmin0, xxmin1, xxmin2;
  int Nxx0, Nxx1, Nxx2;
  int Nxx_plus_2NGHOSTS0, Nxx_plus_2NGHOSTS1, Nxx_plus_2NGHOSTS2;
  int has_outer_boundary;
  int outer_bc_type;
} paramstruct;

/* Precomputed SinhSymTP scale factors: 1-D in xx0 or xx1, 2-D in (xx0,xx1)
 * with index i0 + Nxx_plus_2NGHOSTS0*i1. */
typedef struct __rfmstruct__ {
  REAL *NRPYELL_RESTRICT f0_of_xx0;
  REAL *NRPYELL_RESTRICT f0_of_xx0__D0;
  REAL *NRPYELL_RESTRICT f0_of_xx0__DD00;
  REAL *NRPYELL_RESTRICT f0_of_xx0__DDD000;
  REAL *NRPYELL_RESTRICT f1_of_xx1;
  REAL *NRPYELL_RESTRICT f1_of_xx1__D1;
  REAL *NRPYELL_RESTRICT f1_of_xx1__DD11;
  REAL *NRPYELL_RESTRICT f2_of_xx0_xx1;
  REAL *NRPYELL_RESTRICT f2_of_xx0_xx1__D0;
  REAL *NRPYELL_RESTRICT f2_of_xx0_xx1__D1;
  REAL *NRPYELL_RESTRICT f2_of_xx0_xx1__DD00;
  REAL *NRPYELL_RESTRICT f2_of_xx0_xx1__DD11;
  REAL *NRPYELL_RESTRICT f3_of_xx0;
  REAL *NRPYELL_RESTRICT f3_of_xx0__D0;
  REAL *NRPYELL_RESTRICT f3_of_xx0__DD00;
} rfm_struct;

/* One inner-boundary ghost point: dst takes parity[type] * src. */
typedef struct __innerpt_bc_struct__ {
  int dstpt;
  int srcpt;
  int8_t parity[10];
} innerpt_bc_struct;

/* One pure-outer ghost point and the face it lies on (+1/-1 = min/max face). */
typedef struct __outerpt_bc_struct__ {
  short i0, i1, i2;
  int8_t FACEX0, FACEX1, FACEX2;
} outerpt_bc_struct;

typedef struct __bc_info_struct__ {
  int num_inner_boundary_points;
  int num_pure_outer_boundary_points[NGHOSTS][3];
  int bc_loop_bounds[NGHOSTS][6][6];
} bc_info_struct;

typedef struct __bc_struct__ {
  innerpt_bc_struct *NRPYELL_RESTRICT inner_bc_array;
  /* indexed [dirn + 3*which_gz] */
  outerpt_bc_struct *NRPYELL_RESTRICT pure_outer_bc_array[NGHOSTS * 3];
  bc_info_struct bc_info;
} bc_struct;

typedef struct __MoL_gridfunctions_struct__ {
  REAL *NRPYELL_RESTRICT y_n_gfs;
  REAL *NRPYELL_RESTRICT y_nplus1_running_total_gfs;
  REAL *NRPYELL_RESTRICT k_odd_gfs;
  REAL *NRPYELL_RESTRICT k_even_gfs;
  REAL *NRPYELL_RESTRICT auxevol_gfs;
  /* aliases y_nplus1_running_total_gfs, as in the reference allocator */
  REAL *NRPYELL_RESTRICT diagnostic_output_gfs;
} MoL_gridfunctions_struct;

typedef struct __griddata__ {
  paramstruct params;
  REAL *NRPYELL_RESTRICT xx[3];
  bc_struct bcstruct;
  rfm_struct rfmstruct;
  MoL_gridfunctions_struct gridfuncs;
} griddata_struct;

#ifdef __cplusplus
}
#endif

#endif /* NRPYELL_ABI_H */
