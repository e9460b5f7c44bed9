// Device mirrors of the caller's set-up data ("tables"), built on first use
// and cached by the identity of the caller's arrays.  The caller owns every
// struct and array; the library snapshots what it needs into device memory:
//   * reference-metric tables (rfm_struct) and the folded per-(i0,i1)
//     coefficients of the fused RHS,
//   * the inner-boundary copy map and pure-outer point lists (bc_struct)
//     with the time-invariant radiation-BC geometry (r and d xx^i / d r),
//   * the L2-norm volume weights for one integration radius.
// nrpyell_release_tables() frees all of them.
#pragma once

#include "common.cuh"

namespace nrpyell {

constexpr int kNumCoef = 6;  // fused-RHS coefficients per (i0,i1)

struct RfmTables {
  // key
  const REAL* key_f0;
  const REAL* key_f2;
  Dims d;
  double invdx[3];
  double AMAX, SINHWAA, bScale;  // the content depends on these (host arrays may be reused)
  // device copies of the reference-metric arrays
  double* f0;
  double* f0_D0;
  double* f0_DD00;
  double* f1;
  double* f1_D1;
  double* f2;
  double* f2_D0;
  double* f3;
  double* f3_D0;
  // folded coefficients, structure of arrays: coef[c * N0*N1 + i0 + N0*i1]
  //   0: d22 weight  invdx2^2 / (f0^2 f1^2)
  //   1: d00 weight  invdx0^2 f3^2 / (f0'^2 f2^2)
  //   2: d11 weight  invdx1^2 / f2^2
  //   3: d1  weight  invdx1 f1' / (f1 f2^2)
  //   4: d0  weight  -invdx0 * (first-derivative coefficient of the reference RHS)
  //   5: centre weight  -(5269/1800) (c0 + c1 + c2)
  double* coef;
  float* coef32;
  double* xx01;  // device build: xx0 [N0] then xx1 [N1]
  void* base;
};

// One pure outer point with everything the radiation BC needs, precomputed.
struct OuterPoint {
  int idx3, idx3_int;       // IDX3S of the point and of its interior neighbour
  short i0, i1, i2;         // the point
  short i0n, i1n, i2n;      // the neighbour
  signed char off0, off1;   // upwind offsets of the x0 / x1 stencils at the point
  signed char off0n, off1n; // ... and at the neighbour
  double r, dx0dr, dx1dr;
  double rn, dx0drn, dx1drn;
};

struct BcTables {
  // key
  const innerpt_bc_struct* key_inner;
  const outerpt_bc_struct* key_outer0;
  int key_ninner;
  const REAL* key_xx[3];
  Dims d;
  double AMAX, SINHWAA, bScale, dxx0, dxx1, dxx2;
  // inner copy map
  int n_inner;
  int2* inner;             // (dst, src) 3-D indices
  signed char* inner_par;  // parity[0] of each inner point (scalar gridfunctions)
  // generic pure-outer lists, grouped per (which_gz, dirn) in the reference's order
  int outer_off[NGHOSTS * 3 + 1];
  OuterPoint* outer;
  int n_outer;
  int max_layer;  // largest list size (launch sizing)
  // fused-path column form: every pure outer point lies on the x0max face,
  // layer gz = i0 == N0-NGHOSTS+gz over all interior (i1,i2)
  bool columns_ok;
  // every inner point copies from the SymTP reflection of itself
  // (symtp_ghost_source), so kernels may read ghost values straight from
  // their source points instead of from the ghost zones
  bool analytic_ok;
  // geometry for the column form, [6][N1]: j=0 is the last interior plane,
  // j=1..5 the outer layers; arrays r, dx0dr, dx1dr
  double* colgeo;
  double* xx01;  // xx0 [N0] then xx1 [N1] on the device (bc_tables_layout)
  void* base;
};

struct L2Tables {
  const REAL* key_xx[3];
  Dims d;
  double AMAX, SINHWAA, bScale, dxx0, dxx1, dxx2, R;
  double* w;      // [N0*N1]: sqrt(det gamma) dxx0 dxx1 dxx2 on interior (i0,i1) with r < R, else 0
  double volume;  // sum of dV over interior points with r < R
};

RfmTables* get_rfm_tables(const paramstruct* p, const rfm_struct* rfm);
// Cache lookup only (nullptr when absent), allocation and layout of a new
// entry keyed by rfm / bc, and registration of a filled entry -- shared by
// the host build (get_*_tables) and the device build (tables_gpu.cu).
RfmTables* find_rfm_tables(const paramstruct* p, const rfm_struct* rfm);
RfmTables* new_rfm_tables(const paramstruct* p, const rfm_struct* rfm);
void register_rfm_tables(RfmTables* t);
BcTables* find_bc_tables(const paramstruct* p, const bc_struct* bc, REAL* NRPYELL_RESTRICT const xx[3]);
void bc_tables_set_key(BcTables* t, const paramstruct* p, const bc_struct* bc, REAL* NRPYELL_RESTRICT const xx[3]);
bool bc_tables_layout(BcTables* t, size_t n_inner, size_t n_outer);
void register_bc_tables(BcTables* t);
BcTables* get_bc_tables(const paramstruct* p, const bc_struct* bc, REAL* NRPYELL_RESTRICT const xx[3]);
L2Tables* get_l2_tables(const paramstruct* p, REAL* NRPYELL_RESTRICT const xx[3], double R);
void release_all_tables();

// Scratch device memory owned by the library (reduction partials, flags).
struct Scratch {
  double* partials;  // per-block partial sums
  int n_partials;
  double* result;    // [4]
  unsigned int* counter;
  int* flags;        // [8]
  void* base;
};
// Returns scratch with at least n_partials partial-sum slots.  Never call it
// while a stream is being captured: growing the buffer allocates.
Scratch* get_scratch(int n_partials);
// Incremented whenever the scratch buffer is reallocated.
int scratch_generation();

}  // namespace nrpyell
