// Kernel launchers shared between the C-ABI layer and the relaxation drivers.
#pragma once

#include "common.cuh"
#include "tables.cuh"

namespace nrpyell {

// ---- reference-order kernels (kernels_ref.cu) ----
void launch_rhs_ref(const Dims& d, const paramstruct* p, const RfmTables* rt, const double* aux, const double* in,
                    double* rhs);
void launch_residual_ref(const Dims& d, const RfmTables* rt, const double* aux, const double* in, double* res);
void launch_radiation_bc(const Dims& d, const paramstruct* p, const BcTables* bt, const double c[2],
                         const double finf[2], const double* gfs, double* rhs);
void launch_inner_copy(const Dims& d, const BcTables* bt, double* gfs, int ngfs);
void launch_extrap_bc(const Dims& d, const BcTables* bt, const bc_struct* bc, double* gfs);
// RK4 linear combination over all points, stage 1..4 (MoL_step_forward_in_time.c:33-48,76-92,120-133,161-172)
void launch_rk_update_ref(int stage, long long n, double dt, const double* k, const double* y, double* acc,
                          double* out);
// Deterministic weighted sum of g^2 over the interior: result[0] = sum w g^2.
void launch_l2_sum(const Dims& d, const L2Tables* lt, const double* g, Scratch* s);

// ---- fused kernels (kernels_fused.cu) ----
struct FusedArgs {
  Dims d;
  const void* S;      // stage input state (uu, vv)
  const void* y;      // y_n
  void* acc;          // running total
  void* out;          // stage output (next stage input, or y_n at stage 4)
  const void* aux;    // auxevol (ADD_times_AUU, psi_background, wavespeed)
  double dt, eta, cOB[2];
  const RfmTables* rt;
  const BcTables* bt;
  const L2Tables* lt;  // non-null: accumulate the residual's weighted L2 sum (stage 1)
  void* face;          // [2][Nxx1*Nxx2] RHS on the last interior plane
  Scratch* s;
  const int* done;     // device flag; kernels return immediately when *done != 0
};
template <typename T>
void launch_fused_substep(int stage, const FusedArgs& a);
// Only the interior kernel of a stage (timing helper).
template <typename T>
void launch_fused_interior_only(int stage, const FusedArgs& a);
// L2 finalisation for the relaxation driver: reads the partial sums written by
// the stage-1 kernel, stores log10 L2 into history[n], and sets the done flag.
void launch_relax_check(int nblocks, Scratch* s, double volume, double log10_tol, int max_steps, double* history,
                        int* state);
int fused_interior_blocks(const Dims& d);

}  // namespace nrpyell
