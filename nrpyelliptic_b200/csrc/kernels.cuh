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

// ---- fused substep kernel (kernels_fused.cu) ----
// Requires BcTables::columns_ok && BcTables::analytic_ok.
struct SubstepArgs {
  Dims d;
  const void* S;      // stage input state (uu, vv)
  const void* y;      // y_n
  void* acc;          // running total
  void* out;          // stage output (next stage input, or y_n at stage 4)
  const void* aux;    // auxevol (ADD_times_AUU, psi_background, wavespeed)
  // Correction form (FP32 only, marching shapes only): the base state's RHS
  // (see point_rhs_correction); aux then holds (S(U), psi + U, wavespeed).
  // nullptr: the plain form.
  const void* R0;
  double dt, eta, cOB[2];
  const RfmTables* rt;
  const BcTables* bt;
  // Stop test at stage 1 (relaxation driver); lt == nullptr: none.  The last
  // interior block writes log10 L2 to history[state[0]] and updates state:
  // [0] n, [1] done, [2] converged.
  const L2Tables* lt;
  Scratch* s;
  int* state;
  double* history;
  double log10_tol;
  int max_steps;
  int check_every;  // 0: test every residual (main.c); > 0: the ET thorn's loop
  // 1: the stage-1 blocks only store their per-tile partials and the norm
  // and stop test are left to launch_finalize_forked (relaxation driver).
  int defer_l2;
  const int* done;  // kernels return at entry when *done != 0
  int tile;         // tile shape index (autotuned)
};
template <typename T>
void launch_substep(int stage, const SubstepArgs& a);
// Copies inner ghost points of gfs (2 gridfunctions) from their sources.
template <typename T>
void launch_ghost_fill(const Dims& d, const BcTables* bt, void* gfs);
// Tile shapes: 32 x by x p points per interior tile, of the kinds listed at
// nrpyell_tile_info.
int substep_num_tiles();
void substep_tile_shape(int tile, int* bx, int* by, int* p);
int substep_tile_kind(int tile);  // see nrpyell_tile_info
// Shapes that run the correction form (SubstepArgs::R0).
bool substep_supports_correction(int tile);
int substep_interior_blocks(const Dims& d, int tile);
// One-time per-shape setup (shared-memory opt-in); call before a stream
// capture that launches the shape.
template <typename T>
void prepare_substep(int tile);

// Side stream and events of the stop test (launch_finalize_forked); call
// before a stream capture.
void prepare_columns();

// Stop test of a stage-1 launch made with defer_l2 = 1: one block on
// side_stream() sums the per-tile partials in index order and updates the
// state (finalize_l2), beside the stage-2 launch; join_finalize() makes
// stream() wait for it (before stage 3, the first launch that must see the
// stop decision -- stage 4 writes y_n).
template <typename T>
void launch_finalize_forked(const SubstepArgs& a1);
void join_finalize();

// ---- marching variant (kernels_march.cu): shape v of the list there.  Its
// element offsets are 32-bit: grids with 3 Ntot >= 2^32 do not fit
// (launch_march returns false and launches nothing).
bool march_fits(const Dims& d);
template <typename T>
bool launch_march(int stage, bool resid, int v, const SubstepArgs& a);
// Shared-memory opt-in of a shape's kernels (before a stream capture).
template <typename T>
void prepare_march(int v);
// Interior blocks of shape v's launch on this grid (its split of the planes).
template <typename T>
int march_interior_blocks(int v, const SubstepArgs& a);

}  // namespace nrpyell
