// Relaxation engine of the fused path: per-grid work buffers, the tile
// autotuner and the graph-replayed stop-on-tolerance loop, for FP64 and FP32
// state.  Used by capi.cu (MoL_step_forward_in_time, nrpyell_relax*) and by
// the mixed-precision driver.
#pragma once

#include "kernels.cuh"

namespace nrpyell {

// Per-grid driver state on the device.
struct FusedWork {
  Dims d;
  int* state;      // [0] n, [1] done, [2] converged
  int* zero_flag;  // always 0 (single steps run unconditionally)
  double* history;
  int history_len;
  int tile[3];     // autotuned tile for FP64 / FP32 / FP32 correction form, -1 = not tuned yet
  // FP32 buffers of the mixed-precision driver (allocated on demand): the
  // correction and its RK buffers y, acc, k_odd, k_even (2 gfs each), the
  // pointwise fields (3 gfs) and the base state's RHS R0 (2 gfs)
  float* f32;
  double* cycle_history;  // residual history of one FP32 stretch
};

// Gridfunction buffers of one precision (T = double or float).
struct StateBuffers {
  void* y;
  void* acc;
  void* kodd;
  void* keven;
  const void* aux;
  const void* R0;  // correction form (SubstepArgs::R0), else nullptr
};

struct RelaxParams {
  double dt, eta, cOB[2];
  double log10_tol;
  int max_steps;
  int check_every;  // 0: stop test on every residual (main.c); > 0: ET thorn semantics
  int history_offset;     // history index of step 0 of this run
  double* history_buf;    // where the history goes (nullptr: the work's own)
};

struct RelaxResult {
  int steps;  // index n of the last evaluated residual
  bool converged;
  double last_log10_l2;
};

extern int g_forced_tile;
extern bool g_pdl;  // programmatic dependent launch of the substep kernels
extern int g_work_generation;

FusedWork* get_work(const Dims& d, int history_len);
// Autotuned tile of a grid size (fp32: 0 or 1), -1 if not tuned yet.
int find_tile(const Dims& d, int fp32);
void release_work();
void release_batch();  // batch.cu
void release_graphs();
bool fused_ready(const paramstruct* p, const rfm_struct* rfm, const bc_struct* bc, REAL* NRPYELL_RESTRICT const xx[3],
                 RfmTables** rt, BcTables** bt);
int max_interior_blocks(const Dims& d);
StateBuffers buffers_of(const MoL_gridfunctions_struct* gf);
SubstepArgs substep_args(const Dims& d, RfmTables* rt, BcTables* bt, Scratch* s, const StateBuffers& b,
                         const RelaxParams& rp, int stage, const int* done, int* state, int tile);
// Autotuned tile shape of this grid size, precision and form; lt (nullable):
// time stage 1 with the relaxation's residual partials.  Never call while a
// stream is being captured (it allocates a copy of y_n).
template <typename T>
int tuned_tile(const Dims& d, RfmTables* rt, BcTables* bt, FusedWork* w, Scratch* sc, const StateBuffers& b,
               const RelaxParams& rp, const L2Tables* lt = nullptr);
template <typename T>
RelaxResult relax_loop(const Dims& d, RfmTables* rt, BcTables* bt, L2Tables* lt, FusedWork* w, Scratch* s, int tile,
                       const StateBuffers& b, const RelaxParams& rp);
// Correction form of the mixed-precision driver (nrpyell_relax_mixed): from
// the FP64 base state U, its RHS rhs (interior and radiation ghost points)
// and its residual bracket res (interior), the FP32 inputs of the correction
// kernels: R0 = (uu RHS; bracket at interior points, vv RHS elsewhere) and
// aux32 = (S(U) = ADD_times_AUU / (8 P^7), P = psi_background + U,
// wavespeed), over all points.
void launch_correction_base(const Dims& d, const double* U, const double* aux, const double* rhs, const double* res,
                            float* R0, float* aux32);
// U += correction over n values (both gridfunctions, all points).
void launch_correction_fold(double* U, const float* corr, long long n);
// Elementwise precision conversions on the library stream.
void convert_to_float(const double* in, float* out, long long n);
void convert_to_double(const float* in, double* out, long long n);

}  // namespace nrpyell
