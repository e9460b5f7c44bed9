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
  int* state;      // [0] n, [1] done, [2] converged, [3] stalled
  int* zero_flag;  // always 0 (single steps run unconditionally)
  double* stall;   // [0] log10 L2 at the start of the stall window, [1] its step
  double* history;
  int history_len;
  int tile[2];     // autotuned tile for FP64 / FP32, -1 = not tuned yet
  // FP32 copies of the state for the mixed-precision driver (allocated on demand)
  float* f32;      // y, acc, k_odd, k_even (2 gfs each) and aux (3 gfs)
};

// Gridfunction buffers of one precision (T = double or float).
struct StateBuffers {
  void* y;
  void* acc;
  void* kodd;
  void* keven;
  const void* aux;
};

struct RelaxParams {
  double dt, eta, cOB[2];
  double log10_tol;
  int max_steps;
  int check_every;  // 0: stop test on every residual (main.c); > 0: ET thorn semantics
  int stall_window;       // 0: no stall test
  double stall_log_drop;  // stalled when log10 L2 fell by less than this over the window (negative)
  int history_offset;     // history index of step 0 of this run
};

struct RelaxResult {
  int steps;  // index n of the last evaluated residual
  bool converged, stalled;
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
template <typename T>
int tuned_tile(const Dims& d, RfmTables* rt, BcTables* bt, FusedWork* w, Scratch* sc, const StateBuffers& b,
               const RelaxParams& rp);
template <typename T>
RelaxResult relax_loop(const Dims& d, RfmTables* rt, BcTables* bt, L2Tables* lt, FusedWork* w, Scratch* s, int tile,
                       const StateBuffers& b, const RelaxParams& rp);
// Elementwise precision conversions on the library stream.
void convert_to_float(const double* in, float* out, long long n);
void convert_to_double(const float* in, double* out, long long n);

}  // namespace nrpyell
