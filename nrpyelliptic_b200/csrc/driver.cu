// Relaxation engine of the fused path (see driver.cuh).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "driver.cuh"

namespace nrpyell {

int g_forced_tile = -1;
bool g_pdl = true;
bool pdl_enabled() { return g_pdl; }
int g_work_generation = 0;
static std::vector<FusedWork*> g_work;

// Never call while a stream is being captured (it may allocate).
FusedWork* get_work(const Dims& d, int history_len) {
  for (FusedWork* w : g_work)
    if (w->d.Nxx1 == d.Nxx1 && w->d.Nxx2 == d.Nxx2 && w->d.N0 == d.N0 && w->d.N1 == d.N1 && w->d.N2 == d.N2) {
      if (w->history_len < history_len) {
        g_work_generation++;  // graphs captured with the old history are stale
        NRPYELL_CUDA(cudaStreamSynchronize(stream()));
        NRPYELL_CUDA(cudaFree(w->history));
        NRPYELL_CUDA(dev_alloc(&w->history, sizeof(double) * history_len));
        w->history_len = history_len;
      }
      return w;
    }
  FusedWork* w = new FusedWork();
  w->d = d;
  w->tile[0] = w->tile[1] = w->tile[2] = -1;
  w->f32 = nullptr;
  w->cycle_history = nullptr;
  NRPYELL_CUDA(dev_alloc(&w->state, sizeof(int) * 8 + sizeof(double) * 4));
  NRPYELL_CUDA(cudaMemset(w->state, 0, sizeof(int) * 8 + sizeof(double) * 4));
  w->zero_flag = w->state + 4;
  w->history_len = history_len > 16 ? history_len : 16;
  NRPYELL_CUDA(dev_alloc(&w->history, sizeof(double) * w->history_len));
  g_work.push_back(w);
  return w;
}

void release_work() {
  for (FusedWork* w : g_work) {
    cudaFree(w->state);
    cudaFree(w->history);
    if (w->f32) cudaFree(w->f32);
    if (w->cycle_history) cudaFree(w->cycle_history);
    delete w;
  }
  g_work.clear();
}

int find_tile(const Dims& d, int fp32) {
  for (FusedWork* w : g_work)
    if (w->d.N0 == d.N0 && w->d.N1 == d.N1 && w->d.N2 == d.N2) return w->tile[fp32 >= 0 && fp32 <= 2 ? fp32 : 0];
  return -1;
}

bool fused_ready(const paramstruct* p, const rfm_struct* rfm, const bc_struct* bc, REAL* NRPYELL_RESTRICT const xx[3],
                 RfmTables** rt, BcTables** bt) {
  *rt = get_rfm_tables(p, rfm);
  *bt = get_bc_tables(p, bc, xx);
  return *rt && *bt && (*bt)->columns_ok && (*bt)->analytic_ok && p->outer_bc_type == RADIATION_OUTER_BCS;
}

int max_interior_blocks(const Dims& d) {
  int m = 0;
  for (int t = 0; t < substep_num_tiles(); t++) m = std::max(m, substep_interior_blocks(d, t));
  return m;
}

StateBuffers buffers_of(const MoL_gridfunctions_struct* gf) {
  StateBuffers b;
  b.y = gf->y_n_gfs;
  b.acc = gf->y_nplus1_running_total_gfs;
  b.kodd = gf->k_odd_gfs;
  b.keven = gf->k_even_gfs;
  b.aux = gf->auxevol_gfs;
  b.R0 = nullptr;
  return b;
}

// Stage s reads S and writes O (MoL_step_forward_in_time.c: k_odd / k_even
// alternate, stage 4 updates y_n in place).
SubstepArgs substep_args(const Dims& d, RfmTables* rt, BcTables* bt, Scratch* s, const StateBuffers& b,
                         const RelaxParams& rp, int stage, const int* done, int* state, int tile) {
  SubstepArgs a;
  a.d = d;
  void* S[4] = {b.y, b.kodd, b.keven, b.kodd};
  void* O[4] = {b.kodd, b.keven, b.kodd, b.y};
  a.S = S[stage - 1];
  a.out = O[stage - 1];
  a.y = b.y;
  a.acc = b.acc;
  a.aux = b.aux;
  a.R0 = b.R0;
  a.dt = rp.dt;
  a.eta = rp.eta;
  a.cOB[0] = rp.cOB[0];
  a.cOB[1] = rp.cOB[1];
  a.rt = rt;
  a.bt = bt;
  a.lt = nullptr;
  a.s = s;
  a.state = state;
  a.history = nullptr;
  a.log10_tol = -1e300;
  a.max_steps = 0;
  a.check_every = 0;
  a.defer_l2 = 0;
  a.done = done;
  a.tile = tile;
  return a;
}

// Tile-shape autotuner: times every tile shape on the caller's own buffers
// and keeps the fastest, once per grid size and precision (and form).  Each
// shape is timed on whole RK4 steps as the relaxation runs them -- stage 1
// storing its residual partials when an L2 table is given (the per-tile
// reduction depends on the shape) and the stop test's reduction forked
// beside stage 2 and joined before stage 3, then stages 2, 3 and 4 -- one
// warm-up step and the best of five 8-step timings.  Stage 4 writes y_n, so y_n is
// saved before the timings and restored after them.
template <typename T>
int tuned_tile(const Dims& d, RfmTables* rt, BcTables* bt, FusedWork* w, Scratch* sc, const StateBuffers& b,
               const RelaxParams& rp, const L2Tables* lt) {
  // the correction form runs on the marching and 8-warp direct shapes
  const bool corr = b.R0 != nullptr;
  const int which = sizeof(T) == 8 ? 0 : (corr ? 2 : 1);
  if (g_forced_tile >= 0 && !(corr && !substep_supports_correction(g_forced_tile))) return g_forced_tile;
  if (w->tile[which] >= 0) return w->tile[which];
  const size_t ybytes = sizeof(T) * 2 * (size_t)d.Ntot;
  void* ysave = nullptr;
  NRPYELL_CUDA(dev_alloc(&ysave, ybytes));
  if (!status_ok()) return 0;
  NRPYELL_CUDA(cudaMemcpyAsync(ysave, b.y, ybytes, cudaMemcpyDeviceToDevice, stream()));
  cudaEvent_t e0, e1;
  NRPYELL_CUDA(cudaEventCreate(&e0));
  NRPYELL_CUDA(cudaEventCreate(&e1));
  int best = -1;
  float best_ms = 1e30f;
  for (int t = 0; t < substep_num_tiles(); t++) {
    if (corr && (!substep_supports_correction(t) || !march_fits(d))) continue;
    SubstepArgs a[4];
    for (int st = 1; st <= 4; st++) a[st - 1] = substep_args(d, rt, bt, sc, b, rp, st, w->zero_flag, w->state, t);
    if (lt) {
      a[0].lt = lt;
      a[0].defer_l2 = 1;  // partials only, reduced beside stage 2 as in relax_loop
    }
    // one RK4 step as relax_loop runs it: with an L2 table the stop test's
    // reduction is forked after stage 1 and joined before stage 3 (its
    // state is w->state, which relax_loop resets before every relaxation;
    // the kernels here wait on w->zero_flag, so they always run)
    auto step = [&]() {
      launch_substep<T>(1, a[0]);
      if (lt) launch_finalize_forked<T>(a[0]);
      for (int st = 2; st <= 4; st++) {
        if (lt && st == 3) join_finalize();
        launch_substep<T>(st, a[st - 1]);
      }
    };
    prepare_substep<T>(t);
    step();
    // best of five 8-step timings: the leading one-plane shapes at
    // 128x128x16 differ by 0.5-2 %, within the noise of shorter timings
    float tmin = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
      NRPYELL_CUDA(cudaEventRecord(e0, stream()));
      for (int i = 0; i < 8; i++) step();
      NRPYELL_CUDA(cudaEventRecord(e1, stream()));
      NRPYELL_CUDA(cudaEventSynchronize(e1));
      float ms = 0.0f;
      NRPYELL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      tmin = std::min(tmin, ms);
    }
    if (tmin < best_ms) {
      best_ms = tmin;
      best = t;
    }
  }
  NRPYELL_CUDA(cudaMemcpyAsync(b.y, ysave, ybytes, cudaMemcpyDeviceToDevice, stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  NRPYELL_CUDA(cudaFree(ysave));
  NRPYELL_CUDA(cudaEventDestroy(e0));
  NRPYELL_CUDA(cudaEventDestroy(e1));
  if (best < 0) {
    NRPYELL_FAIL("tile autotuner: no tile shape runs this form on this grid");
    return 0;
  }
  w->tile[which] = best;
  return best;
}
template int tuned_tile<double>(const Dims&, RfmTables*, BcTables*, FusedWork*, Scratch*, const StateBuffers&,
                                const RelaxParams&, const L2Tables*);
template int tuned_tile<float>(const Dims&, RfmTables*, BcTables*, FusedWork*, Scratch*, const StateBuffers&,
                               const RelaxParams&, const L2Tables*);

// ------------------------------------------------------------ relax loop
// A CUDA graph of kStepsPerGraph RK4 steps is replayed until the device-side
// state says done; the stop test runs inside the stage-1 kernel, so kernels
// after the stop return at entry.  Graphs are cached per buffers, grid,
// parameters and tile.
constexpr int kStepsPerGraph = 16;

struct RelaxGraph {
  Dims d;
  StateBuffers b;
  RelaxParams rp;
  int fp32, tile, scratch_gen, work_gen;
  const RfmTables* rt;
  const BcTables* bt;
  const L2Tables* lt;
  cudaGraphExec_t exec;
  size_t nodes;
};
static std::vector<RelaxGraph*> g_graphs;

void release_graphs() {
  for (RelaxGraph* r : g_graphs) {
    cudaGraphExecDestroy(r->exec);
    delete r;
  }
  g_graphs.clear();
}

template <typename T>
RelaxResult relax_loop(const Dims& d, RfmTables* rt, BcTables* bt, L2Tables* lt, FusedWork* w, Scratch* s, int tile,
                       const StateBuffers& b, const RelaxParams& rp) {
  RelaxResult res = {0, false, NAN};
  const int fp32 = sizeof(T) == 4;
  RelaxGraph* rg = nullptr;
  for (size_t i = 0; i < g_graphs.size(); i++) {
    RelaxGraph* r = g_graphs[i];
    if (r->scratch_gen != scratch_generation() || r->work_gen != g_work_generation) {
      NRPYELL_CUDA(cudaGraphExecDestroy(r->exec));
      delete r;
      g_graphs.erase(g_graphs.begin() + i);
      i--;
      continue;
    }
    if (r->fp32 == fp32 && r->tile == tile && r->rt == rt && r->bt == bt && r->lt == lt &&
        memcmp(&r->d, &d, sizeof(Dims)) == 0 && memcmp(&r->b, &b, sizeof(StateBuffers)) == 0 &&
        memcmp(&r->rp, &rp, sizeof(RelaxParams)) == 0)
      rg = r;
  }
  if (!rg) {
    cudaGraph_t graph;
    const long long launches_before = launch_count();
    prepare_substep<T>(tile);
    prepare_columns();
    NRPYELL_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kStepsPerGraph; k++) {
      // stage 1 also evaluates the residual of y_n and runs the stop test
      SubstepArgs a1 = substep_args(d, rt, bt, s, b, rp, 1, w->state + 1, w->state, tile);
      a1.lt = lt;
      a1.history = (rp.history_buf ? rp.history_buf : w->history) + rp.history_offset;
      a1.log10_tol = rp.log10_tol;
      a1.max_steps = rp.max_steps;
      a1.check_every = rp.check_every;
      a1.defer_l2 = 1;
      launch_substep<T>(1, a1);
      launch_finalize_forked<T>(a1);  // the norm and stop test beside stage 2
      for (int st = 2; st <= 4; st++) {
        if (st == 3) join_finalize();
        launch_substep<T>(st, substep_args(d, rt, bt, s, b, rp, st, w->state + 1, w->state, tile));
      }
    }
    NRPYELL_CUDA(cudaStreamEndCapture(stream(), &graph));
    set_launch_count(launches_before);  // captured launches count when the graph runs
    if (!status_ok()) return res;
    rg = new RelaxGraph();
    rg->d = d;
    rg->b = b;
    rg->rp = rp;
    rg->fp32 = fp32;
    rg->tile = tile;
    rg->rt = rt;
    rg->bt = bt;
    rg->lt = lt;
    rg->scratch_gen = scratch_generation();
    rg->work_gen = g_work_generation;
    rg->nodes = 0;
    NRPYELL_CUDA(cudaGraphGetNodes(graph, nullptr, &rg->nodes));
    NRPYELL_CUDA(cudaGraphInstantiate(&rg->exec, graph, 0));
    NRPYELL_CUDA(cudaGraphDestroy(graph));
    g_graphs.push_back(rg);
  }

  static int* pinned = nullptr;
  static cudaEvent_t ev[2];
  if (!pinned) {
    NRPYELL_CUDA(cudaMallocHost(&pinned, sizeof(int) * 16));
    NRPYELL_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    NRPYELL_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  }
  NRPYELL_CUDA(cudaMemsetAsync(w->state, 0, sizeof(int) * 4, stream()));
  // Replay; poll the state of launch k-1 while launch k runs.
  const long long max_launches = (long long)rp.max_steps / kStepsPerGraph + 2;
  for (long long k = 0; k < max_launches; k++) {
    NRPYELL_CUDA(cudaGraphLaunch(rg->exec, stream()));
    count_launch((int)rg->nodes);
    const int slot = (int)(k & 1);
    NRPYELL_CUDA(cudaMemcpyAsync(pinned + 8 * slot, w->state, sizeof(int) * 6, cudaMemcpyDeviceToHost, stream()));
    NRPYELL_CUDA(cudaEventRecord(ev[slot], stream()));
    if (k > 0) {
      NRPYELL_CUDA(cudaEventSynchronize(ev[1 - slot]));
      if (pinned[8 * (1 - slot) + 1]) break;
    }
    if (!status_ok()) return res;
  }
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  int st[6];
  NRPYELL_CUDA(cudaMemcpy(st, w->state, sizeof(st), cudaMemcpyDeviceToHost));
  if (!status_ok()) return res;
  res.steps = st[0];
  res.converged = st[2] != 0;
  NRPYELL_CUDA(cudaMemcpy(&res.last_log10_l2, (rp.history_buf ? rp.history_buf : w->history) + rp.history_offset + st[0],
                          sizeof(double), cudaMemcpyDeviceToHost));
  return res;
}
template RelaxResult relax_loop<double>(const Dims&, RfmTables*, BcTables*, L2Tables*, FusedWork*, Scratch*, int,
                                        const StateBuffers&, const RelaxParams&);
template RelaxResult relax_loop<float>(const Dims&, RfmTables*, BcTables*, L2Tables*, FusedWork*, Scratch*, int,
                                       const StateBuffers&, const RelaxParams&);

__global__ void k_correction_base(Dims d, const double* __restrict__ U, const double* __restrict__ aux,
                                  const double* __restrict__ rhs, const double* __restrict__ res, float* __restrict__ R0,
                                  float* __restrict__ aux32) {
  const long long n = d.Ntot;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(i % d.N0);
    const long long q = i / d.N0;
    const int i1 = (int)(q % d.N1), i2 = (int)(q / d.N1);
    const bool interior = i0 >= NGHOSTS && i0 < NGHOSTS + d.Nxx0 && i1 >= NGHOSTS && i1 < NGHOSTS + d.Nxx1 &&
                          i2 >= NGHOSTS && i2 < NGHOSTS + d.Nxx2;
    const double P = aux[PSI_BACKGROUNDGF * n + i] + U[i];
    const double P2 = P * P, P4 = P2 * P2, P7 = P4 * P2 * P;
    R0[i] = (float)rhs[i];
    R0[n + i] = (float)(interior ? res[i] : rhs[n + i]);
    aux32[ADD_TIMES_AUUGF * n + i] = (float)(0.125 * aux[ADD_TIMES_AUUGF * n + i] / P7);
    aux32[PSI_BACKGROUNDGF * n + i] = (float)P;
    aux32[WAVESPEEDGF * n + i] = (float)aux[WAVESPEEDGF * n + i];
  }
}
void launch_correction_base(const Dims& d, const double* U, const double* aux, const double* rhs, const double* res,
                            float* R0, float* aux32) {
  NRPYELL_LAUNCH(k_correction_base, 148 * 8, 256, 0, d, U, aux, rhs, res, R0, aux32);
}

__global__ void k_correction_fold(double* __restrict__ U, const float* __restrict__ c, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    U[i] += (double)c[i];
}
void launch_correction_fold(double* U, const float* corr, long long n) {
  NRPYELL_LAUNCH(k_correction_fold, 148 * 8, 256, 0, U, corr, n);
}

__global__ void k_to_float(const double* __restrict__ in, float* __restrict__ out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)in[i];
}
__global__ void k_to_double(const float* __restrict__ in, double* __restrict__ out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (double)in[i];
}
void convert_to_float(const double* in, float* out, long long n) {
  NRPYELL_LAUNCH(k_to_float, (unsigned)((n + 255) / 256), 256, 0, in, out, n);
}
void convert_to_double(const float* in, double* out, long long n) {
  NRPYELL_LAUNCH(k_to_double, (unsigned)((n + 255) / 256), 256, 0, in, out, n);
}

}  // namespace nrpyell
