// Batched relaxation: many puncture configurations, on grids of different
// sizes, relaxed together.  Every RK4 substep of all configurations is one
// launch of the shared-memory planes or marching kernel
// (k_substep_planes_batch, k_substep_march_batch): the
// launch's blocks are the concatenated column blocks and interior tiles of
// all grids, and each grid keeps its own launch arguments, stop test and
// done flag, so a grid that has converged costs one flag read per block.
// Sixteen RK4 steps are captured in one CUDA graph and replayed until every
// grid is done; the tile shape is autotuned on the batch.
#include <string.h>

#include <algorithm>
#include <vector>

#include "driver.cuh"
#include "substep.cuh"

namespace nrpyell {

namespace {

constexpr int kBatchStepsPerGraph = 16;
constexpr int kStateInts = 8;  // per grid: [0] n, [1] done, [2] converged

struct BatchWork {
  int n = 0, hist_len = 0, partials_per = 0;
  int* state = nullptr;     // n x kStateInts
  double* history = nullptr;
  double* partials = nullptr;
  unsigned int* tickets = nullptr;
  int* offs = nullptr;      // n
  unsigned char* devs = nullptr;  // 5 x n SubDev<T>: stage 1 with stop test, stages 1..4 (tuning uses 2)
  int* pinned = nullptr;          // host, 2 x n x kStateInts: the polled states of two graph launches
};
BatchWork g_batch;
static_assert(sizeof(SubDev<float>) <= sizeof(SubDev<double>), "batch argument slots hold either precision");

// FP32 buffers of the batched mixed-precision driver, per grid 6 x 2 + 3
// gridfunctions (as FusedWork::f32), and the FP64 evaluations' L2 sums.
struct MixedWork {
  size_t floats = 0;
  float* f32 = nullptr;
  int n = 0;
  double* sums = nullptr;
};
MixedWork g_mixed;

void free_batch() {
  cudaFreeHost(g_batch.pinned);
  cudaFree(g_batch.state);
  cudaFree(g_batch.history);
  cudaFree(g_batch.partials);
  cudaFree(g_batch.tickets);
  cudaFree(g_batch.offs);
  cudaFree(g_batch.devs);
  g_batch = BatchWork();
  cudaFree(g_mixed.f32);
  cudaFree(g_mixed.sums);
  g_mixed = MixedWork();
}

bool ensure_batch(int n, int hist_len, int partials_per) {
  if (g_batch.n >= n && g_batch.hist_len >= hist_len && g_batch.partials_per >= partials_per) return true;
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  cudaFreeHost(g_batch.pinned);
  cudaFree(g_batch.state);
  cudaFree(g_batch.history);
  cudaFree(g_batch.partials);
  cudaFree(g_batch.tickets);
  cudaFree(g_batch.offs);
  cudaFree(g_batch.devs);
  g_batch = BatchWork();
  g_batch.n = n;
  g_batch.hist_len = hist_len;
  g_batch.partials_per = partials_per;
  NRPYELL_CUDA(dev_alloc(&g_batch.state, sizeof(int) * kStateInts * n));
  NRPYELL_CUDA(dev_alloc(&g_batch.history, sizeof(double) * (size_t)hist_len * n));
  NRPYELL_CUDA(dev_alloc(&g_batch.partials, sizeof(double) * (size_t)partials_per * n));
  NRPYELL_CUDA(dev_alloc(&g_batch.tickets, sizeof(unsigned int) * n));
  NRPYELL_CUDA(dev_alloc(&g_batch.offs, sizeof(int) * n));
  NRPYELL_CUDA(dev_alloc(&g_batch.devs, sizeof(SubDev<double>) * 5 * n));
  NRPYELL_CUDA(cudaMemset(g_batch.tickets, 0, sizeof(unsigned int) * n));
  NRPYELL_CUDA(cudaMallocHost(&g_batch.pinned, sizeof(int) * kStateInts * n * 2));
  return status_ok();
}

struct Grid {
  Dims d;
  RfmTables* rt;
  BcTables* bt;
  L2Tables* lt;
  StateBuffers b;
  RelaxParams rp;
  int index;  // position in the caller's array
};

// Launch arguments of every grid for one tile shape: devs_host[5][n] (stage
// 1 with the stop test, then stages 1..4), block offsets, total blocks.
template <typename T>
bool build_devs(const std::vector<Grid>& grids, int tile, std::vector<SubDev<T>>* devs, std::vector<int>* offs,
                int* blocks) {
  const int n = (int)grids.size();
  devs->assign(5 * n, SubDev<T>());
  offs->assign(n, 0);
  int total = 0;
  for (int c = 0; c < n; c++) {
    const Grid& g = grids[c];
    Scratch sc;
    memset(&sc, 0, sizeof(sc));
    sc.partials = g_batch.partials + (size_t)c * g_batch.partials_per;
    sc.n_partials = g_batch.partials_per;
    sc.counter = g_batch.tickets + c;
    int* state = g_batch.state + kStateInts * c;
    for (int k = 0; k < 5; k++) {
      const int stage = (k == 0) ? 1 : k;
      SubstepArgs a = substep_args(g.d, g.rt, g.bt, &sc, g.b, g.rp, stage, state + 1, state, tile);
      if (k == 0) {
        a.lt = g.lt;
        a.history = g_batch.history + (size_t)c * g_batch.hist_len;
        a.log10_tol = g.rp.log10_tol;
        a.max_steps = g.rp.max_steps;
      }
      if (!batch_launch_dev<T>(a, &(*devs)[k * n + c])) return false;
    }
    const SubDev<T>& f = (*devs)[c];
    if (f.n_tiles > g_batch.partials_per) {
      NRPYELL_FAIL("batched relaxation: partial-sum buffer too small");
      return false;
    }
    (*offs)[c] = total;
    total += f.n_col_blocks + f.n_tiles;
  }
  *blocks = total;
  return true;
}

template <typename T>
bool upload_devs(const std::vector<SubDev<T>>& devs, const std::vector<int>& offs) {
  NRPYELL_CUDA(cudaMemcpyAsync(g_batch.devs, devs.data(), sizeof(SubDev<T>) * devs.size(), cudaMemcpyHostToDevice,
                               stream()));
  NRPYELL_CUDA(cudaMemcpyAsync(g_batch.offs, offs.data(), sizeof(int) * offs.size(), cudaMemcpyHostToDevice,
                               stream()));
  return status_ok();
}

// Tile shapes a batch may run: the shared-memory planes and marching shapes
// for FP64, the marching shapes for the FP32 correction form.
bool batch_tile_ok(int t, bool corr) {
  const int kind = substep_tile_kind(t);
  return corr ? kind == 5 : (kind == 4 || kind == 5);
}

struct BatchResult {
  std::vector<int> steps;
  std::vector<char> converged;
  std::vector<double> last;
};

// Relaxes the grids of gs together, each with its own RelaxParams (dt,
// tolerance, max_steps); *tile: the tile shape, -1 = the forced one or the
// fastest on this batch (set on return).  corr: FP32 correction form (every
// grid's b.R0 set).  The results come from the device states and histories.
template <typename T>
bool run_batch(const std::vector<Grid>& gs, bool corr, int* tile, BatchResult* out) {
  const int n = (int)gs.size();
  int max_steps = 0, max_tiles = 0;
  bool fits = true;
  for (const Grid& G : gs) {
    max_steps = std::max(max_steps, G.rp.max_steps);
    max_tiles = std::max(max_tiles, max_interior_blocks(G.d));
    fits = fits && march_fits(G.d);
  }
  if (corr && !fits) {
    NRPYELL_FAIL("batched correction form: a grid is too large for the marching shapes (3 Ntot >= 2^32)");
    return false;
  }
  if (!ensure_batch(n, max_steps + 1, max_tiles)) return false;
  SubDev<T>* devs_dev = reinterpret_cast<SubDev<T>*>(g_batch.devs);
  std::vector<SubDev<T>> devs;
  std::vector<int> offs;
  int blocks = 0;
  if (*tile < 0 && g_forced_tile >= 0 && batch_tile_ok(g_forced_tile, corr)) *tile = g_forced_tile;
  NRPYELL_CUDA(cudaMemsetAsync(g_batch.state, 0, sizeof(int) * kStateInts * n, stream()));
  if (*tile < 0) {  // the fastest shape on this batch, timed on stage 2
    cudaEvent_t e0, e1;
    NRPYELL_CUDA(cudaEventCreate(&e0));
    NRPYELL_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int t = 0; t < substep_num_tiles(); t++) {
      if (!batch_tile_ok(t, corr) || (substep_tile_kind(t) == 5 && !fits)) continue;
      if (!build_devs<T>(gs, t, &devs, &offs, &blocks) || !upload_devs<T>(devs, offs)) return false;
      const SubDev<T>* d2 = devs_dev + 2 * n;  // stage 2: writes only k_even and the running total
      launch_substep_batch<T>(2, false, t, d2, g_batch.offs, n, blocks, corr);
      float tmin = 1e30f;
      for (int rep = 0; rep < 3; rep++) {
        NRPYELL_CUDA(cudaEventRecord(e0, stream()));
        for (int i = 0; i < 5; i++) launch_substep_batch<T>(2, false, t, d2, g_batch.offs, n, blocks, corr);
        NRPYELL_CUDA(cudaEventRecord(e1, stream()));
        NRPYELL_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        NRPYELL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        tmin = std::min(tmin, ms);
      }
      if (tmin < best) {
        best = tmin;
        *tile = t;
      }
    }
    NRPYELL_CUDA(cudaEventDestroy(e0));
    NRPYELL_CUDA(cudaEventDestroy(e1));
  }
  if (*tile < 0 || !build_devs<T>(gs, *tile, &devs, &offs, &blocks) || !upload_devs<T>(devs, offs)) return false;
  NRPYELL_CUDA(cudaMemsetAsync(g_batch.state, 0, sizeof(int) * kStateInts * n, stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  if (!status_ok()) return false;

  // capture sixteen RK4 steps of the whole batch
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  const long long launches_before = launch_count();
  NRPYELL_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < kBatchStepsPerGraph; k++) {
    launch_substep_batch<T>(1, true, *tile, devs_dev, g_batch.offs, n, blocks, corr);
    for (int st = 2; st <= 4; st++)
      launch_substep_batch<T>(st, false, *tile, devs_dev + (size_t)st * n, g_batch.offs, n, blocks, corr);
  }
  NRPYELL_CUDA(cudaStreamEndCapture(stream(), &graph));
  set_launch_count(launches_before);
  if (!status_ok()) return false;
  NRPYELL_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  NRPYELL_CUDA(cudaGraphDestroy(graph));
  if (!status_ok()) return false;

  // replay until every grid is done, polling the states of launch k-1
  // while launch k runs
  int* pinned = g_batch.pinned;
  cudaEvent_t ev[2];
  NRPYELL_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  NRPYELL_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  const long long max_launches = (long long)max_steps / kBatchStepsPerGraph + 2;
  for (long long k = 0; k < max_launches && status_ok(); k++) {
    NRPYELL_CUDA(cudaGraphLaunch(exec, stream()));
    count_launch(4 * kBatchStepsPerGraph);
    const int slot = (int)(k & 1);
    NRPYELL_CUDA(cudaMemcpyAsync(pinned + slot * kStateInts * n, g_batch.state, sizeof(int) * kStateInts * n,
                                 cudaMemcpyDeviceToHost, stream()));
    NRPYELL_CUDA(cudaEventRecord(ev[slot], stream()));
    if (k > 0) {
      NRPYELL_CUDA(cudaEventSynchronize(ev[1 - slot]));
      const int* st = pinned + (1 - slot) * kStateInts * n;
      bool all = true;
      for (int c = 0; c < n && all; c++) all = st[kStateInts * c + 1] != 0;
      if (all) break;
    }
  }
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  cudaGraphExecDestroy(exec);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  std::vector<int> st(kStateInts * n);
  NRPYELL_CUDA(cudaMemcpy(st.data(), g_batch.state, sizeof(int) * kStateInts * n, cudaMemcpyDeviceToHost));
  if (!status_ok()) return false;
  out->steps.assign(n, 0);
  out->converged.assign(n, 0);
  out->last.assign(n, NAN);
  for (int c = 0; c < n; c++) {
    const int steps = st[kStateInts * c];
    out->steps[c] = steps;
    out->converged[c] = st[kStateInts * c + 2] != 0;
    NRPYELL_CUDA(cudaMemcpy(&out->last[c], g_batch.history + (size_t)c * g_batch.hist_len + steps, sizeof(double),
                            cudaMemcpyDeviceToHost));
  }
  return status_ok();
}

// Grids of a batched call, checked; rc 0, -1 (bad arguments or a CUDA
// error) or -2 (a grid the fused path cannot relax).
int make_grids(const char* who, int n, griddata_struct* grids, const REAL* dt, REAL log10_tol, int max_steps,
               REAL integration_radius, std::vector<Grid>* gs) {
  char msg[256];
  if (n <= 0 || !grids || !dt || max_steps < 0) {
    snprintf(msg, sizeof(msg), "%s: need n > 0, grids, dt and max_steps >= 0", who);
    NRPYELL_FAIL(msg);
    return -1;
  }
  gs->assign(n, Grid());
  for (int c = 0; c < n; c++) {
    griddata_struct* g = &grids[c];
    const MoL_gridfunctions_struct* gf = &g->gridfuncs;
    if (!check_device_pointer(gf->y_n_gfs, "y_n_gfs") ||
        !check_device_pointer(gf->y_nplus1_running_total_gfs, "y_nplus1_running_total_gfs") ||
        !check_device_pointer(gf->k_odd_gfs, "k_odd_gfs") || !check_device_pointer(gf->k_even_gfs, "k_even_gfs") ||
        !check_device_pointer(gf->auxevol_gfs, "auxevol_gfs"))
      return -1;
    Grid& G = (*gs)[c];
    if (!fused_ready(&g->params, &g->rfmstruct, &g->bcstruct, g->xx, &G.rt, &G.bt)) {
      snprintf(msg, sizeof(msg), "%s needs radiation outer BCs with the SymTP inner-boundary map", who);
      NRPYELL_FAIL(msg);
      return -2;
    }
    G.lt = get_l2_tables(&g->params, g->xx, integration_radius);
    if (!G.lt) return -1;
    G.d = dims_of(&g->params);
    G.b = buffers_of(gf);
    memset(&G.rp, 0, sizeof(G.rp));
    G.rp.dt = dt[c];
    G.rp.eta = g->params.eta_damping;
    G.rp.cOB[0] = g->params.uu_wavespeed_at_OB;
    G.rp.cOB[1] = g->params.vv_wavespeed_at_OB;
    G.rp.log10_tol = log10_tol;
    G.rp.max_steps = max_steps;
    G.index = c;
  }
  return 0;
}

// Longest FP32 stretch of nrpyell_relax_batch_mixed between two folds.
constexpr int kMaxFoldEvery = 4096;

}  // namespace

void release_batch() { free_batch(); }

}  // namespace nrpyell

using namespace nrpyell;

extern "C" int nrpyell_relax_batch(const int n, griddata_struct* grids, const REAL* dt, const REAL log10_tol,
                                   const int max_steps, const REAL integration_radius, int* steps_taken,
                                   REAL* final_log10_l2) {
  std::vector<Grid> gs;
  const int rc = make_grids("nrpyell_relax_batch", n, grids, dt, log10_tol, max_steps, integration_radius, &gs);
  if (rc) return rc;
  int tile = -1;
  BatchResult r;
  if (!run_batch<double>(gs, false, &tile, &r)) return -1;
  int not_converged = 0;
  for (int c = 0; c < n; c++) {
    if (!r.converged[c]) not_converged++;
    if (steps_taken) steps_taken[c] = r.steps[c];
    if (final_log10_l2) final_log10_l2[c] = r.last[c];
    // ghost zones of the solution, as the reference's all-points update leaves them
    launch_ghost_fill<double>(gs[c].d, gs[c].bt, grids[c].gridfuncs.y_n_gfs);
  }
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return status_ok() ? not_converged : -1;
}

// The correction form of nrpyell_relax_mixed on a batch: every grid follows
// the single-grid driver's schedule (FP64 evaluation of the base state and
// stop test, an FP32 stretch of up to fold_every steps or to log10_switch,
// the fold; the FP64 phase from the switch on), and the FP32 stretches of all
// grids still in that phase, and then their FP64 phases, run as batches.
extern "C" int nrpyell_relax_batch_mixed(const int n, griddata_struct* grids, const REAL* dt, const REAL log10_tol,
                                         const REAL log10_switch, const int fold_every, const int max_steps,
                                         const REAL integration_radius, int* steps_fp32, int* steps_fp64,
                                         REAL* final_log10_l2) {
  std::vector<Grid> gs;
  const int rc = make_grids("nrpyell_relax_batch_mixed", n, grids, dt, log10_tol, max_steps, integration_radius, &gs);
  if (rc) return rc;
  if (fold_every < 1 || fold_every > kMaxFoldEvery) {
    NRPYELL_FAIL("nrpyell_relax_batch_mixed: need 1 <= fold_every <= 4096");
    return -1;
  }
  size_t floats = 0;
  std::vector<size_t> off(n);
  int max_tiles = 0;
  for (int c = 0; c < n; c++) {
    if (!march_fits(gs[c].d)) {
      NRPYELL_FAIL("nrpyell_relax_batch_mixed: grid too large for the FP32 correction kernels (3 Ntot >= 2^32)");
      return -1;
    }
    off[c] = floats;
    floats += 5 * 2 * (size_t)gs[c].d.Ntot + 3 * (size_t)gs[c].d.Ntot;
    max_tiles = std::max(max_tiles, max_interior_blocks(gs[c].d));
  }
  if (g_mixed.floats < floats || g_mixed.n < n) {
    NRPYELL_CUDA(cudaStreamSynchronize(stream()));
    cudaFree(g_mixed.f32);
    cudaFree(g_mixed.sums);
    g_mixed = MixedWork();
    NRPYELL_CUDA(dev_alloc(&g_mixed.f32, sizeof(float) * floats));
    NRPYELL_CUDA(dev_alloc(&g_mixed.sums, sizeof(double) * n));
    if (!status_ok()) return -1;
    g_mixed.floats = floats;
    g_mixed.n = n;
  }
  Scratch* sc = get_scratch(max_tiles);
  if (!status_ok()) return -1;
  // per grid: the FP32 buffers (as in nrpyell_relax_mixed), steps so far,
  // phase (0 FP32 stretches, 1 converged, 2 FP64 phase or out of steps)
  std::vector<StateBuffers> b32(n);
  for (int c = 0; c < n; c++) {
    const long long n2 = 2 * gs[c].d.Ntot;
    float* f = g_mixed.f32 + off[c];
    b32[c].y = f;
    b32[c].acc = f + n2;
    b32[c].kodd = f + 2 * n2;
    b32[c].keven = f + 3 * n2;
    b32[c].aux = f + 4 * n2;
    b32[c].R0 = f + 4 * n2 + 3 * gs[c].d.Ntot;
  }
  std::vector<int> steps(n, 0), phase(n, 0), n64(n, 0);
  std::vector<char> to_fp64(n, 0);
  std::vector<double> l2(n, NAN), sums(n, 0.0);
  const int cycle_len = std::min(fold_every, max_steps);
  const double finf[2] = {0.0, 0.0};
  int tile32 = -1;
  for (;;) {
    // FP64 evaluation of every base state still in the FP32 phase
    int active = 0;
    for (int c = 0; c < n; c++) {
      if (phase[c] != 0) continue;
      active++;
      const Grid& G = gs[c];
      const paramstruct* p = &grids[c].params;
      MoL_gridfunctions_struct* gf = &grids[c].gridfuncs;
      double* U = gf->y_n_gfs;
      const double cw[2] = {p->uu_wavespeed_at_OB, p->vv_wavespeed_at_OB};
      launch_ghost_fill<double>(G.d, G.bt, U);
      launch_rhs_ref(G.d, p, G.rt, gf->auxevol_gfs, U, gf->k_odd_gfs);
      launch_radiation_bc(G.d, p, G.bt, cw, finf, U, gf->k_odd_gfs);
      launch_residual_ref(G.d, G.rt, gf->auxevol_gfs, U, gf->y_nplus1_running_total_gfs);
      launch_l2_sum(G.d, G.lt, gf->y_nplus1_running_total_gfs, sc);
      NRPYELL_CUDA(cudaMemcpyAsync(g_mixed.sums + c, sc->result, sizeof(double), cudaMemcpyDeviceToDevice, stream()));
      launch_correction_base(G.d, U, gf->auxevol_gfs, gf->k_odd_gfs, gf->y_nplus1_running_total_gfs,
                             (float*)b32[c].R0, (float*)b32[c].aux);
    }
    if (!active) break;
    NRPYELL_CUDA(cudaMemcpyAsync(sums.data(), g_mixed.sums, sizeof(double) * n, cudaMemcpyDeviceToHost, stream()));
    NRPYELL_CUDA(cudaStreamSynchronize(stream()));
    if (!status_ok()) return -1;
    std::vector<Grid> sub;
    for (int c = 0; c < n; c++) {
      if (phase[c] != 0) continue;
      l2[c] = log10(1e-16 + sqrt(sums[c] / gs[c].lt->volume));
      if (l2[c] <= log10_tol) {
        phase[c] = 1;
        continue;
      }
      if (l2[c] <= log10_switch || to_fp64[c] || steps[c] >= max_steps) {
        phase[c] = 2;
        continue;
      }
      Grid G = gs[c];
      G.b = b32[c];
      G.rp.log10_tol = log10_switch;
      G.rp.max_steps = std::min(cycle_len, max_steps - steps[c]);
      NRPYELL_CUDA(cudaMemsetAsync(b32[c].y, 0, sizeof(float) * 2 * (size_t)G.d.Ntot, stream()));
      sub.push_back(G);
    }
    if (sub.empty()) continue;
    // one FP32 stretch of every such grid, then the folds
    BatchResult r;
    if (!run_batch<float>(sub, true, &tile32, &r)) return -1;
    for (size_t k = 0; k < sub.size(); k++) {
      const int c = sub[k].index;
      launch_correction_fold(grids[c].gridfuncs.y_n_gfs, (const float*)b32[c].y, 2 * sub[k].d.Ntot);
      steps[c] += r.steps[k];
      if (r.converged[k] || r.steps[k] == 0) to_fp64[c] = 1;
    }
  }
  // the FP64 phase of the grids that reached the switch
  std::vector<Grid> sub;
  for (int c = 0; c < n; c++) {
    if (phase[c] != 2 || steps[c] >= max_steps) continue;
    Grid G = gs[c];
    G.rp.max_steps = max_steps - steps[c];
    sub.push_back(G);
  }
  std::vector<char> converged(n, 0);
  for (int c = 0; c < n; c++) converged[c] = phase[c] == 1;
  if (!sub.empty()) {
    int tile64 = -1;
    BatchResult r;
    if (!run_batch<double>(sub, false, &tile64, &r)) return -1;
    for (size_t k = 0; k < sub.size(); k++) {
      const int c = sub[k].index;
      n64[c] = r.steps[k];
      converged[c] = r.converged[k];
      l2[c] = r.last[k];
    }
  }
  int not_converged = 0;
  for (int c = 0; c < n; c++) {
    launch_ghost_fill<double>(gs[c].d, gs[c].bt, grids[c].gridfuncs.y_n_gfs);
    if (!converged[c]) not_converged++;
    if (steps_fp32) steps_fp32[c] = steps[c];
    if (steps_fp64) steps_fp64[c] = n64[c];
    if (final_log10_l2) final_log10_l2[c] = l2[c];
  }
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return status_ok() ? not_converged : -1;
}
