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
  int* offs = nullptr;                 // n
  SubDev<double>* devs = nullptr;      // 5 x n: stage 1 with stop test, stages 1..4 (tuning uses 2)
};
BatchWork g_batch;

void free_batch() {
  cudaFree(g_batch.state);
  cudaFree(g_batch.history);
  cudaFree(g_batch.partials);
  cudaFree(g_batch.tickets);
  cudaFree(g_batch.offs);
  cudaFree(g_batch.devs);
  g_batch = BatchWork();
}

bool ensure_batch(int n, int hist_len, int partials_per) {
  if (g_batch.n >= n && g_batch.hist_len >= hist_len && g_batch.partials_per >= partials_per) return true;
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  free_batch();
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
  return status_ok();
}

struct Grid {
  Dims d;
  RfmTables* rt;
  BcTables* bt;
  L2Tables* lt;
  StateBuffers b;
  RelaxParams rp;
};

// Launch arguments of every grid for one tile shape: devs_host[5][n] (stage
// 1 with the stop test, then stages 1..4), block offsets, total blocks.
bool build_devs(const std::vector<Grid>& grids, int tile, std::vector<SubDev<double>>* devs, std::vector<int>* offs,
                int* blocks) {
  const int n = (int)grids.size();
  devs->assign(5 * n, SubDev<double>());
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
      if (!batch_launch_dev<double>(a, &(*devs)[k * n + c])) return false;
    }
    const SubDev<double>& f = (*devs)[c];
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

bool upload_devs(const std::vector<SubDev<double>>& devs, const std::vector<int>& offs) {
  NRPYELL_CUDA(cudaMemcpyAsync(g_batch.devs, devs.data(), sizeof(SubDev<double>) * devs.size(),
                               cudaMemcpyHostToDevice, stream()));
  NRPYELL_CUDA(cudaMemcpyAsync(g_batch.offs, offs.data(), sizeof(int) * offs.size(), cudaMemcpyHostToDevice,
                               stream()));
  return status_ok();
}

// Shared-memory planes and marching shapes of the tile table.
std::vector<int> batch_tiles() {
  std::vector<int> t;
  for (int i = 0; i < substep_num_tiles(); i++)
    if (substep_tile_kind(i) == 4 || substep_tile_kind(i) == 5) t.push_back(i);
  return t;
}

}  // namespace

void release_batch() { free_batch(); }

}  // namespace nrpyell

using namespace nrpyell;

extern "C" int nrpyell_relax_batch(const int n, griddata_struct* grids, const REAL* dt, const REAL log10_tol,
                                   const int max_steps, const REAL integration_radius, int* steps_taken,
                                   REAL* final_log10_l2) {
  if (n <= 0 || !grids || !dt || max_steps < 0) {
    NRPYELL_FAIL("nrpyell_relax_batch: need n > 0, grids, dt and max_steps >= 0");
    return -1;
  }
  std::vector<Grid> gs(n);
  int max_tiles = 0;
  for (int c = 0; c < n; c++) {
    griddata_struct* g = &grids[c];
    const MoL_gridfunctions_struct* gf = &g->gridfuncs;
    if (!check_device_pointer(gf->y_n_gfs, "y_n_gfs") ||
        !check_device_pointer(gf->y_nplus1_running_total_gfs, "y_nplus1_running_total_gfs") ||
        !check_device_pointer(gf->k_odd_gfs, "k_odd_gfs") || !check_device_pointer(gf->k_even_gfs, "k_even_gfs") ||
        !check_device_pointer(gf->auxevol_gfs, "auxevol_gfs"))
      return -1;
    Grid& G = gs[c];
    if (!fused_ready(&g->params, &g->rfmstruct, &g->bcstruct, g->xx, &G.rt, &G.bt)) {
      NRPYELL_FAIL("nrpyell_relax_batch needs radiation outer BCs with the SymTP inner-boundary map");
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
    max_tiles = std::max(max_tiles, max_interior_blocks(G.d));
  }
  if (!ensure_batch(n, max_steps + 1, max_tiles)) return -1;

  // tile shape: forced planes or marching shape, else the fastest on this batch
  bool fits = true;
  for (const Grid& G : gs) fits = fits && march_fits(G.d);
  std::vector<int> cands;
  for (int t : batch_tiles())
    if (fits || substep_tile_kind(t) != 5) cands.push_back(t);
  int tile = -1;
  if (g_forced_tile >= 0 && (substep_tile_kind(g_forced_tile) == 4 || substep_tile_kind(g_forced_tile) == 5))
    tile = g_forced_tile;
  std::vector<SubDev<double>> devs;
  std::vector<int> offs;
  int blocks = 0;
  NRPYELL_CUDA(cudaMemsetAsync(g_batch.state, 0, sizeof(int) * kStateInts * n, stream()));
  if (tile < 0) {
    cudaEvent_t e0, e1;
    NRPYELL_CUDA(cudaEventCreate(&e0));
    NRPYELL_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int t : cands) {
      if (!build_devs(gs, t, &devs, &offs, &blocks) || !upload_devs(devs, offs)) return -1;
      const SubDev<double>* d2 = g_batch.devs + 2 * n;  // stage 2: writes only k_even and the running total
      launch_substep_batch<double>(2, false, t, d2, g_batch.offs, n, blocks);
      float tmin = 1e30f;
      for (int rep = 0; rep < 3; rep++) {
        NRPYELL_CUDA(cudaEventRecord(e0, stream()));
        for (int i = 0; i < 5; i++) launch_substep_batch<double>(2, false, t, d2, g_batch.offs, n, blocks);
        NRPYELL_CUDA(cudaEventRecord(e1, stream()));
        NRPYELL_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        NRPYELL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        tmin = std::min(tmin, ms);
      }
      if (tmin < best) {
        best = tmin;
        tile = t;
      }
    }
    NRPYELL_CUDA(cudaEventDestroy(e0));
    NRPYELL_CUDA(cudaEventDestroy(e1));
  }
  if (tile < 0 || !build_devs(gs, tile, &devs, &offs, &blocks) || !upload_devs(devs, offs)) return -1;
  NRPYELL_CUDA(cudaMemsetAsync(g_batch.state, 0, sizeof(int) * kStateInts * n, stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  if (!status_ok()) return -1;

  // capture sixteen RK4 steps of the whole batch
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  const long long launches_before = launch_count();
  NRPYELL_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < kBatchStepsPerGraph; k++) {
    launch_substep_batch<double>(1, true, tile, g_batch.devs, g_batch.offs, n, blocks);
    for (int st = 2; st <= 4; st++)
      launch_substep_batch<double>(st, false, tile, g_batch.devs + (size_t)st * n, g_batch.offs, n, blocks);
  }
  NRPYELL_CUDA(cudaStreamEndCapture(stream(), &graph));
  set_launch_count(launches_before);
  if (!status_ok()) return -1;
  NRPYELL_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  NRPYELL_CUDA(cudaGraphDestroy(graph));
  if (!status_ok()) return -1;

  // replay until every grid is done, polling the states of launch k-1
  // while launch k runs
  int* pinned = nullptr;
  NRPYELL_CUDA(cudaMallocHost(&pinned, sizeof(int) * kStateInts * n * 2));
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
      for (int c = 0; c < n && all; c++) all = st[kStateInts * c + 1] != 0 || st[kStateInts * c + 5] != 0;
      if (all) break;
    }
  }
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  cudaGraphExecDestroy(exec);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  std::vector<int> st(kStateInts * n);
  NRPYELL_CUDA(cudaMemcpy(st.data(), g_batch.state, sizeof(int) * kStateInts * n, cudaMemcpyDeviceToHost));
  cudaFreeHost(pinned);
  if (!status_ok()) return -1;
  int not_converged = 0;
  for (int c = 0; c < n; c++) {
    const int steps = st[kStateInts * c];
    if (st[kStateInts * c + 5]) {
      NRPYELL_FAIL("nrpyell_relax_batch: a bounded wait gave up");
      return -1;
    }
    if (!st[kStateInts * c + 2]) not_converged++;
    double last = NAN;
    NRPYELL_CUDA(cudaMemcpy(&last, g_batch.history + (size_t)c * g_batch.hist_len + steps, sizeof(double),
                            cudaMemcpyDeviceToHost));
    if (steps_taken) steps_taken[c] = steps;
    if (final_log10_l2) final_log10_l2[c] = last;
    // ghost zones of the solution, as the reference's all-points update leaves them
    launch_ghost_fill<double>(gs[c].d, gs[c].bt, grids[c].gridfuncs.y_n_gfs);
  }
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return status_ok() ? not_converged : -1;
}
