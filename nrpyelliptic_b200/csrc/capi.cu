// extern "C" entry points of libnrpyell_gpu: the reference prototypes of the
// hot path (NRPy_function_prototypes.h) plus the library extensions declared
// in include/nrpyell_gpu.h.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace nrpyell {

namespace {
int g_status = 0;
std::string g_error;
bool g_exit_on_error = true;
long long g_launches = 0;
int g_step_mode = NRPYELL_STEP_FUSED;
bool g_async = false;
cudaStream_t g_stream = nullptr;
}  // namespace

void report_error(const char* file, int line, const char* what) {
  char buf[1024];
  snprintf(buf, sizeof(buf), "%s:%d %s", file, line, what);
  if (g_status == 0) {
    g_status = 1;
    g_error = buf;
  }
  fprintf(stderr, "nrpyell_gpu error: %s\n", buf);
  if (g_exit_on_error) exit(1);
}

bool status_ok() { return g_status == 0; }

cudaStream_t stream() {
  if (!g_stream) {
    cudaError_t e = cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      g_stream = nullptr;
      report_error(__FILE__, __LINE__, cudaGetErrorString(e));
    }
  }
  return g_stream;
}

cudaStream_t existing_stream() { return g_stream; }

void count_launch(int n) { g_launches += n; }

bool check_device_pointer(const void* ptr, const char* what) {
  char msg[256];
  if (!ptr) {
    snprintf(msg, sizeof(msg), "%s is NULL", what);
    NRPYELL_FAIL(msg);
    return false;
  }
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    snprintf(msg, sizeof(msg), "%s: cudaPointerGetAttributes failed (%s)", what, cudaGetErrorString(e));
    NRPYELL_FAIL(msg);
    return false;
  }
  if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) return true;
  if (attr.type == cudaMemoryTypeHost && attr.devicePointer == ptr) return true;
  snprintf(msg, sizeof(msg),
           "%s is not device-accessible memory (allocate it with MoL_malloc_*, nrpyell_device_malloc, "
           "cudaMalloc or cudaMallocManaged)",
           what);
  NRPYELL_FAIL(msg);
  return false;
}

// ---------------------------------------------------------------------------
// One RK4 step, reference order: rhs_eval, radiation BC + inner copy on the
// RHS, linear combination over all points (MoL_step_forward_in_time.c:7-178).
static void mol_step_reference_order(griddata_struct* g, double dt) {
  const paramstruct* p = &g->params;
  const Dims d = dims_of(p);
  MoL_gridfunctions_struct* gf = &g->gridfuncs;
  RfmTables* rt = get_rfm_tables(p, &g->rfmstruct);
  BcTables* bt = get_bc_tables(p, &g->bcstruct, g->xx);
  if (!rt || !bt) return;
  const double c[2] = {p->uu_wavespeed_at_OB, p->vv_wavespeed_at_OB};
  const double finf[2] = {0.0, 0.0};
  const long long n = d.Ntot * NUM_EVOL_GFS;
  double* stage_in[4] = {gf->y_n_gfs, gf->k_odd_gfs, gf->k_even_gfs, gf->k_odd_gfs};
  double* stage_k[4] = {gf->k_odd_gfs, gf->k_even_gfs, gf->k_odd_gfs, gf->k_even_gfs};
  for (int s = 0; s < 4; s++) {
    launch_rhs_ref(d, p, rt, gf->auxevol_gfs, stage_in[s], stage_k[s]);
    if (p->outer_bc_type == RADIATION_OUTER_BCS) {
      launch_radiation_bc(d, p, bt, c, finf, stage_in[s], stage_k[s]);
      launch_inner_copy(d, bt, stage_k[s], NUM_EVOL_GFS);
    }
    // stage s writes its combination into the k buffer it just read (k_odd /
    // k_even), or into y_n at stage 4
    double* out = (s == 3) ? gf->y_n_gfs : stage_k[s];
    launch_rk_update_ref(s + 1, n, dt, stage_k[s], gf->y_n_gfs, gf->y_nplus1_running_total_gfs, out);
    if (p->outer_bc_type == EXTRAPOLATION_OUTER_BCS) launch_extrap_bc(d, bt, &g->bcstruct, out);
  }
}

// Driver state of the fused path, per grid size.
struct FusedWork {
  Dims d;
  int* state;        // [0] n, [1] done, [2] converged
  int* zero_flag;    // always 0 (MoL_step_forward_in_time runs unconditionally)
  double* history;
  int history_len;
  int tile[2];       // autotuned tile shape for FP64 / FP32, -1 = not yet tuned
};
static std::vector<FusedWork*> g_work;
static int g_work_generation = 0;  // bumped when a work buffer is reallocated

// Never call while a stream is being captured (it may allocate).
static FusedWork* get_work(const Dims& d, int history_len) {
  for (FusedWork* w : g_work)
    if (w->d.Nxx1 == d.Nxx1 && w->d.Nxx2 == d.Nxx2 && w->d.N0 == d.N0 && w->d.N1 == d.N1 && w->d.N2 == d.N2) {
      if (w->history_len < history_len) {
        g_work_generation++;
        NRPYELL_CUDA(cudaStreamSynchronize(stream()));
        NRPYELL_CUDA(cudaFree(w->history));
        NRPYELL_CUDA(cudaMalloc(&w->history, sizeof(double) * history_len));
        w->history_len = history_len;
      }
      return w;
    }
  FusedWork* w = new FusedWork();
  w->d = d;
  w->tile[0] = w->tile[1] = -1;
  NRPYELL_CUDA(cudaMalloc(&w->state, sizeof(int) * 8));
  NRPYELL_CUDA(cudaMemset(w->state, 0, sizeof(int) * 8));
  w->zero_flag = w->state + 4;
  w->history_len = history_len > 16 ? history_len : 16;
  NRPYELL_CUDA(cudaMalloc(&w->history, sizeof(double) * w->history_len));
  g_work.push_back(w);
  return w;
}

static void release_work() {
  for (FusedWork* w : g_work) {
    cudaFree(w->state);
    cudaFree(w->history);
    delete w;
  }
  g_work.clear();
}

static bool fused_ready(griddata_struct* g, RfmTables** rt, BcTables** bt) {
  const paramstruct* p = &g->params;
  *rt = get_rfm_tables(p, &g->rfmstruct);
  *bt = get_bc_tables(p, &g->bcstruct, g->xx);
  return *rt && *bt && (*bt)->columns_ok && (*bt)->analytic_ok && p->outer_bc_type == RADIATION_OUTER_BCS;
}

static int g_forced_tile = -1;

static SubstepArgs substep_args(griddata_struct* g, RfmTables* rt, BcTables* bt, FusedWork* w, Scratch* s,
                                double dt, int stage, const int* done, int tile) {
  const paramstruct* p = &g->params;
  MoL_gridfunctions_struct* gf = &g->gridfuncs;
  SubstepArgs a;
  a.d = dims_of(p);
  double* S[4] = {gf->y_n_gfs, gf->k_odd_gfs, gf->k_even_gfs, gf->k_odd_gfs};
  double* O[4] = {gf->k_odd_gfs, gf->k_even_gfs, gf->k_odd_gfs, gf->y_n_gfs};
  a.S = S[stage - 1];
  a.out = O[stage - 1];
  a.y = gf->y_n_gfs;
  a.acc = gf->y_nplus1_running_total_gfs;
  a.aux = gf->auxevol_gfs;
  a.dt = dt;
  a.eta = p->eta_damping;
  a.cOB[0] = p->uu_wavespeed_at_OB;
  a.cOB[1] = p->vv_wavespeed_at_OB;
  a.rt = rt;
  a.bt = bt;
  a.lt = nullptr;
  a.s = s;
  a.state = w->state;
  a.history = nullptr;
  a.log10_tol = -1e300;
  a.max_steps = 0;
  a.done = done;
  a.tile = tile;
  (void)w;
  return a;
}

static int max_interior_blocks(const Dims& d) {
  int m = 0;
  for (int t = 0; t < substep_num_tiles(); t++) m = std::max(m, substep_interior_blocks(d, t));
  return m;
}

// Tile-shape autotuner: times the stage-2 fused substep (the most common
// kind) for every tile shape on the caller's own buffers and keeps the
// fastest, once per grid size and precision.  The timing launches write only
// the running-total and k_even buffers, which every RK4 step overwrites
// before reading.
template <typename T>
static int tuned_tile(griddata_struct* g, RfmTables* rt, BcTables* bt, FusedWork* w, Scratch* sc, double dt) {
  const int which = sizeof(T) == 8 ? 0 : 1;
  if (g_forced_tile >= 0) return g_forced_tile;
  if (w->tile[which] >= 0) return w->tile[which];
  cudaEvent_t e0, e1;
  NRPYELL_CUDA(cudaEventCreate(&e0));
  NRPYELL_CUDA(cudaEventCreate(&e1));
  int best = 0;
  float best_ms = 1e30f;
  const int reps = 10;
  for (int t = 0; t < substep_num_tiles(); t++) {
    SubstepArgs a = substep_args(g, rt, bt, w, sc, dt, 2, w->zero_flag, t);
    launch_substep<T>(2, a);  // warm-up
    NRPYELL_CUDA(cudaEventRecord(e0, stream()));
    for (int i = 0; i < reps; i++) launch_substep<T>(2, a);
    NRPYELL_CUDA(cudaEventRecord(e1, stream()));
    NRPYELL_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    NRPYELL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  }
  NRPYELL_CUDA(cudaEventDestroy(e0));
  NRPYELL_CUDA(cudaEventDestroy(e1));
  w->tile[which] = best;
  return best;
}

static void mol_step_fused(griddata_struct* g, double dt) {
  RfmTables* rt;
  BcTables* bt;
  if (!fused_ready(g, &rt, &bt)) {
    mol_step_reference_order(g, dt);
    return;
  }
  const Dims d = dims_of(&g->params);
  FusedWork* w = get_work(d, 16);
  Scratch* sc = get_scratch(max_interior_blocks(d));
  const int tile = tuned_tile<double>(g, rt, bt, w, sc, dt);
  for (int s = 1; s <= 4; s++) launch_substep<double>(s, substep_args(g, rt, bt, w, sc, dt, s, w->zero_flag, tile));
  // the fused kernels read ghost values from their sources; give y_n the
  // ghost zones the reference's all-points update leaves in it
  launch_ghost_fill<double>(d, bt, g->gridfuncs.y_n_gfs);
}

static bool check_gridfuncs(const MoL_gridfunctions_struct* gf) {
  return check_device_pointer(gf->y_n_gfs, "y_n_gfs") &&
         check_device_pointer(gf->y_nplus1_running_total_gfs, "y_nplus1_running_total_gfs") &&
         check_device_pointer(gf->k_odd_gfs, "k_odd_gfs") && check_device_pointer(gf->k_even_gfs, "k_even_gfs") &&
         check_device_pointer(gf->auxevol_gfs, "auxevol_gfs");
}

// Graph-cached relaxation: a CUDA graph of kStepsPerGraph RK4 steps (each
// preceded by the fused residual/L2 test) is replayed until the device-side
// state says done.  Kernels after convergence return at entry.
constexpr int kStepsPerGraph = 16;

struct RelaxGraph {
  griddata_struct key;
  double dt, tol, R;
  int max_steps;
  int scratch_gen, work_gen;  // buffers the graph was captured with
  int tile;
  cudaGraphExec_t exec;
  size_t nodes;
};
static std::vector<RelaxGraph*> g_graphs;

static void release_graphs() {
  for (RelaxGraph* r : g_graphs) {
    cudaGraphExecDestroy(r->exec);
    delete r;
  }
  g_graphs.clear();
}

static bool same_grid(const griddata_struct* a, const griddata_struct* b) {
  return memcmp(&a->params, &b->params, sizeof(paramstruct)) == 0 && a->xx[0] == b->xx[0] && a->xx[1] == b->xx[1] &&
         a->xx[2] == b->xx[2] && a->bcstruct.inner_bc_array == b->bcstruct.inner_bc_array &&
         a->rfmstruct.f0_of_xx0 == b->rfmstruct.f0_of_xx0 &&
         memcmp(&a->gridfuncs, &b->gridfuncs, sizeof(MoL_gridfunctions_struct)) == 0;
}

// The reference's functions return when their work is done, and callers such
// as main.c read managed gridfunctions on the host right after a call; the
// Part-1 entry points therefore wait for their kernels unless the caller
// opted into asynchronous calls.
static void finish_call() {
  if (!g_async) NRPYELL_CUDA(cudaStreamSynchronize(stream()));
}

}  // namespace nrpyell

using namespace nrpyell;

extern "C" {

int nrpyell_last_status(void) { return g_status; }
const char* nrpyell_last_error(void) { return g_error.c_str(); }
void nrpyell_clear_status(void) {
  g_status = 0;
  g_error.clear();
}
void nrpyell_set_exit_on_error(int enable) { g_exit_on_error = enable != 0; }
long long nrpyell_launch_count(void) { return g_launches; }

int nrpyell_abi_layout(int* out, int n) {
  const int v[] = {(int)sizeof(paramstruct),
                   (int)sizeof(rfm_struct),
                   (int)sizeof(innerpt_bc_struct),
                   (int)sizeof(outerpt_bc_struct),
                   (int)sizeof(bc_info_struct),
                   (int)sizeof(bc_struct),
                   (int)sizeof(MoL_gridfunctions_struct),
                   (int)sizeof(griddata_struct),
                   (int)offsetof(paramstruct, Nxx0),
                   (int)offsetof(paramstruct, outer_bc_type),
                   (int)offsetof(griddata_struct, xx),
                   (int)offsetof(griddata_struct, bcstruct),
                   (int)offsetof(griddata_struct, rfmstruct),
                   (int)offsetof(griddata_struct, gridfuncs),
                   NGHOSTS};
  const int m = (int)(sizeof(v) / sizeof(v[0]));
  int k = 0;
  for (; k < m && k < n; k++) out[k] = v[k];
  return k;
}

void nrpyell_set_step_mode(int mode) { g_step_mode = mode; }
void nrpyell_set_async(int enable) { g_async = enable != 0; }

void nrpyell_set_tile(int tile) { g_forced_tile = (tile >= 0 && tile < substep_num_tiles()) ? tile : -1; }

int nrpyell_get_tile(const paramstruct* params, int fp32, int* bx, int* by, int* planes) {
  const Dims d = dims_of(params);
  int tile = g_forced_tile;
  if (tile < 0)
    for (FusedWork* w : g_work)
      if (w->d.N0 == d.N0 && w->d.N1 == d.N1 && w->d.N2 == d.N2) tile = w->tile[fp32 ? 1 : 0];
  if (tile >= 0 && bx && by && planes) substep_tile_shape(tile, bx, by, planes);
  return tile;
}
int nrpyell_get_step_mode(void) { return g_step_mode; }

int nrpyell_set_device(int device) {
  NRPYELL_CUDA(cudaSetDevice(device));
  return g_status;
}

void nrpyell_synchronize(void) { NRPYELL_CUDA(cudaStreamSynchronize(stream())); }

static cudaEvent_t g_events[16];
static bool g_events_made = false;

int nrpyell_event_record(int slot) {
  if (slot < 0 || slot >= 16) {
    NRPYELL_FAIL("nrpyell_event_record: slot out of range");
    return -1;
  }
  if (!g_events_made) {
    for (int i = 0; i < 16; i++) NRPYELL_CUDA(cudaEventCreate(&g_events[i]));
    g_events_made = true;
  }
  NRPYELL_CUDA(cudaEventRecord(g_events[slot], stream()));
  return g_status;
}

float nrpyell_event_elapsed_ms(int a, int b) {
  if (!g_events_made || a < 0 || a >= 16 || b < 0 || b >= 16) {
    NRPYELL_FAIL("nrpyell_event_elapsed_ms: events not recorded");
    return -1.0f;
  }
  float ms = -1.0f;
  NRPYELL_CUDA(cudaEventSynchronize(g_events[b]));
  NRPYELL_CUDA(cudaEventElapsedTime(&ms, g_events[a], g_events[b]));
  return ms;
}

void nrpyell_flush_l2(void) {
  static void* buf = nullptr;
  const size_t bytes = (size_t)256 << 20;
  if (!buf) NRPYELL_CUDA(cudaMalloc(&buf, bytes));
  NRPYELL_CUDA(cudaMemsetAsync(buf, 0x5a, bytes, stream()));
}

int nrpyell_time_fused(griddata_struct* g, const REAL dt, const int stage, const int n_iter, double* ms_interior,
                       double* ms_step) {
  if (!check_gridfuncs(&g->gridfuncs)) return -1;
  RfmTables* rt;
  BcTables* bt;
  if (!fused_ready(g, &rt, &bt) || stage < 1 || stage > 4 || n_iter < 1) {
    NRPYELL_FAIL("nrpyell_time_fused: fused path unavailable for this grid or bad arguments");
    return -2;
  }
  const Dims d = dims_of(&g->params);
  FusedWork* w = get_work(d, 16);
  Scratch* sc = get_scratch(max_interior_blocks(d));
  const int tile = tuned_tile<double>(g, rt, bt, w, sc, dt);
  cudaEvent_t e0, e1;
  NRPYELL_CUDA(cudaEventCreate(&e0));
  NRPYELL_CUDA(cudaEventCreate(&e1));
  for (int which = 0; which < 2; which++) {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    const long long before = g_launches;
    NRPYELL_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < n_iter; i++) {
      if (which == 0) {
        launch_substep<double>(stage, substep_args(g, rt, bt, w, sc, dt, stage, w->zero_flag, tile));
      } else {
        for (int s = 1; s <= 4; s++)
          launch_substep<double>(s, substep_args(g, rt, bt, w, sc, dt, s, w->zero_flag, tile));
      }
    }
    NRPYELL_CUDA(cudaStreamEndCapture(stream(), &graph));
    const long long captured = g_launches - before;
    g_launches = before;
    NRPYELL_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    NRPYELL_CUDA(cudaGraphLaunch(exec, stream()));  // warm-up
    NRPYELL_CUDA(cudaEventRecord(e0, stream()));
    NRPYELL_CUDA(cudaGraphLaunch(exec, stream()));
    NRPYELL_CUDA(cudaEventRecord(e1, stream()));
    g_launches += 2 * captured;
    NRPYELL_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    NRPYELL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (which == 0 && ms_interior) *ms_interior = ms / n_iter;
    if (which == 1 && ms_step) *ms_step = ms / n_iter;
    NRPYELL_CUDA(cudaGraphExecDestroy(exec));
    NRPYELL_CUDA(cudaGraphDestroy(graph));
  }
  NRPYELL_CUDA(cudaEventDestroy(e0));
  NRPYELL_CUDA(cudaEventDestroy(e1));
  return g_status ? -1 : 0;
}

void nrpyell_release_tables(void) {
  if (g_stream) cudaStreamSynchronize(g_stream);
  release_graphs();
  release_work();
  release_all_tables();
}

void* nrpyell_device_malloc(size_t bytes) {
  void* p = nullptr;
  NRPYELL_CUDA(cudaMalloc(&p, bytes));
  return p;
}
void nrpyell_device_free(void* ptr) {
  if (ptr) NRPYELL_CUDA(cudaFree(ptr));
}
void* nrpyell_host_pinned_malloc(size_t bytes) {
  void* p = nullptr;
  NRPYELL_CUDA(cudaMallocHost(&p, bytes));
  return p;
}
void nrpyell_host_pinned_free(void* ptr) {
  if (ptr) NRPYELL_CUDA(cudaFreeHost(ptr));
}
int nrpyell_memcpy(void* dst, const void* src, size_t bytes, int kind) {
  const cudaMemcpyKind k[4] = {cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice,
                               cudaMemcpyDefault};
  if (kind < 0 || kind > 3) kind = 3;
  NRPYELL_CUDA(cudaMemcpyAsync(dst, src, bytes, k[kind], stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return g_status;
}
int nrpyell_memset(void* dst, int value, size_t bytes) {
  NRPYELL_CUDA(cudaMemsetAsync(dst, value, bytes, stream()));
  return g_status;
}

// ---- allocators (MoL_malloc_*.c): managed memory, so the host set-up code
// of the caller can fill the arrays in place.
void MoL_malloc_y_n_gfs(const paramstruct* params, MoL_gridfunctions_struct* gridfuncs) {
  const size_t n = (size_t)params->Nxx_plus_2NGHOSTS0 * params->Nxx_plus_2NGHOSTS1 * params->Nxx_plus_2NGHOSTS2;
  void* p = nullptr;
  NRPYELL_CUDA(cudaMallocManaged(&p, sizeof(REAL) * NUM_EVOL_GFS * n));
  gridfuncs->y_n_gfs = (REAL*)p;
  gridfuncs->diagnostic_output_gfs = gridfuncs->y_nplus1_running_total_gfs;
}
void MoL_free_memory_y_n_gfs(const paramstruct* params, MoL_gridfunctions_struct* gridfuncs) {
  (void)params;
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  NRPYELL_CUDA(cudaFree(gridfuncs->y_n_gfs));
  gridfuncs->y_n_gfs = nullptr;
}
void MoL_malloc_non_y_n_gfs(const paramstruct* params, MoL_gridfunctions_struct* gridfuncs) {
  const size_t n = (size_t)params->Nxx_plus_2NGHOSTS0 * params->Nxx_plus_2NGHOSTS1 * params->Nxx_plus_2NGHOSTS2;
  void* p[4] = {nullptr, nullptr, nullptr, nullptr};
  NRPYELL_CUDA(cudaMallocManaged(&p[0], sizeof(REAL) * NUM_EVOL_GFS * n));
  NRPYELL_CUDA(cudaMallocManaged(&p[1], sizeof(REAL) * NUM_EVOL_GFS * n));
  NRPYELL_CUDA(cudaMallocManaged(&p[2], sizeof(REAL) * NUM_EVOL_GFS * n));
  NRPYELL_CUDA(cudaMallocManaged(&p[3], sizeof(REAL) * NUM_AUXEVOL_GFS * n));
  gridfuncs->y_nplus1_running_total_gfs = (REAL*)p[0];
  gridfuncs->k_odd_gfs = (REAL*)p[1];
  gridfuncs->k_even_gfs = (REAL*)p[2];
  gridfuncs->auxevol_gfs = (REAL*)p[3];
  gridfuncs->diagnostic_output_gfs = gridfuncs->y_nplus1_running_total_gfs;
}
void MoL_free_memory_non_y_n_gfs(const paramstruct* params, MoL_gridfunctions_struct* gridfuncs) {
  (void)params;
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  NRPYELL_CUDA(cudaFree(gridfuncs->y_nplus1_running_total_gfs));
  NRPYELL_CUDA(cudaFree(gridfuncs->k_odd_gfs));
  NRPYELL_CUDA(cudaFree(gridfuncs->k_even_gfs));
  NRPYELL_CUDA(cudaFree(gridfuncs->auxevol_gfs));
  gridfuncs->y_nplus1_running_total_gfs = gridfuncs->k_odd_gfs = gridfuncs->k_even_gfs = nullptr;
  gridfuncs->auxevol_gfs = gridfuncs->diagnostic_output_gfs = nullptr;
}

// ---- hot path ----
void rhs_eval(const paramstruct* params, const rfm_struct* rfmstruct, const REAL* auxevol_gfs, const REAL* in_gfs,
              REAL* rhs_gfs) {
  if (!check_device_pointer(auxevol_gfs, "auxevol_gfs") || !check_device_pointer(in_gfs, "in_gfs") ||
      !check_device_pointer(rhs_gfs, "rhs_gfs"))
    return;
  RfmTables* rt = get_rfm_tables(params, rfmstruct);
  if (!rt) return;
  launch_rhs_ref(dims_of(params), params, rt, auxevol_gfs, in_gfs, rhs_gfs);
  finish_call();
}

void residual_all_points(const paramstruct* params, const rfm_struct* rfmstruct, const REAL* auxevol_gfs,
                         const REAL* in_gfs, REAL* residual_gf) {
  if (!check_device_pointer(auxevol_gfs, "auxevol_gfs") || !check_device_pointer(in_gfs, "in_gfs") ||
      !check_device_pointer(residual_gf, "residual_gf"))
    return;
  RfmTables* rt = get_rfm_tables(params, rfmstruct);
  if (!rt) return;
  launch_residual_ref(dims_of(params), rt, auxevol_gfs, in_gfs, residual_gf);
  finish_call();
}

void apply_bcs_outerradiation_and_inner(const paramstruct* params, const bc_struct* bcstruct,
                                        REAL* NRPYELL_RESTRICT xx[3],
                                        const REAL custom_wavespeed[NUM_EVOL_GFS],
                                        const REAL custom_f_infinity[NUM_EVOL_GFS], REAL* gfs, REAL* rhs_gfs) {
  if (!check_device_pointer(gfs, "gfs") || !check_device_pointer(rhs_gfs, "rhs_gfs")) return;
  BcTables* bt = get_bc_tables(params, bcstruct, xx);
  if (!bt) return;
  const Dims d = dims_of(params);
  launch_radiation_bc(d, params, bt, custom_wavespeed, custom_f_infinity, gfs, rhs_gfs);
  launch_inner_copy(d, bt, rhs_gfs, NUM_EVOL_GFS);
  finish_call();
}

void apply_bcs_inner_only(const paramstruct* params, const bc_struct* bcstruct, REAL* gfs) {
  if (!check_device_pointer(gfs, "gfs")) return;
  REAL* NRPYELL_RESTRICT noxx[3] = {nullptr, nullptr, nullptr};
  BcTables* bt = get_bc_tables(params, bcstruct, noxx);
  if (!bt) return;
  launch_inner_copy(dims_of(params), bt, gfs, NUM_EVOL_GFS);
  finish_call();
}

void apply_bcs_outerextrap_and_inner(const paramstruct* params, const bc_struct* bcstruct, REAL* gfs) {
  if (!check_device_pointer(gfs, "gfs")) return;
  REAL* NRPYELL_RESTRICT noxx[3] = {nullptr, nullptr, nullptr};
  BcTables* bt = get_bc_tables(params, bcstruct, noxx);
  if (!bt) return;
  launch_extrap_bc(dims_of(params), bt, bcstruct, gfs);
  finish_call();
}

void MoL_step_forward_in_time(griddata_struct* griddata, const REAL dt) {
  if (!check_gridfuncs(&griddata->gridfuncs)) return;
  if (g_step_mode == NRPYELL_STEP_REFERENCE_ORDER)
    mol_step_reference_order(griddata, dt);
  else
    mol_step_fused(griddata, dt);
  finish_call();
}

REAL L2_norm_of_gf(const paramstruct* params, const int gf_index, const REAL integration_radius,
                   REAL* NRPYELL_RESTRICT xx[3],
                   const REAL* in_gf) {
  if (!check_device_pointer(in_gf, "in_gf")) return NAN;
  L2Tables* lt = get_l2_tables(params, xx, integration_radius);
  if (!lt) return NAN;
  const Dims d = dims_of(params);
  Scratch* s = get_scratch(1024);
  launch_l2_sum(d, lt, in_gf + (long long)gf_index * d.Ntot, s);
  double sum = 0.0;
  NRPYELL_CUDA(cudaMemcpyAsync(&sum, s->result, sizeof(double), cudaMemcpyDeviceToHost, stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  if (!status_ok()) return NAN;
  return log10(1e-16 + sqrt(sum / lt->volume));
}

int nrpyell_relax(griddata_struct* g, const REAL dt, const REAL log10_tol, const int max_steps,
                  const REAL integration_radius, int* steps_taken, REAL* final_log10_l2, REAL* history) {
  if (max_steps < 0) {
    NRPYELL_FAIL("nrpyell_relax: max_steps < 0");
    return -1;
  }
  if (!check_gridfuncs(&g->gridfuncs)) return -1;
  RfmTables* rt;
  BcTables* bt;
  if (!fused_ready(g, &rt, &bt)) {
    NRPYELL_FAIL("nrpyell_relax needs radiation outer BCs whose pure outer points form the x0max face");
    return -2;
  }
  L2Tables* lt = get_l2_tables(&g->params, g->xx, integration_radius);
  if (!lt) return -1;
  const Dims d = dims_of(&g->params);
  FusedWork* w = get_work(d, max_steps + 1);
  Scratch* s = get_scratch(max_interior_blocks(d));
  const int tile = tuned_tile<double>(g, rt, bt, w, s, dt);

  RelaxGraph* rg = nullptr;
  for (size_t i = 0; i < g_graphs.size(); i++) {
    RelaxGraph* r = g_graphs[i];
    if (r->scratch_gen != scratch_generation() || r->work_gen != g_work_generation) {
      // captured with buffers that have since been reallocated
      NRPYELL_CUDA(cudaGraphExecDestroy(r->exec));
      delete r;
      g_graphs.erase(g_graphs.begin() + i);
      i--;
      continue;
    }
    if (same_grid(&r->key, g) && r->dt == dt && r->tol == log10_tol && r->R == integration_radius &&
        r->max_steps == max_steps && r->tile == tile)
      rg = r;
  }
  if (!rg) {
    cudaGraph_t graph;
    const long long launches_before = g_launches;
    NRPYELL_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kStepsPerGraph; k++) {
      // stage 1 also evaluates the residual of y_n and runs the stop test
      SubstepArgs a1 = substep_args(g, rt, bt, w, s, dt, 1, w->state + 1, tile);
      a1.lt = lt;
      a1.history = w->history;
      a1.log10_tol = log10_tol;
      a1.max_steps = max_steps;
      launch_substep<double>(1, a1);
      for (int st = 2; st <= 4; st++)
        launch_substep<double>(st, substep_args(g, rt, bt, w, s, dt, st, w->state + 1, tile));
    }
    NRPYELL_CUDA(cudaStreamEndCapture(stream(), &graph));
    g_launches = launches_before;  // captured launches run when the graph does
    if (!status_ok()) return -1;
    rg = new RelaxGraph();
    rg->nodes = 0;
    NRPYELL_CUDA(cudaGraphGetNodes(graph, nullptr, &rg->nodes));
    rg->key = *g;
    rg->dt = dt;
    rg->tol = log10_tol;
    rg->R = integration_radius;
    rg->max_steps = max_steps;
    rg->scratch_gen = scratch_generation();
    rg->work_gen = g_work_generation;
    rg->tile = tile;
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
  const long long max_launches = (long long)max_steps / kStepsPerGraph + 2;
  for (long long k = 0; k < max_launches; k++) {
    NRPYELL_CUDA(cudaGraphLaunch(rg->exec, stream()));
    count_launch((int)rg->nodes);
    const int slot = (int)(k & 1);
    NRPYELL_CUDA(cudaMemcpyAsync(pinned + 4 * slot, w->state, sizeof(int) * 4, cudaMemcpyDeviceToHost, stream()));
    NRPYELL_CUDA(cudaEventRecord(ev[slot], stream()));
    if (k > 0) {
      NRPYELL_CUDA(cudaEventSynchronize(ev[1 - slot]));
      if (pinned[4 * (1 - slot) + 1]) break;
    }
    if (!status_ok()) return -1;
  }
  // ghost zones of the solution, as the reference's all-points update leaves them
  launch_ghost_fill<double>(d, bt, g->gridfuncs.y_n_gfs);
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  int st[4];
  NRPYELL_CUDA(cudaMemcpy(st, w->state, sizeof(st), cudaMemcpyDeviceToHost));
  if (!status_ok()) return -1;
  const int n = st[0];
  double last = NAN;
  NRPYELL_CUDA(cudaMemcpy(&last, w->history + n, sizeof(double), cudaMemcpyDeviceToHost));
  if (history) NRPYELL_CUDA(cudaMemcpy(history, w->history, sizeof(double) * (n + 1), cudaMemcpyDeviceToHost));
  if (steps_taken) *steps_taken = n;
  if (final_log10_l2) *final_log10_l2 = last;
  if (!status_ok()) return -1;
  return st[2] ? 0 : 1;
}

int nrpyell_relax_host(const paramstruct* params, REAL* xx[3], const bc_struct* bcstruct, const rfm_struct* rfmstruct,
                       const REAL* auxevol_host, REAL* y_n_host, const REAL dt, const REAL log10_tol,
                       const int max_steps, const REAL integration_radius, int* steps_taken, REAL* final_log10_l2) {
  static griddata_struct g;
  static size_t have = 0;
  const size_t ntot =
      (size_t)params->Nxx_plus_2NGHOSTS0 * params->Nxx_plus_2NGHOSTS1 * params->Nxx_plus_2NGHOSTS2;
  if (have != ntot) {
    if (have) {
      NRPYELL_CUDA(cudaStreamSynchronize(stream()));
      cudaFree(g.gridfuncs.y_n_gfs);
      cudaFree(g.gridfuncs.y_nplus1_running_total_gfs);
      cudaFree(g.gridfuncs.k_odd_gfs);
      cudaFree(g.gridfuncs.k_even_gfs);
      cudaFree(g.gridfuncs.auxevol_gfs);
    }
    void* p[5];
    for (int i = 0; i < 5; i++) NRPYELL_CUDA(cudaMalloc(&p[i], sizeof(REAL) * (i == 4 ? 3 : 2) * ntot));
    g.gridfuncs.y_n_gfs = (REAL*)p[0];
    g.gridfuncs.y_nplus1_running_total_gfs = (REAL*)p[1];
    g.gridfuncs.k_odd_gfs = (REAL*)p[2];
    g.gridfuncs.k_even_gfs = (REAL*)p[3];
    g.gridfuncs.auxevol_gfs = (REAL*)p[4];
    g.gridfuncs.diagnostic_output_gfs = g.gridfuncs.y_nplus1_running_total_gfs;
    have = ntot;
  }
  g.params = *params;
  for (int i = 0; i < 3; i++) g.xx[i] = xx[i];
  g.bcstruct = *bcstruct;
  g.rfmstruct = *rfmstruct;
  NRPYELL_CUDA(cudaMemcpyAsync(g.gridfuncs.auxevol_gfs, auxevol_host, sizeof(REAL) * 3 * ntot,
                               cudaMemcpyHostToDevice, stream()));
  NRPYELL_CUDA(cudaMemcpyAsync(g.gridfuncs.y_n_gfs, y_n_host, sizeof(REAL) * 2 * ntot, cudaMemcpyHostToDevice,
                               stream()));
  const int rc = nrpyell_relax(&g, dt, log10_tol, max_steps, integration_radius, steps_taken, final_log10_l2, nullptr);
  NRPYELL_CUDA(cudaMemcpyAsync(y_n_host, g.gridfuncs.y_n_gfs, sizeof(REAL) * 2 * ntot, cudaMemcpyDeviceToHost,
                               stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  if (!status_ok()) return -1;
  return rc;
}

}  // extern "C"
