// extern "C" entry points of libnrpyell_gpu: the reference prototypes of the
// hot path (NRPy_function_prototypes.h) plus the library extensions declared
// in include/nrpyell_gpu.h.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "driver.cuh"

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

static cudaStream_t g_side_stream = nullptr;
cudaStream_t side_stream() {
  if (!g_side_stream) {
    cudaError_t e = cudaStreamCreateWithFlags(&g_side_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      g_side_stream = nullptr;
      report_error(__FILE__, __LINE__, cudaGetErrorString(e));
    }
  }
  return g_side_stream;
}

void count_launch(int n) { g_launches += n; }
long long launch_count() { return g_launches; }
void set_launch_count(long long n) { g_launches = n; }
static long long g_allocs = 0;
void count_alloc() { g_allocs++; }

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

static RelaxParams relax_params(const paramstruct* p, double dt) {
  RelaxParams rp;
  memset(&rp, 0, sizeof(rp));  // graph keys compare the bytes
  rp.dt = dt;
  rp.eta = p->eta_damping;
  rp.cOB[0] = p->uu_wavespeed_at_OB;
  rp.cOB[1] = p->vv_wavespeed_at_OB;
  rp.log10_tol = -1e300;
  return rp;
}

static void mol_step_fused(griddata_struct* g, double dt) {
  RfmTables* rt;
  BcTables* bt;
  if (!fused_ready(&g->params, &g->rfmstruct, &g->bcstruct, g->xx, &rt, &bt)) {
    mol_step_reference_order(g, dt);
    return;
  }
  const Dims d = dims_of(&g->params);
  FusedWork* w = get_work(d, 16);
  Scratch* sc = get_scratch(max_interior_blocks(d));
  const StateBuffers b = buffers_of(&g->gridfuncs);
  const RelaxParams rp = relax_params(&g->params, dt);
  const int tile = tuned_tile<double>(d, rt, bt, w, sc, b, rp);
  for (int s = 1; s <= 4; s++)
    launch_substep<double>(s, substep_args(d, rt, bt, sc, b, rp, s, w->zero_flag, w->state, tile));
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

// The reference's functions return when their work is done, and callers such
// as main.c read managed gridfunctions on the host right after a call; the
// Part-1 entry points therefore wait for their kernels unless the caller
// opted into asynchronous calls.
static void finish_call() {
  if (!g_async) NRPYELL_CUDA(cudaStreamSynchronize(stream()));
}

// Common preparation of the fused relaxation drivers.
struct RelaxSetup {
  Dims d;
  RfmTables* rt;
  BcTables* bt;
  L2Tables* lt;
  FusedWork* w;
  Scratch* s;
};

// Copy kernel of nrpyell_copy_bandwidth: 16-byte loads and stores, grid-stride.
// `passes` sweeps over the same buffers in one launch, so that a footprint
// that fits in L2 is measured without the launch latency.
__global__ void k_copy_bw(const double2* __restrict__ a, double2* __restrict__ b, long long n, int passes) {
  for (int p = 0; p < passes; p++)
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      b[i] = a[i];
}

// Longest FP32 stretch of nrpyell_relax_mixed between two folds.
constexpr int kMaxFoldEvery = 4096;

static int relax_prepare(griddata_struct* g, int max_steps, double R, RelaxSetup* out, const char* who) {
  char msg[256];
  if (max_steps < 0) {
    snprintf(msg, sizeof(msg), "%s: max_steps < 0", who);
    NRPYELL_FAIL(msg);
    return -1;
  }
  if (!check_gridfuncs(&g->gridfuncs)) return -1;
  if (!fused_ready(&g->params, &g->rfmstruct, &g->bcstruct, g->xx, &out->rt, &out->bt)) {
    snprintf(msg, sizeof(msg),
             "%s needs radiation outer BCs with the SymTP inner-boundary map and x0max-only pure outer points", who);
    NRPYELL_FAIL(msg);
    return -2;
  }
  out->lt = get_l2_tables(&g->params, g->xx, R);
  if (!out->lt) return -1;
  out->d = dims_of(&g->params);
  out->w = get_work(out->d, max_steps + 1);
  out->s = get_scratch(max_interior_blocks(out->d));
  return status_ok() ? 0 : -1;
}

}  // namespace nrpyell

using namespace nrpyell;

extern "C" {

int nrpyell_last_status(void) { return g_status; }
int nrpyell_gpu_last_status(void) { return g_status; }
const char* nrpyell_last_error(void) { return g_error.c_str(); }
void nrpyell_clear_status(void) {
  g_status = 0;
  g_error.clear();
}
void nrpyell_set_exit_on_error(int enable) { g_exit_on_error = enable != 0; }
long long nrpyell_launch_count(void) { return g_launches; }
long long nrpyell_device_alloc_count(void) { return g_allocs; }

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
int nrpyell_get_step_mode(void) { return g_step_mode; }
void nrpyell_set_async(int enable) { g_async = enable != 0; }

void nrpyell_set_tile(int tile) { g_forced_tile = (tile >= 0 && tile < substep_num_tiles()) ? tile : -1; }

void nrpyell_set_programmatic_launch(int on) {
  if (g_pdl == (on != 0)) return;
  if (g_stream) NRPYELL_CUDA(cudaStreamSynchronize(g_stream));
  release_graphs();  // cached relaxation graphs were captured with the other setting
  g_pdl = on != 0;
}
int nrpyell_get_programmatic_launch(void) { return g_pdl ? 1 : 0; }

int nrpyell_get_tile(const paramstruct* params, int fp32, int* bx, int* by, int* planes) {
  int tile = g_forced_tile >= 0 ? g_forced_tile : find_tile(dims_of(params), fp32);
  if (tile >= 0 && bx && by && planes) substep_tile_shape(tile, bx, by, planes);
  return tile;
}

int nrpyell_num_tiles(void) { return substep_num_tiles(); }

int nrpyell_tile_info(int tile, int* by, int* planes, int* kind) {
  if (tile < 0 || tile >= substep_num_tiles()) return -1;
  int bx = 0, b = 0, p = 0;
  substep_tile_shape(tile, &bx, &b, &p);
  if (by) *by = b;
  if (planes) *planes = p;
  if (kind) *kind = substep_tile_kind(tile);
  return 0;
}

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

double nrpyell_copy_bandwidth(size_t bytes, int iters) {
  const long long n = (long long)(bytes / 2 / sizeof(double2));
  if (n < 1 || iters < 1) {
    NRPYELL_FAIL("nrpyell_copy_bandwidth: need bytes >= 32 and iters >= 1");
    return -1.0;
  }
  double2 *a = nullptr, *b = nullptr;
  NRPYELL_CUDA(dev_alloc(&a, sizeof(double2) * n));
  NRPYELL_CUDA(dev_alloc(&b, sizeof(double2) * n));
  cudaEvent_t e0, e1;
  NRPYELL_CUDA(cudaEventCreate(&e0));
  NRPYELL_CUDA(cudaEventCreate(&e1));
  if (!status_ok()) return -1.0;
  NRPYELL_CUDA(cudaMemsetAsync(a, 0, sizeof(double2) * n, stream()));
  int sms = 148;
  int dev = 0;
  NRPYELL_CUDA(cudaGetDevice(&dev));
  NRPYELL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, (long long)sms * 8);
  const int passes = (int)std::max<long long>(1, (1ll << 30) / (long long)(2 * sizeof(double2) * n));
  float best = 1e30f;
  for (int it = 0; it <= iters; it++) {  // the first launch is a warm-up
    NRPYELL_CUDA(cudaEventRecord(e0, stream()));
    NRPYELL_LAUNCH(k_copy_bw, grid, 256, 0, a, b, n, passes);
    NRPYELL_CUDA(cudaEventRecord(e1, stream()));
    NRPYELL_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    NRPYELL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (it > 0) best = std::min(best, ms);
  }
  NRPYELL_CUDA(cudaEventDestroy(e0));
  NRPYELL_CUDA(cudaEventDestroy(e1));
  NRPYELL_CUDA(cudaFree(a));
  NRPYELL_CUDA(cudaFree(b));
  if (!status_ok()) return -1.0;
  return 2.0 * sizeof(double2) * n * passes / (best * 1e-3) / 1e9;
}

void nrpyell_flush_l2(void) {
  static void* buf = nullptr;
  const size_t bytes = (size_t)256 << 20;
  if (!buf) NRPYELL_CUDA(dev_alloc(&buf, bytes));
  NRPYELL_CUDA(cudaMemsetAsync(buf, 0x5a, bytes, stream()));
}

int nrpyell_time_fused(griddata_struct* g, const REAL dt, const int stage, const int n_iter, double* ms_interior,
                       double* ms_step) {
  if (!check_gridfuncs(&g->gridfuncs)) return -1;
  RfmTables* rt;
  BcTables* bt;
  if (!fused_ready(&g->params, &g->rfmstruct, &g->bcstruct, g->xx, &rt, &bt) || stage < 1 || stage > 4 ||
      n_iter < 1) {
    NRPYELL_FAIL("nrpyell_time_fused: fused path unavailable for this grid or bad arguments");
    return -2;
  }
  const Dims d = dims_of(&g->params);
  FusedWork* w = get_work(d, 16);
  Scratch* sc = get_scratch(max_interior_blocks(d));
  const StateBuffers b = buffers_of(&g->gridfuncs);
  const RelaxParams rp = relax_params(&g->params, dt);
  const int tile = tuned_tile<double>(d, rt, bt, w, sc, b, rp);
  prepare_substep<double>(tile);
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
        launch_substep<double>(stage, substep_args(d, rt, bt, sc, b, rp, stage, w->zero_flag, w->state, tile));
      } else {
        for (int s = 1; s <= 4; s++)
          launch_substep<double>(s, substep_args(d, rt, bt, sc, b, rp, s, w->zero_flag, w->state, tile));
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
  release_batch();
  release_all_tables();
}

void* nrpyell_device_malloc(size_t bytes) {
  void* p = nullptr;
  NRPYELL_CUDA(dev_alloc(&p, bytes));
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
  NRPYELL_CUDA(managed_alloc(&p, sizeof(REAL) * NUM_EVOL_GFS * n));
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
  NRPYELL_CUDA(managed_alloc(&p[0], sizeof(REAL) * NUM_EVOL_GFS * n));
  NRPYELL_CUDA(managed_alloc(&p[1], sizeof(REAL) * NUM_EVOL_GFS * n));
  NRPYELL_CUDA(managed_alloc(&p[2], sizeof(REAL) * NUM_EVOL_GFS * n));
  NRPYELL_CUDA(managed_alloc(&p[3], sizeof(REAL) * NUM_AUXEVOL_GFS * n));
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
                                        REAL* NRPYELL_RESTRICT xx[3], const REAL custom_wavespeed[NUM_EVOL_GFS],
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
                   REAL* NRPYELL_RESTRICT xx[3], const REAL* in_gf) {
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

// ---- relaxation drivers ----
int nrpyell_relax(griddata_struct* g, const REAL dt, const REAL log10_tol, const int max_steps,
                  const REAL integration_radius, int* steps_taken, REAL* final_log10_l2, REAL* history) {
  RelaxSetup su;
  const int rc = relax_prepare(g, max_steps, integration_radius, &su, "nrpyell_relax");
  if (rc) return rc;
  const StateBuffers b = buffers_of(&g->gridfuncs);
  RelaxParams rp = relax_params(&g->params, dt);
  rp.log10_tol = log10_tol;
  rp.max_steps = max_steps;
  const int tile = tuned_tile<double>(su.d, su.rt, su.bt, su.w, su.s, b, rp, su.lt);
  const RelaxResult r = relax_loop<double>(su.d, su.rt, su.bt, su.lt, su.w, su.s, tile, b, rp);
  // ghost zones of the solution, as the reference's all-points update leaves them
  launch_ghost_fill<double>(su.d, su.bt, g->gridfuncs.y_n_gfs);
  if (history)
    NRPYELL_CUDA(cudaMemcpyAsync(history, su.w->history, sizeof(double) * (r.steps + 1), cudaMemcpyDeviceToHost,
                                 stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  if (!status_ok()) return -1;
  if (steps_taken) *steps_taken = r.steps;
  if (final_log10_l2) *final_log10_l2 = r.last_log10_l2;
  return r.converged ? 0 : 1;
}

int nrpyell_relax_et(griddata_struct* g, const REAL dt, const REAL log_target_residual, const int max_iterations,
                     const int check_every, const REAL integration_radius, int* iterations, REAL* final_log10_l2) {
  if (check_every < 1 || max_iterations < 0) {
    NRPYELL_FAIL("nrpyell_relax_et: need check_every >= 1 and max_iterations >= 0");
    return -1;
  }
  RelaxSetup su;
  // the thorn's loop takes up to max_iterations + 1 steps and tests after each
  const int rc = relax_prepare(g, max_iterations + 1, integration_radius, &su, "nrpyell_relax_et");
  if (rc) return rc;
  const StateBuffers b = buffers_of(&g->gridfuncs);
  RelaxParams rp = relax_params(&g->params, dt);
  rp.log10_tol = log_target_residual;
  rp.max_steps = max_iterations + 1;
  rp.check_every = check_every;
  const int tile = tuned_tile<double>(su.d, su.rt, su.bt, su.w, su.s, b, rp, su.lt);
  const RelaxResult r = relax_loop<double>(su.d, su.rt, su.bt, su.lt, su.w, su.s, tile, b, rp);
  launch_ghost_fill<double>(su.d, su.bt, g->gridfuncs.y_n_gfs);
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  if (!status_ok()) return -1;
  // r.steps RK4 steps were taken before the last residual: the thorn's
  // loop index at that test is r.steps - 1
  if (iterations) *iterations = r.steps - 1;
  if (final_log10_l2) *final_log10_l2 = r.last_log10_l2;
  return r.converged ? 0 : 1;
}

REAL nrpyell_compute_TRC(const REAL A, const REAL b, const REAL C_0, const REAL dt, const REAL dxx1,
                         const REAL dxx2) {
  // Eq. (B6) of arXiv:2111.02424 in this code's coordinate names
  const double c1 = cos(dxx1 / 2.0), c2 = cos(dxx2 / 2.0);
  return dt / (C_0 * dxx1) * atanh(A / sqrt(A * A + b * b * c1 * c1)) * c1 * c2;
}

void nrpyell_set_optimum_eta_damping(const REAL dt, const REAL CFL_FACTOR, paramstruct* params) {
  // Eq. (36) of arXiv:2111.02424: eta = 6.9 TRC^-0.79 - 0.7
  const double trc = nrpyell_compute_TRC(params->AMAX, params->bScale, CFL_FACTOR, dt, params->dxx1, params->dxx2);
  params->eta_damping = 6.9 * pow(trc, -0.79) - 0.7;
}

int nrpyell_relax_mixed(griddata_struct* g, const REAL dt, const REAL log10_tol, const REAL log10_switch,
                        const int fold_every, const int max_steps, const REAL integration_radius, int* steps_fp32,
                        int* steps_fp64, REAL* final_log10_l2, REAL* history) {
  RelaxSetup su;
  const int rc = relax_prepare(g, max_steps, integration_radius, &su, "nrpyell_relax_mixed");
  if (rc) return rc;
  if (fold_every < 1 || fold_every > kMaxFoldEvery) {
    NRPYELL_FAIL("nrpyell_relax_mixed: need 1 <= fold_every <= 4096");
    return -1;
  }
  if (!march_fits(su.d)) {
    NRPYELL_FAIL("nrpyell_relax_mixed: grid too large for the FP32 correction kernels (3 Ntot >= 2^32)");
    return -1;
  }
  const Dims d = su.d;
  const long long n2 = 2 * d.Ntot;
  FusedWork* w = su.w;
  if (!w->f32) NRPYELL_CUDA(dev_alloc(&w->f32, sizeof(float) * (5 * n2 + 3 * d.Ntot)));
  const int cycle_len = std::min(fold_every, max_steps);
  if (!w->cycle_history) NRPYELL_CUDA(dev_alloc(&w->cycle_history, sizeof(double) * (kMaxFoldEvery + 1)));
  if (!status_ok()) return -1;
  // FP32 buffers: the correction and its RK buffers, the pointwise fields,
  // the base state's RHS
  StateBuffers b32;
  b32.y = w->f32;
  b32.acc = w->f32 + n2;
  b32.kodd = w->f32 + 2 * n2;
  b32.keven = w->f32 + 3 * n2;
  b32.aux = w->f32 + 4 * n2;
  b32.R0 = w->f32 + 4 * n2 + 3 * d.Ntot;
  MoL_gridfunctions_struct* gf = &g->gridfuncs;
  double* U = gf->y_n_gfs;
  double* rhs64 = gf->k_odd_gfs;                   // scratch of the FP64 base evaluation
  double* res64 = gf->y_nplus1_running_total_gfs;  // (both are overwritten by every RK4 step)
  const StateBuffers b64 = buffers_of(gf);
  const paramstruct* p = &g->params;
  const double cw[2] = {p->uu_wavespeed_at_OB, p->vv_wavespeed_at_OB};
  const double finf[2] = {0.0, 0.0};

  RelaxParams rp = relax_params(p, dt);
  rp.log10_tol = log10_switch;
  rp.history_buf = w->cycle_history;
  int n = 0, tile32 = -1;
  bool converged = false, to_fp64 = false;
  double l2 = NAN;
  for (;;) {
    // FP64 evaluation of the base state: its ghost zones, RHS with the
    // radiation BC, residual and L2 norm (the stop test), then the FP32
    // inputs of the correction kernels.
    launch_ghost_fill<double>(d, su.bt, U);
    launch_rhs_ref(d, p, su.rt, gf->auxevol_gfs, U, rhs64);
    launch_radiation_bc(d, p, su.bt, cw, finf, U, rhs64);
    launch_residual_ref(d, su.rt, gf->auxevol_gfs, U, res64);
    launch_l2_sum(d, su.lt, res64, su.s);
    launch_correction_base(d, U, gf->auxevol_gfs, rhs64, res64, (float*)b32.R0, (float*)b32.aux);
    double sum = 0.0;
    NRPYELL_CUDA(cudaMemcpyAsync(&sum, su.s->result, sizeof(double), cudaMemcpyDeviceToHost, stream()));
    NRPYELL_CUDA(cudaStreamSynchronize(stream()));
    if (!status_ok()) return -1;
    l2 = log10(1e-16 + sqrt(sum / su.lt->volume));
    NRPYELL_CUDA(cudaMemcpy(w->history + n, &l2, sizeof(double), cudaMemcpyHostToDevice));
    if (l2 <= log10_tol) {
      converged = true;
      break;
    }
    if (l2 <= log10_switch || to_fp64 || n >= max_steps) break;
    // One FP32 stretch: the correction relaxes from zero for up to
    // fold_every steps, or until its FP32-evaluated residual reaches
    // log10_switch, and is folded into U.
    NRPYELL_CUDA(cudaMemsetAsync(b32.y, 0, sizeof(float) * n2, stream()));
    rp.max_steps = std::min(cycle_len, max_steps - n);
    if (tile32 < 0) tile32 = tuned_tile<float>(d, su.rt, su.bt, w, su.s, b32, rp, su.lt);
    const RelaxResult r = relax_loop<float>(d, su.rt, su.bt, su.lt, w, su.s, tile32, b32, rp);
    if (!status_ok()) return -1;
    launch_correction_fold(U, (const float*)b32.y, n2);
    if (r.steps > 0)
      NRPYELL_CUDA(cudaMemcpyAsync(w->history + n + 1, w->cycle_history + 1, sizeof(double) * r.steps,
                                   cudaMemcpyDeviceToDevice, stream()));
    n += r.steps;
    // the FP32 evaluation met the switch tolerance (the FP64 one decides at
    // the top of the loop) or made no progress: the FP64 phase takes over
    if (r.converged || r.steps == 0) to_fp64 = true;
  }
  const int n32 = n;
  int n64 = 0;
  if (!converged && n < max_steps && status_ok()) {
    RelaxParams rp64 = relax_params(p, dt);
    rp64.log10_tol = log10_tol;
    rp64.max_steps = max_steps - n;
    rp64.history_offset = n;
    const int tile64 = tuned_tile<double>(d, su.rt, su.bt, w, su.s, b64, rp64, su.lt);
    const RelaxResult r64 = relax_loop<double>(d, su.rt, su.bt, su.lt, w, su.s, tile64, b64, rp64);
    n64 = r64.steps;
    converged = r64.converged;
    l2 = r64.last_log10_l2;
  }
  launch_ghost_fill<double>(d, su.bt, U);
  if (history)
    NRPYELL_CUDA(cudaMemcpyAsync(history, w->history, sizeof(double) * (n32 + n64 + 1), cudaMemcpyDeviceToHost,
                                 stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  if (!status_ok()) return -1;
  if (steps_fp32) *steps_fp32 = n32;
  if (steps_fp64) *steps_fp64 = n64;
  if (final_log10_l2) *final_log10_l2 = l2;
  return converged ? 0 : 1;
}

int nrpyell_relax_host(const paramstruct* params, REAL* xx[3], const bc_struct* bcstruct, const rfm_struct* rfmstruct,
                       const REAL* auxevol_host, REAL* y_n_host, const REAL dt, const REAL log10_tol,
                       const int max_steps, const REAL integration_radius, int* steps_taken, REAL* final_log10_l2) {
  static griddata_struct g;
  static size_t have = 0;
  const size_t ntot = (size_t)params->Nxx_plus_2NGHOSTS0 * params->Nxx_plus_2NGHOSTS1 * params->Nxx_plus_2NGHOSTS2;
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
    for (int i = 0; i < 5; i++) NRPYELL_CUDA(dev_alloc(&p[i], sizeof(REAL) * (i == 4 ? 3 : 2) * ntot));
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
