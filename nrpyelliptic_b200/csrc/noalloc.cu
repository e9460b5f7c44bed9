// L2_norm_of_gf_noalloc: the residual L2 norm without any device allocation.
//
// Who needs it.  L2_norm_of_gf builds cached device tables (volume weights)
// and reduction scratch with cudaMalloc the first time it sees a grid.  Some
// callers cannot allow that: frameworks that reserve all device memory for
// their own arena at start-up and forbid later allocations, processes
// running under a hard device-memory quota, and time-critical loops in which
// the implicit device-wide synchronisation of cudaMalloc/cudaFree is not
// acceptable.  For them this entry point computes the same quantity with all
// of its working memory in one fixed, file-scope __device__ array.
//
// Limits and rules.
//   * Grids up to kNoallocMaxN0 x kNoallocMaxN1 points (ghosts included) in
//     the xx0 and xx1 directions; larger grids are rejected with an error and
//     NaN, before any GPU work.  The i2 direction is unlimited.
//   * The array occupies 37.5 KB on every GPU that loads the library, until
//     the process exits.
//   * All calls share the array.  It keeps the last call's contents; the
//     reduction ticket, the only field that must start at zero, is cleared at
//     the start of every call.  Calls that overlap on the GPU (other threads
//     or streams) race on the array and must be serialised by the caller.
//   * The first call on each device looks up the array's device address with
//     cudaGetSymbolAddress while that device is current.  With lazy module
//     loading (CUDA's default) that lookup also loads the library's GPU code,
//     and the driver makes its own allocations for code and globals then:
//     callers with a strict budget make the first call at start-up or run
//     with CUDA_MODULE_LOADING=EAGER.
//   * Every call copies xx0/xx1 from pageable host memory and waits for the
//     result, so no call may be made while the stream it runs on (below) is
//     being captured.
//   * It runs on the library's stream when that stream belongs to the
//     current device (ordering with earlier library calls), otherwise on the
//     legacy default stream of the current device.
//   * No cudaMalloc, cudaFree or other allocating routine is called.  The
//     volume element is evaluated per point on the GPU (as L2_norm_of_gf.c
//     does on the CPU) instead of coming from a cached weight table.
#include <math.h>

#include "common.cuh"

namespace nrpyell {

namespace {
constexpr int kNoallocMaxN0 = 2048;
constexpr int kNoallocMaxN1 = 2048;
constexpr int kNoallocBlocks = 296;  // 2 x 148 SMs
constexpr int kNoallocThreads = 256;
// Layout of the array, in doubles.
constexpr int kOffXX0 = 0;
constexpr int kOffXX1 = kOffXX0 + kNoallocMaxN0;
constexpr int kOffSq = kOffXX1 + kNoallocMaxN1;
constexpr int kOffVol = kOffSq + kNoallocBlocks;
constexpr int kOffRes = kOffVol + kNoallocBlocks;
constexpr int kOffTicket = kOffRes + 2;
constexpr int kScratchDoubles = kOffTicket + 2;
constexpr int kMaxDevices = 64;
}  // namespace

static __device__ __align__(256) double g_l2_noalloc_scratch[kScratchDoubles];

// Device address of g_l2_noalloc_scratch per device (host-side copies of what
// cudaGetSymbolAddress returned; the symbol itself is only a host stand-in).
static double* g_noalloc_addr[kMaxDevices];

__device__ __forceinline__ double noalloc_block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) r += sh[w];
  __syncthreads();
  return r;
}

// Sum of g^2 dV and of dV over interior points with r < R, with dV the
// SinhSymTP volume element of L2_norm_of_gf.c:19-32 times dxx0 dxx1 dxx2.
// Fixed per-block point sets and an index-ordered final sum by the last block
// make the result independent of scheduling.
__global__ void __launch_bounds__(kNoallocThreads)
    k_l2_noalloc(Dims d, double AMAX, double SINHWAA, double bScale, double dV0, double R, const double* __restrict__ g,
                 double* scratch) {
  __shared__ double sh[kNoallocThreads / 32];
  __shared__ bool last;
  const double* xx0 = scratch + kOffXX0;
  const double* xx1 = scratch + kOffXX1;
  const double iw = 1.0 / SINHWAA;
  const double D = exp(iw) - exp(-iw);
  const long long n = (long long)d.Nxx0 * d.Nxx1 * d.Nxx2;
  double sq = 0.0, vol = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(t % d.Nxx0) + NGHOSTS;
    const long long q = t / d.Nxx0;
    const int i1 = (int)(q % d.Nxx1) + NGHOSTS;
    const int i2 = (int)(q / d.Nxx1) + NGHOSTS;
    const double x0 = xx0[i0], x1 = xx1[i1];
    const double s = sin(x1), c = cos(x1);
    const double ep = exp(iw * x0), em = exp(-iw * x0);
    const double E2 = (ep - em) * (ep - em);
    const double A2 = AMAX * AMAX * E2 / (D * D);
    const double B2 = bScale * bScale + A2;
    const double r = sqrt(s * s * A2 + B2 * (c * c));
    if (r < R) {
      const double qq = bScale * bScale * (s * s) + A2;
      const double sdg =
          AMAX * AMAX * sqrt(E2 * (qq * qq) * ((iw * ep + iw * em) * (iw * ep + iw * em)) / (B2 * (D * D * D * D))) * fabs(s);
      const double dV = sdg * dV0;
      const double gv = g[i0 + (long long)d.N0 * (i1 + (long long)d.N1 * i2)];
      sq += gv * gv * dV;
      vol += dV;
    }
  }
  const double bs = noalloc_block_sum(sq, sh);
  const double bv = noalloc_block_sum(vol, sh);
  unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + kOffTicket);
  if (threadIdx.x == 0) {
    scratch[kOffSq + blockIdx.x] = bs;
    scratch[kOffVol + blockIdx.x] = bv;
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
    a += ((volatile double*)scratch)[kOffSq + i];
    b += ((volatile double*)scratch)[kOffVol + i];
  }
  const double ta = noalloc_block_sum(a, sh);
  const double tb = noalloc_block_sum(b, sh);
  if (threadIdx.x == 0) {
    scratch[kOffRes] = ta;
    scratch[kOffRes + 1] = tb;
    *ticket = 0u;
  }
}

}  // namespace nrpyell

using namespace nrpyell;

extern "C" REAL L2_norm_of_gf_noalloc(const paramstruct* params, const int gf_index, const REAL integration_radius,
                                      REAL* NRPYELL_RESTRICT xx[3], const REAL* in_gf) {
  const Dims d = dims_of(params);
  if (d.N0 != d.Nxx0 + 2 * NGHOSTS || d.N1 != d.Nxx1 + 2 * NGHOSTS || d.N2 != d.Nxx2 + 2 * NGHOSTS || d.Nxx0 < 1 ||
      d.Nxx1 < 1 || d.Nxx2 < 1) {
    NRPYELL_FAIL("L2_norm_of_gf_noalloc: Nxx_plus_2NGHOSTSi must equal Nxxi + 2 NGHOSTS with Nxxi >= 1");
    return NAN;
  }
  if (d.N0 > kNoallocMaxN0 || d.N1 > kNoallocMaxN1) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "L2_norm_of_gf_noalloc: grid %d x %d (xx0 x xx1, ghosts included) exceeds the fixed maximum %d x %d",
             d.N0, d.N1, kNoallocMaxN0, kNoallocMaxN1);
    NRPYELL_FAIL(msg);
    return NAN;
  }
  if (gf_index < 0 || gf_index >= NUM_EVOL_GFS) {
    NRPYELL_FAIL("L2_norm_of_gf_noalloc: gf_index out of range");
    return NAN;
  }
  if (!check_device_pointer(in_gf, "in_gf")) return NAN;
  int dev = 0;
  NRPYELL_CUDA(cudaGetDevice(&dev));
  if (!status_ok()) return NAN;
  if (dev < 0 || dev >= kMaxDevices) {
    NRPYELL_FAIL("L2_norm_of_gf_noalloc: device index beyond the supported range");
    return NAN;
  }
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_l2_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      char msg[200];
      snprintf(msg, sizeof(msg), "L2_norm_of_gf_noalloc: cudaGetSymbolAddress failed (%s)", cudaGetErrorString(e));
      NRPYELL_FAIL(msg);
      return NAN;
    }
    g_noalloc_addr[dev] = (double*)p;
  }
  double* s = g_noalloc_addr[dev];
  // The library's stream if it exists and belongs to this device (ordering
  // with earlier library calls), otherwise the default stream; no stream is
  // created here.
  cudaStream_t st = existing_stream();
  if (st) {
    int sdev = -1;
    if (cudaStreamGetDevice(st, &sdev) != cudaSuccess || sdev != dev) st = 0;
  }
  NRPYELL_CUDA(cudaMemcpyAsync(s + kOffXX0, xx[0], sizeof(double) * d.N0, cudaMemcpyHostToDevice, st));
  NRPYELL_CUDA(cudaMemcpyAsync(s + kOffXX1, xx[1], sizeof(double) * d.N1, cudaMemcpyHostToDevice, st));
  NRPYELL_CUDA(cudaMemsetAsync(s + kOffTicket, 0, sizeof(double), st));
  k_l2_noalloc<<<kNoallocBlocks, kNoallocThreads, 0, st>>>(d, params->AMAX, params->SINHWAA, params->bScale,
                                                           params->dxx0 * params->dxx1 * params->dxx2,
                                                           integration_radius, in_gf + (long long)gf_index * d.Ntot, s);
  count_launch();
  NRPYELL_CUDA(cudaGetLastError());
  double res[2] = {0.0, 0.0};
  NRPYELL_CUDA(cudaMemcpyAsync(res, s + kOffRes, sizeof(res), cudaMemcpyDeviceToHost, st));
  NRPYELL_CUDA(cudaStreamSynchronize(st));
  if (!status_ok()) return NAN;
  return log10(1e-16 + sqrt(res[0] / res[1]));
}
