// Shared definitions for the CUDA sources of libnrpyell_gpu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <utility>

#include "nrpyell_gpu.h"

namespace nrpyell {

// Error handling: record the first failure, optionally exit(1) like the
// reference does on set-up errors.
void report_error(const char* file, int line, const char* what);
bool status_ok();
cudaStream_t stream();
// The library's stream if it has been created, else the default stream (0);
// never creates one.
cudaStream_t existing_stream();
// Second stream of the library, created on first use: work that may overlap
// a kernel of stream() (forked from and joined back into stream()).
cudaStream_t side_stream();
void count_launch(int n = 1);
long long launch_count();
void set_launch_count(long long n);

// Every device (and managed) allocation of the library goes through these,
// so a caller can check through nrpyell_device_alloc_count that a call
// allocated nothing.
void count_alloc();
template <typename T>
inline cudaError_t dev_alloc(T** p, size_t bytes) {
  count_alloc();
  return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}
template <typename T>
inline cudaError_t managed_alloc(T** p, size_t bytes) {
  count_alloc();
  return cudaMallocManaged(reinterpret_cast<void**>(p), bytes);
}

#define NRPYELL_CUDA(call)                                                     \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      char b_[512];                                                            \
      snprintf(b_, sizeof(b_), "%s: %s", #call, cudaGetErrorString(e_));       \
      ::nrpyell::report_error(__FILE__, __LINE__, b_);                         \
    }                                                                          \
  } while (0)

#define NRPYELL_FAIL(msg) ::nrpyell::report_error(__FILE__, __LINE__, (msg))

// Launch bookkeeping: every kernel launch of the library goes through this,
// so the process can report how many of its own kernels ran.
#define NRPYELL_LAUNCH(kernel, grid, block, smem, ...)                         \
  do {                                                                         \
    kernel<<<(grid), (block), (smem), ::nrpyell::stream()>>>(__VA_ARGS__);     \
    ::nrpyell::count_launch();                                                 \
    NRPYELL_CUDA(cudaGetLastError());                                          \
  } while (0)
#define NRPYELL_LAUNCH_ON(strm, kernel, grid, block, smem, ...)                \
  do {                                                                         \
    kernel<<<(grid), (block), (smem), (strm)>>>(__VA_ARGS__);                  \
    ::nrpyell::count_launch();                                                 \
    NRPYELL_CUDA(cudaGetLastError());                                          \
  } while (0)

// Programmatic dependent launch of the fused substep kernels (on unless
// nrpyell_set_programmatic_launch(0)): a kernel launched this way may be
// scheduled while the previous kernel of the stream drains, and waits in
// griddepcontrol.wait (pdl_enter) before it touches that kernel's results.
bool pdl_enabled();

template <typename... KArgs, typename... Args>
inline cudaError_t launch_maybe_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                    Args&&... args) {
  if (!pdl_enabled()) {
    kern<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}
#define NRPYELL_LAUNCH_PDL(kernel, grid, block, smem, ...)                                                     \
  do {                                                                                                         \
    NRPYELL_CUDA(::nrpyell::launch_maybe_pdl(kernel, dim3(grid), dim3(block), (smem), ::nrpyell::stream(),     \
                                             __VA_ARGS__));                                                    \
    ::nrpyell::count_launch();                                                                                 \
  } while (0)

// Grid geometry passed by value to kernels.
struct Dims {
  int N0, N1, N2;        // Nxx_plus_2NGHOSTS{0,1,2}
  int Nxx0, Nxx1, Nxx2;  // interior sizes
  long long Ntot;        // N0*N1*N2
};

inline Dims dims_of(const paramstruct* p) {
  Dims d;
  d.N0 = p->Nxx_plus_2NGHOSTS0;
  d.N1 = p->Nxx_plus_2NGHOSTS1;
  d.N2 = p->Nxx_plus_2NGHOSTS2;
  d.Nxx0 = p->Nxx0;
  d.Nxx1 = p->Nxx1;
  d.Nxx2 = p->Nxx2;
  d.Ntot = (long long)d.N0 * d.N1 * d.N2;
  return d;
}

// Checks that ptr can be dereferenced by the GPU (device, managed or mapped
// host memory).  Returns false and records an error otherwise.
bool check_device_pointer(const void* ptr, const char* what);

}  // namespace nrpyell
