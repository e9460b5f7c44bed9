// Set-up on the GPU for batches of configurations: the auxevol
// gridfunctions (psi_background and ADD_times_AUU at all points, as
// auxevol_gfs_all_points.c:6-100, and the wavespeed on the interior, as
// wavespeed_gf_all_points.c:6-45) written straight into device memory, one
// thread per point, from the same closed forms (sinhsymtp.h) the host
// restatement in setup.cpp uses.  A batch of configurations then needs no
// host-side auxevol arrays and no host-to-device copy of them.
#include "common.cuh"
#include "sinhsymtp.h"

namespace nrpyell {

namespace {

struct AuxArgs {
  int N0, N1, N2;
  long long Ntot;
  double AMAX, SINHWAA, bScale, dxx0, dxx1, dxx2;
  double m0, m1;
  ByPuncture b0, b1;
  double CFL, dt;
};

__global__ void k_auxevol(AuxArgs a, const double* __restrict__ xx0, const double* __restrict__ xx1,
                          const double* __restrict__ xx2, double* aux) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.Ntot) return;
  const int i0 = (int)(idx % a.N0), i1 = (int)((idx / a.N0) % a.N1), i2 = (int)(idx / ((long long)a.N0 * a.N1));
  double X[3];
  symtp_xx_to_cart(a.AMAX, a.SINHWAA, a.bScale, xx0[i0], xx1[i1], xx2[i2], X);
  aux[PSI_BACKGROUNDGF * a.Ntot + idx] = bl_psi(a.m0, a.b0.pos, a.m1, a.b1.pos, X);
  aux[ADD_TIMES_AUUGF * a.Ntot + idx] = by_AA(a.b0, a.b1, X);
  double ws = 0.0;  // ghost zones: zero (the reference leaves them unset and never reads them)
  if (i0 >= NGHOSTS && i0 < a.N0 - NGHOSTS && i1 >= NGHOSTS && i1 < a.N1 - NGHOSTS && i2 >= NGHOSTS &&
      i2 < a.N2 - NGHOSTS) {
    double ds[3];
    symtp_ds(a.AMAX, a.SINHWAA, a.bScale, a.dxx0, a.dxx1, a.dxx2, xx0[i0], xx1[i1], ds);
    ws = a.CFL * fmin(ds[0], fmin(ds[1], ds[2])) / a.dt;
  }
  aux[WAVESPEEDGF * a.Ntot + idx] = ws;
}

// Device copy of the coordinate arrays, grown as needed.
double* g_xx_dev = nullptr;
size_t g_xx_cap = 0;

}  // namespace

}  // namespace nrpyell

using namespace nrpyell;

extern "C" int nrpyell_auxevol_device(const paramstruct* p, REAL* xx[3], const REAL CFL_FACTOR, const REAL dt,
                                      REAL* auxevol_gfs) {
  if (!p || !xx || !xx[0] || !xx[1] || !xx[2] || !(dt > 0)) {
    NRPYELL_FAIL("nrpyell_auxevol_device: need params, xx and dt > 0");
    return -1;
  }
  if (!check_device_pointer(auxevol_gfs, "auxevol_gfs")) return -1;
  AuxArgs a;
  a.N0 = p->Nxx_plus_2NGHOSTS0;
  a.N1 = p->Nxx_plus_2NGHOSTS1;
  a.N2 = p->Nxx_plus_2NGHOSTS2;
  a.Ntot = (long long)a.N0 * a.N1 * a.N2;
  a.AMAX = p->AMAX;
  a.SINHWAA = p->SINHWAA;
  a.bScale = p->bScale;
  a.dxx0 = p->dxx0;
  a.dxx1 = p->dxx1;
  a.dxx2 = p->dxx2;
  a.m0 = p->bare_mass_0;
  a.m1 = p->bare_mass_1;
  a.b0 = {{p->puncture_0_x, p->puncture_0_y, p->puncture_0_z}, {p->P0_x, p->P0_y, p->P0_z}, {p->S0_x, p->S0_y, p->S0_z}};
  a.b1 = {{p->puncture_1_x, p->puncture_1_y, p->puncture_1_z}, {p->P1_x, p->P1_y, p->P1_z}, {p->S1_x, p->S1_y, p->S1_z}};
  a.CFL = CFL_FACTOR;
  a.dt = dt;
  const size_t nxx = (size_t)a.N0 + a.N1 + a.N2;
  if (nxx > g_xx_cap) {
    NRPYELL_CUDA(cudaStreamSynchronize(stream()));
    cudaFree(g_xx_dev);
    g_xx_dev = nullptr;
    NRPYELL_CUDA(dev_alloc(&g_xx_dev, sizeof(double) * nxx));
    g_xx_cap = status_ok() ? nxx : 0;
  }
  if (!status_ok()) return -1;
  NRPYELL_CUDA(cudaMemcpyAsync(g_xx_dev, xx[0], sizeof(double) * a.N0, cudaMemcpyHostToDevice, stream()));
  NRPYELL_CUDA(cudaMemcpyAsync(g_xx_dev + a.N0, xx[1], sizeof(double) * a.N1, cudaMemcpyHostToDevice, stream()));
  NRPYELL_CUDA(
      cudaMemcpyAsync(g_xx_dev + a.N0 + a.N1, xx[2], sizeof(double) * a.N2, cudaMemcpyHostToDevice, stream()));
  NRPYELL_LAUNCH(k_auxevol, (unsigned)((a.Ntot + 255) / 256), 256, 0, a, g_xx_dev, g_xx_dev + a.N0,
                 g_xx_dev + a.N0 + a.N1, auxevol_gfs);
  // the coordinate copies read host memory of the caller: finish before returning
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return status_ok() ? 0 : -1;
}
