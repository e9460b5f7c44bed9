// Solution export without Cactus: uu interpolated to arbitrary Cartesian
// points and the ADM quantities of the conformally flat data assembled there
// -- the roles of the Einstein Toolkit thorn's
// NRPyEllipticET_conformally_flat_BBH_Initialize_ADMBase.c (points mapped to
// SinhSymTP coordinates, Lagrange polynomial interpolation of the requested
// order on the uniform (xx0,xx1,xx2) grid including its ghost zones, default
// order 4) and conformally_flat_BBH_compute_ADM_Cartesian_quantities_from_uu.c
// (psi = psi_background + uu, gamma_ij = psi^4 delta_ij, beta = 0,
// K_ij = psi^-2 Abar_ij).
//
// Cartesian -> SinhSymTP: with rho^2 = x^2 + y^2, R^2 = rho^2 + z^2 and b =
// bScale, the SymTP radius A solves rho^2/A^2 + z^2/(A^2 + b^2) = 1, so
//   A^2 = (R^2 - b^2 + sqrt((R^2 - b^2)^2 + 4 b^2 rho^2)) / 2,
//   xx0 = SINHWAA asinh(A sinh(1/SINHWAA) / AMAX),
//   xx1 = acos(z / sqrt(A^2 + b^2)),  xx2 = atan2(y, x).
// Lagrange molecule of order n (n+1 points per direction): for even n
// centred on the nearest grid point, for odd n starting n/2 points below the
// point's cell; shifted to stay inside the array.
#include <string.h>

#include "common.cuh"
#include "sinhsymtp.h"

namespace nrpyell {

namespace {

constexpr int kMaxOrder = 8;

struct ExportArgs {
  int N[3];
  long long Ntot;
  double x0[3], dx[3];  // first grid coordinate and spacing per direction
  double AMAX, SINHWAA, bScale;
  double m0, m1;
  ByPuncture b0, b1;
  int order;
};

__device__ void cart_to_symtp(const ExportArgs& a, const double X[3], double xx[3]) {
  const double b2 = a.bScale * a.bScale;
  const double rho2 = X[0] * X[0] + X[1] * X[1];
  const double R2 = rho2 + X[2] * X[2];
  const double q = R2 - b2;
  const double A2 = 0.5 * (q + sqrt(q * q + 4.0 * b2 * rho2));
  const double iw = 1.0 / a.SINHWAA;
  xx[0] = a.SINHWAA * asinh(sqrt(A2) * sinh(iw) / a.AMAX);
  const double c = X[2] / sqrt(A2 + b2);
  xx[1] = acos(fmin(1.0, fmax(-1.0, c)));
  xx[2] = atan2(X[1], X[0]);
}

// First molecule index and weights along one direction.
__device__ int lagrange_1d(const ExportArgs& a, int d, double x, double* w) {
  const int n = a.order;
  const double t = (x - a.x0[d]) / a.dx[d];
  int s = (n % 2 == 0) ? (int)floor(t + 0.5) - n / 2 : (int)floor(t) - (n - 1) / 2;
  if (s < 0) s = 0;
  if (s > a.N[d] - (n + 1)) s = a.N[d] - (n + 1);
  for (int j = 0; j <= n; j++) {
    double l = 1.0;
    for (int m = 0; m <= n; m++)
      if (m != j) l *= (t - (double)(s + m)) / (double)(j - m);
    w[j] = l;
  }
  return s;
}

__global__ void k_export(ExportArgs a, int npts, const double* __restrict__ xyz, const double* __restrict__ uu,
                         double* out_uu, double* out_psi, double* out_gamma, double* out_K) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const double X[3] = {xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2]};
  double xx[3];
  cart_to_symtp(a, X, xx);
  double w0[kMaxOrder + 1], w1[kMaxOrder + 1], w2[kMaxOrder + 1];
  const int s0 = lagrange_1d(a, 0, xx[0], w0);
  const int s1 = lagrange_1d(a, 1, xx[1], w1);
  const int s2 = lagrange_1d(a, 2, xx[2], w2);
  double u = 0.0;
  for (int k = 0; k <= a.order; k++) {
    double uk = 0.0;
    for (int j = 0; j <= a.order; j++) {
      const double* row = uu + (long long)a.N[0] * ((s1 + j) + (long long)a.N[1] * (s2 + k)) + s0;
      double uj = 0.0;
      for (int i = 0; i <= a.order; i++) uj += w0[i] * row[i];
      uk += w1[j] * uj;
    }
    u += w2[k] * uk;
  }
  if (out_uu) out_uu[p] = u;
  const double psi = bl_psi(a.m0, a.b0.pos, a.m1, a.b1.pos, X) + u;
  if (out_psi) out_psi[p] = psi;
  if (out_gamma) {
    const double g = psi * psi * psi * psi;
    const double v[6] = {g, 0.0, 0.0, g, 0.0, g};  // xx, xy, xz, yy, yz, zz
    for (int c = 0; c < 6; c++) out_gamma[6 * p + c] = v[c];
  }
  if (out_K) {
    double dV[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    by_dV_accumulate(a.b0, X, dV);
    by_dV_accumulate(a.b1, X, dV);
    const double div = dV[0][0] + dV[1][1] + dV[2][2];
    const double ip2 = 1.0 / (psi * psi);
    const int I[6] = {0, 0, 0, 1, 1, 2}, J[6] = {0, 1, 2, 1, 2, 2};
    for (int c = 0; c < 6; c++) {
      double abar = dV[I[c]][J[c]] + dV[J[c]][I[c]];
      if (I[c] == J[c]) abar -= (2.0 / 3.0) * div;
      out_K[6 * p + c] = ip2 * abar;
    }
  }
}

// Initial lapse at points (the thorn's two options,
// conformally_flat_BBH_compute_ADM_Cartesian_quantities_from_uu.c:25-29):
//   mode 0 "NRPyEllipticET-psi^n" (conformally_flat_BBH_lapse_power_of_psi_initial_data.c):
//          alpha = (psi_BL + uu)^n, psi_BL = 1 + m0/(2 r0) + m1/(2 r1);
//   mode 1 "NRPyEllipticET-averaged" (conformally_flat_BBH_lapse_averaged_initial_data.c):
//          alpha = 1/2 (1 - s)/(1 + s) + 1/2, s = m0/(2 r0) + m1/(2 r1)
//          (uu does not enter).
__global__ void k_lapse(ExportArgs a, int npts, const double* __restrict__ xyz, const double* __restrict__ uu,
                        int mode, double n, double* __restrict__ alpha) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const double X = xyz[3 * p], Y = xyz[3 * p + 1], Z = xyz[3 * p + 2];
  const double d0x = X - a.b0.pos[0], d0y = Y - a.b0.pos[1], d0z = Z - a.b0.pos[2];
  const double d1x = X - a.b1.pos[0], d1y = Y - a.b1.pos[1], d1z = Z - a.b1.pos[2];
  const double s = 0.5 * a.m0 / sqrt(d0x * d0x + d0y * d0y + d0z * d0z) +
                   0.5 * a.m1 / sqrt(d1x * d1x + d1y * d1y + d1z * d1z);
  alpha[p] = mode == 0 ? pow(1.0 + s + uu[p], n) : 0.5 * (1.0 - s) / (1.0 + s) + 0.5;
}

}  // namespace

}  // namespace nrpyell

using namespace nrpyell;

extern "C" int nrpyell_initial_lapse(const paramstruct* p, const int npts, const REAL* xyz, const REAL* uu_at_points,
                                     const int mode, const REAL lapse_exponent, REAL* alpha_out) {
  if (!p || npts < 0 || (npts > 0 && (!xyz || !alpha_out)) || (mode != NRPYELL_LAPSE_PSI_POWER &&
                                                                mode != NRPYELL_LAPSE_AVERAGED) ||
      (mode == NRPYELL_LAPSE_PSI_POWER && npts > 0 && !uu_at_points)) {
    NRPYELL_FAIL("nrpyell_initial_lapse: need params, xyz, alpha_out, a known mode and uu_at_points for psi^n");
    return -1;
  }
  if (npts == 0) return 0;
  ExportArgs a;
  memset(&a, 0, sizeof(a));
  a.m0 = p->bare_mass_0;
  a.m1 = p->bare_mass_1;
  a.b0.pos[0] = p->puncture_0_x;
  a.b0.pos[1] = p->puncture_0_y;
  a.b0.pos[2] = p->puncture_0_z;
  a.b1.pos[0] = p->puncture_1_x;
  a.b1.pos[1] = p->puncture_1_y;
  a.b1.pos[2] = p->puncture_1_z;
  const size_t n = (size_t)npts;
  double* buf = nullptr;
  NRPYELL_CUDA(dev_alloc(&buf, sizeof(double) * n * 5));
  if (!status_ok()) return -1;
  double *d_xyz = buf, *d_uu = buf + 3 * n, *d_alpha = buf + 4 * n;
  NRPYELL_CUDA(cudaMemcpyAsync(d_xyz, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, stream()));
  if (mode == NRPYELL_LAPSE_PSI_POWER)
    NRPYELL_CUDA(cudaMemcpyAsync(d_uu, uu_at_points, sizeof(double) * n, cudaMemcpyHostToDevice, stream()));
  NRPYELL_LAUNCH(k_lapse, (unsigned)((n + 127) / 128), 128, 0, a, npts, d_xyz, d_uu, mode, lapse_exponent, d_alpha);
  NRPYELL_CUDA(cudaMemcpyAsync(alpha_out, d_alpha, sizeof(double) * n, cudaMemcpyDeviceToHost, stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  cudaFree(buf);
  return status_ok() ? 0 : -1;
}

extern "C" int nrpyell_interpolate_solution(const paramstruct* p, REAL* xx[3], const REAL* uu, const int npts,
                                            const REAL* xyz, const int order, REAL* uu_out, REAL* psi_out,
                                            REAL* gamma_out, REAL* K_out) {
  if (!p || !xx || !uu || !xyz || npts < 0 || order < 1 || order > kMaxOrder) {
    NRPYELL_FAIL("nrpyell_interpolate_solution: need params, xx, uu, xyz, npts >= 0 and 1 <= order <= 8");
    return -1;
  }
  if (!check_device_pointer(uu, "uu")) return -1;
  ExportArgs a;
  a.N[0] = p->Nxx_plus_2NGHOSTS0;
  a.N[1] = p->Nxx_plus_2NGHOSTS1;
  a.N[2] = p->Nxx_plus_2NGHOSTS2;
  for (int d = 0; d < 3; d++) {
    if (a.N[d] < order + 1) {
      NRPYELL_FAIL("nrpyell_interpolate_solution: grid smaller than the interpolation molecule");
      return -1;
    }
    a.x0[d] = xx[d][0];
    a.dx[d] = xx[d][1] - xx[d][0];
  }
  a.Ntot = (long long)a.N[0] * a.N[1] * a.N[2];
  a.AMAX = p->AMAX;
  a.SINHWAA = p->SINHWAA;
  a.bScale = p->bScale;
  a.m0 = p->bare_mass_0;
  a.m1 = p->bare_mass_1;
  a.b0 = {{p->puncture_0_x, p->puncture_0_y, p->puncture_0_z}, {p->P0_x, p->P0_y, p->P0_z}, {p->S0_x, p->S0_y, p->S0_z}};
  a.b1 = {{p->puncture_1_x, p->puncture_1_y, p->puncture_1_z}, {p->P1_x, p->P1_y, p->P1_z}, {p->S1_x, p->S1_y, p->S1_z}};
  a.order = order;
  if (npts == 0) return 0;
  // one device block: points in, the four outputs (1 + 1 + 6 + 6 per point)
  double* buf = nullptr;
  const size_t n = (size_t)npts;
  NRPYELL_CUDA(dev_alloc(&buf, sizeof(double) * n * 17));
  if (!status_ok()) return -1;
  double *d_xyz = buf, *d_uu = buf + 3 * n, *d_psi = buf + 4 * n, *d_g = buf + 5 * n, *d_K = buf + 11 * n;
  NRPYELL_CUDA(cudaMemcpyAsync(d_xyz, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, stream()));
  NRPYELL_LAUNCH(k_export, (unsigned)((n + 127) / 128), 128, 0, a, npts, d_xyz, uu, d_uu, d_psi, d_g, d_K);
  if (uu_out) NRPYELL_CUDA(cudaMemcpyAsync(uu_out, d_uu, sizeof(double) * n, cudaMemcpyDeviceToHost, stream()));
  if (psi_out) NRPYELL_CUDA(cudaMemcpyAsync(psi_out, d_psi, sizeof(double) * n, cudaMemcpyDeviceToHost, stream()));
  if (gamma_out)
    NRPYELL_CUDA(cudaMemcpyAsync(gamma_out, d_g, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, stream()));
  if (K_out) NRPYELL_CUDA(cudaMemcpyAsync(K_out, d_K, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  cudaFree(buf);
  return status_ok() ? 0 : -1;
}
