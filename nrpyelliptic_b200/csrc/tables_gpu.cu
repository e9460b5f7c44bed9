// The device tables of one grid built on the GPU from its parameters and
// coordinates alone, with no host bc_struct or rfm_struct: the set-up of
// batches of many configurations (the reference builds both on the host:
// rfm_precompute_rfmstruct_define.c:5-93, bcstruct_set_up.c:350-521).
//
//   * reference-metric arrays and the folded RHS weights: the closed forms of
//     the host restatement (symtp_rfm_xx0, symtp_rfm_f2, symtp_fold_rhs_coefs
//     in sinhsymtp.h), one thread per xx0, xx1 or (xx0, xx1) point;
//   * inner-boundary map: every ghost point except the x0max face maps to
//     its SymTP image (symtp_ghost_source, the index form of the reference's
//     Cartesian round trip), parity +1 for the scalar gridfunctions, listed
//     in increasing destination index as bcstruct_set_up lists them.  The
//     position of a point in that list has a closed form -- all N0 N1 points
//     of a ghost i2 plane, all N0 points of a ghost i1 row and the first
//     NGHOSTS points of an interior row are inner points -- so each thread
//     writes its own entry without a scan;
//   * pure outer points: the x0max face only (the x0min, x1 and x2 faces of
//     SinhSymTP map inward), layer by layer, i1 fastest, with the upwind
//     offsets and radial geometry of the radiation BC;
//   * the radiation column geometry [3][6][N1].
// The tables equal the host build's: the integer maps entry by entry, the
// floating-point arrays to rounding (device exp/sin/pow against the host's).
#include <math.h>
#include <string.h>

#include <vector>

#include "sinhsymtp.h"
#include "tables.cuh"

namespace nrpyell {

namespace {

struct SetupArgs {
  Dims d;
  double AMAX, SINHWAA, bScale;
  double ix0, ix1, ix2;
};

__global__ void k_rfm_1d(SetupArgs a, RfmTables t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double* xx0 = t.xx01;
  const double* xx1 = t.xx01 + a.d.N0;
  if (i < a.d.N0) {
    double o[7];
    symtp_rfm_xx0(a.AMAX, a.SINHWAA, a.bScale, xx0[i], o);
    t.f0[i] = o[0];
    t.f0_D0[i] = o[1];
    t.f0_DD00[i] = o[2];
    t.f3[i] = o[4];
    t.f3_D0[i] = o[5];
  }
  if (i < a.d.N1) {
    t.f1[i] = sin(xx1[i]);
    t.f1_D1[i] = cos(xx1[i]);
  }
}

// f2 and the folded weights at (i0, i1); the 1-D arrays come from k_rfm_1d.
__global__ void k_rfm_2d(SetupArgs a, RfmTables t) {
  const int n01 = a.d.N0 * a.d.N1;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n01) return;
  const int i0 = k % a.d.N0, i1 = k / a.d.N0;
  double o[5];
  symtp_rfm_f2(a.AMAX, a.SINHWAA, a.bScale, t.xx01[i0], t.xx01[a.d.N0 + i1], o);
  t.f2[k] = o[0];
  t.f2_D0[k] = o[1];
  double cs[kNumCoef];
  symtp_fold_rhs_coefs(t.f0[i0], t.f0_D0[i0], t.f0_DD00[i0], t.f1[i1], t.f1_D1[i1], o[0], o[1], t.f3[i0],
                       t.f3_D0[i0], a.ix0, a.ix1, a.ix2, cs);
  for (int c = 0; c < kNumCoef; c++) {
    t.coef[c * n01 + k] = cs[c];
    t.coef32[c * n01 + k] = (float)cs[c];
  }
}

// Position of ghost point (i0, i1, i2) in the increasing-index list of inner
// points, or -1 for interior and pure outer points.
__device__ long long inner_slot(const Dims& d, int i0, int i1, int i2) {
  const int G = NGHOSTS;
  const long long n01 = (long long)d.N0 * d.N1;
  const long long plane_int = 2LL * G * d.N0 + (long long)G * d.Nxx1;  // inner points of an interior i2 plane
  if (i2 < G) return i2 * n01 + i0 + (long long)d.N0 * i1;
  if (i2 >= G + d.Nxx2) return G * n01 + (long long)d.Nxx2 * plane_int + (i2 - G - d.Nxx2) * n01 + i0 + (long long)d.N0 * i1;
  const long long base = G * n01 + (long long)(i2 - G) * plane_int;
  if (i1 < G) return base + (long long)i1 * d.N0 + i0;
  if (i1 >= G + d.Nxx1) return base + (long long)G * d.N0 + (long long)G * d.Nxx1 + (long long)(i1 - G - d.Nxx1) * d.N0 + i0;
  if (i0 < G) return base + (long long)G * d.N0 + (long long)(i1 - G) * G + i0;
  return -1;  // interior, or the x0max face (pure outer)
}

__global__ void k_bc_inner(Dims d, int2* __restrict__ inner, signed char* __restrict__ par) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= d.Ntot) return;
  const int i0 = (int)(idx % d.N0);
  const long long q = idx / d.N0;
  const int i1 = (int)(q % d.N1), i2 = (int)(q / d.N1);
  const long long s = inner_slot(d, i0, i1, i2);
  if (s < 0) return;
  int m[3];
  symtp_ghost_source(i0, i1, i2, d.Nxx1, d.Nxx2, m);
  inner[s] = make_int2((int)idx, m[0] + d.N0 * (m[1] + d.N1 * m[2]));
  par[s] = 1;
}

// Pure outer points, layer gz = 0..4 (i0 = N0 - NGHOSTS + gz), i1 fastest,
// face (-1, 0, 0): the interior neighbour is i0 - 1.
__global__ void k_bc_outer(SetupArgs a, const double* __restrict__ xx01, OuterPoint* __restrict__ outer) {
  const Dims& d = a.d;
  const long long per = (long long)d.Nxx1 * d.Nxx2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NGHOSTS * per) return;
  const int gz = (int)(t / per);
  const long long r = t - gz * per;
  const int i1 = NGHOSTS + (int)(r % d.Nxx1), i2 = NGHOSTS + (int)(r / d.Nxx1);
  const int i0 = d.N0 - NGHOSTS + gz;
  OuterPoint q;
  q.i0 = (short)i0;
  q.i1 = (short)i1;
  q.i2 = (short)i2;
  q.i0n = (short)(i0 - 1);
  q.i1n = (short)i1;
  q.i2n = (short)i2;
  q.idx3 = i0 + d.N0 * (i1 + d.N1 * i2);
  q.idx3_int = (i0 - 1) + d.N0 * (i1 + d.N1 * i2);
  q.off0 = (signed char)radiation_upwind_offset(-1, i0, d.N0);
  q.off1 = (signed char)radiation_upwind_offset(0, i1, d.N1);
  q.off0n = (signed char)radiation_upwind_offset(-1, i0 - 1, d.N0);
  q.off1n = (signed char)radiation_upwind_offset(0, i1, d.N1);
  const double* xx0 = xx01;
  const double* xx1 = xx01 + d.N0;
  symtp_radial_geometry(a.AMAX, a.SINHWAA, a.bScale, xx0[i0], xx1[i1], &q.r, &q.dx0dr, &q.dx1dr);
  symtp_radial_geometry(a.AMAX, a.SINHWAA, a.bScale, xx0[i0 - 1], xx1[i1], &q.rn, &q.dx0drn, &q.dx1drn);
  outer[t] = q;
}

// Column geometry: j = 0 is i0 = N0-NGHOSTS-1, j = 1..5 the outer layers.
__global__ void k_bc_colgeo(SetupArgs a, const double* __restrict__ xx01, double* __restrict__ colgeo) {
  const int N1 = a.d.N1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 6 * N1) return;
  const int j = t / N1, i1 = t % N1;
  double r, x0r, x1r;
  symtp_radial_geometry(a.AMAX, a.SINHWAA, a.bScale, xx01[a.d.N0 - NGHOSTS - 1 + j], xx01[a.d.N0 + i1], &r, &x0r, &x1r);
  colgeo[(0 * 6 + j) * N1 + i1] = r;
  colgeo[(1 * 6 + j) * N1 + i1] = x0r;
  colgeo[(2 * 6 + j) * N1 + i1] = x1r;
}

unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

}  // namespace nrpyell

using namespace nrpyell;

extern "C" int nrpyell_setup_tables_device(const paramstruct* p, REAL* xx[3], const rfm_struct* rfm,
                                           const bc_struct* bc) {
  if (!p || !xx || !xx[0] || !xx[1] || !rfm || !bc) {
    NRPYELL_FAIL("nrpyell_setup_tables_device: need params, xx[0], xx[1], rfm and bc");
    return -1;
  }
  const Dims d = dims_of(p);
  if (d.N0 != d.Nxx0 + 2 * NGHOSTS || d.N1 != d.Nxx1 + 2 * NGHOSTS || d.N2 != d.Nxx2 + 2 * NGHOSTS ||
      d.Nxx2 % 2 != 0 || d.Nxx2 < NGHOSTS || d.Nxx0 < 12 || d.Nxx1 < 1 || d.Ntot >= (1LL << 31) ||
      d.N0 > 32767 || d.N1 > 32767 || d.N2 > 32767) {
    NRPYELL_FAIL("nrpyell_setup_tables_device: needs Nxx_plus_2NGHOSTSi = Nxxi + 2 NGHOSTS, an even Nxx2 >= NGHOSTS, "
                 "Nxx0 >= 12 and fewer than 2^31 points");
    return -1;
  }
  SetupArgs a;
  a.d = d;
  a.AMAX = p->AMAX;
  a.SINHWAA = p->SINHWAA;
  a.bScale = p->bScale;
  a.ix0 = p->invdx0;
  a.ix1 = p->invdx1;
  a.ix2 = p->invdx2;
  // reference-metric tables (shared by every grid with these parameters)
  RfmTables* rt = find_rfm_tables(p, rfm);
  RfmTables* rt_new = nullptr;
  if (!rt) {
    rt_new = new_rfm_tables(p, rfm);
    if (!rt_new) return -1;
    NRPYELL_CUDA(cudaMemcpyAsync(rt_new->xx01, xx[0], sizeof(double) * d.N0, cudaMemcpyHostToDevice, stream()));
    NRPYELL_CUDA(cudaMemcpyAsync(rt_new->xx01 + d.N0, xx[1], sizeof(double) * d.N1, cudaMemcpyHostToDevice, stream()));
    NRPYELL_LAUNCH(k_rfm_1d, blocks(d.N0 > d.N1 ? d.N0 : d.N1, 128), 128, 0, a, *rt_new);
    NRPYELL_LAUNCH(k_rfm_2d, blocks((long long)d.N0 * d.N1, 128), 128, 0, a, *rt_new);
    rt = rt_new;
  }
  // boundary tables
  if (!find_bc_tables(p, bc, xx)) {
    const long long n_outer = (long long)NGHOSTS * d.Nxx1 * d.Nxx2;
    const long long n_inner = d.Ntot - (long long)d.Nxx0 * d.Nxx1 * d.Nxx2 - n_outer;
    BcTables* t = new BcTables();
    memset(t->outer_off, 0, sizeof(t->outer_off));
    bc_tables_set_key(t, p, bc, xx);
    if (!bc_tables_layout(t, (size_t)n_inner, (size_t)n_outer)) {
      delete t;
      return -1;
    }
    t->n_inner = (int)n_inner;
    t->n_outer = (int)n_outer;
    t->max_layer = (int)(n_outer / NGHOSTS);
    for (int gz = 0; gz <= NGHOSTS; gz++)
      for (int dirn = 0; dirn < 3; dirn++)
        if (dirn + 3 * gz <= NGHOSTS * 3) t->outer_off[dirn + 3 * gz] = (int)((gz + (dirn > 0)) * (n_outer / NGHOSTS));
    t->outer_off[NGHOSTS * 3] = (int)n_outer;
    t->columns_ok = true;
    t->analytic_ok = true;
    NRPYELL_CUDA(cudaMemcpyAsync(t->xx01, xx[0], sizeof(double) * d.N0, cudaMemcpyHostToDevice, stream()));
    NRPYELL_CUDA(cudaMemcpyAsync(t->xx01 + d.N0, xx[1], sizeof(double) * d.N1, cudaMemcpyHostToDevice, stream()));
    NRPYELL_LAUNCH(k_bc_inner, blocks(d.Ntot, 256), 256, 0, d, t->inner, t->inner_par);
    NRPYELL_LAUNCH(k_bc_outer, blocks(n_outer, 128), 128, 0, a, t->xx01, t->outer);
    NRPYELL_LAUNCH(k_bc_colgeo, blocks(6 * d.N1, 128), 128, 0, a, t->xx01, t->colgeo);
    NRPYELL_CUDA(cudaStreamSynchronize(stream()));
    if (!status_ok()) return -1;
    register_bc_tables(t);
  }
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  if (!status_ok()) return -1;
  if (rt_new) register_rfm_tables(rt_new);
  return 0;
}

extern "C" long long nrpyell_device_tables_read(const paramstruct* p, REAL* xx[3], const rfm_struct* rfm,
                                                const bc_struct* bc, const int what, void* host_out,
                                                const long long capacity) {
  if (!p || !rfm || !bc || !host_out || capacity < 0) {
    NRPYELL_FAIL("nrpyell_device_tables_read: need params, rfm, bc and host_out");
    return -1;
  }
  const Dims d = dims_of(p);
  const long long n0 = d.N0, n1 = d.N1, n01 = n0 * n1;
  auto copy = [&](const void* src, long long n, size_t elem) -> long long {
    if (n > capacity) {
      NRPYELL_FAIL("nrpyell_device_tables_read: host_out too small");
      return -1;
    }
    NRPYELL_CUDA(cudaStreamSynchronize(stream()));
    NRPYELL_CUDA(cudaMemcpy(host_out, src, (size_t)n * elem, cudaMemcpyDeviceToHost));
    return status_ok() ? n : -1;
  };
  if (what >= 5) {
    RfmTables* rt = get_rfm_tables(p, rfm);
    if (!rt) return -1;
    const double* arr[9] = {rt->f0, rt->f0_D0, rt->f0_DD00, rt->f3, rt->f3_D0, rt->f1, rt->f1_D1, rt->f2, rt->f2_D0};
    const long long len[9] = {n0, n0, n0, n0, n0, n1, n1, n01, n01};
    if (what <= 13) return copy(arr[what - 5], len[what - 5], sizeof(double));
    if (what == 14) return copy(rt->coef, kNumCoef * n01, sizeof(double));
    NRPYELL_FAIL("nrpyell_device_tables_read: unknown table");
    return -1;
  }
  BcTables* bt = get_bc_tables(p, bc, xx);
  if (!bt) return -1;
  switch (what) {
    case 0: return copy(bt->inner, 2LL * bt->n_inner, sizeof(int));
    case 1: return copy(bt->inner_par, bt->n_inner, 1);
    case 2:
    case 3: {
      const long long per = what == 2 ? 8 : 6;
      if ((long long)bt->n_outer * per > capacity) {
        NRPYELL_FAIL("nrpyell_device_tables_read: host_out too small");
        return -1;
      }
      std::vector<OuterPoint> o(bt->n_outer > 0 ? bt->n_outer : 1);
      NRPYELL_CUDA(cudaStreamSynchronize(stream()));
      if (bt->n_outer) NRPYELL_CUDA(cudaMemcpy(o.data(), bt->outer, sizeof(OuterPoint) * bt->n_outer, cudaMemcpyDeviceToHost));
      if (!status_ok()) return -1;
      for (int list = 0; list < NGHOSTS * 3; list++)
        for (int k = bt->outer_off[list]; k < bt->outer_off[list + 1]; k++) {
          const OuterPoint& q = o[k];
          if (what == 2) {
            int* r = (int*)host_out + 8 * (long long)k;
            r[0] = list / 3; r[1] = list % 3; r[2] = q.i0; r[3] = q.i1; r[4] = q.i2;
            r[5] = q.i0n - q.i0; r[6] = q.i1n - q.i1; r[7] = q.i2n - q.i2;
          } else {
            double* r = (double*)host_out + 6 * (long long)k;
            r[0] = q.r; r[1] = q.dx0dr; r[2] = q.dx1dr; r[3] = q.rn; r[4] = q.dx0drn; r[5] = q.dx1drn;
          }
        }
      return (long long)bt->n_outer * per;
    }
    case 4: return copy(bt->colgeo, 18 * n1, sizeof(double));
  }
  NRPYELL_FAIL("nrpyell_device_tables_read: unknown table");
  return -1;
}
