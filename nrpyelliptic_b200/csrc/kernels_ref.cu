// Reference-order kernels: the same arithmetic, in the same order, as the
// reference's generated C for rhs_eval, residual_all_points, the boundary
// conditions and the RK4 linear combinations.  Products, sums, quotients and
// fused multiply-adds are spelled with the IEEE round-to-nearest intrinsics
// so the compiler can neither contract nor reorder them; with the AVX-512 /
// AVX2+FMA build of the reference (whose SIMD macros fix every FMA,
// SIMD/SIMD_intrinsics.h:18-21,52-55) rhs_eval and residual_all_points then
// agree bit for bit.
#include "fd_weights.h"
#include "kernels.cuh"

namespace nrpyell {

#define MUL(a, b) __dmul_rn((a), (b))
#define ADD(a, b) __dadd_rn((a), (b))
#define SUB(a, b) __dsub_rn((a), (b))
#define DIV(a, b) __ddiv_rn((a), (b))
#define FMA(a, b, c) __fma_rn((a), (b), (c))
#define FMS(a, b, c) __fma_rn((a), (b), -(c))   // a*b - c, one rounding
#define NFMA(a, b, c) __fma_rn(-(a), (b), (c))  // c - a*b, one rounding

__constant__ double c_fd1_upwind[11][11] = NRPYELL_FD1_UPWIND_INIT;

struct StencilU {
  double c, m[6], p[6], jm[6], jp[6], km[6], kp[6];  // i0-, i0+, i1-, i1+, i2-, i2+ (index 1..5)
};

__device__ __forceinline__ void load_star(const double* __restrict__ u, long long idx, int s1, long long s2,
                                          StencilU& st) {
  st.c = __ldg(u + idx);
#pragma unroll
  for (int k = 1; k <= 5; k++) {
    st.m[k] = __ldg(u + idx - k);
    st.p[k] = __ldg(u + idx + k);
    st.jm[k] = __ldg(u + idx - (long long)k * s1);
    st.jp[k] = __ldg(u + idx + (long long)k * s1);
    st.km[k] = __ldg(u + idx - (long long)k * s2);
    st.kp[k] = __ldg(u + idx + (long long)k * s2);
  }
}

// 10th-order first derivative, rhs_eval.c:87 operation order (times invdx).
__device__ __forceinline__ double d1_ref(const double* m, const double* p, double invdx) {
  return MUL(invdx,
             FMA(5.0 / 504.0, SUB(m[4], p[4]),
                 FMA(5.0 / 6.0, SUB(p[1], m[1]),
                     FMA(5.0 / 84.0, SUB(p[3], m[3]),
                         FMA(1.0 / 1260.0, SUB(p[5], m[5]), MUL(5.0 / 21.0, SUB(m[2], p[2])))))));
}

// 10th-order second derivative, rhs_eval.c:89 operation order.
__device__ __forceinline__ double d2_ref(const double* m, const double* p, double centre_term, double invdx) {
  return MUL(MUL(invdx, invdx),
             FMA(5.0 / 126.0, ADD(m[3], p[3]),
                 FMA(5.0 / 3.0, ADD(m[1], p[1]),
                     FMS(1.0 / 3150.0, ADD(m[5], p[5]),
                         FMA(5.0 / 1008.0, ADD(m[4], p[4]), FMA(5.0 / 21.0, ADD(m[2], p[2]), centre_term))))));
}

// The bracket of the vv right-hand side (equivalently the residual),
// rhs_eval.c:106-110 / residual_all_points.c:103-106.
__device__ __forceinline__ double bracket_ref(const StencilU& st, double invdx0, double invdx1, double invdx2,
                                              double f0, double f0_D0, double f0_DD00, double f1, double f1_D1,
                                              double f2, double f2_D0, double f3, double f3_D0, double psi,
                                              double AA) {
  const double FDPart1_0 = MUL(5269.0 / 1800.0, st.c);
  const double uu_dD0 = d1_ref(st.m, st.p, invdx0);
  const double uu_dD1 = d1_ref(st.jm, st.jp, invdx1);
  const double uu_dDD00 = d2_ref(st.m, st.p, FDPart1_0, invdx0);
  const double uu_dDD11 = d2_ref(st.jm, st.jp, FDPart1_0, invdx1);
  const double uu_dDD22 = d2_ref(st.km, st.kp, FDPart1_0, invdx2);
  const double P0 = DIV(1.0, MUL(f2, f2));
  const double P2 = DIV(MUL(f3, f3), MUL(f0_D0, f0_D0));
  const double P3 = DIV(1.0, MUL(MUL(f2, f2), f2));
  const double pu = ADD(psi, st.c);
  const double pow7 = MUL(MUL(MUL(MUL(MUL(MUL(pu, pu), pu), pu), pu), pu), pu);
  const double ta = DIV(MUL(MUL(P0, -1.0), DIV(MUL(f3, f3), f0_D0)), f0);
  const double tb = FMS(P2, MUL(P3, f2_D0), ta);
  const double tc = DIV(FMS(f3, FMA(f0_D0, f2_D0, MUL(f0_DD00, f2)), MUL(f0_D0, MUL(f2, f3_D0))),
                        MUL(MUL(f0_D0, f0_D0), f0_D0));
  const double td = FMS(MUL(P3, f3), tc, tb);
  const double te = FMS(P0, uu_dDD11, MUL(uu_dD0, td));
  const double tf = FMA(MUL(P0, f1_D1), DIV(uu_dD1, f1), te);
  const double tg = FMA(1.0 / 8.0, DIV(AA, pow7), tf);
  const double th = FMA(P0, MUL(P2, uu_dDD00), tg);
  return FMA(uu_dDD22, DIV(DIV(1.0, MUL(f1, f1)), MUL(f0, f0)), th);
}

struct RefArgs {
  Dims d;
  const double *f0, *f0_D0, *f0_DD00, *f1, *f1_D1, *f2, *f2_D0, *f3, *f3_D0;
  double invdx0, invdx1, invdx2, eta;
};

__device__ __forceinline__ bool interior_index(const Dims& d, int& i0, int& i1, int& i2) {
  i0 = blockIdx.x * blockDim.x + threadIdx.x + NGHOSTS;
  i1 = blockIdx.y * blockDim.y + threadIdx.y + NGHOSTS;
  i2 = blockIdx.z * blockDim.z + threadIdx.z + NGHOSTS;
  return i0 < NGHOSTS + d.Nxx0 && i1 < NGHOSTS + d.Nxx1 && i2 < NGHOSTS + d.Nxx2;
}

// rhs_eval.c:7-117
__global__ void __launch_bounds__(256) k_rhs_ref(RefArgs a, const double* __restrict__ aux,
                                                 const double* __restrict__ in, double* __restrict__ rhs) {
  int i0, i1, i2;
  if (!interior_index(a.d, i0, i1, i2)) return;
  const int N0 = a.d.N0;
  const long long s2 = (long long)N0 * a.d.N1;
  const long long idx = i0 + (long long)N0 * i1 + s2 * i2;
  const long long Ntot = a.d.Ntot;
  StencilU st;
  load_star(in, idx, N0, s2, st);
  const double vv = __ldg(in + Ntot + idx);
  const double AA = __ldg(aux + ADD_TIMES_AUUGF * Ntot + idx);
  const double psi = __ldg(aux + PSI_BACKGROUNDGF * Ntot + idx);
  const double ws = __ldg(aux + WAVESPEEDGF * Ntot + idx);
  const int k2 = i0 + N0 * i1;
  const double b = bracket_ref(st, a.invdx0, a.invdx1, a.invdx2, __ldg(a.f0 + i0), __ldg(a.f0_D0 + i0),
                               __ldg(a.f0_DD00 + i0), __ldg(a.f1 + i1), __ldg(a.f1_D1 + i1), __ldg(a.f2 + k2),
                               __ldg(a.f2_D0 + k2), __ldg(a.f3 + i0), __ldg(a.f3_D0 + i0), psi, AA);
  rhs[idx] = NFMA(a.eta, st.c, vv);
  rhs[Ntot + idx] = MUL(MUL(ws, ws), b);
}

// residual_all_points.c:7-112 (writes the UUGF slot of residual_gf)
__global__ void __launch_bounds__(256) k_residual_ref(RefArgs a, const double* __restrict__ aux,
                                                      const double* __restrict__ in, double* __restrict__ res) {
  int i0, i1, i2;
  if (!interior_index(a.d, i0, i1, i2)) return;
  const int N0 = a.d.N0;
  const long long s2 = (long long)N0 * a.d.N1;
  const long long idx = i0 + (long long)N0 * i1 + s2 * i2;
  const long long Ntot = a.d.Ntot;
  StencilU st;
  load_star(in, idx, N0, s2, st);
  const double AA = __ldg(aux + ADD_TIMES_AUUGF * Ntot + idx);
  const double psi = __ldg(aux + PSI_BACKGROUNDGF * Ntot + idx);
  const int k2 = i0 + N0 * i1;
  res[idx] = bracket_ref(st, a.invdx0, a.invdx1, a.invdx2, __ldg(a.f0 + i0), __ldg(a.f0_D0 + i0),
                         __ldg(a.f0_DD00 + i0), __ldg(a.f1 + i1), __ldg(a.f1_D1 + i1), __ldg(a.f2 + k2),
                         __ldg(a.f2_D0 + k2), __ldg(a.f3 + i0), __ldg(a.f3_D0 + i0), psi, AA);
}

static RefArgs ref_args(const Dims& d, const RfmTables* rt, double invdx0, double invdx1, double invdx2, double eta) {
  RefArgs a;
  a.d = d;
  a.f0 = rt->f0; a.f0_D0 = rt->f0_D0; a.f0_DD00 = rt->f0_DD00;
  a.f1 = rt->f1; a.f1_D1 = rt->f1_D1;
  a.f2 = rt->f2; a.f2_D0 = rt->f2_D0;
  a.f3 = rt->f3; a.f3_D0 = rt->f3_D0;
  a.invdx0 = invdx0; a.invdx1 = invdx1; a.invdx2 = invdx2; a.eta = eta;
  return a;
}

static dim3 interior_grid(const Dims& d, dim3 block) {
  return dim3((d.Nxx0 + block.x - 1) / block.x, (d.Nxx1 + block.y - 1) / block.y, (d.Nxx2 + block.z - 1) / block.z);
}

void launch_rhs_ref(const Dims& d, const paramstruct* p, const RfmTables* rt, const double* aux, const double* in,
                    double* rhs) {
  const dim3 block(32, 4, 2);
  RefArgs a = ref_args(d, rt, p->invdx0, p->invdx1, p->invdx2, p->eta_damping);
  NRPYELL_LAUNCH(k_rhs_ref, interior_grid(d, block), block, 0, a, aux, in, rhs);
}

void launch_residual_ref(const Dims& d, const RfmTables* rt, const double* aux, const double* in, double* res) {
  const dim3 block(32, 4, 2);
  RefArgs a = ref_args(d, rt, rt->invdx[0], rt->invdx[1], rt->invdx[2], 0.0);
  NRPYELL_LAUNCH(k_residual_ref, interior_grid(d, block), block, 0, a, aux, in, res);
}

// ---------------------------------------------------------------------------
// Radiation BC (apply_bcs_outerradiation_and_inner.c:325-408) on one list of
// pure outer points; lists run in the reference's (which_gz, dirn) order so a
// layer sees the RHS of the layer inside it.

// Upwind first derivative along x0 or x1 at (i0,i1,i2) with offset off.
// Terms are summed from the lowest node upwards, as written in
// FD1_arbitrary_upwind_x{0,1}_dirn; the zero centre weight of the centred
// stencil is skipped, as there.
__device__ __forceinline__ double fd1_upwind(const double* __restrict__ f, long long idx, long long stride, int off,
                                             double invdx) {
  const double* w = c_fd1_upwind[off + 5];
  double s = 0.0;
  bool first = true;
#pragma unroll
  for (int j = 0; j < 11; j++) {
    if (off == 0 && j == 5) continue;
    const double t = w[j] * __ldg(f + idx + (long long)(off - 5 + j) * stride);
    s = first ? t : s + t;
    first = false;
  }
  return s * invdx;
}

__global__ void k_radiation_layer(Dims d, const OuterPoint* __restrict__ pts, int n, double invdx0, double invdx1,
                                  double c0, double c1, double finf0, double finf1, const double* __restrict__ gfs,
                                  double* __restrict__ rhs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * n) return;
  const int gf = t / n;
  const OuterPoint q = pts[t - gf * n];
  const long long Ntot = d.Ntot;
  const double* f = gfs + gf * Ntot;
  const int N0 = d.N0;
  const double c = gf ? c1 : c0;
  const double finf = gf ? finf1 : finf0;
  const long long idx = q.idx3, idxn = q.idx3_int;
  const double drf = q.dx0dr * fd1_upwind(f, idx, 1, q.off0, invdx0) + q.dx1dr * fd1_upwind(f, idx, N0, q.off1, invdx1);
  const double drfn =
      q.dx0drn * fd1_upwind(f, idxn, 1, q.off0n, invdx0) + q.dx1drn * fd1_upwind(f, idxn, N0, q.off1n, invdx1);
  const double ptf_int = rhs[gf * Ntot + idxn];
  const double fv = __ldg(f + idx);
  const double fn = __ldg(f + idxn);
  const double out_int = -c * (drfn + (fn - finf) / q.rn);
  const double k = q.rn * q.rn * q.rn * (ptf_int - out_int);
  const double rinv = 1.0 / q.r;
  const double out = -c * (drf + (fv - finf) * rinv);
  rhs[gf * Ntot + idx] = out + k * rinv * rinv * rinv;
}

void launch_radiation_bc(const Dims& d, const paramstruct* p, const BcTables* bt, const double c[2],
                         const double finf[2], const double* gfs, double* rhs) {
  for (int list = 0; list < NGHOSTS * 3; list++) {
    const int n = bt->outer_off[list + 1] - bt->outer_off[list];
    if (n <= 0) continue;
    const int threads = 256;
    NRPYELL_LAUNCH(k_radiation_layer, (2 * n + threads - 1) / threads, threads, 0, d, bt->outer + bt->outer_off[list],
                   n, p->invdx0, p->invdx1, c[0], c[1], finf[0], finf[1], gfs, rhs);
  }
}

// apply_bcs_inner_only.c:18-26
__global__ void k_inner_copy(const int2* __restrict__ map, const signed char* __restrict__ par, int n, long long Ntot,
                             int ngfs, double* __restrict__ gfs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int2 m = map[t];
  const double s = (double)par[t];
  for (int gf = 0; gf < ngfs; gf++) gfs[gf * Ntot + m.x] = s * gfs[gf * Ntot + m.y];
}

void launch_inner_copy(const Dims& d, const BcTables* bt, double* gfs, int ngfs) {
  if (bt->n_inner <= 0) return;
  const int threads = 256;
  NRPYELL_LAUNCH(k_inner_copy, (bt->n_inner + threads - 1) / threads, threads, 0, bt->inner, bt->inner_par,
                 bt->n_inner, d.Ntot, ngfs, gfs);
}

// apply_bcs_outerextrap_and_inner.c:33-60: f0 = 3 f1 - 3 f2 + f3 towards the interior.
__global__ void k_extrap_layer(Dims d, const OuterPoint* __restrict__ pts, int n, double* __restrict__ gfs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const OuterPoint q = pts[t];
  const int F0 = q.i0n - q.i0, F1 = q.i1n - q.i1, F2 = q.i2n - q.i2;
  const int N0 = d.N0, N1 = d.N1;
  // the three points towards the interior must lie on the grid
  const int j0 = q.i0 + 3 * F0, j1 = q.i1 + 3 * F1, j2 = q.i2 + 3 * F2;
  if (j0 < 0 || j0 >= N0 || j1 < 0 || j1 >= N1 || j2 < 0 || j2 >= d.N2) return;
  const long long i1d = q.idx3_int;
  const long long i2d = (q.i0 + 2 * F0) + (long long)N0 * ((q.i1 + 2 * F1) + (long long)N1 * (q.i2 + 2 * F2));
  const long long i3d = (q.i0 + 3 * F0) + (long long)N0 * ((q.i1 + 3 * F1) + (long long)N1 * (q.i2 + 3 * F2));
  for (int gf = 0; gf < NUM_EVOL_GFS; gf++) {
    double* g = gfs + gf * d.Ntot;
    g[q.idx3] = +3.0 * g[i1d] - 3.0 * g[i2d] + 1.0 * g[i3d];
  }
}

void launch_extrap_bc(const Dims& d, const BcTables* bt, const bc_struct* bc, double* gfs) {
  (void)bc;
  for (int list = 0; list < NGHOSTS * 3; list++) {
    const int n = bt->outer_off[list + 1] - bt->outer_off[list];
    if (n <= 0) continue;
    NRPYELL_LAUNCH(k_extrap_layer, (n + 255) / 256, 256, 0, d, bt->outer + bt->outer_off[list], n, gfs);
  }
  launch_inner_copy(d, bt, gfs, NUM_EVOL_GFS);
}

// RK4 linear combinations over all points (MoL_step_forward_in_time.c).
template <int STAGE>
__global__ void k_rk_update_ref(long long n, double dt, const double* k, const double* y, double* acc, double* out) {
  // k and out are the same buffer at stages 1-3, y and out at stage 4.
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double dk = MUL(dt, k[i]);
  if (STAGE == 1) {
    acc[i] = MUL(1.0 / 6.0, dk);
    out[i] = FMA(1.0 / 2.0, dk, y[i]);
  } else if (STAGE == 2) {
    acc[i] = FMA(1.0 / 3.0, dk, acc[i]);
    out[i] = FMA(1.0 / 2.0, dk, y[i]);
  } else if (STAGE == 3) {
    acc[i] = FMA(1.0 / 3.0, dk, acc[i]);
    out[i] = FMA(dt, k[i], y[i]);
  } else {
    out[i] = ADD(y[i], FMA(1.0 / 6.0, dk, acc[i]));
  }
}

void launch_rk_update_ref(int stage, long long n, double dt, const double* k, const double* y, double* acc,
                          double* out) {
  const int threads = 256;
  const long long blocks = (n + threads - 1) / threads;
  switch (stage) {
    case 1: NRPYELL_LAUNCH(k_rk_update_ref<1>, (unsigned)blocks, threads, 0, n, dt, k, y, acc, out); break;
    case 2: NRPYELL_LAUNCH(k_rk_update_ref<2>, (unsigned)blocks, threads, 0, n, dt, k, y, acc, out); break;
    case 3: NRPYELL_LAUNCH(k_rk_update_ref<3>, (unsigned)blocks, threads, 0, n, dt, k, y, acc, out); break;
    default: NRPYELL_LAUNCH(k_rk_update_ref<4>, (unsigned)blocks, threads, 0, n, dt, k, y, acc, out); break;
  }
}

// ---------------------------------------------------------------------------
// Deterministic L2 sum: each block reduces a fixed set of points in a fixed
// tree order into partials[block]; the last block to finish (ticket counter)
// adds the partials in index order.  The result depends only on the data and
// the launch shape, never on scheduling.
constexpr int kL2Threads = 256;
constexpr int kL2Blocks = 592;  // 4 x 148 SMs

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) r += sh[w];
  }
  __syncthreads();
  return r;  // valid in thread 0
}

__global__ void __launch_bounds__(kL2Threads) k_l2_sum(Dims d, const double* __restrict__ w,
                                                       const double* __restrict__ g, double* __restrict__ partials,
                                                       double* __restrict__ result, unsigned int* counter) {
  __shared__ double sh[kL2Threads / 32];
  __shared__ bool last;
  const long long n = (long long)d.Nxx0 * d.Nxx1 * d.Nxx2;
  double acc = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(t % d.Nxx0) + NGHOSTS;
    const long long r = t / d.Nxx0;
    const int i1 = (int)(r % d.Nxx1) + NGHOSTS;
    const int i2 = (int)(r / d.Nxx1) + NGHOSTS;
    const long long idx = i0 + (long long)d.N0 * (i1 + (long long)d.N1 * i2);
    const double gv = g[idx];
    acc += gv * gv * __ldg(w + i0 + d.N0 * i1);
  }
  const double bs = block_sum(acc, sh);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = bs;
    __threadfence();
    const unsigned int ticket = atomicAdd(counter, 1u);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += ((volatile double*)partials)[b];
  const double tot = block_sum(v, sh);
  if (threadIdx.x == 0) {
    result[0] = tot;
    *counter = 0u;  // re-arm for the next launch
  }
}

void launch_l2_sum(const Dims& d, const L2Tables* lt, const double* g, Scratch* s) {
  NRPYELL_LAUNCH(k_l2_sum, kL2Blocks, kL2Threads, 0, d, lt->w, g, s->partials, s->result, s->counter);
}

}  // namespace nrpyell
