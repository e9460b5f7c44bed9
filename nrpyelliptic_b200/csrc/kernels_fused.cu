// Fused RK4 substep kernels (the fast path of MoL_step_forward_in_time and
// of the relaxation drivers).
//
// One RK4 substep of the reference (MoL_step_forward_in_time.c:12-176) is
// rhs_eval over the interior, the radiation BC on the RHS at the pure outer
// points, the inner-BC copy of the RHS, and a linear combination over every
// point.  Here it is three kernels:
//   1. k_fused_interior: the RHS at each interior point straight into the RK
//      combination (the RHS never touches memory), the RHS of the last
//      interior x0 plane into a small face buffer, and at stage 1 optionally
//      the residual's weighted square for the L2 norm (the residual is the
//      vv-RHS bracket before the wavespeed^2 factor, so it comes for free).
//   2. k_fused_outer: the radiation BC for one (i1,i2) column of the x0max
//      face, all NGHOSTS layers inside one thread (layer g needs the RHS of
//      layer g-1), followed by the RK combination at those points.
//   3. k_fused_ghost: inner ghost points of the new stage copied from their
//      source points.  The RK combination is linear and pointwise and the
//      inner BC is a parity copy, so copying the combined stage gives the
//      same bits as combining the copied RHS when the ghost zones of the
//      incoming state already satisfy the inner BC.
// The metric factors of the RHS depend on (i0,i1) only and are folded into
// six per-(i0,i1) weights (tables.cu), leaving one division per point.
#include "fd_weights.h"
#include "kernels.cuh"

namespace nrpyell {

__constant__ double c_fd1w[11][11] = NRPYELL_FD1_UPWIND_INIT;

template <typename T>
struct FusedDev {
  Dims d;
  const T* __restrict__ S;
  const T* y;  // may alias out (stage 4 updates y_n in place)
  T* acc;
  T* out;
  const T* __restrict__ aux;
  const T* __restrict__ coef;
  const double* __restrict__ w;  // L2 weights (stage 1 residual)
  const double* __restrict__ colgeo;
  T* __restrict__ face;
  double* __restrict__ partials;
  const int2* __restrict__ inner;
  const signed char* __restrict__ inner_par;
  const int* __restrict__ done;
  int n_inner;
  T dt, eta;
  T cOB[2];
  double invdx0, invdx1;
};

template <typename T>
__device__ __forceinline__ T ldg(const T* p) {
  return __ldg(p);
}

template <typename T, int STAGE>
__device__ __forceinline__ void rk_combine(T k, T yv, T& acc, T& out, T dt) {
  const T dk = dt * k;
  if (STAGE == 1) {
    acc = (T)(1.0 / 6.0) * dk;
    out = fma((T)0.5, dk, yv);
  } else if (STAGE == 2) {
    acc = fma((T)(1.0 / 3.0), dk, acc);
    out = fma((T)0.5, dk, yv);
  } else if (STAGE == 3) {
    acc = fma((T)(1.0 / 3.0), dk, acc);
    out = fma(dt, k, yv);
  } else {
    out = yv + fma((T)(1.0 / 6.0), dk, acc);
  }
}

constexpr int kBX = 32, kBY = 4, kBZ = 2;
constexpr int kFusedThreads = kBX * kBY * kBZ;

template <typename T, int STAGE, bool RESID>
__global__ void __launch_bounds__(kFusedThreads) k_fused_interior(FusedDev<T> a) {
  __shared__ double sh[kFusedThreads / 32];
  if (*a.done) return;
  const Dims& d = a.d;
  const int i0 = blockIdx.x * kBX + threadIdx.x + NGHOSTS;
  const int i1 = blockIdx.y * kBY + threadIdx.y + NGHOSTS;
  const int i2 = blockIdx.z * kBZ + threadIdx.z + NGHOSTS;
  const bool in = i0 < NGHOSTS + d.Nxx0 && i1 < NGHOSTS + d.Nxx1 && i2 < NGHOSTS + d.Nxx2;
  double r2 = 0.0;
  if (in) {
    const int N0 = d.N0;
    const long long s2 = (long long)N0 * d.N1;
    const long long idx = i0 + (long long)N0 * i1 + s2 * i2;
    const long long Ntot = d.Ntot;
    const T* u = a.S;
    const T c = ldg(u + idx);
    // Raw 10th-order stencil sums (rhs_eval.c:23-27 weights).
    T s0 = 0, s1 = 0, s00 = 0, s11 = 0, s22 = 0;
    const T w1[6] = {0, (T)(5.0 / 6.0), (T)(-5.0 / 21.0), (T)(5.0 / 84.0), (T)(-5.0 / 504.0), (T)(1.0 / 1260.0)};
    const T w2[6] = {0, (T)(5.0 / 3.0), (T)(-5.0 / 21.0), (T)(5.0 / 126.0), (T)(-5.0 / 1008.0), (T)(1.0 / 3150.0)};
#pragma unroll
    for (int k = 1; k <= 5; k++) {
      const T am = ldg(u + idx - k), ap = ldg(u + idx + k);
      const T bm = ldg(u + idx - (long long)k * N0), bp = ldg(u + idx + (long long)k * N0);
      const T cm = ldg(u + idx - (long long)k * s2), cp = ldg(u + idx + (long long)k * s2);
      s0 = fma(w1[k], ap - am, s0);
      s1 = fma(w1[k], bp - bm, s1);
      s00 = fma(w2[k], ap + am, s00);
      s11 = fma(w2[k], bp + bm, s11);
      s22 = fma(w2[k], cp + cm, s22);
    }
    const long long n01 = (long long)N0 * d.N1;
    const int k2 = i0 + N0 * i1;
    const T C22 = ldg(a.coef + k2), C00 = ldg(a.coef + n01 + k2), C11 = ldg(a.coef + 2 * n01 + k2);
    const T C1 = ldg(a.coef + 3 * n01 + k2), C0 = ldg(a.coef + 4 * n01 + k2), Cc = ldg(a.coef + 5 * n01 + k2);
    const T AA = ldg(a.aux + ADD_TIMES_AUUGF * Ntot + idx);
    const T psi = ldg(a.aux + PSI_BACKGROUNDGF * Ntot + idx);
    const T ws = ldg(a.aux + WAVESPEEDGF * Ntot + idx);
    const T pu = psi + c;
    const T pu2 = pu * pu;
    const T pu4 = pu2 * pu2;
    const T pu7 = pu4 * pu2 * pu;
    T lap = Cc * c;
    lap = fma(C00, s00, lap);
    lap = fma(C11, s11, lap);
    lap = fma(C22, s22, lap);
    lap = fma(C1, s1, lap);
    lap = fma(C0, s0, lap);
    const T bracket = fma((T)0.125, AA / pu7, lap);
    const T vv = ldg(u + Ntot + idx);
    const T ku = fma(-a.eta, c, vv);
    const T kv = (ws * ws) * bracket;
    // RK combination for both gridfunctions.
    {
      T accu = (STAGE == 1) ? (T)0 : a.acc[idx];
      T accv = (STAGE == 1) ? (T)0 : a.acc[Ntot + idx];
      const T yu = a.y[idx], yv = a.y[Ntot + idx];
      T ou, ov;
      rk_combine<T, STAGE>(ku, yu, accu, ou, a.dt);
      rk_combine<T, STAGE>(kv, yv, accv, ov, a.dt);
      if (STAGE != 4) {
        a.acc[idx] = accu;
        a.acc[Ntot + idx] = accv;
      }
      a.out[idx] = ou;
      a.out[Ntot + idx] = ov;
    }
    if (i0 == NGHOSTS + d.Nxx0 - 1) {
      const int f = (i1 - NGHOSTS) + d.Nxx1 * (i2 - NGHOSTS);
      a.face[f] = ku;
      a.face[(long long)d.Nxx1 * d.Nxx2 + f] = kv;
    }
    if (RESID) {
      const double b = (double)bracket;
      r2 = b * b * __ldg(a.w + k2);
    }
  }
  if (RESID) {
    const int tid = threadIdx.x + kBX * (threadIdx.y + kBY * threadIdx.z);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
    if ((tid & 31) == 0) sh[tid >> 5] = r2;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int wi = 0; wi < kFusedThreads / 32; wi++) t += sh[wi];
      a.partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = t;
    }
  }
}

// Radiation BC along one (i1,i2) column of the x0max face for one
// gridfunction: apply_bcs_outerradiation_and_inner.c:369-408 for layers
// g = 0..4 (i0 = N0-5+g, FACE = (-1,0,0)).  Point j = 0..5 below is
// i0 = N0-6+j; j = 0 is the last interior plane.  The upwind x0 stencil at
// point j has offset -1 for j = 0, 1 and -j otherwise
// (compute_partial_r_f's rule), so all of them read i0 in [N0-12, N0-1];
// the x1 stencil is centred.  The "interior neighbour" quantities of layer g
// are those of point j = g, identical to the point quantities of layer g-1.
template <typename T, int STAGE>
__global__ void __launch_bounds__(128) k_fused_outer(FusedDev<T> a) {
  if (*a.done) return;
  const Dims& d = a.d;
  const int ncol = d.Nxx1 * d.Nxx2;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * ncol) return;
  const int gf = t / ncol;
  const int col = t - gf * ncol;
  const int i1 = col % d.Nxx1 + NGHOSTS;
  const int i2 = col / d.Nxx1 + NGHOSTS;
  const int N0 = d.N0, N1 = d.N1;
  const long long Ntot = d.Ntot;
  const long long rowbase = (long long)N0 * (i1 + (long long)N1 * i2);
  const T* f = a.S + gf * Ntot;
  T fv[12];
#pragma unroll
  for (int j = 0; j < 12; j++) fv[j] = ldg(f + rowbase + N0 - 12 + j);
  double drf[6];
#pragma unroll
  for (int jj = 0; jj < 6; jj++) {
    const int off = (jj <= 1) ? -1 : -jj;
    const double* wt = c_fd1w[off + 5];
    double d0 = 0.0;
    bool first = true;
#pragma unroll
    for (int m = 0; m < 11; m++) {
      const double term = wt[m] * (double)fv[jj + off + 1 + m];
      d0 = first ? term : d0 + term;
      first = false;
    }
    d0 *= a.invdx0;
    const long long pidx = rowbase + N0 - 6 + jj;
    double d1 = 0.0;
    first = true;
#pragma unroll
    for (int m = 0; m < 11; m++) {
      if (m == 5) continue;
      const double term = c_fd1w[5][m] * (double)ldg(f + pidx + (long long)(m - 5) * N0);
      d1 = first ? term : d1 + term;
      first = false;
    }
    d1 *= a.invdx1;
    const double dx0dr = __ldg(a.colgeo + (1 * 6 + jj) * N1 + i1);
    const double dx1dr = __ldg(a.colgeo + (2 * 6 + jj) * N1 + i1);
    drf[jj] = dx0dr * d0 + dx1dr * d1;
  }
  const double c = (double)a.cOB[gf];
  double kprev = (double)a.face[(long long)gf * ncol + col];
  T* acc = a.acc + gf * Ntot;
  T* out = a.out + gf * Ntot;
  const T* y = a.y + gf * Ntot;
#pragma unroll
  for (int g = 0; g < NGHOSTS; g++) {
    const double rn = __ldg(a.colgeo + (0 * 6 + g) * N1 + i1);
    const double r = __ldg(a.colgeo + (0 * 6 + g + 1) * N1 + i1);
    const double out_int = -c * (drf[g] + (double)fv[6 + g] / rn);
    const double K = rn * rn * rn * (kprev - out_int);
    const double rinv = 1.0 / r;
    const double outw = -c * (drf[g + 1] + (double)fv[7 + g] * rinv);
    const double k = outw + K * rinv * rinv * rinv;
    kprev = k;
    const long long idx = rowbase + N0 - NGHOSTS + g;
    T accv = (STAGE == 1) ? (T)0 : acc[idx];
    T ov;
    rk_combine<T, STAGE>((T)k, y[idx], accv, ov, a.dt);
    if (STAGE != 4) acc[idx] = accv;
    out[idx] = ov;
  }
}

template <typename T>
__global__ void k_fused_ghost(FusedDev<T> a) {
  if (*a.done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_inner) return;
  const int2 m = a.inner[t];
  const T s = (T)a.inner_par[t];
  const long long Ntot = a.d.Ntot;
  a.out[m.x] = s * a.out[m.y];
  a.out[Ntot + m.x] = s * a.out[Ntot + m.y];
}

int fused_interior_blocks(const Dims& d) {
  return ((d.Nxx0 + kBX - 1) / kBX) * ((d.Nxx1 + kBY - 1) / kBY) * ((d.Nxx2 + kBZ - 1) / kBZ);
}

template <typename T>
static FusedDev<T> make_dev(const FusedArgs& a) {
  FusedDev<T> f;
  f.d = a.d;
  f.S = (const T*)a.S;
  f.y = (const T*)a.y;
  f.acc = (T*)a.acc;
  f.out = (T*)a.out;
  f.aux = (const T*)a.aux;
  f.coef = sizeof(T) == 8 ? (const T*)a.rt->coef : (const T*)a.rt->coef32;
  f.w = a.lt ? a.lt->w : nullptr;
  f.colgeo = a.bt->colgeo;
  f.face = (T*)a.face;
  f.partials = a.s->partials;
  f.inner = a.bt->inner;
  f.inner_par = a.bt->inner_par;
  f.n_inner = a.bt->n_inner;
  f.done = a.done;
  f.dt = (T)a.dt;
  f.eta = (T)a.eta;
  f.cOB[0] = (T)a.cOB[0];
  f.cOB[1] = (T)a.cOB[1];
  f.invdx0 = a.rt->invdx[0];
  f.invdx1 = a.rt->invdx[1];
  return f;
}

template <typename T, int STAGE>
static void launch_interior(const FusedArgs& a, const FusedDev<T>& f) {
  const Dims& d = a.d;
  const dim3 block(kBX, kBY, kBZ);
  const dim3 grid((d.Nxx0 + kBX - 1) / kBX, (d.Nxx1 + kBY - 1) / kBY, (d.Nxx2 + kBZ - 1) / kBZ);
  if (STAGE == 1 && a.lt) {
    NRPYELL_LAUNCH((k_fused_interior<T, STAGE, true>), grid, block, 0, f);
  } else {
    NRPYELL_LAUNCH((k_fused_interior<T, STAGE, false>), grid, block, 0, f);
  }
}

template <typename T, int STAGE>
static void launch_stage(const FusedArgs& a) {
  FusedDev<T> f = make_dev<T>(a);
  const Dims& d = a.d;
  launch_interior<T, STAGE>(a, f);
  const int ncol2 = 2 * d.Nxx1 * d.Nxx2;
  NRPYELL_LAUNCH((k_fused_outer<T, STAGE>), (ncol2 + 127) / 128, 128, 0, f);
  if (f.n_inner > 0) NRPYELL_LAUNCH((k_fused_ghost<T>), (f.n_inner + 255) / 256, 256, 0, f);
}

template <typename T>
void launch_fused_substep(int stage, const FusedArgs& a) {
  switch (stage) {
    case 1: launch_stage<T, 1>(a); break;
    case 2: launch_stage<T, 2>(a); break;
    case 3: launch_stage<T, 3>(a); break;
    default: launch_stage<T, 4>(a); break;
  }
}
template void launch_fused_substep<double>(int, const FusedArgs&);
template void launch_fused_substep<float>(int, const FusedArgs&);

template <typename T>
void launch_fused_interior_only(int stage, const FusedArgs& a) {
  FusedDev<T> f = make_dev<T>(a);
  switch (stage) {
    case 1: launch_interior<T, 1>(a, f); break;
    case 2: launch_interior<T, 2>(a, f); break;
    case 3: launch_interior<T, 3>(a, f); break;
    default: launch_interior<T, 4>(a, f); break;
  }
}
template void launch_fused_interior_only<double>(int, const FusedArgs&);
template void launch_fused_interior_only<float>(int, const FusedArgs&);

// state[0] = n (current step index), state[1] = done, state[2] = converged.
__global__ void k_relax_check(const double* __restrict__ partials, int nblocks, double volume, double log10_tol,
                              int max_steps, double* __restrict__ history, int* __restrict__ state) {
  __shared__ double sh[8];
  if (state[1]) return;
  double v = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += partials[b];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += sh[w];
    const double l2 = log10(1e-16 + sqrt(tot / volume));
    const int n = state[0];
    if (history) history[n] = l2;
    if (l2 <= log10_tol) {
      state[1] = 1;
      state[2] = 1;
    } else if (n >= max_steps) {
      state[1] = 1;
    } else {
      state[0] = n + 1;
    }
  }
}

void launch_relax_check(int nblocks, Scratch* s, double volume, double log10_tol, int max_steps, double* history,
                        int* state) {
  NRPYELL_LAUNCH(k_relax_check, 1, 256, 0, s->partials, nblocks, volume, log10_tol, max_steps, history, state);
}

}  // namespace nrpyell
