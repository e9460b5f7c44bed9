// Device code shared by the fused RK4 substep kernels (kernels_fused.cu: one
// thread per (i0,i1) column of P points reading through L1, or the block's
// planes staged in shared memory; kernels_march.cu: blocks marching along i2
// with the planes copied ahead by cp.async): the launch arguments, the point
// RHS, the RK combination, the radiation-BC column work and the stop-test
// reduction.  Every variant evaluates a point with the same
// operations in the same order, so all of them produce identical bits.
#pragma once

#include "fd_weights.h"
#include "kernels.cuh"

namespace nrpyell {

// Upwind first-derivative weights (one copy per translation unit).
static __constant__ double c_fd1w[11][11] = NRPYELL_FD1_UPWIND_INIT;

template <typename T>
struct SubDev {
  int N0, N1, Nxx0, Nxx1, Nxx2, half2;
  long long N01, Ntot;
  int tiles0, tiles1, tiles2;  // interior tile grid
  // marching kernel: each (i0,i1) column tile's planes are mbig chunks of PZ
  // planes (blocks first) and then chunks of msmall planes (blocks last)
  int mbig, msmall;
  int n_tiles, n_col_blocks, ncol;
  int ncz;  // direct kernel: z-layers of its 3-D grid that hold the column blocks
  const T* __restrict__ S;     // stage input
  const T* y;                  // y_n (aliases out at stage 4)
  T* acc;
  T* out;
  const T* __restrict__ aux;
  // Correction form (FP32 relaxation of a correction to an FP64 state, see
  // point_rhs_correction): the RHS of the FP64 base state, R0[0] the uu RHS
  // and R0[1] the residual bracket at interior points / the vv RHS at the
  // radiation ghost points; aux then holds S(U) = ADD_times_AUU/(8 P^7),
  // P = psi_background + U and the wavespeed.  nullptr otherwise.
  const T* __restrict__ R0;
  const T* __restrict__ coef;
  const double* __restrict__ colgeo;
  const double* __restrict__ w;  // L2 weights (stage-1 residual)
  double* partials;
  unsigned int* ticket;
  int* state;  // [0] n, [1] done, [2] converged
  double* history;
  const int* done;
  double volume, log10_tol;
  int max_steps;
  int check_every;  // > 0: Einstein Toolkit thorn semantics (see finalize_l2)
  int defer_l2;     // stage 1: store the per-tile partials only (k_finalize_l2 reduces them)
  T dt, eta;
  T cOB[2];
  double invdx0, invdx1;
};

// Entry of a substep kernel: waits until the kernels before it in the
// stream have completed and their writes are visible (a no-op unless it was
// launched with programmatic stream serialization), then lets the next
// kernel's blocks be scheduled as this grid drains.  Nothing written by an
// earlier kernel -- the state, the done flag -- is read before it.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// Interior index along i2 after a wrap by 2 pi.
__device__ __forceinline__ int wrap2(int j, int Nxx2) {
  j -= NGHOSTS;
  if (j < 0) j += Nxx2;
  if (j >= Nxx2) j -= Nxx2;
  return j + NGHOSTS;
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

// 10th-order weights (rhs_eval.c:23-27): first derivative d_k, second e_k.
template <typename T>
struct W {
  static __device__ __forceinline__ T d(int k) {
    return k == 1 ? (T)(5.0 / 6.0) : k == 2 ? (T)(-5.0 / 21.0) : k == 3 ? (T)(5.0 / 84.0) : k == 4 ? (T)(-5.0 / 504.0) : (T)(1.0 / 1260.0);
  }
  static __device__ __forceinline__ T e(int k) {
    return k == 1 ? (T)(5.0 / 3.0) : k == 2 ? (T)(-5.0 / 21.0) : k == 3 ? (T)(5.0 / 126.0) : k == 4 ? (T)(-5.0 / 1008.0) : (T)(1.0 / 3150.0);
  }
};

// RHS of (uu, vv) at one interior point from the raw stencil sums and the
// pointwise values.  Every variant and the column blocks call this with the
// stencil sums accumulated in the same order, so all produce identical bits.
template <typename T>
__device__ __forceinline__ void point_rhs(T c, T vv, T AA, T psi, T ws, T C22, T C00, T C11, T C1, T C0, T Cc,
                                          T s0, T s1, T s00, T s11, T s22, T eta, T& ku, T& kv, T& bracket) {
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
  bracket = fma((T)0.125, AA / pu7, lap);
  ku = fma(-eta, c, vv);
  kv = (ws * ws) * bracket;
}

// Correction form of point_rhs.  The state is U + d with U an FP64 base state
// that stays fixed over a stretch of steps and d = (c, vv) the correction the
// kernel relaxes (in FP32).  The RHS is affine in the state except for the
// puncture source S(u) = ADD_times_AUU / (8 (psi + u)^7), so
//   uu RHS  = R0u + (vv - eta c)
//   bracket = R0b + lap(c) + [S(U + c) - S(U)]
//   vv RHS  = ws^2 * bracket,
// with R0u = V - eta U and R0b = lap(U) + S(U) evaluated in FP64.  The source
// difference is written as
//   S(U + c) - S(U) = -S(U) (c / (P + c)) (1 + r + ... + r^6),  r = P / (P + c),
// P = psi + U, so every term carries its own relative rounding error and
// the FP32 error of the whole RHS scales with the correction, not with U.
// ju and jv return the correction parts (vv - eta c, ws^2 (lap + dS)): the
// radiation BC, linear in the state, takes them as its interior input.
template <typename T>
__device__ __forceinline__ void point_rhs_correction(T c, T vv, T S, T P, T ws, T C22, T C00, T C11, T C1, T C0, T Cc,
                                                     T s0, T s1, T s00, T s11, T s22, T eta, T R0u, T R0b, T& ku,
                                                     T& kv, T& bracket, T& ju, T& jv) {
  T lap = Cc * c;
  lap = fma(C00, s00, lap);
  lap = fma(C11, s11, lap);
  lap = fma(C22, s22, lap);
  lap = fma(C1, s1, lap);
  lap = fma(C0, s0, lap);
  const T q = (T)1 / (P + c);
  const T r = P * q;
  T sum = fma(r, (T)1, (T)1);
#pragma unroll
  for (int k = 0; k < 5; k++) sum = fma(r, sum, (T)1);
  const T dS = -S * (c * q) * sum;
  const T jb = lap + dS;
  const T w2 = ws * ws;
  bracket = R0b + jb;
  ju = fma(-eta, c, vv);
  ku = R0u + ju;
  kv = w2 * bracket;
  jv = w2 * jb;
}

// Loads the pointwise values at idx / k2 and evaluates point_rhs.
template <typename T>
__device__ __forceinline__ void point_rhs_global(const SubDev<T>& a, long long idx, int k2, T c, T s0, T s1, T s00,
                                                 T s11, T s22, T& ku, T& kv, T& bracket) {
  const long long n01 = a.N01;
  point_rhs<T>(c, __ldg(a.S + a.Ntot + idx), __ldg(a.aux + ADD_TIMES_AUUGF * a.Ntot + idx),
               __ldg(a.aux + PSI_BACKGROUNDGF * a.Ntot + idx), __ldg(a.aux + WAVESPEEDGF * a.Ntot + idx),
               __ldg(a.coef + k2), __ldg(a.coef + n01 + k2), __ldg(a.coef + 2 * n01 + k2), __ldg(a.coef + 3 * n01 + k2),
               __ldg(a.coef + 4 * n01 + k2), __ldg(a.coef + 5 * n01 + k2), s0, s1, s00, s11, s22, a.eta, ku, kv,
               bracket);
}

// Stencil sums along i0 and i1 at interior point (i0,i1,i2) from global
// memory; ghost neighbours are read from their source points.  i2h is the i2
// index shifted by pi.
template <typename T>
__device__ __forceinline__ void stencil01(const SubDev<T>& a, const T* __restrict__ u, int i0, int i1, int i2, int i2h,
                                          T& s0, T& s1, T& s00, T& s11) {
  const long long base = i0 + (long long)a.N0 * i1 + a.N01 * i2;
  const long long rowh = (long long)a.N0 * i1 + a.N01 * i2h;  // (.,i1,i2h)
  const long long colh = i0 + a.N01 * i2h;                     // (i0,.,i2h)
  const int top = NGHOSTS + a.Nxx1;
#pragma unroll
  for (int k = 1; k <= 5; k++) {
    const int j0 = i0 - k;
    const long long im = (j0 >= NGHOSTS) ? base - k : (2 * NGHOSTS - 1 - j0) + rowh;
    const int jm = i1 - k, jp = i1 + k;
    const long long jmi = (jm >= NGHOSTS) ? base - (long long)k * a.N0 : colh + (long long)a.N0 * (2 * NGHOSTS - 1 - jm);
    const long long jpi = (jp < top) ? base + (long long)k * a.N0 : colh + (long long)a.N0 * (2 * top - 1 - jp);
    const T am = __ldg(u + im), ap = __ldg(u + base + k);
    const T bm = __ldg(u + jmi), bp = __ldg(u + jpi);
    s0 = fma(W<T>::d(k), ap - am, s0);
    s1 = fma(W<T>::d(k), bp - bm, s1);
    s00 = fma(W<T>::e(k), ap + am, s00);
    s11 = fma(W<T>::e(k), bp + bm, s11);
  }
}

// RK combination and stores of both gridfunctions at one interior point.
template <typename T, int STAGE>
__device__ __forceinline__ void store_point(const SubDev<T>& a, long long idx, T ku, T kv, T yu, T yv, T accu, T accv) {
  T ou, ov;
  rk_combine<T, STAGE>(ku, yu, accu, ou, a.dt);
  rk_combine<T, STAGE>(kv, yv, accv, ov, a.dt);
  if (STAGE != 4) {
    a.acc[idx] = accu;
    a.acc[a.Ntot + idx] = accv;
  }
  a.out[idx] = ou;
  a.out[a.Ntot + idx] = ov;
}

// Barrier over the NT threads that reduce (the whole block).
struct BlockSync {
  static __device__ __forceinline__ void sync() { __syncthreads(); }
};

// Stop test: the block that completes the last tile sums the per-tile
// partials in index order, writes log10 L2 to history[n] and updates state.
// Threads 0..NT-1 take part.
template <typename T, int NT, class Sync = BlockSync>
__device__ void finalize_l2(const SubDev<T>& a, double* sh) {
  const int tid = threadIdx.x;
  __threadfence();
  double v = 0.0;
  for (int i = tid; i < a.n_tiles; i += NT) v += ((volatile double*)a.partials)[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  Sync::sync();
  if ((tid & 31) == 0) sh[tid >> 5] = v;
  Sync::sync();
  if (tid == 0) {
    double tot = 0.0;
    for (int wi = 0; wi < NT / 32; wi++) tot += sh[wi];
    const double l2 = log10(1e-16 + sqrt(tot / a.volume));
    const int n = a.state[0];
    if (a.history) a.history[n] = l2;
    // main.c semantics: the stop test on every residual, log10 L2 <= tol.
    // The ET thorn's (NRPyEllipticET_..._Hyperbolic_Relaxation.c:185-217):
    // its loop index counts steps already taken minus one, it tests after
    // every check_every-th step and after the last one, with log10 L2 < tol.
    bool test = true;
    if (a.check_every > 0) test = n >= 1 && ((n - 1) % a.check_every == 0 || n >= a.max_steps);
    const bool met = test && (a.check_every > 0 ? l2 < a.log10_tol : l2 <= a.log10_tol);
    if (met) {
      a.state[2] = 1;
      a.state[1] = 1;
    } else if (n >= a.max_steps) {
      a.state[1] = 1;
    } else {
      a.state[0] = n + 1;
    }
    *a.ticket = 0u;
    __threadfence();
  }
}

// Reduces r2 over threads 0..NT-1, stores the tile's partial and returns
// true in each of them if this tile was the last one to complete; with
// `defer` it only stores the partial (a later launch reduces them).
template <int NT, class Sync = BlockSync>
__device__ __forceinline__ bool tile_partial(double r2, int tile, double* partials, unsigned int* ticket, int n_tiles,
                                             double* sh, bool* last, bool defer = false) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
  if ((tid & 31) == 0) sh[tid >> 5] = r2;
  Sync::sync();
  if (tid == 0) {
    double t = 0.0;
    for (int wi = 0; wi < NT / 32; wi++) t += sh[wi];
    partials[tile] = t;
    if (!defer) {
      __threadfence();
      *last = (atomicAdd(ticket, 1u) == (unsigned)n_tiles - 1);
    }
  }
  Sync::sync();
  return !defer && *last;
}

// ------------------------------------------------------------------ columns
constexpr int kColThreadsPerColumn = 16;

// Raw 11-point first-derivative sums of the radiation BC: along x0 with the
// weights w of the point's stencil offset, along x1 with the centred weights
// (the centre term is zero).  v holds the 11 values in stencil order.
__device__ __forceinline__ double radiation_sum_x0(const double* w, const double* v) {
  double d = w[0] * v[0];
#pragma unroll
  for (int m = 1; m < 11; m++) d = d + w[m] * v[m];
  return d;
}
__device__ __forceinline__ double radiation_sum_x1(const double* v) {
  double d = c_fd1w[5][0] * v[0];
#pragma unroll
  for (int m = 1; m < 11; m++)
    if (m != 5) d = d + c_fd1w[5][m] * v[m];
  return d;
}

// d f/d r at one radiation point from the raw x0 / x1 stencil sums.
__device__ __forceinline__ double radiation_drf(double d0, double d1, double invdx0, double invdx1, double dx0dr,
                                                double dx1dr) {
  d0 *= invdx0;
  d1 *= invdx1;
  return dx0dr * d0 + dx1dr * d1;
}

// RHS of one gridfunction on the five outer layers of a column, inner to
// outer (apply_bcs_outerradiation_and_inner.c:400-407): kprev is the RHS of
// the last interior point, drf/fvs the radial derivative and value at the
// last interior point (index 0) and at layers 0..4 (1..5); colgeo the
// column's radial geometry (r at index 0..5, stride N1).
__device__ __forceinline__ void radiation_layers(double cw, double kprev, const double* drf, const double* fvs,
                                                 const double* __restrict__ rcol, int N1, double* kk) {
#pragma unroll
  for (int L = 0; L < NGHOSTS; L++) {
    const double rn = __ldg(rcol + L * N1);
    const double rr = __ldg(rcol + (L + 1) * N1);
    const double out_int = -cw * (drf[L] + fvs[L] / rn);
    const double K = rn * rn * rn * (kprev - out_int);
    const double rinv = 1.0 / rr;
    const double outw = -cw * (drf[L + 1] + fvs[L + 1] * rinv);
    const double k = outw + K * rinv * rinv * rinv;
    kk[L] = k;
    kprev = k;
  }
}

// Radiation BC for CB columns (block-local index cb).  Column c, task r:
// r < 12 -> d f/d r at point jj = r % 6 of gridfunction g = r / 6 (point jj
// is i0 = N0-6+jj; jj = 0 is the last interior plane, jj = 1..5 the outer
// layers 0..4); r == 12 -> RHS at the last interior point.  The upwind x0
// stencil at point jj has offset -1 for jj <= 1 and -jj otherwise
// (compute_partial_r_f's rule); the x1 stencil is centred.  The "interior
// neighbour" derivative of layer L is the point derivative of layer L-1.
template <typename T, int STAGE, int NT>
__device__ void column_block(const SubDev<T>& a, int cb) {
  constexpr int CB = NT / kColThreadsPerColumn;
  __shared__ double drf[CB][2][6], fvs[CB][2][6], kl[CB][2], kk[CB][2][5];
  const int tid = threadIdx.x;
  const int c = tid / kColThreadsPerColumn, r = tid % kColThreadsPerColumn;
  const int colid = cb * CB + c;
  const bool live = colid < a.ncol;
  const int i1 = NGHOSTS + (live ? colid % a.Nxx1 : 0);
  const int i2 = NGHOSTS + (live ? colid / a.Nxx1 : 0);
  const int i2h = wrap2(i2 + a.half2, a.Nxx2);
  const int N0 = a.N0;
  const long long row = (long long)N0 * i1 + a.N01 * i2;
  if (live && r < 12) {
    const int g = r / 6, jj = r % 6;
    const T* f = a.S + g * a.Ntot;
    const int ip = N0 - 6 + jj;
    const int off = (jj <= 1) ? -1 : -jj;
    double v[11];
#pragma unroll
    for (int m = 0; m < 11; m++) v[m] = (double)__ldg(f + row + ip + off - 5 + m);
    const double d0 = radiation_sum_x0(c_fd1w[off + 5], v);
    // centred x1 stencil; points across the axis come from their images
    const int top = NGHOSTS + a.Nxx1;
#pragma unroll
    for (int m = 0; m < 11; m++) {
      const int j1 = i1 + m - 5;
      long long id;
      if (j1 < NGHOSTS)
        id = ip + (long long)N0 * (2 * NGHOSTS - 1 - j1) + a.N01 * i2h;
      else if (j1 >= top)
        id = ip + (long long)N0 * (2 * top - 1 - j1) + a.N01 * i2h;
      else
        id = ip + (long long)N0 * j1 + a.N01 * i2;
      v[m] = (m == 5) ? 0.0 : (double)__ldg(f + id);
    }
    const double d1 = radiation_sum_x1(v);
    drf[c][g][jj] = radiation_drf(d0, d1, a.invdx0, a.invdx1, __ldg(a.colgeo + (1 * 6 + jj) * a.N1 + i1),
                                  __ldg(a.colgeo + (2 * 6 + jj) * a.N1 + i1));
    fvs[c][g][jj] = (double)__ldg(f + row + ip);
  } else if (live && r == 12) {
    const int i0 = N0 - NGHOSTS - 1;
    const T* u = a.S;
    const long long idx = row + i0;
    T s0 = 0, s1 = 0, s00 = 0, s11 = 0, s22 = 0;
    stencil01<T>(a, u, i0, i1, i2, i2h, s0, s1, s00, s11);
    const long long line = i0 + (long long)N0 * i1;
#pragma unroll
    for (int k = 1; k <= 5; k++)
      s22 = fma(W<T>::e(k),
                __ldg(u + line + a.N01 * wrap2(i2 + k, a.Nxx2)) + __ldg(u + line + a.N01 * wrap2(i2 - k, a.Nxx2)), s22);
    T ku, kv, br;
    point_rhs_global<T>(a, idx, i0 + N0 * i1, __ldg(u + idx), s0, s1, s00, s11, s22, ku, kv, br);
    kl[c][0] = (double)ku;
    kl[c][1] = (double)kv;
  }
  __syncthreads();
  if (live && r < 2) {
    const int g = r;
    radiation_layers((double)a.cOB[g], kl[c][g], drf[c][g], fvs[c][g], a.colgeo + i1, a.N1, kk[c][g]);
  }
  __syncthreads();
  if (live && r < 10) {
    const int g = r / 5, L = r % 5;
    const long long idx = g * a.Ntot + row + N0 - NGHOSTS + L;
    T accv = (STAGE == 1) ? (T)0 : a.acc[idx];
    T ov;
    rk_combine<T, STAGE>((T)kk[c][g][L], a.y[idx], accv, ov, a.dt);
    if (STAGE != 4) a.acc[idx] = accv;
    a.out[idx] = ov;
  }
}

// ------------------------------------------------ radiation columns by rows
// The radiation BC of the x0max face: the column blocks of the 8-warp
// direct, shared-memory planes and marching kernels.  A block takes
// kRows consecutive i1 columns at one i2: it copies the outer 12 points of
// uu and vv along i0 on those rows and on 5 rows either side (rows across
// the axis from their images) into shared memory, then computes every
// column's 12 radial derivatives, the RHS of its last interior point, the
// layer recurrence and the RK combination with the same arithmetic as
// column_block.
constexpr int kRows = 32;

// Shared memory of column_rows, in doubles: F[2][kRows+10][12], drf and fvs
// [kRows][2][6], kl [kRows][2], kk [kRows][2][5], and G[kRows][kColG]: per
// column the values the RHS of its last interior point reads outside F
// (uu at i2 +- 1..5, vv, the three auxevol fields, the six metric weights).
// The correction form (CORR) adds R0u and R0b of the last interior point
// (items 20, 21).
constexpr int kColG = 20;
constexpr int kRowsSmem = 2 * (kRows + 10) * 12 + 2 * kRows * 12 + kRows * 2 + kRows * 10 + kRows * kColG;
constexpr int kColGCorr = 22;
constexpr int kRowsSmemCorr = kRowsSmem + kRows * (kColGCorr - kColG);

// CORR: the correction form (point_rhs_correction).  The radiation BC is
// linear in the state and in the interior RHS it starts from, so the layers
// are computed from the correction alone (its radial derivatives and the
// correction part of the last interior point's RHS) and the base state's
// RHS at the ghost point, R0, is added before the RK combination.
template <typename T, int STAGE, int NT, bool CORR = false>
__device__ void column_rows(const SubDev<T>& a, int cb, double* smem) {
  static_assert(NT >= 2 * kRows, "the layer recurrence takes one thread per column and gridfunction");
  constexpr int NCG = CORR ? kColGCorr : kColG;
  constexpr int NRW = kRows + 10, NQ = 12;
  double(*F)[NRW][NQ] = reinterpret_cast<double(*)[NRW][NQ]>(smem);
  double(*drf)[2][6] = reinterpret_cast<double(*)[2][6]>(smem + 2 * NRW * NQ);
  double(*fvs)[2][6] = reinterpret_cast<double(*)[2][6]>(smem + 2 * NRW * NQ + kRows * 12);
  double(*kl)[2] = reinterpret_cast<double(*)[2]>(smem + 2 * NRW * NQ + 2 * kRows * 12);
  double(*kk)[2][5] = reinterpret_cast<double(*)[2][5]>(smem + 2 * NRW * NQ + 2 * kRows * 12 + 2 * kRows);
  double(*G)[NCG] = reinterpret_cast<double(*)[NCG]>(smem + 2 * NRW * NQ + 2 * kRows * 12 + 2 * kRows + 10 * kRows);
  const int tid = threadIdx.x;
  const int nb1 = (a.Nxx1 + kRows - 1) / kRows;
  const int i1a = NGHOSTS + (cb % nb1) * kRows;
  const int i2 = NGHOSTS + cb / nb1;
  const int top = NGHOSTS + a.Nxx1;
  const int ncol = min(kRows, top - i1a);
  const int i2h = wrap2(i2 + a.half2, a.Nxx2);
  const int N0 = a.N0;
  for (int e = tid; e < 2 * NRW * NQ; e += NT) {
    const int q = e % NQ, j = (e / NQ) % NRW, g = e / (NQ * NRW);
    if (j >= ncol + 2 * NGHOSTS) continue;  // not needed
    int i1 = i1a - NGHOSTS + j, i2s = i2;
    if (i1 < NGHOSTS) {
      i1 = 2 * NGHOSTS - 1 - i1;
      i2s = i2h;
    } else if (i1 >= top) {
      i1 = 2 * top - 1 - i1;
      i2s = i2h;
    }
    F[g][j][q] = (double)__ldg(a.S + g * a.Ntot + (N0 - NQ + q) + (long long)N0 * i1 + a.N01 * i2s);
  }
  // the rest of each column's last-interior-point inputs, spread over the
  // block (item m of column c: 0..9 uu at i2 -+ 1..5, 10 vv, 11..13 auxevol,
  // 14..19 metric weights, CORR: 20..21 R0u, R0b)
  for (int e = tid; e < kRows * NCG; e += NT) {
    const int c = e / NCG, m = e - c * NCG;
    if (c >= ncol) continue;
    const long long line = (N0 - NGHOSTS - 1) + (long long)N0 * (i1a + c);
    const T* src;
    if (m < 10) {
      const int k = m / 2 + 1;
      src = a.S + line + a.N01 * wrap2((m & 1) ? i2 + k : i2 - k, a.Nxx2);
    } else if (m == 10) {
      src = a.S + a.Ntot + line + a.N01 * i2;
    } else if (m < 14) {
      const int gf = m == 11 ? ADD_TIMES_AUUGF : (m == 12 ? PSI_BACKGROUNDGF : WAVESPEEDGF);
      src = a.aux + gf * a.Ntot + line + a.N01 * i2;
    } else if (m < 20) {
      src = a.coef + (m - 14) * a.N01 + line;
    } else {
      src = a.R0 + (m - 20) * a.Ntot + line + a.N01 * i2;
    }
    G[c][m] = (double)__ldg(src);
  }
  __syncthreads();
  // radial derivatives at the last interior point and the 5 layers (items
  // c*12 + g*6 + jj), then the RHS of each column's last interior point
  for (int it = tid; it < kRows * 13; it += NT) {
    if (it < kRows * 12) {
      const int c = it / 12, g = (it / 6) % 2, jj = it % 6;
      if (c >= ncol) continue;
      const int off = (jj <= 1) ? -1 : -jj;
      double v[11];
#pragma unroll
      for (int m = 0; m < 11; m++) v[m] = F[g][c + NGHOSTS][1 + jj + off + m];
      const double d0 = radiation_sum_x0(c_fd1w[off + 5], v);
#pragma unroll
      for (int m = 0; m < 11; m++) v[m] = (m == 5) ? 0.0 : F[g][c + m][6 + jj];
      const double d1 = radiation_sum_x1(v);
      const int i1 = i1a + c;
      drf[c][g][jj] = radiation_drf(d0, d1, a.invdx0, a.invdx1, __ldg(a.colgeo + (1 * 6 + jj) * a.N1 + i1),
                                    __ldg(a.colgeo + (2 * 6 + jj) * a.N1 + i1));
      fvs[c][g][jj] = F[g][c + NGHOSTS][6 + jj];
    } else {
      const int c = it - kRows * 12;
      if (c >= ncol) continue;
      const double* row = F[0][c + NGHOSTS];
      T s0 = 0, s1 = 0, s00 = 0, s11 = 0, s22 = 0;
#pragma unroll
      for (int k = 1; k <= 5; k++) {
        const T am = (T)row[6 - k], ap = (T)row[6 + k];
        const T bm = (T)F[0][c + NGHOSTS - k][6], bp = (T)F[0][c + NGHOSTS + k][6];
        s0 = fma(W<T>::d(k), ap - am, s0);
        s1 = fma(W<T>::d(k), bp - bm, s1);
        s00 = fma(W<T>::e(k), ap + am, s00);
        s11 = fma(W<T>::e(k), bp + bm, s11);
      }
      const double* gc = G[c];
#pragma unroll
      for (int k = 1; k <= 5; k++) s22 = fma(W<T>::e(k), (T)gc[2 * k - 1] + (T)gc[2 * k - 2], s22);
      T ku, kv, br;
      if (CORR) {
        T ju, jv;
        point_rhs_correction<T>((T)row[6], (T)gc[10], (T)gc[11], (T)gc[12], (T)gc[13], (T)gc[14], (T)gc[15],
                                (T)gc[16], (T)gc[17], (T)gc[18], (T)gc[19], s0, s1, s00, s11, s22, a.eta,
                                (T)gc[NCG - 2], (T)gc[NCG - 1], ku, kv, br, ju, jv);
        kl[c][0] = (double)ju;
        kl[c][1] = (double)jv;
      } else {
        point_rhs<T>((T)row[6], (T)gc[10], (T)gc[11], (T)gc[12], (T)gc[13], (T)gc[14], (T)gc[15], (T)gc[16],
                     (T)gc[17], (T)gc[18], (T)gc[19], s0, s1, s00, s11, s22, a.eta, ku, kv, br);
        kl[c][0] = (double)ku;
        kl[c][1] = (double)kv;
      }
    }
  }
  __syncthreads();
  if (tid < 2 * ncol) {
    const int c = tid / 2, g = tid % 2;
    radiation_layers((double)a.cOB[g], kl[c][g], drf[c][g], fvs[c][g], a.colgeo + i1a + c, a.N1, kk[c][g]);
  }
  __syncthreads();
  for (int it = tid; it < ncol * 10; it += NT) {
    const int c = it / 10, g = (it / 5) % 2, L = it % 5;
    const long long idx = g * a.Ntot + (long long)N0 * (i1a + c) + a.N01 * i2 + N0 - NGHOSTS + L;
    T accv = (STAGE == 1) ? (T)0 : a.acc[idx];
    T ov;
    const double kfull = CORR ? kk[c][g][L] + (double)__ldg(a.R0 + idx) : kk[c][g][L];
    rk_combine<T, STAGE>((T)kfull, a.y[idx], accv, ov, a.dt);
    if (STAGE != 4) a.acc[idx] = accv;
    a.out[idx] = ov;
  }
}

// Interior index along i2 for any j (a tile that runs past the last plane
// can reach more than one wrap on short grids).
__device__ __forceinline__ int wrapm(int j, int Nxx2) {
  j -= NGHOSTS;
  while (j < 0) j += Nxx2;
  while (j >= Nxx2) j -= Nxx2;
  return j + NGHOSTS;
}

template <typename T>
inline SubDev<T> make_dev(const SubstepArgs& a, int by, int p);

// ---- batched launches (kernels_fused.cu, kernels_march.cu): the
// shared-memory planes or marching kernel over many grids in one launch.
// Launch arguments of one grid for the shape a.tile (kind 4 or 5).
template <typename T>
bool batch_launch_dev(const SubstepArgs& a, SubDev<T>* out);
// One substep of n grids; devs (device) holds the grids' arguments for this
// stage, offs (device) their first block; blocks = total blocks.  corr: the
// correction form (FP32, marching shapes only; every grid has R0).
template <typename T>
void launch_substep_batch(int stage, bool resid, int tile, const SubDev<T>* devs, const int* offs, int n, int blocks,
                          bool corr = false);
// The marching kernel's part of launch_substep_batch: shape v of its list.
template <typename T>
void launch_march_batch(int stage, bool resid, int v, const SubDev<T>* devs, const int* offs, int n, int blocks,
                        bool corr = false);

template <typename T>
inline SubDev<T> make_dev(const SubstepArgs& a, int by, int p) {
  SubDev<T> f;
  const Dims& d = a.d;
  f.N0 = d.N0;
  f.N1 = d.N1;
  f.Nxx0 = d.Nxx0;
  f.Nxx1 = d.Nxx1;
  f.Nxx2 = d.Nxx2;
  f.half2 = d.Nxx2 / 2;
  f.N01 = (long long)d.N0 * d.N1;
  f.Ntot = d.Ntot;
  f.tiles0 = (d.Nxx0 + 31) / 32;
  f.tiles1 = (d.Nxx1 + by - 1) / by;
  f.tiles2 = (d.Nxx2 + p - 1) / p;
  f.n_tiles = f.tiles0 * f.tiles1 * f.tiles2;
  f.mbig = f.tiles2;
  f.msmall = 0;
  f.ncz = 0;
  f.ncol = d.Nxx1 * d.Nxx2;
  f.S = (const T*)a.S;
  f.y = (const T*)a.y;
  f.acc = (T*)a.acc;
  f.out = (T*)a.out;
  f.aux = (const T*)a.aux;
  f.R0 = (const T*)a.R0;
  f.coef = sizeof(T) == 8 ? (const T*)a.rt->coef : (const T*)a.rt->coef32;
  f.colgeo = a.bt->colgeo;
  f.w = a.lt ? a.lt->w : nullptr;
  f.partials = a.s->partials;
  f.ticket = a.s->counter;
  f.state = a.state;
  f.history = a.history;
  f.done = a.done;
  f.volume = a.lt ? a.lt->volume : 1.0;
  f.log10_tol = a.log10_tol;
  f.max_steps = a.max_steps;
  f.check_every = a.check_every;
  f.defer_l2 = a.defer_l2;
  f.dt = (T)a.dt;
  f.eta = (T)a.eta;
  f.cOB[0] = (T)a.cOB[0];
  f.cOB[1] = (T)a.cOB[1];
  f.invdx0 = a.rt->invdx[0];
  f.invdx1 = a.rt->invdx[1];
  return f;
}

}  // namespace nrpyell
