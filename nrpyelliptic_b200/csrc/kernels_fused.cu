// Fused RK4 substep kernel: the fast path of MoL_step_forward_in_time and of
// the relaxation drivers.
//
// One RK4 substep of the reference (MoL_step_forward_in_time.c:12-176) is
// rhs_eval over the interior, the radiation BC on the RHS at the pure outer
// points, the inner-BC copy of the RHS, and a linear combination over every
// point.  Here the whole substep is ONE kernel launch with two kinds of
// blocks:
//   interior blocks: each thread owns an (i0,i1) pair and P consecutive i2
//     planes; it evaluates the RHS and feeds it straight into the RK
//     combination (the RHS never touches memory).  Stencil points that fall
//     in an inner ghost zone are read from their source point (the SymTP
//     reflections of symtp_ghost_source, verified against the caller's
//     bc_struct), so inner ghost zones are never written or read during a
//     relaxation.  At stage 1 the residual -- the vv-RHS bracket before the
//     wavespeed^2 factor -- is squared, weighted and reduced per block; the
//     last block to finish forms the L2 norm in a fixed order and runs the
//     stop test.
//   column blocks: the radiation BC of the x0max face, one (i1,i2) column at
//     a time for both gridfunctions, layers g = 0..4 inner to outer
//     (apply_bcs_outerradiation_and_inner.c:369-408), followed by the RK
//     combination at those points.  A column recomputes the RHS of its last
//     interior point itself, so it never waits for an interior block.
// The metric factors of the RHS depend on (i0,i1) only and are folded into
// six per-(i0,i1) weights (tables.cu), leaving one division per point.
#include "fd_weights.h"
#include "kernels.cuh"

namespace nrpyell {

__constant__ double c_fd1w[11][11] = NRPYELL_FD1_UPWIND_INIT;

template <typename T>
struct SubDev {
  int N0, N1, Nxx0, Nxx1, Nxx2, half2;
  long long N01, Ntot;
  int tiles0, tiles1, tiles2;  // interior tile grid
  int n_int_blocks, ncol, n_col_blocks;
  const T* __restrict__ S;     // stage input
  const T* y;                  // y_n (aliases out at stage 4)
  T* acc;
  T* out;
  const T* __restrict__ aux;
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
  double* stall;
  int stall_window;
  double stall_log_drop;
  T dt, eta;
  T cOB[2];
  double invdx0, invdx1;
};

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

// RHS of (uu, vv) at one interior point from the raw stencil sums.  Shared by
// interior threads and column blocks so both produce identical bits.
template <typename T>
__device__ __forceinline__ void point_rhs(const SubDev<T>& a, long long idx, int k2, T c, T s0, T s1, T s00, T s11,
                                          T s22, T& ku, T& kv, T& bracket) {
  const long long n01 = a.N01;
  const T C22 = __ldg(a.coef + k2), C00 = __ldg(a.coef + n01 + k2), C11 = __ldg(a.coef + 2 * n01 + k2);
  const T C1 = __ldg(a.coef + 3 * n01 + k2), C0 = __ldg(a.coef + 4 * n01 + k2), Cc = __ldg(a.coef + 5 * n01 + k2);
  const T AA = __ldg(a.aux + ADD_TIMES_AUUGF * a.Ntot + idx);
  const T psi = __ldg(a.aux + PSI_BACKGROUNDGF * a.Ntot + idx);
  const T ws = __ldg(a.aux + WAVESPEEDGF * a.Ntot + idx);
  const T vv = __ldg(a.S + a.Ntot + idx);
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
  ku = fma(-a.eta, c, vv);
  kv = (ws * ws) * bracket;
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

// Stencil sums along i0 and i1 at interior point (i0,i1,i2); ghost neighbours
// are read from their source points.  i2h is the i2 index shifted by pi.
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

constexpr int kColThreadsPerColumn = 16;

template <typename T, int STAGE, bool RESID, int BY, int P>
__global__ void __launch_bounds__(32 * BY) k_substep(SubDev<T> a) {
  constexpr int NT = 32 * BY;
  constexpr int CB = NT / kColThreadsPerColumn;
  __shared__ double sh[NT / 32 > 8 ? NT / 32 : 8];
  __shared__ bool last_block;
  __shared__ double drf[CB][2][6], fvs[CB][2][6], kl[CB][2], kk[CB][2][5];
  if (*a.done) return;
  const int tid = threadIdx.x;
  // Column blocks come first in the launch order: their dependent load
  // chains then overlap with the interior blocks instead of forming a tail.
  if ((int)blockIdx.x >= a.n_col_blocks) {
    // ------------------------------------------------------------ interior
    const int b = blockIdx.x - a.n_col_blocks;
    const int t0 = b % a.tiles0, t1 = (b / a.tiles0) % a.tiles1, t2 = b / (a.tiles0 * a.tiles1);
    const int i0 = t0 * 32 + (tid & 31) + NGHOSTS;
    const int i1 = t1 * BY + (tid >> 5) + NGHOSTS;
    const int z0 = t2 * P + NGHOSTS;
    double r2 = 0.0;
    if (i0 < NGHOSTS + a.Nxx0 && i1 < NGHOSTS + a.Nxx1) {
      const T* u = a.S;
      const long long line = i0 + (long long)a.N0 * i1;
      // uu along i2 for planes z0-5 .. z0+P+4 (wrapped by 2 pi)
      T col[P + 10];
#pragma unroll
      for (int q = 0; q < P + 10; q++) col[q] = __ldg(u + line + a.N01 * wrap2(z0 - 5 + q, a.Nxx2));
      const int k2 = i0 + a.N0 * i1;
#pragma unroll
      for (int p = 0; p < P; p++) {
        const int i2 = z0 + p;
        if (i2 < NGHOSTS + a.Nxx2) {
          const int i2h = wrap2(i2 + a.half2, a.Nxx2);
          T s0 = 0, s1 = 0, s00 = 0, s11 = 0, s22 = 0;
          stencil01<T>(a, u, i0, i1, i2, i2h, s0, s1, s00, s11);
#pragma unroll
          for (int k = 1; k <= 5; k++) s22 = fma(W<T>::e(k), col[p + 5 + k] + col[p + 5 - k], s22);
          const long long idx = line + a.N01 * i2;
          T ku, kv, br;
          point_rhs<T>(a, idx, k2, col[p + 5], s0, s1, s00, s11, s22, ku, kv, br);
          T accu = (STAGE == 1) ? (T)0 : a.acc[idx];
          T accv = (STAGE == 1) ? (T)0 : a.acc[a.Ntot + idx];
          const T yu = a.y[idx], yv = a.y[a.Ntot + idx];
          T ou, ov;
          rk_combine<T, STAGE>(ku, yu, accu, ou, a.dt);
          rk_combine<T, STAGE>(kv, yv, accv, ov, a.dt);
          if (STAGE != 4) {
            a.acc[idx] = accu;
            a.acc[a.Ntot + idx] = accv;
          }
          a.out[idx] = ou;
          a.out[a.Ntot + idx] = ov;
          if (RESID) {
            const double bb = (double)br;
            r2 += bb * bb * __ldg(a.w + k2);
          }
        }
      }
    }
    if (RESID) {
      // per-block partial in a fixed order, then the last block forms the norm
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
      if ((tid & 31) == 0) sh[tid >> 5] = r2;
      __syncthreads();
      if (tid == 0) {
        double t = 0.0;
        for (int wi = 0; wi < NT / 32; wi++) t += sh[wi];
        a.partials[b] = t;
        __threadfence();
        last_block = (atomicAdd(a.ticket, 1u) == (unsigned)a.n_int_blocks - 1);
      }
      __syncthreads();
      if (last_block) {
        __threadfence();
        double v = 0.0;
        for (int i = tid; i < a.n_int_blocks; i += NT) v += ((volatile double*)a.partials)[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        __syncthreads();
        if ((tid & 31) == 0) sh[tid >> 5] = v;
        __syncthreads();
        if (tid == 0) {
          double tot = 0.0;
          for (int wi = 0; wi < NT / 32; wi++) tot += sh[wi];
          const double l2 = log10(1e-16 + sqrt(tot / a.volume));
          const int n = a.state[0];
          if (a.history) a.history[n] = l2;
          // Stall test on the best residual so far: the relaxation residual
          // oscillates (and grows for a while after a cold start), so only a
          // lack of progress of the running minimum over a whole window
          // counts, and only once that minimum is within two decades of the
          // tolerance of this phase -- a precision floor shows up there.
          bool stalled = false;
          if (a.stall_window > 0) {
            if (n == 0 || l2 < a.stall[0] + a.stall_log_drop) {
              a.stall[0] = l2;
              a.stall[1] = (double)n;
            } else if (n - (int)a.stall[1] >= a.stall_window && a.stall[0] <= a.log10_tol + 2.0) {
              stalled = true;
            }
          }
          if (l2 <= a.log10_tol) {
            a.state[2] = 1;
            a.state[1] = 1;
          } else if (stalled) {
            a.state[3] = 1;
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
    }
    return;
  }

  // -------------------------------------------------------------- columns
  // Column c of this block, task r: r < 12 -> d f/d r at point jj = r % 6 of
  // gridfunction g = r / 6 (point jj is i0 = N0-6+jj; jj = 0 is the last
  // interior plane, jj = 1..5 the outer layers 0..4); r == 12 -> RHS at the
  // last interior point.
  const int cb = blockIdx.x;
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
    const int off = (jj <= 1) ? -1 : -jj;  // compute_partial_r_f's upwind offset at i0 = ip
    const double* wt = c_fd1w[off + 5];
    double d0 = 0.0;
#pragma unroll
    for (int m = 0; m < 11; m++) {
      const double term = wt[m] * (double)__ldg(f + row + ip + off - 5 + m);
      d0 = (m == 0) ? term : d0 + term;
    }
    d0 *= a.invdx0;
    // centred x1 stencil; points across the axis come from their images
    const int top = NGHOSTS + a.Nxx1;
    double d1 = 0.0;
    bool first = true;
#pragma unroll
    for (int m = 0; m < 11; m++) {
      if (m == 5) continue;
      const int j1 = i1 + m - 5;
      long long id;
      if (j1 < NGHOSTS)
        id = ip + (long long)N0 * (2 * NGHOSTS - 1 - j1) + a.N01 * i2h;
      else if (j1 >= top)
        id = ip + (long long)N0 * (2 * top - 1 - j1) + a.N01 * i2h;
      else
        id = ip + (long long)N0 * j1 + a.N01 * i2;
      const double term = c_fd1w[5][m] * (double)__ldg(f + id);
      d1 = first ? term : d1 + term;
      first = false;
    }
    d1 *= a.invdx1;
    const double dx0dr = __ldg(a.colgeo + (1 * 6 + jj) * a.N1 + i1);
    const double dx1dr = __ldg(a.colgeo + (2 * 6 + jj) * a.N1 + i1);
    drf[c][g][jj] = dx0dr * d0 + dx1dr * d1;
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
    point_rhs<T>(a, idx, i0 + N0 * i1, __ldg(u + idx), s0, s1, s00, s11, s22, ku, kv, br);
    kl[c][0] = (double)ku;
    kl[c][1] = (double)kv;
  }
  __syncthreads();
  if (live && r < 2) {
    const int g = r;
    const double cw = (double)a.cOB[g];
    double kprev = kl[c][g];
#pragma unroll
    for (int L = 0; L < NGHOSTS; L++) {
      const double rn = __ldg(a.colgeo + (0 * 6 + L) * a.N1 + i1);
      const double rr = __ldg(a.colgeo + (0 * 6 + L + 1) * a.N1 + i1);
      const double out_int = -cw * (drf[c][g][L] + fvs[c][g][L] / rn);
      const double K = rn * rn * rn * (kprev - out_int);
      const double rinv = 1.0 / rr;
      const double outw = -cw * (drf[c][g][L + 1] + fvs[c][g][L + 1] * rinv);
      const double k = outw + K * rinv * rinv * rinv;
      kk[c][g][L] = k;
      kprev = k;
    }
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

// Inner ghost points of gfs copied from their sources (apply_bcs_inner_only);
// fills the ghost zones of y_n after a fused step or a relaxation.
template <typename T>
__global__ void k_ghost_fill(const int2* __restrict__ map, const signed char* __restrict__ par, int n, long long Ntot,
                             T* gfs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int2 m = map[t];
  const T s = (T)par[t];
  gfs[m.x] = s * gfs[m.y];
  gfs[Ntot + m.x] = s * gfs[Ntot + m.y];
}

// ------------------------------------------------------------------ tiles

struct TileShape {
  int by, p;
};
static const TileShape kTiles[] = {{4, 1}, {4, 2}, {2, 4}, {8, 1}, {8, 2}, {4, 4}};
constexpr int kNumTiles = sizeof(kTiles) / sizeof(kTiles[0]);

int substep_num_tiles() { return kNumTiles; }
void substep_tile_shape(int tile, int* bx, int* by, int* p) {
  *bx = 32;
  *by = kTiles[tile].by;
  *p = kTiles[tile].p;
}

int substep_interior_blocks(const Dims& d, int tile) {
  const TileShape s = kTiles[tile];
  return ((d.Nxx0 + 31) / 32) * ((d.Nxx1 + s.by - 1) / s.by) * ((d.Nxx2 + s.p - 1) / s.p);
}

template <typename T>
static SubDev<T> make_dev(const SubstepArgs& a) {
  const TileShape ts = kTiles[a.tile];
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
  f.tiles1 = (d.Nxx1 + ts.by - 1) / ts.by;
  f.tiles2 = (d.Nxx2 + ts.p - 1) / ts.p;
  f.n_int_blocks = f.tiles0 * f.tiles1 * f.tiles2;
  f.ncol = d.Nxx1 * d.Nxx2;
  f.S = (const T*)a.S;
  f.y = (const T*)a.y;
  f.acc = (T*)a.acc;
  f.out = (T*)a.out;
  f.aux = (const T*)a.aux;
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
  f.stall = a.stall;
  f.stall_window = a.stall_window;
  f.stall_log_drop = a.stall_log_drop;
  f.dt = (T)a.dt;
  f.eta = (T)a.eta;
  f.cOB[0] = (T)a.cOB[0];
  f.cOB[1] = (T)a.cOB[1];
  f.invdx0 = a.rt->invdx[0];
  f.invdx1 = a.rt->invdx[1];
  return f;
}

template <typename T, int STAGE, bool RESID, int BY, int P>
static void launch_one(const SubstepArgs& a) {
  SubDev<T> f = make_dev<T>(a);
  constexpr int NT = 32 * BY;
  constexpr int CB = NT / kColThreadsPerColumn;
  f.n_col_blocks = (f.ncol + CB - 1) / CB;
  NRPYELL_LAUNCH((k_substep<T, STAGE, RESID, BY, P>), f.n_int_blocks + f.n_col_blocks, NT, 0, f);
}

template <typename T, int STAGE, bool RESID>
static void launch_tile(const SubstepArgs& a) {
  switch (a.tile) {
    case 0: launch_one<T, STAGE, RESID, 4, 1>(a); break;
    case 1: launch_one<T, STAGE, RESID, 4, 2>(a); break;
    case 2: launch_one<T, STAGE, RESID, 2, 4>(a); break;
    case 3: launch_one<T, STAGE, RESID, 8, 1>(a); break;
    case 4: launch_one<T, STAGE, RESID, 8, 2>(a); break;
    default: launch_one<T, STAGE, RESID, 4, 4>(a); break;
  }
}

template <typename T>
void launch_substep(int stage, const SubstepArgs& a) {
  const bool resid = (stage == 1) && a.lt;
  switch (stage) {
    case 1:
      if (resid)
        launch_tile<T, 1, true>(a);
      else
        launch_tile<T, 1, false>(a);
      break;
    case 2: launch_tile<T, 2, false>(a); break;
    case 3: launch_tile<T, 3, false>(a); break;
    default: launch_tile<T, 4, false>(a); break;
  }
}
template void launch_substep<double>(int, const SubstepArgs&);
template void launch_substep<float>(int, const SubstepArgs&);

template <typename T>
void launch_ghost_fill(const Dims& d, const BcTables* bt, void* gfs) {
  if (bt->n_inner <= 0) return;
  NRPYELL_LAUNCH((k_ghost_fill<T>), (bt->n_inner + 255) / 256, 256, 0, bt->inner, bt->inner_par, bt->n_inner, d.Ntot,
                 (T*)gfs);
}
template void launch_ghost_fill<double>(const Dims&, const BcTables*, void*);
template void launch_ghost_fill<float>(const Dims&, const BcTables*, void*);

}  // namespace nrpyell
