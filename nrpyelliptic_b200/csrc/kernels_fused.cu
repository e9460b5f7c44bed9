// Fused RK4 substep kernels: the fast path of MoL_step_forward_in_time and of
// the relaxation drivers.
//
// One RK4 substep of the reference (MoL_step_forward_in_time.c:12-176) is
// rhs_eval over the interior, the radiation BC on the RHS at the pure outer
// points, the inner-BC copy of the RHS, and a linear combination over every
// point.  Here the whole substep is ONE kernel launch with two kinds of
// blocks:
//   column blocks (first in the launch): the radiation BC of the x0max face,
//     one (i1,i2) column at a time for both gridfunctions, layers 0..4 inner
//     to outer (apply_bcs_outerradiation_and_inner.c:369-408), then the RK
//     combination at those points.  A column recomputes the RHS of its last
//     interior point itself, so it never waits for an interior block.
//   interior blocks: the RHS at every interior point straight into the RK
//     combination (the RHS never touches memory).  Stencil points in an
//     inner ghost zone are read from their source point (the SymTP
//     reflections of symtp_ghost_source, verified against the caller's
//     bc_struct), so inner ghost zones are never written or read during a
//     relaxation.  At stage 1 the residual -- the vv-RHS bracket before the
//     wavespeed^2 factor -- is squared, weighted, reduced per tile, and the
//     last tile to finish forms the L2 norm in a fixed order and runs the
//     stop test.
// This file holds the direct variant: each thread owns an (i0,i1) pair and P
// consecutive i2 planes, holds uu along i2 in registers and reads the rest of
// its 31-point star through L1 (optionally loading the pointwise inputs of
// all P planes before the first store), and the shared-memory planes
// variant.  kernels_march.cu holds the marching variant; the autotuner picks
// among the shapes of all of them (the tile table below).
// The metric factors of the RHS depend on (i0,i1) only and are folded into
// six per-(i0,i1) weights (tables.cu), leaving one division per point.
#include "substep.cuh"

namespace nrpyell {

// ------------------------------------------------------- direct interior
// CORR: the correction form of the mixed-precision driver
// (point_rhs_correction; 8-warp shapes without PF only).
// At least MINB resident blocks per SM, which caps the registers.  The
// default caps the one-plane shapes at 1024 threads per SM (64 registers,
// which they fit without spilling) and the two-plane 8-warp shape at 3
// blocks per SM (78 registers, no spills; 47.0 -> 40.8 us per RK4 step at
// 128x128x16), and leaves the prefetching shapes to the compiler.
template <typename T, int STAGE, bool RESID, int BY, int P, bool PF, bool CORR = false,
          int MINB = PF ? 1 : (P == 1 ? 32 / BY : (BY == 8 && P == 2 ? 3 : 1))>
__global__ void __launch_bounds__(32 * BY, MINB) k_substep(SubDev<T> a) {
  constexpr int NT = 32 * BY;
  static_assert(!CORR || (NT >= 256 && !PF), "the correction form runs on 8-warp shapes without PF");
  __shared__ double sh[NT / 32 > 8 ? NT / 32 : 8];
  // radiation columns: blocks of 256 threads take 32 columns by rows
  // (column_rows), narrower blocks 16 threads per column (column_block)
  constexpr bool ROWS = NT >= 256;
  __shared__ double csm[ROWS ? (CORR ? kRowsSmemCorr : kRowsSmem) : 1];
  __shared__ bool last;
  pdl_enter();
  if (*a.done) return;
  // 3-D grid (tiles0, tiles1, ncz + tiles2): the first ncz z-layers hold the
  // column blocks (first in the launch), the rest the interior tiles, so the
  // tile coordinates are the block indices themselves (no integer division)
  const int ncz = a.ncz;
  if ((int)blockIdx.z < ncz) {
    const int cb = ((int)blockIdx.z * a.tiles1 + (int)blockIdx.y) * a.tiles0 + (int)blockIdx.x;
    if (cb >= a.n_col_blocks) return;
    if constexpr (ROWS)
      column_rows<T, STAGE, NT, CORR>(a, cb, csm);
    else
      column_block<T, STAGE, NT>(a, cb);
    return;
  }
  const int tid = threadIdx.x;
  const int t0 = blockIdx.x, t1 = blockIdx.y, t2 = (int)blockIdx.z - ncz;
  const int b = t0 + a.tiles0 * (t1 + a.tiles1 * t2);  // tile index (stop-test partials)
  const int i10 = t1 * BY + NGHOSTS;
  const int i0 = t0 * 32 + (tid & 31) + NGHOSTS;
  const int i1 = i10 + (tid >> 5);
  const int z0 = t2 * P + NGHOSTS;
  const int N0 = a.N0, top = NGHOSTS + a.Nxx1, Nxx2 = a.Nxx2;
  // element offsets fit in 32 bits (the launcher checks march_fits)
  const unsigned N01 = (unsigned)a.N01, Ntot = (unsigned)a.Ntot;
  const bool once = Nxx2 >= 2 * NGHOSTS;  // i2 indices below wrap at most once
  auto wrapz = [&](int j) -> int {
    if (once) return j < NGHOSTS ? j + Nxx2 : (j >= NGHOSTS + Nxx2 ? j - Nxx2 : j);
    return wrapm(j, Nxx2);
  };
  // the i0/i1 arms of every point of this tile stay off the inner ghost zones
  const bool clear = t0 > 0 && i10 >= 2 * NGHOSTS && i10 + BY + NGHOSTS <= top;
  double r2 = 0.0;
  if (i0 < NGHOSTS + a.Nxx0 && i1 < top) {
    const T* __restrict__ u = a.S;
    const unsigned k2 = (unsigned)(i0 + N0 * i1);
    // at stage 1 the stage input is y_n itself: y_n's uu and vv at a point
    // are its col[] value and its vv
    const bool y_is_s = STAGE == 1 && a.y == a.S;
    // uu along i2 for planes z0-5 .. z0+P+4 (wrapped by 2 pi)
    T col[P + 10];
    if (z0 - 5 >= NGHOSTS && z0 + P + 4 < NGHOSTS + Nxx2) {
      // no plane of the column wraps (uniform over the block)
      const T* pz = u + (k2 + N01 * (unsigned)(z0 - 5));
#pragma unroll
      for (int q = 0; q < P + 10; q++) col[q] = __ldg(pz + q * N01);
    } else {
#pragma unroll
      for (int q = 0; q < P + 10; q++) col[q] = __ldg(u + (k2 + N01 * (unsigned)wrapz(z0 - 5 + q)));
    }
    // PF: every pointwise input of the P planes is loaded before the first
    // store (the stores may alias y_n, so the compiler cannot hoist them).
    T pf[8][P];  // unused (and removed) when !PF
    if (PF) {
#pragma unroll
      for (int p = 0; p < P; p++) {
        const unsigned idx = k2 + N01 * (unsigned)(z0 + p < NGHOSTS + Nxx2 ? z0 + p : z0);
        pf[0][p] = __ldg(a.S + (idx + Ntot));
        pf[1][p] = __ldg(a.aux + (idx + ADD_TIMES_AUUGF * Ntot));
        pf[2][p] = __ldg(a.aux + (idx + PSI_BACKGROUNDGF * Ntot));
        pf[3][p] = __ldg(a.aux + (idx + WAVESPEEDGF * Ntot));
        pf[4][p] = y_is_s ? col[p + 5] : a.y[idx];
        pf[5][p] = y_is_s ? pf[0][p] : a.y[idx + Ntot];
        pf[6][p] = (STAGE == 1) ? (T)0 : a.acc[idx];
        pf[7][p] = (STAGE == 1) ? (T)0 : a.acc[idx + Ntot];
      }
    }
#pragma unroll
    for (int p = 0; p < P; p++) {
      const int i2 = z0 + p;
      if (i2 < NGHOSTS + Nxx2) {
        const unsigned idx = k2 + N01 * (unsigned)i2;
        T s0 = 0, s1 = 0, s00 = 0, s11 = 0, s22 = 0;
        if (clear) {
          // the star's i0/i1 arms at fixed offsets from the point
          const T* pc = u + idx;
#pragma unroll
          for (int k = 1; k <= 5; k++) {
            const T am = __ldg(pc - k), ap = __ldg(pc + k);
            const T bm = __ldg(pc - k * N0), bp = __ldg(pc + k * N0);
            s0 = fma(W<T>::d(k), ap - am, s0);
            s1 = fma(W<T>::d(k), bp - bm, s1);
            s00 = fma(W<T>::e(k), ap + am, s00);
            s11 = fma(W<T>::e(k), bp + bm, s11);
          }
        } else {
          stencil01<T>(a, u, i0, i1, i2, wrap2(i2 + a.half2, Nxx2), s0, s1, s00, s11);
        }
#pragma unroll
        for (int k = 1; k <= 5; k++) s22 = fma(W<T>::e(k), col[p + 5 + k] + col[p + 5 - k], s22);
        T ku, kv, br;
        T yu, yv, accu, accv;
        // the six metric weights, loaded per plane (cached in L1; holding
        // them in registers across the planes costs occupancy)
        const T C22 = __ldg(a.coef + k2), C00 = __ldg(a.coef + (k2 + N01)), C11 = __ldg(a.coef + (k2 + 2 * N01));
        const T C1 = __ldg(a.coef + (k2 + 3 * N01)), C0 = __ldg(a.coef + (k2 + 4 * N01));
        const T Cc = __ldg(a.coef + (k2 + 5 * N01));
        if (PF) {
          point_rhs<T>(col[p + 5], pf[0][p], pf[1][p], pf[2][p], pf[3][p], C22, C00, C11, C1, C0, Cc, s0, s1, s00,
                       s11, s22, a.eta, ku, kv, br);
          yu = pf[4][p];
          yv = pf[5][p];
          accu = pf[6][p];
          accv = pf[7][p];
        } else if (CORR) {
          T ju, jv;
          point_rhs_correction<T>(col[p + 5], __ldg(a.S + (idx + Ntot)), __ldg(a.aux + (idx + ADD_TIMES_AUUGF * Ntot)),
                                  __ldg(a.aux + (idx + PSI_BACKGROUNDGF * Ntot)),
                                  __ldg(a.aux + (idx + WAVESPEEDGF * Ntot)), C22, C00, C11, C1, C0, Cc, s0, s1, s00,
                                  s11, s22, a.eta, __ldg(a.R0 + idx), __ldg(a.R0 + (idx + Ntot)), ku, kv, br, ju, jv);
          accu = (STAGE == 1) ? (T)0 : a.acc[idx];
          accv = (STAGE == 1) ? (T)0 : a.acc[idx + Ntot];
          yu = y_is_s ? col[p + 5] : a.y[idx];
          yv = y_is_s ? __ldg(a.S + (idx + Ntot)) : a.y[idx + Ntot];
        } else {
          point_rhs<T>(col[p + 5], __ldg(a.S + (idx + Ntot)), __ldg(a.aux + (idx + ADD_TIMES_AUUGF * Ntot)),
                       __ldg(a.aux + (idx + PSI_BACKGROUNDGF * Ntot)), __ldg(a.aux + (idx + WAVESPEEDGF * Ntot)), C22,
                       C00, C11, C1, C0, Cc, s0, s1, s00, s11, s22, a.eta, ku, kv, br);
          accu = (STAGE == 1) ? (T)0 : a.acc[idx];
          accv = (STAGE == 1) ? (T)0 : a.acc[idx + Ntot];
          yu = y_is_s ? col[p + 5] : a.y[idx];
          yv = y_is_s ? __ldg(a.S + (idx + Ntot)) : a.y[idx + Ntot];
        }
        // RK combination and stores (store_point's arithmetic, 32-bit offsets)
        T ou, ov;
        rk_combine<T, STAGE>(ku, yu, accu, ou, a.dt);
        rk_combine<T, STAGE>(kv, yv, accv, ov, a.dt);
        if (STAGE != 4) {
          a.acc[idx] = accu;
          a.acc[idx + Ntot] = accv;
        }
        a.out[idx] = ou;
        a.out[idx + Ntot] = ov;
        if (RESID) {
          const double bb = (double)br;
          r2 += bb * bb * __ldg(a.w + k2);
        }
      }
    }
  }
  if (RESID && tile_partial<NT>(r2, b, a.partials, a.ticket, a.n_tiles, sh, &last, a.defer_l2 != 0)) finalize_l2<T, NT>(a, sh);
}

// ------------------------------------------------- planes in shared memory
// Same per-point arithmetic as k_substep, but the block first copies uu on
// its P planes, widened by 5 points along i0 and i1, into shared memory (one
// warp per row; ghost points redirected to their sources only in blocks that
// touch an inner boundary), so the i0 and i1 stencil arms are shared-memory
// reads at compile-time offsets and the per-point integer work is small.
// uu along i2 stays in registers and the pointwise inputs of all P planes are
// loaded before the first store.
// Copies uu on plane i2 of an interior tile, widened by 5 points along i0
// and i1 (rows i10-5 .. i10+BY+4, points i00-5 .. i00+36), into su, one row
// per warp iteration; ghost points are redirected to their sources only in
// tiles that touch an inner boundary (`inner`).
template <typename T, int BY>
__device__ __forceinline__ void stage_plane(const SubDev<T>& a, const T* __restrict__ u, int i00, int i10, int i2,
                                            bool inner, T (*su)[42]) {
  constexpr int RWS = 42, NR = BY + 10;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int N0 = a.N0, top = NGHOSTS + a.Nxx1;
  const int N01 = (int)a.N01;
  for (int r = ty; r < NR; r += BY) {
    const int i1 = i10 - NGHOSTS + r;
    if (i1 >= top + NGHOSTS) continue;  // never read
    if (!inner) {
      const T* src = u + (i00 - NGHOSTS) + N0 * i1 + N01 * i2;
      su[r][tx] = __ldg(src + tx);
      if (tx < RWS - 32 && i00 - NGHOSTS + 32 + tx < N0) su[r][32 + tx] = __ldg(src + 32 + tx);
    } else {
      for (int x = tx; x < RWS; x += 32) {
        int j0 = i00 - NGHOSTS + x, j1 = i1;
        if (j0 >= N0) continue;
        bool flip = false;
        if (j1 < NGHOSTS) {
          j1 = 2 * NGHOSTS - 1 - j1;
          flip = true;
        } else if (j1 >= top) {
          j1 = 2 * top - 1 - j1;
          flip = true;
        }
        if (j0 < NGHOSTS) {
          j0 = 2 * NGHOSTS - 1 - j0;
          flip = !flip;
        }
        const int j2 = flip ? wrap2(i2 + a.half2, a.Nxx2) : i2;
        su[r][x] = __ldg(u + j0 + N0 * j1 + N01 * j2);
      }
    }
  }
}

// Shared memory of the planes kernel, in doubles: the planes of an interior
// block, or the rows of a column block.
template <typename T, int BY, int P>
struct PlanesSmem {
  static constexpr int planes = (P * (BY + 10) * 42 * (int)sizeof(T) + 7) / 8;
  static constexpr int value = planes > kRowsSmem ? planes : kRowsSmem;
};

// Block `bid` of one grid's planes launch (column blocks first).
template <typename T, int STAGE, bool RESID, int BY, int P>
__device__ __forceinline__ void planes_block(const SubDev<T>& a, int bid, double* smem, double* sh, bool* lastp) {
  constexpr int NT = 32 * BY;
  constexpr int RWS = 42;       // i0 = i00-5 .. i00+36
  constexpr int NR = BY + 10;   // i1 = i10-5 .. i10+BY+4
  T(*su)[NR][RWS] = reinterpret_cast<T(*)[NR][RWS]>(smem);
  bool& last = *lastp;
  if (bid < a.n_col_blocks) {
    column_rows<T, STAGE, NT>(a, bid, smem);
    return;
  }
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int b = bid - a.n_col_blocks;
  const int t0 = b % a.tiles0, t1 = (b / a.tiles0) % a.tiles1, t2 = b / (a.tiles0 * a.tiles1);
  const int i00 = t0 * 32 + NGHOSTS, i10 = t1 * BY + NGHOSTS, z0 = t2 * P + NGHOSTS;
  const int N0 = a.N0, top = NGHOSTS + a.Nxx1, zend = NGHOSTS + a.Nxx2;
  const int N01 = (int)a.N01;
  const T* __restrict__ u = a.S;
  // ---- stage the planes
  const bool inner = (t0 == 0) || (i10 < 2 * NGHOSTS) || (i10 + BY + NGHOSTS > top);
  for (int p = 0; p < P; p++)
    if (z0 + p < zend) stage_plane<T, BY>(a, u, i00, i10, z0 + p, inner, su[p]);
  const int i0 = i00 + tx, i1 = i10 + ty;
  const bool valid = i0 < NGHOSTS + a.Nxx0 && i1 < top;
  const int k2 = i0 + N0 * i1;
  T col[P + 10];
  T pf[8][P];
  if (valid) {
    // uu along i2 for planes z0-5 .. z0+P+4 (wrapped by 2 pi)
#pragma unroll
    for (int q = 0; q < P + 10; q++) col[q] = __ldg(u + k2 + N01 * wrap2(z0 - 5 + q, a.Nxx2));
    const long long Ntot = a.Ntot;
#pragma unroll
    for (int p = 0; p < P; p++) {
      const int idx = k2 + N01 * (z0 + p < zend ? z0 + p : z0);
      pf[0][p] = __ldg(a.S + Ntot + idx);
      pf[1][p] = __ldg(a.aux + ADD_TIMES_AUUGF * Ntot + idx);
      pf[2][p] = __ldg(a.aux + PSI_BACKGROUNDGF * Ntot + idx);
      pf[3][p] = __ldg(a.aux + WAVESPEEDGF * Ntot + idx);
      pf[4][p] = a.y[idx];
      pf[5][p] = a.y[Ntot + idx];
      pf[6][p] = (STAGE == 1) ? (T)0 : a.acc[idx];
      pf[7][p] = (STAGE == 1) ? (T)0 : a.acc[Ntot + idx];
    }
  }
  __syncthreads();
  double r2 = 0.0;
  if (valid) {
    const T C22 = __ldg(a.coef + k2), C00 = __ldg(a.coef + N01 + k2), C11 = __ldg(a.coef + 2 * N01 + k2);
    const T C1 = __ldg(a.coef + 3 * N01 + k2), C0 = __ldg(a.coef + 4 * N01 + k2), Cc = __ldg(a.coef + 5 * N01 + k2);
#pragma unroll
    for (int p = 0; p < P; p++) {
      const int i2 = z0 + p;
      if (i2 < zend) {
        const T* sp = &su[p][ty + NGHOSTS][tx + NGHOSTS];
        T s0 = 0, s1 = 0, s00 = 0, s11 = 0, s22 = 0;
#pragma unroll
        for (int k = 1; k <= 5; k++) {
          const T am = sp[-k], ap = sp[k];
          const T bm = sp[-k * RWS], bp = sp[k * RWS];
          s0 = fma(W<T>::d(k), ap - am, s0);
          s1 = fma(W<T>::d(k), bp - bm, s1);
          s00 = fma(W<T>::e(k), ap + am, s00);
          s11 = fma(W<T>::e(k), bp + bm, s11);
        }
#pragma unroll
        for (int k = 1; k <= 5; k++) s22 = fma(W<T>::e(k), col[p + 5 + k] + col[p + 5 - k], s22);
        T ku, kv, br;
        point_rhs<T>(col[p + 5], pf[0][p], pf[1][p], pf[2][p], pf[3][p], C22, C00, C11, C1, C0, Cc, s0, s1, s00, s11,
                     s22, a.eta, ku, kv, br);
        store_point<T, STAGE>(a, k2 + (long long)N01 * i2, ku, kv, pf[4][p], pf[5][p], pf[6][p], pf[7][p]);
        if (RESID) {
          const double bb = (double)br;
          r2 += bb * bb * __ldg(a.w + k2);
        }
      }
    }
  }
  if (RESID && tile_partial<NT>(r2, b, a.partials, a.ticket, a.n_tiles, sh, &last, a.defer_l2 != 0)) finalize_l2<T, NT>(a, sh);
}

template <typename T, int STAGE, bool RESID, int BY, int P>
__global__ void __launch_bounds__(32 * BY) k_substep_planes(SubDev<T> a) {
  __shared__ double smem[PlanesSmem<T, BY, P>::value];
  __shared__ double sh[BY > 8 ? BY : 8];
  __shared__ bool last;
  pdl_enter();
  if (*a.done) return;
  planes_block<T, STAGE, RESID, BY, P>(a, blockIdx.x, smem, sh, &last);
}

// One substep of many grids in one launch: the blocks of grid c are
// offs[c] .. offs[c+1]-1 (column blocks first, then interior tiles), each
// grid with its own launch arguments, stop test and done flag.
template <typename T, int STAGE, bool RESID, int BY, int P>
__global__ void __launch_bounds__(32 * BY)
    k_substep_planes_batch(const SubDev<T>* __restrict__ devs, const int* __restrict__ offs, int n) {
  __shared__ double smem[PlanesSmem<T, BY, P>::value];
  __shared__ double sh[BY > 8 ? BY : 8];
  __shared__ bool last;
  pdl_enter();
  int lo = 0, hi = n - 1;
  const int bx = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(offs + mid) <= bx)
      lo = mid;
    else
      hi = mid - 1;
  }
  const SubDev<T>& a = devs[lo];
  if (*a.done) return;
  planes_block<T, STAGE, RESID, BY, P>(a, bx - __ldg(offs + lo), smem, sh, &last);
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

// kind 0: direct; 2: direct with the pointwise inputs of all P planes loaded
// up front; 4: planes in shared memory (its column blocks by rows,
// column_rows); 5: marching along i2 with asynchronous copies
// (kernels_march.cu), p planes per block, v the index of its compiled shape
// there.
struct TileShape {
  int by, p, kind, v;
};
static const TileShape kTiles[] = {{4, 1, 0, 0}, {4, 2, 0, 0}, {2, 4, 0, 0}, {8, 1, 0, 0}, {8, 2, 0, 0},
                                   {4, 4, 0, 0}, {4, 1, 2, 0}, {4, 2, 2, 0}, {2, 4, 2, 0}, {4, 4, 2, 0},
                                   {8, 2, 2, 0}, {4, 2, 4, 0}, {4, 4, 4, 0}, {8, 2, 4, 0}, {2, 4, 4, 0},
                                   {8, 1, 4, 0}, {4, 1, 4, 0}, {8, 4, 4, 0}, {8, 8, 5, 0}, {8, 16, 5, 1},
                                   {8, 4, 5, 2}, {8, 4, 5, 3}, {8, 8, 5, 4}, {8, 32, 5, 5}, {8, 4, 5, 6}};
constexpr int kNumTiles = sizeof(kTiles) / sizeof(kTiles[0]);

int substep_num_tiles() { return kNumTiles; }
void substep_tile_shape(int tile, int* bx, int* by, int* p) {
  *bx = 32;
  *by = kTiles[tile].by;
  *p = kTiles[tile].p;
}
int substep_tile_kind(int tile) { return kTiles[tile].kind; }

int substep_interior_blocks(const Dims& d, int tile) {
  const TileShape s = kTiles[tile];
  // marching shapes: at most one block per (column tile, plane) whatever the
  // split of the planes into chunks
  if (s.kind == 5) return ((d.Nxx0 + 31) / 32) * ((d.Nxx1 + s.by - 1) / s.by) * d.Nxx2;
  return ((d.Nxx0 + 31) / 32) * ((d.Nxx1 + s.by - 1) / s.by) * ((d.Nxx2 + s.p - 1) / s.p);
}

template <typename T, int STAGE, bool RESID, int BY, int P>
static void launch_planes(const SubstepArgs& a);

template <typename T, int STAGE, bool RESID, int BY, int P, bool PF, bool CORR = false,
          int MINB = PF ? 1 : (P == 1 ? 32 / BY : (BY == 8 && P == 2 ? 3 : 1))>
static void launch_direct(const SubstepArgs& a) {
  if (!march_fits(a.d)) {  // 64-bit offsets: the planes kernel
    if (CORR) {
      NRPYELL_FAIL("launch_direct: the correction form needs 3 Ntot < 2^32");
      return;
    }
    launch_planes<T, STAGE, RESID, 8, 1>(a);
    return;
  }
  SubDev<T> f = make_dev<T>(a, BY, P);
  constexpr int NT = 32 * BY;
  constexpr int CB = NT / kColThreadsPerColumn;
  f.n_col_blocks = NT >= 256 ? ((a.d.Nxx1 + kRows - 1) / kRows) * a.d.Nxx2 : (f.ncol + CB - 1) / CB;
  const int plane = f.tiles0 * f.tiles1;
  f.ncz = (f.n_col_blocks + plane - 1) / plane;
  const dim3 grid(f.tiles0, f.tiles1, f.ncz + f.tiles2);
  NRPYELL_LAUNCH_PDL((k_substep<T, STAGE, RESID, BY, P, PF, CORR, MINB>), grid, NT, 0, f);
}

template <typename T, int STAGE, bool RESID, int BY, int P>
static void launch_planes(const SubstepArgs& a) {
  SubDev<T> f = make_dev<T>(a, BY, P);
  constexpr int NT = 32 * BY;
  f.n_col_blocks = ((a.d.Nxx1 + kRows - 1) / kRows) * a.d.Nxx2;
  NRPYELL_LAUNCH_PDL((k_substep_planes<T, STAGE, RESID, BY, P>), f.n_tiles + f.n_col_blocks, NT, 0, f);
}

static cudaEvent_t g_fin_fork = nullptr, g_fin_join = nullptr;

void prepare_columns() {
  side_stream();
  if (!g_fin_fork) {
    NRPYELL_CUDA(cudaEventCreateWithFlags(&g_fin_fork, cudaEventDisableTiming));
    NRPYELL_CUDA(cudaEventCreateWithFlags(&g_fin_join, cudaEventDisableTiming));
  }
}

// The stop test of a deferred stage-1 launch (tile_partial with defer): one
// block sums the per-tile partials in index order (finalize_l2).
template <typename T>
__global__ void __launch_bounds__(256) k_finalize_l2(SubDev<T> a) {
  __shared__ double sh[8];
  if (*a.done) return;
  finalize_l2<T, 256>(a, sh);
}

template <typename T>
void launch_finalize_forked(const SubstepArgs& a1) {
  prepare_columns();
  // the tile grid of the stage-1 launch, as launch_tile chose it: the
  // 32-bit-offset kernels (direct, marching) run the planes 32x8x1 shape on
  // grids too large for them
  const TileShape s = kTiles[a1.tile];
  const bool fits = march_fits(a1.d);
  int by = s.by, p = s.p;
  if (!fits && s.kind != 4) {
    by = 8;
    p = 1;
  }
  SubDev<T> f = make_dev<T>(a1, by, p);
  if (s.kind == 5 && fits) f.n_tiles = march_interior_blocks<T>(s.v, a1);
  cudaStream_t side = side_stream();
  NRPYELL_CUDA(cudaEventRecord(g_fin_fork, stream()));
  NRPYELL_CUDA(cudaStreamWaitEvent(side, g_fin_fork, 0));
  NRPYELL_LAUNCH_ON(side, (k_finalize_l2<T>), 1, 256, 0, f);
  NRPYELL_CUDA(cudaEventRecord(g_fin_join, side));
}
template void launch_finalize_forked<double>(const SubstepArgs&);
template void launch_finalize_forked<float>(const SubstepArgs&);

void join_finalize() { NRPYELL_CUDA(cudaStreamWaitEvent(stream(), g_fin_join, 0)); }

template <typename T>
void prepare_substep(int tile) {
  if (kTiles[tile].kind == 5) prepare_march<T>(kTiles[tile].v);
  prepare_columns();  // side stream and events of the stop test
}
template void prepare_substep<double>(int);
template void prepare_substep<float>(int);

template <typename T, int STAGE, bool RESID>
static void launch_tile(const SubstepArgs& a) {
  switch (a.tile) {
    case 0: launch_direct<T, STAGE, RESID, 4, 1, false>(a); break;
    case 1: launch_direct<T, STAGE, RESID, 4, 2, false>(a); break;
    case 2: launch_direct<T, STAGE, RESID, 2, 4, false>(a); break;
    case 3: launch_direct<T, STAGE, RESID, 8, 1, false>(a); break;
    case 4: launch_direct<T, STAGE, RESID, 8, 2, false>(a); break;
    case 5: launch_direct<T, STAGE, RESID, 4, 4, false>(a); break;
    case 6: launch_direct<T, STAGE, RESID, 4, 1, true>(a); break;
    case 7: launch_direct<T, STAGE, RESID, 4, 2, true>(a); break;
    case 8: launch_direct<T, STAGE, RESID, 2, 4, true>(a); break;
    case 9: launch_direct<T, STAGE, RESID, 4, 4, true>(a); break;
    case 10: launch_direct<T, STAGE, RESID, 8, 2, true>(a); break;
    case 11: launch_planes<T, STAGE, RESID, 4, 2>(a); break;
    case 12: launch_planes<T, STAGE, RESID, 4, 4>(a); break;
    case 13: launch_planes<T, STAGE, RESID, 8, 2>(a); break;
    case 14: launch_planes<T, STAGE, RESID, 2, 4>(a); break;
    case 15: launch_planes<T, STAGE, RESID, 8, 1>(a); break;
    case 16: launch_planes<T, STAGE, RESID, 4, 1>(a); break;
    case 17: launch_planes<T, STAGE, RESID, 8, 4>(a); break;
    case 18:
    case 19:
    case 20:
    case 21:
    case 22:
    case 23:
    case 24:
      if (!launch_march<T>(STAGE, RESID, kTiles[a.tile].v, a)) launch_planes<T, STAGE, RESID, 8, 1>(a);
      break;
    default: NRPYELL_FAIL("launch_substep: tile index out of range"); break;
  }
}

// Shapes that run the correction form: the marching shapes and the 8-warp
// direct shapes without prefetch (32 x 8 x 1, 32 x 8 x 2).
bool substep_supports_correction(int tile) {
  return tile >= 0 && tile < kNumTiles && (kTiles[tile].kind == 5 || tile == 3 || tile == 4);
}

template <typename T, int STAGE, bool RESID>
static void launch_direct_correction(const SubstepArgs& a) {
  if constexpr (sizeof(T) == 4) {
    if (a.tile == 3)
      launch_direct<T, STAGE, RESID, 8, 1, false, true>(a);
    else
      launch_direct<T, STAGE, RESID, 8, 2, false, true>(a);
  }
}

template <typename T>
void launch_substep(int stage, const SubstepArgs& a) {
  if (a.R0 && (sizeof(T) != 4 || !substep_supports_correction(a.tile))) {
    NRPYELL_FAIL("launch_substep: the correction form runs on FP32 marching and 8-warp direct shapes only");
    return;
  }
  const bool resid = (stage == 1) && a.lt;
  if (a.R0 && kTiles[a.tile].kind != 5) {
    switch (stage) {
      case 1:
        if (resid)
          launch_direct_correction<T, 1, true>(a);
        else
          launch_direct_correction<T, 1, false>(a);
        break;
      case 2: launch_direct_correction<T, 2, false>(a); break;
      case 3: launch_direct_correction<T, 3, false>(a); break;
      default: launch_direct_correction<T, 4, false>(a); break;
    }
    return;
  }
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

// ---------------------------------------------------------------- batches

template <typename T>
bool batch_launch_dev(const SubstepArgs& a, SubDev<T>* out) {
  const int t = a.tile;
  if (t < 0 || t >= kNumTiles || (kTiles[t].kind != 4 && kTiles[t].kind != 5)) {
    NRPYELL_FAIL("batched substep: the tile must be a shared-memory planes or marching shape");
    return false;
  }
  if (kTiles[t].kind == 5 && !march_fits(a.d)) {
    NRPYELL_FAIL("batched substep: a grid is too large for the marching shapes (3 Ntot >= 2^32)");
    return false;
  }
  *out = make_dev<T>(a, kTiles[t].by, kTiles[t].p);
  out->n_col_blocks = ((a.d.Nxx1 + kRows - 1) / kRows) * a.d.Nxx2;
  return true;
}
template bool batch_launch_dev<double>(const SubstepArgs&, SubDev<double>*);
template bool batch_launch_dev<float>(const SubstepArgs&, SubDev<float>*);

template <typename T, int STAGE, bool RESID>
static void launch_batch_stage(int tile, const SubDev<T>* devs, const int* offs, int n, int blocks) {
  const int by = kTiles[tile].by, p = kTiles[tile].p;
#define NRPYELL_BATCH(BY, P)                                                                           \
  if (by == BY && p == P) {                                                                            \
    NRPYELL_LAUNCH_PDL((k_substep_planes_batch<T, STAGE, RESID, BY, P>), blocks, 32 * BY, 0, devs, offs, n); \
    return;                                                                                            \
  }
  NRPYELL_BATCH(4, 2)
  NRPYELL_BATCH(4, 4)
  NRPYELL_BATCH(8, 2)
  NRPYELL_BATCH(2, 4)
  NRPYELL_BATCH(8, 1)
  NRPYELL_BATCH(4, 1)
  NRPYELL_BATCH(8, 4)
#undef NRPYELL_BATCH
  NRPYELL_FAIL("batched substep: no kernel for this tile shape");
}

template <typename T>
void launch_substep_batch(int stage, bool resid, int tile, const SubDev<T>* devs, const int* offs, int n, int blocks,
                          bool corr) {
  if (kTiles[tile].kind == 5) {  // batch_launch_dev checked march_fits for every grid
    launch_march_batch<T>(stage, resid, kTiles[tile].v, devs, offs, n, blocks, corr);
    return;
  }
  if (corr || sizeof(T) != 8) {
    NRPYELL_FAIL("batched substep: FP32 and the correction form run on the marching shapes only");
    return;
  }
  if constexpr (sizeof(T) == 8) {
    switch (stage) {
      case 1:
        if (resid)
          launch_batch_stage<T, 1, true>(tile, devs, offs, n, blocks);
        else
          launch_batch_stage<T, 1, false>(tile, devs, offs, n, blocks);
        break;
      case 2: launch_batch_stage<T, 2, false>(tile, devs, offs, n, blocks); break;
      case 3: launch_batch_stage<T, 3, false>(tile, devs, offs, n, blocks); break;
      default: launch_batch_stage<T, 4, false>(tile, devs, offs, n, blocks); break;
    }
  }
}
template void launch_substep_batch<double>(int, bool, int, const SubDev<double>*, const int*, int, int, bool);
template void launch_substep_batch<float>(int, bool, int, const SubDev<float>*, const int*, int, int, bool);

template <typename T>
void launch_ghost_fill(const Dims& d, const BcTables* bt, void* gfs) {
  if (bt->n_inner <= 0) return;
  NRPYELL_LAUNCH((k_ghost_fill<T>), (bt->n_inner + 255) / 256, 256, 0, bt->inner, bt->inner_par, bt->n_inner, d.Ntot,
                 (T*)gfs);
}
template void launch_ghost_fill<double>(const Dims&, const BcTables*, void*);
template void launch_ghost_fill<float>(const Dims&, const BcTables*, void*);

}  // namespace nrpyell
