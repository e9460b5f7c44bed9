// Fused RK4 substep, TMA pipeline variant (FP64).
//
// The interior part of a substep (RHS of MoL_step_forward_in_time.c's
// rhs_eval into the RK combination, plus the stage-1 residual L2) runs as a
// persistent kernel, one CTA per SM, each CTA looping over tiles of
// 32 (i0) x BY (i1) x P (i2) points.  In each CTA one producer warp moves
// what a tile needs from global into shared memory with the tensor memory
// accelerator -- cp.async.bulk.tensor boxes described by tensor maps, their
// completion counted in bytes on an mbarrier -- NS tiles ahead of the
// consumer warps, which compute from shared memory and store the RK outputs.
// A tile takes about 27 box copies, so the copy engine keeps tens of KB per
// SM in flight while the consumers spend their instructions on arithmetic.
//
// A tile stage holds:
//   F  the pointwise fields (vv, ADD_times_AUU, psi_background, wavespeed,
//      y_n uu/vv, and at stages 2-4 the running total uu/vv): 4 boxes;
//   C  the six folded metric weights of the tile's (i0,i1) columns: 1 box;
//   U  uu over the tile widened by 5 points along i0 (the i0 stencil arms);
//   SD at the i0 = 0 tile: the images of the inner ghost points i0 < 5,
//      the points (9-i0, i1, i2+pi) for i0' = 9-i0 in 5..9;
//   Y  uu on the 5 rows below and above the tile along i1, one box per row;
//      rows across the axis are the reflected rows with i2 shifted by pi;
//   Z  uu on the 5 planes below and above the tile along i2 (wrapped by
//      2 pi), one box per plane.
// Boxes start at an even i0 (16-byte aligned, as TMA requires), so rows are
// read from i00-1 (F, C, Y, Z), i00-5 (U) or 4 (SD); this needs an even row
// length N0 and 16-byte aligned arrays (checked on the host, otherwise the
// direct kernel runs).  Tiles that run past the interior along i1 or i2 (grid
// sizes that the tile does not divide) and pieces whose source planes wrap
// inside a box fall back to one plain bulk copy per row.
//
// The radiation-BC columns of the x0max face run as a separate small kernel
// on a second stream, concurrently with the persistent interior kernel, and
// join back before the next substep.
//
// Every wait is bounded: after about two seconds a waiting warp records an
// error code in *err and leaves its loop, so a broken pipeline ends the
// kernel instead of hanging the GPU.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <vector>

#include "substep.cuh"

namespace nrpyell {

namespace {

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits until the phase of bar with the given parity has completed; false
// after about kWaitCycles SM clock cycles.
constexpr long long kWaitCycles = 4000000000LL;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}
// Plain bulk copy: 16-byte aligned addresses, size a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Tensor box copies; x (innermost, elements) must be even for FP64.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_addr(dst)),
      "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(smem_addr(dst)),
      "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_addr(bar))
      : "memory");
}

}  // namespace

// Tensor maps of one launch (boxes in elements, innermost first).
struct BulkMaps {
  CUtensorMap vv;    // S as (N0, N1, N2, 2): box (34, BY, P, 1) at gf 1
  CUtensorMap aux;   // auxevol (N0, N1, N2, 3): box (34, BY, P, 3)
  CUtensorMap y;     // y_n (N0, N1, N2, 2): box (34, BY, P, 2)
  CUtensorMap acc;   // running total (N0, N1, N2, 2): box (34, BY, P, 2)
  CUtensorMap coef;  // folded weights (N0, N1, 6): box (34, BY, 6)
  CUtensorMap U;     // S gf 0 (N0, N1, N2): box (42, BY, P)
  CUtensorMap Yh;    // S gf 0: box (34, 1, P)
  CUtensorMap Zh;    // S gf 0: box (34, BY, 1)
  CUtensorMap SD;    // S gf 0: box (6, BY, P)
};

// Element offsets (doubles) within one tile stage.  Every box destination is
// 128-byte aligned (offsets multiples of 16 doubles); rows inside a box are
// dense, so row strides are the box widths.
template <int BY, int P, int NF>
struct BulkLayout {
  static constexpr int r16(int n) { return (n + 15) & ~15; }
  static constexpr int RW = 34;  // F, C, Y, Z rows: i0 = i00-1 .. i00+32
  static constexpr int UW = 42;  // U rows: i0 = i00-5 .. i00+36
  static constexpr int SW = 6;   // SD rows: i0 = 4 .. 9
  static constexpr int FB = P * BY * RW;  // one field
  static constexpr int YS = r16(P * RW);  // one i1 halo row over the P planes
  static constexpr int ZS = r16(BY * RW);  // one i2 halo plane over the BY rows
  static constexpr int F = 0;
  static constexpr int C = r16(F + NF * FB);
  static constexpr int U = r16(C + 6 * BY * RW);
  static constexpr int SD = r16(U + P * BY * UW);
  static constexpr int Y = r16(SD + P * BY * SW);
  static constexpr int Z = Y + 10 * YS;
  static constexpr int SIZE = r16(Z + 10 * ZS);
  static_assert(FB % 16 == 0, "a field block must keep the next box 128-byte aligned");
  // row slots of the per-row path, in the order it enumerates them
  static constexpr int R_F = 0;
  static constexpr int R_C = R_F + NF * P * BY;
  static constexpr int R_U = R_C + 6 * BY;
  static constexpr int R_SD = R_U + P * BY;
  static constexpr int R_Y = R_SD + P * BY;
  static constexpr int R_Z = R_Y + P * 10;
  static constexpr int ROWS = R_Z + 10 * BY;
};

template <int STAGE>
struct BulkFields {
  static constexpr int value = STAGE == 1 ? 6 : 8;
};

struct TileGeom {
  int t0, i00, i10, z0;
  int n0;  // interior points of the tile along i0
};

__device__ __forceinline__ TileGeom tile_geom(const SubDev<double>& a, int tile, int BY, int P) {
  TileGeom g;
  g.t0 = tile % a.tiles0;
  const int t1 = (tile / a.tiles0) % a.tiles1, t2 = tile / (a.tiles0 * a.tiles1);
  g.i00 = NGHOSTS + 32 * g.t0;
  g.i10 = NGHOSTS + BY * t1;
  g.z0 = NGHOSTS + P * t2;
  g.n0 = min(32, NGHOSTS + a.Nxx0 - g.i00);
  return g;
}

// Source row (i1s, i2s) of uu at (., i1, i2) for i1 in [0, N1) and any i2:
// i1 outside the interior is reflected across the axis with i2 shifted by
// pi; i2 is wrapped by 2 pi.
__device__ __forceinline__ void uu_src_row(const SubDev<double>& a, int i1, int i2, int& i1s, int& i2s) {
  const int top = NGHOSTS + a.Nxx1;
  bool flip = false;
  if (i1 < NGHOSTS) {
    i1 = 2 * NGHOSTS - 1 - i1;
    flip = true;
  } else if (i1 >= top) {
    i1 = 2 * top - 1 - i1;
    flip = true;
  }
  i1s = i1;
  i2s = wrapm(i2 + (flip ? a.half2 : 0), a.Nxx2);
}

__device__ __forceinline__ long long row_off(const SubDev<double>& a, int i1, int i2) {
  return (long long)a.N0 * i1 + a.N01 * i2;
}

// Per-row path: row slot r of a tile -> source, destination (element offset
// in the stage) and length in elements; false if the tile does not need it.
template <int BY, int P, int NF>
__device__ __forceinline__ bool bulk_row(const SubDev<double>& a, const TileGeom& g, int r, const double*& src,
                                         int& dst, int& n) {
  using L = BulkLayout<BY, P, NF>;
  const int top = NGHOSTS + a.Nxx1, zend = NGHOSTS + a.Nxx2;
  const int nrow = (g.n0 + 2) & ~1;  // i00-1 .. i00+n0-1, rounded up to an even count
  int i1s, i2s;
  if (r < L::R_C) {
    const int f = r / (P * BY), rem = r % (P * BY), p = rem / BY, y = rem % BY;
    const int i1 = g.i10 + y, i2 = g.z0 + p;
    if (i1 >= top || i2 >= zend) return false;
    const double* base;
    switch (f) {
      case 0: base = a.S + a.Ntot; break;
      case 1: base = a.aux + ADD_TIMES_AUUGF * a.Ntot; break;
      case 2: base = a.aux + PSI_BACKGROUNDGF * a.Ntot; break;
      case 3: base = a.aux + WAVESPEEDGF * a.Ntot; break;
      case 4: base = a.y; break;
      case 5: base = a.y + a.Ntot; break;
      case 6: base = a.acc; break;
      default: base = a.acc + a.Ntot; break;
    }
    src = base + row_off(a, i1, i2) + (g.i00 - 1);
    dst = L::F + r * L::RW;
    n = nrow;
    return true;
  }
  if (r < L::R_U) {
    const int c = (r - L::R_C) / BY, y = (r - L::R_C) % BY;
    const int i1 = g.i10 + y;
    if (i1 >= top) return false;
    src = a.coef + c * a.N01 + (long long)a.N0 * i1 + (g.i00 - 1);
    dst = L::C + (r - L::R_C) * L::RW;
    n = nrow;
    return true;
  }
  if (r < L::R_SD) {
    const int q = r - L::R_U, p = q / BY, y = q % BY;
    const int i1 = g.i10 + y;
    if (i1 >= top + NGHOSTS) return false;
    uu_src_row(a, i1, g.z0 + p, i1s, i2s);
    src = a.S + row_off(a, i1s, i2s) + (g.i00 - NGHOSTS);
    dst = L::U + q * L::UW;
    n = min(L::UW, a.N0 - (g.i00 - NGHOSTS));
    return true;
  }
  if (r < L::R_Y) {
    const int q = r - L::R_SD, p = q / BY, y = q % BY;
    const int i1 = g.i10 + y, i2 = g.z0 + p;
    if (g.t0 != 0 || i1 >= top || i2 >= zend) return false;
    src = a.S + row_off(a, i1, wrap2(i2 + a.half2, a.Nxx2)) + 4;
    dst = L::SD + q * L::SW;
    n = L::SW;
    return true;
  }
  if (r < L::R_Z) {
    const int q = r - L::R_Y, p = q / 10, h = q % 10;
    const int j1 = (h < 5) ? g.i10 - 5 + h : g.i10 + BY + h - 5;
    const int i2 = g.z0 + p;
    if (i2 >= zend || j1 >= top + NGHOSTS) return false;
    uu_src_row(a, j1, i2, i1s, i2s);
    src = a.S + row_off(a, i1s, i2s) + (g.i00 - 1);
    dst = L::Y + h * L::YS + p * L::RW;
    n = nrow;
    return true;
  }
  {
    const int q = r - L::R_Z, h = q / BY, y = q % BY;
    const int i1 = g.i10 + y;
    const int j2 = (h < 5) ? g.z0 - 5 + h : g.z0 + P + h - 5;
    if (i1 >= top) return false;
    src = a.S + row_off(a, i1, wrapm(j2, a.Nxx2)) + (g.i00 - 1);
    dst = L::Z + h * L::ZS + y * L::RW;
    n = nrow;
    return true;
  }
}

// Box path of a tile that lies inside the interior along i1 and i2: lane
// `job` issues its copies and returns their bytes.  Jobs: 0-3 the field
// boxes, 4 the weights, 5 uu, 6 the ghost side (i0 = 0 tiles), 7-16 the i1
// halo rows, 17-26 the i2 halo planes.
template <int BY, int P, int NF>
__device__ __forceinline__ unsigned tile_boxes(const SubDev<double>& a, const BulkMaps& m, const TileGeom& g, int job,
                                               double* stage, unsigned long long* bar, bool issue) {
  using L = BulkLayout<BY, P, NF>;
  constexpr unsigned FBYTES = 8u * L::FB;
  const int zend = NGHOSTS + a.Nxx2, top = NGHOSTS + a.Nxx1;
  const int x = g.i00 - 1;
  switch (job) {
    case 0:
      if (issue) tma_load_4d(stage + L::F, &m.vv, x, g.i10, g.z0, 1, bar);
      return FBYTES;
    case 1:
      if (issue) tma_load_4d(stage + L::F + L::FB, &m.aux, x, g.i10, g.z0, 0, bar);
      return 3 * FBYTES;
    case 2:
      if (issue) tma_load_4d(stage + L::F + 4 * L::FB, &m.y, x, g.i10, g.z0, 0, bar);
      return 2 * FBYTES;
    case 3:
      if (NF < 8) return 0;
      if (issue) tma_load_4d(stage + L::F + 6 * L::FB, &m.acc, x, g.i10, g.z0, 0, bar);
      return 2 * FBYTES;
    case 4:
      if (issue) tma_load_3d(stage + L::C, &m.coef, x, g.i10, 0, bar);
      return 8u * 6 * BY * L::RW;
    case 5:
      if (issue) tma_load_3d(stage + L::U, &m.U, g.i00 - NGHOSTS, g.i10, g.z0, bar);
      return 8u * P * BY * L::UW;
    case 6: {
      if (g.t0 != 0) return 0;
      const int zh = wrap2(g.z0 + a.half2, a.Nxx2);
      if (zh + P <= zend) {
        if (issue) tma_load_3d(stage + L::SD, &m.SD, 4, g.i10, zh, bar);
      } else if (issue) {
        for (int p = 0; p < P; p++)
          for (int y = 0; y < BY; y++)
            bulk_load(stage + L::SD + (p * BY + y) * L::SW,
                      a.S + row_off(a, g.i10 + y, wrap2(g.z0 + p + a.half2, a.Nxx2)) + 4, 8u * L::SW, bar);
      }
      return 8u * P * BY * L::SW;
    }
    default:
      break;
  }
  if (job < 17) {
    const int h = job - 7;
    const int j1 = (h < 5) ? g.i10 - 5 + h : g.i10 + BY + h - 5;
    if (j1 >= top + NGHOSTS) return 0;
    int j1s, zs;
    uu_src_row(a, j1, g.z0, j1s, zs);
    double* d = stage + L::Y + h * L::YS;
    if (zs + P <= zend) {
      if (issue) tma_load_3d(d, &m.Yh, x, j1s, zs, bar);
      return 8u * P * L::RW;
    }
    // the source planes wrap inside the box: one row per plane
    const int nrow = (g.n0 + 2) & ~1;
    if (issue)
      for (int p = 0; p < P; p++) {
        int a1, a2;
        uu_src_row(a, j1, g.z0 + p, a1, a2);
        bulk_load(d + p * L::RW, a.S + row_off(a, a1, a2) + x, 8u * nrow, bar);
      }
    return 8u * P * nrow;
  }
  if (job < 27) {
    const int h = job - 17;
    const int j2 = wrapm((h < 5) ? g.z0 - 5 + h : g.z0 + P + h - 5, a.Nxx2);
    if (issue) tma_load_3d(stage + L::Z + h * L::ZS, &m.Zh, x, g.i10, j2, bar);
    return 8u * BY * L::RW;
  }
  return 0;
}

template <int STAGE, bool RESID, int BY, int P, int NS, int NCW>
__global__ void __launch_bounds__(32 * (NCW + 1), 1)
    k_substep_bulk(SubDev<double> a, const __grid_constant__ BulkMaps m) {
  constexpr int NF = BulkFields<STAGE>::value;
  constexpr int NCT = 32 * NCW;  // consumer threads
  using L = BulkLayout<BY, P, NF>;
  extern __shared__ __align__(128) double smem_bulk[];
  __shared__ __align__(8) unsigned long long full[NS], empty[NS];
  __shared__ double sh[NCW > 8 ? NCW : 8];
  __shared__ bool last;
  if (*a.done) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < NS; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCT);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  const int top = NGHOSTS + a.Nxx1, zend = NGHOSTS + a.Nxx2;

  if (warp == NCW) {
    // ---------------------------------------------------------- producer
    constexpr int RPL = (L::ROWS + 31) / 32;  // per-row path: rows per lane
    int it = 0;
    for (int tile = blockIdx.x; tile < a.n_tiles; tile += gridDim.x, it++) {
      const int s = it % NS;
      if (it >= NS && !mbar_wait(&empty[s], ((it / NS) - 1) & 1)) {
        atomicExch(a.err, 2);
        break;
      }
      const TileGeom g = tile_geom(a, tile, BY, P);
      double* stage = smem_bulk + s * L::SIZE;
      const bool boxes = g.i10 + BY <= top && g.z0 + P <= zend;
      unsigned bytes = 0;
      if (boxes) {
        bytes = tile_boxes<BY, P, NF>(a, m, g, lane, stage, &full[s], false);
      } else {
        for (int j = 0; j < RPL; j++) {
          const int r = lane + 32 * j;
          const double* src;
          int dst, n;
          if (r < L::ROWS && bulk_row<BY, P, NF>(a, g, r, src, dst, n)) bytes += 8u * n;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
      if (lane == 0) mbar_arrive_expect_tx(&full[s], bytes);
      __syncwarp();
      if (boxes) {
        tile_boxes<BY, P, NF>(a, m, g, lane, stage, &full[s], true);
      } else {
        for (int j = 0; j < RPL; j++) {
          const int r = lane + 32 * j;
          const double* src;
          int dst, n;
          if (r < L::ROWS && bulk_row<BY, P, NF>(a, g, r, src, dst, n))
            bulk_load(stage + dst, src, 8u * n, &full[s]);
        }
      }
    }
    return;
  }

  // ------------------------------------------------------------ consumers
  int it = 0;
  for (int tile = blockIdx.x; tile < a.n_tiles; tile += gridDim.x, it++) {
    const int s = it % NS;
    if (!mbar_wait(&full[s], (it / NS) & 1)) {
      atomicExch(a.err, 1);
      break;
    }
    const TileGeom g = tile_geom(a, tile, BY, P);
    const double* B = smem_bulk + s * L::SIZE;
    const int tx = lane;
    const int i0 = g.i00 + tx;
    double r2 = 0.0;
    for (int item = warp; item < BY * P; item += NCW) {
      const int ty = item % BY, p = item / BY;
      const int i1 = g.i10 + ty, i2 = g.z0 + p;
      if (i0 >= NGHOSTS + a.Nxx0 || i1 >= top || i2 >= zend) continue;
      const int row = p * BY + ty;
      const double* Uc = B + L::U + row * L::UW + NGHOSTS + tx;
      const double c = Uc[0];
      double s0 = 0, s1 = 0, s00 = 0, s11 = 0, s22 = 0;
#pragma unroll
      for (int k = 1; k <= 5; k++) {
        const double am = (g.t0 == 0 && tx < k) ? B[L::SD + row * L::SW + (k - tx)] : Uc[-k];
        const double ap = Uc[k];
        const int ym = ty - k, yp = ty + k;
        const double bm = (ym >= 0) ? B[L::U + (p * BY + ym) * L::UW + NGHOSTS + tx]
                                    : B[L::Y + (5 + ym) * L::YS + p * L::RW + 1 + tx];
        const double bp = (yp < BY) ? B[L::U + (p * BY + yp) * L::UW + NGHOSTS + tx]
                                    : B[L::Y + (5 + yp - BY) * L::YS + p * L::RW + 1 + tx];
        s0 = fma(W<double>::d(k), ap - am, s0);
        s1 = fma(W<double>::d(k), bp - bm, s1);
        s00 = fma(W<double>::e(k), ap + am, s00);
        s11 = fma(W<double>::e(k), bp + bm, s11);
      }
#pragma unroll
      for (int k = 1; k <= 5; k++) {
        const int zm = p - k, zp = p + k;
        const double cm = (zm >= 0) ? B[L::U + (zm * BY + ty) * L::UW + NGHOSTS + tx]
                                    : B[L::Z + (5 + zm) * L::ZS + ty * L::RW + 1 + tx];
        const double cp = (zp < P) ? B[L::U + (zp * BY + ty) * L::UW + NGHOSTS + tx]
                                   : B[L::Z + (5 + zp - P) * L::ZS + ty * L::RW + 1 + tx];
        s22 = fma(W<double>::e(k), cp + cm, s22);
      }
      const double* Fp = B + L::F + row * L::RW + 1 + tx;  // field f at Fp[f * FB]
      constexpr int FB = L::FB;
      const double* Cp = B + L::C + ty * L::RW + 1 + tx;  // weight c at Cp[c * BY * RW]
      constexpr int CS = BY * L::RW;
      double ku, kv, br;
      point_rhs<double>(c, Fp[0], Fp[FB], Fp[2 * FB], Fp[3 * FB], Cp[0], Cp[CS], Cp[2 * CS], Cp[3 * CS], Cp[4 * CS],
                        Cp[5 * CS], s0, s1, s00, s11, s22, a.eta, ku, kv, br);
      const double accu = (NF == 8) ? Fp[6 * FB] : 0.0;
      const double accv = (NF == 8) ? Fp[7 * FB] : 0.0;
      const long long idx = i0 + (long long)a.N0 * i1 + a.N01 * i2;
      store_point<double, STAGE>(a, idx, ku, kv, Fp[4 * FB], Fp[5 * FB], accu, accv);
      if (RESID) r2 += br * br * __ldg(a.w + i0 + a.N0 * i1);
    }
    // every consumer thread releases the stage after its last shared read
    mbar_arrive(&empty[s]);
    if (RESID) {
      if (tile_partial<NCT, NamedSync<1, NCT>>(r2, tile, a.partials, a.ticket, a.n_tiles, sh, &last, a.defer_l2 != 0))
        finalize_l2<double, NCT, NamedSync<1, NCT>>(a, sh);
    }
  }
}

// ---------------------------------------------------------------- host

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    NRPYELL_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p) {
      NRPYELL_FAIL("cuTensorMapEncodeTiled is not available from the driver");
      return nullptr;
    }
    fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

struct MapKey {
  const void* base;
  int rank;
  unsigned long long dims[4];
  unsigned box[4];
};
struct MapEntry {
  MapKey key;
  CUtensorMap map;
};
std::vector<MapEntry> g_maps;

// FP64 tensor map over base with dims (innermost first) and the layout of a
// gridfunction array: strides N0, N0*N1, N0*N1*N2 elements.
bool tensor_map(CUtensorMap* out, const void* base, int rank, const unsigned long long* dims, const unsigned* box) {
  MapKey k;
  memset(&k, 0, sizeof(k));
  k.base = base;
  k.rank = rank;
  for (int i = 0; i < rank; i++) {
    k.dims[i] = dims[i];
    k.box[i] = box[i];
  }
  for (const MapEntry& e : g_maps)
    if (memcmp(&e.key, &k, sizeof(k)) == 0) {
      *out = e.map;
      return true;
    }
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if (!fn) return false;
  cuuint64_t gdim[4], gstride[3];
  cuuint32_t bdim[4], estr[4];
  unsigned long long stride = 8;
  for (int i = 0; i < rank; i++) {
    gdim[i] = dims[i];
    bdim[i] = box[i];
    estr[i] = 1;
    if (i > 0) gstride[i - 1] = stride;
    stride *= dims[i];
  }
  CUtensorMap map;
  const CUresult r = fn(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, rank, const_cast<void*>(base), gdim, gstride, bdim,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char msg[128];
    snprintf(msg, sizeof(msg), "cuTensorMapEncodeTiled failed (%d)", (int)r);
    NRPYELL_FAIL(msg);
    return false;
  }
  if (g_maps.size() > 256) g_maps.clear();
  g_maps.push_back({k, map});
  *out = map;
  return true;
}

template <int BY, int P>
bool bulk_maps(const SubstepArgs& s, BulkMaps* m) {
  const Dims& d = s.d;
  const unsigned long long N0 = d.N0, N1 = d.N1, N2 = d.N2;
  const unsigned long long g2[4] = {N0, N1, N2, 2}, g3[4] = {N0, N1, N2, 3}, c3[3] = {N0, N1, 6};
  const unsigned long long u3[3] = {N0, N1, N2};
  const unsigned bf1[4] = {34, BY, P, 1}, bf2[4] = {34, BY, P, 2}, bf3[4] = {34, BY, P, 3};
  const unsigned bc[3] = {34, BY, 6}, bu[3] = {42, BY, P}, by[3] = {34, 1, P}, bz[3] = {34, BY, 1},
                 bs[3] = {6, BY, P};
  return tensor_map(&m->vv, s.S, 4, g2, bf1) && tensor_map(&m->aux, s.aux, 4, g3, bf3) &&
         tensor_map(&m->y, s.y, 4, g2, bf2) && tensor_map(&m->acc, s.acc, 4, g2, bf2) &&
         tensor_map(&m->coef, s.rt->coef, 3, c3, bc) && tensor_map(&m->U, s.S, 3, u3, bu) &&
         tensor_map(&m->Yh, s.S, 3, u3, by) && tensor_map(&m->Zh, s.S, 3, u3, bz) && tensor_map(&m->SD, s.S, 3, u3, bs);
}

template <int STAGE, bool RESID, int BY, int P, int NS, int NCW>
size_t bulk_smem() {
  return (size_t)NS * BulkLayout<BY, P, BulkFields<STAGE>::value>::SIZE * sizeof(double);
}

// Opts one instantiation in to its shared memory; returns resident CTAs.
template <int STAGE, bool RESID, int BY, int P, int NS, int NCW>
int bulk_opt_in() {
  const size_t smem = bulk_smem<STAGE, RESID, BY, P, NS, NCW>();
  auto kern = k_substep_bulk<STAGE, RESID, BY, P, NS, NCW>;
  NRPYELL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0, dev = 0, sms = 0;
  NRPYELL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * (NCW + 1), smem));
  NRPYELL_CUDA(cudaGetDevice(&dev));
  NRPYELL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return (per_sm > 0 ? per_sm : 1) * sms;
}

// Resident CTA counts of one shape, [0] stage 1 and [1] stages 2-4; set up
// for every stage at once so a launch inside a stream capture finds it done.
template <int BY, int P, int NS, int NCW>
const int* bulk_resident() {
  static int resident[2] = {0, 0};
  if (!resident[0]) {
    const int r1 = bulk_opt_in<1, true, BY, P, NS, NCW>();
    bulk_opt_in<1, false, BY, P, NS, NCW>();
    const int r2 = bulk_opt_in<2, false, BY, P, NS, NCW>();
    bulk_opt_in<3, false, BY, P, NS, NCW>();
    bulk_opt_in<4, false, BY, P, NS, NCW>();
    if (status_ok()) {
      resident[0] = r1;
      resident[1] = r2;
    }
  }
  return resident;
}

template <int STAGE, bool RESID, int BY, int P, int NS, int NCW>
void launch_bulk_t(const SubstepArgs& args) {
  SubDev<double> f = make_dev<double>(args, BY, P);
  f.n_col_blocks = 0;
  const int resident = bulk_resident<BY, P, NS, NCW>()[STAGE == 1 ? 0 : 1];
  if (resident <= 0) return;  // the opt-in failed and set the status
  BulkMaps maps;
  if (!bulk_maps<BY, P>(args, &maps)) return;
  launch_columns_forked<double>(STAGE, args);
  const int grid = f.n_tiles < resident ? f.n_tiles : resident;
  NRPYELL_LAUNCH((k_substep_bulk<STAGE, RESID, BY, P, NS, NCW>), grid, 32 * (NCW + 1),
                 (bulk_smem<STAGE, RESID, BY, P, NS, NCW>()), f, maps);
  join_columns();
}

template <int STAGE, bool RESID>
void launch_bulk_stage(int v, const SubstepArgs& a) {
  switch (v) {
    case 0: launch_bulk_t<STAGE, RESID, 4, 4, 2, 8>(a); break;
    case 1: launch_bulk_t<STAGE, RESID, 4, 4, 3, 8>(a); break;
    case 2: launch_bulk_t<STAGE, RESID, 8, 2, 2, 8>(a); break;
    case 3: launch_bulk_t<STAGE, RESID, 2, 8, 2, 8>(a); break;
    case 4: launch_bulk_t<STAGE, RESID, 4, 2, 2, 4>(a); break;
    default: NRPYELL_FAIL("launch_bulk: shape index out of range"); break;
  }
}

}  // namespace

bool bulk_available(const SubstepArgs& a, size_t elem) {
  auto al = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
  return elem == sizeof(double) && (a.d.N0 % 2) == 0 && al(a.S) && al(a.y) && al(a.acc) && al(a.aux) &&
         al(a.rt->coef);
}

void launch_bulk(int stage, int v, const SubstepArgs& a) {
  const bool resid = (stage == 1) && a.lt;
  switch (stage) {
    case 1:
      if (resid)
        launch_bulk_stage<1, true>(v, a);
      else
        launch_bulk_stage<1, false>(v, a);
      break;
    case 2: launch_bulk_stage<2, false>(v, a); break;
    case 3: launch_bulk_stage<3, false>(v, a); break;
    default: launch_bulk_stage<4, false>(v, a); break;
  }
}

void prepare_bulk(int v) {
  switch (v) {
    case 0: bulk_resident<4, 4, 2, 8>(); break;
    case 1: bulk_resident<4, 4, 3, 8>(); break;
    case 2: bulk_resident<8, 2, 2, 8>(); break;
    case 3: bulk_resident<2, 8, 2, 8>(); break;
    case 4: bulk_resident<4, 2, 2, 4>(); break;
    default: break;
  }
  prepare_columns();
  encode_fn();
}

}  // namespace nrpyell
