// Fused RK4 substep, marching variant (tile kind 5).
//
// Same substep and the same per-point arithmetic as the planes kernel of
// kernels_fused.cu, so every step is bit-identical to it; what differs is how
// uu reaches the stencil.  An interior block owns a 32 x BY tile of (i0,i1)
// columns and PZ consecutive i2 planes, and walks its planes in order:
//   * each plane of uu, widened by 5 points along i0 and i1, and the plane's
//     pointwise inputs (vv of the stage input, the three auxevol fields, y_n
//     and the running total) are copied into shared memory by asynchronous
//     copies (cp.async), issued D-1 planes ahead into a ring of D slots, so
//     the loads of the next D-1 planes are in flight while plane p is
//     computed and the block needs one barrier per plane;
//   * uu along i2 at the thread's own column is a register queue (the 10
//     planes around the first one loaded up front, then one value per plane
//     delivered with the slot), so the i2 stencil arm costs no extra load;
//   * the six metric weights of the column (and the L2 weight) are loaded
//     once per block.
// Per interior point this reads uu from L2 about 2.9-4.6 times (plane halo)
// plus (PZ+10)/PZ times (queue), against 14-16 times in the one-plane planes
// kernel, and the pointwise inputs arrive without a register cost.
// The column blocks (the radiation BC of the x0max face, column_rows) come
// after the interior blocks in a single-grid FP64 launch and before them in
// the correction form's and in batched launches.
#include <functional>
#include <map>
#include <queue>
#include <tuple>
#include <vector>

#include "substep.cuh"

namespace nrpyell {

namespace {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Asynchronous global -> shared copy of BYTES (4, 8: through L1; 16: L2 only).
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  if (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Shared memory of one block, in elements of T per ring slot: the widened uu
// plane [BY+10][42], then NPF pointwise rows of NT values (vv, ADD_TIMES_AUU,
// psi_background, wavespeed, y_n uu, y_n vv, uu at i2+5, and from stage 2 on
// the running totals of uu and vv, and in the correction form R0u and R0b as
// the last two rows).  Rows of 42 doubles are 336 bytes, so every row starts
// on a 16-byte boundary.  (The pointwise fields are copied per point: 16-byte
// pieces of their rows, from i0 = i00-1, were slower.)
template <typename T, int BY, int STAGE, int D, bool CORR = false>
struct MarchSmem {
  static constexpr int NT = 32 * BY, NR = BY + 10, RWS = 42;
  static constexpr int NPF = (STAGE == 1 ? 7 : 9) + (CORR ? 2 : 0);
  static constexpr int plane = NR * RWS;
  static constexpr int slot = plane + NPF * NT;
  static constexpr size_t march = (size_t)D * slot * sizeof(T);
  static constexpr size_t cols = sizeof(double) * (CORR ? kRowsSmemCorr : kRowsSmem);
  static constexpr size_t bytes = march > cols ? march : cols;
};

// Block `bid` of one grid's marching launch; dsm is the block's dynamic
// shared memory (MarchSmem::bytes).  The radiation column blocks come after
// the interior blocks (COLS_LAST: their short, latency-bound blocks fill the
// last wave's free slots) or before them (the batched launch's per-grid
// block ranges).  CORR: the correction form (point_rhs_correction; a.R0 and
// the correction's pointwise fields).
template <typename T, int STAGE, bool RESID, int BY, int PZ, int D, bool COLS_LAST, bool CORR = false>
__device__ __forceinline__ void march_block(const SubDev<T>& a, const int bid, double* dsm, double* sh, bool* lastp) {
  using L = MarchSmem<T, BY, STAGE, D, CORR>;
  constexpr int NT = L::NT, NR = L::NR, RWS = L::RWS, HALF = RWS / 2;
  if (COLS_LAST ? bid >= a.n_tiles : bid < a.n_col_blocks) {
    column_rows<T, STAGE, NT, CORR>(a, COLS_LAST ? bid - a.n_tiles : bid, dsm);
    return;
  }
  T* const ring = reinterpret_cast<T*>(dsm);
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  // block b: chunk b / C of column tile b % C, the PZ-plane chunks first,
  // then the msmall-plane chunks (short blocks last, so the last wave is short)
  const int b = COLS_LAST ? bid : bid - a.n_col_blocks;
  const int C = a.tiles0 * a.tiles1, nbig = C * a.mbig;
  const int s = b - nbig;
  const int col = b < nbig ? b % C : s % C;
  const int z0 = NGHOSTS + (b < nbig ? (b / C) * PZ : a.mbig * PZ + (s / C) * a.msmall);
  const int zc = b < nbig ? PZ : a.msmall;
  const int t0 = col % a.tiles0, t1 = col / a.tiles0;
  const int i00 = t0 * 32 + NGHOSTS, i10 = t1 * BY + NGHOSTS;
  const int N0 = a.N0, top = NGHOSTS + a.Nxx1, Nxx2 = a.Nxx2;
  const int nz = min(zc, NGHOSTS + Nxx2 - z0);
  // element offsets fit in 32 bits (march_fits), so every address is one
  // 32-bit offset scaled onto a base pointer
  const unsigned N01 = (unsigned)a.N01, Ntot = (unsigned)a.Ntot;
  const T* __restrict__ u = a.S;
  // every i2 index below is at most one period outside the interior when
  // Nxx2 >= 10: one conditional add or subtract instead of a loop
  const bool once = Nxx2 >= 2 * NGHOSTS;
  auto wrapz = [&](int j) -> int {
    if (once) return j < NGHOSTS ? j + Nxx2 : (j >= NGHOSTS + Nxx2 ? j - Nxx2 : j);
    return wrapm(j, Nxx2);
  };
  // tiles whose widened planes reach an inner ghost zone gather each point
  // from its source; the others copy rows in pieces of two elements (16
  // bytes for FP64, 8 for FP32) when the pieces are aligned: N0 even and an
  // aligned array
  const bool inner = (t0 == 0) || (i10 < 2 * NGHOSTS) || (i10 + BY + NGHOSTS > top);
  const bool vec = !inner && (N0 & 1) == 0 && (reinterpret_cast<size_t>(u) & (2 * sizeof(T) - 1)) == 0;
  const int i0 = i00 + tx, i1 = i10 + ty;
  const bool valid = i0 < NGHOSTS + a.Nxx0 && i1 < top;
  const unsigned k2 = (unsigned)(i0 + N0 * i1);
  // at stage 1 the stage input is y_n itself: y_n's uu and vv at the point
  // are the plane's centre value and the vv already copied
  const bool y_is_s = STAGE == 1 && a.y == a.S;
  // the two-element pieces of a widened plane this thread copies: offsets within
  // the plane (global, without the plane term) and in the slot; the same for
  // every plane
  constexpr int NV = (NR * HALF + NT - 1) / NT;
  unsigned vg[NV];
  int vs[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) {
    const int e = tid + v * NT;
    const int r = e / HALF, c = 2 * (e - r * HALF);
    const bool ok = e < NR * HALF && i00 - NGHOSTS + c < N0;
    vg[v] = (unsigned)(i00 - NGHOSTS + c + N0 * (i10 - NGHOSTS + r));
    vs[v] = ok ? r * RWS + c : -1;
  }

  // copies of plane p into ring slot p % D (one commit group per plane, empty
  // past the block's last plane)
  auto issue = [&](int p) {
    if (p < nz) {
      T* su = ring + (p % D) * L::slot;
      T* pf = su + L::plane;
      const int i2 = z0 + p;
      const unsigned pl = N01 * (unsigned)i2;
      if (vec) {
#pragma unroll
        for (int v = 0; v < NV; v++)
          if (vs[v] >= 0) cp_async<2 * (int)sizeof(T)>(su + vs[v], u + (vg[v] + pl));
      } else {
        const unsigned plh = N01 * (unsigned)wrap2(i2 + a.half2, Nxx2);
        for (int e = tid; e < NR * RWS; e += NT) {
          const int r = e / RWS, x = e - r * RWS;
          int j0 = i00 - NGHOSTS + x, j1 = i10 - NGHOSTS + r;
          if (j0 >= N0 || j1 >= top + NGHOSTS) continue;  // never read
          bool flip = false;
          if (inner) {
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
          }
          cp_async<(int)sizeof(T)>(su + r * RWS + x, u + ((unsigned)(j0 + N0 * j1) + (flip ? plh : pl)));
        }
      }
      if (valid) {
        const unsigned idx = k2 + pl;
        cp_async<(int)sizeof(T)>(pf + 0 * NT + tid, a.S + (idx + Ntot));
        cp_async<(int)sizeof(T)>(pf + 1 * NT + tid, a.aux + (idx + ADD_TIMES_AUUGF * Ntot));
        cp_async<(int)sizeof(T)>(pf + 2 * NT + tid, a.aux + (idx + PSI_BACKGROUNDGF * Ntot));
        cp_async<(int)sizeof(T)>(pf + 3 * NT + tid, a.aux + (idx + WAVESPEEDGF * Ntot));
        if (!y_is_s) {
          cp_async<(int)sizeof(T)>(pf + 4 * NT + tid, a.y + idx);
          cp_async<(int)sizeof(T)>(pf + 5 * NT + tid, a.y + (idx + Ntot));
        }
        cp_async<(int)sizeof(T)>(pf + 6 * NT + tid, u + (k2 + N01 * (unsigned)wrapz(i2 + NGHOSTS)));
        if (STAGE != 1) {
          cp_async<(int)sizeof(T)>(pf + 7 * NT + tid, a.acc + idx);
          cp_async<(int)sizeof(T)>(pf + 8 * NT + tid, a.acc + (idx + Ntot));
        }
        if (CORR) {
          cp_async<(int)sizeof(T)>(pf + (L::NPF - 2) * NT + tid, a.R0 + idx);
          cp_async<(int)sizeof(T)>(pf + (L::NPF - 1) * NT + tid, a.R0 + (idx + Ntot));
        }
      }
    }
    cp_async_commit();
  };

#pragma unroll
  for (int p = 0; p < D - 1; p++) issue(p);
  // uu along i2: q[j] is plane z0-5+j
  T q[PZ + 10];
  T C22 = 0, C00 = 0, C11 = 0, C1 = 0, C0 = 0, Cc = 0;
  double wl2 = 0.0;
  if (valid) {
#pragma unroll
    for (int j = 0; j < 10; j++) q[j] = __ldg(u + (k2 + N01 * (unsigned)wrapz(z0 - NGHOSTS + j)));
    C22 = __ldg(a.coef + k2);
    C00 = __ldg(a.coef + (k2 + N01));
    C11 = __ldg(a.coef + (k2 + 2 * N01));
    C1 = __ldg(a.coef + (k2 + 3 * N01));
    C0 = __ldg(a.coef + (k2 + 4 * N01));
    Cc = __ldg(a.coef + (k2 + 5 * N01));
    if (RESID) wl2 = __ldg(a.w + k2);
  }
  double r2 = 0.0;
#pragma unroll
  for (int p = 0; p < PZ; p++) {
    if (p >= nz) break;      // uniform over the block
    cp_async_wait<D - 2>();  // this thread's copies of plane p have landed
    __syncthreads();         // everyone's have; slot (p+D-1)%D was last read at plane p-1
    issue(p + D - 1);
    if (valid) {
      const T* su = ring + (p % D) * L::slot;
      const T* pf = su + L::plane + tid;  // this point's pointwise fields, stride NT
      q[p + 10] = pf[6 * NT];
      const T* sp = su + (ty + NGHOSTS) * RWS + tx + NGHOSTS;
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
      for (int k = 1; k <= 5; k++) s22 = fma(W<T>::e(k), q[p + 5 + k] + q[p + 5 - k], s22);
      T ku, kv, br;
      if (CORR) {
        T ju, jv;
        point_rhs_correction<T>(q[p + 5], pf[0], pf[NT], pf[2 * NT], pf[3 * NT], C22, C00, C11, C1, C0, Cc, s0, s1,
                                s00, s11, s22, a.eta, pf[(L::NPF - 2) * NT], pf[(L::NPF - 1) * NT], ku, kv, br, ju,
                                jv);
      } else {
        point_rhs<T>(q[p + 5], pf[0], pf[NT], pf[2 * NT], pf[3 * NT], C22, C00, C11, C1, C0, Cc, s0, s1, s00, s11,
                     s22, a.eta, ku, kv, br);
      }
      // RK combination and stores (store_point's arithmetic, 32-bit offsets)
      T accu = (STAGE == 1) ? (T)0 : pf[7 * NT];
      T accv = (STAGE == 1) ? (T)0 : pf[8 * NT];
      T ou, ov;
      rk_combine<T, STAGE>(ku, y_is_s ? q[p + 5] : pf[4 * NT], accu, ou, a.dt);
      rk_combine<T, STAGE>(kv, y_is_s ? pf[0] : pf[5 * NT], accv, ov, a.dt);
      const unsigned o = k2 + N01 * (unsigned)(z0 + p);
      if (STAGE != 4) {
        a.acc[o] = accu;
        a.acc[o + Ntot] = accv;
      }
      a.out[o] = ou;
      a.out[o + Ntot] = ov;
      if (RESID) {
        const double bb = (double)br;
        r2 += bb * bb * wl2;
      }
    }
  }
  if (RESID && tile_partial<NT>(r2, b, a.partials, a.ticket, a.n_tiles, sh, lastp, a.defer_l2 != 0))
    finalize_l2<T, NT>(a, sh);
}

template <typename T, int STAGE, bool RESID, int BY, int PZ, int D, int MINB, bool CORR = false>
__global__ void __launch_bounds__(32 * BY, MINB) k_substep_march(SubDev<T> a) {
  extern __shared__ __align__(16) double dsm[];
  __shared__ double sh[BY > 8 ? BY : 8];
  __shared__ bool last;
  pdl_enter();
  if (*a.done) return;
  // FP64: column blocks last; correction form: first (its column blocks
  // evaluate the radiation BC in FP64 and were the launch's tail when last:
  // 163.5 -> 151.9 us per RK4 step at 256x256x32)
  march_block<T, STAGE, RESID, BY, PZ, D, !CORR, CORR>(a, blockIdx.x, dsm, sh, &last);
}

// One substep of many grids in one launch: the blocks of grid c are
// offs[c] .. offs[c+1]-1 (column blocks first, then interior tiles), each
// grid with its own launch arguments, stop test and done flag.
template <typename T, int STAGE, bool RESID, int BY, int PZ, int D, int MINB, bool CORR = false>
__global__ void __launch_bounds__(32 * BY, MINB)
    k_substep_march_batch(const SubDev<T>* __restrict__ devs, const int* __restrict__ offs, int n) {
  extern __shared__ __align__(16) double dsm[];
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
  march_block<T, STAGE, RESID, BY, PZ, D, false, CORR>(a, bx - __ldg(offs + lo), dsm, sh, &last);
}

// Opts the kernel into more than 48 KB of dynamic shared memory, once per
// device.
template <typename T, int STAGE, bool RESID, int BY, int PZ, int D, int MINB, bool BATCH = false, bool CORR = false>
bool march_opt_in() {
  static unsigned long long devices = 0;
  const size_t bytes = MarchSmem<T, BY, STAGE, D, CORR>::bytes;
  if (bytes <= 48 * 1024) return true;
  int dev = 0;
  NRPYELL_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !(devices >> dev & 1ull)) {
    if constexpr (BATCH)
      NRPYELL_CUDA(cudaFuncSetAttribute(k_substep_march_batch<T, STAGE, RESID, BY, PZ, D, MINB, CORR>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    else
      NRPYELL_CUDA(cudaFuncSetAttribute(k_substep_march<T, STAGE, RESID, BY, PZ, D, MINB, CORR>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    devices |= 1ull << dev;
  }
  return status_ok();
}

// Split of each column tile's Nz planes into nb chunks of PZ planes and ns
// chunks of `small` planes.  The block scheduler hands out blocks in index
// order as slots free up; with equal chunks the last wave is a partial one
// (1024 chunks on 296 slots leave SMs idle for ~14 % of a 256x256x32 launch).
// Greedy list scheduling of the launch's blocks -- the long chunks, then the
// short ones (cost planes / PZ + 0.15 for the start-up), then the column
// blocks (cost 0.3) -- on `slots` resident blocks picks the split with the
// shortest makespan.
struct MarchSplit {
  int nb, small, ns;
};

MarchSplit choose_split(int C, int Nz, int PZ, int slots, int ncol) {
  auto makespan = [&](int nb, int small, int ns) {
    std::priority_queue<double, std::vector<double>, std::greater<double>> q;
    for (int i = 0; i < slots; i++) q.push(0.0);
    auto take = [&](double d, long long n) {
      for (long long i = 0; i < n; i++) {
        const double t = q.top();
        q.pop();
        q.push(t + d);
      }
    };
    take(1.15, (long long)C * nb);
    if (ns > 0) take((double)small / PZ + 0.15, (long long)C * ns);
    take(0.3, ncol);
    double end = 0.0;
    while (!q.empty()) {
      end = q.top();
      q.pop();
    }
    return end;
  };
  const int nfull = (Nz + PZ - 1) / PZ;
  MarchSplit best = {nfull, 0, 0};
  if (slots <= 0) return best;
  double tbest = makespan(nfull, 0, 0);
  for (int nb = 0; nb < nfull; nb++) {
    const int rest = Nz - nb * PZ;
    for (int small : {PZ / 2, PZ / 4}) {
      if (small < 1) continue;
      const int ns = (rest + small - 1) / small;
      const double t = makespan(nb, small, ns);
      if (t < tbest * 0.99) {  // only for a clear gain
        tbest = t;
        best = {nb, small, ns};
      }
    }
  }
  return best;
}

template <typename T, int STAGE, bool RESID, int BY, int PZ, int D, int MINB>
MarchSplit march_split(const Dims& d, int ncol) {
  static std::map<std::tuple<int, int, int, int>, MarchSplit> cache;
  march_opt_in<T, STAGE, RESID, BY, PZ, D, MINB>();  // the occupancy query needs the shared-memory opt-in
  int dev = 0;
  NRPYELL_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_tuple(dev, d.Nxx0, d.Nxx1, d.Nxx2);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int per_sm = 0, sms = 0;
  NRPYELL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_substep_march<T, STAGE, RESID, BY, PZ, D, MINB>,
                                                             32 * BY, MarchSmem<T, BY, STAGE, D>::bytes));
  NRPYELL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int C = ((d.Nxx0 + 31) / 32) * ((d.Nxx1 + BY - 1) / BY);
  const MarchSplit s = choose_split(C, d.Nxx2, PZ, per_sm * sms, ncol);
  cache[key] = s;
  return s;
}

// The correction form takes the plain form's split (the stop test's
// reduction sums exactly march_interior_blocks partials).
template <typename T, int STAGE, bool RESID, int BY, int PZ, int D, int MINB, bool CORR = false>
void launch_march_shape(const SubstepArgs& a) {
  if (!march_opt_in<T, STAGE, RESID, BY, PZ, D, MINB, false, CORR>()) return;
  SubDev<T> f = make_dev<T>(a, BY, PZ);
  f.n_col_blocks = ((a.d.Nxx1 + kRows - 1) / kRows) * a.d.Nxx2;
  // the split is chosen once per grid size and shape (stage 2's occupancy)
  const MarchSplit sp = march_split<T, 2, false, BY, PZ, D, MINB>(a.d, f.n_col_blocks);
  f.mbig = sp.nb;
  f.msmall = sp.small;
  f.n_tiles = f.tiles0 * f.tiles1 * (sp.nb + sp.ns);
  NRPYELL_LAUNCH_PDL((k_substep_march<T, STAGE, RESID, BY, PZ, D, MINB, CORR>), f.n_tiles + f.n_col_blocks, 32 * BY,
                     (MarchSmem<T, BY, STAGE, D, CORR>::bytes), f);
}

// The compiled shapes, by index: (BY, PZ, ring slots D, minimum resident
// blocks per SM for the register budget).
#define NRPYELL_MARCH_SHAPES(X)                                                                           \
  X(0, 8, 8, 3, 2) X(1, 8, 16, 2, 3) X(2, 8, 4, 2, 4) X(3, 8, 4, 2, 3) X(4, 8, 8, 2, 3) X(5, 8, 32, 2, 3) \
      X(6, 8, 4, 3, 2)

template <typename T, int STAGE, bool RESID, bool CORR = false>
bool march_stage(int v, const SubstepArgs& a) {
  switch (v) {
#define NRPYELL_MARCH(I, BY, PZ, D, MINB)                          \
  case I:                                                          \
    launch_march_shape<T, STAGE, RESID, BY, PZ, D, MINB, CORR>(a); \
    return true;
    NRPYELL_MARCH_SHAPES(NRPYELL_MARCH)
#undef NRPYELL_MARCH
  }
  return false;
}

template <typename T, int STAGE, bool RESID, int BY, int PZ, int D, int MINB, bool CORR = false>
void launch_march_batch_shape(const SubDev<T>* devs, const int* offs, int n, int blocks) {
  if (!march_opt_in<T, STAGE, RESID, BY, PZ, D, MINB, true, CORR>()) return;
  NRPYELL_LAUNCH_PDL((k_substep_march_batch<T, STAGE, RESID, BY, PZ, D, MINB, CORR>), blocks, 32 * BY,
                     (MarchSmem<T, BY, STAGE, D, CORR>::bytes), devs, offs, n);
}

template <typename T, int STAGE, bool RESID, bool CORR = false>
bool march_batch_stage(int v, const SubDev<T>* devs, const int* offs, int n, int blocks) {
  switch (v) {
#define NRPYELL_MARCH(I, BY, PZ, D, MINB)                                                 \
  case I:                                                                                 \
    launch_march_batch_shape<T, STAGE, RESID, BY, PZ, D, MINB, CORR>(devs, offs, n, blocks); \
    return true;
    NRPYELL_MARCH_SHAPES(NRPYELL_MARCH)
#undef NRPYELL_MARCH
  }
  return false;
}

template <typename T, int BY, int PZ, int D, int MINB>
void opt_in_shape() {
  march_opt_in<T, 1, true, BY, PZ, D, MINB>();
  march_opt_in<T, 1, false, BY, PZ, D, MINB>();
  march_opt_in<T, 2, false, BY, PZ, D, MINB>();
  march_opt_in<T, 3, false, BY, PZ, D, MINB>();
  march_opt_in<T, 4, false, BY, PZ, D, MINB>();
  if constexpr (sizeof(T) == 4) {
    march_opt_in<T, 1, true, BY, PZ, D, MINB, false, true>();
    march_opt_in<T, 1, false, BY, PZ, D, MINB, false, true>();
    march_opt_in<T, 2, false, BY, PZ, D, MINB, false, true>();
    march_opt_in<T, 3, false, BY, PZ, D, MINB, false, true>();
    march_opt_in<T, 4, false, BY, PZ, D, MINB, false, true>();
  }
}

}  // namespace

bool march_fits(const Dims& d) { return 3.0 * (double)d.Ntot < 4294967296.0; }

template <typename T>
bool launch_march(int stage, bool resid, int v, const SubstepArgs& a) {
  if (!march_fits(a.d)) return false;
  bool ok = false;
  if (a.R0) {  // the correction form (FP32 only)
    if constexpr (sizeof(T) == 4) {
      switch (stage) {
        case 1: ok = resid ? march_stage<T, 1, true, true>(v, a) : march_stage<T, 1, false, true>(v, a); break;
        case 2: ok = march_stage<T, 2, false, true>(v, a); break;
        case 3: ok = march_stage<T, 3, false, true>(v, a); break;
        default: ok = march_stage<T, 4, false, true>(v, a); break;
      }
    }
    if (!ok) NRPYELL_FAIL("launch_march: the correction form exists for FP32 marching shapes only");
    return true;
  }
  switch (stage) {
    case 1: ok = resid ? march_stage<T, 1, true>(v, a) : march_stage<T, 1, false>(v, a); break;
    case 2: ok = march_stage<T, 2, false>(v, a); break;
    case 3: ok = march_stage<T, 3, false>(v, a); break;
    default: ok = march_stage<T, 4, false>(v, a); break;
  }
  if (!ok) NRPYELL_FAIL("launch_march: no kernel for this shape");
  return true;
}
template bool launch_march<double>(int, bool, int, const SubstepArgs&);
template bool launch_march<float>(int, bool, int, const SubstepArgs&);

template <typename T>
int march_interior_blocks(int v, const SubstepArgs& a) {
  const int ncol = ((a.d.Nxx1 + kRows - 1) / kRows) * a.d.Nxx2;
  switch (v) {
#define NRPYELL_MARCH(I, BY, PZ, D, MINB)                                               \
  case I: {                                                                             \
    const MarchSplit sp = march_split<T, 2, false, BY, PZ, D, MINB>(a.d, ncol);         \
    return ((a.d.Nxx0 + 31) / 32) * ((a.d.Nxx1 + BY - 1) / BY) * (sp.nb + sp.ns);       \
  }
    NRPYELL_MARCH_SHAPES(NRPYELL_MARCH)
#undef NRPYELL_MARCH
  }
  return 0;
}
template int march_interior_blocks<double>(int, const SubstepArgs&);
template int march_interior_blocks<float>(int, const SubstepArgs&);

template <typename T>
void prepare_march(int v) {
  switch (v) {
#define NRPYELL_MARCH(I, BY, PZ, D, MINB) \
  case I: opt_in_shape<T, BY, PZ, D, MINB>(); break;
    NRPYELL_MARCH_SHAPES(NRPYELL_MARCH)
#undef NRPYELL_MARCH
  }
}
template void prepare_march<double>(int);
template void prepare_march<float>(int);

template <typename T>
void launch_march_batch(int stage, bool resid, int v, const SubDev<T>* devs, const int* offs, int n, int blocks,
                        bool corr) {
  bool ok = false;
  if (corr) {  // the correction form (FP32 only)
    if constexpr (sizeof(T) == 4) {
      switch (stage) {
        case 1:
          ok = resid ? march_batch_stage<T, 1, true, true>(v, devs, offs, n, blocks)
                     : march_batch_stage<T, 1, false, true>(v, devs, offs, n, blocks);
          break;
        case 2: ok = march_batch_stage<T, 2, false, true>(v, devs, offs, n, blocks); break;
        case 3: ok = march_batch_stage<T, 3, false, true>(v, devs, offs, n, blocks); break;
        default: ok = march_batch_stage<T, 4, false, true>(v, devs, offs, n, blocks); break;
      }
    }
    if (!ok) NRPYELL_FAIL("launch_march_batch: the correction form exists for FP32 only");
    return;
  }
  if constexpr (sizeof(T) == 8) {  // FP32 batches run the correction form only
    switch (stage) {
      case 1:
        ok = resid ? march_batch_stage<T, 1, true>(v, devs, offs, n, blocks)
                   : march_batch_stage<T, 1, false>(v, devs, offs, n, blocks);
        break;
      case 2: ok = march_batch_stage<T, 2, false>(v, devs, offs, n, blocks); break;
      case 3: ok = march_batch_stage<T, 3, false>(v, devs, offs, n, blocks); break;
      default: ok = march_batch_stage<T, 4, false>(v, devs, offs, n, blocks); break;
    }
  }
  if (!ok) NRPYELL_FAIL("launch_march_batch: no kernel for this shape and precision");
}
template void launch_march_batch<double>(int, bool, int, const SubDev<double>*, const int*, int, int, bool);
template void launch_march_batch<float>(int, bool, int, const SubDev<float>*, const int*, int, int, bool);

}  // namespace nrpyell
