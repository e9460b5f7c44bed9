// Construction and caching of the device tables declared in tables.cuh.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "sinhsymtp.h"
#include "tables.cuh"

namespace nrpyell {

namespace {
std::vector<RfmTables*> g_rfm;
std::vector<BcTables*> g_bc;
std::vector<L2Tables*> g_l2;
Scratch* g_scratch = nullptr;

bool same_dims(const Dims& a, const Dims& b) {
  return a.N0 == b.N0 && a.N1 == b.N1 && a.N2 == b.N2 && a.Nxx0 == b.Nxx0 && a.Nxx1 == b.Nxx1 && a.Nxx2 == b.Nxx2;
}

void* table_alloc(size_t bytes) {
  void* p = nullptr;
  NRPYELL_CUDA(dev_alloc(&p, bytes > 0 ? bytes : 16));
  return p;
}

void upload(void* dst, const void* src, size_t bytes) {
  if (bytes) NRPYELL_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
}

}  // namespace

RfmTables* find_rfm_tables(const paramstruct* p, const rfm_struct* rfm) {
  const Dims d = dims_of(p);
  for (RfmTables* t : g_rfm)
    if (t->key_f0 == rfm->f0_of_xx0 && t->key_f2 == rfm->f2_of_xx0_xx1 && same_dims(t->d, d) &&
        t->invdx[0] == p->invdx0 && t->invdx[1] == p->invdx1 && t->invdx[2] == p->invdx2 && t->AMAX == p->AMAX &&
        t->SINHWAA == p->SINHWAA && t->bScale == p->bScale)
      return t;
  return nullptr;
}

RfmTables* new_rfm_tables(const paramstruct* p, const rfm_struct* rfm) {
  const Dims d = dims_of(p);
  RfmTables* t = new RfmTables();
  t->key_f0 = rfm->f0_of_xx0;
  t->key_f2 = rfm->f2_of_xx0_xx1;
  t->d = d;
  t->invdx[0] = p->invdx0;
  t->invdx[1] = p->invdx1;
  t->invdx[2] = p->invdx2;
  t->AMAX = p->AMAX;
  t->SINHWAA = p->SINHWAA;
  t->bScale = p->bScale;
  const size_t n0 = d.N0, n1 = d.N1, n01 = n0 * n1;
  // the device build stages xx0 and xx1 behind the float weights
  const size_t n_doubles = 5 * n0 + 2 * n1 + 2 * n01 + kNumCoef * n01;
  const size_t bytes = n_doubles * sizeof(double) + kNumCoef * n01 * sizeof(float) + (n0 + n1) * sizeof(double) + 512;
  char* base = (char*)table_alloc(bytes);
  if (!base) {
    delete t;
    return nullptr;
  }
  t->base = base;
  double* q = (double*)base;
  t->f0 = q; q += n0;
  t->f0_D0 = q; q += n0;
  t->f0_DD00 = q; q += n0;
  t->f3 = q; q += n0;
  t->f3_D0 = q; q += n0;
  t->f1 = q; q += n1;
  t->f1_D1 = q; q += n1;
  t->f2 = q; q += n01;
  t->f2_D0 = q; q += n01;
  t->coef = q; q += kNumCoef * n01;
  t->coef32 = (float*)q;
  t->xx01 = (double*)(base + ((n_doubles * sizeof(double) + kNumCoef * n01 * sizeof(float) + 255) / 256) * 256);
  return t;
}

void register_rfm_tables(RfmTables* t) { g_rfm.push_back(t); }

RfmTables* get_rfm_tables(const paramstruct* p, const rfm_struct* rfm) {
  if (RfmTables* f = find_rfm_tables(p, rfm)) return f;
  if (!rfm->f0_of_xx0 || !rfm->f2_of_xx0_xx1 || !rfm->f1_of_xx1 || !rfm->f3_of_xx0) {
    NRPYELL_FAIL("rfm_struct has NULL arrays (call rfm_precompute_rfmstruct_define or nrpyell_setup_tables_device first)");
    return nullptr;
  }
  RfmTables* t = new_rfm_tables(p, rfm);
  if (!t) return nullptr;
  const Dims d = t->d;
  const size_t n0 = d.N0, n1 = d.N1, n01 = n0 * n1;
  upload(t->f0, rfm->f0_of_xx0, n0 * 8);
  upload(t->f0_D0, rfm->f0_of_xx0__D0, n0 * 8);
  upload(t->f0_DD00, rfm->f0_of_xx0__DD00, n0 * 8);
  upload(t->f3, rfm->f3_of_xx0, n0 * 8);
  upload(t->f3_D0, rfm->f3_of_xx0__D0, n0 * 8);
  upload(t->f1, rfm->f1_of_xx1, n1 * 8);
  upload(t->f1_D1, rfm->f1_of_xx1__D1, n1 * 8);
  upload(t->f2, rfm->f2_of_xx0_xx1, n01 * 8);
  upload(t->f2_D0, rfm->f2_of_xx0_xx1__D0, n01 * 8);

  // Fold the metric factors of the vv right-hand side (rhs_eval.c:106-110)
  // into one weight per raw stencil sum.
  std::vector<double> coef(kNumCoef * n01, 0.0);
  std::vector<float> coef32(kNumCoef * n01, 0.0f);
  const double ix0 = p->invdx0, ix1 = p->invdx1, ix2 = p->invdx2;
  for (size_t i1 = 0; i1 < n1; i1++)
    for (size_t i0 = 0; i0 < n0; i0++) {
      const size_t k = i0 + n0 * i1;
      const double f0 = rfm->f0_of_xx0[i0], f0p = rfm->f0_of_xx0__D0[i0], f0pp = rfm->f0_of_xx0__DD00[i0];
      const double f1 = rfm->f1_of_xx1[i1], f1p = rfm->f1_of_xx1__D1[i1];
      const double f2 = rfm->f2_of_xx0_xx1[k], f2_0 = rfm->f2_of_xx0_xx1__D0[k];
      const double f3 = rfm->f3_of_xx0[i0], f3p = rfm->f3_of_xx0__D0[i0];
      double cs[kNumCoef];
      symtp_fold_rhs_coefs(f0, f0p, f0pp, f1, f1p, f2, f2_0, f3, f3p, ix0, ix1, ix2, cs);
      for (int c = 0; c < kNumCoef; c++) {
        coef[c * n01 + k] = cs[c];
        coef32[c * n01 + k] = (float)cs[c];
      }
    }
  upload(t->coef, coef.data(), coef.size() * 8);
  upload(t->coef32, coef32.data(), coef32.size() * 4);
  g_rfm.push_back(t);
  return t;
}

BcTables* find_bc_tables(const paramstruct* p, const bc_struct* bc, REAL* NRPYELL_RESTRICT const xx[3]) {
  const Dims d = dims_of(p);
  for (BcTables* t : g_bc)
    if (t->key_inner == bc->inner_bc_array && t->key_outer0 == bc->pure_outer_bc_array[0] &&
        t->key_ninner == bc->bc_info.num_inner_boundary_points && same_dims(t->d, d) && t->key_xx[0] == xx[0] &&
        t->key_xx[1] == xx[1] && t->key_xx[2] == xx[2] && t->AMAX == p->AMAX && t->SINHWAA == p->SINHWAA &&
        t->bScale == p->bScale && t->dxx0 == p->dxx0 && t->dxx1 == p->dxx1 && t->dxx2 == p->dxx2)
      return t;
  return nullptr;
}

void register_bc_tables(BcTables* t) { g_bc.push_back(t); }

void bc_tables_set_key(BcTables* t, const paramstruct* p, const bc_struct* bc, REAL* NRPYELL_RESTRICT const xx[3]) {
  t->key_inner = bc->inner_bc_array;
  t->key_outer0 = bc->pure_outer_bc_array[0];
  t->key_ninner = bc->bc_info.num_inner_boundary_points;
  for (int i = 0; i < 3; i++) t->key_xx[i] = xx[i];
  t->d = dims_of(p);
  t->AMAX = p->AMAX;
  t->SINHWAA = p->SINHWAA;
  t->bScale = p->bScale;
  t->dxx0 = p->dxx0;
  t->dxx1 = p->dxx1;
  t->dxx2 = p->dxx2;
}

bool bc_tables_layout(BcTables* t, size_t n_inner, size_t n_outer) {
  const size_t b_inner = (n_inner > 0 ? n_inner : 1) * sizeof(int2);
  const size_t b_par = (((n_inner > 0 ? n_inner : 1) + 255) / 256) * 256;
  const size_t b_outer = (n_outer > 0 ? n_outer : 1) * sizeof(OuterPoint);
  const size_t b_col = 3 * 6 * (size_t)t->d.N1 * sizeof(double);
  const size_t b_xx = ((size_t)t->d.N0 + t->d.N1) * sizeof(double);
  char* base = (char*)table_alloc(b_inner + b_par + b_outer + b_col + b_xx + 1280);
  if (!base) return false;
  t->base = base;
  size_t o = 0;
  t->inner = (int2*)(base + o); o += (b_inner + 255) / 256 * 256;
  t->inner_par = (signed char*)(base + o); o += b_par;
  t->outer = (OuterPoint*)(base + o); o += (b_outer + 255) / 256 * 256;
  t->colgeo = (double*)(base + o); o += (b_col + 255) / 256 * 256;
  t->xx01 = (double*)(base + o);
  return true;
}

BcTables* get_bc_tables(const paramstruct* p, const bc_struct* bc, REAL* NRPYELL_RESTRICT const xx[3]) {
  if (BcTables* f = find_bc_tables(p, bc, xx)) return f;
  const Dims d = dims_of(p);
  BcTables* t = new BcTables();
  t->key_inner = bc->inner_bc_array;
  t->key_outer0 = bc->pure_outer_bc_array[0];
  t->key_ninner = bc->bc_info.num_inner_boundary_points;
  for (int i = 0; i < 3; i++) t->key_xx[i] = xx[i];
  t->d = d;
  t->AMAX = p->AMAX;
  t->SINHWAA = p->SINHWAA;
  t->bScale = p->bScale;
  t->dxx0 = p->dxx0;
  t->dxx1 = p->dxx1;
  t->dxx2 = p->dxx2;
  const int N0 = d.N0, N1 = d.N1, N2 = d.N2;

  // Inner map.
  const int ni = bc->bc_info.num_inner_boundary_points;
  std::vector<int2> inner(ni > 0 ? ni : 1);
  std::vector<signed char> par(ni > 0 ? ni : 1);
  for (int i = 0; i < ni; i++) {
    const int dst = bc->inner_bc_array[i].dstpt, src = bc->inner_bc_array[i].srcpt;
    if (dst < 0 || dst >= d.Ntot || src < 0 || src >= d.Ntot) {
      NRPYELL_FAIL("bc_struct inner point index out of range");
      delete t;
      return nullptr;
    }
    inner[i] = make_int2(dst, src);
    par[i] = bc->inner_bc_array[i].parity[0];
  }
  t->n_inner = ni;
  {
    // Inner map == SymTP reflections, and inner + pure outer cover every ghost point.
    bool ok = ((long long)ni == d.Ntot - (long long)d.Nxx0 * d.Nxx1 * d.Nxx2 - (long long)NGHOSTS * d.Nxx1 * d.Nxx2) &&
              d.Nxx2 % 2 == 0 && d.Nxx2 >= NGHOSTS;
    for (int i = 0; i < ni && ok; i++) {
      const int dst = inner[i].x;
      const int i0 = dst % N0, i1 = (dst / N0) % N1, i2 = dst / (N0 * N1);
      int m[3];
      symtp_ghost_source(i0, i1, i2, d.Nxx1, d.Nxx2, m);
      ok = (m[0] + N0 * (m[1] + N1 * m[2]) == inner[i].y) && par[i] == 1;
    }
    t->analytic_ok = ok;
  }

  // Generic outer lists with precomputed geometry.
  std::vector<OuterPoint> outer;
  int max_layer = 0;
  bool columns_ok = true;
  for (int gz = 0; gz < NGHOSTS; gz++)
    for (int dirn = 0; dirn < 3; dirn++) {
      const int list = dirn + 3 * gz;
      t->outer_off[list] = (int)outer.size();
      const int n = bc->bc_info.num_pure_outer_boundary_points[gz][dirn];
      if (n > max_layer) max_layer = n;
      if (dirn == 0) {
        if (n != d.Nxx1 * d.Nxx2) columns_ok = false;
      } else if (n != 0) {
        columns_ok = false;
      }
      for (int k = 0; k < n; k++) {
        const outerpt_bc_struct& o = bc->pure_outer_bc_array[list][k];
        OuterPoint q;
        q.i0 = o.i0; q.i1 = o.i1; q.i2 = o.i2;
        q.i0n = o.i0 + o.FACEX0; q.i1n = o.i1 + o.FACEX1; q.i2n = o.i2 + o.FACEX2;
        if (o.i0 < 0 || o.i0 >= N0 || o.i1 < 0 || o.i1 >= N1 || o.i2 < 0 || o.i2 >= N2 || q.i0n < 0 || q.i0n >= N0 ||
            q.i1n < 0 || q.i1n >= N1 || q.i2n < 0 || q.i2n >= N2) {
          NRPYELL_FAIL("bc_struct outer point index out of range");
          delete t;
          return nullptr;
        }
        if (dirn == 0 && !(o.FACEX0 == -1 && o.FACEX1 == 0 && o.FACEX2 == 0 && o.i0 == N0 - NGHOSTS + gz &&
                           o.i1 >= NGHOSTS && o.i1 < N1 - NGHOSTS && o.i2 >= NGHOSTS && o.i2 < N2 - NGHOSTS))
          columns_ok = false;
        q.idx3 = o.i0 + N0 * (o.i1 + N1 * o.i2);
        q.idx3_int = q.i0n + N0 * (q.i1n + N1 * q.i2n);
        q.off0 = (signed char)radiation_upwind_offset(o.FACEX0, o.i0, N0);
        q.off1 = (signed char)radiation_upwind_offset(o.FACEX1, o.i1, N1);
        q.off0n = (signed char)radiation_upwind_offset(o.FACEX0, q.i0n, N0);
        q.off1n = (signed char)radiation_upwind_offset(o.FACEX1, q.i1n, N1);
        if (xx[0] && xx[1]) {
          symtp_radial_geometry(p->AMAX, p->SINHWAA, p->bScale, xx[0][o.i0], xx[1][o.i1], &q.r, &q.dx0dr, &q.dx1dr);
          symtp_radial_geometry(p->AMAX, p->SINHWAA, p->bScale, xx[0][q.i0n], xx[1][q.i1n], &q.rn, &q.dx0drn, &q.dx1drn);
        } else {
          q.r = q.dx0dr = q.dx1dr = q.rn = q.dx0drn = q.dx1drn = 0.0;
        }
        outer.push_back(q);
      }
    }
  t->outer_off[NGHOSTS * 3] = (int)outer.size();
  t->n_outer = (int)outer.size();
  t->max_layer = max_layer;
  // Without coordinates (inner-only / extrapolation callers) there is no
  // radiation geometry, hence no column form.
  t->columns_ok = columns_ok && d.Nxx0 >= 12 && xx[0] && xx[1];

  // Column geometry: j = 0 is i0 = N0-NGHOSTS-1, j = 1..5 the outer layers.
  std::vector<double> colgeo(3 * 6 * N1, 0.0);
  for (int j = 0; j < 6 && t->columns_ok; j++)
    for (int i1 = 0; i1 < N1; i1++) {
      double r, a, b;
      symtp_radial_geometry(p->AMAX, p->SINHWAA, p->bScale, xx[0][N0 - NGHOSTS - 1 + j], xx[1][i1], &r, &a, &b);
      colgeo[(0 * 6 + j) * N1 + i1] = r;
      colgeo[(1 * 6 + j) * N1 + i1] = a;
      colgeo[(2 * 6 + j) * N1 + i1] = b;
    }

  if (!bc_tables_layout(t, inner.size(), outer.size())) {
    delete t;
    return nullptr;
  }
  upload(t->inner, inner.data(), inner.size() * sizeof(int2));
  upload(t->inner_par, par.data(), par.size());
  if (!outer.empty()) upload(t->outer, outer.data(), outer.size() * sizeof(OuterPoint));
  upload(t->colgeo, colgeo.data(), colgeo.size() * sizeof(double));
  g_bc.push_back(t);
  return t;
}

L2Tables* get_l2_tables(const paramstruct* p, REAL* NRPYELL_RESTRICT const xx[3], double R) {
  const Dims d = dims_of(p);
  for (L2Tables* t : g_l2)
    if (t->key_xx[0] == xx[0] && t->key_xx[1] == xx[1] && t->key_xx[2] == xx[2] && same_dims(t->d, d) &&
        t->AMAX == p->AMAX && t->SINHWAA == p->SINHWAA && t->bScale == p->bScale && t->dxx0 == p->dxx0 &&
        t->dxx1 == p->dxx1 && t->dxx2 == p->dxx2 && t->R == R)
      return t;
  L2Tables* t = new L2Tables();
  for (int i = 0; i < 3; i++) t->key_xx[i] = xx[i];
  t->d = d;
  t->AMAX = p->AMAX; t->SINHWAA = p->SINHWAA; t->bScale = p->bScale;
  t->dxx0 = p->dxx0; t->dxx1 = p->dxx1; t->dxx2 = p->dxx2;
  t->R = R;
  const int N0 = d.N0, N1 = d.N1;
  std::vector<double> w((size_t)N0 * N1, 0.0);
  // Volume element of L2_norm_of_gf.c:19-32, evaluated once per (i0, i1).
  long double vol = 0.0L;
  const double AMAX = p->AMAX, bScale = p->bScale;
  for (int i1 = NGHOSTS; i1 < NGHOSTS + d.Nxx1; i1++)
    for (int i0 = NGHOSTS; i0 < NGHOSTS + d.Nxx0; i0++) {
      const double xx0 = xx[0][i0], xx1 = xx[1][i1];
      const double s = sin(xx1);
      const double iw = 1.0 / p->SINHWAA;
      const double D = exp(iw) - exp(-iw);
      const double ep = exp(iw * xx0), em = exp(-iw * xx0);
      const double E2 = (ep - em) * (ep - em);
      const double A2 = AMAX * AMAX * E2 / (D * D);
      const double B2 = bScale * bScale + A2;
      const double r = sqrt(s * s * A2 + B2 * (cos(xx1) * cos(xx1)));
      const double q = bScale * bScale * (s * s) + A2;
      const double sqrtdetgamma =
          AMAX * AMAX * sqrt(E2 * (q * q) * ((iw * ep + iw * em) * (iw * ep + iw * em)) / (B2 * (D * D * D * D))) * fabs(s);
      if (r < R) {
        const double dV = sqrtdetgamma * p->dxx0 * p->dxx1 * p->dxx2;
        w[i0 + (size_t)N0 * i1] = dV;
        vol += (long double)dV;
      }
    }
  t->volume = (double)(vol * (long double)d.Nxx2);
  t->w = (double*)table_alloc(w.size() * sizeof(double));
  upload(t->w, w.data(), w.size() * sizeof(double));
  g_l2.push_back(t);
  return t;
}

static int g_scratch_generation = 0;
int scratch_generation() { return g_scratch_generation; }

Scratch* get_scratch(int n_partials) {
  if (g_scratch && g_scratch->n_partials >= n_partials) return g_scratch;
  g_scratch_generation++;  // graphs captured with the old buffer are stale
  if (g_scratch) {
    NRPYELL_CUDA(cudaStreamSynchronize(stream()));
    NRPYELL_CUDA(cudaFree(g_scratch->base));
    delete g_scratch;
  }
  Scratch* s = new Scratch();
  s->n_partials = n_partials < 4096 ? 4096 : n_partials;
  const size_t bytes = (size_t)s->n_partials * 8 + 4 * 8 + 64 + 8 * 4 + 256;
  char* base = (char*)table_alloc(bytes);
  NRPYELL_CUDA(cudaMemset(base, 0, bytes));
  s->base = base;
  s->partials = (double*)base;
  s->result = (double*)(base + (size_t)s->n_partials * 8);
  s->counter = (unsigned int*)(base + (size_t)s->n_partials * 8 + 32);
  s->flags = (int*)(base + (size_t)s->n_partials * 8 + 96);
  g_scratch = s;
  return s;
}

void release_all_tables() {
  cudaStreamSynchronize(stream());
  for (RfmTables* t : g_rfm) {
    cudaFree(t->base);
    delete t;
  }
  for (BcTables* t : g_bc) {
    cudaFree(t->base);
    delete t;
  }
  for (L2Tables* t : g_l2) {
    cudaFree(t->w);
    delete t;
  }
  g_rfm.clear();
  g_bc.clear();
  g_l2.clear();
  if (g_scratch) {
    cudaFree(g_scratch->base);
    delete g_scratch;
    g_scratch = nullptr;
  }
}

}  // namespace nrpyell
