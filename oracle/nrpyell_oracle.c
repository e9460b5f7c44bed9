/*
 * nrpyell_oracle.c -- CPU oracle for the hyperbolic-relaxation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * test of __graft_entry__ and bench.py's CPU-baseline leg call it to verify
 * (or time beside) the GPU library.  Nothing in the product links it.
 *
 * It restates, in plain scalar C, the algorithm of NRPyElliptic's generated
 * hot-path code (paths relative to the reference project):
 *   oracle_rhs_eval                 NRPyElliptic_Ccodes/rhs_eval.c:7-117
 *   oracle_residual_all_points      NRPyElliptic_Ccodes/residual_all_points.c:7-112
 *   oracle_apply_bcs_outerradiation_and_inner
 *                                   NRPyElliptic_Ccodes/apply_bcs_outerradiation_and_inner.c:6-469
 *   oracle_apply_bcs_inner_only     NRPyElliptic_Ccodes/apply_bcs_inner_only.c:11-27
 *   oracle_apply_bcs_outerextrap_and_inner
 *                                   NRPyElliptic_Ccodes/apply_bcs_outerextrap_and_inner.c:15-75
 *   oracle_MoL_step_forward_in_time NRPyElliptic_Ccodes/MoL_step_forward_in_time.c:7-178
 *   oracle_L2_norm_of_gf            NRPyElliptic_Ccodes/L2_norm_of_gf.c:6-43
 *   oracle_relax                    NRPyElliptic_Ccodes/main.c:138-187 with the stop test of
 *                                   NRPyEllipticET/.../..._Hyperbolic_Relaxation.c:185-224
 * The reference's SIMD code fixes every fused multiply-add explicitly
 * (SIMD/SIMD_intrinsics.h); here the same operations are written with fma()
 * and the file is compiled with -ffp-contract=off, so rhs_eval and
 * residual_all_points reproduce the AVX2/AVX-512 reference bit for bit.
 * The boundary-condition and L2 code of the reference is scalar C whose
 * multiply-add contraction is left to the compiler, so agreement there is to
 * rounding.  Parity of this file with the reference is pinned by the golden
 * vectors in tests/golden/ (generated from a build of the reference's own
 * sources by tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "nrpyell_abi.h"

#define IDX3(N0, N1, i0, i1, i2) ((long)(i0) + (long)(N0) * ((long)(i1) + (long)(N1) * (long)(i2)))

/* ---------------------------------------------------------------- RHS --- */

typedef struct {
  double c, m[6], p[6], jm[6], jp[6], km[6], kp[6];
} star_t;

static void load_star(const double *u, long idx, long s1, long s2, star_t *s) {
  s->c = u[idx];
  for (int k = 1; k <= 5; k++) {
    s->m[k] = u[idx - k];
    s->p[k] = u[idx + k];
    s->jm[k] = u[idx - k * s1];
    s->jp[k] = u[idx + k * s1];
    s->km[k] = u[idx - k * s2];
    s->kp[k] = u[idx + k * s2];
  }
}

/* first derivative, rhs_eval.c:87 */
static double d1(const double *m, const double *p, double invdx) {
  return invdx * fma(5.0 / 504.0, m[4] - p[4],
                     fma(5.0 / 6.0, p[1] - m[1],
                         fma(5.0 / 84.0, p[3] - m[3], fma(1.0 / 1260.0, p[5] - m[5], (5.0 / 21.0) * (m[2] - p[2])))));
}

/* second derivative, rhs_eval.c:89 */
static double d2(const double *m, const double *p, double centre, double invdx) {
  return (invdx * invdx) *
         fma(5.0 / 126.0, m[3] + p[3],
             fma(5.0 / 3.0, m[1] + p[1],
                 fma(1.0 / 3150.0, m[5] + p[5],
                     -fma(5.0 / 1008.0, m[4] + p[4], fma(5.0 / 21.0, m[2] + p[2], centre)))));
}

/* bracket of the vv RHS (= residual), rhs_eval.c:106-110 */
static double bracket(const paramstruct *P, const rfm_struct *r, int i0, int i1, const star_t *s, double psi,
                      double AA) {
  const int N0 = P->Nxx_plus_2NGHOSTS0;
  const double f0 = r->f0_of_xx0[i0], f0_D0 = r->f0_of_xx0__D0[i0], f0_DD00 = r->f0_of_xx0__DD00[i0];
  const double f1 = r->f1_of_xx1[i1], f1_D1 = r->f1_of_xx1__D1[i1];
  const double f2 = r->f2_of_xx0_xx1[i0 + N0 * i1], f2_D0 = r->f2_of_xx0_xx1__D0[i0 + N0 * i1];
  const double f3 = r->f3_of_xx0[i0], f3_D0 = r->f3_of_xx0__D0[i0];
  const double FD0 = (5269.0 / 1800.0) * s->c;
  const double u0 = d1(s->m, s->p, P->invdx0);
  const double u1 = d1(s->jm, s->jp, P->invdx1);
  const double u00 = d2(s->m, s->p, FD0, P->invdx0);
  const double u11 = d2(s->jm, s->jp, FD0, P->invdx1);
  const double u22 = d2(s->km, s->kp, FD0, P->invdx2);
  const double P0 = 1.0 / (f2 * f2);
  const double P2 = (f3 * f3) / (f0_D0 * f0_D0);
  const double P3 = 1.0 / ((f2 * f2) * f2);
  const double pu = psi + s->c;
  const double pow7 = (((((pu * pu) * pu) * pu) * pu) * pu) * pu;
  const double ta = ((P0 * -1.0) * ((f3 * f3) / f0_D0)) / f0;
  const double tb = fma(P2, P3 * f2_D0, -ta);
  const double tc = fma(f3, fma(f0_D0, f2_D0, f0_DD00 * f2), -(f0_D0 * (f2 * f3_D0))) / ((f0_D0 * f0_D0) * f0_D0);
  const double td = fma(P3 * f3, tc, -tb);
  const double te = fma(P0, u11, -(u0 * td));
  const double tf = fma(P0 * f1_D1, u1 / f1, te);
  const double tg = fma(1.0 / 8.0, AA / pow7, tf);
  const double th = fma(P0, P2 * u00, tg);
  return fma(u22, (1.0 / (f1 * f1)) / (f0 * f0), th);
}

void oracle_rhs_eval(const paramstruct *P, const rfm_struct *r, const double *aux, const double *in, double *rhs) {
  const int N0 = P->Nxx_plus_2NGHOSTS0, N1 = P->Nxx_plus_2NGHOSTS1, N2 = P->Nxx_plus_2NGHOSTS2;
  const long Ntot = (long)N0 * N1 * N2;
#pragma omp parallel for
  for (int i2 = NGHOSTS; i2 < NGHOSTS + P->Nxx2; i2++)
    for (int i1 = NGHOSTS; i1 < NGHOSTS + P->Nxx1; i1++)
      for (int i0 = NGHOSTS; i0 < NGHOSTS + P->Nxx0; i0++) {
        const long idx = IDX3(N0, N1, i0, i1, i2);
        star_t s;
        load_star(in, idx, N0, (long)N0 * N1, &s);
        const double ws = aux[WAVESPEEDGF * Ntot + idx];
        const double b = bracket(P, r, i0, i1, &s, aux[PSI_BACKGROUNDGF * Ntot + idx], aux[ADD_TIMES_AUUGF * Ntot + idx]);
        rhs[UUGF * Ntot + idx] = fma(-P->eta_damping, s.c, in[VVGF * Ntot + idx]);
        rhs[VVGF * Ntot + idx] = (ws * ws) * b;
      }
}

void oracle_residual_all_points(const paramstruct *P, const rfm_struct *r, const double *aux, const double *in,
                                double *res) {
  const int N0 = P->Nxx_plus_2NGHOSTS0, N1 = P->Nxx_plus_2NGHOSTS1, N2 = P->Nxx_plus_2NGHOSTS2;
  const long Ntot = (long)N0 * N1 * N2;
#pragma omp parallel for
  for (int i2 = NGHOSTS; i2 < NGHOSTS + P->Nxx2; i2++)
    for (int i1 = NGHOSTS; i1 < NGHOSTS + P->Nxx1; i1++)
      for (int i0 = NGHOSTS; i0 < NGHOSTS + P->Nxx0; i0++) {
        const long idx = IDX3(N0, N1, i0, i1, i2);
        star_t s;
        load_star(in, idx, N0, (long)N0 * N1, &s);
        res[UUGF * Ntot + idx] =
            bracket(P, r, i0, i1, &s, aux[PSI_BACKGROUNDGF * Ntot + idx], aux[ADD_TIMES_AUUGF * Ntot + idx]);
      }
}

/* ------------------------------------------------------- boundaries --- */

/* Exact 11-point first-derivative weights for upwind offsets -5..5: row
 * k+5, entry j weights node k-5+j (apply_bcs_outerradiation_and_inner.c:6-286). */
static const double FD1W[11][11] = {
    {1.0 / 10, -10.0 / 9, 45.0 / 8, -120.0 / 7, 35.0, -252.0 / 5, 105.0 / 2, -40.0, 45.0 / 2, -10.0, 7381.0 / 2520},
    {-1.0 / 90, 1.0 / 8, -9.0 / 14, 2.0, -21.0 / 5, 63.0 / 10, -7.0, 6.0, -9.0 / 2, 4609.0 / 2520, 1.0 / 10},
    {1.0 / 360, -2.0 / 63, 1.0 / 6, -8.0 / 15, 7.0 / 6, -28.0 / 15, 7.0 / 3, -8.0 / 3, 341.0 / 280, 2.0 / 9, -1.0 / 90},
    {-1.0 / 840, 1.0 / 72, -3.0 / 40, 1.0 / 4, -7.0 / 12, 21.0 / 20, -7.0 / 4, 319.0 / 420, 3.0 / 8, -1.0 / 24, 1.0 / 360},
    {1.0 / 1260, -1.0 / 105, 3.0 / 56, -4.0 / 21, 1.0 / 2, -6.0 / 5, 11.0 / 30, 4.0 / 7, -3.0 / 28, 1.0 / 63, -1.0 / 840},
    {-1.0 / 1260, 5.0 / 504, -5.0 / 84, 5.0 / 21, -5.0 / 6, 0.0, 5.0 / 6, -5.0 / 21, 5.0 / 84, -5.0 / 504, 1.0 / 1260},
    {1.0 / 840, -1.0 / 63, 3.0 / 28, -4.0 / 7, -11.0 / 30, 6.0 / 5, -1.0 / 2, 4.0 / 21, -3.0 / 56, 1.0 / 105, -1.0 / 1260},
    {-1.0 / 360, 1.0 / 24, -3.0 / 8, -319.0 / 420, 7.0 / 4, -21.0 / 20, 7.0 / 12, -1.0 / 4, 3.0 / 40, -1.0 / 72, 1.0 / 840},
    {1.0 / 90, -2.0 / 9, -341.0 / 280, 8.0 / 3, -7.0 / 3, 28.0 / 15, -7.0 / 6, 8.0 / 15, -1.0 / 6, 2.0 / 63, -1.0 / 360},
    {-1.0 / 10, -4609.0 / 2520, 9.0 / 2, -6.0, 7.0, -63.0 / 10, 21.0 / 5, -2.0, 9.0 / 14, -1.0 / 8, 1.0 / 90},
    {-7381.0 / 2520, 10.0, -45.0 / 2, 40.0, -105.0 / 2, 252.0 / 5, -35.0, 120.0 / 7, -45.0 / 8, 10.0 / 9, -1.0 / 10},
};

static double fd1_upwind(const double *f, long idx, long stride, int off, double invdx) {
  double s = 0.0;
  int first = 1;
  for (int j = 0; j < 11; j++) {
    if (off == 0 && j == 5) continue; /* the centred stencil has no centre term */
    const double t = FD1W[off + 5][j] * f[idx + (long)(off - 5 + j) * stride];
    s = first ? t : s + t;
    first = 0;
  }
  return s * invdx;
}

/* r and d xx^i / d r of SinhSymTP, the closed form of
 * apply_bcs_outerradiation_and_inner.c:295-320 */
static void r_and_dxdr(const paramstruct *P, double xx0, double xx1, double *r, double *dx0dr, double *dx1dr) {
  const double s = sin(xx1), c = cos(xx1);
  const double iw = 1.0 / P->SINHWAA;
  const double ep = exp(iw * xx0), em = exp(-iw * xx0);
  const double E = ep - em;
  const double K = (P->AMAX * P->AMAX) / ((exp(iw) - exp(-iw)) * (exp(iw) - exp(-iw)));
  const double A2 = (E * E) * K;
  const double B2 = P->bScale * P->bScale + A2;
  const double Bc2 = B2 * (c * c);
  const double R2 = (s * s) * A2 + Bc2;
  const double R = sqrt(R2);
  const double B = sqrt(B2);
  const double iR = 1.0 / R;
  const double T18 = -s * B2 * c + s * A2 * c;
  const double iR3 = pow(R2, -3.0 / 2.0);
  const double T20 = -s * B * iR - B * T18 * iR3 * c;
  const double T21 = 1.0 / sqrt(-Bc2 / R2 + 1);
  const double dA2h = (1.0 / 2.0) * E * K * (2 * iw * ep + 2 * iw * em);
  const double T24 = (s * s) * dA2h + dA2h * (c * c);
  const double T25 = -B * iR3 * T24 * c + iR * dA2h * c / B;
  const double T26 = T21 / (iR * T18 * T21 * T25 - iR * T20 * T21 * T24);
  *r = R;
  *dx0dr = -T20 * T26;
  *dx1dr = T25 * T26;
}

static int upwind_offset(int face, int i, int n) {
  if (i < 5) return 5 - i;
  if (i > n - 5 - 1) return (n - 5 - 1) - i;
  return face;
}

static double partial_r_f(const paramstruct *P, const double *f, int i0, int i1, int i2, int F0, int F1,
                          double dx0dr, double dx1dr) {
  const int N0 = P->Nxx_plus_2NGHOSTS0, N1 = P->Nxx_plus_2NGHOSTS1;
  const long idx = IDX3(N0, N1, i0, i1, i2);
  const double d0 = fd1_upwind(f, idx, 1, upwind_offset(F0, i0, N0), P->invdx0);
  const double d1v = fd1_upwind(f, idx, N0, upwind_offset(F1, i1, N1), P->invdx1);
  return dx0dr * d0 + dx1dr * d1v + 0.0 * 0.0;
}

void oracle_apply_bcs_inner_only(const paramstruct *P, const bc_struct *bc, double *gfs) {
  const long Ntot = (long)P->Nxx_plus_2NGHOSTS0 * P->Nxx_plus_2NGHOSTS1 * P->Nxx_plus_2NGHOSTS2;
  for (int pt = 0; pt < bc->bc_info.num_inner_boundary_points; pt++)
    for (int gf = 0; gf < NUM_EVOL_GFS; gf++) {
      const innerpt_bc_struct *e = &bc->inner_bc_array[pt];
      gfs[gf * Ntot + e->dstpt] = e->parity[0] * gfs[gf * Ntot + e->srcpt];
    }
}

void oracle_apply_bcs_outerradiation_and_inner(const paramstruct *P, const bc_struct *bc, REAL *NRPYELL_RESTRICT xx[3],
                                               const double c_gf[NUM_EVOL_GFS], const double finf[NUM_EVOL_GFS],
                                               double *gfs, double *rhs) {
  const int N0 = P->Nxx_plus_2NGHOSTS0, N1 = P->Nxx_plus_2NGHOSTS1, N2 = P->Nxx_plus_2NGHOSTS2;
  const long Ntot = (long)N0 * N1 * N2;
  for (int gz = 0; gz < NGHOSTS; gz++)
    for (int dirn = 0; dirn < 3; dirn++)
      for (int k = 0; k < bc->bc_info.num_pure_outer_boundary_points[gz][dirn]; k++) {
        const outerpt_bc_struct *o = &bc->pure_outer_bc_array[dirn + 3 * gz][k];
        const int i0 = o->i0, i1 = o->i1, i2 = o->i2;
        const int F0 = o->FACEX0, F1 = o->FACEX1, F2 = o->FACEX2;
        const int j0 = i0 + F0, j1 = i1 + F1, j2 = i2 + F2;
        double r, a0, a1, rn, b0, b1;
        r_and_dxdr(P, xx[0][i0], xx[1][i1], &r, &a0, &a1);
        r_and_dxdr(P, xx[0][j0], xx[1][j1], &rn, &b0, &b1);
        const long idx = IDX3(N0, N1, i0, i1, i2), idxn = IDX3(N0, N1, j0, j1, j2);
        for (int gf = 0; gf < NUM_EVOL_GFS; gf++) {
          const double *f = gfs + gf * Ntot;
          const double drf = partial_r_f(P, f, i0, i1, i2, F0, F1, a0, a1);
          const double drfn = partial_r_f(P, f, j0, j1, j2, F0, F1, b0, b1);
          const double c = c_gf[gf], fi = finf[gf];
          const double out_int = -c * (drfn + (f[idxn] - fi) / rn);
          const double K = rn * rn * rn * (rhs[gf * Ntot + idxn] - out_int);
          const double rinv = 1.0 / r;
          const double out = -c * (drf + (f[idx] - fi) * rinv);
          rhs[gf * Ntot + idx] = out + K * rinv * rinv * rinv;
        }
      }
  oracle_apply_bcs_inner_only(P, bc, rhs);
}

void oracle_apply_bcs_outerextrap_and_inner(const paramstruct *P, const bc_struct *bc, double *gfs) {
  const int N0 = P->Nxx_plus_2NGHOSTS0, N1 = P->Nxx_plus_2NGHOSTS1, N2 = P->Nxx_plus_2NGHOSTS2;
  const long Ntot = (long)N0 * N1 * N2;
  for (int gz = 0; gz < NGHOSTS; gz++)
    for (int dirn = 0; dirn < 3; dirn++)
      for (int k = 0; k < bc->bc_info.num_pure_outer_boundary_points[gz][dirn]; k++) {
        const outerpt_bc_struct *o = &bc->pure_outer_bc_array[dirn + 3 * gz][k];
        const long i_0 = IDX3(N0, N1, o->i0, o->i1, o->i2);
        const long i_1 = IDX3(N0, N1, o->i0 + o->FACEX0, o->i1 + o->FACEX1, o->i2 + o->FACEX2);
        const long i_2 = IDX3(N0, N1, o->i0 + 2 * o->FACEX0, o->i1 + 2 * o->FACEX1, o->i2 + 2 * o->FACEX2);
        const long i_3 = IDX3(N0, N1, o->i0 + 3 * o->FACEX0, o->i1 + 3 * o->FACEX1, o->i2 + 3 * o->FACEX2);
        for (int gf = 0; gf < NUM_EVOL_GFS; gf++) {
          double *g = gfs + gf * Ntot;
          g[i_0] = +3.0 * g[i_1] - 3.0 * g[i_2] + 1.0 * g[i_3];
        }
      }
  oracle_apply_bcs_inner_only(P, bc, gfs);
}

/* ---------------------------------------------------------- RK4 step --- */

void oracle_MoL_step_forward_in_time(griddata_struct *g, const double dt) {
  const paramstruct *P = &g->params;
  MoL_gridfunctions_struct *G = &g->gridfuncs;
  const long n = (long)P->Nxx_plus_2NGHOSTS0 * P->Nxx_plus_2NGHOSTS1 * P->Nxx_plus_2NGHOSTS2 * NUM_EVOL_GFS;
  const double cw[2] = {P->uu_wavespeed_at_OB, P->vv_wavespeed_at_OB};
  const double finf[2] = {0.0, 0.0};
  double *in[4] = {G->y_n_gfs, G->k_odd_gfs, G->k_even_gfs, G->k_odd_gfs};
  double *kk[4] = {G->k_odd_gfs, G->k_even_gfs, G->k_odd_gfs, G->k_even_gfs};
  double *acc = G->y_nplus1_running_total_gfs, *y = G->y_n_gfs;
  for (int s = 0; s < 4; s++) {
    oracle_rhs_eval(P, &g->rfmstruct, G->auxevol_gfs, in[s], kk[s]);
    if (P->outer_bc_type == RADIATION_OUTER_BCS)
      oracle_apply_bcs_outerradiation_and_inner(P, &g->bcstruct, g->xx, cw, finf, in[s], kk[s]);
    double *k = kk[s];
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
      const double dk = dt * k[i];
      if (s == 0) {
        acc[i] = (1.0 / 6.0) * dk;
        k[i] = fma(1.0 / 2.0, dk, y[i]);
      } else if (s == 1) {
        acc[i] = fma(1.0 / 3.0, dk, acc[i]);
        k[i] = fma(1.0 / 2.0, dk, y[i]);
      } else if (s == 2) {
        acc[i] = fma(1.0 / 3.0, dk, acc[i]);
        k[i] = fma(dt, k[i], y[i]);
      } else {
        y[i] = y[i] + fma(1.0 / 6.0, dk, acc[i]);
      }
    }
    if (P->outer_bc_type == EXTRAPOLATION_OUTER_BCS)
      oracle_apply_bcs_outerextrap_and_inner(P, &g->bcstruct, s == 3 ? y : k);
  }
}

/* ---------------------------------------------------------------- L2 --- */

double oracle_L2_norm_of_gf(const paramstruct *P, const int gf_index, const double R, REAL *NRPYELL_RESTRICT xx[3], const double *in_gf) {
  const int N0 = P->Nxx_plus_2NGHOSTS0, N1 = P->Nxx_plus_2NGHOSTS1, N2 = P->Nxx_plus_2NGHOSTS2;
  const long Ntot = (long)N0 * N1 * N2;
  const double AMAX = P->AMAX, b = P->bScale;
  double sq = 0.0, vol = 0.0;
  for (int i2 = NGHOSTS; i2 < NGHOSTS + P->Nxx2; i2++)
    for (int i1 = NGHOSTS; i1 < NGHOSTS + P->Nxx1; i1++)
      for (int i0 = NGHOSTS; i0 < NGHOSTS + P->Nxx0; i0++) {
        const double x0 = xx[0][i0], x1 = xx[1][i1];
        const double s = sin(x1);
        const double iw = 1.0 / P->SINHWAA;
        const double D = exp(iw) - exp(-iw);
        const double ep = exp(iw * x0), em = exp(-iw * x0);
        const double E2 = (ep - em) * (ep - em);
        const double A2 = AMAX * AMAX * E2 / (D * D);
        const double B2 = b * b + A2;
        const double r = sqrt((s * s) * A2 + B2 * (cos(x1) * cos(x1)));
        const double q = b * b * (s * s) + A2;
        const double sdg = AMAX * AMAX * sqrt(E2 * (q * q) * ((iw * ep + iw * em) * (iw * ep + iw * em)) / (B2 * (D * D * D * D))) * fabs(s);
        if (r < R) {
          const double gv = in_gf[gf_index * Ntot + IDX3(N0, N1, i0, i1, i2)];
          const double dV = sdg * P->dxx0 * P->dxx1 * P->dxx2;
          sq += gv * gv * dV;
          vol += dV;
        }
      }
  return log10(1e-16 + sqrt(sq / vol));
}

/* --------------------------------------------------------- relaxation --- */

int oracle_relax(griddata_struct *g, const double dt, const double log10_tol, const int max_steps, const double R,
                 double *history, int *steps_taken) {
  int n = 0;
  int converged = 0;
  for (n = 0; n <= max_steps; n++) {
    oracle_residual_all_points(&g->params, &g->rfmstruct, g->gridfuncs.auxevol_gfs, g->gridfuncs.y_n_gfs,
                               g->gridfuncs.diagnostic_output_gfs);
    const double l2 = oracle_L2_norm_of_gf(&g->params, UUGF, R, g->xx, g->gridfuncs.diagnostic_output_gfs);
    if (history) history[n] = l2;
    if (l2 <= log10_tol) {
      converged = 1;
      break;
    }
    if (n == max_steps) break;
    oracle_MoL_step_forward_in_time(g, dt);
  }
  if (steps_taken) *steps_taken = n;
  return converged ? 0 : 1;
}

/* Wall time (seconds) of n_iter iterations of the main.c loop body --
 * residual, L2 norm, one RK4 step -- for the CPU-baseline leg of bench.py. */
#include <omp.h>
double oracle_time_iterations(griddata_struct *g, const double dt, const int n_iter, const double R) {
  const double t0 = omp_get_wtime();
  for (int n = 0; n < n_iter; n++) {
    oracle_residual_all_points(&g->params, &g->rfmstruct, g->gridfuncs.auxevol_gfs, g->gridfuncs.y_n_gfs,
                               g->gridfuncs.diagnostic_output_gfs);
    volatile double l2 = oracle_L2_norm_of_gf(&g->params, UUGF, R, g->xx, g->gridfuncs.diagnostic_output_gfs);
    (void)l2;
    oracle_MoL_step_forward_in_time(g, dt);
  }
  return omp_get_wtime() - t0;
}
