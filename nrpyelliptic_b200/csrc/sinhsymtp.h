// SinhSymTP coordinate helpers shared by host set-up code and device set-up
// kernels.  SinhSymTP maps (xx0, xx1, xx2) in (0,1) x (0,pi) x (-pi,pi) to
//   A   = AMAX * sinh(xx0/SINHWAA) / sinh(1/SINHWAA)
//   x   = A sin(xx1) cos(xx2),  y = A sin(xx1) sin(xx2),
//   z   = sqrt(A^2 + bScale^2) cos(xx1)
// (reference: reference_metric.py:308-345; the generated C writes the sinh
// ratio as (exp(a)-exp(-a))/(exp(b)-exp(-b)), e.g.
// rfm_precompute_rfmstruct_define.c:64).
#ifndef NRPYELL_SINHSYMTP_H
#define NRPYELL_SINHSYMTP_H

#include <math.h>

#if defined(__CUDACC__)
#define NRPYELL_HD __host__ __device__ inline
#else
#define NRPYELL_HD static inline
#endif

// A(xx0) written as the generated code writes it in the L2-norm and BC helpers
// (tmp = 1/SINHWAA; exp(tmp*xx0) - exp(-tmp*xx0)).
NRPYELL_HD double symtp_A_invw(double AMAX, double SINHWAA, double xx0) {
  const double iw = 1.0 / SINHWAA;
  return AMAX * (exp(iw * xx0) - exp(-iw * xx0)) / (exp(iw) - exp(-iw));
}

// Cartesian position of a SinhSymTP grid point.
NRPYELL_HD void symtp_xx_to_cart(double AMAX, double SINHWAA, double bScale, double xx0, double xx1,
                                 double xx2, double X[3]) {
  const double iw = 1.0 / SINHWAA;
  const double den = exp(iw) - exp(-iw);
  const double num = exp(iw * xx0) - exp(-iw * xx0);
  const double As = AMAX * num * sin(xx1) / den;
  X[0] = As * cos(xx2);
  X[1] = As * sin(xx2);
  X[2] = sqrt(AMAX * AMAX * num * num / (den * den) + bScale * bScale) * cos(xx1);
}

// A_ij A^ij of the Bowen-York conformal extrinsic curvature (flat conformal
// metric, Cartesian components) for two punctures.  The vector potential is
//   V^i = sum_n [ -7/4 P^i / r - 1/4 (x.P) x^i / r^3 + (x cross S)^i / r^3 ]
// with x the position relative to puncture n (NRPyElliptic_SourceTerm.py:48-74)
// and A_ij = d_j V_i + d_i V_j - 2/3 delta_ij div V (:77-126).  The
// derivatives below are the closed forms of those expressions:
//   d_j V_i = 7/4 P_i x_j/r^3 - 1/4 P_j x_i/r^3 - 1/4 (x.P) delta_ij/r^3
//             + 3/4 (x.P) x_i x_j/r^5 + eps_ijk S_k/r^3 - 3 (x cross S)_i x_j/r^5
struct ByPuncture {
  double pos[3], P[3], S[3];
};

NRPYELL_HD void by_dV_accumulate(const ByPuncture& p, const double X[3], double dV[3][3]) {
  const double x[3] = {X[0] - p.pos[0], X[1] - p.pos[1], X[2] - p.pos[2]};
  const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
  const double r = sqrt(r2);
  const double ir3 = 1.0 / (r2 * r);
  const double ir5 = ir3 / r2;
  const double xP = x[0] * p.P[0] + x[1] * p.P[1] + x[2] * p.P[2];
  const double xS[3] = {x[1] * p.S[2] - x[2] * p.S[1], x[2] * p.S[0] - x[0] * p.S[2],
                        x[0] * p.S[1] - x[1] * p.S[0]};
  // eps_ijk S_k as a matrix
  const double eS[3][3] = {{0.0, p.S[2], -p.S[1]}, {-p.S[2], 0.0, p.S[0]}, {p.S[1], -p.S[0], 0.0}};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double v = 1.75 * p.P[i] * x[j] * ir3 - 0.25 * p.P[j] * x[i] * ir3 + 0.75 * xP * x[i] * x[j] * ir5 +
                 eS[i][j] * ir3 - 3.0 * xS[i] * x[j] * ir5;
      if (i == j) v -= 0.25 * xP * ir3;
      dV[i][j] += v;
    }
}

NRPYELL_HD double by_AA(const ByPuncture& p0, const ByPuncture& p1, const double X[3]) {
  double dV[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  by_dV_accumulate(p0, X, dV);
  by_dV_accumulate(p1, X, dV);
  const double div = dV[0][0] + dV[1][1] + dV[2][2];
  double aa = 0.0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double a = dV[i][j] + dV[j][i];
      if (i == j) a -= (2.0 / 3.0) * div;
      aa += a * a;
    }
  return aa;
}

// Brill-Lindquist background conformal factor, 1 + sum_n m_n / (2 r_n)
// (NRPyElliptic_SourceTerm.py:180-203).
NRPYELL_HD double bl_psi(double m0, const double p0[3], double m1, const double p1[3], const double X[3]) {
  const double a0 = X[0] - p0[0], b0 = X[1] - p0[1], c0 = X[2] - p0[2];
  const double a1 = X[0] - p1[0], b1 = X[1] - p1[1], c1 = X[2] - p1[2];
  return 1.0 + m0 / (2.0 * sqrt(a0 * a0 + b0 * b0 + c0 * c0)) + m1 / (2.0 * sqrt(a1 * a1 + b1 * b1 + c1 * c1));
}

// Proper grid spacings along the three SinhSymTP directions; their minimum
// sets the time step and the wavespeed gridfunction
// (find_timestep.c:24-36, wavespeed_gf_all_points.c:23-35).
NRPYELL_HD void symtp_ds(double AMAX, double SINHWAA, double bScale, double dxx0, double dxx1, double dxx2,
                         double xx0, double xx1, double ds[3]) {
  const double s1 = sin(xx1);
  const double iw = 1.0 / SINHWAA;
  const double den = exp(iw) - exp(-iw);
  const double ep = exp(iw * xx0), em = exp(-iw * xx0);
  const double sh = ep - em;
  const double A2 = AMAX * AMAX * sh * sh / (den * den);
  const double rho = sqrt(bScale * bScale * s1 * s1 + A2);
  const double Aden = AMAX / den;
  ds[0] = dxx0 * Aden * rho * (iw * ep + iw * em) / sqrt(bScale * bScale + A2);
  ds[1] = dxx1 * rho;
  ds[2] = dxx2 * s1 * Aden * sh;
}

// Source point of a ghost point on the cell-centred SymTP grid (NGHOSTS = 5
// ghost layers around Nxx0 x Nxx1 x Nxx2 interior points):
//   xx0 < 0          -> xx0' = -xx0, xx2' = xx2 + pi   (A -> -A flips x and y)
//   xx1 < 0 or > pi  -> xx1' = -xx1 or 2pi - xx1, xx2' = xx2 + pi
//   xx2 outside [-pi, pi) -> wrap by 2pi
// The outer xx0 face has no image: a point there maps to itself unless one of
// its other coordinates is reflected.  This is the round trip
// xx -> Cartesian -> xx of bcstruct_set_up.c:27-194 written on indices.
NRPYELL_HD void symtp_ghost_source(int i0, int i1, int i2, int Nxx1, int Nxx2, int out[3]) {
  const int NG = 5;
  int shift = 0;
  if (i0 < NG) {
    i0 = 2 * NG - 1 - i0;
    shift ^= 1;
  }
  if (i1 < NG) {
    i1 = 2 * NG - 1 - i1;
    shift ^= 1;
  } else if (i1 >= NG + Nxx1) {
    i1 = 2 * (NG + Nxx1) - 1 - i1;
    shift ^= 1;
  }
  int j = i2 - NG;
  if (shift) j += Nxx2 / 2;
  j %= Nxx2;
  if (j < 0) j += Nxx2;
  out[0] = i0;
  out[1] = i1;
  out[2] = j + NG;
}

// Reference-metric scale factors at one xx0 (rfm_precompute_rfmstruct_define.c:5-93).
// With E(x) = exp(x/w) - exp(-x/w), D = exp(1/w) - exp(-1/w), A = AMAX E/D:
// o = {f0 = A, d f0, d2 f0, d3 f0, f3 = sqrt(A^2 + b^2), d f3, d2 f3} (d = d/d xx0).
NRPYELL_HD void symtp_rfm_xx0(double AMAX, double SINHWAA, double bScale, double x, double o[7]) {
  const double D = exp(1.0 / SINHWAA) - exp(-1 / SINHWAA);
  const double ep = exp(x / SINHWAA), em = exp(-x / SINHWAA);
  o[0] = AMAX * (ep - em) / D;
  o[1] = AMAX * (ep / SINHWAA + em / SINHWAA) / D;
  o[2] = AMAX * (ep / pow(SINHWAA, 2) - em / pow(SINHWAA, 2)) / D;
  o[3] = AMAX * (ep / pow(SINHWAA, 3) + em / pow(SINHWAA, 3)) / D;
  const double A2 = pow(AMAX, 2) * pow(ep - em, 2) / pow(D, 2);
  const double f3 = sqrt(A2 + pow(bScale, 2));
  const double dA2 = (1.0 / 2.0) * pow(AMAX, 2) * (2 * ep / SINHWAA + 2 * em / SINHWAA) * (ep - em);  // (A^2)'/2 * D^2
  o[4] = f3;
  o[5] = dA2 / (f3 * pow(D, 2));
  o[6] = -1.0 / 4.0 * pow(AMAX, 4) * pow(2 * ep / SINHWAA + 2 * em / SINHWAA, 2) * pow(ep - em, 2) /
             (pow(A2 + pow(bScale, 2), 3.0 / 2.0) * pow(D, 4)) +
         (1.0 / 2.0) * pow(AMAX, 2) * (2 * ep / pow(SINHWAA, 2) - 2 * em / pow(SINHWAA, 2)) * (ep - em) / (f3 * pow(D, 2)) +
         (1.0 / 2.0) * pow(AMAX, 2) * (ep / SINHWAA + em / SINHWAA) * (2 * ep / SINHWAA + 2 * em / SINHWAA) / (f3 * pow(D, 2));
}

// f2 = sqrt(A^2 + b^2 sin^2 xx1) and its derivatives at (xx0, xx1):
// o = {f2, d f2/d xx0, d f2/d xx1, d2 f2/d xx0^2, d2 f2/d xx1^2}.
NRPYELL_HD void symtp_rfm_f2(double AMAX, double SINHWAA, double bScale, double x, double y, double o[5]) {
  const double D = exp(1.0 / SINHWAA) - exp(-1 / SINHWAA);
  const double s = sin(y), c = cos(y);
  const double ep = exp(x / SINHWAA), em = exp(-x / SINHWAA);
  const double A2 = pow(AMAX, 2) * pow(ep - em, 2) / pow(D, 2);
  const double q = A2 + pow(bScale, 2) * pow(s, 2);
  const double f2 = sqrt(q);
  o[0] = f2;
  o[1] = (1.0 / 2.0) * pow(AMAX, 2) * (2 * ep / SINHWAA + 2 * em / SINHWAA) * (ep - em) / (f2 * pow(D, 2));
  o[2] = pow(bScale, 2) * s * c / f2;
  o[3] = -1.0 / 4.0 * pow(AMAX, 4) * pow(2 * ep / SINHWAA + 2 * em / SINHWAA, 2) * pow(ep - em, 2) /
             (pow(q, 3.0 / 2.0) * pow(D, 4)) +
         (1.0 / 2.0) * pow(AMAX, 2) * (2 * ep / pow(SINHWAA, 2) - 2 * em / pow(SINHWAA, 2)) * (ep - em) / (f2 * pow(D, 2)) +
         (1.0 / 2.0) * pow(AMAX, 2) * (ep / SINHWAA + em / SINHWAA) * (2 * ep / SINHWAA + 2 * em / SINHWAA) / (f2 * pow(D, 2));
  o[4] = -pow(bScale, 4) * pow(s, 2) * pow(c, 2) / pow(q, 3.0 / 2.0) - pow(bScale, 2) * pow(s, 2) / f2 +
         pow(bScale, 2) * pow(c, 2) / f2;
}

// The metric factors of the vv right-hand side (rhs_eval.c:106-110) folded
// into one weight per raw stencil sum (ix = 1/dxx): cs = {d22 weight, d00
// weight, d11 weight, d1 weight, d0 weight, centre weight}.
NRPYELL_HD void symtp_fold_rhs_coefs(double f0, double f0p, double f0pp, double f1, double f1p, double f2,
                                     double f2_0, double f3, double f3p, double ix0, double ix1, double ix2,
                                     double cs[6]) {
  const double P0 = 1.0 / (f2 * f2);
  const double P2 = (f3 * f3) / (f0p * f0p);
  const double P3 = 1.0 / ((f2 * f2) * f2);
  const double ta = ((P0 * -1.0) * ((f3 * f3) / f0p)) / f0;
  const double tb = P2 * (P3 * f2_0) - ta;
  const double tc = (f3 * (f0p * f2_0 + f0pp * f2) - f0p * (f2 * f3p)) / ((f0p * f0p) * f0p);
  const double td = (P3 * f3) * tc - tb;
  const double c22 = ((1.0 / (f1 * f1)) / (f0 * f0)) * (ix2 * ix2);
  const double c00 = P0 * P2 * (ix0 * ix0);
  const double c11 = P0 * (ix1 * ix1);
  cs[0] = c22;
  cs[1] = c00;
  cs[2] = c11;
  cs[3] = (P0 * f1p / f1) * ix1;
  cs[4] = -td * ix0;
  cs[5] = -(5269.0 / 1800.0) * (c00 + c11 + c22);
}

// r and (d xx0/d r, d xx1/d r) at fixed spherical angles, for SinhSymTP at
// (xx0, xx1); the azimuthal component is zero.  The reference evaluates a
// generated closed form (apply_bcs_outerradiation_and_inner.c:290-321); the
// same quantities follow from inverting the 2x2 Jacobian of
// (r, zeta = z/r) with respect to (xx0, xx1):
//   r^2 = A^2 + b^2 cos^2 xx1,  z = sqrt(A^2+b^2) cos xx1,
//   d r/d xx0 = A A'/r,          d r/d xx1 = -b^2 sin xx1 cos xx1 / r,
//   d zeta = (d z - zeta d r)/r,
//   d xx0/d r = (d zeta/d xx1)/det,  d xx1/d r = -(d zeta/d xx0)/det.
NRPYELL_HD void symtp_radial_geometry(double AMAX, double SINHWAA, double bScale, double xx0, double xx1,
                                      double* r_out, double* dx0dr, double* dx1dr) {
  const double iw = 1.0 / SINHWAA;
  const double D = exp(iw) - exp(-iw);
  const double ep = exp(iw * xx0), em = exp(-iw * xx0);
  const double A = AMAX * (ep - em) / D;
  const double Ap = AMAX * (iw * ep + iw * em) / D;
  const double s = sin(xx1), c = cos(xx1);
  const double b2 = bScale * bScale;
  const double B = sqrt(A * A + b2);
  const double r = sqrt(A * A * s * s + (A * A + b2) * c * c);
  const double drdx0 = A * Ap / r;
  const double drdx1 = -b2 * s * c / r;
  const double z = B * c;
  const double zeta = z / r;
  const double dzdx0 = A * Ap * c / B;
  const double dzdx1 = -B * s;
  const double dzetadx0 = (dzdx0 - zeta * drdx0) / r;
  const double dzetadx1 = (dzdx1 - zeta * drdx1) / r;
  const double det = drdx0 * dzetadx1 - drdx1 * dzetadx0;
  *r_out = r;
  *dx0dr = dzetadx1 / det;
  *dx1dr = -dzetadx0 / det;
}

// Upwind offset rule of compute_partial_r_f
// (apply_bcs_outerradiation_and_inner.c:352-360), stencil radius 5.
NRPYELL_HD int radiation_upwind_offset(int face, int i, int n) {
  int off = face;
  if (i < 5)
    off = 5 - i;
  else if (i > n - 5 - 1)
    off = (n - 5 - 1) - i;
  return off;
}

#endif
