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

#endif
