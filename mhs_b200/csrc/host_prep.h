// Host-side preparation shared by the CUDA library and the host test build:
// Gauss-Legendre rules and the per-material image coefficients.
#pragma once

#include <math.h>
#include <string.h>

#include "engine_base.cuh"

namespace mhs {

// Gauss-Legendre nodes (ascending) and weights on [-1, 1] for one order:
// Newton iteration on the three-term recurrence in long double, then the
// rule is symmetrised and its weights normalised to sum 2, as numpy's
// leggauss presents its rules.
inline void gauss_legendre(int n, double* xo, double* wo) {
  long double x[GL_MAX], w[GL_MAX];
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < n; ++i) {
    long double z = cosl(pi * (i + 0.75L) / (n + 0.5L));
    long double dp = 0.0L;
    for (int it = 0; it < 100; ++it) {
      long double p0 = 1.0L, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) { p1 = z; p0 = 1.0L; }
      dp = n * (z * p1 - p0) / (z * z - 1.0L);
      const long double dz = p1 / dp;
      z -= dz;
      if (fabsl(dz) < 1e-19L) break;
    }
    {  // derivative at the converged root
      long double p0 = 1.0L, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) { p1 = z; p0 = 1.0L; }
      dp = n * (z * p1 - p0) / (z * z - 1.0L);
    }
    x[n - 1 - i] = z;   // cos is descending in i
    w[n - 1 - i] = 2.0L / ((1.0L - z * z) * dp * dp);
  }
  long double xs[GL_MAX], ws[GL_MAX], sum = 0.0L;
  for (int i = 0; i < n; ++i) {
    xs[i] = 0.5L * (x[i] - x[n - 1 - i]);
    ws[i] = 0.5L * (w[i] + w[n - 1 - i]);
    sum += ws[i];
  }
  for (int i = 0; i < n; ++i) {
    xo[i] = (double)xs[i];
    wo[i] = (double)(ws[i] * (2.0L / sum));
  }
}

// Packed table of every order 1..GL_MAX (gl_offset layout).
inline void gauss_table(double* x, double* w) {
  for (int n = 1; n <= GL_MAX; ++n) gauss_legendre(n, x + gl_offset(n), w + gl_offset(n));
}

// Per-material image coefficients, laid out for ImageCoef:
//   r_dg[r][pz]  = scale * sum_pnu c[pz][pnu] nu^pnu   (R-family, 3 per record)
//   r_ddg[r][pz] likewise
//   q_dg[r]      = sum_pnu c[pnu] nu^pnu                (Q-family; scale after)
//   q_ddg[r]     likewise
// Total doubles: 3 * (MHS_R_NDG + MHS_R_NDDG) + MHS_Q_NDG + MHS_Q_NDDG.
constexpr int IMAGE_COEF_SIZE = 3 * (MHS_R_NDG + MHS_R_NDDG) + MHS_Q_NDG + MHS_Q_NDDG;

inline void image_coef(const Material& m, double* out) {
  const double nu = m.nu_i, s = m.scale_c;
  const double nup[3] = {1.0, nu, nu * nu};
  double* p = out;
  for (int r = 0; r < MHS_R_NDG; ++r)
    for (int pz = 0; pz < 3; ++pz) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += tab_h::mhs_r_dg_c[r][pz][k] * nup[k];
      *p++ = v * s;
    }
  for (int r = 0; r < MHS_R_NDDG; ++r)
    for (int pz = 0; pz < 3; ++pz) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += tab_h::mhs_r_ddg_c[r][pz][k] * nup[k];
      *p++ = v * s;
    }
  for (int r = 0; r < MHS_Q_NDG; ++r) {
    double v = 0.0;
    for (int k = 0; k < 3; ++k) v += tab_h::mhs_q_dg_c[r][k] * nup[k];
    *p++ = v;
  }
  for (int r = 0; r < MHS_Q_NDDG; ++r) {
    double v = 0.0;
    for (int k = 0; k < 3; ++k) v += tab_h::mhs_q_ddg_c[r][k] * nup[k];
    *p++ = v;
  }
}

}  // namespace mhs
