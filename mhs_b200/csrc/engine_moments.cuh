// Weighted moment tables of one triangle at one observer:
//
//   W_k[n](a, b) = int_T N_k(y) xi_1^a xi_2^b / R_eps^n dS,
//   R_eps^2 = xi_1^2 + xi_2^2 + z^2 + eps^2,
//
// by the divergence-theorem recursion (near field) or a collapsed Gauss
// product rule (far field), exactly the split of mhs/fullspace/moments.py:
// 515-606.  One thread evaluates one (observer, triangle) pair.
#pragma once

#include "engine_base.cuh"

namespace mhs {

// 1/i for the series denominators.
MHS_FI double inv_int(int i) { return 1.0 / (double)i; }

MHS_FI double ipow(double x, int e) {
  double r = 1.0;
  const int n = e < 0 ? -e : e;
  for (int i = 0; i < n; ++i) r *= x;
  return e < 0 ? 1.0 / r : r;
}

// ------------------------------------------------------ edge primitives
// P[m][k] = int_{ua}^{ub} u^k / (u^2 + rho^2)^(m/2) du for the (m, k) of the
// spec, cancellation-free: the small-|u| binomial series where both ends sit
// within rho/2 of the foot, the large-|u| series where both lie beyond 2 rho
// on one side, the closed-form difference forms otherwise
// (mhs/fullspace/primitives.py:131-504; rho > 0 always since eps > 0).

// FAST (the fold's near loads): the same forms with the radii from
// reciprocal square roots and the divisions by R_a, R_b and rho2 taken as
// products with their reciprocals (rounding-level differences).
template <class S, bool FAST = false>
MHS_FI void edge_closed(double ua, double ub, double rho2, double P[MS][8]) {
  constexpr Spec sp = S::spec;
  double Ra, Rb, iRa, iRb, irho2;
  if constexpr (FAST) {
    const double qa = ua * ua + rho2, qb = ub * ub + rho2;
    iRa = rsqrt_r(qa);
    iRb = rsqrt_r(qb);
    Ra = qa * iRa;
    Rb = qb * iRb;
    irho2 = 1.0 / rho2;
  } else {
    Ra = sqrt(ua * ua + rho2);
    Rb = sqrt(ub * ub + rho2);
    iRa = 1.0 / Ra;
    iRb = 1.0 / Rb;
    irho2 = 0.0;
  }
  const double dR = (ub - ua) * (ub + ua) / (Ra + Rb);   // R_b - R_a
  double J[MS], Kk[MS];
  // Delta J_1: log1p forms on one side, the product form across the foot
  if (sp.Jneed[1]) {
    if (ua >= 0.0) J[1] = log1p(((ub - ua) + dR) / (ua + Ra));
    else if (ub <= 0.0) J[1] = log1p(((ub - ua) - dR) / (Rb - ub));
    else J[1] = log(((ub + Rb) * (Ra - ua)) / rho2);
  }
  if (sp.Jneed[2]) {
    if constexpr (FAST) {
      if (ua * ub > 0.0) J[2] = (((ub - ua) * (ub + ua)) * (iRa * iRb)) / (ub * Ra + ua * Rb);
      else J[2] = (ub * iRb - ua * iRa) * irho2;
    } else {
      if (ua * ub > 0.0) J[2] = ((ub - ua) * (ub + ua)) / ((Ra * Rb) * (ub * Ra + ua * Rb));
      else J[2] = (ub / Rb - ua / Ra) / rho2;
    }
  }
  if (sp.Jneed[3]) {  // m = 5 from m = 3
    const double duRm = ub * (iRb * iRb * iRb) - ua * (iRa * iRa * iRa);
    if constexpr (FAST) J[3] = (duRm + 2.0 * J[2]) * (irho2 * (1.0 / 3.0));
    else J[3] = (duRm + 2.0 * J[2]) / (3.0 * rho2);
  }
  if (sp.Jneed[4]) {  // m = 7 from m = 5
    const double a2 = iRa * iRa, b2 = iRb * iRb;
    const double duRm = ub * (b2 * b2 * iRb) - ua * (a2 * a2 * iRa);
    if constexpr (FAST) J[4] = (duRm + 4.0 * J[3]) * (irho2 * 0.2);
    else J[4] = (duRm + 4.0 * J[3]) / (5.0 * rho2);
  }
  if (sp.Jneed[0]) {  // m = -1
    const double duR = 0.5 * (ub - ua) * (Ra + Rb) + 0.5 * (ua + ub) * dR;
    J[0] = 0.5 * (duR + rho2 * J[1]);
  }
  // Delta K_m = Delta R^(2-m) / (2-m), factored through dR
  if (sp.Kneed[0]) Kk[0] = dR * ((Rb * Rb + Ra * Rb) + Ra * Ra) / 3.0;
  if (sp.Kneed[1]) Kk[1] = dR;
  if constexpr (FAST) {
    const double iab = iRa * iRb;
    if (sp.Kneed[2]) Kk[2] = dR * iab;
    if (sp.Kneed[3]) Kk[3] = (dR * ((Rb * Rb + Ra * Rb) + Ra * Ra)) * ((iab * iab * iab) * (1.0 / 3.0));
    if (sp.Kneed[4]) {
      const double a2 = Ra * Ra, b2 = Rb * Rb;
      const double s = (((b2 * b2 + Ra * (b2 * Rb)) + a2 * b2) + (a2 * Ra) * Rb) + a2 * a2;
      const double i2 = iab * iab;
      Kk[4] = (dR * s) * ((i2 * i2 * iab) * 0.2);
    }
  } else {
    if (sp.Kneed[2]) Kk[2] = dR / (Ra * Rb);
    if (sp.Kneed[3]) {
      const double ab = Ra * Rb;
      Kk[3] = dR * ((Rb * Rb + Ra * Rb) + Ra * Ra) / (3.0 * (ab * ab * ab));
    }
    if (sp.Kneed[4]) {
      const double ab = Ra * Rb, a2 = Ra * Ra, b2 = Rb * Rb;
      const double s = (((b2 * b2 + Ra * (b2 * Rb)) + a2 * b2) + (a2 * Ra) * Rb) + a2 * a2;
      Kk[4] = dR * s / (5.0 * (ab * ab * ab * ab * ab));
    }
  }
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int j = 0; j < MS; ++j) {
      if (!sp.Pneed[j][k]) continue;
      if (k == 0) P[j][0] = J[j];
      else if (k == 1) P[j][1] = Kk[j];
      else P[j][k] = P[j - 1][k - 2] - rho2 * P[j][k - 2];
    }
}

// Small-|u| series, P[m][k] = rho^(k+1-m) sum_t C(-m/2, t) E[k + 2t + 1] with
// E[pw] = (yb^pw - ya^pw) / pw, y = u / rho.  E is produced in order of pw
// and every term goes to its sum as it appears: for each (m, k) the terms
// arrive in increasing t, the order of the plain double loop.
template <class S>
MHS_FI void edge_small(double ua, double ub, double rho, double P[MS][8]) {
  constexpr Spec sp = S::spec;
  constexpr int T = cst::SERIES_TERMS;
  constexpr int PWMAX = sp.kmax + 2 * (T - 1) + 1;
  const double ya = ua / rho, yb = ub / rho;
  const bool same = ua * ub > 0.0;
  // E[pw] = (yb^pw - ya^pw) / pw; the same-sign recurrence
  // D_{pw+1} = yb D_pw + ya^pw (yb - ya) has no cancellation.
  const double dy = yb - ya;
  double yap = ya, ybp = yb, D = dy;
  double acc[MS][8];
#pragma unroll
  for (int j = 0; j < MS; ++j)
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[j][k] = 0.0;
#pragma unroll 1
  for (int u = 0; 2 * u + 1 <= PWMAX; ++u) {
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int pw = 2 * u + 1 + half;   // k parity = half
      if (pw > PWMAX) break;
      const double E = D * MHS_TAB(mhs_inv_int)[pw];
      if (same) D = yb * D + yap * dy;
      yap *= ya;
      ybp *= yb;
      if (!same) D = ybp - yap;
#pragma unroll
      for (int j = 0; j < MS; ++j)
#pragma unroll
        for (int k = half; k < 8; k += 2) {
          if (k > sp.edge[j]) continue;
          const int t = u - k / 2;            // pw = k + 2t + 1
          if (t >= 0 && t < T) acc[j][k] += MHS_TAB(mhs_binom_half)[j][t] * E;
        }
    }
  }
#pragma unroll
  for (int j = 0; j < MS; ++j) {
    const int m = 2 * j - 1;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k > sp.edge[j]) continue;
      P[j][k] = ipow(rho, k + 1 - m) * acc[j][k];
    }
  }
}

// Exponent range q = k - m + 1 - 2 t of the large-|u| series over a spec.
MHS_FI constexpr int series_qhi(const Spec& sp) {
  int q = -999;
  for (int j = 0; j < MS; ++j)
    if (sp.edge[j] >= 0) q = imax(q, sp.edge[j] - (2 * j - 1) + 1);
  return q;
}
MHS_FI constexpr int series_qlo(const Spec& sp) {
  int q = 999;
  for (int j = 0; j < MS; ++j)
    if (sp.edge[j] >= 0) q = imin(q, 0 - (2 * j - 1) + 1);
  return q - 2 * (cst::SERIES_TERMS - 1);
}
MHS_FI constexpr int spec_max_need0(const Spec& sp) {
  int d = 0;
  for (int s = 0; s < NS; ++s) d = imax(d, sp.need0[s]);
  return d;
}

// Large-|u| series on one side of the foot (a = min|u|, b = max|u|):
// P[m][k] = +-a^s sum_t C(-m/2, t) x^t dq[s - 2t], s = k - m + 1,
// x = rho^2 / a^2, dq[q] = [t^q / q]_1^(b/a) (log at q = 0).  Near r = b/a = 1
// the geometric sums (r - 1) sum r^i and (1 - 1/r) sum r^-i replace expm1
// without cancellation.  The negative-q values come from one recurrence in
// increasing -q; the sum over t keeps a window of them in registers, and each
// (m, k) sum takes its terms in increasing t as the plain double loop does.
template <class S>
MHS_FI void edge_large(double ua, double ub, double rho2, double P[MS][8]) {
  constexpr Spec sp = S::spec;
  constexpr int T = cst::SERIES_TERMS;
  constexpr int QHI = series_qhi(sp);             // largest s
  constexpr int SMIN = series_qlo(sp) + 2 * (T - 1);   // smallest s
  constexpr int W = QHI - SMIN + 1;               // window width
  static_assert(QHI <= 3, "large-u series exponent above 3");
  static_assert(SMIN <= 0, "window shift assumes a negative exponent at t = 0");
  const bool neg = ua < 0.0;
  const double a = neg ? -ub : ua, b = neg ? -ua : ub;
  const double r = b / a;
  const double log_r = log1p((b - a) / a);
  const bool close = r < 2.0;
  const double x = rho2 / (a * a);
  const double rm1 = (b - a) / a;     // r - 1
  const double omt = (b - a) / b;     // 1 - 1/r
  const double tt = a / b;            // 1/r
  double dpos[4] = {0.0, 0.0, 0.0, 0.0};
  if constexpr (QHI >= 0) dpos[0] = log_r;
  if constexpr (QHI >= 1) dpos[1] = close ? rm1 : r - 1.0;
  if constexpr (QHI >= 2) dpos[2] = (close ? rm1 * (1.0 + r) : r * r - 1.0) * 0.5;
  if constexpr (QHI >= 3) dpos[3] = (close ? rm1 * ((1.0 + r) + r * r) : (r * r) * r - 1.0) / 3.0;
  // recurrence over k = -q = 1, 2, ...: dq[-k] = (close ? omt G_k : 1 - t^k) / k
  double gsum = 0.0, tk = 1.0;
  int kc = 0;
  // win[w] = dq[QHI - w - 2i] at step i
  double win[W];
#pragma unroll
  for (int w = 0; w < W; ++w) {
    const int q = QHI - w;
    if (q >= 0) {
      win[w] = dpos[q >= 0 && q <= 3 ? q : 0];
    } else {
      // generate up to k = -q (k ascending as w grows)
      while (kc < -q) {
        ++kc;
        gsum += tk;
        tk *= tt;
      }
      win[w] = (close ? omt * gsum : 1.0 - tk) * MHS_TAB(mhs_inv_int)[kc];
    }
  }
  double acc[MS][8];
#pragma unroll
  for (int j = 0; j < MS; ++j)
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[j][k] = 0.0;
  double xj = 1.0;
#pragma unroll 1
  for (int i = 0; i < T; ++i) {
    if (i > 0) {
      xj = xj * x;
      // shift by two and append the next two recurrence values
      double g[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        ++kc;
        gsum += tk;
        tk *= tt;
        g[h] = (close ? omt * gsum : 1.0 - tk) * MHS_TAB(mhs_inv_int)[kc];
      }
#pragma unroll
      for (int w = 0; w < W; ++w) win[w] = (w + 2 < W) ? win[w + 2] : g[w - (W - 2)];
    }
#pragma unroll
    for (int j = 0; j < MS; ++j) {
      const double bx = MHS_TAB(mhs_binom_half)[j][i] * xj;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (k > sp.edge[j]) continue;
        const int s = k - (2 * j - 1) + 1;
        acc[j][k] += bx * win[QHI - s];
      }
    }
  }
#pragma unroll
  for (int j = 0; j < MS; ++j) {
    const int m = 2 * j - 1;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k > sp.edge[j]) continue;
      const int s = k - m + 1;
      const double v = ipow(a, s) * acc[j][k];
      P[j][k] = (neg && (k & 1)) ? -v : v;
    }
  }
}

enum : int { EDGE_CLOSED = 0, EDGE_SMALL = 1, EDGE_LARGE = 2 };

// Which of the three forms evaluates an edge (rho = sqrt(rho2)).
// The same test on squares (rho2 = rho^2), without the square root: the
// fold's near batch (a borderline edge may take the other, equally accurate
// form).
MHS_FI int edge_regime_sq(double ua, double ub, double rho2) {
  const double a2 = ua * ua, b2 = ub * ub;
  const double umax2 = a2 > b2 ? a2 : b2;
  const double umin2 = a2 < b2 ? a2 : b2;
  const double s2 = cst::SMALL_U_OVER_RHO_SQ, l2 = cst::SERIES_U_OVER_RHO_SQ;
  if (umax2 <= s2 * rho2) return EDGE_SMALL;
  if (ua * ub > 0.0 && umin2 >= l2 * rho2) return EDGE_LARGE;
  return EDGE_CLOSED;
}

MHS_FI int edge_regime(double ua, double ub, double rho) {
  const double aua = fabs(ua), aub = fabs(ub);
  const double umax = aua > aub ? aua : aub;
  const double umin = aua < aub ? aua : aub;
  if (umax <= cst::SMALL_U_OVER_RHO * rho) return EDGE_SMALL;
  if (ua * ub > 0.0 && umin >= cst::SERIES_U_OVER_RHO * rho) return EDGE_LARGE;
  return EDGE_CLOSED;
}

template <class S>
MHS_HD void edge_table(double ua, double ub, double rho2, double P[MS][8]) {
  const double rho = sqrt(rho2);
  const int r = edge_regime(ua, ub, rho);
  if (r == EDGE_SMALL) edge_small<S>(ua, ub, rho, P);
  else if (r == EDGE_LARGE) edge_large<S>(ua, ub, rho2, P);
  else edge_closed<S>(ua, ub, rho2, P);
}

// ------------------------------------------------- closed-form moment table
// M_n^(a,b)(x) = int_T xi_1^a xi_2^b / R_eps^n dS for the closed degrees of
// the spec, seeded by the solid angle and the vertical identity and filled
// by the horizontal recursion (mhs/fullspace/moments.py:171-355).
template <class S>
struct MomentTable {
  double M[S::spec.m_off[NS] > 0 ? S::spec.m_off[NS] : 1];
  MHS_FI double& at(int s, int a, int b) {
    constexpr Spec sp = S::spec;
    return M[sp.m_off[s] + tri_idx(a, b)];
  }
  MHS_FI double at(int s, int a, int b) const {
    constexpr Spec sp = S::spec;
    return M[sp.m_off[s] + tri_idx(a, b)];
  }
};

// Van Oosterom-Strackee solid angle of the triangle seen from the point at
// in-plane offset -X, height h; the vertices are given relative to the foot
// (pa[i] = p_i - X), so the point sits at (0, 0, h) in the local frame.
MHS_HD double solid_angle_local(const double pr[3][2], double h) {
  double r[3][3];
  for (int i = 0; i < 3; ++i) {
    r[i][0] = pr[i][0];
    r[i][1] = pr[i][1];
    r[i][2] = -h;
  }
  const double R1 = norm3(r[0]), R2 = norm3(r[1]), R3 = norm3(r[2]);
  double cx[3];
  cross3(r[1], r[2], cx);
  const double numer = dot3(r[0], cx);
  const double denom = R1 * R2 * R3 + R3 * dot3(r[0], r[1]) + R1 * dot3(r[1], r[2]) +
                       R2 * dot3(r[0], r[2]);
  return 2.0 * atan2(numer, denom);
}

// One edge of the triangle seen from the foot: tangent (s1, s2), outward
// normal (c1, c2) = (s2, -s1), signed normal distance dp, the foot's
// coordinates ua, ub of the edge ends along the tangent, rho2 = dp^2 + h2.
struct EdgeGeom {
  double s1, s2, dp, ua, ub, rho2;
};

MHS_FI EdgeGeom edge_geom(const double pr[3][2], int e, double h2) {
  const int e2 = e == 2 ? 0 : e + 1;
  const double pa0 = pr[e][0], pa1 = pr[e][1], pb0 = pr[e2][0], pb1 = pr[e2][1];
  const double ev0 = pb0 - pa0, ev1 = pb1 - pa1;
  const double L = sqrt(ev0 * ev0 + ev1 * ev1);
  EdgeGeom g;
  g.s1 = ev0 / L;
  g.s2 = ev1 / L;
  const double c1 = g.s2, c2 = -g.s1;
  g.dp = pa0 * c1 + pa1 * c2;
  g.ua = pa0 * g.s1 + pa1 * g.s2;
  g.ub = pb0 * g.s1 + pb1 * g.s2;
  g.rho2 = g.dp * g.dp + h2;
  return g;
}

// edge_geom with the tangent from one reciprocal square root of the squared
// length (the fold's near loads; rounding-level differences).
MHS_FI EdgeGeom edge_geom_rcp(const double pr[3][2], int e, double h2) {
  const int e2 = e == 2 ? 0 : e + 1;
  const double pa0 = pr[e][0], pa1 = pr[e][1], pb0 = pr[e2][0], pb1 = pr[e2][1];
  const double ev0 = pb0 - pa0, ev1 = pb1 - pa1;
  const double iL = rsqrt_r(ev0 * ev0 + ev1 * ev1);
  EdgeGeom g;
  g.s1 = ev0 * iL;
  g.s2 = ev1 * iL;
  const double c1 = g.s2, c2 = -g.s1;
  g.dp = pa0 * c1 + pa1 * c2;
  g.ua = pa0 * g.s1 + pa1 * g.s2;
  g.ub = pb0 * g.s1 + pb1 * g.s2;
  g.rho2 = g.dp * g.dp + h2;
  return g;
}

// Vertices relative to the foot X (in-plane, centroid frame).
MHS_FI void foot_vertices(const Frame& f, double X0, double X1, double pr[3][2]) {
  for (int k = 0; k < 3; ++k) {
    pr[k][0] = f.p[k][0] - X0;
    pr[k][1] = f.p[k][1] - X1;
  }
}

// Add one edge's boundary terms: BD[j] += dp P[j][0] and the normal
// components of xi_1^a xi_2^b / R^m along the edge, BN1/BN2, expanded as
// polynomials in u (xi_1 = dp c1 + u s1, xi_2 = dp c2 + u s2).
template <class S>
MHS_FI void edge_accumulate(const EdgeGeom& g, const double P[MS][8], double* BN1, double* BN2,
                            double* BD) {
  constexpr Spec sp = S::spec;
  const double s1 = g.s1, s2 = g.s2, dp = g.dp;
  const double c1 = s2, c2 = -s1;
#pragma unroll
  for (int j = 0; j < MS; ++j)
    if (sp.edge[j] >= 0) BD[j] += dp * P[j][0];
  constexpr int KM = sp.kmax;
  double pa_[KM + 1];   // xi_1^a
  pa_[0] = 1.0;
#pragma unroll
  for (int i = 1; i <= KM; ++i) pa_[i] = 0.0;
  const double l0 = dp * c1, l1 = s1, m0 = dp * c2, m1 = s2;
#pragma unroll
  for (int a = 0; a <= KM; ++a) {
    double pb_[KM + 1];
#pragma unroll
    for (int i = 0; i <= KM; ++i) pb_[i] = pa_[i];
#pragma unroll
    for (int b = 0; a + b <= KM; ++b) {
      // pb_ holds xi_1^a xi_2^b (degree a + b)
#pragma unroll
      for (int j = 0; j < MS; ++j) {
        if (sp.edge[j] < a + b) continue;
        double val = 0.0;
#pragma unroll
        for (int i = 0; i <= a + b; ++i) val += pb_[i] * P[j][i];
        BN1[sp.b_off[j] + tri_idx(a, b)] += c1 * val;
        BN2[sp.b_off[j] + tri_idx(a, b)] += c2 * val;
      }
      if (a + b < KM) {  // multiply by xi_2
#pragma unroll
        for (int i = KM; i >= 1; --i) pb_[i] = pb_[i] * m0 + pb_[i - 1] * m1;
        pb_[0] = pb_[0] * m0;
      }
    }
    if (a < KM) {  // multiply by xi_1
#pragma unroll
      for (int i = KM; i >= 1; --i) pa_[i] = pa_[i] * l0 + pa_[i - 1] * l1;
      pa_[0] = pa_[0] * l0;
    }
  }
}

template <class S, bool FAST>
MHS_HD void closed_finish_t(const double pr[3][2], double h2, const double* BN1, const double* BN2,
                            const double* BD, MomentTable<S>& T);

// Seeds (solid angle, vertical identities) and the horizontal recursion
// from the summed boundary terms.
template <class S>
MHS_HD void closed_finish(const double pr[3][2], double h2, const double* BN1, const double* BN2,
                          const double* BD, MomentTable<S>& T) {
  closed_finish_t<S, false>(pr, h2, BN1, BN2, BD, T);
}

// One slot's part of the closed-form table: its upward vertical seed
// I_{n+2} = (E_n + (n-2) I_n) / (n h^2) (slot s = nslot(n + 2)), its
// downward seed I_n = (E_n - n h^2 I_{n+2}) / (2 - n), and its horizontal
// recursion.  The slot and its degree are template constants so every
// index into the tables is a compile-time constant (no local memory).
template <class S, bool FAST, int n>
MHS_FI void seed_up(double h2, double ih2, const double* BD, MomentTable<S>& T) {
  constexpr Spec sp = S::spec;
  if constexpr (n + 2 <= 9) {
    if constexpr (sp.deg[nslot(n + 2)] >= 0) {
      if constexpr (FAST)
        T.at(nslot(n + 2), 0, 0) = (BD[nslot(n)] + (n - 2) * T.at(nslot(n), 0, 0)) * (ih2 * (1.0 / n));
      else
        T.at(nslot(n + 2), 0, 0) = (BD[nslot(n)] + (n - 2) * T.at(nslot(n), 0, 0)) / (n * h2);
      seed_up<S, FAST, n + 2>(h2, ih2, BD, T);
    }
  }
}

template <class S, int n>
MHS_FI void seed_down(double h2, const double* BD, MomentTable<S>& T) {
  constexpr Spec sp = S::spec;
  if constexpr (n >= -1) {
    if constexpr (sp.deg[nslot(n)] >= 0) {
      const double corr = n * h2 * T.at(nslot(n + 2), 0, 0);
      T.at(nslot(n), 0, 0) = (BD[nslot(n)] - corr) / (2.0 - n);
      seed_down<S, n - 2>(h2, BD, T);
    }
  }
}

template <class S, int s>
MHS_FI void recur_slot(const double* BN1, const double* BN2, MomentTable<S>& T) {
  constexpr Spec sp = S::spec;
  if constexpr (s < NS) {
    constexpr int d = sp.deg[s];
    if constexpr (d > 0) {
      constexpr int n = slot_n(s), mj = s - 1;   // m = n - 2
      const double inv = 1.0 / (double)(n - 2);
#pragma unroll
      for (int q = 1; q <= d; ++q)
#pragma unroll
        for (int a = q; a >= 0; --a) {
          const int b = q - a;
          double val;
          if (a >= 1) {
            val = -BN1[sp.b_off[mj] + tri_idx(a - 1, b)];
            if (a >= 2) val = val + (a - 1) * T.at(s - 1, a - 2, b);
          } else {
            val = -BN2[sp.b_off[mj] + tri_idx(0, b - 1)];
            if (b >= 2) val = val + (b - 1) * T.at(s - 1, 0, b - 2);
          }
          T.at(s, a, b) = val * inv;
        }
    }
    recur_slot<S, s + 1>(BN1, BN2, T);
  }
}

// FAST (the fold's near loads): 1/h from a reciprocal square root and the
// seeds' divisions by n h^2 as products with 1/h^2 (rounding-level
// differences).
template <class S, bool FAST>
MHS_HD void closed_finish_t(const double pr[3][2], double h2, const double* BN1, const double* BN2,
                            const double* BD, MomentTable<S>& T) {
  constexpr Spec sp = S::spec;
  double h, I3, ih2 = 0.0;
  if constexpr (FAST) {
    const double ih = rsqrt_r(h2);
    h = h2 * ih;
    I3 = -solid_angle_local(pr, h) * ih;
    ih2 = ih * ih;
  } else {
    h = sqrt(h2);
    I3 = -solid_angle_local(pr, h) / h;
  }
#pragma unroll
  for (int i = 0; i < sp.m_off[NS]; ++i) T.M[i] = 0.0;
  T.at(nslot(3), 0, 0) = I3;
  seed_up<S, FAST, 3>(h2, ih2, BD, T);    // upward seeds from I_3
  seed_down<S, 1>(h2, BD, T);             // downward seeds I_1, I_-1
  recur_slot<S, 0>(BN1, BN2, T);          // horizontal recursion, ascending n
}

template <class S>
MHS_HD void closed_moments(const Frame& f, double X0, double X1, double h2, MomentTable<S>& T) {
  constexpr Spec sp = S::spec;
  constexpr int NB = sp.b_off[MS] > 0 ? sp.b_off[MS] : 1;
  double BN1[NB], BN2[NB], BD[MS];
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    BN1[i] = 0.0;
    BN2[i] = 0.0;
  }
#pragma unroll
  for (int j = 0; j < MS; ++j) BD[j] = 0.0;
  double pr[3][2];
  foot_vertices(f, X0, X1, pr);
#pragma unroll 1
  for (int e = 0; e < 3; ++e) {
    const EdgeGeom g = edge_geom(pr, e, h2);
    double P[MS][8];
    edge_table<S>(g.ua, g.ub, g.rho2, P);
    edge_accumulate<S>(g, P, BN1, BN2, BD);
  }
  closed_finish<S>(pr, h2, BN1, BN2, BD, T);
}

// W_k[n](a, b) = sum_{a'+b'<=P} c_k(a', b') M_n(a + a', b + b'), at the
// constant-slip degrees (mhs/fullspace/moments.py:370-398).
template <class S, int P, int s, class WO>
MHS_FI void weight_slot(const MomentTable<S>& T, const double c[][ntri(P)], int k, WO W) {
  constexpr Spec sp = S::spec;
  if constexpr (s < NS) {
    constexpr int d = sp.need0[s];
    if constexpr (d >= 0) {
#pragma unroll
      for (int a = 0; a <= d; ++a)
#pragma unroll
        for (int b = 0; a + b <= d; ++b) {
          double acc = 0.0;
#pragma unroll
          for (int ap = 0; ap <= P; ++ap)
#pragma unroll
            for (int bp = 0; ap + bp <= P; ++bp)
              acc += c[k][tri_idx(ap, bp)] * T.at(s, a + ap, b + bp);
          W[sp.w_off[s] + tri_idx(a, b)] = acc;
        }
    }
    weight_slot<S, P, s + 1>(T, c, k, W);
  }
}

// W is a pointer or a StridedTable.
template <class S, int P, class WO = double*>
MHS_FI void weight_closed(const MomentTable<S>& T, const double c[][ntri(P)], int k, WO W) {
  weight_slot<S, P, 0>(T, c, k, W);
}

// ----------------------------------------------------- far-field quadrature
// Collapsed Gauss product rule on the reference triangle, mapped onto the
// element: nodes eta (centroid frame), weights wq (area measure) and N_k at
// the nodes (mhs/fullspace/moments.py:401-446).  Built once per source.
template <class T>
struct QuadRuleT {
  int nq;
  const T* eta0;
  const T* eta1;
  const T* wq;
  const T* Nq;   // nq x K, node-major
};
using QuadRule = QuadRuleT<double>;

// Fill a rule for order n from the 1-D Gauss-Legendre table (x in [-1, 1]).
template <int P>
MHS_HD void build_rule(const Frame& f, const double* glx, const double* glw, int n,
                       double* eta0, double* eta1, double* wq, double* Nq) {
  constexpr int K = n_nodes(P);
  const double* x = glx + gl_offset(n);
  const double* w = glw + gl_offset(n);
  int q = 0;
  for (int i = 0; i < n; ++i) {
    const double gi = 0.5 * (x[i] + 1.0), wi = 0.5 * w[i];
    for (int j = 0; j < n; ++j, ++q) {
      const double gj = 0.5 * (x[j] + 1.0), wj = 0.5 * w[j];
      const double x1 = gi, x2 = gj * (1.0 - gi);
      const double ww = wi * wj * (1.0 - gi);
      const double l0 = 1.0 - x1 - x2;
      const double e0 = (l0 * f.p[0][0] + x1 * f.p[1][0]) + x2 * f.p[2][0];
      const double e1 = (l0 * f.p[0][1] + x1 * f.p[1][1]) + x2 * f.p[2][1];
      eta0[q] = e0;
      eta1[q] = e1;
      wq[q] = ww * (2.0 * f.area);
      shape_at<P>(f, e0, e1, Nq + q * K);
    }
  }
}

// W_k[n](a, b) by quadrature of N_k xi_1^a xi_2^b R^-n at the constant-slip
// degrees (mhs/fullspace/moments.py:427-498).  R is float or double: the
// mixed-precision form runs this in float with float accumulation.
// weight_far_nodes evaluates nodes [k0, k0 + KG) into tables out0, out0 + 1,
// ... of Wout: every accumulator adds its point terms in rule order,
// whichever group of nodes it is taken with.
template <class S, int P, class R, int KG, class Q, class WO>
MHS_HD void weight_far_nodes(const Q& q, R x0, R x1, R hh, int k0, int out0, WO Wout) {
  constexpr Spec sp = S::spec;
  constexpr int K = n_nodes(P);
  constexpr int NW = sp.w_off[NS];
  constexpr int DM = spec_max_need0(sp);
  R acc[KG][NW];
#pragma unroll
  for (int k = 0; k < KG; ++k)
#pragma unroll
    for (int i = 0; i < NW; ++i) acc[k][i] = R(0);
#pragma unroll 2
  for (int t = 0; t < q.nq; ++t) {
    const R xi0 = R(q.eta0[t]) - x0, xi1 = R(q.eta1[t]) - x1;
    const R R2 = xi0 * xi0 + xi1 * xi1 + hh;
    const R inv = rsqrt_r(R2);
    const R inv2 = inv * inv;
    // w_s = wq R^-n for the odd n of the spec, then times each monomial
    const R wq = R(q.wq[t]);
    R ws[NS];
    {
      R cur = wq * inv;
#pragma unroll
      for (int s = 1; s < NS; ++s) {
        ws[s] = cur;
        cur = cur * inv2;
      }
    }
    R p0[DM + 1], p1[DM + 1];
    p0[0] = R(1);
    p1[0] = R(1);
#pragma unroll
    for (int i = 1; i <= DM; ++i) {
      p0[i] = p0[i - 1] * xi0;
      p1[i] = p1[i - 1] * xi1;
    }
    R Nk[KG];
#pragma unroll
    for (int k = 0; k < KG; ++k) Nk[k] = R(q.Nq[t * K + k0 + k]);
#pragma unroll
    for (int a = 0; a <= DM; ++a)
#pragma unroll
      for (int b = 0; a + b <= DM; ++b) {
        const R mono = (a && b) ? p0[a] * p1[b] : a ? p0[a] : b ? p1[b] : R(1);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          if (sp.need0[s] < a + b) continue;
          const R v = (a || b) ? ws[s] * mono : ws[s];
          if constexpr (P == 0) {
            acc[0][sp.w_off[s] + tri_idx(a, b)] += v;   // N = 1
          } else {
#pragma unroll
            for (int k = 0; k < KG; ++k) acc[k][sp.w_off[s] + tri_idx(a, b)] += v * Nk[k];
          }
        }
      }
  }
#pragma unroll
  for (int k = 0; k < KG; ++k)
#pragma unroll
    for (int i = 0; i < NW; ++i) Wout[(out0 + k) * NW + i] = double(acc[k][i]);
}

// Far-field weighted tables of all K nodes by the product rule q, in
// passes over the rule of as many nodes as keep at most FAR_ACC_MAX
// accumulators live (P0 and the smaller specs: one pass); each pass repeats
// the per-point powers and leaves every sum's order unchanged.
constexpr int FAR_ACC_MAX = 64;

template <class S, int P, class R, int K0, class Q, class WO>
MHS_HD void weight_far_from(const Q& q, R x0, R x1, R hh, WO Wout) {
  constexpr int K = n_nodes(P);
  constexpr int NW = S::spec.w_off[NS];
  constexpr int KG0 = FAR_ACC_MAX / NW > 0 ? FAR_ACC_MAX / NW : 1;
  constexpr int KG = (K - K0) < KG0 ? (K - K0) : KG0;
  weight_far_nodes<S, P, R, KG>(q, x0, x1, hh, K0, K0, Wout);
  if constexpr (K0 + KG < K) weight_far_from<S, P, R, K0 + KG>(q, x0, x1, hh, Wout);
}

template <class S, int P, class R, class Q = QuadRule, class WO = double*>
MHS_HD void weight_far(const Q& q, double X0, double X1, double h2, WO Wout) {
  weight_far_from<S, P, R, 0>(q, R(X0), R(X1), R(h2), Wout);
}

}  // namespace mhs
