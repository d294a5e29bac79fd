// The folded image of a source whose smeared slip reaches above z = 0
// (mhs/kernels/fold.py): at receivers in a band below the surface the lifted
// Mindlin image is replaced by the mirror element's full-space field plus the
// Boussinesq field of the pair's normal surface traction, integrated on a
// polar grid centred under the receiver.
//
// The grid is rebuilt here from the same rules (radial breaks, composite
// Gauss panels, angular sectors) so the quadrature nodes are the same nodes.
#pragma once

#include "engine_kernels.cuh"

namespace mhs {

// Mirror element's slip columns (fold.py:79).
MHS_FI double mirror_slip_sign(int m) { return m == 2 ? 1.0 : -1.0; }

// Source folded when its shallowest vertex is within FOLD_SOURCE_DEPTH_EPS eps
// of the surface (fold.py:84-87).
MHS_FI bool fold_straddles(const double* tri, double eps) {
  double zmax = tri[2];
  if (tri[5] > zmax) zmax = tri[5];
  if (tri[8] > zmax) zmax = tri[8];
  return -zmax < cst::FOLD_SOURCE_DEPTH_EPS * eps;
}

// Surface disk holding the source's sharp features: centre and radius
// (fold.py:95-107).
MHS_HD void fold_crease(const double* tri, double eps, double* centre, double* radius) {
  double dep[3];
  for (int i = 0; i < 3; ++i) dep[i] = -tri[3 * i + 2];
  bool top[3];
  int nt = 0;
  for (int i = 0; i < 3; ++i) {
    top[i] = dep[i] < cst::FOLD_SOURCE_DEPTH_EPS * eps;
    nt += top[i];
  }
  if (nt == 0) {
    double dmin = dep[0];
    for (int i = 1; i < 3; ++i)
      if (dep[i] < dmin) dmin = dep[i];
    for (int i = 0; i < 3; ++i) {
      top[i] = dep[i] == dmin;
      nt += top[i];
    }
  }
  double cx = 0.0, cy = 0.0;
  for (int i = 0; i < 3; ++i)
    if (top[i]) {
      cx += tri[3 * i];
      cy += tri[3 * i + 1];
    }
  cx /= nt;
  cy /= nt;
  double spread = 0.0, dtop = -INFINITY;
  for (int i = 0; i < 3; ++i)
    if (top[i]) {
      const double dx = tri[3 * i] - cx, dy = tri[3 * i + 1] - cy;
      const double r = sqrt(dx * dx + dy * dy);
      if (r > spread) spread = r;
      if (dep[i] > dtop) dtop = dep[i];
    }
  centre[0] = cx;
  centre[1] = cy;
  *radius = (spread + cst::FOLD_CREASE_MARGIN_EPS * eps) + dtop;
}

// Receiver takes the folded image of this source (fold.py:110-118).
MHS_FI bool fold_band(const double* x, const double* centre, double eps) {
  const double depth = -x[2];
  const double reach = hypot(x[0] - centre[0], x[1] - centre[1]);
  return depth < cst::FOLD_BAND_DEPTH_EPS * eps && reach < cst::FOLD_REACH_EPS * eps;
}

// Largest vertex-to-vertex distance (fold.py:344-345).
MHS_HD double tri_diameter(const double* tri) {
  double d = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double a = tri[3 * i] - tri[3 * j], b = tri[3 * i + 1] - tri[3 * j + 1],
                   c = tri[3 * i + 2] - tri[3 * j + 2];
      const double r = sqrt(a * a + b * b + c * c);
      if (r > d) d = r;
    }
  return d;
}

// ------------------------------------------------ Boussinesq point load
// Unit normal point load on the surface of the body z <= 0: stress (6
// unique components xx, yy, zz, xy, xz, yz) at depth zeta and offset
// (dx, dy) = receiver - load (fold.py:132-166).
MHS_HD void point_stress6(double dx, double dy, double zeta, double nu, double* S) {
  const double r2 = dx * dx + dy * dy;
  const double rho = sqrt(r2 + zeta * zeta);
  const double irho = 1.0 / rho;
  const double irho3 = irho * irho * irho;
  const double irho5 = irho3 * irho * irho;
  const double a = 1.0 / (rho * (rho + zeta));
  const double c = 1.0 - 2.0 * nu;
  const double zr3 = zeta * irho3;
  const double s_th = c * (-a + zr3);
  const double s_r_th = 2.0 * c * a - 3.0 * zeta * r2 * irho5 - c * zr3;
  const double r = sqrt(r2);
  const double ir = r > 0.0 ? 1.0 / r : 0.0;
  const double ex = dx * ir, ey = dy * ir;
  const double pref = 1.0 / (2.0 * cst::PI);
  S[0] = pref * (s_th + s_r_th * ex * ex);
  S[1] = pref * (s_th + s_r_th * ey * ey);
  S[2] = -pref * 3.0 * (zeta * zeta * zeta) * irho5;
  S[3] = pref * s_r_th * ex * ey;
  const double t_rz = pref * 3.0 * r * zeta * zeta * irho5;
  S[4] = t_rz * ex;
  S[5] = t_rz * ey;
}

// point_stress6 with the radii from reciprocal square roots and one
// division (rounding-level differences): the fold's accumulation kernel.
MHS_HD void point_stress6_rcp(double dx, double dy, double zeta, double nu, double* S) {
  const double r2 = dx * dx + dy * dy;
  const double q = r2 + zeta * zeta;
  const double irho = rsqrt_r(q);
  const double rho = q * irho;
  const double irho2 = irho * irho;
  const double irho3 = irho2 * irho;
  const double irho5 = irho3 * irho2;
  const double a = irho / (rho + zeta);
  const double c = 1.0 - 2.0 * nu;
  const double zr3 = zeta * irho3;
  const double s_th = c * (-a + zr3);
  const double s_r_th = 2.0 * c * a - 3.0 * zeta * r2 * irho5 - c * zr3;
  const double ir = r2 > 0.0 ? rsqrt_r(r2) : 0.0;
  const double r = r2 * ir;
  const double ex = dx * ir, ey = dy * ir;
  const double pref = 1.0 / (2.0 * cst::PI);
  S[0] = pref * (s_th + s_r_th * ex * ex);
  S[1] = pref * (s_th + s_r_th * ey * ey);
  S[2] = -pref * 3.0 * (zeta * zeta * zeta) * irho5;
  S[3] = pref * s_r_th * ex * ey;
  const double t_rz = pref * 3.0 * r * zeta * zeta * irho5;
  S[4] = t_rz * ex;
  S[5] = t_rz * ey;
}

// point_disp3 with the radius from a reciprocal square root.
MHS_HD void point_disp3_rcp(double dx, double dy, double zeta, double mu, double nu, double* u) {
  const double q = dx * dx + dy * dy + zeta * zeta;
  const double irho = rsqrt_r(q);
  const double rho = q * irho;
  const double irho3 = irho * irho * irho;
  const double pref = 1.0 / (4.0 * cst::PI * mu);
  const double ur = pref * (zeta * irho3 - (1.0 - 2.0 * nu) * (irho / (rho + zeta)));
  u[0] = ur * dx;
  u[1] = ur * dy;
  u[2] = -pref * (2.0 * (1.0 - nu) * irho + zeta * zeta * irho3);
}

MHS_HD void point_disp3(double dx, double dy, double zeta, double mu, double nu, double* u) {
  const double r2 = dx * dx + dy * dy;
  const double rho = sqrt(r2 + zeta * zeta);
  const double rho3 = rho * rho * rho;
  const double pref = 1.0 / (4.0 * cst::PI * mu);
  const double ur = pref * (zeta / rho3 - (1.0 - 2.0 * nu) / (rho * (rho + zeta)));
  u[0] = ur * dx;
  u[1] = ur * dy;
  u[2] = -pref * (2.0 * (1.0 - nu) / rho + zeta * zeta / rho3);
}

// Love's on-axis field of unit pressure over a disk of radius a
// (fold.py:185-210): diag(srr, srr, szz) and the vertical displacement.
MHS_HD void disk_stress(double a, double zeta, double nu, double* srr, double* szz) {
  const double rho = sqrt(a * a + zeta * zeta);
  const double z3 = (zeta * zeta * zeta) / (rho * rho * rho);
  *szz = -(1.0 - z3);
  *srr = -0.5 * ((1.0 + 2.0 * nu) - 2.0 * (1.0 + nu) * zeta / rho + z3);
}

MHS_HD double disk_disp_z(double a, double zeta, double mu, double nu) {
  const double rho = sqrt(a * a + zeta * zeta);
  return -(0.5 / mu) * (2.0 * (1.0 - nu) * (rho - zeta) + zeta - zeta * zeta / rho);
}

// ---------------------------------------------------------- polar grid
constexpr int FOLD_MAX_BREAKS = 192;

// numpy.linspace(a, b, num)[i]: i * step + a, the last point exactly b.
MHS_FI double linspace_at(double a, double b, int num, int i) {
  if (i == num - 1) return b;
  const double step = (b - a) / (double)(num - 1);
#if defined(__CUDA_ARCH__)
  return __dadd_rn(__dmul_rn((double)i, step), a);
#else
  return (double)i * step + a;
#endif
}

// The same point with the step (b - a) / (num - 1) already formed.
MHS_FI double linspace_step_at(double a, double b, double step, int num, int i) {
  if (i == num - 1) return b;
#if defined(__CUDA_ARCH__)
  return __dadd_rn(__dmul_rn((double)i, step), a);
#else
  return (double)i * step + a;
#endif
}

// One-sided angular half-width of the circles r in [ra, rb] inside the disk
// of `radius` about the crease centre at distance rho_s (fold.py:251-258).
MHS_HD double fold_halfwidth(double ra, double rb, double rho_s, double radius) {
  if (rb < rho_s - radius || ra > rho_s + radius) return 0.0;
  if (rho_s <= radius) return cst::PI;
  double q = radius / rho_s;
  if (q > 1.0) q = 1.0;
  return asin(q);
}

// Angular rule of one radial panel: up to four linspace pieces, each
// composite 4-point Gauss over its intervals (fold.py:261-287).
struct AngRule {
  int npiece;
  double a[4], b[4];
  double step[4];  // (b - a) / m, the linspace step of the piece
  int m[4];        // intervals per piece
  int n;           // total nodes = FOLD_N_ANGULAR * sum(m); -1 past the cap
};

// Intervals per angular piece beyond which a grid is refused (a source
// millions of eps across); keeps every count inside int range.
constexpr double FOLD_MAX_INTERVALS = 1 << 20;

// ceil(v) as an int, or -1 when v is not a finite count below the cap.
MHS_FI int fold_count(double v) {
  const double c = ceil(v);
  return (c >= 0.0 && c <= FOLD_MAX_INTERVALS) ? (int)c : -1;
}

MHS_HD void fold_angular(double theta_c, double w_fine, double w_med, double rb, double eps,
                         AngRule& A) {
  const int n = cst::FOLD_N_ANGULAR;
  const double two_pi = 2.0 * cst::PI;
  A.npiece = 0;
  A.n = 0;
  if (w_fine >= cst::PI || w_med >= cst::PI) {
    const double sp = w_fine >= cst::PI ? cst::FOLD_FINE_SPACING_EPS : cst::FOLD_MEDIUM_SPACING_EPS;
    int m = fold_count(two_pi * rb / ((double)n * sp * eps));
    if (m < 0) { A.n = -1; return; }
    if (m < 8) m = 8;
    A.a[0] = 0.0;
    A.b[0] = two_pi;
    A.step[0] = (two_pi - 0.0) / (double)m;
    A.m[0] = m;
    A.npiece = 1;
    A.n = n * m;
    return;
  }
  double pa[4], pb[4];
  int pm[4], np = 0;
  int mid_first = -1;
  if (w_fine > 0.0) {
    int m = fold_count(2.0 * w_fine * rb / ((double)n * cst::FOLD_FINE_SPACING_EPS * eps));
    if (m < 0) { A.n = -1; return; }
    if (m < 1) m = 1;
    pa[np] = theta_c - w_fine;
    pb[np] = theta_c + w_fine;
    pm[np] = m;
    mid_first = np;
    ++np;
  }
  if (w_med > w_fine) {
    int m = fold_count((w_med - w_fine) * rb / ((double)n * cst::FOLD_MEDIUM_SPACING_EPS * eps));
    if (m < 0) { A.n = -1; return; }
    if (m < 1) m = 1;
    // insert the left flank before the fine sector, append the right one
    for (int i = np; i > 0; --i) {
      pa[i] = pa[i - 1];
      pb[i] = pb[i - 1];
      pm[i] = pm[i - 1];
    }
    pa[0] = theta_c - w_med;
    pb[0] = theta_c - w_fine;
    pm[0] = m;
    ++np;
    pa[np] = theta_c + w_fine;
    pb[np] = theta_c + w_med;
    pm[np] = m;
    ++np;
  }
  (void)mid_first;
  const double start = w_med > 0.0 ? theta_c + w_med : 0.0;
  pa[np] = start;
  pb[np] = (start + two_pi) - 2.0 * w_med;
  pm[np] = imax(1, cst::FOLD_N_COARSE / n);
  ++np;
  for (int i = 0; i < np; ++i) {
    // a piece is used when its last break lies beyond its first
    if (!(pb[i] > pa[i])) continue;
    A.a[A.npiece] = pa[i];
    A.b[A.npiece] = pb[i];
    A.step[A.npiece] = (pb[i] - pa[i]) / (double)pm[i];
    A.m[A.npiece] = pm[i];
    A.n += n * pm[i];
    ++A.npiece;
  }
}

// Sorted, de-duplicated radial breaks of the polar grid about the receiver
// foot (fold.py:290-318).  Returns the count (or -1 past FOLD_MAX_BREAKS)
// and R1, the grid's outer radius.
MHS_HD int fold_breaks(double rho_s, double zeta, double r_f, double eps, double diam,
                       double* br, double* R1out) {
  double geo[64];
  int ng = 0;
  geo[ng++] = 0.0;
  if (0.0 < zeta && zeta < 0.5 * eps) {
    const double zs[4] = {0.5 * zeta, zeta, 2.0 * zeta, 4.0 * zeta};
    for (int i = 0; i < 4; ++i)
      if (zs[i] < 0.5 * eps) geo[ng++] = zs[i];
  }
  const double r1_target = (rho_s + 4.0 * r_f) + cst::FOLD_R1_MARGIN_DIAM * diam;
  double r = 0.5 * eps;
  while (true) {
    if (ng >= 64) return -1;
    geo[ng++] = r;
    if (r >= r1_target) break;
    r *= 2.0;
  }
  const double R1 = geo[ng - 1];
  const double lo_m = rho_s - 4.0 * r_f, hi_m = rho_s + 4.0 * r_f;
  const double lo_f = rho_s - r_f, hi_f = rho_s + r_f;
  int nb = 0;
  for (int i = 0; i < ng; ++i)
    if (geo[i] < lo_m || geo[i] > hi_m) br[nb++] = geo[i];
  const double a0s[3] = {lo_m > 0.0 ? lo_m : 0.0, lo_f > 0.0 ? lo_f : 0.0, hi_f < R1 ? hi_f : R1};
  const double b0s[3] = {lo_f > 0.0 ? lo_f : 0.0, hi_f < R1 ? hi_f : R1, hi_m < R1 ? hi_m : R1};
  const double ws[3] = {cst::FOLD_MEDIUM_SUBPANEL_EPS, cst::FOLD_FINE_SUBPANEL_EPS,
                        cst::FOLD_MEDIUM_SUBPANEL_EPS};
  for (int s = 0; s < 3; ++s) {
    const double a0 = a0s[s], b0 = b0s[s];
    if (!(b0 > a0)) continue;
    const double md = ceil((b0 - a0) / (ws[s] * eps));
    if (!(md <= (double)FOLD_MAX_BREAKS)) return -1;
    int m = (int)md;
    if (m < 1) m = 1;
    if (nb + m + 1 > FOLD_MAX_BREAKS) return -1;
    for (int i = 0; i <= m; ++i) br[nb++] = linspace_at(a0, b0, m + 1, i);
  }
  // sort (insertion) and drop exact duplicates
  for (int i = 1; i < nb; ++i) {
    const double v = br[i];
    int j = i - 1;
    while (j >= 0 && br[j] > v) {
      br[j + 1] = br[j];
      --j;
    }
    br[j + 1] = v;
  }
  int nu = 0;
  const double cap = R1 + 1e-12 * R1;
  for (int i = 0; i < nb; ++i) {
    if (nu > 0 && br[i] == br[nu - 1]) continue;
    if (!(br[i] <= cap)) continue;
    br[nu++] = br[i];
  }
  *R1out = R1;
  return nu;
}

// Everything a band pair's grid walk needs besides the breaks.
struct FoldPair {
  double xh0, xh1, zeta;    // receiver foot and depth
  double rho_s, theta_c;    // crease centre seen from the foot
  double r_f, eps, R1;
};

MHS_HD void fold_pair_setup(const double* x, const double* centre, double r_f, double eps,
                            FoldPair& fp) {
  fp.xh0 = x[0];
  fp.xh1 = x[1];
  fp.zeta = -x[2] > 0.0 ? -x[2] : 0.0;
  const double cx = centre[0] - x[0], cy = centre[1] - x[1];
  fp.rho_s = hypot(cx, cy);
  fp.theta_c = atan2(cy, cx);
  fp.r_f = r_f;
  fp.eps = eps;
}

// Angular rule of panel [ra, rb].
MHS_FI void fold_panel_rule(const FoldPair& fp, double ra, double rb, AngRule& A) {
  fold_angular(fp.theta_c, fold_halfwidth(ra, rb, fp.rho_s, fp.r_f),
               fold_halfwidth(ra, rb, fp.rho_s, 4.0 * fp.r_f), rb, fp.eps, A);
}

// Node j (0 <= j < A.n) of an angular rule: angle and weight.
MHS_HD void fold_ang_node(const AngRule& A, const double* glx4, const double* glw4, int j,
                          double* theta, double* wt) {
  int p = 0;
  while (j >= cst::FOLD_N_ANGULAR * A.m[p]) {
    j -= cst::FOLD_N_ANGULAR * A.m[p];
    ++p;
  }
  const int iv = j / cst::FOLD_N_ANGULAR, nd = j % cst::FOLD_N_ANGULAR;
  const double a = linspace_step_at(A.a[p], A.b[p], A.step[p], A.m[p] + 1, iv);
  const double b = linspace_step_at(A.a[p], A.b[p], A.step[p], A.m[p] + 1, iv + 1);
  const double u = 0.5 * (glx4[nd] + 1.0), wu = 0.5 * glw4[nd];
  *theta = a + (b - a) * u;
  *wt = (b - a) * wu;
}

// Surface load at horizontal point (px, py): twice the element's elastic
// sigma_zz on z = 0 per node and slip component (fold.py:214-228).
template <int P>
MHS_HD void fold_surface_load(const Frame& f, const QuadRule& r12, const QuadRule& r8, double px,
                              double py, double eps, const Material& m, double* s /*K x 3*/) {
  constexpr int K = n_nodes(P);
  double H[K * 27] = {}, E[K] = {};
  const double x[3] = {px, py, 0.0};
  direct_eval<P, W_H | W_E>(f, r12, r8, x, eps, m, nullptr, H, E);
  double ezz[3];
  for (int j = 0; j < 3; ++j) ezz[j] = m.lam * f.n[j] + (j == 2 ? 2.0 * m.mu * f.n[2] : 0.0);
  for (int k = 0; k < K; ++k)
    for (int j = 0; j < 3; ++j) s[3 * k + j] = 2.0 * (H[27 * k + 9 * 2 + 3 * 2 + j] - E[k] * ezz[j]);
}

// Per-source constants of the surface load: the global sigma_zz row of H
// as a linear form in the lifted quantities (per slip component), the
// eigenstress zz factor per slip component, and the blob-weight factor.
struct SurfaceLoadConsts {
  double coef[3][NLIFT];
  double ezz[3];
  double e4;
};

MHS_HD void surface_load_ezz(const Frame& f, double eps, const Material& m, SurfaceLoadConsts& c) {
  for (int j = 0; j < 3; ++j) c.ezz[j] = m.lam * f.n[j] + (j == 2 ? 2.0 * m.mu * f.n[2] : 0.0);
  c.e4 = 15.0 * (eps * eps) * (eps * eps) / (8.0 * cst::PI);
}

MHS_HD void surface_load_consts(const Frame& f, double eps, const Material& m, SurfaceLoadConsts& c) {
  for (int l = 0; l < NLIFT; ++l) {
    double col[3] = {};
    szz_coefficient(f, eps, m, l, col);
    for (int j = 0; j < 3; ++j) c.coef[j][l] = col[j];
  }
  surface_load_ezz(f, eps, m, c);
}

// Surface load of one node from its weighted moments W (one node's block):
// each lifted quantity goes straight into the three sigma_zz accumulators.
MHS_FI void szz_acc(const SurfaceLoadConsts& c, int l, double v, double& a0, double& a1,
                    double& a2) {
  a0 += c.coef[0][l] * v;
  a1 += c.coef[1][l] * v;
  a2 += c.coef[2][l] * v;
}

template <class S>
MHS_HD void surface_load_node(const SurfaceLoadConsts& c, const double* W, double z, double* s3) {
  constexpr Spec sp = S::spec;
  constexpr int o3 = sp.w_off[nslot(3)], o5 = sp.w_off[nslot(5)], o7 = sp.w_off[nslot(7)];
  const double zp[5] = {1.0, z, z * z, z * z * z, z * z * z * z};
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  szz_acc(c, L_I3, W[o3], a0, a1, a2);
  szz_acc(c, L_I5, W[o5], a0, a1, a2);
#pragma unroll
  for (int ca = 0; ca <= 2; ++ca)
#pragma unroll
    for (int cb = 0; ca + cb <= 2; ++cb) {
      const double sg = ((ca + cb) & 1) ? -zp[2 - ca - cb] : zp[2 - ca - cb];
      szz_acc(c, L_T25 + tri_idx(ca, cb), sg * W[o5 + tri_idx(ca, cb)], a0, a1, a2);
      szz_acc(c, L_T27 + tri_idx(ca, cb), sg * W[o7 + tri_idx(ca, cb)], a0, a1, a2);
    }
#pragma unroll
  for (int ca = 0; ca <= 4; ++ca)
#pragma unroll
    for (int cb = 0; ca + cb <= 4; ++cb) {
      const double sg = ((ca + cb) & 1) ? -zp[4 - ca - cb] : zp[4 - ca - cb];
      szz_acc(c, L_T47 + tri_idx(ca, cb), sg * W[o7 + tri_idx(ca, cb)], a0, a1, a2);
    }
  const double E = c.e4 * W[o7];
  s3[0] = 2.0 * (a0 - E * c.ezz[0]);
  s3[1] = 2.0 * (a1 - E * c.ezz[1]);
  s3[2] = 2.0 * (a2 - E * c.ezz[2]);
}

// Moment spec of the surface load (stress and blob weight).
template <int P> using SurfaceSpec = DirectSpec<P, W_H | W_E>;

// Surface load from the closed-form moment table at foot (X0, X1), height z.
template <int P>
MHS_HD void surface_load_near(const Frame& f, const MomentTable<SurfaceSpec<P>>& T,
                              const SurfaceLoadConsts& c, double z, double X0, double X1,
                              double* s /*K x 3*/) {
  using S = SurfaceSpec<P>;
  constexpr Spec sp = S::spec;
  constexpr int K = n_nodes(P);
  constexpr int NW = sp.w_off[NS];
  double cc[K][ntri(P)] = {};
  shape_coeffs<P>(f, X0, X1, cc);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double W[NW] = {};
    weight_closed<S, P>(T, cc, k, W);
    surface_load_node<S>(c, W, z, s + 3 * k);
  }
}

// Surface load by the far-field product rule q.
template <int P, class R_FAR = double, class Q = QuadRule>
MHS_HD void surface_load_far(const Q& q, const SurfaceLoadConsts& c, double z, double X0,
                             double X1, double h2, double* s /*K x 3*/) {
  using S = SurfaceSpec<P>;
  constexpr Spec sp = S::spec;
  constexpr int K = n_nodes(P);
  constexpr int NW = sp.w_off[NS];
  double W[K * NW] = {};
  weight_far<S, P, R_FAR>(q, X0, X1, h2, W);
#pragma unroll
  for (int k = 0; k < K; ++k) surface_load_node<S>(c, W + k * NW, z, s + 3 * k);
}

// Near / far class of a surface point: 0 closed form, 1 the 12 x 12 rule,
// 2 the 8 x 8 rule (the direct term's split, mhs/fullspace/moments.py:551-601).
enum : int { SL_NEAR = 0, SL_FAR12 = 1, SL_FAR8 = 2 };

MHS_FI int surface_class(const Frame& f, double px, double py, double eps) {
  const double d0 = px - f.c[0], d1 = py - f.c[1], d2 = 0.0 - f.c[2];
  const double D = sqrt(((d0 * d0 + d1 * d1) + d2 * d2) + eps * eps);
  if (D <= cst::D_STAR * f.L) return SL_NEAR;
  return (D > cst::D_STAR_DISTANT * f.L) ? SL_FAR8 : SL_FAR12;
}

// The same surface load as fold_surface_load, reading only sigma_zz: the
// weighted moments of each node (as direct_eval forms them), contracted with
// the precomputed sigma_zz row instead of the full H assembly and rotation.
template <int P, class R_FAR = double>
MHS_HD void fold_surface_load_fast(const Frame& f, const QuadRule& r12, const QuadRule& r8,
                                   const SurfaceLoadConsts& c, double px, double py, double eps,
                                   double* s /*K x 3*/) {
  using S = SurfaceSpec<P>;
  const double x[3] = {px, py, 0.0};
  double z, X0, X1;
  to_plane(f, x, z, X0, X1);
  const double h2 = z * z + eps * eps;
  const int cls = surface_class(f, px, py, eps);
  if (cls == SL_NEAR) {
    MomentTable<S> T;
    closed_moments<S>(f, X0, X1, h2, T);
    surface_load_near<P>(f, T, c, z, X0, X1, s);
  } else {
    surface_load_far<P, R_FAR>(cls == SL_FAR8 ? r8 : r12, c, z, X0, X1, h2, s);
  }
}

// Scalar reference walk of one band pair's Boussinesq correction, for the
// host test build and for small launches: H[k][a][b][m] (WANT_H) or
// U[k][i][m].  Returns 0, or -1 if the grid overflowed its capacity.
template <int P, bool WANT_H>
MHS_HD int fold_boussinesq_scalar(const Frame& f, const QuadRule& r12, const QuadRule& r8,
                                  const double* tri, const double* x, double eps,
                                  const Material& m, const double* glx, const double* glw,
                                  double* out) {
  constexpr int K = n_nodes(P);
  double centre[2], r_f;
  fold_crease(tri, eps, centre, &r_f);
  const double diam = tri_diameter(tri);
  FoldPair fp;
  fold_pair_setup(x, centre, r_f, eps, fp);
  double br[FOLD_MAX_BREAKS];
  const int nb = fold_breaks(fp.rho_s, fp.zeta, r_f, eps, diam, br, &fp.R1);
  if (nb < 0) return -1;
  SurfaceLoadConsts slc;
  surface_load_consts(f, eps, m, slc);
  double sh[3 * K] = {};
  fold_surface_load_fast<P>(f, r12, r8, slc, x[0], x[1], eps, sh);
  const double* gx6 = glx + gl_offset(cst::FOLD_N_RADIAL);
  const double* gw6 = glw + gl_offset(cst::FOLD_N_RADIAL);
  const double* gx4 = glx + gl_offset(cst::FOLD_N_ANGULAR);
  const double* gw4 = glw + gl_offset(cst::FOLD_N_ANGULAR);
  constexpr int NC = WANT_H ? 6 : 3;
  double acc[NC][3 * K];
  for (int c = 0; c < NC; ++c)
    for (int j = 0; j < 3 * K; ++j) acc[c][j] = 0.0;
  for (int pi = 0; pi + 1 < nb; ++pi) {
    const double ra = br[pi], rb = br[pi + 1];
    if (rb - ra < 1e-9 * eps) continue;
    AngRule A;
    fold_panel_rule(fp, ra, rb, A);
    if (A.n < 0) return -1;
    for (int ir = 0; ir < cst::FOLD_N_RADIAL; ++ir) {
      const double R = ra + (rb - ra) * (0.5 * (gx6[ir] + 1.0));
      const double wr = (rb - ra) * (0.5 * gw6[ir]);
      for (int j = 0; j < A.n; ++j) {
        double th, wt;
        fold_ang_node(A, gx4, gw4, j, &th, &wt);
        double sn, cs;
        sincos(th, &sn, &cs);
        const double px = fp.xh0 + R * cs, py = fp.xh1 + R * sn;
        const double w = wr * wt * R;
        double s[3 * K] = {};
        fold_surface_load_fast<P>(f, r12, r8, slc, px, py, eps, s);
        double B[NC];
        if (WANT_H) point_stress6(fp.xh0 - px, fp.xh1 - py, fp.zeta, m.nu_f, B);
        else point_disp3(fp.xh0 - px, fp.xh1 - py, fp.zeta, m.mu, m.nu_f, B);
        for (int c = 0; c < NC; ++c)
          for (int jj = 0; jj < 3 * K; ++jj) acc[c][jj] += (w * B[c]) * (s[jj] - sh[jj]);
      }
    }
  }
  if (WANT_H) {
    double srr, szz;
    disk_stress(fp.R1, fp.zeta, m.nu_f, &srr, &szz);
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    for (int k = 0; k < K; ++k)
      for (int mm = 0; mm < 3; ++mm) {
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) out[27 * k + 9 * a + 3 * b + mm] = 0.0;
        for (int c = 0; c < 6; ++c) {
          const double v = acc[c][3 * k + mm];
          out[27 * k + 9 * ia[c] + 3 * ib[c] + mm] = v;
          out[27 * k + 9 * ib[c] + 3 * ia[c] + mm] = v;
        }
        out[27 * k + 9 * 0 + 3 * 0 + mm] += sh[3 * k + mm] * srr;
        out[27 * k + 9 * 1 + 3 * 1 + mm] += sh[3 * k + mm] * srr;
        out[27 * k + 9 * 2 + 3 * 2 + mm] += sh[3 * k + mm] * szz;
      }
  } else {
    const double uz = disk_disp_z(fp.R1, fp.zeta, m.mu, m.nu_f);
    for (int k = 0; k < K; ++k)
      for (int mm = 0; mm < 3; ++mm)
        for (int i = 0; i < 3; ++i)
          out[9 * k + 3 * i + mm] = acc[i][3 * k + mm] + (i == 2 ? sh[3 * k + mm] * uz : 0.0);
  }
  return 0;
}

}  // namespace mhs
