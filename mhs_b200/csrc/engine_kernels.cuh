// Per-(observer, source) influence tensors from the weighted moment tables:
// the direct full-space Kelvin-Cortez kernels U / H / E, the half-space image
// R-family (closed form on the reflected element) and Q-family (per-observer
// Gauss quadrature).  Output layouts, per node k:
//   U[k][i][j]     displacement i from unit Cartesian slip j
//   H[k][a][b][j]  total stress (a, b) from unit Cartesian slip j
//   E[k]           blob weight of the eigenstress
#pragma once

#include "engine_moments.cuh"
#include "tables_q.inc"
#include "tables_r.inc"

namespace mhs {

enum : int { W_U = 1, W_H = 2, W_E = 4, W_G = 8, W_S = 16 };

// Spec of the direct term for a readout mask.
template <int P, int WANT> struct DirectSpec {
  static constexpr Spec spec = (WANT & W_U) ? SpecU<P>::spec
                               : (WANT & W_H) ? SpecH<P>::spec
                                              : SpecE<P>::spec;
};

// Component of a rank-r moment tensor in the element's own frame (basis
// e1, e2, nhat): with (ca, cb, cc) the counts of each basis index the lift
// (mhs/fullspace/kernels.py:90-123) reduces to one table entry,
// (-1)^(ca+cb) z^cc W_n(ca, cb).
template <class S>
MHS_FI double lift_local(const double* W, int s, int ca, int cb, int cc, const double* zp) {
  constexpr Spec sp = S::spec;
  const double v = zp[cc] * W[sp.w_off[s] + tri_idx(ca, cb)];
  return ((ca + cb) & 1) ? -v : v;
}

// Rotate a rank-2 tensor from the local frame: out[a][b] = R[a][x] R[b][y] in[x][y],
// R[a][x] = basis_x[a].
MHS_HD void rotate2(const Frame& f, const double in[3][3], double* out) {
  const double* B[3] = {f.e1, f.e2, f.n};
  double t[3][3];
  for (int a = 0; a < 3; ++a)
    for (int y = 0; y < 3; ++y) t[a][y] = B[0][a] * in[0][y] + B[1][a] * in[1][y] + B[2][a] * in[2][y];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) out[3 * a + b] = t[a][0] * B[0][b] + t[a][1] * B[1][b] + t[a][2] * B[2][b];
}

MHS_HD void rotate3(const Frame& f, const double in[3][3][3], double* out) {
  const double* B[3] = {f.e1, f.e2, f.n};
  double t1[3][3][3], t2[3][3][3];
  for (int a = 0; a < 3; ++a)
    for (int y = 0; y < 3; ++y)
      for (int z = 0; z < 3; ++z)
        t1[a][y][z] = B[0][a] * in[0][y][z] + B[1][a] * in[1][y][z] + B[2][a] * in[2][y][z];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int z = 0; z < 3; ++z)
        t2[a][b][z] = t1[a][0][z] * B[0][b] + t1[a][1][z] * B[1][b] + t1[a][2][z] * B[2][b];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int c = 0; c < 3; ++c)
        out[9 * a + 3 * b + c] = t2[a][b][0] * B[0][c] + t2[a][b][1] * B[1][c] + t2[a][b][2] * B[2][c];
}

// The integrated gradient G1[i][j][k] of the mollified Kelvin solution over
// the element (mhs/fullspace/kernels.py:148-157), in the element frame where
// the normal is e3: read by the slip displacement and the force stress.
template <class S>
MHS_HD void g1_local(const double* W, double z, double eps, const Material& m,
                     double G1[3][3][3]) {
  double zp[4] = {1.0, z, z * z, z * z * z};
  const int s5 = nslot(5);
  constexpr Spec sp = S::spec;
  constexpr int o3 = sp.w_off[nslot(3)], o5 = sp.w_off[nslot(5)];
  const double V3[3] = {-W[o3 + tri_idx(1, 0)], -W[o3 + tri_idx(0, 1)], z * W[o3]};
  const double V5[3] = {-W[o5 + tri_idx(1, 0)], -W[o5 + tri_idx(0, 1)], z * W[o5]};
  const double e2 = eps * eps;
  const double f6 = 6.0 * m.one_m_nu * e2;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) {
        const int ca = (i == 0) + (j == 0) + (k == 0), cb = (i == 1) + (j == 1) + (k == 1);
        const double T = lift_local<S>(W, s5, ca, cb, 3 - ca - cb, zp);
        double g = (i == j ? -m.c34 * V3[k] : 0.0);
        g = g + (i == k ? V3[j] : 0.0);
        g = g + (j == k ? V3[i] : 0.0);
        g = g - 3.0 * T;
        g = g - (i == j ? f6 * V5[k] : 0.0);
        G1[i][j][k] = g * m.C1;
      }
}

// Slip -> displacement (mhs/fullspace/kernels.py:159-163), evaluated in the
// element frame, then rotated.
template <class S>
MHS_HD void kernel_U(const Frame& f, const double* W, double z, double eps, const Material& m,
                     double* U) {
  double G1[3][3][3];
  g1_local<S>(W, z, eps, m, G1);
  double Ul[3][3];
  for (int i = 0; i < 3; ++i) {
    const double tr = G1[i][0][0] + G1[i][1][1] + G1[i][2][2];
    for (int j = 0; j < 3; ++j)
      Ul[i][j] = -(m.mu * G1[i][j][2] + (j == 2 ? m.lam_d * tr : 0.0) + m.mu * G1[i][2][j]);
  }
  rotate2(f, Ul, U);
}

// Force density -> displacement, the Kelvin single layer (mhs/fullspace/
// kernels.py:165-173): C1 [(3 - 4 nu) I1 delta_ij + T23_ij + 2 (1 - nu)
// eps^2 I3 delta_ij], in the element frame, then rotated.
template <class S>
MHS_HD void kernel_G(const Frame& f, const double* W, double z, double eps, const Material& m,
                     double* G) {
  const double zp[3] = {1.0, z, z * z};
  constexpr Spec sp = S::spec;
  const double I1 = W[sp.w_off[nslot(1)]], I3 = W[sp.w_off[nslot(3)]];
  const double f2 = 2.0 * m.one_m_nu * (eps * eps);
  double Gl[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const int ca = (i == 0) + (j == 0), cb = (i == 1) + (j == 1);
      double g = (i == j ? m.c34 * I1 : 0.0);
      g = g + lift_local<S>(W, nslot(3), ca, cb, 2 - ca - cb, zp);
      g = g + (i == j ? f2 * I3 : 0.0);
      Gl[i][j] = m.C1 * g;
    }
  rotate2(f, Gl, G);
}

// Force density -> stress (mhs/fullspace/kernels.py:175-181):
// S[i][j][c] = lam delta_ij G1[a][c][a] + mu (G1[i][c][j] + G1[j][c][i]),
// in the element frame, then rotated in all three indices.
template <class S>
MHS_HD void kernel_S(const Frame& f, const double* W, double z, double eps, const Material& m,
                     double* Sout) {
  double G1[3][3][3];
  g1_local<S>(W, z, eps, m, G1);
  double Sl[3][3][3];
  for (int c = 0; c < 3; ++c) {
    const double tr = G1[0][c][0] + G1[1][c][1] + G1[2][c][2];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        Sl[i][j][c] = (i == j ? m.lam_d * tr : 0.0) + m.mu * G1[i][c][j] + m.mu * G1[j][c][i];
  }
  rotate3(f, Sl, Sout);
}

// Lifted local-frame quantities of the stress kernel, one vector per node:
// I3, I5, then T25(a, b) and T27(a, b) over the six components of a
// symmetric rank-2 tensor and T47 over the fifteen of a symmetric rank-4
// tensor, each at tri_idx(count of e1, count of e2).  H is linear in them.
constexpr int NLIFT = 29;
constexpr int L_I3 = 0, L_I5 = 1, L_T25 = 2, L_T27 = 8, L_T47 = 14;

template <class S>
MHS_HD void lift_H(const double* W, double z, double* L) {
  const double zp[5] = {1.0, z, z * z, z * z * z, z * z * z * z};
  const int s5 = nslot(5), s7 = nslot(7);
  constexpr Spec sp = S::spec;
  L[L_I3] = W[sp.w_off[nslot(3)]];
  L[L_I5] = W[sp.w_off[nslot(5)]];
#pragma unroll
  for (int ca = 0; ca <= 2; ++ca)
#pragma unroll
    for (int cb = 0; ca + cb <= 2; ++cb) {
      L[L_T25 + tri_idx(ca, cb)] = lift_local<S>(W, s5, ca, cb, 2 - ca - cb, zp);
      L[L_T27 + tri_idx(ca, cb)] = lift_local<S>(W, s7, ca, cb, 2 - ca - cb, zp);
    }
#pragma unroll
  for (int ca = 0; ca <= 4; ++ca)
#pragma unroll
    for (int cb = 0; ca + cb <= 4; ++cb)
      L[L_T47 + tri_idx(ca, cb)] = lift_local<S>(W, s7, ca, cb, 4 - ca - cb, zp);
}

// Slip -> total stress (mhs/fullspace/kernels.py:182-210) from the lifted
// quantities, assembled in the element frame and rotated.
MHS_HD void H_from_lift(const Frame& f, const double* L, double eps, const Material& m, double* H) {
  const double I3 = L[L_I3];
  const double I5 = L[L_I5];
  const double e2 = eps * eps;
  const double f2 = 2.0 * m.one_m_nu * e2;
  double T25[3][3], T27[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const int ca = (i == 0) + (j == 0), cb = (i == 1) + (j == 1);
      T25[i][j] = L[L_T25 + tri_idx(ca, cb)];
      T27[i][j] = L[L_T27 + tri_idx(ca, cb)];
    }
  // D2[r][p][s][q] / C1
  double D2[3][3][3][3];
  for (int r = 0; r < 3; ++r)
    for (int p = 0; p < 3; ++p)
      for (int s = 0; s < 3; ++s)
        for (int q = 0; q < 3; ++q) {
          const double drp = r == p, dsq = s == q, drs = r == s, dpq = p == q, dps = p == s,
                       drq = r == q;
          const int ca = (r == 0) + (p == 0) + (s == 0) + (q == 0);
          const int cb = (r == 1) + (p == 1) + (s == 1) + (q == 1);
          const double T47 = L[L_T47 + tri_idx(ca, cb)];
          double d = -m.c34 * (drp * dsq * I3 - 3.0 * (drp * T25[s][q]));
          d += drs * dpq * I3 - 3.0 * (drs * T25[p][q]);
          d += dps * drq * I3 - 3.0 * (dps * T25[r][q]);
          d += -3.0 * ((drq * T25[p][s] + dpq * T25[r][s]) + dsq * T25[r][p]);
          d += 15.0 * T47;
          d += f2 * (-3.0 * (drp * dsq * I5) + 15.0 * (drp * T27[s][q]));
          D2[r][p][s][q] = d * m.C1;
        }
  double B[3][3][3];
  for (int r = 0; r < 3; ++r)
    for (int s = 0; s < 3; ++s) {
      const double trD = D2[r][0][s][0] + D2[r][1][s][1] + D2[r][2][s][2];
      for (int j = 0; j < 3; ++j)
        B[r][s][j] = (j == 2 ? m.lam_d * trD : 0.0) + m.mu * D2[r][j][s][2] + m.mu * D2[r][2][s][j];
    }
  double Hl[3][3][3];
  for (int j = 0; j < 3; ++j) {
    const double trB = B[0][0][j] + B[1][1][j] + B[2][2][j];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        Hl[a][b][j] = -((a == b ? m.lam_d * trB : 0.0) + m.mu * (B[a][b][j] + B[b][a][j]));
  }
  rotate3(f, Hl, H);
}

template <class S>
MHS_HD void kernel_H(const Frame& f, const double* W, double z, double eps, const Material& m,
                     double* H) {
  double L[NLIFT] = {};
  lift_H<S>(W, z, L);
  H_from_lift(f, L, eps, m, H);
}

// Coefficients of the global sigma_zz row: H[2][2][j] = sum_l col[l][j] L_l,
// read off by evaluating H_from_lift on the unit vector of lifted slot l.
MHS_HD void szz_coefficient(const Frame& f, double eps, const Material& m, int l, double* col3) {
  double e[NLIFT] = {};
  e[l] = 1.0;
  double H[27] = {};
  H_from_lift(f, e, eps, m, H);
  for (int j = 0; j < 3; ++j) col3[j] = H[9 * 2 + 3 * 2 + j];
}

// ----------------------------------------------------------- direct term
// One source triangle at one observer, all K nodes: near field by the
// closed-form recursion (sqrt(|x - c|^2 + eps^2) <= D_STAR L), far field by
// the product rule r12 (12 x 12), r8 (8 x 8) beyond far_switch_l L
// (D_STAR_DISTANT: mhs/fullspace/moments.py:551-601,
// mhs/fullspace/kernels.py:126-215).  R_FAR is the arithmetic type of the
// far-field quadrature; the mixed form passes its own float rules and
// switch distance.
// The node loops are fully unrolled so that every output offset is a
// compile-time constant: a -O3 device build with them kept rolled returned
// wrong P >= 1 tensors where this function is inlined into the fold kernels.
template <int P, int WANT, class R_FAR = double, class Q = QuadRule>
MHS_HD void direct_eval(const Frame& f, const Q& r12, const Q& r8,
                        const double* x, double eps, const Material& m,
                        double* U, double* H, double* E, double near_l = cst::D_STAR,
                        double far_switch_l = cst::D_STAR_DISTANT) {
  using S = DirectSpec<P, WANT>;
  constexpr Spec sp = S::spec;
  constexpr int K = n_nodes(P);
  constexpr int NW = sp.w_off[NS];
  const double d0 = x[0] - f.c[0], d1 = x[1] - f.c[1], d2 = x[2] - f.c[2];
  const double D = sqrt(((d0 * d0 + d1 * d1) + d2 * d2) + eps * eps);
  double z, X0, X1;
  to_plane(f, x, z, X0, X1);
  const double h2 = z * z + eps * eps;
  const double e4 = 15.0 * (eps * eps) * (eps * eps) / (8.0 * cst::PI);
  // closed form within near_l element lengths: D_STAR (mhs's hybrid split),
  // the mixed form's narrower zone, or (the full-space API's far_field
  // options) everywhere / nowhere; the far rule beyond
  if (D <= near_l * f.L) {
    MomentTable<S> T;
    closed_moments<S>(f, X0, X1, h2, T);
    double c[K][ntri(P)];
    shape_coeffs<P>(f, X0, X1, c);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double W[NW] = {};
      weight_closed<S, P>(T, c, k, W);
      if (WANT & W_U) kernel_U<S>(f, W, z, eps, m, U + 9 * k);
      if (WANT & W_H) kernel_H<S>(f, W, z, eps, m, H + 27 * k);
      if (WANT & W_E) E[k] = e4 * W[sp.w_off[nslot(7)]];
    }
  } else {
    const Q& q = (D > far_switch_l * f.L) ? r8 : r12;
    double Wbuf[K * NW] = {};
    double* W = P > 0 ? in_memory(Wbuf) : Wbuf;   // K * NW doubles at P >= 1
    weight_far<S, P, R_FAR>(q, X0, X1, h2, W);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (WANT & W_U) kernel_U<S>(f, W + k * NW, z, eps, m, U + 9 * k);
      if (WANT & W_H) kernel_H<S>(f, W + k * NW, z, eps, m, H + 27 * k);
      if (WANT & W_E) E[k] = e4 * W[k * NW + sp.w_off[nslot(7)]];
    }
  }
}

// Force (Kelvin single-layer) source of one triangle at one observer, all K
// nodes: G[k] (9) and / or S[k] (27), from the force source's weighted
// tables with the same near / far split as direct_eval (node loops fully
// unrolled, as there).
template <int P, int WANT, class Q = QuadRule>
MHS_HD void force_eval(const Frame& f, const Q& r12, const Q& r8, const double* x, double eps,
                       const Material& m, double* G, double* S, double near_l = cst::D_STAR,
                       double far_switch_l = cst::D_STAR_DISTANT) {
  using Sp = SpecF<P>;
  constexpr Spec sp = Sp::spec;
  constexpr int K = n_nodes(P);
  constexpr int NW = sp.w_off[NS];
  const double d0 = x[0] - f.c[0], d1 = x[1] - f.c[1], d2 = x[2] - f.c[2];
  const double D = sqrt(((d0 * d0 + d1 * d1) + d2 * d2) + eps * eps);
  double z, X0, X1;
  to_plane(f, x, z, X0, X1);
  const double h2 = z * z + eps * eps;
  if (D <= near_l * f.L) {
    MomentTable<Sp> T;
    closed_moments<Sp>(f, X0, X1, h2, T);
    double c[K][ntri(P)];
    shape_coeffs<P>(f, X0, X1, c);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double W[NW] = {};
      weight_closed<Sp, P>(T, c, k, W);
      if (WANT & W_G) kernel_G<Sp>(f, W, z, eps, m, G + 9 * k);
      if (WANT & W_S) kernel_S<Sp>(f, W, z, eps, m, S + 27 * k);
    }
  } else {
    const Q& q = (D > far_switch_l * f.L) ? r8 : r12;
    double Wbuf[K * NW] = {};
    double* W = P > 0 ? in_memory(Wbuf) : Wbuf;
    weight_far<Sp, P, double>(q, X0, X1, h2, W);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (WANT & W_G) kernel_G<Sp>(f, W + k * NW, z, eps, m, G + 9 * k);
      if (WANT & W_S) kernel_S<Sp>(f, W + k * NW, z, eps, m, S + 27 * k);
    }
  }
}

// ------------------------------------------------------------ image data
// Per-material image coefficients (built on the host from the generated
// rationals): R records c(z) = cz[r][0] + z cz[r][1] + z^2 cz[r][2], scale
// included; Q records a single number each, scale applied after the sum
// (mhs/kernels/image.py:95-104, 257-297).
struct ImageCoef {
  const double* r_dg;    // [MHS_R_NDG][3]
  const double* r_ddg;   // [MHS_R_NDDG][3]
  const double* q_dg;    // [MHS_Q_NDG]
  const double* q_ddg;   // [MHS_Q_NDDG]
};

// View of the packed coefficient block (host_prep.h: image_coef).
MHS_HD ImageCoef image_coef_view(const double* base) {
  ImageCoef c;
  c.r_dg = base;
  c.r_ddg = c.r_dg + 3 * MHS_R_NDG;
  c.q_dg = c.r_ddg + 3 * MHS_R_NDDG;
  c.q_ddg = c.q_dg + MHS_Q_NDG;
  return c;
}

// Basis-product coefficients G_abc(alpha, beta): the coefficient of
// x^alpha y^beta w^gamma in prod over the a+b+c Cartesian slots of
// (e1_i x + e2_i y + n_i w), i.e. the geometry the lift sums per (alpha, beta)
// group (mhs/fullspace/kernels.py:63-87), one polynomial per (a, b, c).
constexpr int G_RMAX = 5;
MHS_FI constexpr int abc_idx(int a, int b, int c) {
  return (a + b + c) * (a + b + c + 1) * (a + b + c + 2) / 6 + tri_idx(b, c);
}
MHS_FI constexpr int g_rank_off(int r) {  // sum_{r' < r} ntri(r')^2
  int s = 0;
  for (int i = 0; i < r; ++i) s += ntri(i) * ntri(i);
  return s;
}
MHS_FI constexpr int g_off(int a, int b, int c) {
  return g_rank_off(a + b + c) + tri_idx(b, c) * ntri(a + b + c);
}
constexpr int G_SIZE = g_rank_off(G_RMAX + 1);

MHS_HD void build_basis_products(const Frame& f, double* G) {
  G[0] = 1.0;
  for (int r = 1; r <= G_RMAX; ++r)
    for (int b = 0; b <= r; ++b)
      for (int c = 0; b + c <= r; ++c) {
        const int a = r - b - c;
        int pa = a, pb = b, pc = c, comp;
        if (c > 0) { pc = c - 1; comp = 2; }
        else if (b > 0) { pb = b - 1; comp = 1; }
        else { pa = a - 1; comp = 0; }
        const double* src = G + g_off(pa, pb, pc);
        double* dst = G + g_off(a, b, c);
        const double ux = f.e1[comp], uy = f.e2[comp], uw = f.n[comp];
        for (int al = 0; al <= r; ++al)
          for (int be = 0; al + be <= r; ++be) {
            double v = 0.0;
            if (al >= 1) v += ux * src[tri_idx(al - 1, be)];
            if (be >= 1) v += uy * src[tri_idx(al, be - 1)];
            if (al + be <= r - 1) v += uw * src[tri_idx(al, be)];
            dst[tri_idx(al, be)] = v;
          }
      }
}

// Traction-operator contraction of DG (slip -> displacement) with the real
// element's normal (mhs/kernels/image.py:127-137).
MHS_HD void contract_dg(const double* DG, const double* nrm, const Material& m, double* U) {
  for (int i = 0; i < 3; ++i) {
    const double tr = DG[9 * i + 0] + DG[9 * i + 4] + DG[9 * i + 8];
    for (int k = 0; k < 3; ++k) {
      double s1 = 0.0, s2 = 0.0;
      for (int l = 0; l < 3; ++l) {
        s1 += nrm[l] * DG[9 * i + 3 * k + l];
        s2 += nrm[l] * DG[9 * i + 3 * l + k];
      }
      U[3 * i + k] = m.mu * s1 + m.mu * s2 + m.lam * nrm[k] * tr;
    }
  }
}

// H from the traction-operator image S[i][p][k] of DDG: the symmetric part
// in (i, p) through Hooke's law, per slip component k.
MHS_HD void hooke_from_traction(const double (&S)[3][3][3], const Material& m, double* H) {
  for (int k = 0; k < 3; ++k) {
    double e[3][3];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) e[a][b] = 0.5 * (S[a][b][k] + S[b][a][k]);
    const double tr = e[0][0] + e[1][1] + e[2][2];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double v = 2.0 * m.mu * e[a][b];
        if (a == b) v += m.lam * tr;
        H[9 * a + 3 * b + k] = v;
      }
  }
}

// DDG (i, j, p, m) -> displacement gradient -> symmetric Hooke stress
// (mhs/kernels/image.py:138-161).
MHS_HD void contract_ddg(const double* DDG, const double* nrm, const Material& m, double* H) {
  double S[3][3][3];
  for (int i = 0; i < 3; ++i)
    for (int p = 0; p < 3; ++p) {
      const double trm = DDG[27 * i + 9 * 0 + 3 * p + 0] + DDG[27 * i + 9 * 1 + 3 * p + 1] +
                         DDG[27 * i + 9 * 2 + 3 * p + 2];
      for (int k = 0; k < 3; ++k) {
        double s1 = 0.0, s2 = 0.0;
        for (int l = 0; l < 3; ++l) {
          s1 += nrm[l] * DDG[27 * i + 9 * k + 3 * p + l];
          s2 += nrm[l] * DDG[27 * i + 9 * l + 3 * p + k];
        }
        S[i][p][k] = m.mu * s1 + m.mu * s2 + m.lam * nrm[k] * trm;
      }
    }
  hooke_from_traction(S, m, H);
}

// --------------------------------------------------------- image R-family
// The records of one node: the monomial moments in monomial order, each
// followed by its own records (sorted by monomial, so every slot receives
// its records in table order) with coefficient c(z) = c0 + z (c1 + z c2) at
// the observer's depth.  The displacement readout accumulates DG (27
// slots); the stress readout contracts each DDG record straight into the
// traction-operator image S[i][p][k] (27 entries, as 9 i + 3 p + k): record
// slot (i, a, p, b) adds mun[b] v to S[i][p][a], mun[a] v to S[i][p][b] and,
// when a = b, lamn[k] v to every S[i][p][k] (mun = mu n, lamn = lam n; the
// scale is already in the coefficients).  One instantiation per monomial:
// its records are straight-line code with literal slots.
template <class S, int WANT, int MI>
MHS_FI void r_mono_records(double tm, double zo, const ImageCoef& ic, double* D,
                           const double* mun, const double* lamn) {
  if constexpr (WANT == W_U) {
#define MHS_RTU(r, mi, slot)                                           \
  if constexpr ((mi) == MI) {                                          \
    const double* cz = ic.r_dg + 3 * (r);                              \
    D[slot] += (cz[0] + zo * (cz[1] + zo * cz[2])) * tm;               \
  }
    MHS_R_TERMS_DG(MHS_RTU)
#undef MHS_RTU
  } else {
#define MHS_RTD(r, mi, slot)                                                        \
  if constexpr ((mi) == MI) {                                                       \
    const double* cz = ic.r_ddg + 3 * (r);                                          \
    const double v = (cz[0] + zo * (cz[1] + zo * cz[2])) * tm;                      \
    constexpr int qi = (slot) / 27, qa = ((slot) / 9) % 3, qp = ((slot) / 3) % 3;  \
    constexpr int qb = (slot) % 3;                                                  \
    D[9 * qi + 3 * qp + qa] += mun[qb] * v;                                         \
    D[9 * qi + 3 * qp + qb] += mun[qa] * v;                                         \
    if constexpr (qa == qb) {                                                       \
      D[9 * qi + 3 * qp + 0] += lamn[0] * v;                                        \
      D[9 * qi + 3 * qp + 1] += lamn[1] * v;                                        \
      D[9 * qi + 3 * qp + 2] += lamn[2] * v;                                        \
    }                                                                               \
  }
    MHS_R_TERMS_DDG(MHS_RTD)
#undef MHS_RTD
  }
}

// Cartesian monomial moment D1^A D2^B D3^C / R2^N of one node from the
// basis products G and the node's weighted table Wr (mhs/kernels/image.py:
// 456-480): sum over t of (-1)^t zp^(r - t) sum_al G[al, t - al]
// W_N[al, t - al], with every exponent and table index known at compile time.
template <class S, int A, int B, int C, int N>
MHS_FI double r_moment_ct(const double* G, const double* Wr, const double (&zpow)[G_RMAX + 1]) {
  constexpr Spec sp = S::spec;
  constexpr int r = A + B + C;
  constexpr int wo = sp.w_off[nslot(N)];
  const double* g = G + g_off(A, B, C);
  double acc = 0.0;
#pragma unroll
  for (int t = 0; t <= r; ++t) {
    double part = 0.0;
#pragma unroll
    for (int al = 0; al <= t; ++al) part += g[tri_idx(al, t - al)] * Wr[wo + tri_idx(al, t - al)];
    const double v = zpow[r - t] * part;
    acc += (t & 1) ? -v : v;
  }
  return acc;
}

// The records of one node.  The node's table is read once into registers;
// the monomial loop runs at run time (its counter opaque, so the compiler
// neither unrolls it nor threads it into its cases) and dispatches to one
// case per monomial whose moment and records are straight-line code with
// literal indices: only the table, the 27 sums and the moment are live, and
// nothing is addressed at run time but the shared tables.
template <class S, int WANT, class WT>
MHS_FI void image_r_records(const double* G, WT W, const double (&zpow)[G_RMAX + 1], double zo,
                            const ImageCoef& ic, double* D, const double* mun,
                            const double* lamn) {
  constexpr int NW = S::spec.w_off[NS];
  double Wr[NW];
#pragma unroll
  for (int j = 0; j < NW; ++j) Wr[j] = W[j];
#pragma unroll 1
  for (int i = 0; i < MHS_R_NMONO; ++i) {
    switch (opaque(i)) {
#define MHS_RCASE(mi_, a, b, c, n)                                                       \
  case mi_:                                                                              \
    r_mono_records<S, WANT, mi_>(r_moment_ct<S, a, b, c, n>(G, Wr, zpow), zo, ic, D, mun, \
                                 lamn);                                                  \
    break;
      MHS_R_MONO(MHS_RCASE)
#undef MHS_RCASE
      default:
        break;
    }
  }
}

// Powers zp^0..zp^G_RMAX of the observer's height over the reflected
// element's plane (the moments' sign-alternating z factors).
MHS_FI void image_r_zpow(const Frame& fi, const double* x, double (&zpow)[G_RMAX + 1]) {
  double zp, X0, X1;
  to_plane(fi, x, zp, X0, X1);
  zpow[0] = 1.0;
  for (int i = 1; i <= G_RMAX; ++i) zpow[i] = zpow[i - 1] * zp;
}

// Weighted tables of the image frame for every node k, written to
// Wall + k NW (a pointer or a StridedTable): the closed form within near_l
// element lengths (every node's table from one moment table), else the
// 12 x 12 / 8 x 8 far rules, one pass per node.  PART restricts the call
// to the observers of one form (TAB_CLOSED, TAB_FAR; others are left
// untouched), so that each form can run in its own kernel with its own
// registers.
enum : int { TAB_BOTH = 0, TAB_CLOSED = 1, TAB_FAR = 2 };

template <int P, class R_FAR = double, int PART = TAB_BOTH, class Q = QuadRule,
          class WO = double*>
MHS_HD void image_r_tables(const Frame& fi, const Q& r12, const Q& r8, const double* x,
                           double eps, WO Wall, double near_l = cst::D_STAR,
                           double far_switch_l = cst::D_STAR_DISTANT) {
  using S = SpecImg<P>;
  constexpr int K = n_nodes(P);
  constexpr int NW = S::spec.w_off[NS];
  const double d0 = x[0] - fi.c[0], d1 = x[1] - fi.c[1], d2 = x[2] - fi.c[2];
  const double D = sqrt(((d0 * d0 + d1 * d1) + d2 * d2) + eps * eps);
  const bool closed = D <= near_l * fi.L;
  if ((PART == TAB_CLOSED && !closed) || (PART == TAB_FAR && closed)) return;
  double zp, X0, X1;
  to_plane(fi, x, zp, X0, X1);
  const double h2 = zp * zp + eps * eps;
  if constexpr (PART != TAB_FAR) {
    if (closed) {
      MomentTable<S> T;
      closed_moments<S>(fi, X0, X1, h2, T);
      double c[K][ntri(P)];
      shape_coeffs<P>(fi, X0, X1, c);
      for (int k = 0; k < K; ++k) weight_closed<S, P>(T, c, k, Wall + k * NW);
      return;
    }
  }
  if constexpr (PART != TAB_CLOSED) {
    const Q& q = (D > far_switch_l * fi.L) ? r8 : r12;
    if constexpr (K == 1 || PART == TAB_BOTH) {
      weight_far<S, P, R_FAR>(q, X0, X1, h2, Wall);
    } else {
      // one pass per node (as weight_far makes them: NW accumulators are
      // a pass's limit), kept as a loop so that only one pass is live
#pragma unroll 1
      for (int k = 0; k < K; ++k) {
        const int kk = opaque(k);
        weight_far_nodes<S, P, R_FAR, 1>(q, R_FAR(X0), R_FAR(X1), R_FAR(h2), kk, kk, Wall);
      }
    }
  }
}
static_assert(FAR_ACC_MAX / SpecImg<1>::spec.w_off[NS] == 1 &&
                  FAR_ACC_MAX / SpecImg<2>::spec.w_off[NS] == 1,
              "the image tables' far passes take one node each");

// The records of one node from its weighted table W (a pointer or a
// StridedTable), contracted into the node's displacement (U, 9 entries) or
// total-stress (H, 27 entries) influence.
template <int P, int WANT, class WT>
MHS_FI void image_r_node(const double* G, WT W, const double (&zpow)[G_RMAX + 1], double zo,
                         const double* nrm, const Material& m, const ImageCoef& ic, double* U,
                         double* H) {
  using S = SpecImg<P>;
  const double mun[3] = {m.mu * nrm[0], m.mu * nrm[1], m.mu * nrm[2]};
  const double lamn[3] = {m.lam * nrm[0], m.lam * nrm[1], m.lam * nrm[2]};
  if constexpr ((WANT & W_U) != 0) {
    double DG[27] = {};
    image_r_records<S, W_U>(G, W, zpow, zo, ic, DG, mun, lamn);
    contract_dg(DG, nrm, m, U);
  }
  if constexpr ((WANT & W_H) != 0) {
    double Sf[27] = {};
    image_r_records<S, W_H>(G, W, zpow, zo, ic, Sf, mun, lamn);
    double St[3][3][3];
    for (int i = 0; i < 3; ++i)
      for (int p = 0; p < 3; ++p)
        for (int c = 0; c < 3; ++c) St[i][p][c] = Sf[9 * i + 3 * p + c];
    hooke_from_traction(St, m, H);
  }
}

// The closed-form R-family on the reflected element (mhs/kernels/image.py:
// 435-497): weighted tables of the image frame, Cartesian monomial moments
// D1^a D2^b D3^c / R2^n from the basis products G, then the generated records.
// The device pipeline runs the two halves as separate kernels over a table
// buffer (image_r_tables, image_r_node); this composition serves the
// single-point paths.
template <int P, int WANT, class R_FAR = double, class Q = QuadRule>
MHS_HD void image_r_eval(const Frame& fi, const double* G, const double* nrm,
                         const Q& r12, const Q& r8, const double* x, double eps,
                         const Material& m, const ImageCoef& ic, double* U, double* H,
                         double near_l = cst::D_STAR,
                         double far_switch_l = cst::D_STAR_DISTANT) {
  using S = SpecImg<P>;
  constexpr int K = n_nodes(P);
  constexpr int NW = S::spec.w_off[NS];
  double zpow[G_RMAX + 1];
  image_r_zpow(fi, x, zpow);
  double Wbuf[K * NW];
  double* Wall = P > 0 ? in_memory(Wbuf) : Wbuf;
  image_r_tables<P, R_FAR>(fi, r12, r8, x, eps, Wall, near_l, far_switch_l);
#pragma unroll 1
  for (int k = 0; k < K; ++k)
    image_r_node<P, WANT>(G, Wall + k * NW, zpow, x[2], nrm, m, ic, U ? U + 9 * k : nullptr,
                          H ? H + 27 * k : nullptr);
}

// --------------------------------------------------------- image Q-family
// Exact distance from a point to a closed triangle (mhs/kernels/image.py:
// 170-208), used by the Q-family order law.
MHS_HD double triangle_distance(const double* x, const double* t) {
  const double* a = t;
  const double* b = t + 3;
  const double* c = t + 6;
  double ab[3], ac[3], ap[3], nr[3];
  for (int j = 0; j < 3; ++j) {
    ab[j] = b[j] - a[j];
    ac[j] = c[j] - a[j];
    ap[j] = x[j] - a[j];
  }
  cross3(ab, ac, nr);
  const double d20 = dot3(ap, ab), d21 = dot3(ap, ac);
  const double d00 = dot3(ab, ab), d01 = dot3(ab, ac), d11 = dot3(ac, ac);
  const double den = d00 * d11 - d01 * d01;
  const double v = (d11 * d20 - d01 * d21) / den;
  const double w = (d00 * d21 - d01 * d20) / den;
  const double u = 1.0 - v - w;
  if (u >= 0.0 && v >= 0.0 && w >= 0.0) return fabs(dot3(ap, nr)) / norm3(nr);
  double best = INFINITY;
  const double* P0[3] = {a, b, c};
  const double* P1[3] = {b, c, a};
  for (int e = 0; e < 3; ++e) {
    double ev[3], d[3];
    for (int j = 0; j < 3; ++j) {
      ev[j] = P1[e][j] - P0[e][j];
      d[j] = x[j] - P0[e][j];
    }
    double tt = dot3(d, ev) / dot3(ev, ev);
    tt = tt < 0.0 ? 0.0 : (tt > 1.0 ? 1.0 : tt);
    double q[3];
    for (int j = 0; j < 3; ++j) q[j] = x[j] - (P0[e][j] + tt * ev[j]);
    const double dist = norm3(q);
    if (dist < best) best = dist;
  }
  return best;
}

// Gauss order per observer: clip(ceil(C L / sqrt(delta^2 + eps^2)) + order)
// with delta the distance to the image triangle (image.py:211-254).
MHS_HD int q_gauss_order(const double* x, const double* tri_img, double eps, double L, int order) {
  const double delta = triangle_distance(x, tri_img);
  const double scale = sqrt(delta * delta + eps * eps);
  double nq = ceil(cst::IMAGE_Q_BUDGET_C * L / scale) + (double)order;
  if (nq < cst::IMAGE_Q_GAUSS_MIN) nq = cst::IMAGE_Q_GAUSS_MIN;
  if (nq > cst::IMAGE_Q_GAUSS_MAX) nq = cst::IMAGE_Q_GAUSS_MAX;
  return (int)nq;
}

// A Q-family rule on the REAL element held in arrays: Cartesian nodes y,
// weights wN[k] = area weight x N_k (image.py:325-339).
template <int P>
struct QRule {
  static constexpr int K = n_nodes(P);
  int nq;
  const double* y;    // nq x 3
  const double* wN;   // nq x K
  MHS_HD int count() const { return nq; }
  MHS_HD void node(int t, double* yy, double* w) const {
    yy[0] = y[3 * t];
    yy[1] = y[3 * t + 1];
    yy[2] = y[3 * t + 2];
    for (int k = 0; k < K; ++k) w[k] = wN[t * K + k];
  }
};

template <int P>
MHS_HD void build_qrule(const Frame& f, const double* glx, const double* glw, int n,
                        double* y, double* wN) {
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
      for (int c = 0; c < 3; ++c) y[3 * q + c] = (l0 * f.v[0][c] + x1 * f.v[1][c]) + x2 * f.v[2][c];
      const double e0 = (l0 * f.p[0][0] + x1 * f.p[1][0]) + x2 * f.p[2][0];
      const double e1 = (l0 * f.p[0][1] + x1 * f.p[1][1]) + x2 * f.p[2][1];
      double N[K];
      shape_at<P>(f, e0, e1, N);
      const double wq = ww * (2.0 * f.area);
      for (int k = 0; k < K; ++k) wN[q * K + k] = wq * N[k];
    }
  }
}

// Q-family moments by quadrature, contracted (image.py:315-432).
//
// Per node k, the basis sums B_m = sum_t wN_t[k] D1^a D2^b D3^c / (R2^n Q^q)
// of exactly the monomials the contraction reads, in passes over ranges of
// the monomial index: a pass keeps its range's sums in registers through the
// point loop (the generated lists spell every monomial's exponents as
// literals, so the products and the record-by-record contraction are
// straight-line code) and then contracts that range's records.  Each
// monomial is formed as the ordered product p1[a] p2[b] p3[c] pr[n] pq[q]
// with p[0] = 1 (a factor of one is exact), the points are summed in rule
// order, and -- the records being sorted by monomial -- passes in
// increasing range add the records in table order, as mhs does.  Rule:
// count() and node(t, y, wN[K]) in the arithmetic type R of the point sums
// (double; float for the mixed form's far pairs).
//
// The stress readout contracts each DDG record straight into the 27 entries
// of its traction-operator image S[i][p][k] = mu sum_l n_l (DDG[i,k,p,l] +
// DDG[i,l,p,k]) + lam n_k sum_j DDG[i,j,p,j] (contract_ddg), so a pass holds
// 27 accumulators instead of 81: with mun = mu n and lamn = lam n, record
// slot (i, a, p, b) adds mun[b] v to S[i][p][a], mun[a] v to S[i][p][b] and,
// when a = b, lamn[k] v to every S[i][p][k].  D is DG (27) for the
// displacement readout, S (27, as 9 i + 3 p + k) for the stress readout.
template <int P, int WANT, int LO, int HI, class Rule, class R>
MHS_HD void image_q_pass(const Rule& q, int k, R x0, R x1, R x2, R e2, const ImageCoef& ic,
                         double* D, const double* mun, const double* lamn) {
  constexpr int K = n_nodes(P);
  R bs[HI - LO];
#define MHS_QZ(i, a, b, c, n, qq) \
  if constexpr ((i) >= LO && (i) < HI) bs[(i) - LO] = R(0);
  if constexpr (WANT == W_U) { MHS_Q_MONO_DG(MHS_QZ) }
  else { MHS_Q_MONO_DDG(MHS_QZ) }
#undef MHS_QZ
  const int nq = q.count();
#pragma unroll 1
  for (int t = 0; t < nq; ++t) {
    R y[3], wN[K];
    q.node(t, y, wN);
    const R d1 = x0 - y[0];
    const R d2 = x1 - y[1];
    const R d3 = x2 + y[2];
    const R r2 = sqrt(((d1 * d1 + d2 * d2) + d3 * d3) + e2);
    const R ir = R(1) / r2, iq = R(1) / (r2 - d3);
    R p1[5], p2[5], p3[5], pr[8], pq[5];
    p1[0] = R(1); p2[0] = R(1); p3[0] = R(1); pr[0] = R(1); pq[0] = R(1);
    p1[1] = d1; p2[1] = d2; p3[1] = d3; pr[1] = ir; pq[1] = iq;
#pragma unroll
    for (int i = 2; i < 5; ++i) {
      p1[i] = p1[i - 1] * d1;
      p2[i] = p2[i - 1] * d2;
      p3[i] = p3[i - 1] * d3;
      pq[i] = pq[i - 1] * iq;
    }
#pragma unroll
    for (int i = 2; i < 8; ++i) pr[i] = pr[i - 1] * ir;
    const R w = wN[k];
#define MHS_QA(i, a, b, c, n, qq) \
  if constexpr ((i) >= LO && (i) < HI) \
    bs[(i) - LO] += ((((p1[a] * p2[b]) * p3[c]) * pr[n]) * pq[qq]) * w;
    if constexpr (WANT == W_U) { MHS_Q_MONO_DG(MHS_QA) }
    else { MHS_Q_MONO_DDG(MHS_QA) }
#undef MHS_QA
  }
#define MHS_QTD(r, mi, slot)                                                     \
  if constexpr ((mi) >= LO && (mi) < HI) {                                      \
    const double v = ic.q_ddg[r] * bs[(mi) - LO];                                \
    constexpr int qi = (slot) / 27, qa = ((slot) / 9) % 3, qp = ((slot) / 3) % 3; \
    constexpr int qb = (slot) % 3;                                               \
    D[9 * qi + 3 * qp + qa] += mun[qb] * v;                                      \
    D[9 * qi + 3 * qp + qb] += mun[qa] * v;                                      \
    if constexpr (qa == qb) {                                                    \
      D[9 * qi + 3 * qp + 0] += lamn[0] * v;                                     \
      D[9 * qi + 3 * qp + 1] += lamn[1] * v;                                     \
      D[9 * qi + 3 * qp + 2] += lamn[2] * v;                                     \
    }                                                                            \
  }
#define MHS_QTU(r, mi, slot) \
  if constexpr ((mi) >= LO && (mi) < HI) D[slot] += ic.q_dg[r] * bs[(mi) - LO];
  if constexpr (WANT == W_U) { MHS_Q_TERMS_DG(MHS_QTU) }
  else { MHS_Q_TERMS_DDG(MHS_QTD) }
#undef MHS_QTD
#undef MHS_QTU
}

template <int P, int WANT, class Rule, class R = double>
MHS_HD void image_q_eval(const Rule& q, const double* nrm, const double* x, double eps,
                         const Material& m, const ImageCoef& ic, double* U, double* H) {
  static_assert(WANT == W_U || WANT == W_H, "one contraction per call");
  constexpr int K = n_nodes(P);
  const R e2 = R(eps * eps);
  const R x0 = R(x[0]), x1 = R(x[1]), x2 = R(x[2]);
  const double mun[3] = {m.mu * nrm[0], m.mu * nrm[1], m.mu * nrm[2]};
  const double lamn[3] = {m.lam * nrm[0], m.lam * nrm[1], m.lam * nrm[2]};
#pragma unroll 1
  for (int k = 0; k < K; ++k) {
    // float sums take half the registers: fewer, wider passes
    constexpr bool F32 = std::is_same<R, float>::value;
    if constexpr (WANT == W_U) {
      double DG[27] = {};
      if constexpr (F32) {
        image_q_pass<P, WANT, 0, MHS_Q_NMONO>(q, k, x0, x1, x2, e2, ic, DG, mun, lamn);
      } else {
        // two ranges of 34-35 of the 69 monomials
        image_q_pass<P, WANT, 0, 73>(q, k, x0, x1, x2, e2, ic, DG, mun, lamn);
        image_q_pass<P, WANT, 73, MHS_Q_NMONO>(q, k, x0, x1, x2, e2, ic, DG, mun, lamn);
      }
      for (int i = 0; i < 27; ++i) DG[i] *= m.scale_c;
      contract_dg(DG, nrm, m, U + 9 * k);
    } else {
      double Sf[27] = {};
      if constexpr (F32) {
        // two ranges of 84 and 83 of the 167 monomials
        image_q_pass<P, WANT, 0, 144>(q, k, x0, x1, x2, e2, ic, Sf, mun, lamn);
        image_q_pass<P, WANT, 144, MHS_Q_NMONO>(q, k, x0, x1, x2, e2, ic, Sf, mun, lamn);
      } else {
        // six ranges of 27-28 of the 167 monomials
        image_q_pass<P, WANT, 0, 55>(q, k, x0, x1, x2, e2, ic, Sf, mun, lamn);
        image_q_pass<P, WANT, 55, 107>(q, k, x0, x1, x2, e2, ic, Sf, mun, lamn);
        image_q_pass<P, WANT, 107, 144>(q, k, x0, x1, x2, e2, ic, Sf, mun, lamn);
        image_q_pass<P, WANT, 144, 180>(q, k, x0, x1, x2, e2, ic, Sf, mun, lamn);
        image_q_pass<P, WANT, 180, 208>(q, k, x0, x1, x2, e2, ic, Sf, mun, lamn);
        image_q_pass<P, WANT, 208, MHS_Q_NMONO>(q, k, x0, x1, x2, e2, ic, Sf, mun, lamn);
      }
      double S[3][3][3];
      for (int i = 0; i < 3; ++i)
        for (int p = 0; p < 3; ++p)
          for (int c = 0; c < 3; ++c) S[i][p][c] = Sf[9 * i + 3 * p + c] * m.scale_c;
      hooke_from_traction(S, m, H + 27 * k);
    }
  }
}

}  // namespace mhs
