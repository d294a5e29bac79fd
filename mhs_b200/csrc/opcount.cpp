// Algorithmic operation counts of the fold's work units and of one ordinary
// pair's direct and image terms, for the roofline.
//
// The engine headers are compiled here with `double` replaced by CountD, a
// scalar that performs the same IEEE arithmetic and counts every operation:
// add, subtract and multiply count one flop each (a fused multiply-add is a
// multiply plus an add, two flops); divisions, square roots and the other
// library functions are counted apart as special operations.  The entry
// points evaluate one work unit of the fold stage on caller-given inputs and
// return its counts; mhs_b200/flops.py combines them with the device census
// of a run (nodes per surface-load class, near-field edges per form).
// Nothing in the compute path uses this file.
#include <math.h>
#include <stdint.h>
#include <string.h>

namespace opc {
struct Ops {
  long long flop, div, sqrt, special;
};
static Ops g;
}  // namespace opc

struct CountD {
  double v;
  constexpr CountD() : v(0.0) {}
  constexpr CountD(double x) : v(x) {}
  constexpr CountD(long double x) : v((double)x) {}
  constexpr CountD(float x) : v((double)x) {}
  constexpr CountD(int x) : v((double)x) {}
  constexpr CountD(long x) : v((double)x) {}
  constexpr CountD(long long x) : v((double)x) {}
  constexpr CountD(unsigned x) : v((double)x) {}
  explicit constexpr operator double() const { return v; }
  explicit constexpr operator int() const { return (int)v; }
  explicit constexpr operator long long() const { return (long long)v; }
  CountD& operator+=(CountD o) { ++opc::g.flop; v += o.v; return *this; }
  CountD& operator-=(CountD o) { ++opc::g.flop; v -= o.v; return *this; }
  CountD& operator*=(CountD o) { ++opc::g.flop; v *= o.v; return *this; }
  CountD& operator/=(CountD o) { ++opc::g.div; v /= o.v; return *this; }
};
inline CountD operator+(CountD a, CountD b) { ++opc::g.flop; return CountD(a.v + b.v); }
inline CountD operator-(CountD a, CountD b) { ++opc::g.flop; return CountD(a.v - b.v); }
inline CountD operator*(CountD a, CountD b) { ++opc::g.flop; return CountD(a.v * b.v); }
inline CountD operator/(CountD a, CountD b) { ++opc::g.div; return CountD(a.v / b.v); }
inline CountD operator-(CountD a) { return CountD(-a.v); }
inline CountD operator+(CountD a) { return a; }
inline bool operator<(CountD a, CountD b) { return a.v < b.v; }
inline bool operator<=(CountD a, CountD b) { return a.v <= b.v; }
inline bool operator>(CountD a, CountD b) { return a.v > b.v; }
inline bool operator>=(CountD a, CountD b) { return a.v >= b.v; }
inline bool operator==(CountD a, CountD b) { return a.v == b.v; }
inline bool operator!=(CountD a, CountD b) { return a.v != b.v; }
inline CountD sqrt(CountD a) { ++opc::g.sqrt; return CountD(::sqrt(a.v)); }
inline CountD fabs(CountD a) { return CountD(::fabs(a.v)); }
inline CountD ceil(CountD a) { return CountD(::ceil(a.v)); }
inline CountD log(CountD a) { ++opc::g.special; return CountD(::log(a.v)); }
inline CountD log1p(CountD a) { ++opc::g.special; return CountD(::log1p(a.v)); }
inline CountD asin(CountD a) { ++opc::g.special; return CountD(::asin(a.v)); }
inline CountD atan2(CountD a, CountD b) { ++opc::g.special; return CountD(::atan2(a.v, b.v)); }
inline CountD hypot(CountD a, CountD b) { ++opc::g.special; return CountD(::hypot(a.v, b.v)); }
inline void sincos(CountD a, CountD* s, CountD* c) {
  opc::g.special += 2;
  *s = CountD(::sin(a.v));
  *c = CountD(::cos(a.v));
}

#define double CountD
#include "engine_fold.cuh"
#undef double

using namespace mhs;

namespace {

CountD g_glx[GL_TABLE], g_glw[GL_TABLE];   // set by oc_set_gauss

void ensure_gl() {}

void take(long long* out) {
  out[0] = opc::g.flop;
  out[1] = opc::g.div;
  out[2] = opc::g.sqrt;
  out[3] = opc::g.special;
  opc::g = opc::Ops{0, 0, 0, 0};
}

void frame_of(const double* tri, Frame& f) {
  CountD t[9];
  for (int i = 0; i < 9; ++i) t[i] = tri[i];
  make_frame(t, f);
}

template <int P>
struct Rules {
  static constexpr int K = n_nodes(P);
  CountD e0[208], e1[208], wq[208], Nq[208 * 6];
  QuadRule r12, r8;
  void build(const Frame& f) {
    build_rule<P>(f, g_glx, g_glw, cst::FAR_GAUSS_N, e0, e1, wq, Nq);
    build_rule<P>(f, g_glx, g_glw, cst::FAR_GAUSS_N_DISTANT, e0 + 144, e1 + 144, wq + 144,
                  Nq + 144 * K);
    r12 = QuadRule{144, e0, e1, wq, Nq};
    r8 = QuadRule{64, e0 + 144, e1 + 144, wq + 144, Nq + 144 * K};
  }
};

template <int P>
void consts(const Frame& f, double eps, double mu, double lam, SurfaceLoadConsts& c) {
  const Material m = make_material(CountD(mu), CountD(lam));
  surface_load_consts(f, CountD(eps), m, c);
}

// One edge integral of the surface-load spec in form `form`.
template <int P>
void edge_unit(int form, double ua, double ub, double rho2) {
  using S = SurfaceSpec<P>;
  CountD Pt[MS][8];
  if (form == EDGE_CLOSED) edge_closed<S, true>(ua, ub, rho2, Pt);   // the fold's form
  else if (form == EDGE_SMALL) edge_small<S>(ua, ub, sqrt(CountD(rho2)), Pt);
  else edge_large<S>(ua, ub, rho2, Pt);
}

// A near node without its three edge integrals: foot, edge geometry and form
// tests, boundary accumulation, seeds and recursion, weights and sigma_zz.
template <int P>
void near_rest(const Frame& f, const SurfaceLoadConsts& c, double px, double py, double eps) {
  using S = SurfaceSpec<P>;
  constexpr Spec sp = S::spec;
  constexpr int NB = sp.b_off[MS] > 0 ? sp.b_off[MS] : 1;
  constexpr int K = n_nodes(P);
  const CountD x[3] = {px, py, 0.0};
  CountD z, X0, X1;
  to_plane(f, x, z, X0, X1);
  const CountD h2 = z * z + CountD(eps) * CountD(eps);
  CountD pr[3][2];
  foot_vertices(f, X0, X1, pr);
  CountD BN1[NB], BN2[NB], BD[MS];
  for (int i = 0; i < NB; ++i) BN1[i] = BN2[i] = 0.0;
  for (int j = 0; j < MS; ++j) BD[j] = 0.0;
  for (int e = 0; e < 3; ++e) {
    const EdgeGeom g = edge_geom_rcp(pr, e, h2);   // the fold's form
    (void)edge_regime_sq(g.ua, g.ub, g.rho2);
    CountD Pt[MS][8] = {};
    for (int j = 0; j < MS; ++j)
      for (int k = 0; k < 8; ++k) Pt[j][k] = 0.5;
    edge_accumulate<S>(g, Pt, BN1, BN2, BD);
  }
  MomentTable<S> T;
  closed_finish_t<S, true>(pr, h2, BN1, BN2, BD, T);
  CountD s[3 * K];
  surface_load_near<P>(f, T, c, z, X0, X1, s);
}

template <int P>
void far_unit(const Frame& f, const Rules<P>& r, const SurfaceLoadConsts& c, int n, double px,
              double py, double eps) {
  constexpr int K = n_nodes(P);
  const CountD x[3] = {px, py, 0.0};
  CountD z, X0, X1;
  to_plane(f, x, z, X0, X1);
  (void)surface_class(f, px, py, eps);
  CountD s[3 * K];
  surface_load_far<P>(n == 8 ? r.r8 : r.r12, c, z, X0, X1, z * z + CountD(eps) * CountD(eps), s);
}

}  // namespace

extern "C" {

// The packed Gauss-Legendre table (orders 1..GL_MAX, as the device uses).
int oc_set_gauss(const double* x, const double* w, int n) {
  if (n != GL_TABLE) return -1;
  for (int i = 0; i < n; ++i) {
    g_glx[i] = x[i];
    g_glw[i] = w[i];
  }
  return 0;
}

// ops[4] per call: flops, divisions, square roots, other special functions.
int oc_edge(int P, int form, double ua, double ub, double rho2, long long* ops) {
  take(ops);
  if (P == 0) edge_unit<0>(form, ua, ub, rho2);
  else if (P == 1) edge_unit<1>(form, ua, ub, rho2);
  else edge_unit<2>(form, ua, ub, rho2);
  take(ops);
  return 0;
}

int oc_near_rest(int P, const double* tri, double eps, double mu, double lam, double px, double py,
                 long long* ops) {
  ensure_gl();
  Frame f;
  frame_of(tri, f);
  SurfaceLoadConsts c;
  take(ops);
  if (P == 0) { consts<0>(f, eps, mu, lam, c); take(ops); near_rest<0>(f, c, px, py, eps); }
  else if (P == 1) { consts<1>(f, eps, mu, lam, c); take(ops); near_rest<1>(f, c, px, py, eps); }
  else { consts<2>(f, eps, mu, lam, c); take(ops); near_rest<2>(f, c, px, py, eps); }
  take(ops);
  return 0;
}

int oc_far(int P, int n, const double* tri, double eps, double mu, double lam, double px, double py,
           long long* ops) {
  ensure_gl();
  Frame f;
  frame_of(tri, f);
  SurfaceLoadConsts c;
#define OC_FAR(PP)                       \
  {                                      \
    static Rules<PP> r;                  \
    r.build(f);                          \
    consts<PP>(f, eps, mu, lam, c);      \
    take(ops);                           \
    far_unit<PP>(f, r, c, n, px, py, eps); \
  }
  if (P == 0) OC_FAR(0) else if (P == 1) OC_FAR(1) else OC_FAR(2)
#undef OC_FAR
  take(ops);
  return 0;
}

// Per grid node besides its surface load: angular node, position, class
// test, point-load tensor (6 stress or 3 displacement components) and its
// weighting; the ordered sum adds nc x 3K products per node (2 flops each).
int oc_node(int P, int want_h, double zeta, long long* ops) {
  ensure_gl();
  const int K = (P + 1) * (P + 2) / 2;
  AngRule A;
  FoldPair fp;
  const CountD x[3] = {0.3, -0.2, -zeta};
  const CountD centre[2] = {1.0, 0.5};
  fold_pair_setup(x, centre, 0.8, 0.1, fp);
  fold_angular(0.4, 0.3, 0.9, 2.0, 0.1, A);
  Frame f;
  const double tri[9] = {0.0, 0.0, 0.0, 1.5, 0.2, -0.05, 0.3, 0.9, -1.1};
  frame_of(tri, f);
  const Material m = make_material(CountD(30.0), CountD(22.0));
  const CountD* gx6 = g_glx + gl_offset(cst::FOLD_N_RADIAL);
  const CountD* gw6 = g_glw + gl_offset(cst::FOLD_N_RADIAL);
  const CountD* gx4 = g_glx + gl_offset(cst::FOLD_N_ANGULAR);
  const CountD* gw4 = g_glw + gl_offset(cst::FOLD_N_ANGULAR);
  take(ops);
  const CountD ra = 0.5, rb = 0.75;
  const int j = A.n / 2, ir = 2;
  const CountD R = ra + (rb - ra) * (0.5 * (gx6[ir] + 1.0));
  const CountD wr = (rb - ra) * (0.5 * gw6[ir]);
  CountD th, wt;
  fold_ang_node(A, gx4, gw4, j, &th, &wt);
  CountD sn, cs;
  sincos(th, &sn, &cs);
  const CountD px = fp.xh0 + R * cs, py = fp.xh1 + R * sn;
  const CountD w = wr * wt * R;
  (void)surface_class(f, px, py, 0.1);
  CountD B[6];
  const int nc = want_h ? 6 : 3;
  if (want_h) point_stress6(fp.xh0 - px, fp.xh1 - py, fp.zeta, m.nu_f, B);
  else point_disp3(fp.xh0 - px, fp.xh1 - py, fp.zeta, m.mu, m.nu_f, B);
  for (int c = 0; c < nc; ++c) B[c] = w * B[c];
  opc::g.flop += 3 * K;              // load minus the load at the foot
  opc::g.flop += 2LL * nc * 3 * K;   // ordered sum of the products
  take(ops);
  return 0;
}

// Per band pair besides its grid: setup, breaks, the foot load (taken as a
// near node), the mirror element's full-space H + E (near form) and the
// Boussinesq assembly.  Per panel: its angular rule.
int oc_pair(int P, int want_h, const double* tri, double eps, double mu, double lam,
            const double* x, long long* pair_ops, long long* panel_ops) {
  ensure_gl();
  const int K = (P + 1) * (P + 2) / 2;
  Frame f, fi;
  frame_of(tri, f);
  double ti[9];
  for (int i = 0; i < 9; ++i) ti[i] = (i % 3 == 2) ? -tri[i] : tri[i];
  frame_of(ti, fi);
  const Material m = make_material(CountD(mu), CountD(lam));
  CountD tt[9], xx[3] = {x[0], x[1], x[2]};
  for (int i = 0; i < 9; ++i) tt[i] = tri[i];
  take(pair_ops);
  CountD centre[2], r_f;
  fold_crease(tt, eps, centre, &r_f);
  const CountD diam = tri_diameter(tt);
  FoldPair fp;
  fold_pair_setup(xx, centre, r_f, eps, fp);
  CountD br[FOLD_MAX_BREAKS], R1;
  const int nb = fold_breaks(fp.rho_s, fp.zeta, r_f, eps, diam, br, &R1);
  long long scratch[4];
#define OC_MIRROR(PP)                                                                       \
  {                                                                                         \
    static Rules<PP> r;                                                                     \
    r.build(fi);                                                                            \
    take(scratch);                                                                          \
    CountD Hm[27 * 6], Um[9 * 6], E[6];                                                     \
    if (want_h) direct_eval<PP, W_H | W_E>(fi, r.r12, r.r8, xx, eps, m, nullptr, Hm, E);   \
    else direct_eval<PP, W_U>(fi, r.r12, r.r8, xx, eps, m, Um, nullptr, nullptr);          \
  }
  {
    long long keep[4];
    take(keep);
    for (int i = 0; i < 4; ++i) pair_ops[i] += keep[i];
  }
  if (P == 0) OC_MIRROR(0) else if (P == 1) OC_MIRROR(1) else OC_MIRROR(2)
#undef OC_MIRROR
  CountD srr, szz;
  disk_stress(R1, fp.zeta, m.nu_f, &srr, &szz);
  opc::g.flop += (want_h ? 12LL : 6LL) * 3 * K;   // assembly of the correction
  {
    long long keep[4];
    take(keep);
    for (int i = 0; i < 4; ++i) pair_ops[i] += keep[i];
  }
  // one panel's angular rule
  AngRule A;
  if (nb > 1) fold_panel_rule(fp, br[0], br[1], A);
  take(panel_ops);
  return nb;
}

}  // extern "C"

namespace {
// The per-material coefficient block in ImageCoef's layout (values only:
// built before the counted evaluation).
constexpr int OC_COEF_SIZE = 3 * (MHS_R_NDG + MHS_R_NDDG) + MHS_Q_NDG + MHS_Q_NDDG;
void oc_image_coef(const Material& m, CountD* out) {
  const CountD nup[3] = {1.0, m.nu_i, m.nu_i * m.nu_i};
  CountD* p = out;
  for (int r = 0; r < MHS_R_NDG; ++r)
    for (int pz = 0; pz < 3; ++pz) {
      CountD v = 0.0;
      for (int k = 0; k < 3; ++k) v += tab_h::mhs_r_dg_c[r][pz][k] * nup[k];
      *p++ = v * m.scale_c;
    }
  for (int r = 0; r < MHS_R_NDDG; ++r)
    for (int pz = 0; pz < 3; ++pz) {
      CountD v = 0.0;
      for (int k = 0; k < 3; ++k) v += tab_h::mhs_r_ddg_c[r][pz][k] * nup[k];
      *p++ = v * m.scale_c;
    }
  for (int r = 0; r < MHS_Q_NDG; ++r) {
    CountD v = 0.0;
    for (int k = 0; k < 3; ++k) v += tab_h::mhs_q_dg_c[r][k] * nup[k];
    *p++ = v;
  }
  for (int r = 0; r < MHS_Q_NDDG; ++r) {
    CountD v = 0.0;
    for (int k = 0; k < 3; ++k) v += tab_h::mhs_q_ddg_c[r][k] * nup[k];
    *p++ = v;
  }
}
}  // namespace

extern "C" {

// One ordinary (observer, source) pair as the pair kernels evaluate it:
// the direct term (closed form within D_STAR L, else the 12 x 12 rule, 8 x 8
// beyond D_STAR_DISTANT L), the image R-family on the reflected element and
// the image Q-family at the pair's Gauss order (nodes precomputed, as the
// device holds the floor order's per source).  *band = 1 when the receiver
// lies in the fold band of a straddling source: the image terms are then
// replaced by the fold and are not evaluated (their counts are zero).
int oc_pair_terms(int P, int want_h, const double* tri, double eps, double mu, double lam,
                  const double* x, long long* direct_ops, long long* image_r_ops,
                  long long* image_q_ops, int* q_order, int* band) {
  ensure_gl();
  CountD tt[9], ti[9], xx[3] = {x[0], x[1], x[2]};
  for (int i = 0; i < 9; ++i) {
    tt[i] = tri[i];
    ti[i] = (i % 3 == 2) ? -tri[i] : tri[i];
  }
  Frame f, fi;
  make_frame(tt, f);
  make_frame(ti, fi);
  const Material m = make_material(CountD(mu), CountD(lam));
  CountD centre[2], r_f;
  fold_crease(tt, CountD(eps), centre, &r_f);
  const bool in_band = fold_straddles(tt, CountD(eps)) && fold_band(xx, centre, CountD(eps));
  *band = in_band ? 1 : 0;
  long long scratch[4];
#define OC_TERMS(PP)                                                                         \
  {                                                                                          \
    constexpr int K = n_nodes(PP);                                                           \
    static Rules<PP> rd, ri;                                                                 \
    rd.build(f);                                                                             \
    ri.build(fi);                                                                            \
    static CountD G[G_SIZE], coef[OC_COEF_SIZE];                                          \
    build_basis_products(fi, G);                                                             \
    oc_image_coef(m, coef);                                                                  \
    const ImageCoef ic = image_coef_view(coef);                                              \
    take(scratch);                                                                           \
    CountD A[27 * 6], E[6];                                                                  \
    if (want_h) direct_eval<PP, W_H | W_E>(f, rd.r12, rd.r8, xx, CountD(eps), m, nullptr, A, E); \
    else direct_eval<PP, W_U>(f, rd.r12, rd.r8, xx, CountD(eps), m, A, nullptr, nullptr);    \
    take(direct_ops);                                                                        \
    for (int i = 0; i < 4; ++i) image_r_ops[i] = image_q_ops[i] = 0;                         \
    *q_order = 0;                                                                            \
    if (!in_band) {                                                                          \
      CountD B[27 * 6];                                                                      \
      if (want_h) image_r_eval<PP, W_H>(fi, G, f.n, ri.r12, ri.r8, xx, CountD(eps), m, ic,   \
                                        nullptr, B);                                         \
      else image_r_eval<PP, W_U>(fi, G, f.n, ri.r12, ri.r8, xx, CountD(eps), m, ic, B,       \
                                 nullptr);                                                   \
      take(image_r_ops);                                                                     \
      CountD tv[9];                                                                          \
      for (int a = 0; a < 3; ++a)                                                            \
        for (int b = 0; b < 3; ++b) tv[3 * a + b] = fi.v[a][b];                              \
      const int n = q_gauss_order(xx, tv, CountD(eps), f.L, PP);                             \
      *q_order = n;                                                                          \
      static CountD qy[3 * GL_MAX * GL_MAX], qw[6 * GL_MAX * GL_MAX];                        \
      build_qrule<PP>(f, g_glx, g_glw, n, qy, qw);                                           \
      const QRule<PP> q{n * n, qy, qw};                                                      \
      take(scratch);                                                                         \
      if (want_h) image_q_eval<PP, W_H>(q, f.n, xx, CountD(eps), m, ic, nullptr, B);         \
      else image_q_eval<PP, W_U>(q, f.n, xx, CountD(eps), m, ic, B, nullptr);                \
      take(image_q_ops);                                                                     \
      (void)K;                                                                               \
    }                                                                                        \
  }
  if (P == 0) OC_TERMS(0) else if (P == 1) OC_TERMS(1) else OC_TERMS(2)
#undef OC_TERMS
  return 0;
}

// The image Q-family of one pair at a given Gauss order n (its work is a
// fixed part plus a part per rule point, n^2 of them).
int oc_image_q_n(int P, int want_h, const double* tri, double eps, double mu, double lam,
                 const double* x, int n, long long* ops) {
  ensure_gl();
  if (n < 1 || n > GL_MAX) return -1;
  CountD tt[9], xx[3] = {x[0], x[1], x[2]};
  for (int i = 0; i < 9; ++i) tt[i] = tri[i];
  Frame f;
  make_frame(tt, f);
  const Material m = make_material(CountD(mu), CountD(lam));
  long long scratch[4];
#define OC_Q(PP)                                                                  \
  {                                                                               \
    static CountD coef[OC_COEF_SIZE];                                             \
    oc_image_coef(m, coef);                                                       \
    const ImageCoef ic = image_coef_view(coef);                                   \
    static CountD qy[3 * GL_MAX * GL_MAX], qw[6 * GL_MAX * GL_MAX];               \
    build_qrule<PP>(f, g_glx, g_glw, n, qy, qw);                                  \
    const QRule<PP> q{n * n, qy, qw};                                             \
    CountD B[27 * 6];                                                             \
    take(scratch);                                                                \
    if (want_h) image_q_eval<PP, W_H>(q, f.n, xx, CountD(eps), m, ic, nullptr, B); \
    else image_q_eval<PP, W_U>(q, f.n, xx, CountD(eps), m, ic, B, nullptr);      \
    take(ops);                                                                    \
  }
  if (P == 0) OC_Q(0) else if (P == 1) OC_Q(1) else OC_Q(2)
#undef OC_Q
  return 0;
}

}  // extern "C"
