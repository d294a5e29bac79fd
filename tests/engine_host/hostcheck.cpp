// CPU build of the device engine's per-pair arithmetic, for tests only.
//
// The kernels in mhs_b200/csrc are __host__ __device__; compiling them here
// with g++ lets the CPU test suite check the engine's mathematics term by
// term (direct, image R, image Q) against golden vectors without a GPU.
// Nothing in the package loads this library.
#include <vector>

#include "../../mhs_b200/csrc/engine_fold.cuh"
#include "../../mhs_b200/csrc/host_prep.h"

using namespace mhs;

namespace {

std::vector<double> g_glx, g_glw;

void ensure_gl() {
  if (g_glx.empty()) {
    g_glx.resize(GL_TABLE);
    g_glw.resize(GL_TABLE);
    gauss_table(g_glx.data(), g_glw.data());
  }
}

template <int P>
struct Rule {
  std::vector<double> e0, e1, wq, Nq;
  QuadRule q;
  void build(const Frame& f, int n) {
    const int nq = n * n, K = n_nodes(P);
    e0.resize(nq); e1.resize(nq); wq.resize(nq); Nq.resize(nq * K);
    build_rule<P>(f, g_glx.data(), g_glw.data(), n, e0.data(), e1.data(), wq.data(), Nq.data());
    q = QuadRule{nq, e0.data(), e1.data(), wq.data(), Nq.data()};
  }
};

template <int P, int WANT>
void direct_all(const double* obs, int nobs, const double* tri, double mu, double lam, double eps,
                double* U, double* H, double* E) {
  ensure_gl();
  constexpr int K = n_nodes(P);
  Frame f;
  make_frame(tri, f);
  Rule<P> r12, r8;
  r12.build(f, cst::FAR_GAUSS_N);
  r8.build(f, cst::FAR_GAUSS_N_DISTANT);
  const Material m = make_material(mu, lam);
  for (int o = 0; o < nobs; ++o)
    direct_eval<P, WANT>(f, r12.q, r8.q, obs + 3 * o, eps, m, U ? U + o * K * 9 : nullptr,
                         H ? H + o * K * 27 : nullptr, E ? E + o * K : nullptr);
}

template <int P, int WANT>
void force_all(const double* obs, int nobs, const double* tri, double mu, double lam, double eps,
               double near_l, double* G, double* S) {
  ensure_gl();
  constexpr int K = n_nodes(P);
  Frame f;
  make_frame(tri, f);
  Rule<P> r12, r8;
  r12.build(f, cst::FAR_GAUSS_N);
  r8.build(f, cst::FAR_GAUSS_N_DISTANT);
  const Material m = make_material(mu, lam);
  for (int o = 0; o < nobs; ++o)
    force_eval<P, WANT>(f, r12.q, r8.q, obs + 3 * o, eps, m, G ? G + o * K * 9 : nullptr,
                        S ? S + o * K * 27 : nullptr, near_l);
}

template <int P, int WANT>
void image_r_all(const double* obs, int nobs, const double* tri, double mu, double lam, double eps,
                 double* U, double* H) {
  ensure_gl();
  constexpr int K = n_nodes(P);
  double ti[9];
  for (int i = 0; i < 9; ++i) ti[i] = (i % 3 == 2) ? -tri[i] : tri[i];
  Frame f, fi;
  make_frame(tri, f);
  make_frame(ti, fi);
  Rule<P> r12, r8;
  r12.build(fi, cst::FAR_GAUSS_N);
  r8.build(fi, cst::FAR_GAUSS_N_DISTANT);
  std::vector<double> G(G_SIZE);
  build_basis_products(fi, G.data());
  const Material m = make_material(mu, lam);
  std::vector<double> coef(IMAGE_COEF_SIZE);
  image_coef(m, coef.data());
  const ImageCoef ic = image_coef_view(coef.data());
  for (int o = 0; o < nobs; ++o)
    image_r_eval<P, WANT>(fi, G.data(), f.n, r12.q, r8.q, obs + 3 * o, eps, m, ic,
                          U ? U + o * K * 9 : nullptr, H ? H + o * K * 27 : nullptr);
}

template <int P, int WANT>
void image_q_all(const double* obs, int nobs, const double* tri, double mu, double lam, double eps,
                 int nq_force, double* U, double* H, int* orders) {
  ensure_gl();
  constexpr int K = n_nodes(P);
  double ti[9];
  for (int i = 0; i < 9; ++i) ti[i] = (i % 3 == 2) ? -tri[i] : tri[i];
  Frame f;
  make_frame(tri, f);
  const Material m = make_material(mu, lam);
  std::vector<double> coef(IMAGE_COEF_SIZE);
  image_coef(m, coef.data());
  const ImageCoef ic = image_coef_view(coef.data());
  std::vector<double> y, wN;
  for (int o = 0; o < nobs; ++o) {
    const int n = nq_force > 0 ? nq_force : q_gauss_order(obs + 3 * o, ti, eps, f.L, P);
    if (orders) orders[o] = n;
    y.resize(3 * n * n);
    wN.resize(K * n * n);
    build_qrule<P>(f, g_glx.data(), g_glw.data(), n, y.data(), wN.data());
    const QRule<P> q{n * n, y.data(), wN.data()};
    image_q_eval<P, WANT>(q, f.n, obs + 3 * o, eps, m, ic, U ? U + o * K * 9 : nullptr,
                          H ? H + o * K * 27 : nullptr);
  }
}

// Folded image at band receivers: mirror element (slip columns signed) plus
// the Boussinesq correction.
template <int P, int WANT>
void fold_all(const double* obs, int nobs, const double* tri, double mu, double lam, double eps,
              double* U, double* H) {
  ensure_gl();
  constexpr int K = n_nodes(P);
  double tm[9];
  for (int i = 0; i < 9; ++i) tm[i] = (i % 3 == 2) ? -tri[i] : tri[i];
  Frame f, fm;
  make_frame(tri, f);
  make_frame(tm, fm);
  Rule<P> r12, r8, m12, m8;
  r12.build(f, cst::FAR_GAUSS_N);
  r8.build(f, cst::FAR_GAUSS_N_DISTANT);
  m12.build(fm, cst::FAR_GAUSS_N);
  m8.build(fm, cst::FAR_GAUSS_N_DISTANT);
  const Material m = make_material(mu, lam);
  for (int o = 0; o < nobs; ++o) {
    const double* x = obs + 3 * o;
    if (WANT & W_U) {
      double Um[9 * K], Ub[9 * K];
      direct_eval<P, W_U>(fm, m12.q, m8.q, x, eps, m, Um, nullptr, nullptr);
      fold_boussinesq_scalar<P, false>(f, r12.q, r8.q, tri, x, eps, m, g_glx.data(), g_glw.data(), Ub);
      for (int i = 0; i < 9 * K; ++i) U[o * 9 * K + i] = Um[i] * mirror_slip_sign(i % 3) + Ub[i];
    } else {
      double Hm[27 * K], Hb[27 * K];
      direct_eval<P, W_H>(fm, m12.q, m8.q, x, eps, m, nullptr, Hm, nullptr);
      fold_boussinesq_scalar<P, true>(f, r12.q, r8.q, tri, x, eps, m, g_glx.data(), g_glw.data(), Hb);
      for (int i = 0; i < 27 * K; ++i) H[o * 27 * K + i] = Hm[i] * mirror_slip_sign(i % 3) + Hb[i];
    }
  }
}

// Surface load sigma_zz at surface points (x, y, 0) for every node and slip
// component: fast = 1 reads the contracted sigma_zz row, 0 the full H.
template <int P, int FAST>
void surface_load_all(const double* pts, int npts, const double* tri, double mu, double lam,
                      double eps, double* s) {
  ensure_gl();
  constexpr int K = n_nodes(P);
  Frame f;
  make_frame(tri, f);
  Rule<P> r12, r8;
  r12.build(f, cst::FAR_GAUSS_N);
  r8.build(f, cst::FAR_GAUSS_N_DISTANT);
  const Material m = make_material(mu, lam);
  SurfaceLoadConsts c;
  surface_load_consts(f, eps, m, c);
  for (int i = 0; i < npts; ++i) {
    if (FAST) fold_surface_load_fast<P>(f, r12.q, r8.q, c, pts[2 * i], pts[2 * i + 1], eps, s + 3 * K * i);
    else fold_surface_load<P>(f, r12.q, r8.q, pts[2 * i], pts[2 * i + 1], eps, m, s + 3 * K * i);
  }
}

}  // namespace

#define DISPATCH_P(FN, WANT, ...)                 \
  switch (P) {                                    \
    case 0: FN<0, WANT>(__VA_ARGS__); return 0;   \
    case 1: FN<1, WANT>(__VA_ARGS__); return 0;   \
    case 2: FN<2, WANT>(__VA_ARGS__); return 0;   \
  }                                               \
  return -1;

extern "C" {

int hc_gauss(int n, double* x, double* w) {
  if (n < 1 || n > GL_MAX) return -1;
  gauss_legendre(n, x, w);
  return 0;
}

// want: 1 = U, 2 = H, 6 = H + E, 4 = E
int hc_direct(int P, int want, const double* obs, int nobs, const double* tri, double mu,
              double lam, double eps, double* U, double* H, double* E) {
  if (want == W_U) { DISPATCH_P(direct_all, W_U, obs, nobs, tri, mu, lam, eps, U, H, E) }
  if (want == W_H) { DISPATCH_P(direct_all, W_H, obs, nobs, tri, mu, lam, eps, U, H, E) }
  if (want == (W_H | W_E)) { DISPATCH_P(direct_all, W_H | W_E, obs, nobs, tri, mu, lam, eps, U, H, E) }
  if (want == W_E) { DISPATCH_P(direct_all, W_E, obs, nobs, tri, mu, lam, eps, U, H, E) }
  return -2;
}

// want: 8 = G, 16 = S, 24 = both; near_l: the closed form within near_l L
int hc_force(int P, int want, const double* obs, int nobs, const double* tri, double mu,
             double lam, double eps, double near_l, double* G, double* S) {
  if (want == W_G) { DISPATCH_P(force_all, W_G, obs, nobs, tri, mu, lam, eps, near_l, G, S) }
  if (want == W_S) { DISPATCH_P(force_all, W_S, obs, nobs, tri, mu, lam, eps, near_l, G, S) }
  if (want == (W_G | W_S)) { DISPATCH_P(force_all, W_G | W_S, obs, nobs, tri, mu, lam, eps, near_l, G, S) }
  return -2;
}

int hc_image_r(int P, int want, const double* obs, int nobs, const double* tri, double mu,
               double lam, double eps, double* U, double* H) {
  if (want == W_U) { DISPATCH_P(image_r_all, W_U, obs, nobs, tri, mu, lam, eps, U, H) }
  if (want == W_H) { DISPATCH_P(image_r_all, W_H, obs, nobs, tri, mu, lam, eps, U, H) }
  return -2;
}

int hc_image_q(int P, int want, const double* obs, int nobs, const double* tri, double mu,
               double lam, double eps, int nq_force, double* U, double* H, int* orders) {
  if (want == W_U) { DISPATCH_P(image_q_all, W_U, obs, nobs, tri, mu, lam, eps, nq_force, U, H, orders) }
  if (want == W_H) { DISPATCH_P(image_q_all, W_H, obs, nobs, tri, mu, lam, eps, nq_force, U, H, orders) }
  return -2;
}

int hc_fold_image(int P, int want, const double* obs, int nobs, const double* tri, double mu,
                  double lam, double eps, double* U, double* H) {
  if (want == W_U) { DISPATCH_P(fold_all, W_U, obs, nobs, tri, mu, lam, eps, U, H) }
  if (want == W_H) { DISPATCH_P(fold_all, W_H, obs, nobs, tri, mu, lam, eps, U, H) }
  return -2;
}

int hc_surface_load(int P, int fast, const double* pts, int npts, const double* tri, double mu,
                    double lam, double eps, double* s) {
  if (fast) { DISPATCH_P(surface_load_all, 1, pts, npts, tri, mu, lam, eps, s) }
  DISPATCH_P(surface_load_all, 0, pts, npts, tri, mu, lam, eps, s)
}

// One closed-form edge of the surface-load spec: the plain form or the
// fold's reciprocal form (fast = 1); P[j][k] for j < 5, k < 8 into out.
int hc_edge_closed(int P, int fast, double ua, double ub, double rho2, double* out) {
  double Pt[MS][8] = {};
#define HC_EC(PP)                                                                   \
  {                                                                                 \
    if (fast) edge_closed<SurfaceSpec<PP>, true>(ua, ub, rho2, Pt);                 \
    else edge_closed<SurfaceSpec<PP>, false>(ua, ub, rho2, Pt);                     \
  }
  if (P == 0) HC_EC(0) else if (P == 1) HC_EC(1) else HC_EC(2)
#undef HC_EC
  for (int j = 0; j < MS; ++j)
    for (int k = 0; k < 8; ++k) out[8 * j + k] = Pt[j][k];
  return 0;
}

// Seeds and recursion of one near node (surface-load spec, P0) from given
// boundary sums: the plain form or the fold's reciprocal form (fast = 1).
int hc_closed_finish(int fast, const double* pr6, double h2, const double* bn, double* out) {
  using S = SurfaceSpec<0>;
  constexpr Spec sp = S::spec;
  constexpr int NB = sp.b_off[MS];
  double pr[3][2] = {{pr6[0], pr6[1]}, {pr6[2], pr6[3]}, {pr6[4], pr6[5]}};
  double BN1[NB], BN2[NB], BD[MS];
  for (int i = 0; i < NB; ++i) { BN1[i] = bn[i]; BN2[i] = bn[NB + i]; }
  for (int j = 0; j < MS; ++j) BD[j] = bn[2 * NB + j];
  MomentTable<S> T;
  if (fast) closed_finish_t<S, true>(pr, h2, BN1, BN2, BD, T);
  else closed_finish_t<S, false>(pr, h2, BN1, BN2, BD, T);
  for (int i = 0; i < sp.m_off[NS]; ++i) out[i] = T.M[i];
  return sp.m_off[NS];
}

}  // extern "C"
