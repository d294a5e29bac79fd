// Scalar building blocks shared by every kernel of the engine: constants,
// compile-time degree specs, triangle frames, shape functions and the
// Gauss-Legendre rules.  Everything here is __host__ __device__ so the same
// arithmetic can be exercised on the CPU by the test build.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define MHS_HD __host__ __device__ inline
#define MHS_FI __host__ __device__ __forceinline__
#else
#define MHS_HD inline
#define MHS_FI inline
#endif

// Generated coefficient tables, once for host code and, under nvcc, once in
// __constant__ memory for device code; MHS_TAB(name) picks the right copy.
namespace mhs {
namespace tab_h {
#define MHS_TBL static const
#define MHS_TBLC static const
#include "tables.inc"
#undef MHS_TBL
#undef MHS_TBLC
}  // namespace tab_h
#if defined(__CUDACC__)
namespace tab_d {
#define MHS_TBL static __constant__ const
#define MHS_TBLC static __device__ const
#include "tables.inc"
#undef MHS_TBL
#undef MHS_TBLC
}  // namespace tab_d
#endif
}  // namespace mhs
#if defined(__CUDA_ARCH__)
#define MHS_TAB(x) ::mhs::tab_d::x
#else
#define MHS_TAB(x) ::mhs::tab_h::x
#endif

namespace mhs {

// ----------------------------------------------------------------- constants
// Algorithm thresholds; each value changes results and equals mhs's
// (mhs/defaults.py:60-143, mhs/fullspace/defaults.py:20-35).
namespace cst {
constexpr double D_STAR = 10.0;              // near/far switch, units of L
constexpr int FAR_GAUSS_N = 12;              // far rule, points per direction
constexpr int FAR_GAUSS_N_DISTANT = 8;       // beyond D_STAR_DISTANT * L
constexpr double D_STAR_DISTANT = 40.0;
constexpr double SERIES_U_OVER_RHO = 2.0;    // large-|u| edge series regime
constexpr int SERIES_TERMS = 32;
constexpr double SMALL_U_OVER_RHO = 0.5;     // small-|u| edge series regime
// Squares of the two edge-regime thresholds (exact in binary), for the tests
// on squared lengths; tied to the thresholds by a static_assert in the
// device build (pipeline.cuh).
constexpr double SERIES_U_OVER_RHO_SQ = 4.0;
constexpr double SMALL_U_OVER_RHO_SQ = 0.25;
constexpr double DEGENERATE_AREA_REL = 1e-14;
constexpr double IMAGE_Q_BUDGET_C = 10.0;    // Q-family Gauss order law
constexpr int IMAGE_Q_GAUSS_MIN = 8;
constexpr int IMAGE_Q_GAUSS_MAX = 192;
constexpr double FOLD_SOURCE_DEPTH_EPS = 3.0;
constexpr double FOLD_BAND_DEPTH_EPS = 10.0;
constexpr double FOLD_REACH_EPS = 60.0;
constexpr int FOLD_N_RADIAL = 6;
constexpr int FOLD_N_ANGULAR = 4;
constexpr double FOLD_CREASE_MARGIN_EPS = 5.0;
constexpr double FOLD_FINE_SPACING_EPS = 0.25;
constexpr double FOLD_MEDIUM_SPACING_EPS = 2.0;
constexpr int FOLD_N_COARSE = 24;
constexpr double FOLD_FINE_SUBPANEL_EPS = 6.0;
constexpr double FOLD_MEDIUM_SUBPANEL_EPS = 16.0;
constexpr double FOLD_R1_MARGIN_DIAM = 8.0;
constexpr double PI = 3.141592653589793;
}  // namespace cst

// Largest Gauss-Legendre order any rule asks for (the Q-family ceiling).
// The array behind p stays in (local) memory: once its address has passed
// through an opaque move the compiler can no longer promote the array to
// registers.  For per-thread arrays too large to live in registers.
// An int the compiler cannot see through (an opaque move): a loop whose
// counter passes through it is not unrolled or threaded into its cases.
MHS_FI int opaque(int v) {
#if defined(__CUDA_ARCH__)
  asm volatile("mov.b32 %0, %0;" : "+r"(v));
#endif
  return v;
}

template <class T>
MHS_FI T* in_memory(T* p) {
#if defined(__CUDA_ARCH__)
  asm volatile("mov.b64 %0, %0;" : "+l"(p));
#endif
  return p;
}

// A table whose entries lie `st` words apart in device memory (the
// observer index innermost, so one warp's threads touch consecutive words
// for every entry).  Indexing and offsets count entries, as on a pointer.
struct StridedTable {
  double* p;
  int64_t st;
  MHS_FI double& operator[](int i) const { return p[(int64_t)i * st]; }
  MHS_FI StridedTable operator+(int i) const { return {p + (int64_t)i * st, st}; }
};

constexpr int GL_MAX = cst::IMAGE_Q_GAUSS_MAX;
// Offset of order n's nodes in the packed 1-D rule table (orders 1..GL_MAX).
MHS_FI constexpr int gl_offset(int n) { return (n - 1) * n / 2; }
constexpr int GL_TABLE = gl_offset(GL_MAX + 1);

// 1 / sqrt(x): the device's reciprocal square root (within an ulp), one
// division and square root on the host.
MHS_FI double rsqrt_r(double x) {
#if defined(__CUDA_ARCH__)
  return ::rsqrt(x);
#else
  return 1.0 / sqrt(x);
#endif
}
MHS_FI float rsqrt_r(float x) {
#if defined(__CUDA_ARCH__)
  return ::rsqrtf(x);
#else
  return 1.0f / sqrtf(x);
#endif
}

// ------------------------------------------------------ triangular packing
// Index of (a, b), a + b <= D, independent of D: ordered by total degree,
// then by b.  ntri(D) entries cover every degree <= D.
MHS_FI constexpr int tri_idx(int a, int b) { return (a + b) * (a + b + 1) / 2 + b; }
MHS_FI constexpr int ntri(int d) { return d < 0 ? 0 : (d + 1) * (d + 2) / 2; }
MHS_FI constexpr int imax(int a, int b) { return a > b ? a : b; }
MHS_FI constexpr int imin(int a, int b) { return a < b ? a : b; }
MHS_FI constexpr int n_nodes(int p) { return (p + 1) * (p + 2) / 2; }

// ------------------------------------------------------------ degree specs
// Moment orders n are odd, n in {-1, 1, 3, 5, 7, 9} -> slot (n + 1) / 2.
// Edge primitive orders m in {-1, 1, 3, 5, 7} -> slot (m + 1) / 2.
constexpr int NS = 6;
constexpr int MS = 5;
MHS_FI constexpr int nslot(int n) { return (n + 1) / 2; }
MHS_FI constexpr int slot_n(int s) { return 2 * s - 1; }

struct Spec {
  int order;
  int need0[NS];   // constant-slip table degree per n (-1 = absent)
  int need[NS];    // raised by the slip order (closed form)
  int deg[NS];     // after closing the recursion
  int edge[MS];    // edge primitive degree kmax per m (-1 = absent)
  bool Pneed[MS][8];  // closed-form closure of P_k^m
  bool Jneed[MS];
  bool Kneed[MS];
  int m_off[NS + 1];   // packed offsets of M_n tables (deg)
  int w_off[NS + 1];   // packed offsets of W_n tables (need0)
  int b_off[MS + 1];   // packed offsets of edge BN tables (edge)
  int kmax;            // max edge degree
  int dmax;            // max closed degree
};

// Required table degrees from the constant-slip ones: the recursion for M_n
// at degree D consumes M_{n-2} at degree D-2 down to the lowest odd n, and
// the vertical seeds need I_3 and every I_m between (mhs/fullspace/
// moments.py:94-116, restated).
MHS_FI constexpr Spec make_spec(int d1, int d3, int d5, int d7, int d9, int order) {
  Spec s{};
  s.order = order;
  const int in0[NS] = {-1, d1, d3, d5, d7, d9};
  for (int i = 0; i < NS; ++i) {
    s.need0[i] = in0[i];
    s.need[i] = in0[i] >= 0 ? in0[i] + order : -1;
    s.deg[i] = s.need[i];
  }
  // --- close the degrees
  int nmax = -99;
  for (int i = 0; i < NS; ++i)
    if (s.deg[i] >= 0) nmax = slot_n(i);
  int n = nmax;
  while (true) {
    const int d = s.deg[nslot(n)];
    if (d >= 2) s.deg[nslot(n - 2)] = imax(s.deg[nslot(n - 2)], d - 2);
    int nmin = 99;
    for (int i = 0; i < NS; ++i)
      if (s.deg[i] >= 0 && slot_n(i) < nmin) nmin = slot_n(i);
    if (n - 2 < nmin) break;
    n -= 2;
  }
  s.deg[nslot(3)] = imax(s.deg[nslot(3)], 0);
  bool present[NS] = {};
  for (int i = 0; i < NS; ++i) present[i] = s.deg[i] >= 0;
  for (int i = 0; i < NS; ++i) {
    if (!present[i]) continue;
    const int nn = slot_n(i);
    if (nn >= 5)
      for (int m = 3; m < nn; m += 2) s.deg[nslot(m)] = imax(s.deg[nslot(m)], 0);
    if (nn <= 1)
      for (int m = nn; m < 4; m += 2) s.deg[nslot(m)] = imax(s.deg[nslot(m)], 0);
  }
  // --- edge primitive degrees (mhs/fullspace/moments.py:224-233, restated)
  for (int j = 0; j < MS; ++j) s.edge[j] = -1;
  for (int i = 0; i < NS; ++i) {
    if (s.deg[i] < 0) continue;
    const int nn = slot_n(i), d = s.deg[i];
    if (d >= 1) s.edge[(nn - 1) / 2] = imax(s.edge[(nn - 1) / 2], d - 1);  // m = n - 2
  }
  for (int i = 0; i < NS; ++i) {
    if (s.deg[i] < 0) continue;
    const int nn = slot_n(i);
    if (nn >= 5) s.edge[(nn - 1) / 2] = imax(s.edge[(nn - 1) / 2], 0);
    if (nn <= 1) s.edge[i] = imax(s.edge[i], 0);                      // m = n
  }
  // --- closed-form closure: P_k^m = P_{k-2}^{m-2} - rho^2 P_{k-2}^m
  for (int j = 0; j < MS; ++j)
    for (int k = 0; k < 8; ++k) s.Pneed[j][k] = k <= s.edge[j];
  for (int k = 7; k >= 2; --k)
    for (int j = 0; j < MS; ++j)
      if (s.Pneed[j][k]) {
        if (j >= 1) s.Pneed[j - 1][k - 2] = true;
        s.Pneed[j][k - 2] = true;
      }
  for (int j = 0; j < MS; ++j) {
    s.Jneed[j] = s.Pneed[j][0];
    s.Kneed[j] = s.Pneed[j][1];
  }
  for (int j = MS - 1; j >= 3; --j)  // J_m, m >= 5, recurses on J_{m-2}
    if (s.Jneed[j]) s.Jneed[j - 1] = true;
  if (s.Jneed[0]) s.Jneed[1] = true;  // J_{-1} reads J_1
  // --- packed layouts
  s.m_off[0] = 0;
  s.w_off[0] = 0;
  for (int i = 0; i < NS; ++i) {
    s.m_off[i + 1] = s.m_off[i] + ntri(s.deg[i]);
    s.w_off[i + 1] = s.w_off[i] + ntri(s.need0[i]);
  }
  s.b_off[0] = 0;
  s.kmax = -1;
  for (int j = 0; j < MS; ++j) {
    s.b_off[j + 1] = s.b_off[j] + ntri(s.edge[j]);
    s.kmax = imax(s.kmax, s.edge[j]);
  }
  s.dmax = -1;
  for (int i = 0; i < NS; ++i) s.dmax = imax(s.dmax, s.deg[i]);
  return s;
}

// Constant-slip degrees per readout (mhs/fullspace/moments.py:63-91):
//   U -> {3: 1, 5: 3};  H (and H + E) -> {3: 0, 5: 2, 7: 4};  E -> {7: 0};
// the image R-family reads {3: 1, 5: 3, 7: 4, 9: 5} (its generated table);
// the force source G -> {1: 0, 3: 2}, S -> {3: 1, 5: 3}.
template <int P> struct SpecU { static constexpr Spec spec = make_spec(-1, 1, 3, -1, -1, P); };
template <int P> struct SpecH { static constexpr Spec spec = make_spec(-1, 0, 2, 4, -1, P); };
template <int P> struct SpecE { static constexpr Spec spec = make_spec(-1, -1, -1, 0, -1, P); };
template <int P> struct SpecImg { static constexpr Spec spec = make_spec(-1, 1, 3, 4, 5, P); };
// the force (Kelvin single-layer) source: G reads {1: 0, 3: 2}, S the U degrees
template <int P> struct SpecF { static constexpr Spec spec = make_spec(0, 2, 3, -1, -1, P); };

// ------------------------------------------------------------------ frames
struct Frame {
  double v[3][3];     // vertices (rows)
  double e1[3], e2[3], n[3], c[3];
  double p[3][2];     // in-plane vertex coordinates about the centroid
  double area, L;     // area, longest edge
  double abc[3][3];   // barycentric affine rows (A_k, B_k, C_k)
  int ok;             // 0 for a degenerate triangle
};

MHS_FI double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
MHS_FI void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
MHS_FI double norm3(const double* a) { return sqrt(dot3(a, a)); }

// Local frame of one flat triangle: e1 along v2 - v1, nhat from the vertex
// order, centroid origin, L the longest edge (mhs/fullspace/frame.py:282-302).
// Also the affine barycentric coefficients in that frame
// (mhs/fullspace/shape.py:107-111), here by the closed-form inverse.
MHS_HD void make_frame(const double* tri, Frame& f) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) f.v[i][j] = tri[3 * i + j];
  double e1v[3], e2v[3], e3v[3], nn[3];
  for (int j = 0; j < 3; ++j) {
    e1v[j] = f.v[1][j] - f.v[0][j];
    e2v[j] = f.v[2][j] - f.v[0][j];
    e3v[j] = f.v[0][j] - f.v[2][j];
  }
  cross3(e1v, e2v, nn);
  const double area2 = norm3(nn);
  double d12[3];
  for (int j = 0; j < 3; ++j) d12[j] = f.v[2][j] - f.v[1][j];
  const double l0 = norm3(e1v), l1 = norm3(d12), l2 = norm3(e3v);
  double L = l0;
  if (l1 > L) L = l1;
  if (l2 > L) L = l2;
  f.L = L;
  f.area = 0.5 * area2;
  f.ok = (L != 0.0 && !(0.5 * area2 < cst::DEGENERATE_AREA_REL * L * L)) ? 1 : 0;
  for (int j = 0; j < 3; ++j) {
    f.n[j] = nn[j] / area2;
    f.e1[j] = e1v[j] / l0;
  }
  cross3(f.n, f.e1, f.e2);
  for (int j = 0; j < 3; ++j) f.c[j] = ((f.v[0][j] + f.v[1][j]) + f.v[2][j]) / 3.0;
  for (int k = 0; k < 3; ++k) {
    double d[3];
    for (int j = 0; j < 3; ++j) d[j] = f.v[k][j] - f.c[j];
    f.p[k][0] = dot3(d, f.e1);
    f.p[k][1] = dot3(d, f.e2);
  }
  // lam_k(eta) = A_k + B_k eta_1 + C_k eta_2 with lam_k(p_j) = delta_kj
  const double det = (f.p[1][0] - f.p[0][0]) * (f.p[2][1] - f.p[0][1]) -
                     (f.p[2][0] - f.p[0][0]) * (f.p[1][1] - f.p[0][1]);
  for (int k = 0; k < 3; ++k) {
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    f.abc[k][0] = (f.p[i][0] * f.p[j][1] - f.p[j][0] * f.p[i][1]) / det;
    f.abc[k][1] = (f.p[i][1] - f.p[j][1]) / det;
    f.abc[k][2] = (f.p[j][0] - f.p[i][0]) / det;
  }
}

// Signed height and in-plane coordinates of a point (frame.py:251-256).
MHS_FI void to_plane(const Frame& f, const double* x, double& z, double& X0, double& X1) {
  const double d[3] = {x[0] - f.c[0], x[1] - f.c[1], x[2] - f.c[2]};
  z = dot3(d, f.n);
  X0 = dot3(d, f.e1);
  X1 = dot3(d, f.e2);
}

// --------------------------------------------------------- shape functions
// Monomial coefficients c[k][tri_idx(a, b)] of the order-P Lagrange shape
// functions in the observer-centred coordinate xi = eta - X
// (mhs/fullspace/shape.py:114-147).  Node order: P0 centroid; P1 v1 v2 v3;
// P2 v1 v2 v3 m12 m23 m31.
template <int P>
MHS_HD void shape_coeffs(const Frame& f, double X0, double X1, double c[][ntri(P) > 0 ? ntri(P) : 1]) {
  if constexpr (P == 0) {
    c[0][0] = 1.0;
  } else {
    double l0[3], lx[3], ly[3];  // affine lam_i(xi) = l0 + lx xi1 + ly xi2
    for (int i = 0; i < 3; ++i) {
      l0[i] = f.abc[i][0] + X0 * f.abc[i][1] + X1 * f.abc[i][2];
      lx[i] = f.abc[i][1];
      ly[i] = f.abc[i][2];
    }
    if constexpr (P == 1) {
      for (int k = 0; k < 3; ++k) {
        c[k][tri_idx(0, 0)] = l0[k];
        c[k][tri_idx(1, 0)] = lx[k];
        c[k][tri_idx(0, 1)] = ly[k];
      }
    } else {
      // vertex k: lam_k (2 lam_k - 1) = (2 lam_k) * (lam_k - 1/2)
      for (int k = 0; k < 3; ++k) {
        const double a0 = 2.0 * l0[k], ax = 2.0 * lx[k], ay = 2.0 * ly[k];
        const double b0 = l0[k] - 0.5, bx = lx[k], by = ly[k];
        c[k][tri_idx(0, 0)] = a0 * b0;
        c[k][tri_idx(1, 0)] = a0 * bx + ax * b0;
        c[k][tri_idx(0, 1)] = a0 * by + ay * b0;
        c[k][tri_idx(2, 0)] = ax * bx;
        c[k][tri_idx(1, 1)] = ax * by + ay * bx;
        c[k][tri_idx(0, 2)] = ay * by;
      }
      // edge node (i, j): (2 lam_i)(2 lam_j)
      const int ei[3] = {0, 1, 2}, ej[3] = {1, 2, 0};
      for (int e = 0; e < 3; ++e) {
        const int i = ei[e], j = ej[e];
        const double a0 = 2.0 * l0[i], ax = 2.0 * lx[i], ay = 2.0 * ly[i];
        const double b0 = 2.0 * l0[j], bx = 2.0 * lx[j], by = 2.0 * ly[j];
        double* ck = c[3 + e];
        ck[tri_idx(0, 0)] = a0 * b0;
        ck[tri_idx(1, 0)] = a0 * bx + ax * b0;
        ck[tri_idx(0, 1)] = a0 * by + ay * b0;
        ck[tri_idx(2, 0)] = ax * bx;
        ck[tri_idx(1, 1)] = ax * by + ay * bx;
        ck[tri_idx(0, 2)] = ay * by;
      }
    }
  }
}

// Shape functions at centroid-frame point eta (the far/quadrature rules
// evaluate N_k at their nodes, i.e. shape_coeffs about X = 0 at xi = eta).
template <int P>
MHS_HD void shape_at(const Frame& f, double eta0, double eta1, double* N) {
  constexpr int K = n_nodes(P);
  if constexpr (P == 0) {
    N[0] = 1.0;
  } else {
    double c[K][ntri(P)];
    shape_coeffs<P>(f, 0.0, 0.0, c);
    for (int k = 0; k < K; ++k) {
      double acc = 0.0;
      for (int a = 0; a <= P; ++a)
        for (int b = 0; b <= P - a; ++b) {
          double m = 1.0;
          for (int i = 0; i < a; ++i) m *= eta0;
          for (int i = 0; i < b; ++i) m *= eta1;
          acc += c[k][tri_idx(a, b)] * m;
        }
      N[k] = acc;
    }
  }
}

// ----------------------------------------------------------- material data
// Derived constants, formed exactly as mhs forms them at each seam:
// the full-space engine takes (mu, nu) with nu = lam / (2 (lam + mu)) and
// rebuilds lam from it (mhs/kernels/assemble.py:58-66, fullspace/kernels.py:58);
// the image uses nu = lam / (2 (lam + mu)) and 1 / (pi mu (1 - nu)) written
// in (mu, lam) (mhs/kernels/image.py:451-456).
struct Material {
  double mu, lam;        // as given
  double nu_d, lam_d;    // full-space engine
  double C1, c34, one_m_nu;
  double nu_i, scale_c;  // image
  double nu_f;           // fold / Boussinesq
};

MHS_HD Material make_material(double mu, double lam) {
  Material m;
  m.mu = mu;
  m.lam = lam;
  m.nu_d = 0.5 * lam / (lam + mu);
  m.lam_d = 2.0 * mu * m.nu_d / (1.0 - 2.0 * m.nu_d);
  m.one_m_nu = 1.0 - m.nu_d;
  m.C1 = 1.0 / (16.0 * cst::PI * mu * (1.0 - m.nu_d));
  m.c34 = 3.0 - 4.0 * m.nu_d;
  m.nu_i = lam / (2.0 * (lam + mu));
  m.scale_c = 2.0 * (lam + mu) / (cst::PI * mu * (lam + 2.0 * mu));
  m.nu_f = 0.5 * lam / (lam + mu);
  return m;
}

}  // namespace mhs
