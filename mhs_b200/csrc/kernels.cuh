// Device side of the assembly pipeline: the kernels and the per-request
// launch sequence (run).  Included only by the kernel units (unit.cu), each
// of which instantiates one (order, readout, precision) combination.
#pragma once

#include <algorithm>
#include <type_traits>
#include <vector>

#include "pipeline.cuh"

namespace mhs {
namespace pipe {
namespace {

// ------------------------------------------------------------ device data
// Gauss-Legendre nodes and weights of every order (gl_offset layout); one
// copy per unit, filled by the unit's init entry point.
__device__ double d_glx[GL_TABLE];
__device__ double d_glw[GL_TABLE];

// --------------------------------------------------------------- helpers
__device__ __forceinline__ void atomic_status(int* st, int bits) { atomicOr(st, bits); }

// One node of the collapsed Gauss product rule of order n (q = i * n + j).
template <int P>
__device__ __forceinline__ void rule_node(const Frame& f, int n, int q, double& e0, double& e1,
                                          double& wq, double* N) {
  const double* x = d_glx + gl_offset(n);
  const double* w = d_glw + gl_offset(n);
  const int i = q / n, j = q % n;
  const double gi = 0.5 * (x[i] + 1.0), wi = 0.5 * w[i];
  const double gj = 0.5 * (x[j] + 1.0), wj = 0.5 * w[j];
  const double x1 = gi, x2 = gj * (1.0 - gi);
  const double ww = wi * wj * (1.0 - gi);
  const double l0 = 1.0 - x1 - x2;
  e0 = (l0 * f.p[0][0] + x1 * f.p[1][0]) + x2 * f.p[2][0];
  e1 = (l0 * f.p[0][1] + x1 * f.p[1][1]) + x2 * f.p[2][1];
  wq = ww * (2.0 * f.area);
  shape_at<P>(f, e0, e1, N);
}

// Shared-memory far-field rules of one frame (orders 12 and 8).
template <int P>
struct SmemRules {
  static constexpr int K = n_nodes(P);
  static constexpr int N12 = cst::FAR_GAUSS_N * cst::FAR_GAUSS_N;
  static constexpr int N8 = cst::FAR_GAUSS_N_DISTANT * cst::FAR_GAUSS_N_DISTANT;
  double e0[N12 + N8], e1[N12 + N8], wq[N12 + N8], Nq[(N12 + N8) * K];
  __device__ void build(const Frame& f, int tid, int nthr) {
    for (int t = tid; t < N12 + N8; t += nthr) {
      const int n = t < N12 ? cst::FAR_GAUSS_N : cst::FAR_GAUSS_N_DISTANT;
      const int q = t < N12 ? t : t - N12;
      rule_node<P>(f, n, q, e0[t], e1[t], wq[t], Nq + t * K);
    }
  }
  __device__ QuadRule r12() const { return QuadRule{N12, e0, e1, wq, Nq}; }
  __device__ QuadRule r8() const { return QuadRule{N8, e0 + N12, e1 + N12, wq + N12, Nq + N12 * K}; }
};

// The mixed form's far rules, in float: MIXED_GAUSS_N x MIXED_GAUSS_N for
// MIXED_NEAR_L L < D <= D_STAR L, MIXED_GAUSS_N_FAR x MIXED_GAUSS_N_FAR beyond.
template <int P>
struct FloatRules {
  static constexpr int NM = MIXED_GAUSS_N * MIXED_GAUSS_N;
  static constexpr int NF = MIXED_GAUSS_N_FAR * MIXED_GAUSS_N_FAR;
  static constexpr int N = NM + NF;
  float e0[N], e1[N], wq[N], Nq[N * n_nodes(P)];
};
struct NoRules {};

// Nodes formed in double, then rounded.
template <int P>
__device__ void build_float_rules(const Frame& f, FloatRules<P>& fr, int tid, int nthr) {
  constexpr int NM = FloatRules<P>::NM, K = n_nodes(P);
  for (int t = tid; t < FloatRules<P>::N; t += nthr) {
    const int n = t < NM ? MIXED_GAUSS_N : MIXED_GAUSS_N_FAR;
    const int q = t < NM ? t : t - NM;
    double e0, e1, wq, Nq[K];
    rule_node<P>(f, n, q, e0, e1, wq, Nq);
    fr.e0[t] = (float)e0;
    fr.e1[t] = (float)e1;
    fr.wq[t] = (float)wq;
    for (int k = 0; k < K; ++k) fr.Nq[t * K + k] = (float)Nq[k];
  }
}

template <int P>
__device__ QuadRuleT<float> float_rule_mid(const FloatRules<P>& fr) {
  return QuadRuleT<float>{FloatRules<P>::NM, fr.e0, fr.e1, fr.wq, fr.Nq};
}
template <int P>
__device__ QuadRuleT<float> float_rule_far(const FloatRules<P>& fr) {
  constexpr int O = FloatRules<P>::NM;
  return QuadRuleT<float>{FloatRules<P>::NF, fr.e0 + O, fr.e1 + O, fr.wq + O,
                          fr.Nq + O * n_nodes(P)};
}

// ---------------------------------------------------------------- k_coef
// Record coefficients t of one material (t < MHS_Q_NDDG covers every table).
__device__ __forceinline__ void coef_entry(double mu, double lam, double* out, int t) {
  const Material m = make_material(mu, lam);
  const double nu = m.nu_i, s = m.scale_c;
  const double nup[3] = {1.0, nu, nu * nu};
  double* r_dg = out;
  double* r_ddg = r_dg + 3 * MHS_R_NDG;
  double* q_dg = r_ddg + 3 * MHS_R_NDDG;
  double* q_ddg = q_dg + MHS_Q_NDG;
  if (t < MHS_R_NDG)
    for (int pz = 0; pz < 3; ++pz) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += tab_d::mhs_r_dg_c[t][pz][k] * nup[k];
      r_dg[3 * t + pz] = v * s;
    }
  if (t < MHS_R_NDDG)
    for (int pz = 0; pz < 3; ++pz) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += tab_d::mhs_r_ddg_c[t][pz][k] * nup[k];
      r_ddg[3 * t + pz] = v * s;
    }
  if (t < MHS_Q_NDG) {
    double v = 0.0;
    for (int k = 0; k < 3; ++k) v += tab_d::mhs_q_dg_c[t][k] * nup[k];
    q_dg[t] = v;
  }
  if (t < MHS_Q_NDDG) {
    double v = 0.0;
    for (int k = 0; k < 3; ++k) v += tab_d::mhs_q_ddg_c[t][k] * nup[k];
    q_ddg[t] = v;
  }
}

// Per-pass image coefficients (and the pass's status word cleared).
__global__ void k_coef(const ReqDesc* __restrict__ D, const long long* __restrict__ off, int nreq) {
  const int r = find_req(off, nreq, blockIdx.x);
  const ReqDesc& d = D[r];
  const long long b = blockIdx.x - off[r];
  if (b == 0 && threadIdx.x == 0) *d.status = 0;
  coef_entry(d.fa.mu, d.fa.lam, d.coef, (int)(b * blockDim.x + threadIdx.x));
}

// The same for one material (diagnostics).
__global__ void k_coef1(double mu, double lam, double* out) {
  coef_entry(mu, lam, out, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------- k_prep
__global__ void k_prep(const ReqDesc* __restrict__ D, const long long* __restrict__ off, int nreq,
                       int want_g) {
  const int r = find_req(off, nreq, blockIdx.x);
  const ReqDesc& d = D[r];
  const int64_t s = (blockIdx.x - off[r]) * (int64_t)blockDim.x + threadIdx.x;
  if (s >= d.fa.n_src) return;
  const double* __restrict__ tris = d.tris;
  const double* __restrict__ eps = d.eps;
  const int fold = d.fold;
  SrcPrep* __restrict__ prep = d.prep;
  double* __restrict__ G = d.G;
  SrcPrep p;
  const double* t = tris + 9 * s;
  double ti[9];
  for (int i = 0; i < 9; ++i) ti[i] = (i % 3 == 2) ? -t[i] : t[i];
  make_frame(t, p.f);
  make_frame(ti, p.fi);
  p.eps = eps[s];
  fold_crease(t, p.eps, p.centre, &p.r_f);
  p.diam = tri_diameter(t);
  p.straddle = (fold && fold_straddles(t, p.eps)) ? 1 : 0;
  p.pad = 0;
  prep[s] = p;
  if (want_g) build_basis_products(p.fi, G + s * G_SIZE);
}

// ---------------------------------------------------------------- k_pair
// Direct term of one (observer, source) pair, stored as the pair's row of
// the table (the image kernels add to it).  RF: arithmetic type of the
// far-field quadrature (double; float in the mixed form).
template <int P, int KC, class RF>
__global__ void __launch_bounds__(TB)
k_pair(const ReqDesc* __restrict__ D, const long long* __restrict__ off, int nreq,
       double near_l_mixed) {
  constexpr int K = n_nodes(P);
  constexpr int NR = row_of(KC);
  const int r = find_req(off, nreq, blockIdx.x);
  const ReqDesc& d = D[r];
  const int64_t lo = d.fa.lo, n_chunk = d.fa.n_chunk, n_src = d.fa.n_src;
  const long long local = blockIdx.x - off[r];
  const int64_t s = local % n_src, tile = local / n_src;
  const double* __restrict__ obs = d.obs;
  const SrcPrep* __restrict__ prep = d.prep;
  const double mu = d.fa.mu, lam = d.fa.lam;
  double* __restrict__ T = d.T;
  constexpr bool F32 = std::is_same<RF, float>::value;
  // far rules of the element: double, or float only in the mixed form
  __shared__ SrcPrep sp;
  __shared__ std::conditional_t<F32, NoRules, SmemRules<P>> rd;
  __shared__ std::conditional_t<F32, FloatRules<P>, NoRules> rdf;
  if (threadIdx.x == 0) sp = prep[s];
  __syncthreads();
  if constexpr (F32) build_float_rules<P>(sp.f, rdf, threadIdx.x, blockDim.x);
  else rd.build(sp.f, threadIdx.x, blockDim.x);
  __syncthreads();
  const double near_l = F32 ? near_l_mixed : cst::D_STAR;
  const int64_t oc = tile * (int64_t)blockDim.x + threadIdx.x;
  if (oc >= n_chunk) return;
  const int64_t o = lo + oc;
  const double x[3] = {obs[3 * o], obs[3 * o + 1], obs[3 * o + 2]};
  const Material m = make_material(mu, lam);
  const double eps = sp.eps;
  double* row = T + ((oc * n_src + s) * K) * NR;
  if constexpr (KC == KD_E) {
    double E[K] = {};
    if constexpr (F32)
      direct_eval<P, W_E, RF>(sp.f, float_rule_mid<P>(rdf), float_rule_far<P>(rdf), x, eps, m,
                              nullptr, nullptr, E, near_l, cst::D_STAR);
    else
      direct_eval<P, W_E, RF>(sp.f, rd.r12(), rd.r8(), x, eps, m, nullptr, nullptr, E);
    for (int k = 0; k < K; ++k) {
      row[k * NR + 0] = E[k];
      row[k * NR + 1] = 0.0;
    }
  } else {
    constexpr int C = comps_of(KC);
    double Abuf[K * C] = {}, E[K] = {};
    // at P >= 1 the node tensors stay in memory (K * C doubles)
    double* A = P > 0 ? in_memory(Abuf) : Abuf;
    if constexpr (F32) {
      const QuadRuleT<float> f12 = float_rule_mid<P>(rdf), f8 = float_rule_far<P>(rdf);
      if constexpr (KC == KD_DISP)
        direct_eval<P, W_U, RF>(sp.f, f12, f8, x, eps, m, A, nullptr, nullptr, near_l, cst::D_STAR);
      else
        direct_eval<P, W_H | W_E, RF>(sp.f, f12, f8, x, eps, m, nullptr, A, E, near_l,
                                      cst::D_STAR);
    } else {
      if constexpr (KC == KD_DISP)
        direct_eval<P, W_U, RF>(sp.f, rd.r12(), rd.r8(), x, eps, m, A, nullptr, nullptr);
      else
        direct_eval<P, W_H | W_E, RF>(sp.f, rd.r12(), rd.r8(), x, eps, m, nullptr, A, E);
    }
    for (int k = 0; k < K; ++k) {
      for (int c = 0; c < C; ++c) row[k * NR + c] = A[k * C + c];
      row[k * NR + C] = (KC == KD_HE) ? E[k] : 0.0;
      row[k * NR + C + 1] = 0.0;
    }
  }
}

// ------------------------------------------------- k_image_w, k_image_r
// Image R-family of one (observer, source) pair outside the source's fold
// band (the fold replaces it there), in two kernels over the request's
// table buffer Wimg[s][k][j][oc] (observer innermost): k_image_w forms the
// image frame's weighted tables of every node (one launch for the pairs in
// closed-form range, one for the far rules), k_image_r reads them back,
// runs the generated records and adds the result to the pair's row.  Apart,
// each kernel keeps its own working set in registers: the moment table, the
// far rule's accumulators or the records' 27 sums.
template <int P>
__device__ __forceinline__ StridedTable image_table(const ReqDesc& d, int64_t s, int k,
                                                    int64_t oc) {
  const int64_t n_chunk = d.fa.n_chunk;
  return {d.Wimg + ((s * n_nodes(P) + k) * IMG_NW) * n_chunk + oc, n_chunk};
}

template <int P, int KC, class RF, int PART>
__global__ void __launch_bounds__(TB)
k_image_w(const ReqDesc* __restrict__ D, const long long* __restrict__ off, int nreq,
          double near_l_mixed) {
  static_assert(KC != KD_E, "the eigenstress readout has no image term");
  const int r = find_req(off, nreq, blockIdx.x);
  const ReqDesc& d = D[r];
  const int64_t lo = d.fa.lo, n_chunk = d.fa.n_chunk, n_src = d.fa.n_src;
  const long long local = blockIdx.x - off[r];
  const int64_t s = local % n_src, tile = local / n_src;
  constexpr bool F32 = std::is_same<RF, float>::value;
  // far rules of the reflected element
  __shared__ SrcPrep sp;
  __shared__ std::conditional_t<F32, NoRules, SmemRules<P>> ri;
  __shared__ std::conditional_t<F32, FloatRules<P>, NoRules> rif;
  if (threadIdx.x == 0) sp = d.prep[s];
  __syncthreads();
  if constexpr (PART != TAB_CLOSED) {
    if constexpr (F32) build_float_rules<P>(sp.fi, rif, threadIdx.x, blockDim.x);
    else ri.build(sp.fi, threadIdx.x, blockDim.x);
    __syncthreads();
  }
  const int64_t oc = tile * (int64_t)blockDim.x + threadIdx.x;
  if (oc >= n_chunk) return;
  const int64_t o = lo + oc;
  const double x[3] = {d.obs[3 * o], d.obs[3 * o + 1], d.obs[3 * o + 2]};
  const double eps = sp.eps;
  if (sp.straddle && fold_band(x, sp.centre, eps)) return;
  const StridedTable W = image_table<P>(d, s, 0, oc);
  if constexpr (F32) {
    const QuadRuleT<float> i12 = float_rule_mid<P>(rif), i8 = float_rule_far<P>(rif);
    image_r_tables<P, float, PART>(sp.fi, i12, i8, x, eps, W, near_l_mixed, cst::D_STAR);
  } else {
    image_r_tables<P, double, PART>(sp.fi, ri.r12(), ri.r8(), x, eps, W);
  }
}

template <int P, int KC>
__global__ void __launch_bounds__(TB)
k_image_r(const ReqDesc* __restrict__ D, const long long* __restrict__ off, int nreq) {
  static_assert(KC != KD_E, "the eigenstress readout has no image term");
  constexpr int K = n_nodes(P);
  constexpr int NR = row_of(KC);
  constexpr int C = comps_of(KC);
  const int r = find_req(off, nreq, blockIdx.x);
  const ReqDesc& d = D[r];
  const int64_t lo = d.fa.lo, n_chunk = d.fa.n_chunk, n_src = d.fa.n_src;
  const long long local = blockIdx.x - off[r];
  const int64_t s = local % n_src, tile = local / n_src;
  // the source's basis products and the R-family coefficients of the
  // request's material (read record by record, K times per pair)
  __shared__ SrcPrep sp;
  __shared__ double sG[G_SIZE];
  __shared__ double sRc[3 * (MHS_R_NDG + MHS_R_NDDG)];
  if (threadIdx.x == 0) sp = d.prep[s];
  for (int i = threadIdx.x; i < G_SIZE; i += blockDim.x) sG[i] = d.G[s * G_SIZE + i];
  for (int i = threadIdx.x; i < 3 * (MHS_R_NDG + MHS_R_NDDG); i += blockDim.x) sRc[i] = d.coef[i];
  __syncthreads();
  const int64_t oc = tile * (int64_t)blockDim.x + threadIdx.x;
  if (oc >= n_chunk) return;
  const int64_t o = lo + oc;
  const double x[3] = {d.obs[3 * o], d.obs[3 * o + 1], d.obs[3 * o + 2]};
  if (sp.straddle && fold_band(x, sp.centre, sp.eps)) return;
  const Material m = make_material(d.fa.mu, d.fa.lam);
  ImageCoef ic = image_coef_view(d.coef);
  ic.r_dg = sRc;
  ic.r_ddg = sRc + 3 * MHS_R_NDG;
  double zpow[G_RMAX + 1];
  image_r_zpow(sp.fi, x, zpow);
  double* row = d.T + ((oc * n_src + s) * K) * NR;
#pragma unroll 1
  for (int k = 0; k < K; ++k) {
    double B[C];
    if constexpr (KC == KD_DISP)
      image_r_node<P, W_U>(sG, image_table<P>(d, s, k, oc), zpow, x[2], sp.f.n, m, ic, B,
                           nullptr);
    else
      image_r_node<P, W_H>(sG, image_table<P>(d, s, k, oc), zpow, x[2], sp.f.n, m, ic, nullptr,
                           B);
    for (int c = 0; c < C; ++c) row[k * NR + c] += B[c];
  }
}

// -------------------------------------------------------------- k_imageq
// Image Q-family of one pair, added to the scratch row.  The floor order
// (8 x 8 points, almost every pair) reads a shared-memory rule; higher
// orders generate their nodes on the fly.
template <int P, class E = double>
struct QRuleSmem {
  static constexpr int K = n_nodes(P);
  const E* y;
  const E* wN;
  int nq;
  __device__ int count() const { return nq; }
  __device__ void node(int t, E* yy, E* w) const {
    yy[0] = y[3 * t];
    yy[1] = y[3 * t + 1];
    yy[2] = y[3 * t + 2];
    for (int k = 0; k < K; ++k) w[k] = wN[t * K + k];
  }
};

template <int P>
struct QRuleFly {
  static constexpr int K = n_nodes(P);
  const Frame* f;
  int n;
  __device__ int count() const { return n * n; }
  __device__ void node(int t, double* yy, double* w) const {
    double e0, e1, wq, N[K];
    rule_node<P>(*f, n, t, e0, e1, wq, N);
    // Cartesian node on the real element: barycentric (l0, x1, x2) @ tri
    const double* x = d_glx + gl_offset(n);
    const int i = t / n, j = t % n;
    const double gi = 0.5 * (x[i] + 1.0), gj = 0.5 * (x[j] + 1.0);
    const double x1 = gi, x2 = gj * (1.0 - gi), l0 = 1.0 - x1 - x2;
    for (int c = 0; c < 3; ++c) yy[c] = (l0 * f->v[0][c] + x1 * f->v[1][c]) + x2 * f->v[2][c];
    for (int k = 0; k < K; ++k) w[k] = wq * N[k];
  }
};

// RF = float (the mixed form): pairs at the floor order -- at least about an
// element from the image triangle -- sum their points in float.
// At P0 in double three blocks per SM (168 registers) run 11 % faster than
// two; the float sums keep their registers.
template <int P, int KC, class RF>
__global__ void __launch_bounds__(TB, (P == 0 && std::is_same<RF, double>::value) ? 3 : 1)
k_imageq(const ReqDesc* __restrict__ D, const long long* __restrict__ off, int nreq,
         unsigned long long* __restrict__ census) {
  constexpr int K = n_nodes(P);
  constexpr int NR = row_of(KC);
  constexpr int C = comps_of(KC);
  const int r = find_req(off, nreq, blockIdx.x);
  const ReqDesc& d = D[r];
  const int64_t lo = d.fa.lo, n_chunk = d.fa.n_chunk, n_src = d.fa.n_src;
  const long long local = blockIdx.x - off[r];
  const int64_t s = local % n_src, tile = local / n_src;
  const double* __restrict__ obs = d.obs;
  const SrcPrep* __restrict__ prep = d.prep;
  const double* __restrict__ coef = d.coef;
  const double mu = d.fa.mu, lam = d.fa.lam;
  double* __restrict__ T = d.T;
  __shared__ SrcPrep sp;
  __shared__ double qy[QFLOOR * QFLOOR * 3];
  __shared__ double qw[QFLOOR * QFLOOR * K];
  constexpr bool F32 = std::is_same<RF, float>::value;
  __shared__ float qyf[F32 ? QFLOOR * QFLOOR * 3 : 1];
  __shared__ float qwf[F32 ? QFLOOR * QFLOOR * K : 1];
  if (threadIdx.x == 0) sp = prep[s];
  __syncthreads();
  {
    QRuleFly<P> fly{&sp.f, QFLOOR};
    for (int t = threadIdx.x; t < QFLOOR * QFLOOR; t += blockDim.x) fly.node(t, qy + 3 * t, qw + K * t);
  }
  __syncthreads();
  if constexpr (F32) {
    for (int t = threadIdx.x; t < QFLOOR * QFLOOR * 3; t += blockDim.x) qyf[t] = (float)qy[t];
    for (int t = threadIdx.x; t < QFLOOR * QFLOOR * K; t += blockDim.x) qwf[t] = (float)qw[t];
    __syncthreads();
  }
  const int64_t oc = tile * (int64_t)blockDim.x + threadIdx.x;
  if (oc >= n_chunk) return;
  const int64_t o = lo + oc;
  const double x[3] = {obs[3 * o], obs[3 * o + 1], obs[3 * o + 2]};
  const double eps = sp.eps;
  if (sp.straddle && fold_band(x, sp.centre, eps)) return;
  const Material m = make_material(mu, lam);
  const ImageCoef ic = image_coef_view(coef);
  double ti[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) ti[3 * i + j] = sp.fi.v[i][j];
  const int n = q_gauss_order(x, ti, eps, sp.f.L, P);
  if (census) {
    atomicAdd(&census[MHS_CENSUS_Q_PAIRS], 1ull);
    atomicAdd(&census[MHS_CENSUS_Q_POINTS], (unsigned long long)n * (unsigned long long)n);
  }
  double B[K * C] = {};
  constexpr int WANT = KC == KD_DISP ? W_U : W_H;
  bool done = false;
  if constexpr (F32) {
    if (n == QFLOOR) {
      QRuleSmem<P, float> r{qyf, qwf, QFLOOR * QFLOOR};
      image_q_eval<P, WANT, QRuleSmem<P, float>, float>(r, sp.f.n, x, eps, m, ic, B, B);
      done = true;
    }
  }
  if (done) {
  } else if (n == QFLOOR) {
    QRuleSmem<P> r{qy, qw, QFLOOR * QFLOOR};
    image_q_eval<P, WANT>(r, sp.f.n, x, eps, m, ic, B, B);
  } else {
    QRuleFly<P> r{&sp.f, n};
    image_q_eval<P, WANT>(r, sp.f.n, x, eps, m, ic, B, B);
  }
  double* row = T + ((oc * n_src + s) * K) * NR;
  for (int k = 0; k < K; ++k)
    for (int c = 0; c < C; ++c) row[k * NR + c] += B[k * C + c];
}

// ---------------------------------------------------------------- k_band
// Ordered list of the band receivers of each straddling source, in slots
// [s * n_chunk, s * n_chunk + cnt[s]).
__global__ void __launch_bounds__(256)
k_band(int64_t lo, int64_t n_chunk, const double* __restrict__ obs,
       const SrcPrep* __restrict__ prep, int* __restrict__ cnt, int* __restrict__ list) {
  const int64_t s = blockIdx.x;
  __shared__ int warp_n[8];
  __shared__ int base;
  const SrcPrep& p = prep[s];
  if (!p.straddle) {
    if (threadIdx.x == 0) cnt[s] = 0;
    return;
  }
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t t0 = 0; t0 < n_chunk; t0 += 256) {
    const int64_t oc = t0 + threadIdx.x;
    bool pred = false;
    if (oc < n_chunk) {
      const double x[3] = {obs[3 * (lo + oc)], obs[3 * (lo + oc) + 1], obs[3 * (lo + oc) + 2]};
      pred = fold_band(x, p.centre, p.eps);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, pred);
    if (lane == 0) warp_n[wid] = __popc(bal);
    __syncthreads();
    int off = base;
    for (int w = 0; w < wid; ++w) off += warp_n[w];
    if (pred) list[s * n_chunk + off + __popc(bal & ((1u << lane) - 1u))] = (int)oc;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < 8; ++w) tot += warp_n[w];
      base += tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) cnt[s] = base;
}

// --------------------------------------------------------- k_fold_mirror
// The mirror element of every band pair, one thread per pair: its
// full-space field with the slip signs of the reflection (fold.py:334-350)
// added to the pair's row, and its blob weight (the mirror eigenstress).
template <int P, int KC, class RF>
__global__ void __launch_bounds__(TB)
k_fold_mirror(int64_t lo, int64_t n_chunk, int64_t n_src, const double* __restrict__ obs,
              const SrcPrep* __restrict__ prep, const int* __restrict__ cnt,
              const int* __restrict__ list, double mu, double lam, double* __restrict__ T) {
  constexpr int K = n_nodes(P);
  constexpr int NR = row_of(KC);
  constexpr int C = comps_of(KC);
  const int64_t s = blockIdx.x;
  const int n_band = cnt[s];
  if ((int64_t)blockIdx.y * TB >= n_band) return;
  __shared__ SrcPrep sp;
  __shared__ SmemRules<P> rm;
  if (threadIdx.x == 0) sp = prep[s];
  __syncthreads();
  rm.build(sp.fi, threadIdx.x, TB);
  __syncthreads();
  const int bi = blockIdx.y * TB + threadIdx.x;
  if (bi >= n_band) return;
  const int64_t oc = list[s * n_chunk + bi];
  const int64_t o = lo + oc;
  const double x[3] = {obs[3 * o], obs[3 * o + 1], obs[3 * o + 2]};
  const Material m = make_material(mu, lam);
  const double eps = sp.eps;
  double* row = T + ((oc * n_src + s) * K) * NR;
  double E[K] = {};
  if constexpr (KC == KD_E) {
    direct_eval<P, W_E, RF>(sp.fi, rm.r12(), rm.r8(), x, eps, m, nullptr, nullptr, E);
    for (int k = 0; k < K; ++k) row[k * NR + 1] = E[k];
  } else if constexpr (KC == KD_HE) {
    double Mv[K * 27] = {};
    direct_eval<P, W_H | W_E, RF>(sp.fi, rm.r12(), rm.r8(), x, eps, m, nullptr, Mv, E);
    for (int k = 0; k < K; ++k) {
      for (int i = 0; i < 27; ++i) row[k * NR + i] += Mv[27 * k + i] * mirror_slip_sign(i % 3);
      row[k * NR + C + 1] = E[k];
    }
  } else {
    double Mv[K * 9] = {};
    direct_eval<P, W_U, RF>(sp.fi, rm.r12(), rm.r8(), x, eps, m, Mv, nullptr, nullptr);
    for (int k = 0; k < K; ++k)
      for (int i = 0; i < 9; ++i) row[k * NR + i] += Mv[9 * k + i] * mirror_slip_sign(i % 3);
  }
}

#include "fold_waves.cuh"

// --------------------------------------------------------------- k_final

// Eigenstress C:sym(slip (x) n) of one row: phi C(n) + phi_m C(n_m) sign.
__device__ __forceinline__ double eig_comp(const SrcPrep& p, double phi, double phim, double mu,
                                           double lam, int a, int b, int m) {
  const double* n = p.f.n;
  const double* nm = p.fi.n;
  const double c = (a == b ? lam * n[m] : 0.0) + mu * ((a == m ? n[b] : 0.0) + (b == m ? n[a] : 0.0));
  const double cm = (a == b ? lam * nm[m] : 0.0) + mu * ((a == m ? nm[b] : 0.0) + (b == m ? nm[a] : 0.0));
  return phi * c + phim * (cm * mirror_slip_sign(m));
}

template <class OUT>
__device__ __forceinline__ void store(void* out, int64_t i, double v) {
  reinterpret_cast<OUT*>(out)[i] = (OUT)v;
}

// Value of output component `comp` of one (observer, source, node) row.
template <int KC>
__device__ void row_values(const FinalArgs& a, const SrcPrep& p, const double* row, int64_t o,
                           int64_t scol, double* v, int nv) {
  constexpr int C = comps_of(KC);
  const double phi = row[C], phim = row[C + 1];
  const double mu = a.mu, lam = a.lam;
  switch (a.kind) {
    case MHS_DISP:
      for (int i = 0; i < 9; ++i) v[i] = row[i];
      break;
    case MHS_TOTAL_STRESS:
      for (int i = 0; i < 27; ++i) v[i] = row[i];
      break;
    case MHS_EIGENSTRESS:
      for (int aa = 0; aa < 3; ++aa)
        for (int b = 0; b < 3; ++b)
          for (int m = 0; m < 3; ++m) v[9 * aa + 3 * b + m] = eig_comp(p, row[0], row[1], mu, lam, aa, b, m);
      break;
    case MHS_STRESS:
    case MHS_STRAIN:
      for (int aa = 0; aa < 3; ++aa)
        for (int b = 0; b < 3; ++b)
          for (int m = 0; m < 3; ++m) {
            double s = row[9 * aa + 3 * b + m];
            if (a.subtract) s -= eig_comp(p, phi, phim, mu, lam, aa, b, m);
            v[9 * aa + 3 * b + m] = s;
          }
      if (a.kind == MHS_STRAIN)
        for (int m = 0; m < 3; ++m) {
          const double tr = v[m] + v[12 + m] + v[24 + m];
          const double tre = tr / (3.0 * lam + 2.0 * mu);
          for (int d = 0; d < 3; ++d) v[12 * d + m] -= lam * tre;
          for (int i = 0; i < 9; ++i) v[3 * i + m] /= (2.0 * mu);
        }
      break;
    default: {  // traction / interaction
      const double* n = a.normals + 3 * o;
      double t[3][3];
      for (int i = 0; i < 3; ++i)
        for (int m = 0; m < 3; ++m) {
          double s = row[9 * i + 3 * 0 + m] * n[0] + row[9 * i + 3 * 1 + m] * n[1] + row[9 * i + 3 * 2 + m] * n[2];
          if (a.subtract) {
            double e = 0.0;
            for (int j = 0; j < 3; ++j) e += eig_comp(p, phi, phim, mu, lam, i, j, m) * n[j];
            s -= e;
          }
          t[i][m] = s;
        }
      if (a.kind == MHS_TRACTION) {
        for (int i = 0; i < 3; ++i)
          for (int m = 0; m < 3; ++m) v[3 * i + m] = t[i][m];
      } else {
        const double* rb = a.rec_basis + o * a.n_a * 3;
        const double* sb = a.src_basis + scol * a.n_b * 3;
        for (int ia = 0; ia < a.n_a; ++ia)
          for (int ib = 0; ib < a.n_b; ++ib) {
            double acc = 0.0;
            for (int i = 0; i < 3; ++i)
              for (int m = 0; m < 3; ++m) acc += rb[3 * ia + i] * t[i][m] * sb[3 * ib + m];
            v[ia * a.n_b + ib] = acc;
          }
      }
    }
  }
}

__device__ __forceinline__ void store_any(void* out, int64_t i, double v, int f32) {
  if (f32) reinterpret_cast<float*>(out)[i] = (float)v;
  else reinterpret_cast<double*>(out)[i] = v;
}

// Values of output column `col` of observer row `o` of one pass: the
// element's scratch row (discontinuous) or the ordered gather of its shared
// column (continuous).
template <int P, int KC>
__device__ __forceinline__ void column_values(const FinalArgs& a, const SrcPrep* __restrict__ prep,
                                              const double* __restrict__ T, int64_t oc, int64_t o,
                                              int64_t col, double* v, int nv) {
  constexpr int K = n_nodes(P);
  constexpr int NR = row_of(KC);
  if (!a.col_ptr) {
    const int64_t s = col / K;
    const double* row = T + (oc * a.n_src * K + col) * NR;
    row_values<KC>(a, prep[s], row, o, s, v, nv);
  } else {
    for (int i = 0; i < nv; ++i) v[i] = 0.0;
    for (int e = a.col_ptr[col]; e < a.col_ptr[col + 1]; ++e) {
      const int ent = a.col_ent[e];
      const int64_t s = ent / 6;
      const double* row = T + (oc * a.n_src * K + ent) * NR;
      double w[27];
      row_values<KC>(a, prep[s], row, o, col, w, nv);
      for (int i = 0; i < nv; ++i) v[i] += w[i];
    }
  }
}

// Output stage of every pass: the store of each (observer, column) value in
// the caller's layout, or -- in apply mode -- the matrix times the slip
// vector, y[o][c] = sum over columns and slip components of M[o][c][col][s]
// slip[col][s], without storing M (one block per observer row; each thread
// takes a stride of columns and the block's sums are reduced in a fixed
// tree order).  blockDim is a power of two.
template <int P, int KC>
__global__ void __launch_bounds__(TB)
k_out(const ReqDesc* __restrict__ D, const long long* __restrict__ off, int nreq) {
  const int r = find_req(off, nreq, blockIdx.x);
  const ReqDesc& d = D[r];
  const FinalArgs& a = d.fa;
  const SrcPrep* __restrict__ prep = d.prep;
  const double* __restrict__ T = d.T;
  const long long local = blockIdx.x - off[r];
  int nv, ns;
  switch (a.kind) {
    case MHS_DISP:
    case MHS_TRACTION: nv = 9; ns = 3; break;
    case MHS_INTERACTION: nv = a.n_a * a.n_b; ns = a.n_b; break;
    default: nv = 27; ns = 3;
  }
  if (a.slip) {
    const int64_t oc = local;
    const int64_t o = a.lo + oc;
    const int nc = nv / ns;
    double y[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) y[c] = 0.0;
    for (int64_t col = threadIdx.x; col < a.n_dof; col += blockDim.x) {
      double v[27];
      column_values<P, KC>(a, prep, T, oc, o, col, v, nv);
      const double* sl = a.slip + col * ns;
      for (int c = 0; c < nc; ++c) {
        double acc = 0.0;
        for (int m = 0; m < ns; ++m) acc += v[c * ns + m] * sl[m];
        y[c] += acc;
      }
    }
    __shared__ double red[TB][9];
    for (int c = 0; c < 9; ++c) red[threadIdx.x][c] = y[c];
    __syncthreads();
    for (int h = blockDim.x / 2; h >= 1; h >>= 1) {
      if (threadIdx.x < h)
        for (int c = 0; c < 9; ++c) red[threadIdx.x][c] += red[threadIdx.x + h][c];
      __syncthreads();
    }
    if (threadIdx.x < nc) store_any(a.out, o * nc + threadIdx.x, red[0][threadIdx.x], a.out_f32);
    return;
  }
  const long long ctiles = (a.n_dof + blockDim.x - 1) / blockDim.x;
  const int64_t col = (local % ctiles) * (int64_t)blockDim.x + threadIdx.x;
  const int64_t oc = local / ctiles;
  if (col >= a.n_dof) return;
  const int64_t o = a.lo + oc;
  double v[27];
  column_values<P, KC>(a, prep, T, oc, o, col, v, nv);
  // store in the caller's layout
  switch (a.kind) {
    case MHS_DISP:
    case MHS_TRACTION:  // (N, 3, n_dof, 3)
      for (int i = 0; i < 3; ++i)
        for (int m = 0; m < 3; ++m)
          store_any(a.out, ((o * 3 + i) * a.n_dof + col) * 3 + m, v[3 * i + m], a.out_f32);
      break;
    case MHS_INTERACTION:  // (N, n_dof, n_a, n_b)
      for (int i = 0; i < nv; ++i) store_any(a.out, (o * a.n_dof + col) * nv + i, v[i], a.out_f32);
      break;
    default:  // (N, 3, 3, n_dof, 3)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int m = 0; m < 3; ++m)
            store_any(a.out, (((o * 3 + i) * 3 + j) * a.n_dof + col) * 3 + m, v[9 * i + 3 * j + m],
                      a.out_f32);
  }
}

// One pass of one request: its observer chunk [lo, lo + nc) on its own
// workspace; `first` marks the request's first pass (coefficients and
// per-source data are formed once).
struct Pass {
  const mhs_request* r;
  const Layout* L;
  int64_t lo, nc;
  bool first;
};

template <int P, int KC>
void fill_desc(const Pass& p, ReqDesc& d) {
  constexpr int K = n_nodes(P);
  const mhs_request* r = p.r;
  char* ws = (char*)r->workspace;
  const bool cont = r->ids != nullptr;
  FinalArgs& a = d.fa;
  a.kind = r->kind;
  a.subtract = r->subtract_eigenstress;
  a.out_f32 = r->out_f32;
  a.n_a = r->n_a;
  a.n_b = r->n_b;
  a.lo = p.lo;
  a.n_chunk = p.nc;
  a.n_src = r->n_src;
  a.n_obs = r->n_obs;
  a.n_dof = cont ? r->n_cols : r->n_src * K;
  a.normals = r->normals;
  a.rec_basis = r->rec_basis;
  a.src_basis = r->src_basis;
  a.col_ptr = cont ? r->col_ptr : nullptr;
  a.col_ent = cont ? r->col_ent : nullptr;
  a.mu = r->mu;
  a.lam = r->lam;
  a.out = r->out;
  a.slip = r->slip;
  d.obs = r->obs;
  d.tris = r->tris;
  d.eps = r->eps;
  d.prep = (SrcPrep*)(ws + p.L->prep);
  d.G = (double*)(ws + p.L->G);
  d.coef = (double*)(ws + p.L->coef);
  d.T = (double*)(ws + p.L->T);
  d.Wimg = (double*)(ws + p.L->Wimg);
  d.status = (int*)(ws + p.L->status);
  d.fold = r->fold;
  d.pad = 0;
}

// Descriptors and stage block prefixes of n passes (host image of the
// device block at desc_bytes(n)).
template <int P, int KC>
void build_descs(const Pass* ps, int n, const Tune& tune, std::vector<char>& host) {
  host.assign(desc_bytes(n), 0);
  ReqDesc* hd = (ReqDesc*)host.data();
  long long* off = (long long*)(host.data() + align_up(sizeof(ReqDesc) * (size_t)n));
  for (int i = 0; i < n; ++i) fill_desc<P, KC>(ps[i], hd[i]);
  for (int j = 0; j < N_OFF; ++j) off[j * (n + 1)] = 0;
  for (int i = 0; i < n; ++i) {
    const FinalArgs& a = hd[i].fa;
    const long long b[N_OFF] = {
        ps[i].first ? (MHS_Q_NDDG + 255) / 256 : 0,
        ps[i].first ? (a.n_src + 127) / 128 : 0,
        a.n_src * ((a.n_chunk + tune.pair_tb - 1) / tune.pair_tb),
        a.slip ? a.n_chunk : ((a.n_dof + tune.final_tb - 1) / tune.final_tb) * a.n_chunk};
    for (int j = 0; j < N_OFF; ++j) off[j * (n + 1) + i + 1] = off[j * (n + 1) + i] + b[j];
  }
}

// The stages of n passes of this unit, each stage in one launch over all of
// them; the fold runs per pass between the pair stages and the output.  The
// descriptors live at desc (device); upload = 0 when they are there already.
template <int P, int KC, class RF>
int run_passes(const Pass* ps, int n, void* desc, bool upload, cudaStream_t st,
               unsigned long long* census, const Tune& tune) {
  std::vector<char> host;
  build_descs<P, KC>(ps, n, tune, host);
  const long long* hoff = (const long long*)(host.data() + align_up(sizeof(ReqDesc) * (size_t)n));
  if (upload)
    MHS_CUDA_TRY(cudaMemcpyAsync(desc, host.data(), host.size(), cudaMemcpyHostToDevice, st));
  const ReqDesc* D = (const ReqDesc*)desc;
  const long long* off = (const long long*)((const char*)desc + align_up(sizeof(ReqDesc) * (size_t)n));
  auto total = [&](int j) { return hoff[j * (n + 1) + n]; };
  auto offs = [&](int j) { return off + j * (n + 1); };
  if (total(OFF_COEF) > 0) {
    StageTimer t(MHS_STAGE_PREP, st);
    k_coef<<<(unsigned)total(OFF_COEF), 256, 0, st>>>(D, offs(OFF_COEF), n);
    k_prep<<<(unsigned)total(OFF_PREP), 128, 0, st>>>(D, offs(OFF_PREP), n, KC != KD_E);
    count_kernels(2);
  }
  {
    StageTimer t(MHS_STAGE_PAIR, st);
    {
      StageTimer td(MHS_STAGE_PAIR_DIRECT, st);
      k_pair<P, KC, RF><<<(unsigned)total(OFF_PAIR), tune.pair_tb, 0, st>>>(D, offs(OFF_PAIR), n,
                                                                            MIXED_NEAR_L);
      count_kernels(1);
    }
    if constexpr (KC != KD_E) {
      StageTimer ti(MHS_STAGE_PAIR_IMAGE_R, st);
      k_image_w<P, KC, RF, TAB_CLOSED><<<(unsigned)total(OFF_PAIR), tune.pair_tb, 0, st>>>(
          D, offs(OFF_PAIR), n, MIXED_NEAR_L);
      k_image_w<P, KC, RF, TAB_FAR><<<(unsigned)total(OFF_PAIR), tune.pair_tb, 0, st>>>(
          D, offs(OFF_PAIR), n, MIXED_NEAR_L);
      k_image_r<P, KC><<<(unsigned)total(OFF_PAIR), tune.pair_tb, 0, st>>>(D, offs(OFF_PAIR), n);
      count_kernels(3);
    }
  }
  if constexpr (KC != KD_E) {
    StageTimer t(MHS_STAGE_IMAGEQ, st);
    k_imageq<P, KC, RF><<<(unsigned)total(OFF_PAIR), tune.pair_tb, 0, st>>>(D, offs(OFF_PAIR), n,
                                                                            census);
    count_kernels(1);
  }
  for (int i = 0; i < n; ++i) {
    const mhs_request* r = ps[i].r;
    if (!r->fold) continue;
    const Layout& L = *ps[i].L;
    char* ws = (char*)r->workspace;
    int* status = (int*)(ws + L.status);
    SrcPrep* prep = (SrcPrep*)(ws + L.prep);
    int* cnt = (int*)(ws + L.cnt);
    int* list = (int*)(ws + L.list);
    double* T = (double*)(ws + L.T);
    const int64_t lo = ps[i].lo, nc = ps[i].nc;
    StageTimer t(MHS_STAGE_FOLD, st);
    k_band<<<(unsigned)r->n_src, 256, 0, st>>>(lo, nc, r->obs, prep, cnt, list);
    count_kernels(1);
    if constexpr (KC != KD_E) {
      const int rc = fold_waves::run_fold<P, KC, RF>(r, st, ws + L.fold, L.fold_bytes, lo, nc, prep,
                                                     cnt, list, T, status, census, tune);
      if (rc) return rc;
    }
    dim3 gm((unsigned)r->n_src, (unsigned)((nc + TB - 1) / TB));
    k_fold_mirror<P, KC, RF><<<gm, TB, 0, st>>>(lo, nc, r->n_src, r->obs, prep, cnt, list, r->mu,
                                                r->lam, T);
    count_kernels(1);
  }
  {
    StageTimer t(MHS_STAGE_FINAL, st);
    const bool apply = n > 0 && ps[0].r->slip;
    k_out<P, KC><<<(unsigned)total(OFF_FINAL), apply ? TB : tune.final_tb, 0, st>>>(
        D, offs(OFF_FINAL), n);
    count_kernels(1);
  }
  MHS_CUDA_TRY(cudaGetLastError());
  return MHS_OK;
}

// One request on its workspace: its observer chunks one pass after another.
template <int P, int KC, class RF>
int run(const mhs_request* r, cudaStream_t st, const Layout& L, unsigned long long* census,
        const Tune& tune) {
  void* desc = (char*)r->workspace + L.desc;
  for (int64_t lo = 0; lo < r->n_obs; lo += L.chunk) {
    const Pass p{r, &L, lo, std::min<int64_t>(L.chunk, r->n_obs - lo), lo == 0};
    const int rc = run_passes<P, KC, RF>(&p, 1, desc, true, st, census, tune);
    if (rc) return rc;
  }
  return MHS_OK;
}

// A batch of requests of this unit, each in one pass.  Requests in apply
// mode and the rest must not be mixed (the output stage's block size).
// upload: 1 copies the descriptors to desc and launches, 0 launches with
// the descriptors already there (a batch bound before stream capture), 2
// only copies them.
template <int P, int KC, class RF>
int run_batch(const mhs_request* const* rs, const Layout* L, int n, void* desc, int upload,
              cudaStream_t st, unsigned long long* census, const Tune& tune) {
  std::vector<Pass> ps((size_t)n);
  for (int i = 0; i < n; ++i) {
    if (L[i].chunk < rs[i]->n_obs) return fail(MHS_ERR_WORKSPACE, "batched request %d needs one pass", i);
    if ((rs[i]->slip != nullptr) != (rs[0]->slip != nullptr))
      return fail(MHS_ERR_ARG, "a batch mixes apply-mode and matrix requests");
    ps[i] = Pass{rs[i], &L[i], 0, rs[i]->n_obs, true};
  }
  if (upload == 2) {
    std::vector<char> host;
    build_descs<P, KC>(ps.data(), n, tune, host);
    MHS_CUDA_TRY(cudaMemcpyAsync(desc, host.data(), host.size(), cudaMemcpyHostToDevice, st));
    return MHS_OK;
  }
  return run_passes<P, KC, RF>(ps.data(), n, desc, upload == 1, st, census, tune);
}

// ---------------------------------------------------- per-term diagnostics
// One source, n observers, one thread per observer: a single influence term
// exactly as the pipeline evaluates it.  term 0 direct (H + E or U), 1 image
// R-family, 2 image Q-family, 3 folded image (mirror + Boussinesq); with
// H, 4 and 5 the fold's surface load at (x, y, 0) (K x 3 values), from the
// sigma_zz row and from the full H.
// out per observer: K x C tensor values, then K blob weights (direct only).
template <int P, int WANT>
__global__ void k_terms(int term, int n, const double* __restrict__ obs,
                        const double* __restrict__ tri, double mu, double lam, double eps,
                        const double* __restrict__ coef, double* __restrict__ out) {
  constexpr int K = n_nodes(P);
  constexpr int C = (WANT & W_U) ? 9 : 27;
  __shared__ Frame f, fi;
  __shared__ SmemRules<P> rd, ri;
  __shared__ double sG[G_SIZE];
  if (threadIdx.x == 0) {
    double ti[9];
    for (int i = 0; i < 9; ++i) ti[i] = (i % 3 == 2) ? -tri[i] : tri[i];
    make_frame(tri, f);
    make_frame(ti, fi);
    build_basis_products(fi, sG);
  }
  __syncthreads();
  rd.build(f, threadIdx.x, blockDim.x);
  ri.build(fi, threadIdx.x, blockDim.x);
  __syncthreads();
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  const double x[3] = {obs[3 * o], obs[3 * o + 1], obs[3 * o + 2]};
  const Material m = make_material(mu, lam);
  const ImageCoef ic = image_coef_view(coef);
  double A[K * C] = {}, E[K] = {};
  for (int k = 0; k < K; ++k) E[k] = 0.0;
  if (term == 0) {
    if (WANT & W_U) direct_eval<P, W_U>(f, rd.r12(), rd.r8(), x, eps, m, A, nullptr, nullptr);
    else direct_eval<P, W_H | W_E>(f, rd.r12(), rd.r8(), x, eps, m, nullptr, A, E);
  } else if (term == 1) {
    image_r_eval<P, WANT>(fi, sG, f.n, ri.r12(), ri.r8(), x, eps, m, ic, A, A);
  } else if (term == 2) {
    double ti[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) ti[3 * i + j] = fi.v[i][j];
    const int nq = q_gauss_order(x, ti, eps, f.L, P);
    QRuleFly<P> r{&f, nq};
    image_q_eval<P, WANT>(r, f.n, x, eps, m, ic, A, A);
  } else if (term >= 4) {
    if (!(WANT & W_U)) {
      if (term == 4) {
        SurfaceLoadConsts c;
        surface_load_consts(f, eps, m, c);
        fold_surface_load_fast<P>(f, rd.r12(), rd.r8(), c, x[0], x[1], eps, A);
      } else {
        fold_surface_load<P>(f, rd.r12(), rd.r8(), x[0], x[1], eps, m, A);
      }
    }
  } else {
    double Mv[K * C] = {}, Bq[K * C] = {};
    if (WANT & W_U) direct_eval<P, W_U>(fi, ri.r12(), ri.r8(), x, eps, m, Mv, nullptr, nullptr);
    else direct_eval<P, W_H>(fi, ri.r12(), ri.r8(), x, eps, m, nullptr, Mv, nullptr);
    fold_boussinesq_scalar<P, !(WANT & W_U)>(f, rd.r12(), rd.r8(), tri, x, eps, m, d_glx, d_glw, Bq);
    for (int i = 0; i < K * C; ++i) A[i] = Mv[i] * mirror_slip_sign(i % 3) + Bq[i];
  }
  for (int i = 0; i < K * C; ++i) out[o * (K * C + K) + i] = A[i];
  for (int k = 0; k < K; ++k) out[o * (K * C + K) + K * C + k] = E[k];
}

template <int P>
int debug_terms(int term, int want_u, int n, const double* obs, const double* tri, double mu,
                double lam, double eps, double* coef, double* out, cudaStream_t st) {
  k_coef1<<<(MHS_Q_NDDG + 255) / 256, 256, 0, st>>>(mu, lam, coef);
  const int nb = (n + 63) / 64;
  if (want_u) k_terms<P, W_U><<<nb, 64, 0, st>>>(term, n, obs, tri, mu, lam, eps, coef, out);
  else k_terms<P, W_H><<<nb, 64, 0, st>>>(term, n, obs, tri, mu, lam, eps, coef, out);
  MHS_CUDA_TRY(cudaGetLastError());
  return MHS_OK;
}

// ------------------------------------------------------------ full space
// The full-space single-triangle API (mhs/fullspace/api.py:90-175): the
// nodal influence tensors of one triangle at n observers, one thread per
// observer -- slip source U (K x 9), total stress H (K x 27), eigenstress
// weight E (K); force source G (K x 9), S (K x 27) -- for the kernels in
// `want`, with the closed form within near_l element lengths (D_STAR: the
// hybrid far field; +inf: analytic; -1: quadrature everywhere).
struct FsTri {
  double v[9];
};
static_assert(int(MHS_FS_U) == int(W_U) && int(MHS_FS_H) == int(W_H) &&
                  int(MHS_FS_E) == int(W_E) && int(MHS_FS_G) == int(W_G) &&
                  int(MHS_FS_S) == int(W_S),
              "the ABI's kernel flags are the engine's");

template <int P>
__global__ void __launch_bounds__(64)
k_fullspace(int want, double near_l, int64_t n, const double* __restrict__ obs, FsTri tri,
            double mu, double lam, double eps, double* U, double* H, double* E, double* G,
            double* S) {
  constexpr int K = n_nodes(P);
  __shared__ Frame f;
  __shared__ SmemRules<P> rd;
  if (threadIdx.x == 0) make_frame(tri.v, f);
  __syncthreads();
  rd.build(f, threadIdx.x, blockDim.x);
  __syncthreads();
  const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  const double x[3] = {obs[3 * o], obs[3 * o + 1], obs[3 * o + 2]};
  const Material m = make_material(mu, lam);
  const QuadRule r12 = rd.r12(), r8 = rd.r8();
  if (want & W_U) direct_eval<P, W_U>(f, r12, r8, x, eps, m, U + o * K * 9, nullptr, nullptr, near_l);
  if ((want & W_H) && (want & W_E))
    direct_eval<P, W_H | W_E>(f, r12, r8, x, eps, m, nullptr, H + o * K * 27, E + o * K, near_l);
  else if (want & W_H)
    direct_eval<P, W_H>(f, r12, r8, x, eps, m, nullptr, H + o * K * 27, nullptr, near_l);
  else if (want & W_E)
    direct_eval<P, W_E>(f, r12, r8, x, eps, m, nullptr, nullptr, E + o * K, near_l);
  if ((want & W_G) && (want & W_S))
    force_eval<P, W_G | W_S>(f, r12, r8, x, eps, m, G + o * K * 9, S + o * K * 27, near_l);
  else if (want & W_G)
    force_eval<P, W_G>(f, r12, r8, x, eps, m, G + o * K * 9, nullptr, near_l);
  else if (want & W_S)
    force_eval<P, W_S>(f, r12, r8, x, eps, m, nullptr, S + o * K * 27, near_l);
}

template <int P>
int fullspace_run(int want, double near_l, int64_t n, const double* obs, const double* tri,
                  double mu, double lam, double eps, double* U, double* H, double* E, double* G,
                  double* S, cudaStream_t st) {
  if (n <= 0) return MHS_OK;
  FsTri t;
  for (int i = 0; i < 9; ++i) t.v[i] = tri[i];
  const int64_t nb = (n + 63) / 64;
  if (nb > INT32_MAX) return fail(MHS_ERR_ARG, "fullspace: too many observers");
  k_fullspace<P><<<(unsigned)nb, 64, 0, st>>>(want, near_l, n, obs, t, mu, lam, eps, U, H, E, G, S);
  count_kernels(1);
  MHS_CUDA_TRY(cudaGetLastError());
  return MHS_OK;
}

}  // namespace
}  // namespace pipe
}  // namespace mhs
