// Declarations shared by the host translation unit (mhs_b200.cu, the C ABI)
// and the kernel units (unit.cu, compiled once per order / readout /
// precision so the library builds in parallel).
//
// A request runs as a short pipeline on the caller's stream, per chunk of
// observers (kernels.cuh):
//   k_coef   per-material image coefficients (once per request)
//   k_prep   per-source frames, reflected frames, basis products, fold data
//   k_pair   one thread per (observer, source): direct term + image R-family
//   k_imageq one thread per (observer, source): image Q-family
//   k_band   per straddling source, the ordered list of band receivers
//   k_fold*  the folded image of every band pair
//   k_final  one thread per (observer, output column): eigenstress,
//            traction / interaction contraction, continuous-layout gather,
//            and the store in the caller's layout
// Per-pair tensors travel between stages in an element-major scratch table
// (workspace), so every stage writes disjoint rows and no result depends on
// atomics or scheduling order.
#pragma once

#include <cuda_runtime.h>

#include <stddef.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/mhs_b200.h"
#include "engine_fold.cuh"
#include "host_prep.h"

namespace mhs {

static_assert(cst::SMALL_U_OVER_RHO_SQ == cst::SMALL_U_OVER_RHO * cst::SMALL_U_OVER_RHO &&
                  cst::SERIES_U_OVER_RHO_SQ == cst::SERIES_U_OVER_RHO * cst::SERIES_U_OVER_RHO,
              "edge-regime thresholds and their squares disagree");

namespace pipe {

struct SrcPrep {
  Frame f;        // element
  Frame fi;       // reflected element (image R-family and fold mirror)
  double eps;
  double centre[2], r_f, diam;
  int straddle;   // folded (fold requested and the source reaches the band)
  int pad;
};

constexpr int TB = 128;          // threads per block for pair-parallel kernels
// The mixed form's far field: the pair kernel takes the closed-form near
// field only within MIXED_NEAR_L element lengths (sqrt(|x - c|^2 + eps^2)
// <= MIXED_NEAR_L * L), a float MIXED_GAUSS_N x MIXED_GAUSS_N product rule
// out to D_STAR L and a float MIXED_GAUSS_N_FAR x MIXED_GAUSS_N_FAR rule
// beyond (the fold's far surface loads, all beyond D_STAR L, take the
// latter).  At those distances these orders already resolve the kernels:
// at P2 the 8 x 8 rule at 3 L and the 6 x 6 rule at 10 L agree with a
// 40 x 40 rule to 2e-13 of the largest entry, far below float rounding.
// The FP64 form keeps mhs's rules (12 x 12, 8 x 8 beyond D_STAR_DISTANT L).
constexpr double MIXED_NEAR_L = 3.0;
constexpr int MIXED_GAUSS_N = 8;
constexpr int MIXED_GAUSS_N_FAR = 6;
constexpr int QFLOOR = cst::IMAGE_Q_GAUSS_MIN;

enum : int { KD_DISP = 0, KD_HE = 1, KD_E = 2 };   // what the stages compute

MHS_FI constexpr int kind_class(int kind) {
  return kind == MHS_DISP ? KD_DISP : (kind == MHS_EIGENSTRESS ? KD_E : KD_HE);
}
MHS_FI constexpr int comps_of(int kc) { return kc == KD_DISP ? 9 : (kc == KD_HE ? 27 : 0); }
// Scratch row per (observer, source, node): tensor comps, phi, phi_mirror.
MHS_FI constexpr int row_of(int kc) { return comps_of(kc) + 2; }

inline size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// ----------------------------------------------------- request descriptors
// What the output stage needs of one pass (one observer chunk of one
// request).
struct FinalArgs {
  int kind, subtract, out_f32, n_a, n_b;
  int64_t lo, n_chunk, n_src, n_obs, n_dof;
  const double* normals;
  const double* rec_basis;
  const double* src_basis;
  const int32_t* col_ptr;
  const int32_t* col_ent;
  double mu, lam;
  void* out;
  const double* slip;   // apply mode: (n_dof, n_s) slip; out is (n_obs, nv / n_s)
};

// One pass of one request as the batched stage kernels read it: a group of
// passes of the same (order, readout, precision) runs each stage in one
// launch, every block finding its pass by the prefix of block counts.
struct ReqDesc {
  FinalArgs fa;
  const double* obs;
  const double* tris;
  const double* eps;
  SrcPrep* prep;
  double* G;
  double* coef;
  double* T;
  double* Wimg;   // the image R-family's weighted tables per pair and node
  int* status;
  int fold, pad;
};

// Stages' block counts per pass, as exclusive prefixes over the group
// (n + 1 entries each), following the descriptors in device memory.
enum : int { OFF_COEF = 0, OFF_PREP = 1, OFF_PAIR = 2, OFF_FINAL = 3, N_OFF = 4 };

MHS_FI int find_req(const long long* off, int n, long long b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

inline size_t desc_bytes(int n) {
  return align_up(sizeof(ReqDesc) * (size_t)n) + sizeof(long long) * (size_t)N_OFF * (n + 1);
}

// Launch shapes the autotuner picks per (order, readout, precision) and
// device: threads per block of the pair kernels (observer tile) and of the
// output stage (column tile), and the grid multipliers (blocks per SM x
// this factor) of the fold's grid-stride load kernels.
struct Tune {
  int pair_tb = 128;
  int final_tb = 128;
  int far_mult = 4;
  int near_mult = 4;
};

// Workspace carve-up for a chunk of `chunk` observers plus `fold_bytes`
// for the fold's plan, pair batches and node waves.
struct Layout {
  size_t status, desc, coef, prep, G, cnt, list, T, Wimg, fold, fold_bytes, total;
  int64_t chunk;
};

// Weighted-table entries per node of the image R-family (the same at every
// order: its spec's constant-slip degrees do not depend on the order).
constexpr int IMG_NW = SpecImg<0>::spec.w_off[NS];
static_assert(IMG_NW == SpecImg<1>::spec.w_off[NS] && IMG_NW == SpecImg<2>::spec.w_off[NS],
              "image tables per node independent of the order");

inline Layout plan(const mhs_request* r, int64_t chunk, size_t fold_bytes = 0) {
  const int kc = kind_class(r->kind);
  const int K = n_nodes(r->order);
  Layout L;
  size_t off = 0;
  L.status = off; off = align_up(off + 256);
  L.desc = off; off = align_up(off + desc_bytes(1));
  L.coef = off; off = align_up(off + sizeof(double) * IMAGE_COEF_SIZE);
  L.prep = off; off = align_up(off + sizeof(SrcPrep) * (size_t)r->n_src);
  L.G = off;
  if (kc != KD_E) off = align_up(off + sizeof(double) * G_SIZE * (size_t)r->n_src);
  L.cnt = off; off = align_up(off + sizeof(int) * (size_t)r->n_src);
  L.list = off; off = align_up(off + sizeof(int) * (size_t)r->n_src * (size_t)chunk);
  L.T = off; off = align_up(off + sizeof(double) * (size_t)chunk * r->n_src * K * row_of(kc));
  L.Wimg = off;
  if (kc != KD_E) off = align_up(off + sizeof(double) * (size_t)chunk * r->n_src * K * IMG_NW);
  L.fold = off; off = align_up(off + fold_bytes);
  L.fold_bytes = fold_bytes;
  L.total = off;
  L.chunk = chunk;
  return L;
}

// Fold region: none without the fold or for the blob-only readout; else at
// least FOLD_MIN_BYTES, at most the request's useful size (`cap`, less for
// small requests), otherwise half of what the workspace holds beyond one
// observer row.  A request assembled alone takes up to FOLD_GOOD_BYTES:
// bigger node waves leave fewer wave tails (on the 2,400-triangle
// interaction the fold takes 207 ms with 4 GiB against 209 ms with 2 GiB);
// a request of a batch takes up to FOLD_BATCH_BYTES, so that batches keep
// many requests per pass.
constexpr size_t FOLD_MIN_BYTES = size_t(8) << 20;
constexpr size_t FOLD_GOOD_BYTES = size_t(4) << 30;
constexpr size_t FOLD_BATCH_BYTES = size_t(2) << 30;

inline size_t fold_good_bytes(const mhs_request* r, size_t cap = FOLD_GOOD_BYTES) {
  if (!r->fold || kind_class(r->kind) == KD_E) return 0;
  const double want = 4096.0 * (double)r->n_obs * (double)r->n_src;
  if (want >= (double)cap) return cap;
  return std::max<size_t>(FOLD_MIN_BYTES * 8, align_up((size_t)want));
}

inline size_t fold_bytes_for(const mhs_request* r, size_t workspace_bytes) {
  const size_t good = fold_good_bytes(r);
  if (!good) return 0;
  const size_t row = plan(r, 1, 0).total;
  const size_t half = workspace_bytes > row ? (workspace_bytes - row) / 2 : 0;
  return align_up(std::min(good, std::max(FOLD_MIN_BYTES, half)));
}

// ------------------------------------------- services of the host unit
// Error text of this thread (mhs_last_error); returns `code`.
int fail(int code, const char* fmt, ...);
// Stage timing: whether it is on, and the record of one stage's events.
bool prof_enabled();
void prof_record(int stage, cudaEvent_t a, cudaEvent_t b);
// Count of kernels queued (mhs_kernel_count).
void count_kernels(int n);

#define MHS_CUDA_TRY(x)                                                                     \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess)                                                                  \
      return ::mhs::pipe::fail(MHS_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_));          \
  } while (0)

// Brackets one stage's launches with CUDA events on the request's stream
// while stage timing is on.
struct StageTimer {
  int stage;
  cudaStream_t st;
  cudaEvent_t a = nullptr, b = nullptr;
  StageTimer(int s, cudaStream_t stream) : stage(s), st(stream) {
    if (prof_enabled()) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, st);
    }
  }
  ~StageTimer() {
    if (a) {
      cudaEventRecord(b, st);
      prof_record(stage, a, b);
    }
  }
};

// ------------------------------------------------ kernel unit entry points
// Each kernel unit holds its own copy of the Gauss-Legendre table (device
// globals are per translation unit): `init` copies it in on the current
// device; `run` queues one request's pipeline.  census: device counters
// of the fold's work units, or null.
using UnitInit = int (*)(const double* glx, const double* glw);
using UnitRun = int (*)(const mhs_request* r, cudaStream_t st, const Layout& L,
                        unsigned long long* census, const Tune& tune);
// A batch: n requests of this unit, request i on its own workspace part with
// layout L[i] (one pass, all its observers); descriptors at desc (device,
// desc_bytes(n), already holding what batch_descs wrote when upload = 0).
using UnitBatch = int (*)(const mhs_request* const* r, const Layout* L, int n, void* desc,
                          int upload, cudaStream_t st, unsigned long long* census,
                          const Tune& tune);
using UnitTerms = int (*)(int term, int want_u, int n, const double* obs, const double* tri,
                          double mu, double lam, double eps, double* coef, double* out,
                          cudaStream_t st);
using UnitFullspace = int (*)(int want, double near_l, int64_t n, const double* obs,
                              const double* tri, double mu, double lam, double eps, double* U,
                              double* H, double* E, double* G, double* S, cudaStream_t st);

#define MHS_UNIT_LIST(X) \
  X(0, 0, 0) X(0, 0, 1) X(0, 1, 0) X(0, 1, 1) X(0, 2, 0) X(0, 2, 1) \
  X(1, 0, 0) X(1, 0, 1) X(1, 1, 0) X(1, 1, 1) X(1, 2, 0) X(1, 2, 1) \
  X(2, 0, 0) X(2, 0, 1) X(2, 1, 0) X(2, 1, 1) X(2, 2, 0) X(2, 2, 1)

#define MHS_UNIT_DECL(P, KC, RF)                                                     \
  int unit_init_##P##_##KC##_##RF(const double* glx, const double* glw);             \
  int unit_run_##P##_##KC##_##RF(const mhs_request* r, cudaStream_t st, const Layout& L, \
                                 unsigned long long* census, const Tune& tune);      \
  int unit_batch_##P##_##KC##_##RF(const mhs_request* const* r, const Layout* L, int n,  \
                                   void* desc, int upload, cudaStream_t st,          \
                                   unsigned long long* census, const Tune& tune);
MHS_UNIT_LIST(MHS_UNIT_DECL)
#undef MHS_UNIT_DECL

#define MHS_TERMS_DECL(P)                                                                \
  int unit_init_terms_##P(const double* glx, const double* glw);                         \
  int unit_terms_##P(int term, int want_u, int n, const double* obs, const double* tri,  \
                     double mu, double lam, double eps, double* coef, double* out,       \
                     cudaStream_t st);                                                   \
  int unit_fullspace_##P(int want, double near_l, int64_t n, const double* obs,          \
                         const double* tri, double mu, double lam, double eps, double* U, \
                         double* H, double* E, double* G, double* S, cudaStream_t st);
MHS_TERMS_DECL(0)
MHS_TERMS_DECL(1)
MHS_TERMS_DECL(2)
#undef MHS_TERMS_DECL

}  // namespace pipe
}  // namespace mhs
