// Host unit of the B200 Green's-function assembler: the C ABI
// (include/mhs_b200.h), request checks, the per-device tables, stage
// timing, the fold census counters and the allocation-free scratch array.
// The kernels live in the kernel units (unit.cu, one per order / readout /
// precision); this unit dispatches to them.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "host_prep.h"
#include "pipeline.cuh"

using namespace mhs;
using namespace mhs::pipe;

namespace mhs {
namespace pipe {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

// ------------------------------------------------------ stage timing
// When enabled, each stage launch is bracketed by CUDA events on the
// request's stream; mhs_profile_read sums them per stage.
struct ProfRec {
  int stage;
  cudaEvent_t a, b;
};
std::mutex g_prof_mu;
std::vector<ProfRec> g_prof;
int g_prof_on = 0;

std::atomic<unsigned long long> g_kernels{0};
void count_kernels(int n) { g_kernels.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

bool prof_enabled() { return __atomic_load_n(&g_prof_on, __ATOMIC_RELAXED) != 0; }

void prof_record(int stage, cudaEvent_t a, cudaEvent_t b) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof.push_back({stage, a, b});
}

}  // namespace pipe
}  // namespace mhs

namespace {

#define CUDA_TRY MHS_CUDA_TRY

// ------------------------------------------------------ kernel units
struct UnitEntry {
  int P, KC, RF;
  UnitInit init;
  UnitRun run;
  UnitBatch batch;
};
#define MHS_UNIT_ENTRY(P, KC, RF) \
  {P, KC, RF, unit_init_##P##_##KC##_##RF, unit_run_##P##_##KC##_##RF, unit_batch_##P##_##KC##_##RF},
const UnitEntry g_units[] = {MHS_UNIT_LIST(MHS_UNIT_ENTRY)};
#undef MHS_UNIT_ENTRY
const UnitInit g_terms_init[3] = {unit_init_terms_0, unit_init_terms_1, unit_init_terms_2};
const UnitTerms g_terms[3] = {unit_terms_0, unit_terms_1, unit_terms_2};
const UnitFullspace g_fullspace[3] = {unit_fullspace_0, unit_fullspace_1, unit_fullspace_2};

std::mutex g_init_mu;
std::vector<int> g_init_done;

// Gauss-Legendre tables of every unit on the current device, once.
int ensure_device_tables() {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_init_mu);
  if ((int)g_init_done.size() <= dev) g_init_done.resize(dev + 1, 0);
  if (g_init_done[dev]) return MHS_OK;
  std::vector<double> x(GL_TABLE), w(GL_TABLE);
  gauss_table(x.data(), w.data());
  for (const UnitEntry& u : g_units) {
    const int rc = u.init(x.data(), w.data());
    if (rc) return rc;
  }
  for (UnitInit f : g_terms_init) {
    const int rc = f(x.data(), w.data());
    if (rc) return rc;
  }
  g_init_done[dev] = 1;
  return MHS_OK;
}

// Independent FMA chains: the FP64 (or FP32) issue ceiling of the device.
template <class R>
__device__ __forceinline__ void fma_chains(R* out, int iters, R b, R c) {
  R a0 = R(threadIdx.x) * R(1e-9), a1 = a0 + R(1e-9), a2 = a0 + R(2e-9), a3 = a0 + R(3e-9);
  R a4 = a0 + R(4e-9), a5 = a0 + R(5e-9), a6 = a0 + R(6e-9), a7 = a0 + R(7e-9);
  for (int i = 0; i < iters; ++i) {
    a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
    a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
  }
  const R s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == R(-1)) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
__global__ void k_fma_peak_f64(double* out, int iters, double b, double c) {
  fma_chains<double>(out, iters, b, c);
}
__global__ void k_fma_peak_f32(float* out, int iters, float b, float c) {
  fma_chains<float>(out, iters, b, c);
}

int check_request(const mhs_request* r) {
  if (!r) return fail(MHS_ERR_ARG, "null request");
  if (r->kind < MHS_DISP || r->kind > MHS_INTERACTION) return fail(MHS_ERR_ARG, "bad kind %d", r->kind);
  if (r->order < 0 || r->order > 2) return fail(MHS_ERR_ARG, "order must be 0, 1 or 2");
  if (r->n_obs <= 0 || r->n_src <= 0) return fail(MHS_ERR_ARG, "empty request");
  if (r->n_src > INT32_MAX / 6) return fail(MHS_ERR_ARG, "n_src %lld above %d", (long long)r->n_src, INT32_MAX / 6);
  if (!r->obs || !r->tris || !r->eps || !r->out) return fail(MHS_ERR_ARG, "null array");
  if (!(r->mu > 0.0)) return fail(MHS_ERR_ARG, "mu must be positive");
  if ((r->kind == MHS_TRACTION || r->kind == MHS_INTERACTION) && !r->normals)
    return fail(MHS_ERR_ARG, "normals required");
  if (r->kind == MHS_INTERACTION &&
      (!r->rec_basis || !r->src_basis || r->n_a < 1 || r->n_a > 3 || r->n_b < 1 || r->n_b > 3))
    return fail(MHS_ERR_ARG, "interaction bases");
  if (r->ids && (r->order != 2 || !r->col_ptr || !r->col_ent || r->n_cols <= 0))
    return fail(MHS_ERR_ARG, "continuous layout needs order 2 and a column plan");
  if (r->precision != MHS_FP64 && r->precision != MHS_MIXED) return fail(MHS_ERR_ARG, "precision");
  return MHS_OK;
}

// ------------------------------------------------------ fold census
__device__ unsigned long long g_census[MHS_CENSUS_N];
std::atomic<int> g_census_on{0};

// Queue the request on the unit of its (order, readout, precision).
// Unit of a request: its (order, readout class, precision).
const UnitEntry* unit_of(const mhs_request* r) {
  const int kc = kind_class(r->kind);
  const int rf = r->precision == MHS_MIXED ? 1 : 0;
  for (const UnitEntry& u : g_units)
    if (u.P == r->order && u.KC == kc && u.RF == rf) return &u;
  return nullptr;
}

// ------------------------------------------------------ launch shapes
// Per device and unit, the launch shapes in use: defaults until the
// autotuner (mhs_autotune) or the caller (mhs_set_tune) sets them.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, Tune> g_tune;

int tune_for(const mhs_request* r, Tune* t) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find({dev, r->order, kind_class(r->kind), r->precision});
  *t = it == g_tune.end() ? Tune{} : it->second;
  return MHS_OK;
}

int set_tune(const mhs_request* r, const Tune& t) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[{dev, r->order, kind_class(r->kind), r->precision}] = t;
  return MHS_OK;
}

unsigned long long* census_ptr() {
  unsigned long long* census = nullptr;
  if (g_census_on.load(std::memory_order_relaxed) &&
      cudaGetSymbolAddress((void**)&census, g_census) != cudaSuccess)
    census = nullptr;
  return census;
}

// Queue the request on the unit of its (order, readout, precision).
int run_request(const mhs_request* r, cudaStream_t st, const Layout& L) {
  const UnitEntry* u = unit_of(r);
  if (!u) return fail(MHS_ERR_ARG, "no kernel unit for order %d", r->order);
  Tune t;
  const int rc = tune_for(r, &t);
  if (rc) return rc;
  return u->run(r, st, L, census_ptr(), t);
}

// Layout of the largest observer chunk whose workspace fits `bytes`
// (plan() is monotone in the chunk), beside the fold region the workspace
// size affords; chunk 0 when not even one row fits.
Layout fit_layout(const mhs_request* r, size_t bytes) {
  const size_t fb = fold_bytes_for(r, bytes);
  Layout none = plan(r, 1, fb);
  if (none.total > bytes) {
    none.chunk = 0;
    return none;
  }
  int64_t lo = 1, hi = std::min<int64_t>(r->n_obs, 65535);
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo + 1) / 2;
    if (plan(r, mid, fb).total <= bytes) lo = mid;
    else hi = mid - 1;
  }
  return plan(r, lo, fb);
}

// Per-chunk pair tables (the pair table and the image tables) of the good
// workspace size: the 2,400-triangle interaction fits in one chunk.
constexpr size_t GOOD_T_BYTES = size_t(4) << 30;

// ------------------------------------------- allocation-free scratch
// Scratch of mhs_assemble_noalloc: one file-scope device array that every
// device loading this library holds until the process exits.  Host code
// never dereferences the symbol; it passes the device address that
// cudaGetSymbolAddress returns, looked up once per device.
__device__ __align__(256) unsigned char g_noalloc_scratch[MHS_NOALLOC_SCRATCH_BYTES];
std::mutex g_noalloc_mu;
std::vector<void*> g_noalloc_ptr;

int noalloc_scratch(void** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if ((int)g_noalloc_ptr.size() <= dev) g_noalloc_ptr.resize(dev + 1, nullptr);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(MHS_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return MHS_OK;
}

// ------------------------------------------------------------ batches
constexpr size_t BATCH_PASS_MAX = size_t(8) << 30;

}  // namespace

struct mhs_batch {
  struct Group {
    const UnitEntry* unit;
    std::vector<int> idx;       // requests of the group
    size_t desc_off;            // its descriptors in the arena
  };
  std::vector<mhs_request> reqs;
  std::vector<Layout> L;
  std::vector<size_t> ws_off;
  std::vector<Group> groups;
  size_t bytes = 0;
  char* arena = nullptr;
  cudaEvent_t done = nullptr;
  bool submitted = false;
};

extern "C" {

int mhs_workspace_bytes(const mhs_request* req, size_t* min_bytes, size_t* good_bytes) {
  int rc = check_request(req);
  if (rc) return rc;
  const size_t fgood = fold_good_bytes(req);
  const size_t fmin = fgood ? FOLD_MIN_BYTES : 0;
  const Layout one = plan(req, 1, 0);
  const size_t row = plan(req, 2, 0).total - one.total;
  int64_t chunk = std::min<int64_t>(req->n_obs, 65535);
  if (plan(req, chunk, 0).total - one.total > GOOD_T_BYTES && row > 0)
    chunk = std::max<int64_t>(1, (int64_t)(GOOD_T_BYTES / row));
  if (min_bytes) *min_bytes = plan(req, 1, fmin).total;
  if (good_bytes) *good_bytes = plan(req, chunk, fgood).total;
  return MHS_OK;
}

int mhs_assemble(const mhs_request* req, void* stream) {
  int rc = check_request(req);
  if (rc) return rc;
  rc = ensure_device_tables();
  if (rc) return rc;
  // largest chunk the workspace holds
  const Layout L = fit_layout(req, req->workspace ? req->workspace_bytes : 0);
  if (L.chunk == 0) {
    size_t mn = 0;
    mhs_workspace_bytes(req, &mn, nullptr);
    return fail(MHS_ERR_WORKSPACE, "workspace %zu bytes, need at least %zu", req->workspace_bytes,
                mn);
  }
  return run_request(req, (cudaStream_t)stream, L);
}

int mhs_assemble_noalloc(const mhs_request* req, void* stream, int* status_bits) {
  int rc = check_request(req);
  if (rc) return rc;
  rc = ensure_device_tables();
  if (rc) return rc;
  void* scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  const size_t cap = MHS_NOALLOC_SCRATCH_BYTES;
  const Layout L = fit_layout(req, cap);
  if (L.chunk == 0)
    return fail(MHS_ERR_WORKSPACE,
                "request needs %zu bytes of scratch for one observer row, above the %zu-byte "
                "array of the allocation-free entry point (MHS_NOALLOC_SCRATCH_BYTES); pass "
                "fewer sources per call or use mhs_assemble with a caller workspace",
                L.total, cap);
  mhs_request r = *req;
  r.workspace = scratch;
  r.workspace_bytes = cap;
  cudaStream_t st = (cudaStream_t)stream;
  rc = run_request(&r, st, L);
  if (rc || !status_bits) return rc;
  CUDA_TRY(cudaMemcpyAsync(status_bits, (char*)scratch + L.status, sizeof(int),
                           cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return MHS_OK;
}

int mhs_read_status(void* workspace, void* stream, int* bits) {
  cudaStream_t st = (cudaStream_t)stream;
  if (!workspace) {  // the allocation-free entry point's array on this device
    const int rc = noalloc_scratch(&workspace);
    if (rc) return rc;
  }
  int h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, workspace, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (h) CUDA_TRY(cudaMemsetAsync(workspace, 0, sizeof(int), st));
  if (bits) *bits = h;
  return MHS_OK;
}

int mhs_column_plan(const int64_t* ids, int64_t n_src, int64_t n_cols, int32_t* col_ptr,
                    int32_t* col_ent) {
  if (!ids || !col_ptr || !col_ent || n_src <= 0 || n_cols <= 0) return fail(MHS_ERR_ARG, "column plan args");
  std::vector<int32_t> count(n_cols + 1, 0);
  for (int64_t i = 0; i < n_src * 6; ++i) {
    if (ids[i] < 0 || ids[i] >= n_cols) return fail(MHS_ERR_ARG, "ids[%lld] out of range", (long long)i);
    count[ids[i] + 1]++;
  }
  for (int64_t c = 0; c < n_cols; ++c) count[c + 1] += count[c];
  for (int64_t c = 0; c <= n_cols; ++c) col_ptr[c] = count[c];
  for (int64_t i = 0; i < n_src * 6; ++i) col_ent[count[ids[i]]++] = (int32_t)i;  // ascending i
  return MHS_OK;
}

int mhs_debug_terms(int order, int term, int want_u, int n, const double* obs, const double* tri,
                    double mu, double lam, double eps, double* coef_scratch, double* out,
                    void* stream) {
  int rc = ensure_device_tables();
  if (rc) return rc;
  if (n <= 0 || term < 0 || term > 5 || (term >= 4 && want_u) || !obs || !tri || !coef_scratch ||
      !out)
    return fail(MHS_ERR_ARG, "debug_terms args");
  if (order < 0 || order > 2) return fail(MHS_ERR_ARG, "order");
  return g_terms[order](term, want_u, n, obs, tri, mu, lam, eps, coef_scratch, out,
                        (cudaStream_t)stream);
}

int mhs_fullspace_influence(const mhs_fullspace_request* q, void* stream) {
  if (!q) return fail(MHS_ERR_ARG, "fullspace: null request");
  if (q->order < 0 || q->order > 2) return fail(MHS_ERR_ARG, "fullspace: order must be 0, 1 or 2");
  const int all = MHS_FS_U | MHS_FS_H | MHS_FS_E | MHS_FS_G | MHS_FS_S;
  if (q->want == 0 || (q->want & ~all)) return fail(MHS_ERR_ARG, "fullspace: want");
  if (q->n_obs < 0 || (q->n_obs > 0 && !q->obs)) return fail(MHS_ERR_ARG, "fullspace: obs");
  if (((q->want & MHS_FS_U) && !q->U) || ((q->want & MHS_FS_H) && !q->H) ||
      ((q->want & MHS_FS_E) && !q->E) || ((q->want & MHS_FS_G) && !q->G) ||
      ((q->want & MHS_FS_S) && !q->S))
    return fail(MHS_ERR_ARG, "fullspace: an output of `want` is NULL");
  if (!(q->mu > 0.0) || !(q->nu > -1.0 && q->nu < 0.5) || !(q->eps >= 0.0))
    return fail(MHS_ERR_ARG, "fullspace: mu > 0, -1 < nu < 1/2, eps >= 0");
  double near_l;
  switch (q->far_field) {
    case MHS_FAR_HYBRID: near_l = cst::D_STAR; break;
    case MHS_FAR_ANALYTIC: near_l = INFINITY; break;
    case MHS_FAR_QUADRATURE: near_l = -1.0; break;
    default: return fail(MHS_ERR_ARG, "fullspace: far_field");
  }
  int rc = ensure_device_tables();
  if (rc) return rc;
  const double lam = 2.0 * q->mu * q->nu / (1.0 - 2.0 * q->nu);
  return g_fullspace[q->order](q->want, near_l, q->n_obs, q->obs, q->tri, q->mu, lam, q->eps,
                               q->U, q->H, q->E, q->G, q->S, (cudaStream_t)stream);
}

int mhs_census_enable(int on) {
  if (on) {
    const unsigned long long zero[MHS_CENSUS_N] = {};
    if (cudaMemcpyToSymbol(g_census, zero, sizeof(zero)) != cudaSuccess)
      return fail(MHS_ERR_CUDA, "census: clearing the counters failed");
  }
  g_census_on.store(on ? 1 : 0, std::memory_order_relaxed);
  return MHS_OK;
}

int mhs_census_read(unsigned long long* counts) {
  if (!counts) return fail(MHS_ERR_ARG, "census: null counts");
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpyFromSymbol(counts, g_census, sizeof(unsigned long long) * MHS_CENSUS_N) != cudaSuccess)
    return fail(MHS_ERR_CUDA, "census: reading the counters failed");
  const unsigned long long zero[MHS_CENSUS_N] = {};
  if (cudaMemcpyToSymbol(g_census, zero, sizeof(zero)) != cudaSuccess)
    return fail(MHS_ERR_CUDA, "census: clearing the counters failed");
  return MHS_OK;
}

int mhs_profile_enable(int on) {
  __atomic_store_n(&g_prof_on, on ? 1 : 0, __ATOMIC_RELAXED);
  return MHS_OK;
}

int mhs_profile_read(double* ms, int* launches) {
  std::vector<ProfRec> recs;
  {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    recs.swap(g_prof);
  }
  for (int i = 0; i < MHS_N_STAGES; ++i) {
    if (ms) ms[i] = 0.0;
    if (launches) launches[i] = 0;
  }
  int rc = MHS_OK;
  for (auto& r : recs) {
    float t = 0.0f;
    if (cudaEventSynchronize(r.b) != cudaSuccess || cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess)
      rc = fail(MHS_ERR_CUDA, "profile event");
    if (ms) ms[r.stage] += t;
    if (launches) launches[r.stage] += 1;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  return rc;
}

int mhs_fp_peak(int fp64, int iters, double* tflops, void* stream) {
  int rc = ensure_device_tables();
  if (rc) return rc;
  int dev = 0, sms = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  cudaStream_t st = (cudaStream_t)stream;
  const int blocks = sms * 8, threads = 256;
  cudaEvent_t a, b;
  CUDA_TRY(cudaEventCreate(&a));
  CUDA_TRY(cudaEventCreate(&b));
  float ms = 0.0f;
  for (int rep = 0; rep < 2; ++rep) {  // first pass warms up
    CUDA_TRY(cudaEventRecord(a, st));
    if (fp64) k_fma_peak_f64<<<blocks, threads, 0, st>>>(nullptr, iters, 0.999999, 1e-7);
    else k_fma_peak_f32<<<blocks, threads, 0, st>>>(nullptr, iters, 0.999999f, 1e-7f);
    CUDA_TRY(cudaEventRecord(b, st));
    CUDA_TRY(cudaEventSynchronize(b));
    CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
  if (tflops) *tflops = flops / (ms * 1e-3) / 1e12;
  return MHS_OK;
}

int mhs_batch_pass_bytes(const mhs_request* r, size_t* bytes, size_t* limit) {
  if (!r || !bytes) return fail(MHS_ERR_ARG, "batch: null");
  mhs_request q = *r;
  q.workspace = nullptr;
  q.workspace_bytes = 0;
  int rc = check_request(&q);
  if (rc) return rc;
  *bytes = plan(&q, q.n_obs, fold_good_bytes(&q, FOLD_BATCH_BYTES)).total;
  if (limit) *limit = BATCH_PASS_MAX;
  return MHS_OK;
}

int mhs_batch_create(const mhs_request* reqs, int n, mhs_batch** out) {
  if (!out || !reqs || n < 1) return fail(MHS_ERR_ARG, "batch: empty or null");
  std::unique_ptr<mhs_batch> b(new mhs_batch);
  b->reqs.assign(reqs, reqs + n);
  size_t off = 0;
  for (int i = 0; i < n; ++i) {
    mhs_request& r = b->reqs[i];
    r.workspace = nullptr;
    r.workspace_bytes = 0;
    int rc = check_request(&r);
    if (rc) {
      char msg[512];
      snprintf(msg, sizeof(msg), "%s", mhs_last_error());
      return fail(rc, "batch request %d: %s", i, msg);
    }
    const Layout L = plan(&r, r.n_obs, fold_good_bytes(&r, FOLD_BATCH_BYTES));
    if (L.total > BATCH_PASS_MAX)
      return fail(MHS_ERR_WORKSPACE, "batch request %d needs %zu bytes of scratch for one pass, "
                  "above the batch limit of %zu; assemble it alone", i, L.total, BATCH_PASS_MAX);
    b->L.push_back(L);
    b->ws_off.push_back(off);
    off = align_up(off + L.total);
    const UnitEntry* u = unit_of(&r);
    if (!u) return fail(MHS_ERR_ARG, "batch request %d: no kernel unit", i);
    bool placed = false;
    for (auto& g : b->groups)
      if (g.unit == u && (b->reqs[g.idx[0]].slip != nullptr) == (r.slip != nullptr)) {
        g.idx.push_back(i);
        placed = true;
        break;
      }
    if (!placed) b->groups.push_back({u, {i}, 0});
  }
  for (auto& g : b->groups) {
    g.desc_off = off;
    off = align_up(off + desc_bytes((int)g.idx.size()));
  }
  b->bytes = off;
  *out = b.release();
  return MHS_OK;
}

int mhs_batch_workspace_bytes(const mhs_batch* b, size_t* bytes) {
  if (!b || !bytes) return fail(MHS_ERR_ARG, "batch: null");
  *bytes = b->bytes;
  return MHS_OK;
}

int mhs_batch_bind(mhs_batch* b, void* workspace, size_t bytes, void* stream) {
  if (!b || !workspace) return fail(MHS_ERR_ARG, "batch: null");
  if (bytes < b->bytes)
    return fail(MHS_ERR_WORKSPACE, "batch workspace %zu bytes, need %zu", bytes, b->bytes);
  int rc = ensure_device_tables();
  if (rc) return rc;
  b->arena = (char*)workspace;
  for (size_t i = 0; i < b->reqs.size(); ++i) {
    b->reqs[i].workspace = b->arena + b->ws_off[i];
    b->reqs[i].workspace_bytes = b->L[i].total;
  }
  cudaStream_t st = (cudaStream_t)stream;
  for (auto& g : b->groups) {
    std::vector<const mhs_request*> rp;
    std::vector<Layout> lp;
    for (int i : g.idx) {
      rp.push_back(&b->reqs[i]);
      lp.push_back(b->L[i]);
    }
    Tune t;
    rc = tune_for(rp[0], &t);
    if (rc) return rc;
    rc = g.unit->batch(rp.data(), lp.data(), (int)rp.size(), b->arena + g.desc_off, 2, st, nullptr,
                       t);
    if (rc) return rc;
  }
  if (!b->done) CUDA_TRY(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
  return MHS_OK;
}

int mhs_submit_batch(mhs_batch* b, void* stream) {
  if (!b || !b->arena) return fail(MHS_ERR_ARG, "batch: not bound to a workspace");
  cudaStream_t st = (cudaStream_t)stream;
  for (auto& g : b->groups) {
    std::vector<const mhs_request*> rp;
    std::vector<Layout> lp;
    for (int i : g.idx) {
      rp.push_back(&b->reqs[i]);
      lp.push_back(b->L[i]);
    }
    Tune t;
    int rc = tune_for(rp[0], &t);
    if (rc) return rc;
    rc = g.unit->batch(rp.data(), lp.data(), (int)rp.size(), b->arena + g.desc_off, 0, st,
                       census_ptr(), t);
    if (rc) return rc;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CUDA_TRY(cudaStreamIsCapturing(st, &cap));
  if (cap == cudaStreamCaptureStatusNone) {  // a captured submission is polled by its graph's stream
    CUDA_TRY(cudaEventRecord(b->done, st));
    b->submitted = true;
  }
  return MHS_OK;
}

int mhs_poll(mhs_batch* b, int* done, int* status_bits) {
  if (!b || !done) return fail(MHS_ERR_ARG, "batch: null");
  *done = 0;
  if (!b->submitted) return fail(MHS_ERR_ARG, "batch: nothing submitted");
  const cudaError_t e = cudaEventQuery(b->done);
  if (e == cudaErrorNotReady) return MHS_OK;
  if (e != cudaSuccess) return fail(MHS_ERR_CUDA, "batch event: %s", cudaGetErrorString(e));
  int bits = 0;
  for (size_t i = 0; i < b->reqs.size(); ++i) {
    int h = 0;
    CUDA_TRY(cudaMemcpy(&h, b->arena + b->ws_off[i] + b->L[i].status, sizeof(int),
                        cudaMemcpyDeviceToHost));
    bits |= h;
  }
  *done = 1;
  if (status_bits) *status_bits = bits;
  return MHS_OK;
}

int mhs_batch_destroy(mhs_batch* b) {
  if (!b) return MHS_OK;
  if (b->done) cudaEventDestroy(b->done);
  delete b;
  return MHS_OK;
}

int mhs_set_tune(const mhs_request* like, const mhs_tune* t) {
  if (!like || !t) return fail(MHS_ERR_ARG, "tune: null");
  auto ok = [](int v, int lo, int hi) { return v >= lo && v <= hi; };
  const bool pow2 = t->final_tb > 0 && (t->final_tb & (t->final_tb - 1)) == 0;
  if (!ok(t->pair_tb, 32, TB) || !ok(t->final_tb, 32, TB) || !pow2 || !ok(t->far_mult, 1, 16) ||
      !ok(t->near_mult, 1, 16))
    return fail(MHS_ERR_ARG, "tune out of range");
  return set_tune(like, Tune{t->pair_tb, t->final_tb, t->far_mult, t->near_mult});
}

int mhs_get_tune(const mhs_request* like, mhs_tune* t) {
  if (!like || !t) return fail(MHS_ERR_ARG, "tune: null");
  Tune v;
  const int rc = tune_for(like, &v);
  if (rc) return rc;
  *t = mhs_tune{v.pair_tb, v.final_tb, v.far_mult, v.near_mult};
  return MHS_OK;
}

int mhs_autotune(const mhs_request* sample, void* stream, mhs_tune* chosen, double* best_ms) {
  int rc = check_request(sample);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t a, b;
  CUDA_TRY(cudaEventCreate(&a));
  CUDA_TRY(cudaEventCreate(&b));
  Tune keep;
  rc = tune_for(sample, &keep);
  if (rc) return rc;
  Tune best = keep;
  double best_t = 1e300;
  rc = mhs_assemble(sample, stream);   // warm-up at the current shape
  for (int ptb : {64, 128})
    for (int ftb : {64, 128})
      for (int mult : {2, 4, 8}) {
        if (rc) break;
        const Tune t{ptb, ftb, mult, mult};
        set_tune(sample, t);
        CUDA_TRY(cudaEventRecord(a, st));
        rc = mhs_assemble(sample, stream);
        CUDA_TRY(cudaEventRecord(b, st));
        CUDA_TRY(cudaEventSynchronize(b));
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
        if (!rc && ms < best_t) {
          best_t = ms;
          best = t;
        }
      }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  set_tune(sample, rc ? keep : best);
  if (rc) return rc;
  if (chosen) *chosen = mhs_tune{best.pair_tb, best.final_tb, best.far_mult, best.near_mult};
  if (best_ms) *best_ms = best_t;
  return MHS_OK;
}

int mhs_kernel_count(unsigned long long* n) {
  if (!n) return fail(MHS_ERR_ARG, "null count");
  *n = g_kernels.exchange(0, std::memory_order_relaxed);
  return MHS_OK;
}

const char* mhs_last_error(void) { return g_err; }

const char* mhs_version(void) { return "mhs_b200 0.1.0"; }

}  // extern "C"

