// One kernel unit of the library.  The build compiles this file once per
// (order P, readout class KC, far-field type RF) with
//   -DMHS_UNIT_P=<0|1|2> -DMHS_UNIT_KC=<0 disp|1 stress+blob|2 blob> -DMHS_UNIT_RF=<0 double|1 float>
// and once per order with -DMHS_UNIT_TERMS=<P> for the per-term diagnostics
// and the full-space single-triangle API,
// so the units compile in parallel; the host unit (mhs_b200.cu) dispatches.
#include "kernels.cuh"

#define MHS_CAT4_(a, b, c, d) a##b##_##c##_##d
#define MHS_CAT4(a, b, c, d) MHS_CAT4_(a, b, c, d)
#define MHS_CAT2_(a, b) a##b
#define MHS_CAT2(a, b) MHS_CAT2_(a, b)

namespace mhs {
namespace pipe {

namespace {
int copy_tables(const double* glx, const double* glw) {
  MHS_CUDA_TRY(cudaMemcpyToSymbol(d_glx, glx, sizeof(double) * GL_TABLE));
  MHS_CUDA_TRY(cudaMemcpyToSymbol(d_glw, glw, sizeof(double) * GL_TABLE));
  return MHS_OK;
}
}  // namespace

#if defined(MHS_UNIT_TERMS)

int MHS_CAT2(unit_init_terms_, MHS_UNIT_TERMS)(const double* glx, const double* glw) {
  return copy_tables(glx, glw);
}

int MHS_CAT2(unit_terms_, MHS_UNIT_TERMS)(int term, int want_u, int n, const double* obs,
                                          const double* tri, double mu, double lam, double eps,
                                          double* coef, double* out, cudaStream_t st) {
  return debug_terms<MHS_UNIT_TERMS>(term, want_u, n, obs, tri, mu, lam, eps, coef, out, st);
}

int MHS_CAT2(unit_fullspace_, MHS_UNIT_TERMS)(int want, double near_l, int64_t n,
                                              const double* obs, const double* tri, double mu,
                                              double lam, double eps, double* U, double* H,
                                              double* E, double* G, double* S, cudaStream_t st) {
  return fullspace_run<MHS_UNIT_TERMS>(want, near_l, n, obs, tri, mu, lam, eps, U, H, E, G, S,
                                       st);
}

#else

int MHS_CAT4(unit_init_, MHS_UNIT_P, MHS_UNIT_KC, MHS_UNIT_RF)(const double* glx,
                                                               const double* glw) {
  return copy_tables(glx, glw);
}

using UnitRF = std::conditional_t<MHS_UNIT_RF == 1, float, double>;

int MHS_CAT4(unit_run_, MHS_UNIT_P, MHS_UNIT_KC, MHS_UNIT_RF)(const mhs_request* r,
                                                              cudaStream_t st, const Layout& L,
                                                              unsigned long long* census,
                                                              const Tune& tune) {
  return run<MHS_UNIT_P, MHS_UNIT_KC, UnitRF>(r, st, L, census, tune);
}

int MHS_CAT4(unit_batch_, MHS_UNIT_P, MHS_UNIT_KC, MHS_UNIT_RF)(const mhs_request* const* r,
                                                                const Layout* L, int n,
                                                                void* desc, int upload,
                                                                cudaStream_t st,
                                                                unsigned long long* census,
                                                                const Tune& tune) {
  return run_batch<MHS_UNIT_P, MHS_UNIT_KC, UnitRF>(r, L, n, desc, upload, st, census, tune);
}

#endif

}  // namespace pipe
}  // namespace mhs
