/* C ABI of the B200 Green's-function assembler.
 *
 * One entry point fills one matrix on one CUDA device, asynchronously on the
 * caller's stream.  Every pointer in mhs_request is DEVICE memory owned by
 * the caller; the library allocates nothing per call (it keeps a small
 * per-device table of Gauss-Legendre rules, built on first use).  Scratch
 * comes from the caller's workspace, sized by mhs_workspace_bytes.
 *
 * The request mirrors mhs's internal assembly seam (mhs/kernels/assemble.py:
 * 190-366), which sees only C-contiguous float64 arrays and plain floats:
 * obs (N, 3), tris (S, 3, 3), eps (S,), mu, lam, a preallocated output,
 * order, ids (S, 6) for shared columns, fold, plus receiver normals for
 * traction and receiver/source bases for interaction.  Validation of user
 * input (shapes, z <= 0, eps > 0, the byte ceiling) happens in the caller,
 * as in mhs/matrices.py:75-227; the library re-checks what would make a
 * launch unsafe and returns an error code instead.
 */
#ifndef MHS_B200_H
#define MHS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Output kinds, each one of mhs's public matrix functions. */
enum mhs_kind {
  MHS_DISP = 0,          /* disp_matrix          (N, 3, n_dof, 3)    matrices.py:231 */
  MHS_STRESS = 1,        /* stress_matrix        (N, 3, 3, n_dof, 3) matrices.py:251 */
  MHS_TOTAL_STRESS = 2,  /* total_stress_matrix  (N, 3, 3, n_dof, 3) matrices.py:494 */
  MHS_EIGENSTRESS = 3,   /* eigenstress_matrix   (N, 3, 3, n_dof, 3) matrices.py:518 */
  MHS_STRAIN = 4,        /* elastic_strain_matrix(N, 3, 3, n_dof, 3) matrices.py:546 */
  MHS_TRACTION = 5,      /* traction_matrix      (N, 3, n_dof, 3)    matrices.py:298 */
  MHS_INTERACTION = 6    /* interaction_matrix   (N, n_dof, n_a, n_b) matrices.py:378 */
};

enum mhs_precision {
  MHS_FP64 = 0,   /* every term in float64 */
  MHS_MIXED = 1   /* far-field quadrature bulk in float32, the rest float64 */
};

enum mhs_status_code {
  MHS_OK = 0,
  MHS_ERR_ARG = 1,        /* invalid request field */
  MHS_ERR_WORKSPACE = 2,  /* workspace too small */
  MHS_ERR_CUDA = 3,       /* a CUDA call failed */
  MHS_ERR_DEVICE = 4      /* a device-side check failed (see mhs_read_status) */
};

/* Device-side status bits (mhs_read_status). */
#define MHS_DEV_FOLD_GRID_OVERFLOW 1

typedef struct mhs_request {
  int kind;                  /* enum mhs_kind */
  int order;                 /* 0, 1, 2 (P0, P1, P2) */
  int fold;                  /* 1: fold surface-reaching sources (default) */
  int subtract_eigenstress;  /* STRESS/STRAIN/TRACTION/INTERACTION */
  int precision;             /* enum mhs_precision */
  int out_f32;               /* 1: output stored as float32 */
  int64_t n_obs, n_src;
  const double* obs;         /* (n_obs, 3) */
  const double* tris;        /* (n_src, 3, 3) */
  const double* eps;         /* (n_src,) */
  double mu, lam;
  const double* normals;     /* TRACTION / INTERACTION: (n_obs, 3) unit */
  const double* rec_basis;   /* INTERACTION: (n_obs, n_a, 3) */
  const double* src_basis;   /* INTERACTION: (n_src, n_b, 3), or (n_cols, n_b, 3) with ids */
  int n_a, n_b;
  /* continuous layout: per-column gather plan built by mhs_column_plan */
  const int64_t* ids;        /* (n_src, 6) or NULL (discontinuous) */
  int64_t n_cols;
  const int32_t* col_ptr;    /* (n_cols + 1,) */
  const int32_t* col_ent;    /* (n_src * 6,) entries s * 6 + k, ascending s per column */
  void* out;                 /* output, C-contiguous, zero not required */
  void* workspace;
  size_t workspace_bytes;
} mhs_request;

/* Bytes of workspace a request needs: *min_bytes for one observer row per
 * pass, *good_bytes for the whole request in one pass (capped at 2 GiB). */
int mhs_workspace_bytes(const mhs_request* req, size_t* min_bytes, size_t* good_bytes);

/* Assemble req->out on `stream` (a cudaStream_t; NULL = legacy default).
 * Returns MHS_OK once every kernel is queued; device-side checks are read
 * later with mhs_read_status.  Replaces mhs.kernels.assemble's
 * assemble_halfspace_disp / _total_stress / _traction, assemble_interaction
 * and assemble_eigenstress (assemble.py:190-366) plus the eigenstress
 * subtraction and strain readout of matrices.py:287-294 and :572-579. */
int mhs_assemble(const mhs_request* req, void* stream);

/* Allocation-free variant of mhs_assemble, for callers that must not
 * allocate device memory while they run: a solver whose memory pool owns
 * the device after start-up, a host framework that pre-reserves nearly all
 * of HBM (so even a small cudaMalloc can fail or stall), or real-time code
 * where an allocation's implicit synchronisation is not allowed.  It takes
 * the same request -- the caller still owns inputs and output -- but
 * ignores workspace / workspace_bytes and uses one fixed scratch array
 * inside this library instead (MHS_NOALLOC_SCRATCH_BYTES per device, held
 * by every device that loads the library until the process exits).  It
 * calls no cudaMalloc or cudaFree.
 *
 * Limit: the request's per-source tables plus one observer row of
 * per-pair tensors must fit the array (about 8.6 KB per source at P2,
 * so a few thousand sources per call); larger requests are refused with
 * MHS_ERR_WORKSPACE and a message that says so, and observers beyond what
 * fits in one pass are processed in chunks.
 *
 * The first call on each device does one-time set-up with that device
 * current (the Gauss-Legendre tables and the scratch array's device
 * address, via cudaGetSymbolAddress); make that first call before any
 * stream capture.  Every call shares the one array and it keeps the last
 * call's contents (the pipeline clears what must start at zero), so calls
 * whose work overlaps on the GPU -- on different streams, or from
 * different threads -- race: serialise them.
 *
 * status_bits: NULL to return once queued (read the status later with
 * mhs_read_status(NULL, stream, &bits)); otherwise the call synchronises
 * `stream` and stores the device status bits there.
 * No counterpart in mhs (which never runs on a device). */
#define MHS_NOALLOC_SCRATCH_BYTES ((size_t)64 << 20)
int mhs_assemble_noalloc(const mhs_request* req, void* stream, int* status_bits);

/* Synchronise `stream` and return the device status bits of the last
 * request that used `workspace` (0 = clean), clearing them.  workspace =
 * NULL reads the status of the last mhs_assemble_noalloc call on the
 * current device (the word lives in its scratch array). */
int mhs_read_status(void* workspace, void* stream, int* bits);

/* Host helper: the per-column gather plan of a continuous layout from its
 * (n_src, 6) ids (mhs/shared.py:175-273), entries in ascending source order
 * so the sum runs in the order mhs's scatter-add does (assemble.py:69-93).
 * col_ptr has n_cols + 1 entries, col_ent n_src * 6. */
int mhs_column_plan(const int64_t* ids_host, int64_t n_src, int64_t n_cols, int32_t* col_ptr,
                    int32_t* col_ent);

/* Diagnostics: one influence term of ONE source at n observers, one thread
 * per observer, as the pipeline evaluates it (term 0 direct, 1 image
 * R-family, 2 image Q-family, 3 folded image; with want_u = 0, 4 and 5 the
 * fold's surface load at (x, y, 0) as K x 3 values, from the contracted
 * sigma_zz row and from the full stress kernel).  out (device) receives per
 * observer K x C values (C = 9 for want_u, else 27) then K blob weights.
 * coef_scratch: device buffer of at least 4096 doubles.  No counterpart in
 * mhs; the per-term split follows mhs/kernels/assemble.py:96-120. */
int mhs_debug_terms(int order, int term, int want_u, int n, const double* obs, const double* tri,
                    double mu, double lam, double eps, double* coef_scratch, double* out,
                    void* stream);

/* Stage timing (tracing).  While enabled, every stage launch of every
 * request is bracketed by CUDA events on its stream; mhs_profile_read waits
 * for them and returns per-stage milliseconds and launch counts since the
 * last read (arrays of MHS_N_STAGES).  No counterpart in mhs, which has no
 * tracing. */
enum mhs_stage {
  MHS_STAGE_PREP = 0,    /* per-material coefficients, per-source frames */
  MHS_STAGE_PAIR = 1,    /* direct term + image R-family */
  MHS_STAGE_IMAGEQ = 2,  /* image Q-family */
  MHS_STAGE_FOLD = 3,    /* band lists + folded image */
  MHS_STAGE_FINAL = 4,   /* eigenstress, contraction, layout stores */
  MHS_N_STAGES = 5
};
int mhs_profile_enable(int on);
int mhs_profile_read(double* ms, int* launches);

/* Fold work census (measurement).  While enabled, the fold kernel counts its
 * work units into device counters: band pairs, radial panels, polar-grid
 * nodes per surface-load form (closed form, 12 x 12 rule, 8 x 8 rule) and
 * near-field edge integrals per form (closed, small-|u| series, large-|u|
 * series).  mhs_census_read synchronises the device, returns the
 * MHS_CENSUS_N counts accumulated since the last read or enable, and clears
 * them.  Multiplied by the per-unit operation counts of the op-counting build
 * (mhs_b200/csrc/opcount.cpp) they give the fold's algorithmic flops.  No
 * counterpart in mhs. */
enum mhs_census_item {
  MHS_CENSUS_PAIRS = 0,
  MHS_CENSUS_PANELS = 1,
  MHS_CENSUS_NEAR = 2,
  MHS_CENSUS_FAR12 = 3,
  MHS_CENSUS_FAR8 = 4,
  MHS_CENSUS_EDGE_CLOSED = 5,
  MHS_CENSUS_EDGE_SMALL = 6,
  MHS_CENSUS_EDGE_LARGE = 7,
  MHS_CENSUS_N = 8
};
int mhs_census_enable(int on);
int mhs_census_read(unsigned long long* counts);

/* Issue ceiling of the device: independent FMA chains on every SM, FP64
 * (fp64 = 1) or FP32, in TFLOP/s (2 flops per FMA).  The roofline
 * denominator of the FP64 and mixed forms. */
int mhs_fp_peak(int fp64, int iters, double* tflops, void* stream);

/* Last error message of this thread. */
const char* mhs_last_error(void);

/* Library version string. */
const char* mhs_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MHS_B200_H */
