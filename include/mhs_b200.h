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
  /* Apply mode (slip != NULL): out receives the matrix times a slip vector,
   * y[o][c] = sum over columns and slip components of M[o][c][col][s]
   * slip[col][s], and the matrix itself is never stored.  slip is (n_dof,
   * n_s) with n_s = 3 (Cartesian slip) or n_b (INTERACTION); out is (n_obs,
   * C) with C = 3 (DISP, TRACTION), 9 (the stress-like kinds, [a][b]) or n_a
   * (INTERACTION).  This is the product a cycle or cascade model reads
   * (studies/active_fractal/kernel.py:1-30 keeps the whole K for it). */
  const double* slip;
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

/* ------------------------------------------------------------- batches
 * A batch: n requests queued as one group of launches per (order, readout
 * class, precision).  Each stage -- image coefficients, per-source data, the
 * two pair kernels, the output stage -- runs once over every request of the
 * group, its blocks finding their request by a prefix of block counts; the
 * fold of a request with fold = 1 runs per request between the pair kernels
 * and the output stage.  Every request runs in one pass over all its
 * observers (a request whose one-pass scratch would exceed 8 GiB is refused;
 * run it alone with mhs_assemble).  Apply-mode requests (slip != NULL) are
 * grouped apart from matrix requests.
 *   mhs_batch_pass_bytes  one request's one-pass scratch and the batch
 *                         limit (host only), to split a list of requests
 *                         into batches and requests to assemble alone
 *   mhs_batch_create      checks and plans the requests (host only; their
 *                         workspace fields are ignored; the array is copied)
 *   mhs_batch_workspace_bytes   bytes of the one device arena of the batch
 *   mhs_batch_bind        places each request's scratch and the launch
 *                         descriptors in the arena (copies queued on stream)
 *   mhs_submit_batch      queues the batch's kernels on stream.  With no
 *                         request at fold = 1 it queues kernels only, so it
 *                         can be captured into a CUDA graph and replayed
 *                         (a request whose sources all lie deeper than
 *                         FOLD_SOURCE_DEPTH_EPS eps gives the same result at
 *                         fold = 0); a request at fold = 1 makes the call
 *                         synchronise the stream to read its fold plan.
 *   mhs_poll              *done = 1 once the last submission has completed,
 *                         and then *status_bits = the OR of the requests'
 *                         device status bits
 *   mhs_batch_destroy
 * Inputs and outputs stay the caller's device buffers; a replay reads them
 * as they are at the time.  No counterpart in mhs, which has no launch to
 * amortise (mhs/chunking.py:3-6) and batches only by processes
 * (mhs/parallel.py:132-221). */
typedef struct mhs_batch mhs_batch;
int mhs_batch_pass_bytes(const mhs_request* req, size_t* bytes, size_t* limit);
int mhs_batch_create(const mhs_request* reqs, int n, mhs_batch** batch);
int mhs_batch_workspace_bytes(const mhs_batch* batch, size_t* bytes);
int mhs_batch_bind(mhs_batch* batch, void* workspace, size_t bytes, void* stream);
int mhs_submit_batch(mhs_batch* batch, void* stream);
int mhs_poll(mhs_batch* batch, int* done, int* status_bits);
int mhs_batch_destroy(mhs_batch* batch);

/* Launch shapes of one (order, readout class, precision) on the current
 * device: threads per block of the two pair kernels (observer tile, 32 to
 * 128) and of the output stage (column tile, 32 to 128), and the grid
 * multipliers of the fold's far- and near-load kernels (blocks per SM at
 * full occupancy x the multiplier, 1 to 16).  None of them changes a
 * result: each thread's arithmetic is the same under every shape.
 * mhs_autotune times the sample request (its workspace included) under each
 * candidate shape -- pair and output tiles 64 or 128, multipliers 2, 4 or
 * 8 -- keeps the fastest for the sample's class, returns it and its time.
 * No counterpart in mhs. */
typedef struct mhs_tune {
  int pair_tb, final_tb, far_mult, near_mult;
} mhs_tune;
int mhs_autotune(const mhs_request* sample, void* stream, mhs_tune* chosen, double* best_ms);
int mhs_set_tune(const mhs_request* like, const mhs_tune* tune);
int mhs_get_tune(const mhs_request* like, mhs_tune* tune);

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

/* The full-space single-triangle API (mhs/fullspace/api.py:90-175): the
 * nodal influence tensors of ONE triangle at n_obs observers (one thread per
 * observer), for the kernels in `want` (OR of MHS_FS_*):
 *   U (n, K, 3, 3)     slip -> displacement       (MHS_FS_U)
 *   H (n, K, 3, 3, 3)  slip -> TOTAL stress       (MHS_FS_H)
 *   E (n, K)           eigenstress weight         (MHS_FS_E)
 *   G (n, K, 3, 3)     force density -> displacement, Kelvin single layer (MHS_FS_G)
 *   S (n, K, 3, 3, 3)  force density -> stress    (MHS_FS_S)
 * with K = 1, 3, 6 nodes at order 0, 1, 2 (the nodes of the matrix
 * functions).  far_field: MHS_FAR_HYBRID (closed form within D_STAR element
 * lengths, Gauss quadrature beyond, as mhs's default), MHS_FAR_ANALYTIC
 * (closed form everywhere), MHS_FAR_QUADRATURE (quadrature everywhere).
 * tri: the vertex rows, by value in the request; obs and the outputs on
 * the device.  Material by (mu, nu), as mhs's full-space API.  eps >= 0; with
 * eps = 0 every observer must lie off the triangle's plane (the caller
 * checks: this engine has no on-plane limit). */
enum { MHS_FS_U = 1, MHS_FS_H = 2, MHS_FS_E = 4, MHS_FS_G = 8, MHS_FS_S = 16 };
enum { MHS_FAR_HYBRID = 0, MHS_FAR_ANALYTIC = 1, MHS_FAR_QUADRATURE = 2 };
typedef struct mhs_fullspace_request {
  int order;
  int want;
  int far_field;
  int pad;
  int64_t n_obs;
  const double* obs;   /* (n_obs, 3), device */
  double tri[9];       /* vertex rows, by value */
  double mu, nu, eps;
  double* U;           /* device outputs; NULL where not wanted */
  double* H;
  double* E;
  double* G;
  double* S;
} mhs_fullspace_request;
int mhs_fullspace_influence(const mhs_fullspace_request* req, void* stream);

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
  MHS_STAGE_PAIR = 1,    /* direct term + image R-family (two kernels) */
  MHS_STAGE_IMAGEQ = 2,  /* image Q-family */
  MHS_STAGE_FOLD = 3,    /* band lists + folded image */
  MHS_STAGE_FINAL = 4,   /* eigenstress, contraction, layout stores */
  /* parts of the fold stage (their time is inside MHS_STAGE_FOLD's) */
  MHS_STAGE_FOLD_PLAN = 5,   /* band scan, pair and panel plan, foot loads */
  MHS_STAGE_FOLD_NODES = 6,  /* polar-grid nodes and their class lists */
  MHS_STAGE_FOLD_FAR = 7,    /* far-field surface loads (12 x 12, 8 x 8 rules) */
  MHS_STAGE_FOLD_NEAR = 8,   /* near-field surface loads (closed form) */
  MHS_STAGE_FOLD_ACCUM = 9,  /* point-load products, panel sums, disk term */
  /* parts of the pair stage (their time is inside MHS_STAGE_PAIR's) */
  MHS_STAGE_PAIR_DIRECT = 10,   /* direct term */
  MHS_STAGE_PAIR_IMAGE_R = 11,  /* image R-family */
  MHS_N_STAGES = 12
};
int mhs_profile_enable(int on);
int mhs_profile_read(double* ms, int* launches);

/* Kernels this library queued (all devices, all threads) since the last
 * call; the count is returned and reset.  No counterpart in mhs. */
int mhs_kernel_count(unsigned long long* n);

/* Work census (measurement).  While enabled, the fold kernels count their
 * work units into device counters: band pairs, radial panels, polar-grid
 * nodes per surface-load form (closed form, 12 x 12 rule, 8 x 8 rule) and
 * near-field edge integrals per form (closed, small-|u| series, large-|u|
 * series); the image Q-family kernel counts its pairs and their rule points
 * (n^2 at Gauss order n).  mhs_census_read synchronises the device, returns the
 * MHS_CENSUS_N counts accumulated since the last read or enable, and clears
 * them.  Multiplied by the per-unit operation counts of the op-counting build
 * (mhs_b200/csrc/opcount.cpp) they give the algorithmic flops.  No
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
  /* the image Q-family stage: pairs it evaluates and their rule points */
  MHS_CENSUS_Q_PAIRS = 8,
  MHS_CENSUS_Q_POINTS = 9,
  MHS_CENSUS_N = 10
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
