/*
 * bcmg.h -- C ABI of the B200-native alpha-AMG + flexible-CG solve path.
 *
 * This header is the drop-in boundary for BootCMatchG's solve path.  Every
 * entry point names the reference interface it replaces (paths are relative
 * to the BootCMatchG source tree).  Plain C types only: int32 indices, FP64
 * values, opaque handles, status codes.  No CUDA or torch types appear here;
 * device pointers are passed as plain pointers and streams as void*.
 *
 * Threading: every piece of solver state lives in a bcmg_handle.  Distinct
 * handles may be used from distinct threads concurrently; one handle must be
 * used by one thread at a time.  (The reference keeps its state in global
 * singletons: FCG::context, Relax::context, GAMGcycle::Res_buffer,
 * matchingAggregationContext -- src/SOLVER/FCG.h:72-74,
 * src/AMG/relaxation.cu:8-9, src/SOLVER/GAMG_cycle.cu:7-8,
 * src/AMG/matchingAggregation.h:3-6.)
 */
#ifndef BCMG_H
#define BCMG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference terminates the process on every error
 * (exit()/assert in src/utility/utils.h:36-71, src/AMG/AMG.cu:8-18,
 * src/SOLVER/FCG.cu:459-462); this library returns one of these instead and
 * leaves a message in bcmg_last_error(). */
typedef enum bcmg_status {
  BCMG_OK = 0,
  BCMG_ERR_PARAM = 1,           /* invalid setting (checkP, AMG.cu:8-18)         */
  BCMG_ERR_IO = 2,              /* file missing or unparsable                     */
  BCMG_ERR_ALLOC = 3,           /* host or device allocation failed               */
  BCMG_ERR_CUDA = 4,            /* CUDA runtime error                             */
  BCMG_ERR_INDEFINITE = 5,      /* FCG met a non-positive curvature (A not SPD)   */
  BCMG_ERR_NOT_CONVERGED = 6,   /* reserved: non-convergence is reported in info  */
  BCMG_ERR_DEVICE_TIMEOUT = 7,  /* a bounded device loop ran out of iterations    */
  BCMG_ERR_INVALID_MATRIX = 8,  /* not square, missing diagonal, bad index, NaN   */
  BCMG_ERR_UNSUPPORTED = 9,     /* option the path does not implement             */
  BCMG_ERR_INTERNAL = 10,
  BCMG_ERR_PENDING = 11         /* bcmg_server_wait: the request is not done yet  */
} bcmg_status;

/* Host CSR matrix: 0-based, int32 row pointers and column indices, FP64
 * values; n rows, m columns.  Mirrors struct CSR, src/matrix/CSR.h:13-28
 * (host side; the device flag and cuSPARSE descriptor are dropped). */
typedef struct bcmg_csr {
  int32_t n;
  int32_t m;
  int32_t nnz;
  int32_t *row;   /* n+1 */
  int32_t *col;   /* nnz */
  double  *val;   /* nnz */
} bcmg_csr;

/* The 14 file settings plus the forced matchtype, in the same field order
 * as struct params, src/AMG/AMG.cu:20-37.  The settings file lists them in a
 * different order (AMG.cu:491-522, AMGsettings_base:1-14); see
 * bcmg_params_from_file. */
typedef struct bcmg_params {
  int    solver_type;        /* 0 multiplicative, 1 symmetrized, 2 additive   */
  int    max_hrc;            /* max hierarchies built by the bootstrap        */
  double conv_ratio;         /* rho: desired composite convergence rate       */
  int    matchtype;          /* always 3 (AMG.cu:497)                         */
  int    aggrsweeps;         /* pairwise aggregation sweeps per level         */
  int    aggrtype;           /* 0 unsmoothed, 1 smoothed (P = S P_tent)       */
  int    max_levels;         /* max levels per hierarchy                      */
  int    cycle_type;         /* 0 V, 1 H, 2 W, 3 K-cycle                      */
  int    coarse_solver;      /* 0 Jacobi, 4 l1-Jacobi                         */
  int    relax_type;         /* 0 Jacobi, 4 l1-Jacobi                         */
  int    prerelax_sweeps;
  int    postrelax_sweeps;
  int    itnlim;             /* FCG iteration limit                           */
  double rtol;               /* FCG relative tolerance on ||r||_2             */
  int    relaxnumber_coarse; /* sweeps on the coarsest level                  */
} bcmg_params;

/* Extensions that do not exist in the reference.  They never change the
 * meaning of the 14 settings above. */
enum { BCMG_PREC_FP64 = 0, BCMG_PREC_MIXED = 1 };
enum { BCMG_STORE_FP32 = 0, BCMG_STORE_BF16 = 1, BCMG_STORE_FP16 = 2 };

typedef struct bcmg_ext {
  int    precision;       /* BCMG_PREC_FP64 (default): FP64 hierarchy and cycle.
                             BCMG_PREC_MIXED: FP32 hierarchy values and cycle,
                             FP64 FCG, dots, recurrences and matching weights. */
  int    coarse_storage;  /* mixed mode: value storage of levels >= 1          */
  int    replace_every;   /* mixed mode: recompute r = b - A x in FP64 every k
                             iterations and at convergence (0 disables)        */
  int    use_graphs;      /* capture the FCG iteration in a CUDA graph         */
  int    device;          /* CUDA device ordinal                               */
  int    verbose;         /* 0 quiet, 1 #META lines, 2 per-iteration residual  */
  double max_device_seconds; /* bound, in seconds, on each wait of a pipelined
                             row pass for its staged copies (default 2); a
                             wait that runs out makes the call return
                             BCMG_ERR_DEVICE_TIMEOUT and leaves the handle
                             usable (bcmg_set_max_device_seconds changes it) */
  void  *stream;          /* cudaStream_t to run on from setup on (NULL: the
                             handle creates its own); the caller keeps it alive */
  int    sliced;          /* solve on the sliced copies of the levels (default 1) */
  int    autotune;        /* batched solves: time the row-kernel shapes of every
                             level once per batch width (default 1); 0 uses a
                             fixed rule.  Results are identical either way.   */
  int    narrow_values;   /* store the values of the FP64 and FP32
                             solve-phase copies (cycle, FCG SpMV) in BF16,
                             FP16 or (FP64 copies) FP32 when every value
                             converts exactly (default 1); the kernels widen
                             them, so results are bit-identical with 0.      */
  int64_t match_step_limit; /* bound on the steps (proposals and displacements)
                             of each suitor-matching thread; 0 (default): 8 nnz
                             + 1024 of the level.  A thread that runs out makes
                             setup return BCMG_ERR_DEVICE_TIMEOUT.           */
} bcmg_ext;

/* Per-solve report.  residual is the recursive ||r||_2 that FCG returns
 * (flexibileConjugateGradients_v3 return value, src/SOLVER/FCG.cu:584);
 * true_rel_residual is ||b - A x||_2 / ||b - A x0||_2 recomputed in FP64. */
typedef struct bcmg_solve_info {
  int    iters;              /* num_iter as the reference counts it (FCG.cu:569) */
  int    converged;
  double residual;
  double rel_residual;
  double true_rel_residual;
  double setup_ms;
  double solve_ms;
  int    num_hrc;
  double estimated_ratio;
} bcmg_solve_info;

typedef struct bcmg_handle bcmg_handle;

/* ---- errors ------------------------------------------------------------- */
const char *bcmg_last_error(void);            /* thread-local message          */
const char *bcmg_status_string(int status);
const char *bcmg_version(void);
/* Number of CUDA kernels this library has launched in this process. */
unsigned long long bcmg_kernel_launches(void);

/* ---- failure detection (no counterpart in the reference, which exit()s or
 * asserts: src/utility/utils.h:36-71) ---------------------------------------
 * Every device-side wait of the library is bounded.  This changes the bound
 * of a handle's pipelined row passes (bcmg_ext.max_device_seconds); the next
 * solve recaptures its CUDA graph with it.  seconds > 0. */
bcmg_status bcmg_set_max_device_seconds(bcmg_handle *h, double seconds);
/* Self-test of that mechanism on `device`: a pipeline wait that nothing ever
 * completes, bounded by `seconds` (0 < seconds <= 10), beside a real staged
 * copy that must land before its kernel exits.  Returns
 * BCMG_ERR_DEVICE_TIMEOUT -- what a solve returns when one of its waits runs
 * out -- when the wait gave up and the copy drained, BCMG_ERR_INTERNAL if
 * either did not happen.  The device stays usable either way. */
bcmg_status bcmg_wait_selftest(int device, double seconds);
/* Host-side failure injection for tests of the error paths: the device
 * allocation that follows `after` further successful ones fails with
 * BCMG_ERR_ALLOC, as an out-of-memory cudaMallocAsync would (one shot,
 * process-wide; after < 0 disarms).  Nothing reaches the GPU. */
bcmg_status bcmg_debug_fail_alloc(int64_t after);
/* Device allocations of the library: *live held right now over all handles
 * (a failed call leaves it where it found it), *made since the library was
 * loaded.  Either pointer may be NULL. */
bcmg_status bcmg_debug_alloc_stats(int64_t *live, int64_t *made);

/* ---- matrix input (replaces readMatrixFromFile, src/matrix/matrixIO.cu:4) --
 * m_type 0: Matrix Market coordinate real/integer, general or symmetric
 * (readMTXDouble, matrixIO.cu:33-192); m_type 1: the reference's plain COO
 * list "n nnz rows... cols... vals..." (readMTX2Double, matrixIO.cu:194-289).
 * Columns of each row are sorted and duplicate entries summed on ingest (the
 * reference keeps file order, which its AH builder silently assumes sorted,
 * src/AMG/matching.cu:216-231).  Arrays are allocated by the library and
 * released with bcmg_csr_free. */
bcmg_status bcmg_read_matrix(const char *path, int m_type, bcmg_csr *out);
/* Matrix Market writer (CSRMatrixPrintMM, src/matrix/matrixIO.cu:292-335). */
bcmg_status bcmg_write_matrix_mm(const char *path, const bcmg_csr *A);
void        bcmg_csr_free(bcmg_csr *A);
/* Validates a caller CSR: square, in-range strictly increasing columns,
 * a diagonal entry in every row, finite values. */
bcmg_status bcmg_csr_check(const bcmg_csr *A);

/* ---- settings (replaces AMG::Params::initFromFile, src/AMG/AMG.cu:480-526) */
void        bcmg_params_default(bcmg_params *p);   /* = AMGsettings_base       */
bcmg_status bcmg_params_from_file(const char *path, bcmg_params *p);
bcmg_status bcmg_params_check(const bcmg_params *p); /* checkP, AMG.cu:492-516  */
void        bcmg_ext_default(bcmg_ext *e);

/* ---- setup and solve -----------------------------------------------------
 * bcmg_setup: host CSR in; uploads it and runs the bootstrap
 * (solve() lines src/SOLVER/solver.cu:37-62: BootBuildData::initByParams,
 * ApplyData::setGridSweeps, Bootstrap::bootstrap).  The handle owns all
 * device memory.  bcmg_setup_device: same, the CSR already resident in device
 * memory (the library copies it).  For inputs of 131,072 rows and more the
 * setup starts one helper thread and one stream of its own, which build the
 * coarse levels' solve copies while the setup goes on coarsening; both end
 * before the call returns. */
bcmg_status bcmg_setup(const bcmg_csr *A, const bcmg_params *p,
                       const bcmg_ext *ext, bcmg_handle **out);
bcmg_status bcmg_setup_device(int32_t n, int32_t nnz, const int32_t *d_row,
                              const int32_t *d_col, const double *d_val,
                              const bcmg_params *p, const bcmg_ext *ext,
                              bcmg_handle **out);
/* Flexible CG (flexibileConjugateGradients_v3, src/SOLVER/FCG.cu:433-585)
 * preconditioned by the bootstrap composite.  b and x have n entries; x is
 * the initial guess on input and the solution on output.  on_device != 0
 * means b and x are device pointers.  An already-converged start returns
 * BCMG_OK with iters = 0 (the reference calls exit(1), FCG.cu:459-462). */
bcmg_status bcmg_solve(bcmg_handle *h, const double *b, double *x,
                       int on_device, bcmg_solve_info *info);
/* Exactly the reference's solve(A_host, p, rhs) (solver.cu:20-129): setup,
 * solve from x0 = 0, teardown.  Host arrays in and out. */
bcmg_status bcmg_solve_legacy(const bcmg_csr *A, const bcmg_params *p,
                              const bcmg_ext *ext, const double *b, double *x,
                              bcmg_solve_info *info);
/* ---- multiple right-hand sides (no counterpart in the reference, which
 * solves one right-hand side per solve() call) ------------------------------
 * Solves A X = B for nrhs right-hand sides sharing the handle's hierarchy.
 * B and X are column-major n x nrhs with leading dimensions ldb, ldx >= n, on
 * the host or (on_device) the handle's device; X holds the initial guesses on
 * entry and the solutions on return.  Up to 32 columns run together: one
 * cycle per FCG iteration serves all of them and every column keeps its own
 * FCG scalars, iteration count and stopping test, exactly as bcmg_solve would
 * for that column alone.  infos: nrhs entries (or NULL); solve_ms is the time
 * of the group of up to 32 columns the entry belongs to.  Returns
 * BCMG_ERR_INDEFINITE if any column broke down (the others are still solved
 * and reported). */
bcmg_status bcmg_solve_batch(bcmg_handle *h, int32_t nrhs, const double *B, int64_t ldb,
                             double *X, int64_t ldx, int on_device, bcmg_solve_info *infos);
/* Z = M R for nrhs device columns (column-major, leading dimensions >= n):
 * the batched preconditioner of bcmg_solve_batch, from Z = 0. */
bcmg_status bcmg_precond_apply_batch(bcmg_handle *h, int32_t nrhs, const double *d_R,
                                     int64_t ldr, double *d_Z, int64_t ldz);
/* k batched smoother sweeps on level `level` of hierarchy `hrc` for `width`
 * interleaved columns (width a power of two <= 32; element (i, c) at
 * u[i * width + c]), in the cycle's precision (FP32 for BCMG_PREC_MIXED,
 * else FP64), exactly as the batched cycle runs them.  f and u must be
 * 16-byte aligned. */
bcmg_status bcmg_level_relax_batch(bcmg_handle *h, int hrc, int level, int32_t width,
                                   const void *d_f, void *d_u, int k);
/* The row-kernel shape a batch of nrhs columns uses on level `level` of
 * hierarchy `hrc` (hrc < 0: the FCG SpMV on the input matrix): batch width,
 * columns per lane and threads per block, plus the time the batch state took
 * to build and tune (ms). */
bcmg_status bcmg_batch_config(bcmg_handle *h, int32_t nrhs, int hrc, int level,
                              int32_t *width, int32_t *cols_per_lane, int32_t *block_threads,
                              double *tune_ms);

/* Device memory the handle holds, in bytes (hierarchies, their solve-phase
 * copies, cycle and Krylov work vectors, batch state); no counterpart in the
 * reference. */
bcmg_status bcmg_device_bytes(const bcmg_handle *h, uint64_t *bytes);
/* Frees everything the handle owns (the frees at the end of solve():
 * CSRm::free, AMG::Hierarchy / Boot frees, src/SOLVER/solver.cu:120-126). */
bcmg_status bcmg_destroy(bcmg_handle *h);

/* ---- hierarchy files -------------------------------------------------------
 * Save a set-up handle's hierarchies (settings, input matrix, every level's
 * CSR, D, M, w, aggregates and prolongator values, and with smoothed
 * aggregation every level's smoothed prolongator P) to a binary file, and
 * build a handle from such a file without running setup again.  The
 * reference only dumps single vectors (Vector::dump / Vector::load,
 * src/matrix/vector.cu:468-505) and rebuilds every hierarchy per solve();
 * this lets a cache of hierarchies outlive the process.  bcmg_load takes its
 * own extensions (e.g. a hierarchy built in FP64 mode can be loaded for
 * mixed-precision solves); NULL selects the defaults.  Little-endian files. */
bcmg_status bcmg_save(const bcmg_handle *h, const char *path);
bcmg_status bcmg_load(const char *path, const bcmg_ext *ext, bcmg_handle **out);
/* The settings a handle was set up (or loaded) with. */
bcmg_status bcmg_get_params(const bcmg_handle *h, bcmg_params *p);

/* ---- solve server (no counterpart in the reference) ------------------------
 * Continuous batching of solve requests on one GPU: `slots` worker threads
 * with their own CUDA streams run requests from a FIFO queue.  A request
 * starts when a slot is free and the estimated device footprint of all
 * resident hierarchies and work blocks plus its own stays under mem_cap_gb
 * (idle cached hierarchies are evicted least-recently-used to make room).
 * Finished hierarchies stay cached by matrix key up to cache_cap_gb, and
 * queued requests on the same key (up to max_batch) run together as one
 * bcmg_solve_batch on the shared hierarchy. */
typedef struct bcmg_server bcmg_server;
typedef struct bcmg_server_opts {
  int         device;
  int         slots;          /* requests in flight (default 4)               */
  double      mem_cap_gb;     /* admission cap on device footprint (150)      */
  double      cache_cap_gb;   /* budget of cached idle hierarchies (60)       */
  int         max_batch;      /* same-key requests solved together (<= 32)    */
  bcmg_params params;         /* settings of every request                    */
  bcmg_ext    ext;            /* precision etc.; stream and device are set
                                 by the server                                */
} bcmg_server_opts;
typedef struct bcmg_request_info {
  bcmg_solve_info solve;
  double latency_ms;          /* submit -> result written                     */
  double queue_ms;            /* submit -> start on a slot                    */
  int    group;               /* requests solved together with it (1 alone)   */
  int    cache_hit;           /* hierarchy came from the cache                */
} bcmg_request_info;
typedef struct bcmg_server_stats {
  uint64_t submitted, completed, failed, setups, cache_hits, batches, evictions;
  uint64_t peak_resident_bytes, resident_bytes;
  int      cached_hierarchies, queued, running;
} bcmg_server_stats;
void bcmg_server_opts_default(bcmg_server_opts *o);
bcmg_status bcmg_server_create(const bcmg_server_opts *opt, bcmg_server **out);
/* Queues one solve A x = b from x0 = 0.  key identifies the matrix (0: a
 * hash of A's arrays).  A's arrays are read only if the key needs a setup and
 * must stay valid until the request is done; b is copied; x (n doubles) is
 * written when the request finishes. */
bcmg_status bcmg_server_submit(bcmg_server *s, const bcmg_csr *A, uint64_t key,
                               const double *b, double *x, uint64_t *ticket);
/* Waits up to timeout_s seconds (< 0: forever) for a request; returns its
 * status (BCMG_ERR_PENDING if it is not done) and releases the ticket once
 * done. */
bcmg_status bcmg_server_wait(bcmg_server *s, uint64_t ticket, double timeout_s,
                             bcmg_request_info *info);
bcmg_status bcmg_server_stats_get(bcmg_server *s, bcmg_server_stats *out);
/* Finishes every queued request, then frees the cache and the streams. */
bcmg_status bcmg_server_destroy(bcmg_server *s);
/* Binds the handle to a CUDA stream (cudaStream_t passed as void*); no
 * counterpart in the reference, which runs on the default stream with
 * global handles (src/utility/handles.cu). */
bcmg_status bcmg_set_stream(bcmg_handle *h, void *stream);
/* z = B r for the composite preconditioner (preconditionApply,
 * src/SOLVER/FCG.cu:112-187) with z's initial content as initial guess.
 * Device pointers, n entries each. */
bcmg_status bcmg_precond_apply(bcmg_handle *h, const double *d_r, double *d_z);

/* ---- hierarchy introspection (parity tests, #META output) --------------
 * What the reference prints rather than returns: the number of hierarchies
 * and the estimated ratio (#META agg;hierarchy_levels_num and
 * agg;final_estimated_ratio, src/SOLVER/solver.cu:106-107), per hierarchy
 * the level count, operator complexities and average coarsening ratio
 * (AMG::Hierarchy::finalize_cmplx / finalize_wcmplx / printInfo,
 * src/AMG/AMG.cu:221-251, called at src/AMG/matchingAggregation.cu:404-414),
 * and one level's data (hrrch->A_array / P_array and the relaxPrepare
 * vectors). */
bcmg_status bcmg_hierarchy_count(const bcmg_handle *h, int *num_hrc,
                                 double *estimated_ratio);
bcmg_status bcmg_hierarchy_info(const bcmg_handle *h, int hrc, int *num_levels,
                                double *op_cmplx, double *op_wcmplx,
                                double *avg_cratio);
bcmg_status bcmg_level_info(const bcmg_handle *h, int hrc, int level,
                            int32_t *n, int32_t *nnz, int32_t *n_coarse);
/* Copies one level to host buffers (any pointer may be NULL).  row n+1,
 * col/val nnz, D/M/w n entries; agg/p n entries (absent on the last level):
 * agg[i] is the coarse index of fine row i and p[i] the prolongator value
 * (P has exactly one entry per row for unsmoothed aggregation). */
bcmg_status bcmg_level_copy(const bcmg_handle *h, int hrc, int level,
                            int32_t *row, int32_t *col, double *val, double *D,
                            double *M, int32_t *agg, double *p, double *w);

/* k smoother sweeps of one level exactly as the solve-phase cycle runs them
 * (relax, src/AMG/relaxation.cu:357-377, with relax_type's diagonal, in the
 * level's solve format and precision).  f and u
 * are device vectors of the level's size: FP64 for BCMG_PREC_FP64 handles,
 * FP32 for BCMG_PREC_MIXED handles.  Used to time the dominant kernel. */
bcmg_status bcmg_level_relax(bcmg_handle *h, int hrc, int level, const void *d_f,
                             void *d_u, int k);
/* Storage of one level's solve-phase copy (no counterpart in the reference,
 * which solves from CSR): value slots (32 values each),
 * slots of slices with explicit columns (the rest share column offsets and
 * store no indices), slices, bytes per value (0: the level is solved from
 * CSR). */
bcmg_status bcmg_level_format(const bcmg_handle *h, int hrc, int level,
                              int64_t *slots, int64_t *column_slots,
                              int32_t *slices, int32_t *value_bytes);

/* ---- single-step entry points on device pointers --------------------------
 * Used by the parity tests; stream may be NULL (legacy default stream).
 *
 * One pairwise aggregation sweep: weights (Matching::makeAH +
 * toMaximumProductMatrix, src/AMG/matching.cu:293-317,437-472), suitor
 * matching (approx_match_gpu_suitor, src/AMG/suitor.cu:427-454), unsymFix
 * (src/AMG/unsymMatching.cu:58-71) and _aggregate_symmetric
 * (src/AMG/matchingAggregation.cu:92-137).  Outputs agg (n), p (n) and the
 * number of aggregates; optional W (nnz, 0 on the diagonal), suitor (n) and
 * symmetric matching (n). */
bcmg_status bcmg_k_pair_aggregate(int32_t n, int32_t nnz, const int32_t *d_row,
                                  const int32_t *d_col, const double *d_val,
                                  const double *d_w, int32_t *d_agg,
                                  double *d_p, int32_t *n_coarse,
                                  double *d_W, int32_t *d_suitor,
                                  int32_t *d_match, void *stream);
/* Galerkin product A_c = P^T A P for a one-entry-per-row P given as (agg, p)
 * (matchingAggregation.cu:239-244 via nsparse spgemm_kernel_hash,
 * src/EXTERNAL/nsparse-master/cuda-c/src/kernel/kernel_spgemm_hash_d.cu:1035).
 * Call with d_crow only to get *c_nnz; then again with d_ccol/d_cval of that
 * size. */
bcmg_status bcmg_k_galerkin(int32_t n, int32_t nnz, const int32_t *d_row,
                            const int32_t *d_col, const double *d_val,
                            int32_t n_coarse, const int32_t *d_agg,
                            const double *d_p, int32_t *d_crow,
                            int32_t *c_nnz, int32_t *d_ccol, double *d_cval,
                            void *stream);
/* C = X Y for device CSR matrices (X: n rows, x_nnz entries; Y: y_n rows,
 * m columns, rows with distinct columns), each entry summed over X's row
 * order from the first term — the products of smoothed aggregation
 * (CSRm::CSRCSR_product, src/matrix/CSR.cu:1069-1082, whose cuSPARSE order
 * is unspecified; matchingAggregation.cu:372-384).  Rows come out sorted by
 * column.  Call with d_crow (n+1) only to get *c_nnz; then again with
 * d_ccol/d_cval of that size. */
bcmg_status bcmg_k_spgemm(int32_t n, int32_t m, int32_t x_nnz, const int32_t *d_xrow,
                          const int32_t *d_xcol, const double *d_xval, int32_t y_n,
                          int32_t y_nnz, const int32_t *d_yrow, const int32_t *d_ycol,
                          const double *d_yval, int32_t *d_crow, int32_t *c_nnz,
                          int32_t *d_ccol, double *d_cval, void *stream);
/* k Jacobi / l1-Jacobi sweeps u <- u + (f - A u) ./ d
 * (_jacobi_it, src/AMG/relaxation.cu:176-209).  d is D (Jacobi) or the
 * absolute row sums (l1).  u is updated in place. */
bcmg_status bcmg_k_relax(int32_t n, int32_t nnz, const int32_t *d_row,
                         const int32_t *d_col, const double *d_val,
                         const double *d_d, const double *d_f, double *d_u,
                         int k, void *stream);
/* bcmg_k_relax without any device allocation; no counterpart in the
 * reference.  For callers that may not allocate device memory at the point
 * of the call (another framework's allocator owns the device, a plugin with
 * a fixed footprint, a latency-critical loop).  Its ping-pong vector is a
 * process-lifetime device buffer of 1,048,576 doubles (8 MiB on every GPU
 * that loads the library): n above that is rejected with BCMG_ERR_PARAM.
 * The first call on a device looks the buffer up and should come before any
 * stream capture; the address stays cached for the process, so do not call
 * it after resetting the device or destroying its primary context.  stream
 * must belong to the current device, and each call synchronises it before
 * returning.  Calls that overlap on the GPU share the buffer and race. */
bcmg_status bcmg_k_relax_noalloc(int32_t n, int32_t nnz, const int32_t *d_row,
                                 const int32_t *d_col, const double *d_val,
                                 const double *d_d, const double *d_f, double *d_u,
                                 int k, void *stream);
/* y = alpha A x + beta y (CSRVector_product_adaptive_miniwarp,
 * src/matrix/CSR.cu:926-960). */
bcmg_status bcmg_k_spmv(int32_t n, int32_t nnz, const int32_t *d_row,
                        const int32_t *d_col, const double *d_val,
                        double alpha, const double *d_x, double beta,
                        double *d_y, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* BCMG_H */
