/*
 * oracle.h -- CPU FP64 restatement of BootCMatchG's alpha-AMG + FCG path.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is the parity checker and the timed
 * CPU baseline; nothing in the product library links, loads or calls it.
 *
 * Parity status: partially pinned.  The reference ships no tests, golden
 * vectors or sample matrices, and its solve path does not build unmodified
 * with CUDA 12 (legacy cuSPARSE routines).  oracle/ref/ compiles its sources
 * with a compatibility shim into oracle/_ref/libref.so, which pins this
 * restatement where the reference's own code could run: one matching +
 * aggregation sweep recorded on a B200 and the reference's sequential suitor
 * matcher on three more inputs with tie-free weights (tests/golden/, checked
 * by tests/test_ref_fixtures.py), and its host code run on the CPU
 * (tests/test_ref_io.py: the Matrix-Market reader and writer, the settings
 * file, the coarsest-size rule and the grid-sweep table).  The rest is
 * pinned by the reference's own invariants (a valid symmetric matching,
 * every vertex in one aggregate, P^T P = I on good aggregates,
 * A_c = P^T A P), by hand-checked known answers, and by a second
 * restatement in plain Python on small cases (weights, matching,
 * aggregates, Galerkin, the cycle and composites, the bootstrap's inner
 * iterations, flexible CG) that this code must equal bit for bit
 * (tests/test_cpu_oracle.py).
 *
 * Every function follows the reference file:line cited beside it.  Where
 * the reference is nondeterministic (atomicAdd aggregate numbering, FP64
 * atomics in the Galerkin product, racy suitor ties) the oracle fixes one
 * valid execution; the GPU library implements the same one:
 *   - matching: the suitor (proposer-optimal) outcome under strict keys
 *     (weight, id) -- the race-free reading of suitor.cu:118-214;
 *   - unsymFix second pass: all claims resolved in lockstep;
 *   - aggregate numbering: ascending by the aggregate's smallest vertex;
 *   - Galerkin sums: terms (p_i p_j) a_ij summed in ascending
 *     (min(i,j), max(i,j), i) order, which keeps A_c exactly symmetric.
 */
#ifndef BCMG_ORACLE_H
#define BCMG_ORACLE_H

#include "../include/bcmg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_handle orc_handle;

void orc_set_threads(int nthreads);

/* maxcoarsesize = (int)(40 n^(1/3)) (BuildData::setMaxCoarseSize) and the
 * grid-sweep table of the first max_levels - 1 levels
 * (ApplyData::setGridSweeps); returns the number of entries written. */
int32_t orc_max_coarse_size(int32_t n);
int orc_grid_sweeps(int cycle_type, int max_levels, int32_t *out);
int orc_get_threads(void);

int orc_setup(const bcmg_csr *A, const bcmg_params *p, orc_handle **out);
/* One hierarchy (adaptiveCoarsening) from a given smooth vector w, without
 * the bootstrap loop: checks a bootstrapped hierarchy from identical inputs. */
int orc_setup_from_w(const bcmg_csr *A, const bcmg_params *p, const double *w,
                     orc_handle **out);
int orc_solve(orc_handle *h, const double *b, double *x, bcmg_solve_info *info);
int orc_precond_apply(orc_handle *h, const double *r, double *z);
void orc_destroy(orc_handle *h);
/* Runs `iters` FCG iterations from x (used to time a bounded sample). */
int orc_fcg_sample(orc_handle *h, const double *b, double *x, int iters,
                   double *seconds);

int orc_hierarchy_count(const orc_handle *h, int *num_hrc, double *est_ratio);
int orc_hierarchy_info(const orc_handle *h, int hrc, int *num_levels,
                       double *op_cmplx, double *op_wcmplx, double *avg_cratio);
int orc_level_info(const orc_handle *h, int hrc, int level, int32_t *n,
                   int32_t *nnz, int32_t *n_coarse);
int orc_level_copy(const orc_handle *h, int hrc, int level, int32_t *row,
                   int32_t *col, double *val, double *D, double *M,
                   int32_t *agg, double *p, double *w);

/* Single steps on host arrays (same contracts as the bcmg_k_* entries). */
int orc_pair_aggregate(int32_t n, int32_t nnz, const int32_t *row,
                       const int32_t *col, const double *val, const double *w,
                       int32_t *agg, double *p, int32_t *n_coarse, double *W,
                       int32_t *suitor, int32_t *match);
int orc_galerkin(int32_t n, int32_t nnz, const int32_t *row, const int32_t *col,
                 const double *val, int32_t n_coarse, const int32_t *agg,
                 const double *p, int32_t *crow, int32_t *c_nnz, int32_t *ccol,
                 double *cval);
int orc_relax(int32_t n, const int32_t *row, const int32_t *col,
              const double *val, const double *d, const double *f, double *u,
              int k);
int orc_spmv(int32_t n, const int32_t *row, const int32_t *col, const double *val,
             double alpha, const double *x, double beta, double *y);
/* Sequential greedy matching on descending key (W, max id, min id) for a
 * symmetric weight matrix; match[v] = partner or -1.  Self-check of the
 * suitor restatement. */
int orc_greedy_match(int32_t n, const int32_t *row, const int32_t *col,
                     const double *W, int32_t *match);

#ifdef __cplusplus
}
#endif

#endif
