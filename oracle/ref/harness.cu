// BootCMatchG's own solve path, compiled from the unmodified sources of the
// reference tree (the unity header below pulls them in; the Makefile adds the
// separately compiled files and compat.h/compat.cu for the cuSPARSE routines
// CUDA 11 removed), behind a small C entry layer:
//   ref_pair_aggregate  one matching + aggregation sweep with the reference's
//                       kernels (matchingPairAggregation, src/AMG/
//                       matchingAggregation.cu:181-208, and the W of
//                       Matching::makeAH/toMaximumProductMatrix);
//   ref_galerkin        R (A P) with nsparse (matchingAggregation.cu:239-244);
//   ref_solve           the stock solve(A, p, rhs) (src/SOLVER/solver.cu:20).
// TEST INFRASTRUCTURE ONLY: it generates golden fixtures that pin the oracle
// and times the reference's GPU solve; nothing in the product links it.
#define VERBOSE 0
#include "BootCMatchG.h"

namespace {

CSR *wrap_host(int n, int nnz, const int *row, const int *col, const double *val) {
  CSR *A = CSRm::init(n, n, nnz, false, false, false);
  A->row = const_cast<int *>(row);
  A->col = const_cast<int *>(col);
  A->val = const_cast<double *>(val);
  return A;
}

void drop_host_wrapper(CSR *A) {
  cusparseDestroyMatDescr(*A->descr);
  std::free(A->descr);
  std::free(A);
}

}  // namespace

extern "C" {

int ref_pair_aggregate(int n, int nnz, const int *row, const int *col, const double *val,
                       const double *w_host, int *agg, double *p, int *nc, int *match,
                       double *W) {
  CSR *Ah = wrap_host(n, nnz, row, col, val);
  CSR *A = CSRm::copyToDevice(Ah);
  vector<vtype> *w = Vector::init<vtype>(n, true, true);
  cudaMemcpy(w->val, w_host, sizeof(double) * n, cudaMemcpyHostToDevice);
  matchingAggregationContext::initContext(n);
  if (W) {
    CSR *AH = Matching::makeAH(A, w);
    Matching::toMaximumProductMatrix(AH);
    cudaMemcpy(W, AH->val, sizeof(double) * (nnz - n), cudaMemcpyDeviceToHost);
    CSRm::free(AH);
  }
  // Matching::suitor = weights + suitor kernel + unsymFix; then the
  // aggregation kernel on that matching, as matchingPairAggregation does.
  vector<itype> *M = Matching::suitor(A, w);
  cudaMemcpy(match, M->val, sizeof(int) * n, cudaMemcpyDeviceToHost);
  CSR *P = CSRm::init(n, 1, n, true, true, false);
  scalar<itype> *nuns = Scalar::init<itype>(0, true);
  gridblock gb = gb1d(n, aggregate_BLOCKSIZE);
  _aggregate_symmetric<<<gb.g, gb.b>>>(n, A->row, P->val, M->val, P->col, w->val, nuns->val);
  int *nl = Scalar::getvalueFromDevice(nuns);
  *nc = nl[0];
  cudaMemcpy(agg, P->col, sizeof(int) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(p, P->val, sizeof(double) * n, cudaMemcpyDeviceToHost);
  std::free(nl);
  Scalar::free(nuns);
  CSRm::free(P);
  Vector::free(M);
  Vector::free(w);
  CSRm::free(A);
  matchingAggregationContext::freeContext();
  drop_host_wrapper(Ah);
  return static_cast<int>(cudaDeviceSynchronize());
}

int ref_galerkin(int n, int nnz, const int *row, const int *col, const double *val, int nc,
                 const int *agg, const double *p, int *crow, int *cnnz, int *ccol,
                 double *cval) {
  handles *h = Handles::init();
  CSR *Ah = wrap_host(n, nnz, row, col, val);
  CSR *A = CSRm::copyToDevice(Ah);
  CSR *Ph = CSRm::init(n, nc, n, true, false, false);
  for (int i = 0; i <= n; ++i) Ph->row[i] = i;
  for (int i = 0; i < n; ++i) {
    Ph->col[i] = agg[i];
    Ph->val[i] = p[i];
  }
  CSR *P = CSRm::copyToDevice(Ph);
  CSR *R = CSRm::T(h->cusparse_h0, P);
  CSR *AP = CSRm::CSRCSR_product(h->cusparse_h0, A, P);
  CSR *Ac = CSRm::CSRCSR_product(h->cusparse_h0, R, AP);
  *cnnz = Ac->nnz;
  cudaMemcpy(crow, Ac->row, sizeof(int) * (nc + 1), cudaMemcpyDeviceToHost);
  if (ccol) cudaMemcpy(ccol, Ac->col, sizeof(int) * Ac->nnz, cudaMemcpyDeviceToHost);
  if (cval) cudaMemcpy(cval, Ac->val, sizeof(double) * Ac->nnz, cudaMemcpyDeviceToHost);
  CSRm::free(Ac);
  CSRm::free(AP);
  CSRm::free(R);
  CSRm::free(P);
  CSRm::free(Ph);
  CSRm::free(A);
  drop_host_wrapper(Ah);
  Handles::free(h);
  return static_cast<int>(cudaDeviceSynchronize());
}

// prm: solver_type, max_hrc, aggrsweeps, aggrtype, max_levels, cycle_type,
// coarse_solver, relax_type, relaxnumber_coarse, prerelax, postrelax, itnlim;
// dprm: conv_ratio, rtol.
int ref_solve(int n, int nnz, const int *row, const int *col, const double *val,
              const int *prm, const double *dprm, const double *b, double *x) {
  params pp;
  pp.solver_type = prm[0];
  pp.max_hrc = prm[1];
  pp.aggrsweeps = prm[2];
  pp.aggrtype = prm[3];
  pp.max_levels = prm[4];
  pp.cycle_type = prm[5];
  pp.coarse_solver = prm[6];
  pp.relax_type = prm[7];
  pp.relaxnumber_coarse = prm[8];
  pp.prerelax_sweeps = prm[9];
  pp.postrelax_sweeps = prm[10];
  pp.itnlim = prm[11];
  pp.conv_ratio = dprm[0];
  pp.rtol = dprm[1];
  pp.matchtype = 3;
  CSR *Ah = wrap_host(n, nnz, row, col, val);
  vector<vtype> *rhs = Vector::init<vtype>(n, true, true);
  cudaMemcpy(rhs->val, b, sizeof(double) * n, cudaMemcpyHostToDevice);
  vector<vtype> *sol = solve(Ah, pp, rhs);
  cudaMemcpy(x, sol->val, sizeof(double) * n, cudaMemcpyDeviceToHost);
  Vector::free(sol);
  Vector::free(rhs);
  drop_host_wrapper(Ah);
  return static_cast<int>(cudaDeviceSynchronize());
}

}  // extern "C"
