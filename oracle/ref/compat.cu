// The legacy cuSPARSE routines of compat.h.  The two on BootCMatchG's solve
// path are implemented with the current generic API: cusparseDcsrmv
// (y = alpha op(A) x + beta y) with cusparseSpMV, and cusparseDcsr2csc with
// cusparseCsr2cscEx2.  The off-path ones report CUSPARSE_STATUS_NOT_SUPPORTED.
// TEST INFRASTRUCTURE ONLY.
#include <cuda_runtime.h>

#include "compat.h"

extern "C" {

cusparseStatus_t cusparseDcsrmv(cusparseHandle_t handle, cusparseOperation_t transA, int m,
                                int n, int nnz, const double *alpha,
                                const cusparseMatDescr_t, const double *val,
                                const int *rowPtr, const int *colInd, const double *x,
                                const double *beta, double *y) {
  cusparseSpMatDescr_t A;
  cusparseDnVecDescr_t X, Y;
  cusparseStatus_t st = cusparseCreateCsr(&A, m, n, nnz, const_cast<int *>(rowPtr),
                                          const_cast<int *>(colInd), const_cast<double *>(val),
                                          CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                                          CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F);
  if (st != CUSPARSE_STATUS_SUCCESS) return st;
  const bool t = transA != CUSPARSE_OPERATION_NON_TRANSPOSE;
  cusparseCreateDnVec(&X, t ? m : n, const_cast<double *>(x), CUDA_R_64F);
  cusparseCreateDnVec(&Y, t ? n : m, y, CUDA_R_64F);
  size_t bytes = 0;
  st = cusparseSpMV_bufferSize(handle, transA, alpha, A, X, beta, Y, CUDA_R_64F,
                               CUSPARSE_SPMV_ALG_DEFAULT, &bytes);
  void *buf = nullptr;
  if (st == CUSPARSE_STATUS_SUCCESS && bytes) cudaMalloc(&buf, bytes);
  if (st == CUSPARSE_STATUS_SUCCESS)
    st = cusparseSpMV(handle, transA, alpha, A, X, beta, Y, CUDA_R_64F,
                      CUSPARSE_SPMV_ALG_DEFAULT, buf);
  if (buf) cudaFree(buf);
  cusparseDestroyDnVec(X);
  cusparseDestroyDnVec(Y);
  cusparseDestroySpMat(A);
  return st;
}

cusparseStatus_t cusparseDcsr2csc(cusparseHandle_t handle, int m, int n, int nnz,
                                  const double *csrVal, const int *csrRowPtr,
                                  const int *csrColInd, double *cscVal, int *cscRowInd,
                                  int *cscColPtr, cusparseAction_t copyValues,
                                  cusparseIndexBase_t idxBase) {
  size_t bytes = 0;
  cusparseStatus_t st = cusparseCsr2cscEx2_bufferSize(
      handle, m, n, nnz, csrVal, csrRowPtr, csrColInd, cscVal, cscColPtr, cscRowInd,
      CUDA_R_64F, copyValues, idxBase, CUSPARSE_CSR2CSC_ALG1, &bytes);
  if (st != CUSPARSE_STATUS_SUCCESS) return st;
  void *buf = nullptr;
  if (bytes) cudaMalloc(&buf, bytes);
  st = cusparseCsr2cscEx2(handle, m, n, nnz, csrVal, csrRowPtr, csrColInd, cscVal, cscColPtr,
                          cscRowInd, CUDA_R_64F, copyValues, idxBase, CUSPARSE_CSR2CSC_ALG1,
                          buf);
  if (buf) cudaFree(buf);
  return st;
}

cusparseStatus_t cusparseCreateSolveAnalysisInfo(cusparseSolveAnalysisInfo_t *) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
cusparseStatus_t cusparseDestroySolveAnalysisInfo(cusparseSolveAnalysisInfo_t) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
cusparseStatus_t cusparseDcsr2dense(cusparseHandle_t, int, int, const cusparseMatDescr_t,
                                    const double *, const int *, const int *, double *, int) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
cusparseStatus_t cusparseXcsrgemmNnz(cusparseHandle_t, cusparseOperation_t, cusparseOperation_t,
                                     int, int, int, const cusparseMatDescr_t, int, const int *,
                                     const int *, const cusparseMatDescr_t, int, const int *,
                                     const int *, const cusparseMatDescr_t, int *, int *) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
cusparseStatus_t cusparseDcsrgemm(cusparseHandle_t, cusparseOperation_t, cusparseOperation_t,
                                  int, int, int, const cusparseMatDescr_t, int, const double *,
                                  const int *, const int *, const cusparseMatDescr_t, int,
                                  const double *, const int *, const int *,
                                  const cusparseMatDescr_t, double *, const int *, int *) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
cusparseStatus_t cusparseDcsrsv_analysis(cusparseHandle_t, cusparseOperation_t, int, int,
                                         const cusparseMatDescr_t, const double *, const int *,
                                         const int *, cusparseSolveAnalysisInfo_t) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
cusparseStatus_t cusparseDcsrsv_solve(cusparseHandle_t, cusparseOperation_t, int,
                                      const double *, const cusparseMatDescr_t, const double *,
                                      const int *, const int *, cusparseSolveAnalysisInfo_t,
                                      const double *, double *) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
cusparseStatus_t cusparseDcsrilu0(cusparseHandle_t, cusparseOperation_t, int,
                                  const cusparseMatDescr_t, double *, const int *, const int *,
                                  cusparseSolveAnalysisInfo_t) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}

}  // extern "C"
