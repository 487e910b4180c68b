// Declarations of the legacy cuSPARSE routines BootCMatchG calls that CUDA 11
// removed, so its unmodified sources compile against CUDA 12.9.  Force-included
// (-include) into every translation unit of the reference build in
// oracle/ref/Makefile.  Names and argument lists follow the reference's call
// sites (src/matrix/CSR.cu:281,378,551-585,875,1026-1032,
// src/AMG/relaxation.cu:339-341).  TEST INFRASTRUCTURE ONLY.
#pragma once

#include <cfloat>  // src/matrix/vector.cu uses DBL_EPSILON without including it
#include <cusparse.h>

typedef struct bcmg_ref_csrsv_info *cusparseSolveAnalysisInfo_t;

#ifdef __cplusplus
extern "C" {
#endif

cusparseStatus_t cusparseCreateSolveAnalysisInfo(cusparseSolveAnalysisInfo_t *info);
cusparseStatus_t cusparseDestroySolveAnalysisInfo(cusparseSolveAnalysisInfo_t info);
cusparseStatus_t cusparseDcsrmv(cusparseHandle_t handle, cusparseOperation_t transA, int m,
                                int n, int nnz, const double *alpha,
                                const cusparseMatDescr_t descrA, const double *val,
                                const int *rowPtr, const int *colInd, const double *x,
                                const double *beta, double *y);
cusparseStatus_t cusparseDcsr2csc(cusparseHandle_t handle, int m, int n, int nnz,
                                  const double *csrVal, const int *csrRowPtr,
                                  const int *csrColInd, double *cscVal, int *cscRowInd,
                                  int *cscColPtr, cusparseAction_t copyValues,
                                  cusparseIndexBase_t idxBase);
cusparseStatus_t cusparseDcsr2dense(cusparseHandle_t handle, int m, int n,
                                    const cusparseMatDescr_t descrA, const double *val,
                                    const int *rowPtr, const int *colInd, double *A, int lda);
cusparseStatus_t cusparseXcsrgemmNnz(cusparseHandle_t handle, cusparseOperation_t transA,
                                     cusparseOperation_t transB, int m, int n, int k,
                                     const cusparseMatDescr_t descrA, int nnzA,
                                     const int *rowPtrA, const int *colIndA,
                                     const cusparseMatDescr_t descrB, int nnzB,
                                     const int *rowPtrB, const int *colIndB,
                                     const cusparseMatDescr_t descrC, int *rowPtrC,
                                     int *nnzTotal);
cusparseStatus_t cusparseDcsrgemm(cusparseHandle_t handle, cusparseOperation_t transA,
                                  cusparseOperation_t transB, int m, int n, int k,
                                  const cusparseMatDescr_t descrA, int nnzA,
                                  const double *valA, const int *rowPtrA, const int *colIndA,
                                  const cusparseMatDescr_t descrB, int nnzB,
                                  const double *valB, const int *rowPtrB, const int *colIndB,
                                  const cusparseMatDescr_t descrC, double *valC,
                                  const int *rowPtrC, int *colIndC);
cusparseStatus_t cusparseDcsrsv_analysis(cusparseHandle_t handle, cusparseOperation_t transA,
                                         int m, int nnz, const cusparseMatDescr_t descrA,
                                         const double *val, const int *rowPtr,
                                         const int *colInd, cusparseSolveAnalysisInfo_t info);
cusparseStatus_t cusparseDcsrsv_solve(cusparseHandle_t handle, cusparseOperation_t transA,
                                      int m, const double *alpha,
                                      const cusparseMatDescr_t descrA, const double *val,
                                      const int *rowPtr, const int *colInd,
                                      cusparseSolveAnalysisInfo_t info, const double *f,
                                      double *x);
cusparseStatus_t cusparseDcsrilu0(cusparseHandle_t handle, cusparseOperation_t trans, int m,
                                  const cusparseMatDescr_t descrA, double *val,
                                  const int *rowPtr, const int *colInd,
                                  cusparseSolveAnalysisInfo_t info);

#ifdef __cplusplus
}
#endif
