// cusparse_legacy.h — placeholders for the legacy cuSPARSE routines that the
// reference's GPU-side functions (hybrid_makeYbus, hybrid_makeB in
// src/powerflow/makeYbus.h:372-510 and makeB.h:109-309) call and that CUDA 12 removed
// (csrgemm, csrgeam, gthr).  TEST INFRASTRUCTURE: only oracle/ref_pf.cu includes it.
// The reference's CPU path (mkl_*), which is what oracle/_ref/librefpf.so runs, never
// reaches them; they exist so that the reference's headers compile and link
// unmodified, and each returns CUSPARSE_STATUS_NOT_SUPPORTED if ever called.
#ifndef REFSHIM_CUSPARSE_LEGACY_H_
#define REFSHIM_CUSPARSE_LEGACY_H_

#include <cuComplex.h>
#include <cusparse.h>

inline cusparseStatus_t cusparseXcsrgemmNnz(cusparseHandle_t, cusparseOperation_t, cusparseOperation_t, int, int, int,
                                            const cusparseMatDescr_t, int, const int*, const int*,
                                            const cusparseMatDescr_t, int, const int*, const int*,
                                            const cusparseMatDescr_t, int*, int*) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
inline cusparseStatus_t cusparseZcsrgemm(cusparseHandle_t, cusparseOperation_t, cusparseOperation_t, int, int, int,
                                         const cusparseMatDescr_t, int, const cuDoubleComplex*, const int*, const int*,
                                         const cusparseMatDescr_t, int, const cuDoubleComplex*, const int*, const int*,
                                         const cusparseMatDescr_t, cuDoubleComplex*, const int*, int*) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
inline cusparseStatus_t cusparseXcsrgeamNnz(cusparseHandle_t, int, int, const cusparseMatDescr_t, int, const int*,
                                            const int*, const cusparseMatDescr_t, int, const int*, const int*,
                                            const cusparseMatDescr_t, int*, int*) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
inline cusparseStatus_t cusparseZcsrgeam(cusparseHandle_t, int, int, const cuDoubleComplex*, const cusparseMatDescr_t,
                                         int, const cuDoubleComplex*, const int*, const int*, const cuDoubleComplex*,
                                         const cusparseMatDescr_t, int, const cuDoubleComplex*, const int*, const int*,
                                         const cusparseMatDescr_t, cuDoubleComplex*, int*, int*) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
inline cusparseStatus_t cusparseZgthr(cusparseHandle_t, int, const cuDoubleComplex*, cuDoubleComplex*, const int*,
                                      cusparseIndexBase_t) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
inline cusparseStatus_t cusparseDgthr(cusparseHandle_t, int, const double*, double*, const int*, cusparseIndexBase_t) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}

#endif  // REFSHIM_CUSPARSE_LEGACY_H_
