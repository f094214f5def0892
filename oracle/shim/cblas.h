/* Minimal CBLAS interface for building the reference sources as a CPU oracle (test infrastructure).
 * The reference calls cblas_zgemm (src/operator.cpp:183-210,242-269) and, in dead solver variants,
 * cblas_zaxpy / cblas_zcopy (src/solver.cpp:183-1158). They are forwarded by blas_shim.c to the
 * exported scipy_cblas_* symbols of the OpenBLAS build bundled with scipy (LP64). */
#ifndef HHG_ORACLE_CBLAS_SHIM_H
#define HHG_ORACLE_CBLAS_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
void cblas_zgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n,
                 int k, const void* alpha, const void* a, int lda, const void* b, int ldb, const void* beta,
                 void* c, int ldc);
void cblas_zaxpy(int n, const void* alpha, const void* x, int incx, void* y, int incy);
void cblas_zcopy(int n, const void* x, int incx, void* y, int incy);
#ifdef __cplusplus
}
#endif
#endif
