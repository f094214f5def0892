/* Forwarders from the CBLAS / LAPACKE names the reference uses to the exported scipy_* names of
 * scipy's bundled OpenBLAS (the library is linked and called, never inspected). Test infrastructure. */
#include "cblas.h"
#include "lapacke.h"

extern void scipy_cblas_zgemm(int, int, int, int, int, int, const void*, const void*, int, const void*, int,
                              const void*, void*, int);
extern void scipy_cblas_zaxpy(int, const void*, const void*, int, void*, int);
extern void scipy_cblas_zcopy(int, const void*, int, void*, int);
extern int scipy_LAPACKE_zheevd(int, char, char, int, void*, int, double*);

void cblas_zgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n,
                 int k, const void* alpha, const void* a, int lda, const void* b, int ldb, const void* beta,
                 void* c, int ldc) {
  scipy_cblas_zgemm((int)order, (int)ta, (int)tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
void cblas_zaxpy(int n, const void* alpha, const void* x, int incx, void* y, int incy) {
  scipy_cblas_zaxpy(n, alpha, x, incx, y, incy);
}
void cblas_zcopy(int n, const void* x, int incx, void* y, int incy) { scipy_cblas_zcopy(n, x, incx, y, incy); }
lapack_int LAPACKE_zheevd(int layout, char jobz, char uplo, lapack_int n, lapack_complex_double* a,
                          lapack_int lda, double* w) {
  return scipy_LAPACKE_zheevd(layout, jobz, uplo, n, (void*)a, lda, w);
}
