/* Minimal LAPACKE interface for building the reference sources as a CPU oracle (test infrastructure).
 * The reference calls LAPACKE_zheevd (src/hamiltonian.cpp:83-91); blas_shim.c forwards it to the
 * exported scipy_LAPACKE_zheevd of the OpenBLAS build bundled with scipy (LP64). */
#ifndef HHG_ORACLE_LAPACKE_SHIM_H
#define HHG_ORACLE_LAPACKE_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
typedef int lapack_int;
typedef struct { double re, im; } lapack_complex_double;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
lapack_int LAPACKE_zheevd(int matrix_layout, char jobz, char uplo, lapack_int n, lapack_complex_double* a,
                          lapack_int lda, double* w);
#ifdef __cplusplus
}
#endif
#endif
