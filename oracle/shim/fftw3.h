/* Minimal FFTW3-compatible interface used to build the reference sources as a CPU oracle.
 *
 * Test infrastructure only. The reference (src/fftw_helper.cpp:5-33, src/solver.cpp:1439-1440,
 * src/velocity.cpp:51-54, src/operator.cpp:46-48,70-72, src/solver_kspace.cpp:124-126) calls FFTW3's
 * fftw_plan_dft_2d / fftw_execute / fftw_malloc / fftw_free. FFTW3 is an un-vendored third-party
 * dependency (no pinned version; README "FFTW3 >= 3.3") that is absent from this image, so these
 * entry points are served by fft_shim.c: an FP64 mixed-radix Stockham FFT with FFTW's conventions
 * (sign -1 forward, +1 backward, unnormalised, row-major n0 x n1 with n1 contiguous). */
#ifndef HHG_ORACLE_FFTW3_SHIM_H
#define HHG_ORACLE_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct oracle_fft_plan* fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);
void* fftw_malloc(size_t n);
void fftw_free(void* p);
/* Shim extensions (not FFTW API): an in-place 2D transform on caller memory, used by the tests. */
void oracle_fft2d(int n0, int n1, double* data, int sign);
#ifdef __cplusplus
}
#endif
#endif
