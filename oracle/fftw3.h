/* Minimal FFTW-3 API shim (test infrastructure only).
 *
 * FFTW 3 is a third-party dependency of the reference (diskfft/Makefile:2-6, Homebrew,
 * no pinned version) that is not vendored and not installed here.  This header declares
 * exactly the subset that diskfft/src/kalnajs.hpp uses (lines 15, 35-45, 52, 57, 102-103,
 * 114) with FFTW's published semantics, backed by the project's own offt.c, so the
 * reference sources compile unmodified.  Results differ from FFTW's by round-off only. */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
double *fftw_alloc_real(size_t n);
fftw_complex *fftw_alloc_complex(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif
#endif
