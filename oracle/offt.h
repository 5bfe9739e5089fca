/* offt — CPU FFT used by the oracle (test infrastructure only).
 *
 * A mixed-radix Stockham autosort FFT for complex double data of any length
 * (explicit radix 4, 2, 3, 5 butterflies; any other prime factor uses an O(p^2)
 * butterfly).  It backs two things that both stand in for FFTW, which the
 * reference links (diskfft/Makefile:6) but which is not present here:
 *   - the FFTW-API shim in fftw3.h / fftw_shim.c that lets the reference's own
 *     sources (diskfft/src/kalnajs.hpp, diskmain.cpp, test_kalnajs.cpp) compile
 *     unmodified, and
 *   - the plain-C restatement of the time step in diskoracle.c.
 * Conventions follow FFTW: forward uses exp(-2 pi i jk/n), no normalisation on
 * either direction; r2c keeps n1/2+1 outputs of the last dimension; c2r assumes
 * Hermitian symmetry and ignores the imaginary parts of self-conjugate bins.
 */
#ifndef OFFT_H
#define OFFT_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct offt_plan1d offt_plan1d;

offt_plan1d *offt_plan1d_create(int n);
void offt_plan1d_destroy(offt_plan1d *p);
/* In-place complex transform of interleaved (re,im) data; sign -1 forward, +1 inverse.
 * work must hold 2*n doubles. */
void offt_exec1d(const offt_plan1d *p, double *data, double *work, int sign);

/* 2-D real-to-complex: in n0 x n1 real (row-major), out n0 x (n1/2+1) complex. */
void offt_r2c_2d(int n0, int n1, const double *in, double *out, int nthreads);
/* 2-D complex-to-real (unnormalised inverse): in n0 x (n1/2+1) complex, out n0 x n1 real.
 * The input is not modified. */
void offt_c2r_2d(int n0, int n1, const double *in, double *out, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
