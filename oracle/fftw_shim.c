/* FFTW-3 API shim implementation over offt (test infrastructure only). */
#include "fftw3.h"
#include "offt.h"
#include <stdlib.h>

struct fftw_plan_s {
  int kind; /* 0 = r2c, 1 = c2r */
  int n0, n1, nthreads;
  void *in, *out;
};

static int g_nthreads = 1;

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads > 0 ? nthreads : 1; }
void fftw_cleanup_threads(void) {}

double *fftw_alloc_real(size_t n) {
  void *p = NULL;
  if (posix_memalign(&p, 64, n * sizeof(double) + 64)) return NULL;
  return (double *)p;
}
fftw_complex *fftw_alloc_complex(size_t n) {
  void *p = NULL;
  if (posix_memalign(&p, 64, n * sizeof(fftw_complex) + 64)) return NULL;
  return (fftw_complex *)p;
}
void fftw_free(void *p) { free(p); }

static fftw_plan mk(int kind, int n0, int n1, void *in, void *out) {
  fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
  p->kind = kind; p->n0 = n0; p->n1 = n1; p->in = in; p->out = out; p->nthreads = g_nthreads;
  return p;
}
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags) {
  (void)flags;
  return mk(0, n0, n1, in, out);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags) {
  (void)flags;
  return mk(1, n0, n1, in, out);
}
void fftw_execute(const fftw_plan p) {
  if (p->kind == 0) offt_r2c_2d(p->n0, p->n1, (const double *)p->in, (double *)p->out, p->nthreads);
  else offt_c2r_2d(p->n0, p->n1, (const double *)p->in, (double *)p->out, p->nthreads);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }
