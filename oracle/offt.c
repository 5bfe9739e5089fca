/* offt — mixed-radix Stockham FFT for the oracle (test infrastructure only).
 * Stand-in for FFTW's r2c/c2r 2-D transforms used by diskfft/src/kalnajs.hpp:39-40,52,57,114.
 * See offt.h for conventions. */
#include "offt.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OFFT_MAXF 64

struct offt_plan1d {
  int n;
  int nf;
  int fac[OFFT_MAXF];
  double *root; /* root[2t], root[2t+1] = cos, -sin of 2 pi t / n  (forward roots) */
};

offt_plan1d *offt_plan1d_create(int n) {
  if (n < 1) return NULL;
  offt_plan1d *p = (offt_plan1d *)calloc(1, sizeof(*p));
  p->n = n;
  int m = n;
  while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
  for (int f = 3; m > 1; f += 2)
    while (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
  p->root = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (int t = 0; t < n; ++t) {
    /* reduce the angle to the first octant by symmetry for accuracy */
    double a = 2.0 * M_PI * (double)t / (double)n;
    p->root[2 * t] = cos(a);
    p->root[2 * t + 1] = -sin(a);
  }
  return p;
}

void offt_plan1d_destroy(offt_plan1d *p) {
  if (!p) return;
  free(p->root);
  free(p);
}

/* complex multiply helpers on (re,im) pairs */
static inline void cmul(double ar, double ai, double br, double bi, double *cr, double *ci) {
  *cr = ar * br - ai * bi;
  *ci = ar * bi + ai * br;
}

void offt_exec1d(const offt_plan1d *p, double *data, double *work, int sign) {
  const int n = p->n;
  if (n == 1) return;
  double *x = data, *y = work;
  double vr[OFFT_MAXF * 4], vi[OFFT_MAXF * 4]; /* radix scratch; generic radix <= 256 */
  double *gr = NULL, *gi = NULL;
  int Ns = 1;
  for (int s = 0; s < p->nf; ++s) {
    const int R = p->fac[s];
    const int m = n / R;
    const int tstep = n / (Ns * R);
    double *ur = vr, *ui = vi;
    if (R > OFFT_MAXF * 4) {
      gr = (double *)realloc(gr, sizeof(double) * 2 * R);
      gi = gr + R;
      ur = gr; ui = gi;
    }
    for (int j = 0; j < m; ++j) {
      const int k = j % Ns;
      for (int r = 0; r < R; ++r) {
        double a = x[2 * (j + r * m)], b = x[2 * (j + r * m) + 1];
        if (r && k) {
          long t = ((long)r * k * tstep) % n;
          double wr = p->root[2 * t], wi = sign < 0 ? p->root[2 * t + 1] : -p->root[2 * t + 1];
          cmul(a, b, wr, wi, &a, &b);
        }
        ur[r] = a; ui[r] = b;
      }
      double orr[4], oii[4];
      double *outr = orr, *outi = oii;
      if (R == 2) {
        orr[0] = ur[0] + ur[1]; oii[0] = ui[0] + ui[1];
        orr[1] = ur[0] - ur[1]; oii[1] = ui[0] - ui[1];
      } else if (R == 4) {
        double a0r = ur[0] + ur[2], a0i = ui[0] + ui[2];
        double a1r = ur[0] - ur[2], a1i = ui[0] - ui[2];
        double a2r = ur[1] + ur[3], a2i = ui[1] + ui[3];
        double dr = ur[1] - ur[3], di = ui[1] - ui[3];
        /* a3 = d * (-i) forward, d * (+i) inverse */
        double a3r = sign < 0 ? di : -di, a3i = sign < 0 ? -dr : dr;
        orr[0] = a0r + a2r; oii[0] = a0i + a2i;
        orr[2] = a0r - a2r; oii[2] = a0i - a2i;
        orr[1] = a1r + a3r; oii[1] = a1i + a3i;
        orr[3] = a1r - a3r; oii[3] = a1i - a3i;
      } else if (R == 3) {
        const double h = 0.86602540378443864676; /* sqrt(3)/2 */
        double t1r = ur[1] + ur[2], t1i = ui[1] + ui[2];
        double t2r = ur[0] - 0.5 * t1r, t2i = ui[0] - 0.5 * t1i;
        double dr = ur[1] - ur[2], di = ui[1] - ui[2];
        /* t3 = (v1 - v2) * (-i h) forward, (+i h) inverse */
        double t3r = sign < 0 ? h * di : -h * di, t3i = sign < 0 ? -h * dr : h * dr;
        orr[0] = ur[0] + t1r; oii[0] = ui[0] + t1i;
        orr[1] = t2r + t3r; oii[1] = t2i + t3i;
        orr[2] = t2r - t3r; oii[2] = t2i - t3i;
      } else {
        /* generic O(R^2) butterfly using the n-th roots: exp(-2 pi i rq/R) = root[(rq mod R) * (n/R)] */
        static __thread double tr_[OFFT_MAXF * 4], ti_[OFFT_MAXF * 4];
        double *tr = tr_, *ti = ti_, *big = NULL;
        if (R > OFFT_MAXF * 4) { big = (double *)malloc(sizeof(double) * 2 * R); tr = big; ti = big + R; }
        const int nr = n / R;
        for (int q = 0; q < R; ++q) {
          double sr = 0.0, si = 0.0;
          for (int r = 0; r < R; ++r) {
            long t = ((long)r * q % R) * nr;
            double wr = p->root[2 * t], wi = sign < 0 ? p->root[2 * t + 1] : -p->root[2 * t + 1];
            sr += ur[r] * wr - ui[r] * wi;
            si += ur[r] * wi + ui[r] * wr;
          }
          tr[q] = sr; ti[q] = si;
        }
        const int base = (j / Ns) * Ns * R + k;
        for (int q = 0; q < R; ++q) { y[2 * (base + q * Ns)] = tr[q]; y[2 * (base + q * Ns) + 1] = ti[q]; }
        free(big);
        continue;
      }
      const int base = (j / Ns) * Ns * R + k;
      for (int q = 0; q < R; ++q) { y[2 * (base + q * Ns)] = outr[q]; y[2 * (base + q * Ns) + 1] = outi[q]; }
    }
    Ns *= R;
    double *tmp = x; x = y; y = tmp;
  }
  free(gr);
  if (x != data) memcpy(data, x, sizeof(double) * 2 * (size_t)n);
}

void offt_r2c_2d(int n0, int n1, const double *in, double *out, int nthreads) {
  const int nc = n1 / 2 + 1;
  offt_plan1d *p1 = offt_plan1d_create(n1), *p0 = offt_plan1d_create(n0);
  (void)nthreads;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)(n0 > n1 ? n0 : n1));
    double *wrk = (double *)malloc(sizeof(double) * 2 * (size_t)(n0 > n1 ? n0 : n1));
#pragma omp for schedule(static)
    for (int i = 0; i < n0; ++i) {
      for (int j = 0; j < n1; ++j) { buf[2 * j] = in[(size_t)i * n1 + j]; buf[2 * j + 1] = 0.0; }
      offt_exec1d(p1, buf, wrk, -1);
      memcpy(out + 2 * (size_t)i * nc, buf, sizeof(double) * 2 * nc);
    }
#pragma omp for schedule(static)
    for (int k = 0; k < nc; ++k) {
      for (int i = 0; i < n0; ++i) {
        buf[2 * i] = out[2 * ((size_t)i * nc + k)];
        buf[2 * i + 1] = out[2 * ((size_t)i * nc + k) + 1];
      }
      offt_exec1d(p0, buf, wrk, -1);
      for (int i = 0; i < n0; ++i) {
        out[2 * ((size_t)i * nc + k)] = buf[2 * i];
        out[2 * ((size_t)i * nc + k) + 1] = buf[2 * i + 1];
      }
    }
    free(buf); free(wrk);
  }
  offt_plan1d_destroy(p1); offt_plan1d_destroy(p0);
}

void offt_c2r_2d(int n0, int n1, const double *in, double *out, int nthreads) {
  const int nc = n1 / 2 + 1;
  offt_plan1d *p1 = offt_plan1d_create(n1), *p0 = offt_plan1d_create(n0);
  double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n0 * nc);
  (void)nthreads;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)(n0 > n1 ? n0 : n1));
    double *wrk = (double *)malloc(sizeof(double) * 2 * (size_t)(n0 > n1 ? n0 : n1));
#pragma omp for schedule(static)
    for (int k = 0; k < nc; ++k) {
      for (int i = 0; i < n0; ++i) {
        buf[2 * i] = in[2 * ((size_t)i * nc + k)];
        buf[2 * i + 1] = in[2 * ((size_t)i * nc + k) + 1];
      }
      offt_exec1d(p0, buf, wrk, +1);
      for (int i = 0; i < n0; ++i) {
        tmp[2 * ((size_t)i * nc + k)] = buf[2 * i];
        tmp[2 * ((size_t)i * nc + k) + 1] = buf[2 * i + 1];
      }
    }
#pragma omp for schedule(static)
    for (int i = 0; i < n0; ++i) {
      const double *row = tmp + 2 * (size_t)i * nc;
      for (int k = 0; k < nc; ++k) { buf[2 * k] = row[2 * k]; buf[2 * k + 1] = row[2 * k + 1]; }
      for (int k = nc; k < n1; ++k) { buf[2 * k] = row[2 * (n1 - k)]; buf[2 * k + 1] = -row[2 * (n1 - k) + 1]; }
      offt_exec1d(p1, buf, wrk, +1);
      for (int j = 0; j < n1; ++j) out[(size_t)i * n1 + j] = buf[2 * j];
    }
    free(buf); free(wrk);
  }
  free(tmp);
  offt_plan1d_destroy(p1); offt_plan1d_destroy(p0);
}
