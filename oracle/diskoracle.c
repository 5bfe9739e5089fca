/* diskoracle — plain-C restatement of the reference diskfft time step.
 * TEST INFRASTRUCTURE ONLY (see diskoracle.h).  Loop structure and floating-point
 * operation order follow the cited reference lines so that, compiled with the same
 * flags, results match the reference sources bit for bit. */
#include "diskoracle.h"
#include "offt.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static double *zalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* hydro.hpp:16-18 */
static inline double vanleer(double a, double b) { return (a * b > 0.0) ? 2.0 * a * b / (a + b) : 0.0; }

/* hydro.hpp:28-43 */
orc_hydro *orc_hydro_create(int Nu, int Nphi, double Rin, double Rout, double K, double g, double GMstar) {
  orc_hydro *h = (orc_hydro *)calloc(1, sizeof(*h));
  h->Nu = Nu; h->Nphi = Nphi; h->Kpoly = K; h->gamma_gas = g; h->gmstar = GMstar; h->nthreads = 1;
  h->umin = log(Rin); h->umax = log(Rout);
  h->du = (h->umax - h->umin) / Nu; h->dphi = 2.0 * M_PI / Nphi;
  h->R = zalloc(Nu); h->Rf = zalloc(Nu + 1); h->Vol = zalloc(Nu);
  for (int i = 0; i <= Nu; ++i) h->Rf[i] = exp(h->umin + i * h->du);
  for (int i = 0; i < Nu; ++i) {
    h->R[i] = exp(h->umin + (i + 0.5) * h->du);
    h->Vol[i] = h->R[i] * (h->Rf[i + 1] - h->Rf[i]) * h->dphi;
  }
  size_t n = (size_t)Nu * Nphi, nf = (size_t)(Nu + 1) * Nphi;
  h->Sig = zalloc(n); h->vR = zalloc(n); h->vp = zalloc(n);
  h->wA = zalloc(n); h->wB = zalloc(n); h->mR = zalloc(n); h->mp = zalloc(n);
  h->Fm = zalloc(nf); h->FmR = zalloc(nf); h->FmP = zalloc(nf);
  return h;
}

void orc_hydro_destroy(orc_hydro *h) {
  if (!h) return;
  free(h->R); free(h->Rf); free(h->Vol); free(h->Sig); free(h->vR); free(h->vp);
  free(h->wA); free(h->wB); free(h->mR); free(h->mp); free(h->Fm); free(h->FmR); free(h->FmP);
  free(h);
}

double *orc_hydro_field(orc_hydro *h, int which) {
  switch (which) {
    case 0: return h->Sig; case 1: return h->vR; case 2: return h->vp;
    case 3: return h->R; case 4: return h->Rf; case 5: return h->Vol;
  }
  return NULL;
}

void orc_set_threads(orc_hydro *h, int nthreads) { h->nthreads = nthreads > 0 ? nthreads : 1; }

#define IDX(i, j) ((size_t)(i) * Nphi + (j))

/* hydro.hpp:45-46 */
static inline double cs2(const orc_hydro *h, double s) { return h->gamma_gas * h->Kpoly * pow(s, h->gamma_gas - 1.0); }
static inline double pres(const orc_hydro *h, double s) { return h->Kpoly * pow(s, h->gamma_gas); }

/* hydro.hpp:48-61 */
double orc_timestep(const orc_hydro *h, double cfl) {
  const int Nu = h->Nu, Nphi = h->Nphi;
  double dtinv = 1e-30;
#pragma omp parallel for reduction(max : dtinv) schedule(static) num_threads(h->nthreads)
  for (int i = 0; i < Nu; ++i) {
    double dR = h->Rf[i + 1] - h->Rf[i];
    for (int j = 0; j < Nphi; ++j) {
      double s = h->Sig[IDX(i, j)];
      double cs = sqrt(cs2(h, (s < 1e-12) ? 1e-12 : s)); /* std::max(s, 1e-12) */
      double sR = (fabs(h->vR[IDX(i, j)]) + cs) / dR;
      double sp = (fabs(h->vp[IDX(i, j)]) + cs) / (h->R[i] * h->dphi);
      if (sR + sp > dtinv) dtinv = sR + sp;
    }
  }
  return cfl / dtinv;
}

/* hydro.hpp:73-96 */
void orc_source(orc_hydro *h, double dt, const double *gR_sg, const double *gp_sg) {
  const int Nu = h->Nu, Nphi = h->Nphi;
  double *nvR = h->wA, *nvp = h->wB;
  const double *Sig = h->Sig, *vR = h->vR, *vp = h->vp, *R = h->R;
#pragma omp parallel for schedule(static) num_threads(h->nthreads)
  for (int i = 0; i < Nu; ++i) {
    int im = i - 1 > 0 ? i - 1 : 0, ip = i + 1 < Nu - 1 ? i + 1 : Nu - 1;
    double dRc = R[ip] - R[im];
    for (int j = 0; j < Nphi; ++j) {
      size_t c = IDX(i, j);
      size_t jm = IDX(i, (j - 1 + Nphi) % Nphi), jp = IDX(i, (j + 1) % Nphi);
      double s = Sig[c];
      double dPdR = (pres(h, Sig[IDX(ip, j)]) - pres(h, Sig[IDX(im, j)])) / dRc;
      double dPdphi = (pres(h, Sig[jp]) - pres(h, Sig[jm])) / (2.0 * h->dphi);
      double gR = -h->gmstar / (R[i] * R[i]);
      double gp = 0.0;
      if (gR_sg) gR += gR_sg[c];
      if (gp_sg) gp += gp_sg[c];
      double aR = -dPdR / s + gR + vp[c] * vp[c] / R[i];
      double ap = -(1.0 / (s * R[i])) * dPdphi + gp - vR[c] * vp[c] / R[i];
      nvR[c] = vR[c] + dt * aR;
      nvp[c] = vp[c] + dt * ap;
    }
  }
  double *t;
  t = h->vR; h->vR = h->wA; h->wA = t;
  t = h->vp; h->vp = h->wB; h->wB = t;
}

/* hydro.hpp:107-110 */
static inline double slopeR(const orc_hydro *h, const double *a, int i, int j) {
  const int Nu = h->Nu, Nphi = h->Nphi;
  if (i <= 0 || i >= Nu - 1) return 0.0;
  return vanleer(a[IDX(i + 1, j)] - a[IDX(i, j)], a[IDX(i, j)] - a[IDX(i - 1, j)]);
}

/* hydro.hpp:99-140 */
void orc_transportR(orc_hydro *h, double dt) {
  const int Nu = h->Nu, Nphi = h->Nphi;
  double *Sig = h->Sig, *vR = h->vR, *vp = h->vp, *mR = h->mR, *mp = h->mp;
  double *Fm = h->Fm, *FmR = h->FmR, *FmP = h->FmP;
  const double *Rf = h->Rf;
  const size_t n = (size_t)Nu * Nphi;
#pragma omp parallel for schedule(static) num_threads(h->nthreads)
  for (size_t k = 0; k < n; ++k) { mR[k] = Sig[k] * vR[k]; mp[k] = Sig[k] * vp[k]; }
  for (int j = 0; j < Nphi; ++j) {
    Fm[j] = FmR[j] = FmP[j] = 0.0;
    Fm[(size_t)Nu * Nphi + j] = FmR[(size_t)Nu * Nphi + j] = FmP[(size_t)Nu * Nphi + j] = 0.0;
  }
#pragma omp parallel for schedule(static) num_threads(h->nthreads)
  for (int f = 1; f < Nu; ++f) {
    double Af = Rf[f] * h->dphi;
    double dRl = Rf[f] - Rf[f - 1], dRr = Rf[f + 1] - Rf[f];
    for (int j = 0; j < Nphi; ++j) {
      double vf = 0.5 * (vR[IDX(f - 1, j)] + vR[IDX(f, j)]);
      double sf, vRf, vpf;
      if (vf > 0) {
        sf = Sig[IDX(f - 1, j)] + 0.5 * slopeR(h, Sig, f - 1, j) * (1.0 - vf * dt / dRl);
        vRf = vR[IDX(f - 1, j)] + 0.5 * slopeR(h, vR, f - 1, j) * (1.0 - vf * dt / dRl);
        vpf = vp[IDX(f - 1, j)] + 0.5 * slopeR(h, vp, f - 1, j) * (1.0 - vf * dt / dRl);
      } else {
        sf = Sig[IDX(f, j)] - 0.5 * slopeR(h, Sig, f, j) * (1.0 + vf * dt / dRr);
        vRf = vR[IDX(f, j)] - 0.5 * slopeR(h, vR, f, j) * (1.0 + vf * dt / dRr);
        vpf = vp[IDX(f, j)] - 0.5 * slopeR(h, vp, f, j) * (1.0 + vf * dt / dRr);
      }
      double fm = vf * sf * Af;
      Fm[(size_t)f * Nphi + j] = fm; FmR[(size_t)f * Nphi + j] = fm * vRf; FmP[(size_t)f * Nphi + j] = fm * vpf;
    }
  }
#pragma omp parallel for schedule(static) num_threads(h->nthreads)
  for (int i = 0; i < Nu; ++i)
    for (int j = 0; j < Nphi; ++j) {
      size_t c = IDX(i, j);
      double ns = Sig[c] + dt * (Fm[(size_t)i * Nphi + j] - Fm[(size_t)(i + 1) * Nphi + j]) / h->Vol[i];
      double nmR = mR[c] + dt * (FmR[(size_t)i * Nphi + j] - FmR[(size_t)(i + 1) * Nphi + j]) / h->Vol[i];
      double nmP = mp[c] + dt * (FmP[(size_t)i * Nphi + j] - FmP[(size_t)(i + 1) * Nphi + j]) / h->Vol[i];
      double d = (ns < 1e-10) ? 1e-10 : ns; /* std::max(ns, 1e-10) */
      Sig[c] = ns; vR[c] = nmR / d; vp[c] = nmP / d;
    }
}

/* hydro.hpp:146-149 */
static inline double slopeP(const orc_hydro *h, const double *a, int i, int j) {
  const int Nphi = h->Nphi;
  int jm = (j - 1 + Nphi) % Nphi, jp = (j + 1) % Nphi;
  return vanleer(a[IDX(i, jp)] - a[IDX(i, j)], a[IDX(i, j)] - a[IDX(i, jm)]);
}

/* hydro.hpp:143-179 */
void orc_transportPhi(orc_hydro *h, double dt) {
  const int Nu = h->Nu, Nphi = h->Nphi;
  double *Sig = h->Sig, *vR = h->vR, *vp = h->vp, *mR = h->mR, *mp = h->mp;
  double *Fm = h->Fm, *FmR = h->FmR, *FmP = h->FmP;
  const size_t n = (size_t)Nu * Nphi;
#pragma omp parallel for schedule(static) num_threads(h->nthreads)
  for (size_t k = 0; k < n; ++k) { mR[k] = Sig[k] * vR[k]; mp[k] = Sig[k] * vp[k]; }
#pragma omp parallel for schedule(static) num_threads(h->nthreads)
  for (int i = 0; i < Nu; ++i) {
    double dl = h->R[i] * h->dphi, Aface = h->Rf[i + 1] - h->Rf[i];
    for (int j = 0; j < Nphi; ++j) {
      int jm = (j - 1 + Nphi) % Nphi;
      double vf = 0.5 * (vp[IDX(i, jm)] + vp[IDX(i, j)]);
      double sf, vRf, vpf;
      if (vf > 0) {
        sf = Sig[IDX(i, jm)] + 0.5 * slopeP(h, Sig, i, jm) * (1.0 - vf * dt / dl);
        vRf = vR[IDX(i, jm)] + 0.5 * slopeP(h, vR, i, jm) * (1.0 - vf * dt / dl);
        vpf = vp[IDX(i, jm)] + 0.5 * slopeP(h, vp, i, jm) * (1.0 - vf * dt / dl);
      } else {
        sf = Sig[IDX(i, j)] - 0.5 * slopeP(h, Sig, i, j) * (1.0 + vf * dt / dl);
        vRf = vR[IDX(i, j)] - 0.5 * slopeP(h, vR, i, j) * (1.0 + vf * dt / dl);
        vpf = vp[IDX(i, j)] - 0.5 * slopeP(h, vp, i, j) * (1.0 + vf * dt / dl);
      }
      double fm = vf * sf * Aface;
      Fm[IDX(i, j)] = fm; FmR[IDX(i, j)] = fm * vRf; FmP[IDX(i, j)] = fm * vpf;
    }
  }
#pragma omp parallel for schedule(static) num_threads(h->nthreads)
  for (int i = 0; i < Nu; ++i)
    for (int j = 0; j < Nphi; ++j) {
      size_t c = IDX(i, j), jp = IDX(i, (j + 1) % Nphi);
      double ns = Sig[c] + dt * (Fm[c] - Fm[jp]) / h->Vol[i];
      double nmR = mR[c] + dt * (FmR[c] - FmR[jp]) / h->Vol[i];
      double nmP = mp[c] + dt * (FmP[c] - FmP[jp]) / h->Vol[i];
      double d = (ns < 1e-10) ? 1e-10 : ns; /* std::max(ns, 1e-10) */
      Sig[c] = ns; vR[c] = nmR / d; vp[c] = nmP / d;
    }
}

/* hydro.hpp:63-70 */
void orc_step(orc_hydro *h, double dt, const double *gR, const double *gp) {
  orc_source(h, dt, gR, gp);
  orc_transportR(h, dt);
  orc_transportPhi(h, dt);
  const size_t n = (size_t)h->Nu * h->Nphi;
#pragma omp parallel for schedule(static) num_threads(h->nthreads)
  for (size_t k = 0; k < n; ++k) h->Sig[k] = (h->Sig[k] < 1e-10) ? 1e-10 : h->Sig[k];
}

/* kalnajs.hpp:105-116 */
static void build_kernel(orc_kalnajs *k) {
  const int M = k->M, Nphi = k->Nphi, Nc = k->Nc;
  for (int p = 0; p < M; ++p) {
    int ioff = (p <= M / 2) ? p : p - M;
    double Du = ioff * k->du;
    for (int q = 0; q < Nphi; ++q) {
      double Dphi = q * k->dphi;
      k->rbuf[(size_t)p * Nphi + q] = 1.0 / sqrt(2.0 * cosh(Du) - 2.0 * cos(Dphi) + k->eps);
    }
  }
  offt_r2c_2d(M, Nphi, k->rbuf, k->cbuf, k->nthreads);
  memcpy(k->Khat, k->cbuf, sizeof(double) * 2 * (size_t)M * Nc);
}

/* kalnajs.hpp:25-42 */
orc_kalnajs *orc_kalnajs_create(int Nu, int Nphi, double Rin, double Rout, double eps, double G, int nthreads) {
  orc_kalnajs *k = (orc_kalnajs *)calloc(1, sizeof(*k));
  k->Nu = Nu; k->Nphi = Nphi; k->M = 2 * Nu; k->Nc = Nphi / 2 + 1; k->eps = eps; k->G = G;
  k->nthreads = nthreads > 0 ? nthreads : 1;
  k->umin = log(Rin); k->umax = log(Rout);
  k->du = (k->umax - k->umin) / Nu; k->dphi = 2.0 * M_PI / Nphi;
  k->R = zalloc(Nu); k->sqrtR = zalloc(Nu); k->R32 = zalloc(Nu);
  for (int i = 0; i < Nu; ++i) {
    k->R[i] = exp(k->umin + (i + 0.5) * k->du);
    k->sqrtR[i] = sqrt(k->R[i]); k->R32[i] = k->R[i] * k->sqrtR[i];
  }
  k->rbuf = zalloc((size_t)k->M * Nphi);
  k->cbuf = zalloc(2 * (size_t)k->M * k->Nc);
  k->Khat = zalloc(2 * (size_t)k->M * k->Nc);
  build_kernel(k);
  return k;
}

void orc_kalnajs_destroy(orc_kalnajs *k) {
  if (!k) return;
  free(k->R); free(k->sqrtR); free(k->R32); free(k->rbuf); free(k->cbuf); free(k->Khat);
  free(k);
}

const double *orc_khat(const orc_kalnajs *k) { return k->Khat; }

/* kalnajs.hpp:48-63 */
void orc_potential(orc_kalnajs *k, const double *Sigma, double *Phi) {
  const int Nu = k->Nu, Nphi = k->Nphi, M = k->M, Nc = k->Nc;
  for (size_t q = 0; q < (size_t)M * Nphi; ++q) k->rbuf[q] = 0.0;
  for (int i = 0; i < Nu; ++i)
    for (int j = 0; j < Nphi; ++j) k->rbuf[IDX(i, j)] = k->R32[i] * Sigma[IDX(i, j)];
  offt_r2c_2d(M, Nphi, k->rbuf, k->cbuf, k->nthreads);
  for (size_t q = 0; q < (size_t)M * Nc; ++q) {
    double a = k->cbuf[2 * q], b = k->cbuf[2 * q + 1], c = k->Khat[2 * q], d = k->Khat[2 * q + 1];
    k->cbuf[2 * q] = a * c - b * d; k->cbuf[2 * q + 1] = a * d + b * c;
  }
  offt_c2r_2d(M, Nphi, k->cbuf, k->rbuf, k->nthreads);
  double pref = -k->G * k->du * k->dphi / ((double)M * Nphi);
  for (int i = 0; i < Nu; ++i)
    for (int j = 0; j < Nphi; ++j) Phi[IDX(i, j)] = pref * k->rbuf[IDX(i, j)] / k->sqrtR[i];
}

/* kalnajs.hpp:65-80 */
void orc_forces(const orc_kalnajs *k, const double *Phi, double *gR, double *gphi) {
  const int Nu = k->Nu, Nphi = k->Nphi;
#pragma omp parallel for schedule(static) num_threads(k->nthreads)
  for (int i = 0; i < Nu; ++i)
    for (int j = 0; j < Nphi; ++j) {
      int jm = (j - 1 + Nphi) % Nphi, jp = (j + 1) % Nphi;
      double dPhidphi = (Phi[IDX(i, jp)] - Phi[IDX(i, jm)]) / (2.0 * k->dphi);
      double dPhidu;
      if (i == 0) dPhidu = (Phi[IDX(i + 1, j)] - Phi[IDX(i, j)]) / k->du;
      else if (i == Nu - 1) dPhidu = (Phi[IDX(i, j)] - Phi[IDX(i - 1, j)]) / k->du;
      else dPhidu = (Phi[IDX(i + 1, j)] - Phi[IDX(i - 1, j)]) / (2.0 * k->du);
      gR[IDX(i, j)] = -dPhidu / k->R[i];
      gphi[IDX(i, j)] = -dPhidphi / k->R[i];
    }
}

/* kalnajs.hpp:83-99 */
void orc_potential_direct(const orc_kalnajs *k, const double *Sigma, double *Phi) {
  const int Nu = k->Nu, Nphi = k->Nphi;
  double pref = -k->G * k->du * k->dphi;
#pragma omp parallel for schedule(static) num_threads(k->nthreads)
  for (int i = 0; i < Nu; ++i)
    for (int j = 0; j < Nphi; ++j) {
      double V = 0.0;
      for (int ip = 0; ip < Nu; ++ip) {
        double Du = (i - ip) * k->du;
        for (int jp = 0; jp < Nphi; ++jp) {
          double Dphi = (j - jp) * k->dphi;
          V += k->R32[ip] * Sigma[IDX(ip, jp)] / sqrt(2.0 * cosh(Du) - 2.0 * cos(Dphi) + k->eps);
        }
      }
      Phi[IDX(i, j)] = pref * V / k->sqrtR[i];
    }
}

/* diskmain.cpp:17-29 */
void orc_params_default(orc_params *p) {
  p->Nu = 128; p->Nphi = 128; p->eps = 0.02; p->tlim = 8.0; p->selfgrav = 1; p->amp = 1e-3; p->nthreads = 1;
  p->Rin = 0.25; p->Rout = 1.0; p->R0 = 0.45; p->w2 = 0.05; p->S0 = 0.372;
  p->Kpoly = 0.25; p->gamma_gas = 2.0; p->gmstar = 0.6; p->G = 1.0;
  p->phase0 = 0.0;
}

/* diskmain.cpp:34 */
static inline double sigma0(const orc_params *p, double R) { return p->S0 * exp(-(R - p->R0) * (R - p->R0) / p->w2); }

/* diskmain.cpp:36-63 */
void orc_init_standard(const orc_params *p, orc_hydro *h, orc_kalnajs *k) {
  const int Nu = h->Nu, Nphi = h->Nphi;
  double *gRdisk = zalloc(Nu);
  if (p->selfgrav) {
    size_t n = (size_t)Nu * Nphi;
    double *Sig_axi = zalloc(n), *Phi_eq = zalloc(n), *gR_eq = zalloc(n), *gp_eq = zalloc(n);
    for (int i = 0; i < Nu; ++i)
      for (int j = 0; j < Nphi; ++j) Sig_axi[IDX(i, j)] = sigma0(p, h->R[i]);
    orc_potential(k, Sig_axi, Phi_eq);
    orc_forces(k, Phi_eq, gR_eq, gp_eq);
    for (int i = 0; i < Nu; ++i) {
      double s = 0;
      for (int j = 0; j < Nphi; ++j) s += gR_eq[IDX(i, j)];
      gRdisk[i] = s / Nphi;
    }
    free(Sig_axi); free(Phi_eq); free(gR_eq); free(gp_eq);
  }
  for (int i = 0; i < Nu; ++i) {
    double R = h->R[i];
    double dSig = sigma0(p, R) * (-2.0 * (R - p->R0) / p->w2);
    double dPdR = p->Kpoly * p->gamma_gas * pow(sigma0(p, R), p->gamma_gas - 1.0) * dSig;
    double v2 = p->gmstar / R + (R / sigma0(p, R)) * dPdR - R * gRdisk[i];
    double vphi = (v2 > 0) ? sqrt(v2) : 0.0;
    for (int j = 0; j < Nphi; ++j) {
      double phi = (j + 0.5) * h->dphi;
      /* phase0 == 0 reproduces the reference seed cos(2 phi) exactly */
      double c = p->phase0 == 0.0 ? cos(2.0 * phi) : cos(2.0 * (phi - p->phase0));
      h->Sig[IDX(i, j)] = sigma0(p, R) * (1.0 + p->amp * c);
      h->vR[IDX(i, j)] = 0.0;
      h->vp[IDX(i, j)] = vphi;
    }
  }
  free(gRdisk);
}

/* diskmain.cpp:66-70 */
double orc_disk_mass(const orc_hydro *h) {
  const int Nu = h->Nu, Nphi = h->Nphi;
  double mD = 0.0;
  for (int i = 0; i < Nu; ++i) {
    double dA = h->R[i] * (h->Rf[i + 1] - h->Rf[i]) * h->dphi;
    for (int j = 0; j < Nphi; ++j) mD += h->Sig[IDX(i, j)] * dA;
  }
  return mD;
}

/* diskmain.cpp:72-84 */
void orc_cm(const orc_hydro *h, int m, double mD, double *mag, double *phase) {
  const int Nu = h->Nu, Nphi = h->Nphi;
  double re = 0, im = 0;
  for (int i = 0; i < Nu; ++i) {
    double dA = h->R[i] * (h->Rf[i + 1] - h->Rf[i]) * h->dphi;
    for (int j = 0; j < Nphi; ++j) {
      double phi = (j + 0.5) * h->dphi;
      re += h->Sig[IDX(i, j)] * cos(m * phi) * dA;
      im -= h->Sig[IDX(i, j)] * sin(m * phi) * dA;
    }
  }
  *mag = sqrt(re * re + im * im) / mD;
  *phase = atan2(im, re);
}

/* diskmain.cpp:86-112 */
long orc_run(const orc_params *p, orc_hydro *h, orc_kalnajs *k, long max_steps, double *t_out, FILE *modes) {
  const size_t n = (size_t)h->Nu * h->Nphi;
  double mD = orc_disk_mass(h);
  double *Phi = zalloc(n), *gR = zalloc(n), *gp = zalloc(n);
  if (modes) fprintf(modes, "# t  |C0|  |C2|  arg(C2)\n");
  double t = 0.0, dtout = 0.25, tnext = 0.0;
  double c0, c2, ph2, ph0;
  long step = 0;
  while (t < p->tlim && (max_steps < 0 || step < max_steps)) {
    if (t >= tnext - 1e-12) {
      orc_cm(h, 0, mD, &c0, &ph0);
      orc_cm(h, 2, mD, &c2, &ph2);
      if (modes) { fprintf(modes, "%.5f %.6e %.6e %.6e\n", t, c0, c2, ph2); fflush(modes); }
      tnext += dtout;
    }
    double dt = orc_timestep(h, 0.3);
    if (t + dt > p->tlim) dt = p->tlim - t;
    if (p->selfgrav) {
      orc_potential(k, h->Sig, Phi);
      orc_forces(k, Phi, gR, gp);
      orc_step(h, dt, gR, gp);
    } else {
      orc_step(h, dt, NULL, NULL);
    }
    t += dt; ++step;
  }
  free(Phi); free(gR); free(gp);
  if (t_out) *t_out = t;
  return step;
}
