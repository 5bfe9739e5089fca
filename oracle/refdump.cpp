// refdump — drives the reference's own DiskHydro / KalnajsSolver classes
// (diskfft/src/hydro.hpp, diskfft/src/kalnajs.hpp, compiled unmodified against the
// FFTW shim) and dumps fields for golden fixtures.  TEST INFRASTRUCTURE ONLY.
//
// The initial condition and loop body restate diskfft/src/diskmain.cpp:28-63 and
// :100-109 (timestep 0.3 -> potential -> forces -> step), without the tlim clip.
//
// usage: refdump Nu Nphi eps selfgrav amp nsteps out.bin [nthreads [gamma_gas Kpoly S0]]
// The optional physics arguments replace the constants of diskmain.cpp:28-29 (the
// reference's DiskHydro takes K and Gamma as constructor arguments, hydro.hpp:28), so
// fixtures can pin the general-Gamma pressure and sound-speed branches (hydro.hpp:45-46).
// out.bin: int32 Nu, Nphi, nsteps, selfgrav; float64 eps, amp, mD; then float64 arrays
//   Sig0 vR0 vp0 Phi0 gR0 gp0 (Nu*Nphi each, initial state and its gravity),
//   dt[nsteps], SigN vRN vpN, c0 ph0 c2 ph2 (modes of the final state).
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "hydro.hpp"
#include "kalnajs.hpp"

using namespace diskfft;

static void wr(FILE *f, const std::vector<double> &v) { fwrite(v.data(), sizeof(double), v.size(), f); }

int main(int argc, char **argv) {
  if (argc < 8) {
    fprintf(stderr, "usage: refdump Nu Nphi eps selfgrav amp nsteps out.bin [nthreads [gamma_gas Kpoly S0]]\n");
    return 2;
  }
  int Nu = atoi(argv[1]), Nphi = atoi(argv[2]);
  double eps = atof(argv[3]);
  int selfgrav = atoi(argv[4]);
  double amp = atof(argv[5]);
  int nsteps = atoi(argv[6]);
  int nthreads = argc > 8 ? atoi(argv[8]) : 1;
#ifdef _OPENMP
  omp_set_num_threads(nthreads);
#endif
  double Rin = 0.25, Rout = 1.0, R0 = 0.45, w2 = 0.05, S0 = 0.372;
  double Kpoly = 0.25, gamma_gas = 2.0, gmstar = 0.6, G = 1.0;
  if (argc > 11) {
    gamma_gas = atof(argv[9]);
    Kpoly = atof(argv[10]);
    S0 = atof(argv[11]);
  }
  DiskHydro hyd(Nu, Nphi, Rin, Rout, Kpoly, gamma_gas, gmstar);
  KalnajsSolver grav(Nu, Nphi, Rin, Rout, eps, G, nthreads);
  auto Sigma0 = [&](double R) { return S0 * std::exp(-(R - R0) * (R - R0) / w2); };
  std::vector<double> gR_eq(Nu * Nphi, 0.0), gp_eq, Phi_eq, Sig_axi(Nu * Nphi);
  for (int i = 0; i < Nu; ++i)
    for (int j = 0; j < Nphi; ++j) Sig_axi[i * Nphi + j] = Sigma0(hyd.R[i]);
  std::vector<double> gRdisk(Nu, 0.0);
  if (selfgrav) {
    grav.potential(Sig_axi, Phi_eq);
    grav.forces(Phi_eq, gR_eq, gp_eq);
    for (int i = 0; i < Nu; ++i) {
      double s = 0; for (int j = 0; j < Nphi; ++j) s += gR_eq[i * Nphi + j];
      gRdisk[i] = s / Nphi;
    }
  }
  for (int i = 0; i < Nu; ++i) {
    double R = hyd.R[i];
    double dSig = Sigma0(R) * (-2.0 * (R - R0) / w2);
    double dPdR = Kpoly * gamma_gas * std::pow(Sigma0(R), gamma_gas - 1.0) * dSig;
    double v2 = gmstar / R + (R / Sigma0(R)) * dPdR - R * gRdisk[i];
    double vphi = (v2 > 0) ? std::sqrt(v2) : 0.0;
    for (int j = 0; j < Nphi; ++j) {
      double phi = (j + 0.5) * hyd.dphi;
      hyd.Sig[i * Nphi + j] = Sigma0(R) * (1.0 + amp * std::cos(2.0 * phi));
      hyd.vR[i * Nphi + j] = 0.0;
      hyd.vp[i * Nphi + j] = vphi;
    }
  }
  double mD = 0.0;
  for (int i = 0; i < Nu; ++i) {
    double dA = hyd.R[i] * (hyd.Rf[i + 1] - hyd.Rf[i]) * hyd.dphi;
    for (int j = 0; j < Nphi; ++j) mD += hyd.Sig[i * Nphi + j] * dA;
  }
  auto Cm = [&](int m, double &mag, double &phase) {
    double re = 0, im = 0;
    for (int i = 0; i < Nu; ++i) {
      double dA = hyd.R[i] * (hyd.Rf[i + 1] - hyd.Rf[i]) * hyd.dphi;
      for (int j = 0; j < Nphi; ++j) {
        double phi = (j + 0.5) * hyd.dphi;
        re += hyd.Sig[i * Nphi + j] * std::cos(m * phi) * dA;
        im -= hyd.Sig[i * Nphi + j] * std::sin(m * phi) * dA;
      }
    }
    mag = std::sqrt(re * re + im * im) / mD;
    phase = std::atan2(im, re);
  };

  FILE *f = fopen(argv[7], "wb");
  if (!f) { perror("fopen"); return 1; }
  int hdr[4] = {Nu, Nphi, nsteps, selfgrav};
  fwrite(hdr, sizeof(int), 4, f);
  double dh[3] = {eps, amp, mD};
  fwrite(dh, sizeof(double), 3, f);
  std::vector<double> Phi, gR, gp;
  grav.potential(hyd.Sig, Phi);
  grav.forces(Phi, gR, gp);
  wr(f, hyd.Sig); wr(f, hyd.vR); wr(f, hyd.vp); wr(f, Phi); wr(f, gR); wr(f, gp);
  std::vector<double> dts;
  for (int s = 0; s < nsteps; ++s) {
    double dt = hyd.timestep(0.3);
    dts.push_back(dt);
    if (selfgrav) {
      grav.potential(hyd.Sig, Phi);
      grav.forces(Phi, gR, gp);
      hyd.step(dt, &gR, &gp);
    } else {
      hyd.step(dt);
    }
  }
  wr(f, dts);
  wr(f, hyd.Sig); wr(f, hyd.vR); wr(f, hyd.vp);
  double c0, ph0, c2, ph2;
  Cm(0, c0, ph0); Cm(2, c2, ph2);
  double md[4] = {c0, ph0, c2, ph2};
  fwrite(md, sizeof(double), 4, f);
  fclose(f);
  return 0;
}
