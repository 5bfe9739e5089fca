// refbench — times the reference's own time step on the host cores.  TEST AND CPU-BASELINE
// INFRASTRUCTURE ONLY.  It drives diskfft/src/hydro.hpp and diskfft/src/kalnajs.hpp
// (compiled unmodified against the FFTW shim) through the loop body of
// diskfft/src/diskmain.cpp:100-109: timestep(0.3) -> potential -> forces -> step, and
// reports zone-updates/s = Nu*Nphi*steps / wall time of the timed steps (the reference's
// own metric, diskfft/README.md:39-43).
//
// usage: refbench Nu Nphi eps nthreads warmup steps
// prints one JSON line.
#include <chrono>
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

int main(int argc, char **argv) {
  if (argc < 7) { fprintf(stderr, "usage: refbench Nu Nphi eps nthreads warmup steps\n"); return 2; }
  int Nu = atoi(argv[1]), Nphi = atoi(argv[2]);
  double eps = atof(argv[3]);
  int nthreads = atoi(argv[4]), warm = atoi(argv[5]), steps = atoi(argv[6]);
#ifdef _OPENMP
  omp_set_num_threads(nthreads);
#endif
  double Rin = 0.25, Rout = 1.0, R0 = 0.45, w2 = 0.05, S0 = 0.372;
  DiskHydro hyd(Nu, Nphi, Rin, Rout, 0.25, 2.0, 0.6);
  KalnajsSolver grav(Nu, Nphi, Rin, Rout, eps, 1.0, nthreads);
  // standard disk with an m=2 seed (equilibrium support from the star and pressure only;
  // the timing does not depend on the exact rotation curve)
  for (int i = 0; i < Nu; ++i) {
    double R = hyd.R[i];
    double s0 = S0 * std::exp(-(R - R0) * (R - R0) / w2);
    double dPdR = 0.25 * 2.0 * s0 * s0 * (-2.0 * (R - R0) / w2);
    double v2 = 0.6 / R + (R / s0) * dPdR;
    for (int j = 0; j < Nphi; ++j) {
      double phi = (j + 0.5) * hyd.dphi;
      hyd.Sig[i * Nphi + j] = s0 * (1.0 + 1e-3 * std::cos(2.0 * phi));
      hyd.vR[i * Nphi + j] = 0.0;
      hyd.vp[i * Nphi + j] = v2 > 0 ? std::sqrt(v2) : 0.0;
    }
  }
  std::vector<double> Phi, gR, gp;
  auto one = [&]() {
    double dt = hyd.timestep(0.3);
    grav.potential(hyd.Sig, Phi);
    grav.forces(Phi, gR, gp);
    hyd.step(dt, &gR, &gp);
  };
  for (int s = 0; s < warm; ++s) one();
  auto t0 = std::chrono::steady_clock::now();
  for (int s = 0; s < steps; ++s) one();
  auto t1 = std::chrono::steady_clock::now();
  double sec = std::chrono::duration<double>(t1 - t0).count();
  printf("{\"Nu\": %d, \"Nphi\": %d, \"threads\": %d, \"steps\": %d, \"seconds\": %.6f, "
         "\"zone_updates_per_s\": %.6e}\n",
         Nu, Nphi, nthreads, steps, sec, (double)Nu * Nphi * steps / sec);
  return 0;
}
