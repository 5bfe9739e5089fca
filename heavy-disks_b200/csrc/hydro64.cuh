// Plain-method (FP64) hydro: one fused kernel per time step.
//
// It restates DiskHydro::step (diskfft/src/hydro.hpp:63-70) =
//   source (:73-96) -> transportR (:99-140) -> transportPhi (:143-179) -> floor (:69)
// with the self-gravity forces of KalnajsSolver::forces (kalnajs.hpp:65-80) computed
// from the potential in the same pass, and the CFL reduction of DiskHydro::timestep
// (:48-61) for the NEXT step fused into the epilogue.  The floating-point expressions
// keep the reference's operation order, so results agree to round-off.
//
// Tiling: a CTA owns TI x TJ output cells and stages a (TI+6) x (TJ+6) halo region of
// Sigma, vR, vphi, Phi in shared memory (3 cells each side: transportPhi needs +-2 cells
// of the transportR output, which needs +-2 rows of the source output, which needs +-1
// cell of pressure / potential).  phi is periodic (wrapped loads); at the radial edges
// the reference's clamps, one-sided differences, zero slopes and zero boundary fluxes
// apply, so halo rows outside [0, Nu) are never consumed.
#pragma once

#include "dg_common.cuh"

namespace dg {

struct Geom64 {
  const double *R, *Rf, *Vol;
  // per-row constants: -GM*/R^2, 1/R, 1/(R[ip]-R[im]), 1/Vol, 1/(Rf[i+1]-Rf[i]), 1/(R dphi)
  const double *gstar, *invR, *invdRc, *invVol, *invdR, *invdl;
  // per-face constants: 1/(Rf[f]-Rf[f-1]), 1/(Rf[f+1]-Rf[f])
  const double *invdRl, *invdRr;
  int Nu, Nphi;
  double dphi, du, Kpoly, gamma, gmstar;
  double inv2dphi, invdu, inv2du;
  int gamma2;  // gamma == 2: P = K s^2, cs^2 = 2 K s without pow
};

// Which self-gravity the kernel applies (hydro.hpp:86-88).
enum ForceMode : int { kForceNone = 0, kForcePhi = 1, kForceArrays = 2 };

constexpr int kTI = 8, kTJ = 32, kH = 3;
constexpr int kLI = kTI + 2 * kH, kLJ = kTJ + 2 * kH;  // loaded region
constexpr int kSI = kTI + 4, kSJ = kTJ + 4;            // source-stage region
constexpr int kHydroThreads = 256;

__device__ __forceinline__ double vanleer64(double a, double b) {  // hydro.hpp:16-18
  return (a * b > 0.0) ? 2.0 * a * b / (a + b) : 0.0;
}
__device__ __forceinline__ double dmax_ref(double a, double b) { return (a < b) ? b : a; }  // std::max

__device__ __forceinline__ double pres64(const Geom64 &g, double s) {  // hydro.hpp:46
  return g.gamma2 ? g.Kpoly * (s * s) : g.Kpoly * pow(s, g.gamma);
}
__device__ __forceinline__ double cs2_64(const Geom64 &g, double s) {  // hydro.hpp:45
  return g.gamma2 ? g.gamma * g.Kpoly * s : g.gamma * g.Kpoly * pow(s, g.gamma - 1.0);
}
// (|vR| + cs)/dR + (|vp| + cs)/(R dphi)  (hydro.hpp:54-57)
__device__ __forceinline__ double cfl_rate64(const Geom64 &g, int i, double s, double vr, double vp) {
  double cs = sqrt(cs2_64(g, dmax_ref(s, 1e-12)));
  double sR = (fabs(vr) + cs) * g.invdR[i];
  double sp = (fabs(vp) + cs) * g.invdl[i];
  return sR + sp;
}

}  // namespace dg
