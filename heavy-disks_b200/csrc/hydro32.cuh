// Mixed-precision hydro: the same time step as hydro.hpp:63-179, written for an FP32
// perturbation (sigma, u, w) = (Sigma - Sigma0(R), vR, vphi - V0(R)) about an FP64
// axisymmetric basic state (Sigma0, V0, vR0 = 0).
//
// Every operator of the reference is rewritten so that the large basic-state terms
// cancel analytically instead of numerically:
//   source:  aR = a0(R) + (dP0/dR sigma / Sigma0 - d(dP)/dR) / Sigma + dgR + (2 V0 + w) w / R,
//            with a0 the FP64 residual of the discrete radial balance of the basic state and
//            dP = P(Sigma0 + sigma) - P(Sigma0) evaluated without cancellation;
//   R sweep: slopes of the full fields use FP64 basic-state differences; the phi-momentum
//            flux is carried as F (vphi_f - V0(cell)) so the V0 F part cancels exactly;
//   phi sweep: the mass flux is carried as A (V0 sigma_f + dv_f Sigma_f) (the V0 Sigma0 A
//            part is the same on every face of a row), the phi-momentum flux as F w_f.
// Reconstruction, limiter, upwinding, reflecting radial faces, periodic phi, the Sigma
// floor and the CFL rate follow the reference expressions.
#pragma once

#include <cuda_bf16.h>

#include "dg_common.cuh"

namespace dg {

// Per-row constants (FP64 values rounded once to FP32) and per-face constants.
struct Rows32 {
  // rows i in [0, Nu)
  const float *R, *invR, *invdRc, *dP0dR, *S0, *invS0, *V0, *a0, *dR, *dl, *Aphi, *invVol, *R32, *P0;
  const double *S0d, *V0d, *Rd, *dAd;  // FP64 copies for the global sums
  // faces f in [0, Nu]
  const float *Af, *dRl, *dRr, *dV, *dS0;
  const float *invdR, *invdl, *invdRl, *invdRr;  // reciprocals (rows, rows, faces, faces)
  // the packed hydro kernel's row constants, row-major [Nu + 24][20]: row r holds the
  // constants of i = r - 3 (hydro32p.cuh), zero outside the grid, so one tile's rows are
  // one contiguous copy
  const float *rowtab;
  int Nu, Nphi;
  float dphi, inv2dphi, invdu, inv2du, Kpoly, gamma, gmstar;
  int gamma2;  // gamma == 2: P = K Sigma^2 exactly
};

// hydro.hpp:16-18; a*b > 0 means |a + b| >= max(|a|, |b|) > 0, so the fast divide is safe
__device__ __forceinline__ float vanleer32(float a, float b) {
  return (a * b > 0.f) ? __fdividef(2.f * a * b, a + b) : 0.f;
}

// P(Sigma0 + s) - P(Sigma0) for P = K Sigma^gamma
__device__ __forceinline__ float dpres32(const Rows32 &g, int i, float s) {
  if (g.gamma2) return g.Kpoly * s * (2.f * g.S0[i] + s);
  return g.P0[i] * expm1f(g.gamma * log1pf(s * g.invS0[i]));
}

__device__ __forceinline__ float cfl_rate32(const Rows32 &g, int i, float sig, float u, float w) {
  float s = g.S0[i] + sig;
  s = (s < 1e-12f) ? 1e-12f : s;
  float cs2 = g.gamma2 ? g.gamma * g.Kpoly * s : g.gamma * g.Kpoly * powf(s, g.gamma - 1.f);
  float cs = sqrtf(cs2);
  return (fabsf(u) + cs) * g.invdR[i] + (fabsf(g.V0[i] + w) + cs) * g.invdl[i];
}

}  // namespace dg
