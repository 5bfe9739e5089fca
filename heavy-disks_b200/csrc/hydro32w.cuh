// Warp-marching form of the mixed-precision hydro step (same arithmetic as the
// perturbation operators documented in hydro32.cuh).
//
// One warp owns a strip of 32 azimuthal columns j0-2 .. j0+29 (lane l <-> column
// j0-2+l, periodic) and a band of kBand32 radial rows.  It marches outward one row per
// iteration, keeping every radial neighbour it needs in registers:
//   iteration k loads input row L = i0-3+k (prefetched one iteration ahead),
//   computes the source kick of row L-1, the radial face L-2, gathers row L-3 from faces
//   L-3 and L-2, and runs the azimuthal sweep of row L-3 with neighbours from shuffles.
// The azimuthal faces of lanes 2..30 are complete (they need lanes l-2..l+1), so lanes
// 2..29 (28 columns) write output.  The two edge lanes additionally load their outer
// neighbour column for the pressure and potential differences of the source step.
// No CTA barrier is needed until the end-of-launch reduction.
#pragma once

#include "hydro32.cuh"
#include "step_ctl.cuh"

namespace dg {

constexpr int kBand32 = 16;        // radial rows per warp
constexpr int kOutCols32 = 28;     // output columns per warp
constexpr int kWarps32 = 4;        // warps per CTA (adjacent strips of one band)

struct SplitBf16 {
  __nv_bfloat16 *hi, *lo;
};

__device__ __forceinline__ int wrap_col(int j, int N) {
  j += (j < 0) ? N : 0;
  j -= (j >= N) ? N : 0;
  return j;
}

__global__ void __launch_bounds__(kWarps32 * 32) k_hydro32w(
    const float *__restrict__ sig, const float *__restrict__ uu, const float *__restrict__ ww,
    const float *__restrict__ Phi, const double *__restrict__ gRin, const double *__restrict__ gpin, int force_mode,
    float *__restrict__ so, float *__restrict__ uo, float *__restrict__ wo, SplitBf16 Sx, Ctl *ctl, Rows32 g,
    int nstrips) {
  __shared__ double red[kWarps32];
  // per-row / per-face constants of rows i0-3 .. i0+kBand32+2, staged once per CTA
  enum { cS0, cInvS0, cV0, cA0, cDP0, cInvdRc, cInvR, cR, cInvVol, cInvdl, cAphi, cR32, cInvdR, cP0,
         cDS0, cDV, cAf, cInvdRl, cInvdRr, cNConst };
  constexpr int kRows = kBand32 + 6;
  __shared__ float rc[cNConst][kRows];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int strip = blockIdx.x * kWarps32 + warp;
  const int i0 = blockIdx.y * kBand32;
  const int Nu = g.Nu, Nphi = g.Nphi;
  const int ib = i0 - 3;
  for (int t = threadIdx.x; t < cNConst * kRows; t += blockDim.x) {
    const int k = t / kRows, r = t - k * kRows, i = ib + r;
    float v = 0.f;
    if (i >= 0 && i <= Nu) {
      const bool row = i < Nu;
      switch (k) {
        case cS0: v = row ? g.S0[i] : 0.f; break;
        case cInvS0: v = row ? g.invS0[i] : 0.f; break;
        case cV0: v = row ? g.V0[i] : 0.f; break;
        case cA0: v = row ? g.a0[i] : 0.f; break;
        case cDP0: v = row ? g.dP0dR[i] : 0.f; break;
        case cInvdRc: v = row ? g.invdRc[i] : 0.f; break;
        case cInvR: v = row ? g.invR[i] : 0.f; break;
        case cR: v = row ? g.R[i] : 0.f; break;
        case cInvVol: v = row ? g.invVol[i] : 0.f; break;
        case cInvdl: v = row ? g.invdl[i] : 0.f; break;
        case cAphi: v = row ? g.Aphi[i] : 0.f; break;
        case cR32: v = row ? g.R32[i] : 0.f; break;
        case cInvdR: v = row ? g.invdR[i] : 0.f; break;
        case cP0: v = row ? g.P0[i] : 0.f; break;
        case cDS0: v = g.dS0[i]; break;
        case cDV: v = g.dV[i]; break;
        case cAf: v = g.Af[i]; break;
        case cInvdRl: v = g.invdRl[i]; break;
        case cInvdRr: v = g.invdRr[i]; break;
      }
    }
    rc[k][r] = v;
  }
  __syncthreads();
#define RC(k, i) rc[k][(i) - ib]
  const StepInfo si = read_step_info(ctl, true);
  const float dt = (float)si.dt;
  const int nmodes = si.nmodes;
  double msum[2 * kMaxModes];
#pragma unroll
  for (int q = 0; q < 2 * kMaxModes; ++q) msum[q] = 0.0;
  float lmaxf = 0.f;
  double lmax = 0.0;
  bool bad = false;

  const bool wact = strip < nstrips;
  const int j0 = strip * kOutCols32;
  const int jg = wrap_col(j0 - 2 + lane, Nphi);
  const int jx = wrap_col(lane == 0 ? jg - 1 : jg + 1, Nphi);  // outer neighbour of the edge lanes
  const bool edge = (lane == 0 || lane == 31);
  const bool outlane = wact && lane >= 2 && lane <= 29 && (j0 + lane - 2) < Nphi;
  const int iend = (i0 + kBand32 < Nu) ? i0 + kBand32 : Nu;

  if (!si.active) {
    if (outlane) {
      for (int i = i0; i < iend; ++i) {
        const int k = i * Nphi + jg;
        so[k] = sig[k]; uo[k] = uu[k]; wo[k] = ww[k];
        lmax = fmax(lmax, (double)cfl_rate32(g, i, sig[k], uu[k], ww[k]));
      }
    }
    finish_launch<kWarps32 * 32>(ctl, si, lmax, msum, red);
    return;
  }

  // ---- register windows (index 0 = oldest row) ----
  float sg[5] = {0.f, 0.f, 0.f, 0.f, 0.f};   // sigma, rows L-4 .. L
  float u0[2] = {0.f, 0.f}, w0[2] = {0.f, 0.f};  // raw u, w, rows L-1, L
  float dp[3] = {0.f, 0.f, 0.f}, ph[3] = {0.f, 0.f, 0.f};  // dP, dPhi, rows L-2 .. L
  float dpx[2] = {0.f, 0.f}, phx[2] = {0.f, 0.f};  // edge lanes: outer neighbour, rows L-1, L
  float u1[4] = {0.f, 0.f, 0.f, 0.f}, w1[4] = {0.f, 0.f, 0.f, 0.f};  // source output, rows L-4 .. L-1
  float fF = 0.f, fFR = 0.f, fGB = 0.f;  // radial face L-3 (previous iteration)
  // prefetched next row
  float nsg = 0.f, nu = 0.f, nw = 0.f, nph = 0.f, nsx = 0.f, nphx = 0.f;

  auto load_row = [&](int L) {
    nsg = nu = nw = nph = nsx = nphx = 0.f;
    if (wact && L >= 0 && L < Nu) {
      const int k = L * Nphi + jg;
      nsg = sig[k];
      nu = uu[k];
      nw = ww[k];
      if (force_mode == kForcePhi) nph = Phi[k];
      if (edge) {
        const int kx = L * Nphi + jx;
        nsx = sig[kx];
        if (force_mode == kForcePhi) nphx = Phi[kx];
      }
    }
  };

  const int nit = kBand32 + 6;
  load_row(i0 - 3);
  for (int it = 0; it < nit; ++it) {
    const int L = i0 - 3 + it;
    // shift windows and insert the prefetched row L
#pragma unroll
    for (int q = 0; q < 4; ++q) sg[q] = sg[q + 1];
    u0[0] = u0[1]; w0[0] = w0[1];
    dp[0] = dp[1]; dp[1] = dp[2]; ph[0] = ph[1]; ph[1] = ph[2];
    dpx[0] = dpx[1]; phx[0] = phx[1];
    const bool Lok = L >= 0 && L < Nu;
    sg[4] = nsg; u0[1] = nu; w0[1] = nw; ph[2] = nph; phx[1] = nphx;
    if (g.gamma2) {
      const float twoS0 = 2.f * RC(cS0, L);
      dp[2] = Lok ? g.Kpoly * nsg * (twoS0 + nsg) : 0.f;
      dpx[1] = (Lok && edge) ? g.Kpoly * nsx * (twoS0 + nsx) : 0.f;
    } else {
      dp[2] = Lok ? RC(cP0, L) * expm1f(g.gamma * log1pf(nsg * RC(cInvS0, L))) : 0.f;
      dpx[1] = (Lok && edge) ? RC(cP0, L) * expm1f(g.gamma * log1pf(nsx * RC(cInvS0, L))) : 0.f;
    }
    // prefetch row L+1 while this row is processed
    if (it + 1 < nit) load_row(L + 1);

    // ---- source kick of row Ls = L-1 (hydro.hpp:73-96, perturbation form) ----
    const int Ls = L - 1;
    float nu1 = 0.f, nw1 = 0.f;
    {
      // azimuthal neighbours of dP and dPhi at row Ls
      float pm = __shfl_up_sync(0xffffffffu, dp[1], 1), pp = __shfl_down_sync(0xffffffffu, dp[1], 1);
      float fm = __shfl_up_sync(0xffffffffu, ph[1], 1), fp = __shfl_down_sync(0xffffffffu, ph[1], 1);
      if (lane == 0) { pm = dpx[0]; fm = phx[0]; }
      if (lane == 31) { pp = dpx[0]; fp = phx[0]; }
      if (Ls >= 0 && Ls < Nu) {
        const float s_g = sg[3];
        const float s = RC(cS0, Ls) + s_g;
        const float pim = (Ls == 0) ? dp[1] : dp[0];
        const float pip = (Ls == Nu - 1) ? dp[1] : dp[2];
        const float ddP = (pip - pim) * RC(cInvdRc, Ls);
        const float dPdphi = (pp - pm) * g.inv2dphi;
        const float iR = RC(cInvR, Ls);
        float dgR = 0.f, dgp = 0.f;
        if (force_mode == kForcePhi) {
          float dPhidu;
          if (Ls == 0) dPhidu = (ph[2] - ph[1]) * g.invdu;
          else if (Ls == Nu - 1) dPhidu = (ph[1] - ph[0]) * g.invdu;
          else dPhidu = (ph[2] - ph[0]) * g.inv2du;
          dgR = -dPhidu * iR;
          dgp = -(fp - fm) * g.inv2dphi * iR;
        } else if (force_mode == kForceArrays && wact) {
          const int k = Ls * Nphi + jg;
          dgR = (float)gRin[k];
          dgp = (float)gpin[k];
        }
        const float uc = u0[0], wc = w0[0];
        const float V = RC(cV0, Ls);
        const float aR = RC(cA0, Ls) + __fdividef(RC(cDP0, Ls) * s_g * RC(cInvS0, Ls) - ddP, s) + dgR +
                         (2.f * V + wc) * wc * iR;
        const float ap = __fdividef(-dPdphi, s * RC(cR, Ls)) + dgp - uc * (V + wc) * iR;
        nu1 = uc + dt * aR;
        nw1 = wc + dt * ap;
      }
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) { u1[q] = u1[q + 1]; w1[q] = w1[q + 1]; }
    u1[3] = nu1; w1[3] = nw1;

    // ---- radial face f = L-2 (hydro.hpp:107-130): cells f-2..f+1 are window slots 0..3 ----
    const int f = L - 2;
    float F = 0.f, FR = 0.f, GA = 0.f, GB = 0.f;
    if (f >= 1 && f <= Nu - 1) {
      const float vf = 0.5f * (u1[1] + u1[2]);
      const bool up = vf > 0.f;
      const int cc = up ? f - 1 : f;
      const float hf = up ? 0.5f * (1.f - vf * dt * RC(cInvdRl, f)) : -0.5f * (1.f + vf * dt * RC(cInvdRr, f));
      // slots of cc-1, cc, cc+1
      const float sa = up ? sg[0] : sg[1], sb = up ? sg[1] : sg[2], sc = up ? sg[2] : sg[3];
      const float ua = up ? u1[0] : u1[1], ub = up ? u1[1] : u1[2], uc = up ? u1[2] : u1[3];
      const float wa = up ? w1[0] : w1[1], wb = up ? w1[1] : w1[2], wc = up ? w1[2] : w1[3];
      float kS = 0.f, kU = 0.f, kV = 0.f;
      if (cc > 0 && cc < Nu - 1) {
        kS = vanleer32(RC(cDS0, cc + 1) + (sc - sb), RC(cDS0, cc) + (sb - sa));
        kU = vanleer32(uc - ub, ub - ua);
        kV = vanleer32(RC(cDV, cc + 1) + (wc - wb), RC(cDV, cc) + (wb - wa));
      }
      const float Sf = RC(cS0, cc) + sb + hf * kS;
      const float uf = ub + hf * kU;
      const float dVf = RC(cDV, f);
      const float Df = (up ? 0.f : dVf) + wb + hf * kV;  // vphi_f - V0(f-1)
      F = vf * Sf * RC(cAf, f);
      FR = F * uf;
      GA = F * Df;
      GB = F * (Df - dVf);
    }

    // ---- radial gather of row i = L-3 from faces i (previous) and i+1 (= f) ----
    const int i = L - 3;
    float s2 = 0.f, u2 = 0.f, w2 = 0.f;
    const bool iok = i >= i0 && i < iend;
    if (iok) {
      const float sgi = sg[1], u1i = u1[1], w1i = w1[1];
      const float S0 = RC(cS0, i);
      const float s = S0 + sgi;
      const float iv = RC(cInvVol, i);
      s2 = sgi + dt * (fF - F) * iv;
      const float sn = S0 + s2;
      const float d = (sn < 1e-10f) ? 1e-10f : sn;
      u2 = __fdividef(s * u1i + dt * (fFR - FR) * iv, d);
      w2 = __fdividef(s * w1i + dt * (fGB - GA) * iv, d);
    }
    fF = F; fFR = FR; fGB = GB;

    // ---- azimuthal sweep of row i (hydro.hpp:150-178), neighbours by shuffle ----
    if (i >= i0 && i < iend) {  // warp-uniform
      const float s_m2 = __shfl_up_sync(0xffffffffu, s2, 2), s_m1 = __shfl_up_sync(0xffffffffu, s2, 1);
      const float s_p1 = __shfl_down_sync(0xffffffffu, s2, 1);
      const float u_m2 = __shfl_up_sync(0xffffffffu, u2, 2), u_m1 = __shfl_up_sync(0xffffffffu, u2, 1);
      const float u_p1 = __shfl_down_sync(0xffffffffu, u2, 1);
      const float w_m2 = __shfl_up_sync(0xffffffffu, w2, 2), w_m1 = __shfl_up_sync(0xffffffffu, w2, 1);
      const float w_p1 = __shfl_down_sync(0xffffffffu, w2, 1);
      // left face of this lane (between column l-1 and l)
      const float V = RC(cV0, i);
      const float dv = 0.5f * (w_m1 + w2);
      const float vf = V + dv;
      const bool up = vf > 0.f;
      const float idl = RC(cInvdl, i);
      const float hf = up ? 0.5f * (1.f - vf * dt * idl) : -0.5f * (1.f + vf * dt * idl);
      const float sa = up ? s_m2 : s_m1, sb = up ? s_m1 : s2, sc = up ? s2 : s_p1;
      const float ua = up ? u_m2 : u_m1, ub = up ? u_m1 : u2, uc = up ? u2 : u_p1;
      const float wa = up ? w_m2 : w_m1, wb = up ? w_m1 : w2, wc = up ? w2 : w_p1;
      const float sf = sb + hf * vanleer32(sc - sb, sb - sa);
      const float Sf = RC(cS0, i) + sf;
      const float uf = ub + hf * vanleer32(uc - ub, ub - ua);
      const float wf = wb + hf * vanleer32(wc - wb, wb - wa);
      const float A = RC(cAphi, i);
      const float Ffull = vf * Sf * A;
      const float Fm = A * (V * sf + dv * Sf);
      const float FRp = Ffull * uf;
      const float Gp = Ffull * wf;
      // right face = left face of lane l+1
      const float Fm_r = __shfl_down_sync(0xffffffffu, Fm, 1);
      const float FR_r = __shfl_down_sync(0xffffffffu, FRp, 1);
      const float G_r = __shfl_down_sync(0xffffffffu, Gp, 1);
      if (outlane) {
        const float iv = RC(cInvVol, i);
        const float S0 = RC(cS0, i);
        const float sn2 = S0 + s2;
        float s3 = s2 + dt * (Fm - Fm_r) * iv;
        const float sn3 = S0 + s3;
        const float d = (sn3 < 1e-10f) ? 1e-10f : sn3;
        const float u3 = __fdividef(sn2 * u2 + dt * (FRp - FR_r) * iv, d);
        const float w3 = __fdividef(sn2 * w2 + dt * (Gp - G_r) * iv, d);
        if (sn3 < 1e-10f) s3 = 1e-10f - S0;  // floor (hydro.hpp:69)
        const int k = i * Nphi + jg;
        so[k] = s3; uo[k] = u3; wo[k] = w3;
        const float x = RC(cR32, i) * s3;
        const __nv_bfloat16 hx = __float2bfloat16_rn(x);
        Sx.hi[k] = hx;
        Sx.lo[k] = __float2bfloat16_rn(x - __bfloat162float(hx));
        // CFL rate of the new state (hydro.hpp:54-57)
        const float sc_ = (sn3 < 1e-10f) ? 1e-10f : sn3;
        const float cs = sqrtf(g.gamma2 ? g.gamma * g.Kpoly * sc_ : g.gamma * g.Kpoly * powf(sc_, g.gamma - 1.f));
        const float rate = (fabsf(u3) + cs) * RC(cInvdR, i) + (fabsf(V + w3) + cs) * idl;
        bad |= !(rate == rate) || !(u3 == u3) || !(w3 == w3);
        lmaxf = fmaxf(lmaxf, rate);
        if (nmodes) {
          const double sfull = g.S0d[i] + (double)s3;
          const double phi = (jg + 0.5) * (double)g.dphi;
          for (int m = 0; m < nmodes; ++m) {
            double sn, cs;
            sincos(m * phi, &sn, &cs);
            msum[2 * m] += sfull * cs * g.dAd[i];
            msum[2 * m + 1] -= sfull * sn * g.dAd[i];
          }
        }
      }
    }
  }
  lmax = (double)lmaxf;
  if (bad) lmax = __longlong_as_double(0x7ff8000000000000ll);
  finish_launch<kWarps32 * 32>(ctl, si, lmax, msum, red);
#undef RC
}

}  // namespace dg
