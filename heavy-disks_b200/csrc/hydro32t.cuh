// Tiled form of the mixed-precision hydro step (same arithmetic as the perturbation
// operators documented in hydro32.cuh, stage by stage as in hydro32w.cuh).
//
// One CTA owns an output tile of kTileI radial rows x kTileJ azimuthal columns and stages
// rows i0-3 .. i0+kTileI+2, columns j0-3 .. j0+kTileJ+2 (periodic in phi) in shared memory
// as rows of exactly 64 floats.  Each thread owns one stored column c = j - (j0 - 3) for the
// whole launch (lane + 32 x (warp & 1)) and steps through the rows (warp >> 1) + 4k with
// fully unrolled loops, so a warp always works on one row (row constants are broadcasts,
// addresses are base + immediate) and its 32 lanes touch 32 consecutive floats.  Stages,
// separated by CTA barriers:
//   S0 load sigma, dP = P(Sigma0 + sigma) - P(Sigma0) and dPhi (u, w go to registers)
//   S2 source kick (hydro.hpp:73-96) of rows i0-2 .. i0+kTileI+1
//   S3 radial faces i0 .. i0+kTileI (hydro.hpp:107-130)
//   S4 radial gather of the tile rows (hydro.hpp:131-139), in place over sigma
//   S5 azimuthal faces j0 .. j0+kTileJ (hydro.hpp:150-170)
//   S6 azimuthal gather, Sigma floor (hydro.hpp:69), outputs, CFL rate of the new state
// Only the halo of the source stage (2 rows, 3 columns a side) is computed twice.
#pragma once

#include "hydro32.cuh"
#include "hydro32w.cuh"
#include "step_ctl.cuh"

namespace dg {

constexpr int kTileI = 16;                // output rows per CTA
constexpr int kLd32t = 64;                // stored columns per row: c in [0, 64) <-> j = j0 - 3 + c
constexpr int kTileJ = kLd32t - 6;        // output columns per CTA (58)
constexpr int kThreads32t = 256;          // 4 row groups x 64 columns
constexpr int kRowGroups32t = kThreads32t / kLd32t;
constexpr int kRows32t = kTileI + 6;      // stored rows r = i - (i0 - 3)
constexpr int kSrcRows32t = kTileI + 4;   // source rows i0-2 .. i0+kTileI+1 (r in [1, kTileI + 5))
constexpr int kFaceRows32t = kTileI + 1;  // radial faces i0 .. i0+kTileI
// rows of each stage a thread visits (ceil over the 4 row groups)
constexpr int kItLoad = (kRows32t + kRowGroups32t - 1) / kRowGroups32t;
constexpr int kItSrc = (kSrcRows32t + kRowGroups32t - 1) / kRowGroups32t;
constexpr int kItFace = (kFaceRows32t + kRowGroups32t - 1) / kRowGroups32t;
constexpr int kItOut = (kTileI + kRowGroups32t - 1) / kRowGroups32t;
// row and face constants staged per CTA (same set as the warp form)
enum { tS0, tInvS0, tV0, tA0, tDP0, tInvdRc, tInvR, tR, tInvVol, tInvdl, tAphi, tR32, tInvdR, tP0,
       tDS0, tDV, tAf, tInvdRl, tInvdRr, tNConst };
// shared-memory plan in floats
constexpr int kOffRc32t = 0;
constexpr int kOffSg32t = kOffRc32t + tNConst * kRows32t;      // sigma, then s2 in place
constexpr int kOffDp32t = kOffSg32t + kRows32t * kLd32t;       // dP, then u2
constexpr int kOffPh32t = kOffDp32t + kRows32t * kLd32t;       // dPhi, then w2
constexpr int kOffU132t = kOffPh32t + kRows32t * kLd32t;       // u1 (source rows), then s3 for the mode sums
constexpr int kOffW132t = kOffU132t + kSrcRows32t * kLd32t;    // w1
constexpr int kOffF32t = kOffW132t + kSrcRows32t * kLd32t;     // radial F, FR, GA, GB; then phi Fm, FR, G
constexpr int kFaceArr32t = kFaceRows32t * kLd32t;
constexpr int kFloats32t = kOffF32t + 4 * kFaceArr32t;
constexpr size_t kSmem32t = (size_t)kFloats32t * sizeof(float);
static_assert(kItOut * kRowGroups32t == kTileI, "output rows split evenly over the row groups");

// One tile's step.  G2: Gamma = 2 (P = K Sigma^2); FM: force mode; IN: the tile's rows
// i0-3 .. i0+kTileI+2 all lie in 1 .. Nu-2 for the stages that need it (no reflecting face,
// one-sided difference or missing row inside the tile), so those tests compile away.
template <bool G2, int FM, bool IN>
__device__ __forceinline__ void hydro32t_tile(
    const float *__restrict__ sig, const float *__restrict__ uu, const float *__restrict__ ww,
    const float *__restrict__ Phi, const double *__restrict__ gRin, const double *__restrict__ gpin,
    float *__restrict__ so, float *__restrict__ uo, float *__restrict__ wo, const SplitBf16 &Sx, Ctl *ctl,
    const Rows32 &g, float *sm32t, double *red, double *bsum, double *zsum) {
  constexpr int force_mode = FM;
  float *rc = sm32t + kOffRc32t;
  float *SG = sm32t + kOffSg32t, *DP = sm32t + kOffDp32t, *PH = sm32t + kOffPh32t;
  float *U1 = sm32t + kOffU132t, *W1 = sm32t + kOffW132t;
  float *FF = sm32t + kOffF32t, *FR = FF + kFaceArr32t, *GA = FR + kFaceArr32t, *GB = GA + kFaceArr32t;
  float *U2 = DP, *W2 = PH;               // S4 outputs over the dead source inputs
  float *PF = FF, *PR = FR, *PG = GA;     // S5 outputs over the dead radial fluxes
  float *S3 = U1;                         // new sigma for the mode sums, over the dead u1

  const int tid = threadIdx.x;
  const int c = tid & (kLd32t - 1);       // this thread's stored column
  const int rg = tid / kLd32t;            // row group: rows rg, rg + 4, ...
  const int Nu = g.Nu, Nphi = g.Nphi;
  const int i0 = blockIdx.y * kTileI, j0 = blockIdx.x * kTileJ;
  const int ib = i0 - 3;
  const int iend = (i0 + kTileI < Nu) ? i0 + kTileI : Nu;
  const int jc = wrap_col(j0 - 3 + c, Nphi);                 // global column of c
  const bool out_col = c >= 3 && c < 3 + kTileJ && j0 + c - 3 < Nphi;
#define RC(k, i) rc[(k) * kRows32t + (i) - ib]
  // row / face tests that an interior tile never fails
  auto row_ok = [&](int i) { return IN || (i >= 0 && i < Nu); };
  auto first_row = [&](int i) { return !IN && i == 0; };
  auto last_row = [&](int i) { return !IN && i == Nu - 1; };

  for (int t = tid; t < tNConst * kRows32t; t += kThreads32t) {
    const int k = t / kRows32t, r = t - k * kRows32t, i = ib + r;
    float v = 0.f;
    if (i >= 0 && i <= Nu) {
      const bool row = i < Nu;
      switch (k) {
        case tS0: v = row ? g.S0[i] : 0.f; break;
        case tInvS0: v = row ? g.invS0[i] : 0.f; break;
        case tV0: v = row ? g.V0[i] : 0.f; break;
        case tA0: v = row ? g.a0[i] : 0.f; break;
        case tDP0: v = row ? g.dP0dR[i] : 0.f; break;
        case tInvdRc: v = row ? g.invdRc[i] : 0.f; break;
        case tInvR: v = row ? g.invR[i] : 0.f; break;
        case tR: v = row ? g.R[i] : 0.f; break;
        case tInvVol: v = row ? g.invVol[i] : 0.f; break;
        case tInvdl: v = row ? g.invdl[i] : 0.f; break;
        case tAphi: v = row ? g.Aphi[i] : 0.f; break;
        case tR32: v = row ? g.R32[i] : 0.f; break;
        case tInvdR: v = row ? g.invdR[i] : 0.f; break;
        case tP0: v = row ? g.P0[i] : 0.f; break;
        case tDS0: v = g.dS0[i]; break;
        case tDV: v = g.dV[i]; break;
        case tAf: v = g.Af[i]; break;
        case tInvdRl: v = g.invdRl[i]; break;
        case tInvdRr: v = g.invdRr[i]; break;
      }
    }
    rc[t] = v;
  }
  if (tid < 2 * kMaxModes) {
    bsum[tid] = 0.0;
    zsum[tid] = 0.0;
  }
  pdl_wait();  // dt, the state and dPhi come from earlier kernels on the stream
  pdl_trigger();
  const StepInfo si = read_step_info(ctl, true);
  const float dt = (float)si.dt;
  float lmaxf = 0.f;
  bool bad = false;

  if (!si.active) {
    // pass-through: copy the tile and report the CFL rate of the unchanged state
    if (out_col) {
#pragma unroll
      for (int k = 0; k < kItOut; ++k) {
        const int i = i0 + rg + kRowGroups32t * k;
        if (i < Nu) {
          const size_t q = (size_t)i * Nphi + jc;
          so[q] = sig[q]; uo[q] = uu[q]; wo[q] = ww[q];
          lmaxf = fmaxf(lmaxf, cfl_rate32(g, i, sig[q], uu[q], ww[q]));
        }
      }
    }
    __syncthreads();
    finish_launch_deferred<kThreads32t>(ctl, si, (double)lmaxf, tid == 0 ? bsum : zsum, red);
    return;
  }

  // ---- S0: every global load of the thread first: raw u, w of its source points (kept
  // in registers) and sigma, dPhi of its stored points ----
  float ur[kItSrc], wr[kItSrc], sv[kItLoad], pv[kItLoad];
#pragma unroll
  for (int k = 0; k < kItSrc; ++k) {
    const int i = ib + 1 + rg + kRowGroups32t * k;
    ur[k] = wr[k] = 0.f;
    if (row_ok(i)) {
      const size_t q = (size_t)i * Nphi + jc;
      ur[k] = uu[q];
      wr[k] = ww[q];
    }
  }
#pragma unroll
  for (int k = 0; k < kItLoad; ++k) {
    const int r = rg + kRowGroups32t * k, i = ib + r;
    sv[k] = pv[k] = 0.f;
    if (r < kRows32t && row_ok(i)) {
      const size_t q = (size_t)i * Nphi + jc;
      sv[k] = sig[q];
      if (force_mode == kForcePhi) pv[k] = Phi[q];
    }
  }
  __syncthreads();  // row constants staged
#pragma unroll
  for (int k = 0; k < kItLoad; ++k) {
    const int r = rg + kRowGroups32t * k, i = ib + r;
    if (r < kRows32t) {
      const float s = sv[k];
      float d = 0.f;
      if (row_ok(i)) {
        if (G2) d = g.Kpoly * s * (2.f * RC(tS0, i) + s);
        else d = RC(tP0, i) * expm1f(g.gamma * log1pf(s * RC(tInvS0, i)));
      }
      SG[r * kLd32t + c] = s;
      DP[r * kLd32t + c] = d;
      PH[r * kLd32t + c] = pv[k];
    }
  }
  __syncthreads();

  // ---- S2: source kick of rows i0-2 .. i0+kTileI+1, columns c in [1, 63) ----
  const bool src_col = c >= 1 && c < kLd32t - 1;
#pragma unroll
  for (int k = 0; k < kItSrc; ++k) {
    const int rs = rg + kRowGroups32t * k, r = rs + 1, i = ib + r;
    if (rs < kSrcRows32t && src_col) {
      float nu1 = 0.f, nw1 = 0.f;
      if (row_ok(i)) {
        const int x = r * kLd32t + c;
        const float s_g = SG[x];
        const float s = RC(tS0, i) + s_g;
        const float pim = first_row(i) ? DP[x] : DP[x - kLd32t];
        const float pip = last_row(i) ? DP[x] : DP[x + kLd32t];
        const float ddP = (pip - pim) * RC(tInvdRc, i);
        const float dPdphi = (DP[x + 1] - DP[x - 1]) * g.inv2dphi;
        const float iR = RC(tInvR, i);
        float dgR = 0.f, dgp = 0.f;
        if (force_mode == kForcePhi) {
          float dPhidu;
          if (first_row(i)) dPhidu = (PH[x + kLd32t] - PH[x]) * g.invdu;
          else if (last_row(i)) dPhidu = (PH[x] - PH[x - kLd32t]) * g.invdu;
          else dPhidu = (PH[x + kLd32t] - PH[x - kLd32t]) * g.inv2du;
          dgR = -dPhidu * iR;
          dgp = -(PH[x + 1] - PH[x - 1]) * g.inv2dphi * iR;
        } else if (force_mode == kForceArrays) {
          const size_t q = (size_t)i * Nphi + jc;
          dgR = (float)gRin[q];
          dgp = (float)gpin[q];
        }
        const float uc = ur[k], wc = wr[k];
        const float V = RC(tV0, i);
        const float aR = RC(tA0, i) + __fdividef(RC(tDP0, i) * s_g * RC(tInvS0, i) - ddP, s) + dgR +
                         (2.f * V + wc) * wc * iR;
        const float ap = __fdividef(-dPdphi, s * RC(tR, i)) + dgp - uc * (V + wc) * iR;
        nu1 = uc + dt * aR;
        nw1 = wc + dt * ap;
      }
      U1[rs * kLd32t + c] = nu1;
      W1[rs * kLd32t + c] = nw1;
    }
  }
  __syncthreads();

  // ---- S3: radial faces f = i0 .. i0+kTileI, columns c in [1, 63) ----
#pragma unroll
  for (int k = 0; k < kItFace; ++k) {
    const int fr = rg + kRowGroups32t * k, f = i0 + fr;
    if (fr < kFaceRows32t && src_col) {
      float F = 0.f, FRv = 0.f, GAv = 0.f, GBv = 0.f;
      if (IN || (f >= 1 && f <= Nu - 1)) {
        const int xs = (f - 2 - ib) * kLd32t + c;   // sigma at row f-2
        const int xu = (f - 3 - ib) * kLd32t + c;   // u1 / w1 at row f-2
        const float vf = 0.5f * (U1[xu + kLd32t] + U1[xu + 2 * kLd32t]);
        const bool up = vf > 0.f;
        const int cc = up ? f - 1 : f;
        const float hf = up ? 0.5f * (1.f - vf * dt * RC(tInvdRl, f)) : -0.5f * (1.f + vf * dt * RC(tInvdRr, f));
        const int o = up ? 0 : kLd32t;  // cells cc-1, cc, cc+1 start at row f-2 (up) or f-1
        const float sa = SG[xs + o], sb = SG[xs + o + kLd32t], sc = SG[xs + o + 2 * kLd32t];
        const float ua = U1[xu + o], ub = U1[xu + o + kLd32t], uc = U1[xu + o + 2 * kLd32t];
        const float wa = W1[xu + o], wb = W1[xu + o + kLd32t], wc = W1[xu + o + 2 * kLd32t];
        float kS = 0.f, kU = 0.f, kV = 0.f;
        if (IN || (cc > 0 && cc < Nu - 1)) {
          kS = vanleer32(RC(tDS0, cc + 1) + (sc - sb), RC(tDS0, cc) + (sb - sa));
          kU = vanleer32(uc - ub, ub - ua);
          kV = vanleer32(RC(tDV, cc + 1) + (wc - wb), RC(tDV, cc) + (wb - wa));
        }
        const float Sf = RC(tS0, cc) + sb + hf * kS;
        const float uf = ub + hf * kU;
        const float dVf = RC(tDV, f);
        const float Df = (up ? 0.f : dVf) + wb + hf * kV;  // vphi_f - V0(f-1)
        F = vf * Sf * RC(tAf, f);
        FRv = F * uf;
        GAv = F * Df;
        GBv = F * (Df - dVf);
      }
      const int x = fr * kLd32t + c;
      FF[x] = F; FR[x] = FRv; GA[x] = GAv; GB[x] = GBv;
    }
  }
  __syncthreads();

  // ---- S4: radial gather of rows i0 .. iend-1, columns c in [1, 63) ----
#pragma unroll
  for (int k = 0; k < kItOut; ++k) {
    const int ri = rg + kRowGroups32t * k, i = i0 + ri;
    if ((IN || i < iend) && src_col) {
      const int xs = (i - ib) * kLd32t + c, xu = (i - ib - 1) * kLd32t + c, xf = ri * kLd32t + c;
      const float sgi = SG[xs], u1i = U1[xu], w1i = W1[xu];
      const float S0 = RC(tS0, i);
      const float s = S0 + sgi;
      const float iv = RC(tInvVol, i);
      const float s2 = sgi + dt * (FF[xf] - FF[xf + kLd32t]) * iv;
      const float sn = S0 + s2;
      const float d = (sn < 1e-10f) ? 1e-10f : sn;
      const float u2 = __fdividef(s * u1i + dt * (FR[xf] - FR[xf + kLd32t]) * iv, d);
      const float w2 = __fdividef(s * w1i + dt * (GB[xf] - GA[xf + kLd32t]) * iv, d);
      SG[xs] = s2;
      U2[xs] = u2;
      W2[xs] = w2;
    }
  }
  __syncthreads();

  // ---- S5: azimuthal faces (left face of column c) for c in [3, 3 + kTileJ] ----
  const bool face_col = c >= 3 && c <= 3 + kTileJ;
#pragma unroll
  for (int k = 0; k < kItOut; ++k) {
    const int ri = rg + kRowGroups32t * k, i = i0 + ri;
    if ((IN || i < iend) && face_col) {
      const int x = (i - ib) * kLd32t + c;
      const float V = RC(tV0, i);
      const float dv = 0.5f * (W2[x - 1] + W2[x]);
      const float vf = V + dv;
      const bool up = vf > 0.f;
      const float idl = RC(tInvdl, i);
      const float hf = up ? 0.5f * (1.f - vf * dt * idl) : -0.5f * (1.f + vf * dt * idl);
      const int o = up ? x - 2 : x - 1;  // cells cc-1, cc, cc+1
      const float sa = SG[o], sb = SG[o + 1], sc = SG[o + 2];
      const float ua = U2[o], ub = U2[o + 1], uc = U2[o + 2];
      const float wa = W2[o], wb = W2[o + 1], wc = W2[o + 2];
      const float sf = sb + hf * vanleer32(sc - sb, sb - sa);
      const float Sf = RC(tS0, i) + sf;
      const float uf = ub + hf * vanleer32(uc - ub, ub - ua);
      const float wf = wb + hf * vanleer32(wc - wb, wb - wa);
      const float A = RC(tAphi, i);
      const float Ffull = vf * Sf * A;
      const int xf = ri * kLd32t + c;
      PF[xf] = A * (V * sf + dv * Sf);
      PR[xf] = Ffull * uf;
      PG[xf] = Ffull * wf;
    }
  }
  __syncthreads();

  // ---- S6: azimuthal gather, floor, outputs, CFL rate ----
#pragma unroll
  for (int k = 0; k < kItOut; ++k) {
    const int ri = rg + kRowGroups32t * k, i = i0 + ri;
    if ((IN || i < iend) && out_col) {
      const int x = (i - ib) * kLd32t + c, xf = ri * kLd32t + c;
      const float iv = RC(tInvVol, i);
      const float S0 = RC(tS0, i);
      const float s2 = SG[x], u2 = U2[x], w2 = W2[x];
      const float sn2 = S0 + s2;
      float s3 = s2 + dt * (PF[xf] - PF[xf + 1]) * iv;
      const float sn3 = S0 + s3;
      const float d = (sn3 < 1e-10f) ? 1e-10f : sn3;
      const float u3 = __fdividef(sn2 * u2 + dt * (PR[xf] - PR[xf + 1]) * iv, d);
      const float w3 = __fdividef(sn2 * w2 + dt * (PG[xf] - PG[xf + 1]) * iv, d);
      if (sn3 < 1e-10f) s3 = 1e-10f - S0;  // floor (hydro.hpp:69)
      const size_t q = (size_t)i * Nphi + jc;
      so[q] = s3; uo[q] = u3; wo[q] = w3;
      const float xr = RC(tR32, i) * s3;
      const __nv_bfloat16 hx = __float2bfloat16_rn(xr);
      Sx.hi[q] = hx;
      Sx.lo[q] = __float2bfloat16_rn(xr - __bfloat162float(hx));
      // CFL rate of the new state (hydro.hpp:54-57)
      const float sc_ = (sn3 < 1e-10f) ? 1e-10f : sn3;
      const float cs = sqrtf(G2 ? g.gamma * g.Kpoly * sc_ : g.gamma * g.Kpoly * powf(sc_, g.gamma - 1.f));
      const float rate = (fabsf(u3) + cs) * RC(tInvdR, i) + (fabsf(RC(tV0, i) + w3) + cs) * RC(tInvdl, i);
      bad |= !(rate == rate) || !(u3 == u3) || !(w3 == w3);
      lmaxf = fmaxf(lmaxf, rate);
      S3[ri * kLd32t + c] = s3;
    }
  }
  // mode sums of the new state (output times and per-step diagnostics only)
  if (si.nmodes) {
    __syncthreads();
    const double phi = (jc + 0.5) * (double)g.dphi;
    for (int m = 0; m < si.nmodes; ++m) {
      double re = 0.0, im = 0.0;
      if (out_col) {
        double sn, cs;
        sincos(m * phi, &sn, &cs);
#pragma unroll 1
        for (int k = 0; k < kItOut; ++k) {
          const int ri = rg + kRowGroups32t * k, i = i0 + ri;
          if (i < iend) {
            const double sfull = g.S0d[i] + (double)S3[ri * kLd32t + c];
            re += sfull * cs * g.dAd[i];
            im -= sfull * sn * g.dAd[i];
          }
        }
      }
      re = warp_sum(re);
      im = warp_sum(im);
      if ((tid & 31) == 0) {
        atomicAdd(&bsum[2 * m], re);
        atomicAdd(&bsum[2 * m + 1], im);
      }
    }
  }
  __syncthreads();
  double lmax = (double)lmaxf;
  if (bad) lmax = __longlong_as_double(0x7ff8000000000000ll);
  finish_launch_deferred<kThreads32t>(ctl, si, lmax, tid == 0 ? bsum : zsum, red);
#undef RC
}

template <bool G2, int FM>
__global__ void __launch_bounds__(kThreads32t, 4) k_hydro32t(
    const float *__restrict__ sig, const float *__restrict__ uu, const float *__restrict__ ww,
    const float *__restrict__ Phi, const double *__restrict__ gRin, const double *__restrict__ gpin,
    float *__restrict__ so, float *__restrict__ uo, float *__restrict__ wo, SplitBf16 Sx, Ctl *ctl, Rows32 g,
    int *rowpend) {
  extern __shared__ float sm32t[];
  __shared__ double red[kThreads32t / 32];
  __shared__ double bsum[2 * kMaxModes], zsum[2 * kMaxModes];
  const int i0 = blockIdx.y * kTileI;
  if (i0 >= 3 && i0 + kTileI + 3 <= g.Nu)
    hydro32t_tile<G2, FM, true>(sig, uu, ww, Phi, gRin, gpin, so, uo, wo, Sx, ctl, g, sm32t, red, bsum, zsum);
  else
    hydro32t_tile<G2, FM, false>(sig, uu, ww, Phi, gRin, gpin, so, uo, wo, Sx, ctl, g, sm32t, red, bsum, zsum);
  if (rowpend) rowtile_done(rowpend + blockIdx.y);  // this tile's outputs are written
}

}  // namespace dg
