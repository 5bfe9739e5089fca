// Plain-method (FP64) kernels: fused hydro step, CFL reduction, forces, mode sums,
// Kalnajs kernel samples, and launchers for the shared-memory FFT passes.
#include "kernels.h"
#include "hydro64.cuh"
#include "fft_smem.cuh"
#include "step_ctl.cuh"

namespace dg {

// Mode-sum contribution of one cell: Sigma cos(m phi) dA and -Sigma sin(m phi) dA
// (diskmain.cpp:76-80).
__device__ __forceinline__ void add_modes(double *msum, int nmodes, double s, int j, double dphi, double dA) {
  double phi = (j + 0.5) * dphi;
  for (int m = 0; m < nmodes; ++m) {
    double sn, cs;
    sincos(m * phi, &sn, &cs);
    msum[2 * m] += s * cs * dA;
    msum[2 * m + 1] -= s * sn * dA;
  }
}

// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(kHydroThreads) k_hydro64(
    const double *__restrict__ Sig, const double *__restrict__ vR, const double *__restrict__ vp,
    const double *__restrict__ Phi, const double *__restrict__ gRin, const double *__restrict__ gpin, int force_mode,
    double *__restrict__ So, double *__restrict__ vRo, double *__restrict__ vpo, Ctl *ctl, Geom64 g) {
  __shared__ double sS[kLI][kLJ], sVR[kLI][kLJ], sVP[kLI][kLJ], sP[kLI][kLJ], sPh[kLI][kLJ];
  __shared__ double sVR1[kSI][kSJ], sVP1[kSI][kSJ];
  __shared__ double fF[kTI + 1][kSJ], fFR[kTI + 1][kSJ], fFP[kTI + 1][kSJ];
  __shared__ double pF[3 * kTI][kTJ + 1];  // phi-face fluxes: rows [0,TI) F, [TI,2TI) FR, [2TI,3TI) FP
  __shared__ double red[kHydroThreads / 32];
  // transportR outputs reuse the (dead after the source stage) pressure / velocity tiles
  double(*s2S)[kLJ] = sP;
  double(*s2VR)[kLJ] = sVR;
  double(*s2VP)[kLJ] = sVP;

  const int Nu = g.Nu, Nphi = g.Nphi;
  const int i0 = blockIdx.y * kTI, j0 = blockIdx.x * kTJ;
  const StepInfo si = read_step_info(ctl, true);
  const double dt = si.dt;
  const int tid = threadIdx.x;
  double msum[2 * kMaxModes];
#pragma unroll
  for (int q = 0; q < 2 * kMaxModes; ++q) msum[q] = 0.0;
  double lmax = 0.0;

  if (!si.active) {
    // pass-through so a launch after the loop has ended leaves the state unchanged
    for (int c = tid; c < kTI * kTJ; c += kHydroThreads) {
      int i = i0 + c / kTJ, j = j0 + c % kTJ;
      if (i < Nu && j < Nphi) {
        size_t k = (size_t)i * Nphi + j;
        So[k] = Sig[k]; vRo[k] = vR[k]; vpo[k] = vp[k];
        lmax = fmax(lmax, cfl_rate64(g, i, So[k], vRo[k], vpo[k]));
      }
    }
    finish_launch<kHydroThreads>(ctl, si, lmax, msum, red);
    return;
  }

  // ---- load the halo region ----
  for (int c = tid; c < kLI * kLJ; c += kHydroThreads) {
    int li = c / kLJ, lj = c % kLJ;
    int i = i0 - kH + li;
    int j = j0 - kH + lj;
    j = ((j % Nphi) + Nphi) % Nphi;
    double s = 0.0, a = 0.0, b = 0.0, ph = 0.0;
    if (i >= 0 && i < Nu) {
      size_t k = (size_t)i * Nphi + j;
      s = Sig[k]; a = vR[k]; b = vp[k];
      if (force_mode == kForcePhi) ph = Phi[k];
    }
    sS[li][lj] = s; sVR[li][lj] = a; sVP[li][lj] = b; sPh[li][lj] = ph;
    sP[li][lj] = (i >= 0 && i < Nu) ? pres64(g, s) : 0.0;
  }
  __syncthreads();

  // ---- source (hydro.hpp:73-96) on rows i0-2 .. i0+TI+1 ----
  for (int c = tid; c < kSI * kSJ; c += kHydroThreads) {
    int si_ = c / kSJ, sj = c % kSJ;
    int i = i0 - 2 + si_;
    int li = si_ + 1, lj = sj + 1;
    double nvr = 0.0, nvp = 0.0;
    if (i >= 0 && i < Nu) {
      int im = i - 1 > 0 ? i - 1 : 0, ip = i + 1 < Nu - 1 ? i + 1 : Nu - 1;
      int lim = li + (im - i), lip = li + (ip - i);
      double Ri = g.R[i], iR = g.invR[i];
      double s = sS[li][lj];
      double dPdR = (sP[lip][lj] - sP[lim][lj]) * g.invdRc[i];
      double dPdphi = (sP[li][lj + 1] - sP[li][lj - 1]) * g.inv2dphi;
      double gR = g.gstar[i];
      double gp = 0.0;
      if (force_mode == kForcePhi) {  // kalnajs.hpp:71-78
        double dPhidphi = (sPh[li][lj + 1] - sPh[li][lj - 1]) * g.inv2dphi;
        double dPhidu;
        if (i == 0) dPhidu = (sPh[li + 1][lj] - sPh[li][lj]) * g.invdu;
        else if (i == Nu - 1) dPhidu = (sPh[li][lj] - sPh[li - 1][lj]) * g.invdu;
        else dPhidu = (sPh[li + 1][lj] - sPh[li - 1][lj]) * g.inv2du;
        gR += -dPhidu * iR;
        gp += -dPhidphi * iR;
      } else if (force_mode == kForceArrays) {
        int j = ((j0 - 2 + sj) % Nphi + Nphi) % Nphi;
        size_t k = (size_t)i * Nphi + j;
        gR += gRin[k];
        gp += gpin[k];
      }
      double vrc = sVR[li][lj], vpc = sVP[li][lj];
      double aR = -dPdR / s + gR + vpc * vpc * iR;
      double ap = -(1.0 / (s * Ri)) * dPdphi + gp - vrc * vpc * iR;
      nvr = vrc + dt * aR;
      nvp = vpc + dt * ap;
    }
    sVR1[si_][sj] = nvr;
    sVP1[si_][sj] = nvp;
  }
  __syncthreads();

  // ---- transportR fluxes (hydro.hpp:107-130) at faces f = i0 .. i0+TI ----
  // cell index i in source coordinates: si_ = i - (i0 - 2); Sigma at sS[si_ + 1][sj + 1]
  auto Ssrc = [&](int i, int sj) { return sS[i - (i0 - 2) + 1][sj + 1]; };
  auto VRsrc = [&](int i, int sj) { return sVR1[i - (i0 - 2)][sj]; };
  auto VPsrc = [&](int i, int sj) { return sVP1[i - (i0 - 2)][sj]; };
  for (int c = tid; c < (kTI + 1) * kSJ; c += kHydroThreads) {
    int fi = c / kSJ, sj = c % kSJ;
    int f = i0 + fi;
    double F = 0.0, FR = 0.0, FP = 0.0;
    if (f >= 1 && f <= Nu - 1) {
      double Af = g.Rf[f] * g.dphi;
      double idRl = g.invdRl[f], idRr = g.invdRr[f];
      double vf = 0.5 * (VRsrc(f - 1, sj) + VRsrc(f, sj));
      double sf, vRf, vpf;
      if (vf > 0) {
        int u = f - 1;
        bool sl = (u > 0 && u < Nu - 1);
        double kS = sl ? vanleer64(Ssrc(u + 1, sj) - Ssrc(u, sj), Ssrc(u, sj) - Ssrc(u - 1, sj)) : 0.0;
        double kR = sl ? vanleer64(VRsrc(u + 1, sj) - VRsrc(u, sj), VRsrc(u, sj) - VRsrc(u - 1, sj)) : 0.0;
        double kP = sl ? vanleer64(VPsrc(u + 1, sj) - VPsrc(u, sj), VPsrc(u, sj) - VPsrc(u - 1, sj)) : 0.0;
        sf = Ssrc(u, sj) + 0.5 * kS * (1.0 - vf * dt * idRl);
        vRf = VRsrc(u, sj) + 0.5 * kR * (1.0 - vf * dt * idRl);
        vpf = VPsrc(u, sj) + 0.5 * kP * (1.0 - vf * dt * idRl);
      } else {
        int u = f;
        bool sl = (u > 0 && u < Nu - 1);
        double kS = sl ? vanleer64(Ssrc(u + 1, sj) - Ssrc(u, sj), Ssrc(u, sj) - Ssrc(u - 1, sj)) : 0.0;
        double kR = sl ? vanleer64(VRsrc(u + 1, sj) - VRsrc(u, sj), VRsrc(u, sj) - VRsrc(u - 1, sj)) : 0.0;
        double kP = sl ? vanleer64(VPsrc(u + 1, sj) - VPsrc(u, sj), VPsrc(u, sj) - VPsrc(u - 1, sj)) : 0.0;
        sf = Ssrc(u, sj) - 0.5 * kS * (1.0 + vf * dt * idRr);
        vRf = VRsrc(u, sj) - 0.5 * kR * (1.0 + vf * dt * idRr);
        vpf = VPsrc(u, sj) - 0.5 * kP * (1.0 + vf * dt * idRr);
      }
      double fm = vf * sf * Af;
      F = fm; FR = fm * vRf; FP = fm * vpf;
    }
    fF[fi][sj] = F; fFR[fi][sj] = FR; fFP[fi][sj] = FP;
  }
  __syncthreads();

  // ---- transportR gather (hydro.hpp:131-139) on rows i0 .. i0+TI-1 ----
  for (int c = tid; c < kTI * kSJ; c += kHydroThreads) {
    int ri = c / kSJ, sj = c % kSJ;
    int i = i0 + ri;
    double ns = 0.0, a = 0.0, b = 0.0;
    if (i < Nu) {
      double s = Ssrc(i, sj), vr1 = VRsrc(i, sj), vp1 = VPsrc(i, sj);
      double mR = s * vr1, mp = s * vp1;
      double iV = g.invVol[i];
      ns = s + dt * (fF[ri][sj] - fF[ri + 1][sj]) * iV;
      double nmR = mR + dt * (fFR[ri][sj] - fFR[ri + 1][sj]) * iV;
      double nmP = mp + dt * (fFP[ri][sj] - fFP[ri + 1][sj]) * iV;
      double d = dmax_ref(ns, 1e-10);
      a = nmR / d;
      b = nmP / d;
    }
    s2S[ri][sj] = ns; s2VR[ri][sj] = a; s2VP[ri][sj] = b;
  }
  __syncthreads();

  // ---- transportPhi fluxes (hydro.hpp:150-169): face pj is j-1/2 of cell j0+pj ----
  // cells in R-output coordinates: column c <-> global j0 - 2 + c
  for (int c = tid; c < kTI * (kTJ + 1); c += kHydroThreads) {
    int ri = c / (kTJ + 1), pj = c % (kTJ + 1);
    int i = i0 + ri;
    double F = 0.0, FR = 0.0, FP = 0.0;
    if (i < Nu) {
      double idl = g.invdl[i], Aface = g.Rf[i + 1] - g.Rf[i];
      int cm = pj + 1, cc = pj + 2;  // cells j-1, j
      double vf = 0.5 * (s2VP[ri][cm] + s2VP[ri][cc]);
      double sf, vRf, vpf;
      int u = (vf > 0) ? cm : cc;
      double kS = vanleer64(s2S[ri][u + 1] - s2S[ri][u], s2S[ri][u] - s2S[ri][u - 1]);
      double kR = vanleer64(s2VR[ri][u + 1] - s2VR[ri][u], s2VR[ri][u] - s2VR[ri][u - 1]);
      double kP = vanleer64(s2VP[ri][u + 1] - s2VP[ri][u], s2VP[ri][u] - s2VP[ri][u - 1]);
      if (vf > 0) {
        sf = s2S[ri][u] + 0.5 * kS * (1.0 - vf * dt * idl);
        vRf = s2VR[ri][u] + 0.5 * kR * (1.0 - vf * dt * idl);
        vpf = s2VP[ri][u] + 0.5 * kP * (1.0 - vf * dt * idl);
      } else {
        sf = s2S[ri][u] - 0.5 * kS * (1.0 + vf * dt * idl);
        vRf = s2VR[ri][u] - 0.5 * kR * (1.0 + vf * dt * idl);
        vpf = s2VP[ri][u] - 0.5 * kP * (1.0 + vf * dt * idl);
      }
      double fm = vf * sf * Aface;
      F = fm; FR = fm * vRf; FP = fm * vpf;
    }
    pF[ri][pj] = F; pF[kTI + ri][pj] = FR; pF[2 * kTI + ri][pj] = FP;
  }
  __syncthreads();

  // ---- transportPhi gather (hydro.hpp:170-178) + floor (:69) + next-step CFL ----
  bool bad = false;
  for (int c = tid; c < kTI * kTJ; c += kHydroThreads) {
    int ri = c / kTJ, pj = c % kTJ;
    int i = i0 + ri, j = j0 + pj;
    if (i < Nu && j < Nphi) {
      int cc = pj + 2;
      double s = s2S[ri][cc], vr = s2VR[ri][cc], vpp = s2VP[ri][cc];
      double mR = s * vr, mp = s * vpp;
      double iV = g.invVol[i];
      double ns = s + dt * (pF[ri][pj] - pF[ri][pj + 1]) * iV;
      double nmR = mR + dt * (pF[kTI + ri][pj] - pF[kTI + ri][pj + 1]) * iV;
      double nmP = mp + dt * (pF[2 * kTI + ri][pj] - pF[2 * kTI + ri][pj + 1]) * iV;
      double d = dmax_ref(ns, 1e-10);
      double vro = nmR / d, vpo_ = nmP / d;
      double so = dmax_ref(ns, 1e-10);
      size_t k = (size_t)i * Nphi + j;
      So[k] = so; vRo[k] = vro; vpo[k] = vpo_;
      double rate = cfl_rate64(g, i, so, vro, vpo_);
      bad |= !(rate == rate) || !(vro == vro) || !(vpo_ == vpo_);
      lmax = fmax(lmax, rate);
      if (si.nmodes) {
        double dA = g.R[i] * (g.Rf[i + 1] - g.Rf[i]) * g.dphi;
        add_modes(msum, si.nmodes, so, j, g.dphi, dA);
      }
    }
  }
  if (bad) lmax = __longlong_as_double(0x7ff8000000000000ll);
  finish_launch<kHydroThreads>(ctl, si, lmax, msum, red);
}

// CFL reduction over a state (DiskHydro::timestep, hydro.hpp:48-61); the last CTA stores
// dt = cfl / max (clipped to tlim unless fixed_dt).  Optionally accumulates mode sums.
__global__ void __launch_bounds__(256) k_cfl64(const double *__restrict__ Sig, const double *__restrict__ vR,
                                               const double *__restrict__ vp, Ctl *ctl, Geom64 g, int nmodes,
                                               int record) {
  __shared__ double red[8];
  StepInfo si;
  si.t = ctl->t; si.dt = 0.0; si.tlim = ctl->tlim;
  si.active = false; si.advance_t = false;
  si.record = record != 0;
  si.nmodes = record && nmodes < 3 ? 3 : nmodes;
  nmodes = si.nmodes;
  double msum[2 * kMaxModes];
#pragma unroll
  for (int q = 0; q < 2 * kMaxModes; ++q) msum[q] = 0.0;
  double lmax = 0.0;
  const size_t n = (size_t)g.Nu * g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / g.Nphi), j = (int)(k % g.Nphi);
    double r = cfl_rate64(g, i, Sig[k], vR[k], vp[k]);
    if (!(r == r)) lmax = r;
    else if (lmax == lmax) lmax = fmax(lmax, r);
    if (nmodes) {
      double dA = g.R[i] * (g.Rf[i + 1] - g.Rf[i]) * g.dphi;
      add_modes(msum, nmodes, Sig[k], j, g.dphi, dA);
    }
  }
  finish_launch<256>(ctl, si, lmax, msum, red);
}

// Sums Sigma e^{-i m phi} dA for m < nmodes (diskmain.cpp:72-84) into out[2m], out[2m+1].
__global__ void __launch_bounds__(256) k_modes64(const double *__restrict__ Sig, Geom64 g, int nmodes,
                                                 double *__restrict__ out) {
  __shared__ double red[8];
  double msum[2 * kMaxModes];
#pragma unroll
  for (int q = 0; q < 2 * kMaxModes; ++q) msum[q] = 0.0;
  const size_t n = (size_t)g.Nu * g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / g.Nphi), j = (int)(k % g.Nphi);
    double dA = g.R[i] * (g.Rf[i + 1] - g.Rf[i]) * g.dphi;
    add_modes(msum, nmodes, Sig[k], j, g.dphi, dA);
  }
  for (int q = 0; q < 2 * nmodes; ++q) {
    double v = warp_sum(msum[q]);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < 8; ++w) s += red[w];
      atomicAdd(&out[q], s);
    }
    __syncthreads();
  }
}

// KalnajsSolver::forces (kalnajs.hpp:65-80) as a standalone pass.
__global__ void k_forces64(const double *__restrict__ Phi, double *__restrict__ gR, double *__restrict__ gp,
                           Geom64 g) {
  const size_t n = (size_t)g.Nu * g.Nphi;
  const int Nu = g.Nu, Nphi = g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / Nphi), j = (int)(k % Nphi);
    int jm = (j - 1 + Nphi) % Nphi, jp = (j + 1) % Nphi;
    double dPhidphi = (Phi[(size_t)i * Nphi + jp] - Phi[(size_t)i * Nphi + jm]) / (2.0 * g.dphi);
    double dPhidu;
    if (i == 0) dPhidu = (Phi[(size_t)(i + 1) * Nphi + j] - Phi[k]) / g.du;
    else if (i == Nu - 1) dPhidu = (Phi[k] - Phi[(size_t)(i - 1) * Nphi + j]) / g.du;
    else dPhidu = (Phi[(size_t)(i + 1) * Nphi + j] - Phi[(size_t)(i - 1) * Nphi + j]) / (2.0 * g.du);
    gR[k] = -dPhidu / g.R[i];
    gp[k] = -dPhidphi / g.R[i];
  }
}

// Samples of the softened log-spiral kernel at wrapped offsets (kalnajs.hpp:106-112).
__global__ void k_kernel_samples64(double *__restrict__ out, int M, int Nphi, double du, double dphi, double eps) {
  const size_t n = (size_t)M * Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int p = (int)(k / Nphi), q = (int)(k % Nphi);
    int ioff = (p <= M / 2) ? p : p - M;
    double Du = ioff * du;
    double Dphi = q * dphi;
    out[k] = 1.0 / sqrt(2.0 * cosh(Du) - 2.0 * cos(Dphi) + eps);
  }
}

// global sums mass = sum Sigma dA, angmom = sum Sigma vphi R dA (FP64)
__global__ void k_conserved64(const double *__restrict__ Sig, const double *__restrict__ vp, Geom64 g,
                              double *__restrict__ out) {
  __shared__ double red[2][8];
  double m = 0.0, L = 0.0;
  const size_t n = (size_t)g.Nu * g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / g.Nphi);
    double dA = g.R[i] * (g.Rf[i + 1] - g.Rf[i]) * g.dphi;
    m += Sig[k] * dA;
    L += Sig[k] * vp[k] * g.R[i] * dA;
  }
  m = warp_sum(m);
  L = warp_sum(L);
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = m; red[1][threadIdx.x >> 5] = L; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += red[0][w]; b += red[1][w]; }
    atomicAdd(&out[0], a);
    atomicAdd(&out[1], b);
  }
}

// ---------------------------------------------------------------------------------
// host launchers
static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

cudaError_t launch_hydro64(const double *Sig, const double *vR, const double *vp, const double *Phi,
                           const double *gR, const double *gp, int force_mode, double *So, double *vRo, double *vpo,
                           Ctl *ctl, const Geom64 &g, cudaStream_t st) {
  dim3 grid((g.Nphi + kTJ - 1) / kTJ, (g.Nu + kTI - 1) / kTI);
  k_hydro64<<<grid, kHydroThreads, 0, st>>>(Sig, vR, vp, Phi, gR, gp, force_mode, So, vRo, vpo, ctl, g);
  return cudaGetLastError();
}

cudaError_t launch_cfl64(const double *Sig, const double *vR, const double *vp, Ctl *ctl, const Geom64 &g,
                         int nmodes, int record, cudaStream_t st) {
  size_t n = (size_t)g.Nu * g.Nphi;
  int blocks = (int)((n + 255) / 256);
  int cap = sm_count() * 4;
  if (blocks > cap) blocks = cap;
  k_cfl64<<<blocks, 256, 0, st>>>(Sig, vR, vp, ctl, g, nmodes, record);
  return cudaGetLastError();
}

cudaError_t launch_modes64(const double *Sig, const Geom64 &g, int nmodes, double *out, cudaStream_t st) {
  size_t n = (size_t)g.Nu * g.Nphi;
  int blocks = (int)((n + 255) / 256);
  if (blocks > sm_count() * 4) blocks = sm_count() * 4;
  cudaMemsetAsync(out, 0, 2 * nmodes * sizeof(double), st);
  k_modes64<<<blocks, 256, 0, st>>>(Sig, g, nmodes, out);
  return cudaGetLastError();
}

cudaError_t launch_forces64(const double *Phi, double *gR, double *gp, const Geom64 &g, cudaStream_t st) {
  size_t n = (size_t)g.Nu * g.Nphi;
  int blocks = (int)((n + 255) / 256);
  if (blocks > sm_count() * 8) blocks = sm_count() * 8;
  k_forces64<<<blocks, 256, 0, st>>>(Phi, gR, gp, g);
  return cudaGetLastError();
}

cudaError_t launch_conserved64(const double *Sig, const double *vp, const Geom64 &g, double *out2,
                               cudaStream_t st) {
  size_t n = (size_t)g.Nu * g.Nphi;
  int blocks = (int)((n + 255) / 256);
  if (blocks > sm_count() * 4) blocks = sm_count() * 4;
  cudaMemsetAsync(out2, 0, 2 * sizeof(double), st);
  k_conserved64<<<blocks, 256, 0, st>>>(Sig, vp, g, out2);
  return cudaGetLastError();
}

cudaError_t launch_kernel_samples64(double *out, int M, int Nphi, double du, double dphi, double eps,
                                    cudaStream_t st) {
  size_t n = (size_t)M * Nphi;
  int blocks = (int)((n + 255) / 256);
  if (blocks > sm_count() * 8) blocks = sm_count() * 8;
  k_kernel_samples64<<<blocks, 256, 0, st>>>(out, M, Nphi, du, dphi, eps);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// FFT pass launchers.  Each picks (E, nb, threads) with nb * n <= E * threads.
bool make_fft_plan(int n, FftPlan *pl) {
  pl->n = n;
  pl->n4 = pl->n2 = pl->n3 = pl->n5 = 0;
  int m = n;
  while (m % 4 == 0) { pl->n4++; m /= 4; }
  while (m % 2 == 0) { pl->n2++; m /= 2; }
  while (m % 3 == 0) { pl->n3++; m /= 3; }
  while (m % 5 == 0) { pl->n5++; m /= 5; }
  return m == 1 && n >= 1;
}

struct FftShape {
  int E, nb, threads;
  size_t smem;
};

template <typename V>
static FftShape fft_shape(int n, int count) {
  // Prefer 256 threads and 8 elements per thread; shrink nb to fill >= 2 waves of SMs.
  FftShape s;
  s.E = 8;
  s.threads = 256;
  if (n > s.E * s.threads) {
    s.threads = (n + s.E - 1) / s.E;
    s.threads = ((s.threads + 31) / 32) * 32;
    if (s.threads > 1024) s.threads = 1024;  // n <= 8192
  }
  s.nb = (s.E * s.threads) / n;
  if (s.nb < 1) s.nb = 1;
  int want = 2 * sm_count();
  while (s.nb > 1 && (count + s.nb - 1) / s.nb < want) s.nb /= 2;
  s.smem = (size_t)s.nb * n * sizeof(V);
  return s;
}


// Raise the dynamic shared-memory limit of every FFT pass once, outside any graph capture.
cudaError_t prepare_fft_kernels() {
  static bool done = false;
  if (done) return cudaSuccess;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const void *fns[] = {(const void *)k_phi_fwd<double, 8>, (const void *)k_u_conv<double, 8>,
                       (const void *)k_phi_inv<double, 8>};
  for (const void *f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e != cudaSuccess) return e;
  }
  done = true;
  return cudaSuccess;
}

template <typename T>
cudaError_t launch_phi_fwd(const T *src, int nrows, int Nphi, const T *rowscale, typename cplx_of<T>::type *W,
                           int ldw, const FftPlan &pl, const typename cplx_of<T>::type *roots, cudaStream_t st) {
  using V = typename cplx_of<T>::type;
  FftShape s = fft_shape<V>(Nphi, (nrows + 1) / 2);
  int blocks = (nrows + 2 * s.nb - 1) / (2 * s.nb);
  {
    k_phi_fwd<T, 8><<<blocks, s.threads, s.smem, st>>>(src, nrows, Nphi, rowscale, W, ldw, pl, roots, s.nb);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_u_conv(typename cplx_of<T>::type *W, int ldw, int Nc, int nin, int nout, const FftPlan &pl,
                          const typename cplx_of<T>::type *roots, const typename cplx_of<T>::type *khat,
                          typename cplx_of<T>::type *kout, cudaStream_t st) {
  using V = typename cplx_of<T>::type;
  FftShape s = fft_shape<V>(pl.n, Nc);
  int blocks = (Nc + s.nb - 1) / s.nb;
  {
    k_u_conv<T, 8><<<blocks, s.threads, s.smem, st>>>(W, ldw, Nc, nin, nout, pl, roots, khat, kout, s.nb);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_phi_inv(const typename cplx_of<T>::type *W, int ldw, int nrows, int Nphi, const FftPlan &pl,
                           const typename cplx_of<T>::type *roots, T pref, const T *sqrtR, T *out, cudaStream_t st) {
  using V = typename cplx_of<T>::type;
  FftShape s = fft_shape<V>(Nphi, (nrows + 1) / 2);
  int blocks = (nrows + 2 * s.nb - 1) / (2 * s.nb);
  {
    k_phi_inv<T, 8><<<blocks, s.threads, s.smem, st>>>(W, ldw, nrows, Nphi, pl, roots, pref, sqrtR, out, s.nb);
  }
  return cudaGetLastError();
}

template cudaError_t launch_phi_fwd<double>(const double *, int, int, const double *, double2 *, int,
                                            const FftPlan &, const double2 *, cudaStream_t);
template cudaError_t launch_u_conv<double>(double2 *, int, int, int, int, const FftPlan &, const double2 *,
                                           const double2 *, double2 *, cudaStream_t);
template cudaError_t launch_phi_inv<double>(const double2 *, int, int, int, const FftPlan &, const double2 *,
                                            double, const double *, double *, cudaStream_t);

}  // namespace dg
