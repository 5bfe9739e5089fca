// End-of-launch protocol shared by the FP64 and mixed hydro / CFL kernels.
#pragma once

#include "dg_common.cuh"

namespace dg {

// ---------------------------------------------------------------------------------
// End-of-launch bookkeeping shared by the hydro and CFL kernels.  Every CTA folds its
// partial max of (sR + sphi) and its mode sums into the control block; the last CTA to
// finish advances t, derives the next dt (diskmain.cpp:100-101: dt = cfl / max, clipped
// so that t lands on tlim), appends a mode record when one is due (diskmain.cpp:93-99),
// and resets the accumulators for the next launch.
struct StepInfo {
  double t, dt, tlim;
  bool active;     // this launch advances the state
  bool advance_t;  // the last CTA adds dt to t (hydro launches)
  bool record;     // the new state is due for a mode record
  int nmodes;      // number of m accumulated (0 = none)
};

// The control-block fields a launch decides on, loaded in one go (a kernel can issue these
// loads early and derive its StepInfo after other waits).
struct StepRaw {
  double t, dt, tlim, tnext;
  int status, fixed_dt, mode_every_step, mmax;
};
__device__ __forceinline__ StepRaw load_step_raw(const Ctl *ctl) {
  StepRaw r;
  r.t = ctl->t;
  r.dt = ctl->dt;
  r.tlim = ctl->tlim;
  r.tnext = ctl->tnext;
  r.status = ctl->status;
  r.fixed_dt = ctl->fixed_dt;
  r.mode_every_step = ctl->mode_every_step;
  r.mmax = ctl->mmax;
  return r;
}

// force_active >= 0 replaces the status / tlim test (k_step_finalize: the decision the hydro
// launch took at its start, before its own CTAs could raise status bits)
__device__ __forceinline__ StepInfo step_info_from(const StepRaw &r, bool advance_t, int force_active = -1) {
  StepInfo s;
  s.t = r.t;
  s.dt = r.dt;
  s.tlim = r.tlim;
  s.advance_t = advance_t;
  s.active = force_active >= 0 ? force_active != 0 : (r.status == 0) && (r.fixed_dt || s.t < s.tlim);
  s.record = false;
  s.nmodes = 0;
  if (advance_t && s.active && !r.fixed_dt) {
    double tn = s.t + s.dt;
    s.record = (tn < s.tlim) && (tn >= r.tnext - 1e-12);
  }
  if (s.record) s.nmodes = 3;  // C0, C1, C2
  if (r.mode_every_step && s.active) s.nmodes = r.mmax + 1 > s.nmodes ? r.mmax + 1 : s.nmodes;
  if (s.nmodes > kMaxModes) s.nmodes = kMaxModes;
  return s;
}

__device__ __forceinline__ StepInfo read_step_info(const Ctl *ctl, bool advance_t, int force_active = -1) {
  return step_info_from(load_step_raw(ctl), advance_t, force_active);
}

// A CTA's share of the launch: its CFL max and mode sums, folded into the control block
// with fire-and-forget atomics (the result of thread 0's block reduction).
template <int NT>
__device__ __forceinline__ double fold_launch_sums(Ctl *ctl, const StepInfo &si, double local_max, const double *msum,
                                                   double *red) {
  double bmax = block_max_nan<NT>(local_max, red);
  // mode sums: block reduce each component
  for (int q = 0; q < 2 * si.nmodes; ++q) {
    double v = warp_sum(msum[q]);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int k = 0; k < NT / 32; ++k) s += red[k];
      atomicAdd(&ctl->modesum[q], s);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) atomic_max_pos(&ctl->dtinv_bits, bmax);
  return bmax;
}

// The end of a launch: t, dt, records and diagnostics from the folded sums (thread 0 of
// the last CTA, or k_step_finalize after the whole launch).
__device__ __forceinline__ void finalize_launch(Ctl *ctl, const StepInfo &si);

template <int NT>
__device__ __forceinline__ void finish_launch(Ctl *ctl, const StepInfo &si, double local_max, const double *msum, double *red) {
  __shared__ bool am_last;
  fold_launch_sums<NT>(ctl, si, local_max, msum, red);
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned prev = atomicAdd(&ctl->done_ctas, 1u);
    am_last = (prev == gridDim.x * gridDim.y - 1);
  }
  __syncthreads();
  if (!am_last || threadIdx.x != 0) return;
  __threadfence();
  finalize_launch(ctl, si);
}

// Deferred end of launch (the mixed tile hydro kernels): the CTAs only fold their sums;
// k_step_finalize, launched right after with programmatic dependence, waits for the whole
// launch and finalises, so no CTA waits on a control-block round trip before it exits.
template <int NT>
__device__ __forceinline__ void finish_launch_deferred(Ctl *ctl, const StepInfo &si, double local_max,
                                                       const double *msum, double *red) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.y == 0) ctl->pend_active = si.active ? 1 : 0;
  fold_launch_sums<NT>(ctl, si, local_max, msum, red);
}

__device__ __forceinline__ void finalize_launch(Ctl *ctl, const StepInfo &si) {
  double dtinv = __longlong_as_double((long long)atomicAdd(&ctl->dtinv_bits, 0ull));
  dtinv = (dtinv < 1e-30) ? 1e-30 : dtinv;  // reduction starts at 1e-30 (hydro.hpp:49)
  double t = si.t;
  if (si.active && si.advance_t) {
    t = si.t + si.dt;
    ctl->t = t;
    ctl->step += 1;
  }
  double dtn = ctl->cfl / dtinv;
  if (!(dtn > 0.0) || !(dtn < 1e300)) ctl->status |= kStNonFinite;
  if (!ctl->fixed_dt && t + dtn > ctl->tlim) dtn = ctl->tlim - t;  // diskmain.cpp:101
  ctl->dt = dtn;
  if (si.nmodes > 0) {
    for (int q = 0; q < 2 * si.nmodes; ++q) ctl->last_modes[q] = ctl->modesum[q];
    if (si.record) {
      const double mD = ctl->mD;
      double re0 = ctl->modesum[0], im0 = ctl->modesum[1];
      double re2 = ctl->modesum[4], im2 = ctl->modesum[5];
      int k = ctl->nrec;
      if (k < kMaxRecords) {
        ctl->rec[k][0] = t;
        ctl->rec[k][1] = sqrt(re0 * re0 + im0 * im0) / mD;
        ctl->rec[k][2] = sqrt(re2 * re2 + im2 * im2) / mD;
        ctl->rec[k][3] = atan2(im2, re2);
        ctl->nrec = k + 1;
      }
      ctl->tnext += ctl->dtout;
    }
    // per-step diagnostic row: t, then Re/Im of sum Sigma e^{-i m phi} dA for m = 0..mmax
    if (ctl->mode_every_step && si.active && si.advance_t && ctl->diag && ctl->ndiag < ctl->diag_cap) {
      const int w = 1 + 2 * (ctl->mmax + 1);
      double *row = ctl->diag + (size_t)ctl->ndiag * w;
      row[0] = t;
      for (int q = 0; q < 2 * (ctl->mmax + 1); ++q) row[1 + q] = ctl->modesum[q];
      ctl->ndiag += 1;
    }
    for (int q = 0; q < 2 * kMaxModes; ++q) ctl->modesum[q] = 0.0;
  }
  ctl->dtinv_bits = 0ull;
  __threadfence();
  ctl->done_ctas = 0u;
}

}  // namespace dg
