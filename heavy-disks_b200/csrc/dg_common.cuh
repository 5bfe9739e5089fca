// Shared device-side definitions for the diskgpu kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dg {

// Status bits raised on the device and read by the host at the end of a chunk.
enum : int {
  kStNonFinite = 1,   // dt or state became non-finite / non-positive
  kStTimeout = 2,     // a bounded device wait gave up
};

constexpr int kMaxModes = 9;        // C_0 .. C_8 accumulated on device
constexpr int kMaxRecords = 4096;   // device ring of mode records between host drains

// Device-resident control block of one disk: the step loop runs without host sync.
// Written only by the last CTA of the hydro kernel (and by host-side set-up).
struct Ctl {
  // --- host-written configuration (copied as one prefix, up to dtinv_bits) ---
  double t;          // simulation time at the start of the next step (advanced by the device)
  double tlim;       // loop stops when !(t < tlim)
  double cfl;        // Courant number of the next dt (0.3 in diskmain.cpp:100)
  double dt;         // dt of the next step
  double tnext;      // next mode-record time (diskmain.cpp:93)
  double dtout;      // record cadence (0.25)
  double mD;         // disk mass used to normalise C_m
  int fixed_dt;      // 1: dt was supplied by the host; no clip to tlim, no records
  int mode_every_step;  // accumulate C_0..C_mmax every step (diagnostic mode)
  int mmax;          // highest m accumulated in that mode
  int pad0;
  // --- device-maintained ---
  unsigned long long dtinv_bits;   // running max of (sR + sphi) as ordered bits
  unsigned int done_ctas;          // CTAs of the current launch that have finished
  int status;                      // kSt* bits
  long long step;                  // completed steps
  int nrec;                        // records written since the last host drain
  int ndiag;                       // per-step diagnostic rows written since the last drain
  double *diag;                    // per-step diagnostic ring (host-allocated on request), or null
  int diag_cap;                    // rows the ring holds
  int pend_active;                 // the running hydro launch advances the state (for k_step_finalize)
  double modesum[2 * kMaxModes];   // re/im sums for the record being built
  double last_modes[2 * kMaxModes];// the most recent per-step sums (mode_every_step)
  double rec[kMaxRecords][4];      // t, |C0|, |C2|, arg C2
};

template <typename T> struct cplx_of;
template <> struct cplx_of<double> { using type = double2; };
template <> struct cplx_of<float> { using type = float2; };

template <typename V>
__device__ __forceinline__ V cmul(V a, V b) {
  V r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

// Programmatic dependent launch.  A kernel launched with programmatic stream serialization
// may start while the kernel before it on the stream is still running: it does its
// prologue (shared memory, TMEM, constant tables), then pdl_wait() blocks until that kernel
// (and, transitively, everything before it) has completed with its writes visible.  With no
// such predecessor pdl_wait() returns at once.  pdl_trigger() lets the next kernel start.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Row-tile hand-over from the hydro step to the forward phi transform of the next step.
// The inverse phi transform (the hydro's predecessor) arms one counter per 16-row tile row
// with the hydro launch's column-tile count.  Each hydro CTA, once all of its writes are
// issued, decrements its row's counter with release semantics (rowtile_done).  A phi
// transform CTA waits, with acquire semantics, until the counter of the rows it reads is
// zero (rowtile_wait) instead of waiting for the whole hydro grid, so early rows are
// transformed while the hydro's last CTAs still run.  The phi transform is launched with
// programmatic dependence, i.e. only after every hydro CTA has started, so the counters
// always reach zero; the wait is bounded all the same (~1 s of SM clock, then kStTimeout).
__device__ __forceinline__ void rowtile_done(int *cnt) {
  __syncthreads();  // every thread's stores precede the release below
  if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.s32 [%0], -1;" ::"l"(cnt) : "memory");
}
__device__ __forceinline__ bool rowtile_wait(const int *cnt, int *status) {
  if (status && *(volatile int *)status) return false;  // an earlier wait gave up: the step is void
  long long start = 0;
  for (uint32_t it = 0;; ++it) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(cnt) : "memory");
    if (v <= 0) return true;
    if (it == 64) start = clock64();
    if (it > 64 && clock64() - start > (1ll << 31)) {
      if (status) atomicOr(status, kStTimeout);
      return false;
    }
    __nanosleep(128);
  }
}

// Ordered atomic max for non-negative doubles (NaN compares above +inf, so a NaN
// propagates into the max and is caught by the non-finite check).
__device__ __forceinline__ void atomic_max_pos(unsigned long long *addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide max that keeps NaN (fmax drops NaN, so NaN is tracked separately).
template <int NT>
__device__ __forceinline__ double block_max_nan(double v, double *red) {
  bool bad = !(v == v);
  v = bad ? 0.0 : v;
  v = warp_max(v);
  unsigned anybad = __any_sync(0xffffffffu, bad);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = anybad ? __longlong_as_double(0x7ff8000000000000ll) : v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    r = red[0];
    for (int k = 1; k < NT / 32; ++k) {
      double x = red[k];
      if (!(x == x) || !(r == r)) r = __longlong_as_double(0x7ff8000000000000ll);
      else r = fmax(r, x);
    }
  }
  __syncthreads();
  return r;  // valid in thread 0
}

}  // namespace dg
