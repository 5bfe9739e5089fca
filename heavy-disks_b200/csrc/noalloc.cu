// Allocation-free variant of the CFL time step (dg_timestep_static, include/diskgpu.h).
//
// Some callers cannot allocate device memory at the moment they need a time step: hosts
// whose device memory is owned by a pool or framework that forbids any other allocation
// after start-up, and fixed-budget loops that must not call into the allocator (a
// cudaMalloc can synchronise the device and its cost is unbounded).  This entry point
// computes dt = cfl / max_ij (sR + sphi) (the reference's DiskHydro::timestep) from
// caller-owned device arrays into a caller-owned device double, using no memory of its
// own except the file-scope scratch array below.
//
// The scratch holds one per-row maximum, so the largest grid is kMaxRows radial rows.
// It lives in every device that loads this library until the process exits.  Its device
// address is looked up once per device (cudaGetSymbolAddress) on the first call made with
// that device current; make that first call before any stream capture.  The looked-up
// address is kept for the life of the process: after cudaDeviceReset on a device, this
// entry point must not be called on that device again.  A non-finite value in the state
// makes dt NaN (the reference's std::max would skip it).  All calls share
// the one array and it keeps the last call's contents: calls that overlap on the GPU
// (different streams, no ordering between them) race on it.  Every row slot a call reads
// is written by the same call first, so nothing needs clearing between calls.
#include <cmath>
#include <cstring>
#include <mutex>

#include "diskgpu.h"

namespace {

constexpr int kMaxRows = 8192;  // 64 KiB of scratch per device
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_cfl_row_max[kMaxRows];

std::mutex g_mu;
double *g_scratch[kMaxDevices] = {};

__device__ __forceinline__ double nan_max(double a, double b) {
  if (!(a == a) || !(b == b)) return __longlong_as_double(0x7ff8000000000000ll);
  return a > b ? a : b;
}

// One block per radial row i: the row's max of (|vR| + cs)/dR + (|vphi| + cs)/(R dphi)
// with the grid of hydro.hpp:31-38 recomputed on the device.
__global__ void __launch_bounds__(256) k_cfl_rows(const double *__restrict__ S, const double *__restrict__ vR,
                                                  const double *__restrict__ vp, int Nphi, double umin, double du,
                                                  double dphi, double K, double gam, double *__restrict__ rowmax) {
  __shared__ double red[8];
  const int i = blockIdx.x;
  const double R = exp(umin + (i + 0.5) * du);
  const double dR = exp(umin + (i + 1) * du) - exp(umin + i * du);
  const double dl = R * dphi;
  double m = 0.0;
  for (int j = threadIdx.x; j < Nphi; j += blockDim.x) {
    const size_t k = (size_t)i * Nphi + j;
    double s = S[k];
    s = (s < 1e-12) ? 1e-12 : s;
    const double cs = sqrt(gam * K * pow(s, gam - 1.0));
    m = nan_max(m, (fabs(vR[k]) + cs) / dR + (fabs(vp[k]) + cs) / dl);
  }
  for (int o = 16; o > 0; o >>= 1) m = nan_max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = nan_max(r, red[w]);
    rowmax[i] = r;
  }
}

__global__ void __launch_bounds__(256) k_cfl_rows_to_dt(const double *__restrict__ rowmax, int Nu, double cfl,
                                                        double *__restrict__ dt) {
  __shared__ double red[8];
  double m = 0.0;
  for (int i = threadIdx.x; i < Nu; i += blockDim.x) m = nan_max(m, rowmax[i]);
  for (int o = 16; o > 0; o >>= 1) m = nan_max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = red[0];
    for (int w = 1; w < 8; ++w) r = nan_max(r, red[w]);
    if (r == r && r < 1e-30) r = 1e-30;  // the reference's reduction starts at 1e-30
    *dt = cfl / r;
  }
}

}  // namespace

extern "C" int dg_timestep_static(const double *Sig, const double *vR, const double *vp, int Nu, int Nphi, double Rin,
                                  double Rout, double Kpoly, double gamma_gas, double cfl, double *dt, void *stream) {
  if (!Sig || !vR || !vp || !dt || Nu < 1 || Nphi < 1 || !(Rin > 0) || !(Rout > Rin) || !(cfl > 0))
    return DG_ERR_INVALID;
  if (Nu > kMaxRows) return DG_ERR_UNSUPPORTED;  // more radial rows than the scratch holds
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DG_ERR_CUDA;
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
      double *ptr = nullptr;
      if (cudaGetSymbolAddress((void **)&ptr, g_cfl_row_max) != cudaSuccess || !ptr) return DG_ERR_CUDA;
      g_scratch[dev] = ptr;
    }
    scratch = g_scratch[dev];
  }
  const double umin = std::log(Rin), umax = std::log(Rout);
  const double du = (umax - umin) / Nu, dphi = 2.0 * M_PI / Nphi;
  cudaStream_t st = (cudaStream_t)stream;
  // an error left by earlier work is not this call's: report it without launching
  if (cudaPeekAtLastError() != cudaSuccess) return DG_ERR_CUDA;
  k_cfl_rows<<<Nu, 256, 0, st>>>(Sig, vR, vp, Nphi, umin, du, dphi, Kpoly, gamma_gas, scratch);
  if (cudaGetLastError() != cudaSuccess) return DG_ERR_CUDA;
  k_cfl_rows_to_dt<<<1, 256, 0, st>>>(scratch, Nu, cfl, dt);
  if (cudaGetLastError() != cudaSuccess) return DG_ERR_CUDA;
  return DG_OK;
}
