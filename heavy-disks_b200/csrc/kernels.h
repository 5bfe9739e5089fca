// Host-side declarations of the diskgpu kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include "dg_common.cuh"
#include "hydro64.cuh"
#include "fft_smem.cuh"

namespace dg {

// plain-method (FP64) path
cudaError_t launch_hydro64(const double *Sig, const double *vR, const double *vp, const double *Phi,
                           const double *gR, const double *gp, int force_mode, double *So, double *vRo, double *vpo,
                           Ctl *ctl, const Geom64 &g, cudaStream_t st);
cudaError_t launch_cfl64(const double *Sig, const double *vR, const double *vp, Ctl *ctl, const Geom64 &g,
                         int nmodes, int record, cudaStream_t st);
cudaError_t launch_modes64(const double *Sig, const Geom64 &g, int nmodes, double *out, cudaStream_t st);
cudaError_t launch_forces64(const double *Phi, double *gR, double *gp, const Geom64 &g, cudaStream_t st);
cudaError_t launch_conserved64(const double *Sig, const double *vp, const Geom64 &g, double *out2, cudaStream_t st);
cudaError_t launch_kernel_samples64(double *out, int M, int Nphi, double du, double dphi, double eps,
                                    cudaStream_t st);

bool make_fft_plan(int n, FftPlan *pl);
cudaError_t prepare_fft_kernels();
template <typename T>
cudaError_t launch_phi_fwd(const T *src, int nrows, int Nphi, const T *rowscale, typename cplx_of<T>::type *W,
                           int ldw, const FftPlan &pl, const typename cplx_of<T>::type *roots, cudaStream_t st);
template <typename T>
cudaError_t launch_u_conv(typename cplx_of<T>::type *W, int ldw, int Nc, int nin, int nout, const FftPlan &pl,
                          const typename cplx_of<T>::type *roots, const typename cplx_of<T>::type *khat,
                          typename cplx_of<T>::type *kout, cudaStream_t st);
template <typename T>
cudaError_t launch_phi_inv(const typename cplx_of<T>::type *W, int ldw, int nrows, int Nphi, const FftPlan &pl,
                           const typename cplx_of<T>::type *roots, T pref, const T *sqrtR, T *out, cudaStream_t st);

}  // namespace dg
