// Shared-memory mixed-radix (4, 2, 3, 5) Stockham FFT used by the plain (FP64) gravity
// path, and the three passes of the Kalnajs convolution built from it.
//
// The convolution restates diskfft/src/kalnajs.hpp:48-63 (potential) and :105-116
// (kernel table): a 2-D real-to-complex transform of the M x Nphi zero-padded field
// (M = 2 Nu), a complex multiply by khat, and the inverse.  It is split into:
//   pass 1  (phi_fwd)  rows i -> half spectrum in phi, two real rows packed per complex
//                      transform, written transposed as W[m][i] (mode-major);
//   pass 2  (u_conv)   per mode m: length-M transform along u (rows >= Nu are the
//                      implicit zero padding), multiply by khat[m][p], inverse, keep Nu;
//   pass 3  (phi_inv)  rows i <- Hermitian half spectrum (c2r), scaled by
//                      -G du dphi / (M Nphi) / sqrt(R_i).
// Each CTA holds nb whole transforms in shared memory; one stage reads every element
// into registers, applies twiddles and the radix-R butterfly, syncs, and writes the
// Stockham-permuted result back in place.
#pragma once

#include "dg_common.cuh"

namespace dg {

// n = 4^n4 * 2^n2 * 3^n3 * 5^n5; stages run in that order.
struct FftPlan {
  int n;
  int n4, n2, n3, n5;
};

template <typename V>
__device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V>
__device__ __forceinline__ V csub(V a, V b) { V r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
// multiply by -i (sign < 0) or +i (sign > 0)
template <typename V>
__device__ __forceinline__ V cmul_i(V a, int sign) {
  V r;
  if (sign < 0) { r.x = a.y; r.y = -a.x; } else { r.x = -a.y; r.y = a.x; }
  return r;
}

template <typename V, int R> struct Bfly;

template <typename V> struct Bfly<V, 2> {
  static __device__ __forceinline__ void run(V *v, int) {
    V a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <typename V> struct Bfly<V, 4> {
  static __device__ __forceinline__ void run(V *v, int sign) {
    V a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    V a2 = cadd(v[1], v[3]), a3 = cmul_i(csub(v[1], v[3]), sign);
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3);
    v[3] = csub(a1, a3);
  }
};

template <typename V> struct Bfly<V, 3> {
  static __device__ __forceinline__ void run(V *v, int sign) {
    using T = decltype(v[0].x);
    const T h = (T)0.86602540378443864676;  // sqrt(3)/2
    V t1 = cadd(v[1], v[2]);
    V t2;
    t2.x = v[0].x - (T)0.5 * t1.x;
    t2.y = v[0].y - (T)0.5 * t1.y;
    V d = csub(v[1], v[2]);
    V t3 = cmul_i(d, sign);
    t3.x *= h;
    t3.y *= h;
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};

template <typename V> struct Bfly<V, 5> {
  static __device__ __forceinline__ void run(V *v, int sign) {
    using T = decltype(v[0].x);
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;  // cos 2pi/5, cos 4pi/5
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;   // sin 2pi/5, sin 4pi/5
    V t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    V t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    V a1, a2, b1, b2;
    a1.x = v[0].x + c1 * t1.x + c2 * t2.x; a1.y = v[0].y + c1 * t1.y + c2 * t2.y;
    a2.x = v[0].x + c2 * t1.x + c1 * t2.x; a2.y = v[0].y + c2 * t1.y + c1 * t2.y;
    b1.x = s1 * t3.x + s2 * t4.x; b1.y = s1 * t3.y + s2 * t4.y;
    b2.x = s2 * t3.x - s1 * t4.x; b2.y = s2 * t3.y - s1 * t4.y;
    V ib1 = cmul_i(b1, sign), ib2 = cmul_i(b2, sign);
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, ib1);
    v[4] = csub(a1, ib1);
    v[2] = cadd(a2, ib2);
    v[3] = csub(a2, ib2);
  }
};

// One Stockham stage over nb transforms of length n held contiguously in buf.
// roots[t] = exp(-2 pi i t / n); the inverse uses the conjugate.
template <typename V, int R, int PER>
__device__ __forceinline__ void fft_stage(V *buf, int n, int nb, int Ns, int sign, const V *__restrict__ roots) {
  const int m = n / R;
  const int nbf = nb * m;
  const int tstep = n / (Ns * R);
  V v[PER][R];
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int b = threadIdx.x + q * blockDim.x;
    if (b < nbf) {
      const int t = b / m, j = b - t * m;
      const V *x = buf + t * n;
      const int k = j % Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        V a = x[j + r * m];
        if (r > 0 && k > 0) {
          V w = __ldg(&roots[r * k * tstep]);
          if (sign > 0) w.y = -w.y;
          a = cmul(a, w);
        }
        v[q][r] = a;
      }
      Bfly<V, R>::run(v[q], sign);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int b = threadIdx.x + q * blockDim.x;
    if (b < nbf) {
      const int t = b / m, j = b - t * m;
      V *x = buf + t * n;
      const int k = j % Ns;
      const int base = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) x[base + r * Ns] = v[q][r];
    }
  }
  __syncthreads();
}

// Full transform of nb sequences of length plan.n in shared memory.  Requires
// nb * n <= E * blockDim.x (each thread holds at most E elements per stage).
template <typename V, int E>
__device__ __forceinline__ void smem_fft(V *buf, int nb, const FftPlan &pl, int sign, const V *__restrict__ roots) {
  int Ns = 1;
  for (int s = 0; s < pl.n4; ++s, Ns *= 4) fft_stage<V, 4, (E + 3) / 4>(buf, pl.n, nb, Ns, sign, roots);
  for (int s = 0; s < pl.n2; ++s, Ns *= 2) fft_stage<V, 2, (E + 1) / 2>(buf, pl.n, nb, Ns, sign, roots);
  for (int s = 0; s < pl.n3; ++s, Ns *= 3) fft_stage<V, 3, (E + 2) / 3>(buf, pl.n, nb, Ns, sign, roots);
  for (int s = 0; s < pl.n5; ++s, Ns *= 5) fft_stage<V, 5, (E + 4) / 5>(buf, pl.n, nb, Ns, sign, roots);
}

// ---------------------------------------------------------------------------------
// pass 1: rows -> transposed half spectrum.  Rows row0 .. row0+2nb-1 of src (nrows x Nphi)
// are multiplied by rowscale[i] (kalnajs.hpp:51: R^{3/2} Sigma; NULL = 1), packed two rows
// per complex transform, transformed forward along phi and unpacked into
// W[m * ldw + i], m < Nc.
template <typename T, int E>
__global__ void __launch_bounds__(1024) k_phi_fwd(const T *__restrict__ src, int nrows, int Nphi,
                                                 const T *__restrict__ rowscale,
                                                 typename cplx_of<T>::type *__restrict__ W, int ldw,
                                                 FftPlan pl, const typename cplx_of<T>::type *__restrict__ roots,
                                                 int nb) {
  using V = typename cplx_of<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *buf = reinterpret_cast<V *>(smem_raw);
  const int row0 = blockIdx.x * 2 * nb;
  const int total = nb * Nphi;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int t = idx / Nphi, j = idx - t * Nphi;
    const int r0 = row0 + 2 * t, r1 = r0 + 1;
    V z;
    z.x = (r0 < nrows) ? (rowscale ? rowscale[r0] * src[(size_t)r0 * Nphi + j] : src[(size_t)r0 * Nphi + j]) : (T)0;
    z.y = (r1 < nrows) ? (rowscale ? rowscale[r1] * src[(size_t)r1 * Nphi + j] : src[(size_t)r1 * Nphi + j]) : (T)0;
    buf[idx] = z;
  }
  __syncthreads();
  smem_fft<V, E>(buf, nb, pl, -1, roots);
  const int Nc = Nphi / 2 + 1;
  const int tot2 = nb * Nc;
  for (int idx = threadIdx.x; idx < tot2; idx += blockDim.x) {
    const int m = idx / nb, t = idx - m * nb;
    const int r0 = row0 + 2 * t;
    const V *Z = buf + t * Nphi;
    const V a = Z[m], c = Z[(Nphi - m) % Nphi];
    V A, B;
    A.x = (T)0.5 * (a.x + c.x);
    A.y = (T)0.5 * (a.y - c.y);
    B.x = (T)0.5 * (a.y + c.y);
    B.y = (T)0.5 * (c.x - a.x);
    if (r0 < nrows) W[(size_t)m * ldw + r0] = A;
    if (r0 + 1 < nrows) W[(size_t)m * ldw + r0 + 1] = B;
  }
}

// pass 2: per mode m (column of W): forward length-M transform of W[m][0..nin) (zero
// beyond), then either (build) store the whole spectrum to K[m][0..M), or multiply by
// khat[m][p] (kalnajs.hpp:53-56), inverse-transform and store W[m][0..nout).
template <typename T, int E>
__global__ void __launch_bounds__(1024) k_u_conv(typename cplx_of<T>::type *__restrict__ W, int ldw, int Nc, int nin,
                                                int nout, FftPlan pl,
                                                const typename cplx_of<T>::type *__restrict__ roots,
                                                const typename cplx_of<T>::type *__restrict__ khat,
                                                typename cplx_of<T>::type *__restrict__ kout, int nb) {
  using V = typename cplx_of<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *buf = reinterpret_cast<V *>(smem_raw);
  const int M = pl.n;
  const int m0 = blockIdx.x * nb;
  const int total = nb * M;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int t = idx / M, p = idx - t * M;
    const int m = m0 + t;
    V z;
    z.x = (T)0;
    z.y = (T)0;
    if (m < Nc && p < nin) z = W[(size_t)m * ldw + p];
    buf[idx] = z;
  }
  __syncthreads();
  smem_fft<V, E>(buf, nb, pl, -1, roots);
  if (kout) {
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int t = idx / M, p = idx - t * M;
      const int m = m0 + t;
      if (m < Nc) kout[(size_t)m * M + p] = buf[idx];
    }
    return;
  }
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int t = idx / M, p = idx - t * M;
    const int m = m0 + t;
    if (m < Nc) buf[idx] = cmul(buf[idx], khat[(size_t)m * M + p]);
  }
  __syncthreads();
  smem_fft<V, E>(buf, nb, pl, +1, roots);
  for (int idx = threadIdx.x; idx < nb * nout; idx += blockDim.x) {
    const int t = idx / nout, p = idx - t * nout;
    const int m = m0 + t;
    if (m < Nc) W[(size_t)m * ldw + p] = buf[t * M + p];
  }
}

// pass 3: transposed half spectrum -> rows.  Two Hermitian rows are packed into one
// complex inverse transform (FFTW c2r semantics: the imaginary parts of the m=0 and
// Nyquist bins are ignored), then out[i][j] = (pref * x) / sqrtR[i] (kalnajs.hpp:58-62).
template <typename T, int E>
__global__ void __launch_bounds__(1024) k_phi_inv(const typename cplx_of<T>::type *__restrict__ W, int ldw, int nrows,
                                                 int Nphi, FftPlan pl,
                                                 const typename cplx_of<T>::type *__restrict__ roots, T pref,
                                                 const T *__restrict__ sqrtR, T *__restrict__ out, int nb) {
  using V = typename cplx_of<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *buf = reinterpret_cast<V *>(smem_raw);
  const int row0 = blockIdx.x * 2 * nb;
  const int Nc = Nphi / 2 + 1;
  const bool even = (Nphi % 2) == 0;
  const int tot = nb * Nc;
  for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
    const int m = idx / nb, t = idx - m * nb;
    const int r0 = row0 + 2 * t;
    V A, B;
    A.x = A.y = B.x = B.y = (T)0;
    if (r0 < nrows) A = W[(size_t)m * ldw + r0];
    if (r0 + 1 < nrows) B = W[(size_t)m * ldw + r0 + 1];
    if (m == 0 || (even && m == Nphi / 2)) { A.y = (T)0; B.y = (T)0; }
    V *Z = buf + t * Nphi;
    V z;
    z.x = A.x - B.y;
    z.y = A.y + B.x;
    Z[m] = z;
    if (m > 0 && Nphi - m >= Nc) {
      V w;
      w.x = A.x + B.y;
      w.y = B.x - A.y;
      Z[Nphi - m] = w;
    }
  }
  __syncthreads();
  smem_fft<V, E>(buf, nb, pl, +1, roots);
  const int total = nb * Nphi;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int t = idx / Nphi, j = idx - t * Nphi;
    const int r0 = row0 + 2 * t, r1 = r0 + 1;
    const V z = buf[idx];
    if (r0 < nrows) out[(size_t)r0 * Nphi + j] = (pref * z.x) / sqrtR[r0];
    if (r1 < nrows) out[(size_t)r1 * Nphi + j] = (pref * z.y) / sqrtR[r1];
  }
}

}  // namespace dg
