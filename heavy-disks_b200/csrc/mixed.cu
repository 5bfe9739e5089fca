// Mixed-precision path: FP32 perturbation state about an FP64 axisymmetric basic state,
// gravity of the perturbation as a split-BF16 tensor-core DFT (four tcgen05 GEMMs).
//
// Gravity (kalnajs.hpp:48-63 restated as dense real DFT contractions; s = R^{3/2} sigma):
//   G1  X[c][i]  = sum_j Fphi[c][j] s[i][j]     phi DFT, c in [0, Nphi): Re m = 0, Re m = Nphi/2,
//                                               then (Re, Im) of m = 1..Nphi/2-1 interleaved
//                                               (the other imaginary parts vanish)
//   G2  W[c][p]  = KW[c][p] sum_i Cu[p][i] X[c][i]
//                                               u DFT on 2 Nu rows (cos p=0..Nu, sin p=1..Nu-1)
//                                               times (w_p / M) khat(p, m(c)) (khat is real and
//                                               even in p, so cos and sin rows decouple)
//   G3  Z[i][c]  = sum_p Cu[p][i] W[c][p]       inverse u DFT (only the Nu physical rows)
//   G4  dPhi[i][j] = (-G du dphi / sqrt(R_i)) sum_c Z[i][c] Gphi[j][c]   inverse phi DFT
// Each GEMM's epilogue writes the next GEMM's operand as a BF16 (hi, lo) pair in the
// K-major layout it needs; the hydro kernel writes s for G1 and reads dPhi.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include <cudaTypedefs.h>

#include "engine.h"
#include "hydro32.cuh"
#include "tc_gemm.cuh"
#include "step_ctl.cuh"
#include "hydro32w.cuh"
#include "hydro32t.cuh"
#include "hydro32p.cuh"
#include "uconv.cuh"
#include "phifwd.cuh"
#include "phiinv.cuh"

using namespace dg;

namespace {

struct SplitBuf {
  __nv_bfloat16 *hi = nullptr, *lo = nullptr;
};

}  // namespace

struct MixedState {
  int Nu = 0, Nphi = 0;
  // per-row / per-face tables
  float *rowbuf = nullptr;    // packed FP32 row and face arrays
  float *rowtab = nullptr;    // the same constants row-major for k_hydro32p (Rows32::rowtab)
  double *rowbufd = nullptr;  // packed FP64 row arrays
  Rows32 rows{};
  std::vector<double> S0, V0, g0;  // FP64 basic state (host)
  // state ping-pong
  float *sig[2] = {nullptr, nullptr}, *u[2] = {nullptr, nullptr}, *w[2] = {nullptr, nullptr};
  // gravity operands and outputs
  SplitBuf Sx, X1, Wt, Z, Fphi, Cu, CuT, Gphi;
  float *KW = nullptr, *dPhi = nullptr, *phiscale = nullptr;
  CUtensorMap mFphi[2], mSx[2], mX1[2], mCu[2], mCuT[2], mWt[2], mZ[2], mGphi[2];
  // factored u-direction (Nu a multiple of 1024): M = 2 Nu = 64 A, A = Nu / 32
  bool factored = false;
  int fa = 0, nm = 0;  // A and the padded complex-mode count
  SplitBuf Xin, Tb, Yk, Ub, RB, RA, RGA, RGB;
  float *KW2 = nullptr;
  float2 *tw = nullptr;
  // hydro kernel: the tiled form (hydro32t.cuh), its packed two-column form (hydro32p.cuh)
  // or the warp-marching form (hydro32w.cuh), chosen by DISKGPU_HYDRO32 = tile | packed |
  // warp; all compute the same step
  enum HydroKind : int { kHydroWarp = 0, kHydroTile = 1, kHydroPacked = 2 };
  int hydro_kind = kHydroTile;
  // pipeline stages of each gravity product (slots: 0 phi DFT, 1-4 the u passes, 5 inverse
  // phi DFT; 0 = chosen by K, kPersist / kPersistWide = the persistent kernel) and the tuner's record
  // (autotune below)
  int ns[6] = {0, 0, 0, 0, 0, 0};
  // FP32 field tiles of the packed hydro kernel: sigma, u, w of both ping-pong buffers, dPhi
  CUtensorMap mSig[2], mU[2], mW[2], mPhi;
  // row-tile counters between a step's hydro kernel and the next step's fused phi transform
  // (dg_common.cuh rowtile_*); zero between steps.  rs_arm: the gravity being enqueued is
  // part of a time step whose hydro counts them down (its inverse transform arms them);
  // rs_wait: its phi transform waits on them, which needs the hydro enqueued just before it
  // to have counted them down (prev_rs; otherwise it waits for its predecessor kernel).
  // DISKGPU_ROWSYNC=0 turns the hand-over off.
  int *rowpend = nullptr;
  bool rs_arm = false, rs_wait = false, prev_rs = false, rowsync = true;
  bool rowsync_ok() const {
    return rowsync && fused_phi && rowpend && (hydro_kind == kHydroTile || hydro_kind == kHydroPacked);
  }
  bool tuned = false;
  std::string tune_info;
  // A = 32 (Nu = 1024): the four u passes run as one fused kernel (uconv.cuh)
  bool fused_u = false;
  float *khm = nullptr;  // khat[m][p] / M, [nm][M]
  // Nu = Nphi = 1024: the forward and inverse phi transforms as fused kernels (phifwd.cuh,
  // phiinv.cuh); khm then carries the inverse real DFT's weights w_m / Nphi as well
  bool fused_phi = false;
  SplitBuf PA, PB;       // forward: stage-A (real 32-point) and stage-B (complex 32-point) operands
  SplitBuf IA, IB;       // inverse: stage-A (complex 32-point) and stage-B (real-output 32-point) operands
  SplitBuf Zt;           // the radial convolution's output rows, [Nu][kZtLd]
  float2 *twphi = nullptr;  // W^{m2 j1}, [32][32]
  CUtensorMap mPA[2], mPB[2], mIA[2], mIB[2];
  float2 *twp = nullptr; // W_M^{p2 i1} with padded rows, [64][kUcTwLd]
  CUtensorMap mXin[2], mTb[2], mYk[2], mUb[2], mRB[2], mRA[2], mRGA[2], mRGB[2], mZmn[2];
  bool tables_ready = false;
  // Nphi = 4096 on grids whose u convolution runs as four passes: both phi transforms in
  // two split-BF16 passes each (64 x 64, four-step) instead of the dense DFT products
  bool phi4096 = false;
  SplitBuf PhA1, PhB2f, PhB1i, PhB2i, PhT, PhX, PhV;
  float2 *twph = nullptr;  // W_4096^{m1 j2}, [64][64]
  CUtensorMap mSxBlk[2], mPhA1[2], mPhB2f[2], mPhB1i[2], mPhB2i[2], mPhT[2], mPhX[2], mPhV[2];
  // Failure-detection test: DISKGPU_TEST_ROWTILE_STALL=<row tile> at handle creation makes
  // the first self-gravity step enqueued outside a graph capture raise that tile row's
  // counter once more after its hydro has finished, so the next phi transform's bounded
  // wait on it runs out (~1 s) and the step reports DG_ERR_TIMEOUT.  Off (-1) otherwise.
  int test_stall = -1;
};

// One extra count on a row-tile counter (the failure-detection test above): no hydro CTA
// will count it down.  Launched in plain stream order, so the hydro before it has finished.
__global__ void k_rowtile_stall(int *cnt) { atomicAdd(cnt, 1); }

// ---------------------------------------------------------------------------------
// TMA descriptors

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// Dynamic shared memory of a step kernel, and the largest shared-memory carveout for all of
// them: the step's kernels alternate between 1 and 4 CTAs per SM with 46 to 214 KB each, and
// one common L1 / shared split spares the SMs a reconfiguration at every kernel boundary.
static cudaError_t smem_attrs(const void *fn, size_t bytes) {
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
}

// every instantiation of the tiled hydro kernels takes more than 48 KB of shared memory
static cudaError_t hydro32t_prepare() {
  const void *fns[] = {(const void *)k_hydro32t<true, kForcePhi>, (const void *)k_hydro32t<false, kForcePhi>,
                       (const void *)k_hydro32t<true, kForceArrays>, (const void *)k_hydro32t<false, kForceArrays>,
                       (const void *)k_hydro32t<true, kForceNone>, (const void *)k_hydro32t<false, kForceNone>,
                       (const void *)k_hydro32p<true, kForcePhi>, (const void *)k_hydro32p<false, kForcePhi>,
                       (const void *)k_hydro32p<true, kForceArrays>, (const void *)k_hydro32p<false, kForceArrays>,
                       (const void *)k_hydro32p<true, kForceNone>, (const void *)k_hydro32p<false, kForceNone>};
  for (int q = 0; q < 12; ++q) {
    cudaError_t e = smem_attrs(fns[q], q < 6 ? kSmem32t : kSmem32p);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// radial-direction layout of the split-BF16 gravity: factored (M = 2 Nu = 64 x Nu/32) when
// Nu is a multiple of 1024, and the four factored passes fused into one kernel at Nu = 1024
static bool u_factored(int Nu) { return Nu % 1024 == 0; }
static bool u_fused(int Nu) { return Nu == 1024; }
// the forward phi transform as a fused two-stage kernel (phifwd.cuh) when both are 1024
static bool phi_fused(int Nu, int Nphi) { return Nu == 1024 && Nphi == 1024; }

// Row-major FP32 field [rows][cols] -> boxes of 68 columns x 22 rows, no swizzle (the
// packed hydro kernel's input tile; rows outside the field read as zero).
static bool make_map_f32(CUtensorMap *m, const void *base, uint64_t rows, uint64_t cols) {
  auto fn = encode_fn();
  if (!fn) return false;
  if (((uintptr_t)base & 15) || (cols * 4) % 16) return false;
  cuuint64_t gdim[2] = {cols, rows};
  cuuint64_t gstride[1] = {cols * 4};
  cuuint32_t box[2] = {(cuuint32_t)kLdP, (cuuint32_t)kRows32t};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), gdim, gstride, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// K-major BF16 matrix [rows][cols] -> tiles of box_rows x 64 with 128-byte swizzle.
static bool make_map(CUtensorMap *m, const void *base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  if (((uintptr_t)base & 15) || (cols * 2) % 16) return false;
  cuuint64_t gdim[2] = {cols, rows};
  cuuint64_t gstride[1] = {cols * 2};
  cuuint32_t box[2] = {64, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), gdim, gstride, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// the same map for other files of the library (the surrogate network's operands)
bool dg_bf16_tensor_map(CUtensorMap *m, const void *base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
  return make_map(m, base, rows, cols, box_rows);
}

// ---------------------------------------------------------------------------------
// DFT tables (built on the device in FP64, stored as BF16 pairs)

__device__ __forceinline__ void put_split(SplitBuf b, size_t k, double x) {
  float f = (float)x;
  __nv_bfloat16 h = __float2bfloat16_rn(f);
  b.hi[k] = h;
  b.lo[k] = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
}

// phi index c -> (m, is_imag), interleaved: c = 0 -> Re m = 0, c = 1 -> Re m = Nphi/2,
// c = 2m + ri for 1 <= m < Nphi/2 (Nphi even; the imaginary parts of m = 0 and Nphi/2 vanish)
__device__ __forceinline__ void phi_mode(int c, int Nphi, int &m, bool &im) {
  if (c == 0) { m = 0; im = false; }
  else if (c == 1) { m = Nphi / 2; im = false; }
  else { m = c >> 1; im = (c & 1) != 0; }
}

__global__ void k_tab_phi(SplitBuf F, SplitBuf Gt, int N) {
  const size_t n = (size_t)N * N;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int a = (int)(k / N), b = (int)(k % N);
    // F[c = a][j = b]
    {
      int m; bool im;
      phi_mode(a, N, m, im);
      long long r = ((long long)m * b) % N;
      double sn, cs;
      sincospi(2.0 * (double)r / N, &sn, &cs);
      put_split(F, k, im ? -sn : cs);
    }
    // Gt[j = a][c = b]: inverse real DFT weights (1/N, doubled off the self-conjugate bins)
    {
      int m; bool im;
      phi_mode(b, N, m, im);
      long long r = ((long long)m * a) % N;
      double sn, cs;
      sincospi(2.0 * (double)r / N, &sn, &cs);
      double wgt = (m == 0 || (N % 2 == 0 && m == N / 2)) ? 1.0 : 2.0;
      put_split(Gt, k, (im ? -sn : cs) * wgt / N);
    }
  }
}

// Cu[p][i] (2Nu x Nu): p <= Nu cos(2 pi p i / M), p > Nu sin(2 pi (p - Nu) i / M); CuT = Cu^T
__global__ void k_tab_u(SplitBuf Cu, SplitBuf CuT, int Nu) {
  const int M = 2 * Nu;
  const size_t n = (size_t)M * Nu;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int p = (int)(k / Nu), i = (int)(k % Nu);
    bool sn_row = p > Nu;
    int pp = sn_row ? p - Nu : p;
    long long r = ((long long)pp * i) % M;
    double sn, cs;
    sincospi(2.0 * (double)r / M, &sn, &cs);
    double v = sn_row ? sn : cs;
    put_split(Cu, k, v);
    put_split(CuT, (size_t)i * M + p, v);
  }
}

// KW[c][p] = (w_p / M) Re khat(p, m(c)); khat is the FP64 r2c table [m][0..M)
__global__ void k_tab_kw(float *KW, const double2 *khat, int Nu, int Nphi) {
  const int M = 2 * Nu;
  const size_t n = (size_t)Nphi * M;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int c = (int)(k / M), p = (int)(k % M);
    int m; bool im;
    phi_mode(c, Nphi, m, im);
    int pp = p > Nu ? p - Nu : p;
    double wgt = (p == 0 || p == Nu) ? 1.0 : 2.0;
    KW[k] = (float)(wgt / M * khat[(size_t)m * M + pp].x);
  }
}

// Tables of the four-step phi transforms at Nphi = 4096 (m = m1 + 64 m2, j = 64 j1 + j2):
// PhA1[(m1, ri)][j1] = cos / -sin (2 pi m1 j1 / 64), the real-input 64-point DFT over j1;
// PhB2i[j1][(m1, ri)] = cos / -sin (2 pi j1 m1 / 64) / N, the real part of the inverse
// 64-point DFT over m1 with the inverse transform's 1 / N;
// PhB2f[(m2, ro)][(ri, j2)]: the complex 64-point DFT W_64^{m2 j2} in real block form with
// its K index planar (the real parts of the 64 inputs, then the imaginary parts).
__global__ void k_tab_ph4096(SplitBuf A1, SplitBuf B2i, SplitBuf B2f, int N) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 128 * 128; q += gridDim.x * blockDim.x) {
    const int row = q / 128, col = q % 128, m2 = row >> 1, ro = row & 1, ri = col >> 6, j2 = col & 63;
    double sn, cs;
    sincospi(2.0 * (double)((m2 * j2) % 64) / 64.0, &sn, &cs);
    const double Fr = cs, Fi = -sn;  // W_64^{m2 j2} = exp(-2 pi i m2 j2 / 64)
    put_split(B2f, q, ro == 0 ? (ri == 0 ? Fr : -Fi) : (ri == 0 ? Fi : Fr));
    if (q >= 128 * 64) continue;
    {
      const int row = q / 64, j1 = q % 64, m1 = row >> 1, ri = row & 1;
      double sn, cs;
      sincospi(2.0 * (double)((m1 * j1) % 64) / 64.0, &sn, &cs);
      put_split(A1, q, ri ? -sn : cs);
    }
    {
      const int j1 = q / 128, col = q % 128, m1 = col >> 1, ri = col & 1;
      double sn, cs;
      sincospi(2.0 * (double)((j1 * m1) % 64) / 64.0, &sn, &cs);
      put_split(B2i, q, (ri ? -sn : cs) / N);
    }
  }
}

// Real block form [[Fr, -Fi], [Fi, Fr]] of a complex matrix F[r][k] = exp(sgn 2 pi i r k / L):
// rows (r, ri) for r < nr, cols (k, ri') for k < nk.
__global__ void k_tab_cblock(SplitBuf T, int nr, int nk, int L, int sgn) {
  const size_t n = (size_t)4 * nr * nk;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(q / (2 * nk)), col = (int)(q % (2 * nk));
    const int r = row >> 1, ri = row & 1, k = col >> 1, rk = col & 1;
    double sn, cs;
    sincospi(2.0 * (double)(((long long)r * k) % L) / L, &sn, &cs);
    const double Fr = cs, Fi = sgn * sn;
    const double v = (ri == 0) ? (rk == 0 ? Fr : -Fi) : (rk == 0 ? Fi : Fr);
    put_split(T, q, v);
  }
}

// KW2[(m, p2)][(p1, ri)] = Re khat(p2 + 64 p1, m) / M for m <= Nphi/2 (padding modes: 0)
__global__ void k_tab_kw2(float *KW2, const double2 *khat, int nm, int A, int Nphi) {
  const int M = 64 * A;
  const size_t n = (size_t)nm * 64 * 2 * A;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(q / (2 * A)), col = (int)(q % (2 * A));
    const int m = row >> 6, p2 = row & 63, p1 = col >> 1;
    KW2[q] = (m <= Nphi / 2) ? (float)(khat[(size_t)m * M + p2 + 64 * p1].x / M) : 0.f;
  }
}

// twiddles of k_phifwd: W_N^{m2 j1} = e^{-2 pi i m2 j1 / N}, [32][32]
__global__ void k_tab_twphi(float2 *tw, int N) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 32 * 32; q += gridDim.x * blockDim.x) {
    const int m2 = q / 32, j1 = q % 32;
    double sn, cs;
    sincospi(2.0 * (double)(m2 * j1) / N, &sn, &cs);
    tw[q] = make_float2((float)cs, (float)-sn);
  }
}

// stage-A operand of k_phifwd: C[(m2, ro)][j2] = cos / -sin (2 pi m2 j2 / 32), 64 x 64 with
// columns 32.. zero
__global__ void k_tab_phiA(SplitBuf C) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 64 * 64; q += gridDim.x * blockDim.x) {
    const int r = q / 64, k = q % 64;
    double v = 0.0;
    if (k < 32) {
      double sn, cs;
      sincospi(2.0 * (double)(((r >> 1) * k) % 32) / 32.0, &sn, &cs);
      v = (r & 1) ? -sn : cs;
    }
    put_split(C, q, v);
  }
}

// KHM[m][p] = Re khat(p, m) / M for m <= Nphi/2 (padding modes: 0); with real_dft_weights
// also times w_m / Nphi (w = 1 at m = 0 and Nphi/2, else 2), the inverse real DFT's weights
__global__ void k_tab_khm(float *KHM, const double2 *khat, int nm, int M, int Nphi, bool real_dft_weights) {
  const size_t n = (size_t)nm * M;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(q / M);
    const double w = !real_dft_weights ? 1.0 : ((m == 0 || 2 * m == Nphi) ? 1.0 : 2.0) / Nphi;
    KHM[q] = (m <= Nphi / 2) ? (float)(khat[q].x / M * w) : 0.f;
  }
}

// stage-B operand of k_phiinv: B[j2][(m2, ri)] = cos / -sin (2 pi j2 m2 / 32), 32 x 64
// (the real part of e^{+2 pi i j2 m2 / 32} (Y_re + i Y_im))
__global__ void k_tab_phiIB(SplitBuf B) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 32 * 64; q += gridDim.x * blockDim.x) {
    const int j2 = q / 64, m2 = (q % 64) >> 1, ri = q & 1;
    double sn, cs;
    sincospi(2.0 * (double)((j2 * m2) % 32) / 32.0, &sn, &cs);
    put_split(B, q, ri ? -sn : cs);
  }
}

// twiddles W_M^{p2 i1}, [64][ld] (ld >= A; columns A.. are zero)
__global__ void k_tab_tw(float2 *tw, int A, int ld) {
  const int M = 64 * A;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 64 * ld; q += gridDim.x * blockDim.x) {
    const int p2 = q / ld, i1 = q % ld;
    double sn = 0.0, cs = 0.0;
    if (i1 < A) sincospi(2.0 * (double)(((long long)p2 * i1) % M) / M, &sn, &cs);
    tw[q] = make_float2((float)cs, (float)-sn);
  }
}

// ---------------------------------------------------------------------------------
// state conversion (FP64 full fields <-> basic state + FP32 perturbation)

__global__ void k_to_pert(const double *S, const double *vR, const double *vp, float *sig, float *u, float *w,
                          SplitBuf Sx, Rows32 g) {
  const size_t n = (size_t)g.Nu * g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / g.Nphi);
    float s = (float)(S[k] - g.S0d[i]);
    sig[k] = s;
    u[k] = (float)vR[k];
    w[k] = (float)(vp[k] - g.V0d[i]);
    float x = g.R32[i] * s;
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    Sx.hi[k] = h;
    Sx.lo[k] = __float2bfloat16_rn(x - __bfloat162float(h));
  }
}

__global__ void k_from_pert(const float *sig, const float *u, const float *w, double *S, double *vR, double *vp,
                            Rows32 g) {
  const size_t n = (size_t)g.Nu * g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / g.Nphi);
    S[k] = g.S0d[i] + (double)sig[k];
    vR[k] = (double)u[k];
    vp[k] = g.V0d[i] + (double)w[k];
  }
}

// s = R^{3/2} Sigma of a full FP64 field (dg_potential in mixed precision)
__global__ void k_full_to_sx(const double *S, SplitBuf Sx, const double *R32d, int Nu, int Nphi) {
  const size_t n = (size_t)Nu * Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / Nphi);
    float x = (float)(R32d[i] * S[k]);
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    Sx.hi[k] = h;
    Sx.lo[k] = __float2bfloat16_rn(x - __bfloat162float(h));
  }
}

// s = R^{3/2} sigma of the current perturbation (the G1 operand)
__global__ void k_sig_to_sx(const float *sig, SplitBuf Sx, Rows32 g) {
  const size_t n = (size_t)g.Nu * g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / g.Nphi);
    float x = g.R32[i] * sig[k];
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    Sx.hi[k] = h;
    Sx.lo[k] = __float2bfloat16_rn(x - __bfloat162float(h));
  }
}

__global__ void k_f32_to_f64(const float *a, double *b, size_t n) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    b[k] = (double)a[k];
}

// CFL (and optional mode sums) over the perturbation state
__global__ void __launch_bounds__(256) k_cfl32(const float *sig, const float *uu, const float *ww, Ctl *ctl, Rows32 g,
                                               int nmodes, int record) {
  __shared__ double red[8];
  double msum[2 * kMaxModes];
#pragma unroll
  for (int q = 0; q < 2 * kMaxModes; ++q) msum[q] = 0.0;
  if (record && nmodes < 3) nmodes = 3;
  double lmax = 0.0;
  bool bad = false;
  const size_t n = (size_t)g.Nu * g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / g.Nphi), j = (int)(k % g.Nphi);
    float r = cfl_rate32(g, i, sig[k], uu[k], ww[k]);
    bad |= !(r == r);
    lmax = fmax(lmax, (double)r);
    if (nmodes) {
      const double sfull = g.S0d[i] + (double)sig[k];
      const double phi = (j + 0.5) * (double)g.dphi;
      for (int m = 0; m < nmodes; ++m) {
        double sn, cs;
        sincos(m * phi, &sn, &cs);
        msum[2 * m] += sfull * cs * g.dAd[i];
        msum[2 * m + 1] -= sfull * sn * g.dAd[i];
      }
    }
  }
  if (bad) lmax = __longlong_as_double(0x7ff8000000000000ll);
  StepInfo si;
  si.t = ctl->t; si.dt = 0.0; si.tlim = ctl->tlim;
  si.active = false; si.advance_t = false; si.record = record != 0; si.nmodes = nmodes;
  finish_launch<256>(ctl, si, lmax, msum, red);
}

__global__ void __launch_bounds__(256) k_modes32(const float *sig, Rows32 g, int nmodes, double *out) {
  __shared__ double red[8];
  double msum[2 * kMaxModes];
#pragma unroll
  for (int q = 0; q < 2 * kMaxModes; ++q) msum[q] = 0.0;
  const size_t n = (size_t)g.Nu * g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / g.Nphi), j = (int)(k % g.Nphi);
    const double sfull = g.S0d[i] + (double)sig[k];
    const double phi = (j + 0.5) * (double)g.dphi;
    for (int m = 0; m < nmodes; ++m) {
      double sn, cs;
      sincos(m * phi, &sn, &cs);
      msum[2 * m] += sfull * cs * g.dAd[i];
      msum[2 * m + 1] -= sfull * sn * g.dAd[i];
    }
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

__global__ void __launch_bounds__(256) k_conserved32(const float *sig, const float *ww, Rows32 g, double *out) {
  __shared__ double red[2][8];
  double m = 0.0, L = 0.0;
  const size_t n = (size_t)g.Nu * g.Nphi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k / g.Nphi);
    const double s = g.S0d[i] + (double)sig[k];
    const double vp = g.V0d[i] + (double)ww[k];
    m += s * g.dAd[i];
    L += s * vp * g.Rd[i] * g.dAd[i];
  }
  m = warp_sum(m);
  L = warp_sum(L);
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = m; red[1][threadIdx.x >> 5] = L; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < 8; ++w) { a += red[0][w]; b += red[1][w]; }
    atomicAdd(&out[0], a);
    atomicAdd(&out[1], b);
  }
}

// ---------------------------------------------------------------------------------
// host side

#define XK(call)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) return fail(DG_ERR_CUDA, #call, cudaGetErrorString(e_)); \
  } while (0)

static int grid_for(size_t n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  size_t b = (n + 255) / 256;
  size_t cap = (size_t)sms * 8;
  return (int)(b < cap ? b : cap);
}

template <typename T>
static cudaError_t dalloc(T **p, size_t n) {
  return cudaMalloc((void **)p, (n ? n : 1) * sizeof(T));
}

static cudaError_t alloc_split(SplitBuf &b, size_t n) {
  cudaError_t e = dalloc(&b.hi, n);
  if (e != cudaSuccess) return e;
  return dalloc(&b.lo, n);
}

static void free_split(SplitBuf &b) {
  if (b.hi) cudaFree(b.hi);
  if (b.lo) cudaFree(b.lo);
  b.hi = b.lo = nullptr;
}

// Launch with programmatic stream serialization: the kernel may begin (its prologue up to
// pdl_wait) while the previous kernel on the stream drains.
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// a product slot's "stages" values that select the persistent GEMM (tc_gemm.cuh), with
// 128 x 128 or (where N is a multiple of 256) 128 x 256 tiles
constexpr int kPersist = 8, kPersistWide = 16;

// SMs of the current device (the persistent products' grid)
static int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      n <= 0)
    n = 148;
  return n;
}

// gemm(): one split-BF16 product.  ns = pipeline stages of the tile kernel (1, 2 or 4; 0
// picks by K), or kPersist for the persistent kernel.
template <int MODE, bool A_MN = false, bool B_MN = false>
static cudaError_t gemm(const CUtensorMap &Ah, const CUtensorMap &Al, const CUtensorMap &Bh, const CUtensorMap &Bl,
                        int M, int N, int K, const tc::GemmArgs &base, cudaStream_t st, int ns = 0) {
  tc::GemmArgs a = base;
  a.M = M; a.N = N; a.K = K;
  if (M % tc::BM || N % tc::BN || K % tc::BK) return cudaErrorInvalidValue;
  if (ns == kPersistWide) {
    if (N % 256 == 0) {
      tc::GemmDisk b;
      b.hi = Bh; b.lo = Bl; b.args = a;
      const int tn = N / 256, tm = M / tc::BM, nt = tn * tm, nsm = sm_count();
      return launch_pdl(tc::k_gemm_persist<MODE, A_MN, B_MN, 256>, dim3(nt < nsm ? nt : nsm),
                        dim3(tc::threads_persist(tc::kEpiWarpsLone)), tc::smem_persist(256), st, Ah, Al, b, tn, tm, nt);
    }
    ns = kPersist;  // N not a multiple of 256: 128 x 128 tiles
  }
  if (ns == kPersist) {
    // the persistent warp-specialised kernel: one CTA per SM walks 128 x 128 tiles, the
    // epilogue of one tile overlapping the loads and MMAs of the next
    if (N % tc::BN2 == 0) {
      tc::GemmDisk b;
      b.hi = Bh; b.lo = Bl; b.args = a;
      const int tn = N / tc::BN2, tm = M / tc::BM, nt = tn * tm, nsm = sm_count();
      return launch_pdl(tc::k_gemm_persist<MODE, A_MN, B_MN>, dim3(nt < nsm ? nt : nsm),
                        dim3(tc::threads_persist(tc::kEpiWarpsLone)),
                        tc::kSmemP, st, Ah, Al, b, tn, tm, nt);
    }
    ns = 0;  // N not a multiple of 128: the tile kernel, stages by K
  }
  dim3 grid(N / tc::BN, M / tc::BM);
  // short contractions (one or two K chunks) need no deep pipeline: fewer stages let more
  // CTAs share an SM and hide each tile's load / epilogue latency
  const int nk = K / tc::BK;
  if (ns == 0) ns = nk <= 1 ? 1 : (nk <= 2 ? 2 : tc::STAGES);
  if (ns <= 1)
    return launch_pdl(tc::k_gemm_split<MODE, A_MN, B_MN, 1>, grid, dim3(tc::kThreads), tc::smem_bytes(1), st, Ah, Al,
                      Bh, Bl, a);
  if (ns <= 2)
    return launch_pdl(tc::k_gemm_split<MODE, A_MN, B_MN, 2>, grid, dim3(tc::kThreads), tc::smem_bytes(2), st, Ah, Al,
                      Bh, Bl, a);
  return launch_pdl(tc::k_gemm_split<MODE, A_MN, B_MN, tc::STAGES>, grid, dim3(tc::kThreads),
                    tc::smem_bytes(tc::STAGES), st, Ah, Al, Bh, Bl, a);
}

// The smem limit of every instantiation gemm() may launch, raised once at set-up.
template <int MODE, bool A_MN, bool B_MN>
static cudaError_t prepare_gemm() {
  cudaError_t e;
  e = smem_attrs((const void *)tc::k_gemm_persist<MODE, A_MN, B_MN>, tc::kSmemP);
  if (e != cudaSuccess) return e;
  e = smem_attrs((const void *)tc::k_gemm_persist<MODE, A_MN, B_MN, 256>, tc::smem_persist(256));
  if (e != cudaSuccess) return e;
  e = smem_attrs((const void *)tc::k_gemm_split<MODE, A_MN, B_MN, 1>, tc::smem_bytes(1));
  if (e != cudaSuccess) return e;
  e = smem_attrs((const void *)tc::k_gemm_split<MODE, A_MN, B_MN, 2>, tc::smem_bytes(2));
  if (e != cudaSuccess) return e;
  return smem_attrs((const void *)tc::k_gemm_split<MODE, A_MN, B_MN, tc::STAGES>, tc::smem_bytes(tc::STAGES));
}

int dg_handle::mixed_init() {
  const int Nu = p.Nu, Nphi = p.Nphi;
  if (Nu % tc::BM || Nphi % tc::BM) {
    char b[160];
    snprintf(b, sizeof b, "Nu=%d Nphi=%d: the tensor-core gravity needs multiples of %d", Nu, Nphi, tc::BM);
    return fail(DG_ERR_UNSUPPORTED, "mixed precision", b);
  }
  if (!encode_fn()) return fail(DG_ERR_UNSUPPORTED, "mixed precision", "cuTensorMapEncodeTiled unavailable");
  mx = new MixedState();
  MixedState &X = *mx;
  X.Nu = Nu;
  X.Nphi = Nphi;
  const size_t n = (size_t)Nu * Nphi;
  for (int b = 0; b < 2; ++b) {
    XK(dalloc(&X.sig[b], n)); XK(dalloc(&X.u[b], n)); XK(dalloc(&X.w[b], n));
  }
  XK(alloc_split(X.Sx, n)); XK(alloc_split(X.X1, n)); XK(alloc_split(X.Z, n));
  XK(alloc_split(X.Wt, (size_t)Nphi * 2 * Nu));
  XK(alloc_split(X.Fphi, (size_t)Nphi * Nphi)); XK(alloc_split(X.Gphi, (size_t)Nphi * Nphi));
  XK(alloc_split(X.Cu, (size_t)2 * Nu * Nu)); XK(alloc_split(X.CuT, (size_t)2 * Nu * Nu));
  XK(dalloc(&X.KW, (size_t)Nphi * 2 * Nu));
  XK(dalloc(&X.dPhi, n));
  static_assert(kTileI == tc::kPfHydroRows && kTileI % tc::kPfRows == 0, "row tiles of the hand-over");
  XK(dalloc(&X.rowpend, (size_t)(Nu + kTileI - 1) / kTileI));
  {
    const char *rs = getenv("DISKGPU_ROWSYNC");
    X.rowsync = !(rs && strcmp(rs, "0") == 0);
  }
  XK(cudaMemsetAsync(X.rowpend, 0, (size_t)(Nu + kTileI - 1) / kTileI * sizeof(int), st));
  XK(dalloc(&X.phiscale, Nu));
  XK(dalloc(&X.rowbuf, (size_t)24 * (Nu + 1)));
  XK(dalloc(&X.rowtab, (size_t)(Nu + kRowTabExtra) * kRowTabW));
  XK(dalloc(&X.rowbufd, (size_t)4 * Nu));
  // DFT tables
  k_tab_phi<<<grid_for((size_t)Nphi * Nphi), 256, 0, st>>>(X.Fphi, X.Gphi, Nphi);
  XK(cudaGetLastError());
  k_tab_u<<<grid_for((size_t)2 * Nu * Nu), 256, 0, st>>>(X.Cu, X.CuT, Nu);
  XK(cudaGetLastError());
  k_tab_kw<<<grid_for((size_t)Nphi * 2 * Nu), 256, 0, st>>>(X.KW, Khat, Nu, Nphi);
  XK(cudaGetLastError());
  std::vector<float> ps(Nu);
  for (int i = 0; i < Nu; ++i) ps[i] = (float)(-p.G * du * dphi / sqrtR[i]);
  XK(cudaMemcpy(X.phiscale, ps.data(), Nu * sizeof(float), cudaMemcpyHostToDevice));
  // tensor maps: A operands are read in 128-row boxes, B operands in 64-row boxes
  bool okm = make_map(&X.mFphi[0], X.Fphi.hi, Nphi, Nphi, tc::BM) && make_map(&X.mFphi[1], X.Fphi.lo, Nphi, Nphi, tc::BM) &&
             make_map(&X.mSx[0], X.Sx.hi, Nu, Nphi, tc::BN) && make_map(&X.mSx[1], X.Sx.lo, Nu, Nphi, tc::BN) &&
             make_map(&X.mX1[0], X.X1.hi, Nphi, Nu, tc::BM) && make_map(&X.mX1[1], X.X1.lo, Nphi, Nu, tc::BM) &&
             make_map(&X.mCu[0], X.Cu.hi, 2 * Nu, Nu, tc::BN) && make_map(&X.mCu[1], X.Cu.lo, 2 * Nu, Nu, tc::BN) &&
             make_map(&X.mCuT[0], X.CuT.hi, Nu, 2 * Nu, tc::BM) && make_map(&X.mCuT[1], X.CuT.lo, Nu, 2 * Nu, tc::BM) &&
             make_map(&X.mWt[0], X.Wt.hi, Nphi, 2 * Nu, tc::BN) && make_map(&X.mWt[1], X.Wt.lo, Nphi, 2 * Nu, tc::BN) &&
             make_map(&X.mZ[0], X.Z.hi, Nu, Nphi, tc::BM) && make_map(&X.mZ[1], X.Z.lo, Nu, Nphi, tc::BM) &&
             make_map(&X.mGphi[0], X.Gphi.hi, Nphi, Nphi, tc::BN) && make_map(&X.mGphi[1], X.Gphi.lo, Nphi, Nphi, tc::BN);
  if (!okm) return fail(DG_ERR_CUDA, "mixed precision", "tensor map encoding failed");
  // factored u-direction when Nu is a multiple of 1024 (F1: 64-point stage on 128 rows)
  X.factored = u_factored(Nu);
  if (X.factored) {
    const int A = Nu / 32, nm = ((Nphi / 2 + 1) + 3) / 4 * 4;
    X.fa = A;
    X.nm = nm;
    XK(alloc_split(X.Xin, (size_t)64 * nm * A));
    XK(cudaMemset(X.Xin.hi, 0, sizeof(__nv_bfloat16) * 64 * nm * A));
    XK(cudaMemset(X.Xin.lo, 0, sizeof(__nv_bfloat16) * 64 * nm * A));
    XK(alloc_split(X.Tb, (size_t)2 * A * nm * 64));
    XK(alloc_split(X.Yk, (size_t)nm * 64 * 2 * A));
    XK(alloc_split(X.Ub, (size_t)nm * A * 128));
    XK(alloc_split(X.RB, (size_t)128 * 64));
    XK(alloc_split(X.RA, (size_t)2 * A * 2 * A));
    XK(alloc_split(X.RGA, (size_t)2 * A * 2 * A));
    XK(alloc_split(X.RGB, (size_t)64 * 128));
    XK(dalloc(&X.KW2, (size_t)nm * 64 * 2 * A));
    XK(dalloc(&X.tw, (size_t)64 * A));
    k_tab_cblock<<<64, 256, 0, st>>>(X.RB, 64, 32, 64, -1);    // W_64^{p2 i2}, i2 < 32
    k_tab_cblock<<<64, 256, 0, st>>>(X.RA, A, A, A, -1);       // W_A^{p1 i1}
    k_tab_cblock<<<64, 256, 0, st>>>(X.RGA, A, A, A, +1);      // W_A^{-i1 p1}
    k_tab_cblock<<<64, 256, 0, st>>>(X.RGB, 32, 64, 64, +1);   // W_64^{-i2 p2}
    k_tab_kw2<<<grid_for((size_t)nm * 128 * A), 256, 0, st>>>(X.KW2, Khat, nm, A, Nphi);
    k_tab_tw<<<64, 256, 0, st>>>(X.tw, A, A);
    XK(cudaGetLastError());
    X.fused_u = u_fused(Nu);
    X.fused_phi = X.fused_u && phi_fused(Nu, Nphi);
    if (X.fused_u) {
      XK(dalloc(&X.khm, (size_t)nm * 64 * A));
      XK(dalloc(&X.twp, (size_t)64 * tc::kUcTwLd));
      k_tab_tw<<<64, 256, 0, st>>>(X.twp, A, tc::kUcTwLd);
      k_tab_khm<<<grid_for((size_t)nm * 64 * A), 256, 0, st>>>(X.khm, Khat, nm, 64 * A, Nphi, X.fused_phi);
      XK(cudaGetLastError());
      XK(smem_attrs((const void *)tc::k_uconv, tc::kUcSmem));
    }
    if (X.fused_phi) {
      static_assert(tc::kZtModes >= 1024 / 2 + 1 && tc::kZtModes % 32 == 0, "Zt row layout");
      XK(alloc_split(X.Zt, (size_t)Nu * tc::kZtLd));
      XK(cudaMemset(X.Zt.hi, 0, sizeof(__nv_bfloat16) * (size_t)Nu * tc::kZtLd));  // modes above Nphi/2 stay 0
      XK(cudaMemset(X.Zt.lo, 0, sizeof(__nv_bfloat16) * (size_t)Nu * tc::kZtLd));
      XK(alloc_split(X.IA, (size_t)64 * 64));
      XK(alloc_split(X.IB, (size_t)32 * 64));
      k_tab_cblock<<<32, 256, 0, st>>>(X.IA, 32, 32, 32, +1);  // W_32^{-j1 m1}
      k_tab_phiIB<<<8, 256, 0, st>>>(X.IB);                     // Re W_32^{-j2 m2}
      XK(cudaGetLastError());
      bool oki = make_map(&X.mIA[0], X.IA.hi, 64, 64, tc::BN) && make_map(&X.mIA[1], X.IA.lo, 64, 64, tc::BN) &&
                 make_map(&X.mIB[0], X.IB.hi, 32, 64, 32) && make_map(&X.mIB[1], X.IB.lo, 32, 64, 32);
      if (!oki) return fail(DG_ERR_CUDA, "mixed precision", "tensor map encoding failed (fused inverse phi transform)");
      XK(smem_attrs((const void *)tc::k_phiinv, tc::kPiSmem));
      XK(alloc_split(X.PA, (size_t)64 * 64));
      XK(alloc_split(X.PB, (size_t)64 * 64));
      XK(dalloc(&X.twphi, (size_t)32 * 32));
      k_tab_phiA<<<32, 256, 0, st>>>(X.PA);
      k_tab_cblock<<<32, 256, 0, st>>>(X.PB, 32, 32, 32, -1);  // W_32^{m1 j1}
      k_tab_twphi<<<8, 128, 0, st>>>(X.twphi, Nphi);            // W_Nphi^{m2 j1}
      XK(cudaGetLastError());
      bool okp = make_map(&X.mPA[0], X.PA.hi, 64, 64, tc::BN) && make_map(&X.mPA[1], X.PA.lo, 64, 64, tc::BN) &&
                 make_map(&X.mPB[0], X.PB.hi, 64, 64, tc::BN) && make_map(&X.mPB[1], X.PB.lo, 64, 64, tc::BN);
      if (!okp) return fail(DG_ERR_CUDA, "mixed precision", "tensor map encoding failed (fused phi transform)");
      XK(smem_attrs((const void *)tc::k_phifwd, tc::kPfSmem));
    }
    bool okf = make_map(&X.mXin[0], X.Xin.hi, 64, (uint64_t)nm * A, 64) && make_map(&X.mXin[1], X.Xin.lo, 64, (uint64_t)nm * A, 64) &&
               make_map(&X.mTb[0], X.Tb.hi, 2 * A, (uint64_t)nm * 64, 64) && make_map(&X.mTb[1], X.Tb.lo, 2 * A, (uint64_t)nm * 64, 64) &&
               make_map(&X.mYk[0], X.Yk.hi, (uint64_t)nm * 64, 2 * A, tc::BM) && make_map(&X.mYk[1], X.Yk.lo, (uint64_t)nm * 64, 2 * A, tc::BM) &&
               make_map(&X.mUb[0], X.Ub.hi, (uint64_t)nm * A, 128, tc::BM) && make_map(&X.mUb[1], X.Ub.lo, (uint64_t)nm * A, 128, tc::BM) &&
               make_map(&X.mRB[0], X.RB.hi, 128, 64, tc::BM) && make_map(&X.mRB[1], X.RB.lo, 128, 64, tc::BM) &&
               make_map(&X.mRA[0], X.RA.hi, 2 * A, 2 * A, tc::BN) && make_map(&X.mRA[1], X.RA.lo, 2 * A, 2 * A, tc::BN) &&
               make_map(&X.mRGA[0], X.RGA.hi, 2 * A, 2 * A, tc::BN) && make_map(&X.mRGA[1], X.RGA.lo, 2 * A, 2 * A, tc::BN) &&
               make_map(&X.mRGB[0], X.RGB.hi, 64, 128, tc::BN) && make_map(&X.mRGB[1], X.RGB.lo, 64, 128, tc::BN) &&
               make_map(&X.mZmn[0], X.Z.hi, Nphi, Nu, 64) && make_map(&X.mZmn[1], X.Z.lo, Nphi, Nu, 64);
    if (!okf) return fail(DG_ERR_CUDA, "mixed precision", "tensor map encoding failed (factored path)");
    X.phi4096 = !X.fused_u && Nphi == 4096;
    if (X.phi4096) {
      const size_t big = (size_t)64 * Nu * 128;  // T, X, V: [64 Nu][128]
      XK(alloc_split(X.PhA1, (size_t)128 * 64)); XK(alloc_split(X.PhB2i, (size_t)64 * 128));
      XK(alloc_split(X.PhB2f, (size_t)128 * 128)); XK(alloc_split(X.PhB1i, (size_t)128 * 128));
      XK(alloc_split(X.PhT, big)); XK(alloc_split(X.PhX, big)); XK(alloc_split(X.PhV, big));
      XK(dalloc(&X.twph, (size_t)64 * 64));
      k_tab_ph4096<<<64, 256, 0, st>>>(X.PhA1, X.PhB2i, X.PhB2f, Nphi);
      k_tab_cblock<<<64, 256, 0, st>>>(X.PhB1i, 64, 64, 64, +1);  // W_64^{-j2 m2}
      k_tab_tw<<<64, 256, 0, st>>>(X.twph, 64, 64);                // W_4096^{m1 j2}
      XK(cudaGetLastError());
      bool ok4 = make_map(&X.mSxBlk[0], X.Sx.hi, (uint64_t)Nu * 64, 64, 64) &&
                 make_map(&X.mSxBlk[1], X.Sx.lo, (uint64_t)Nu * 64, 64, 64) &&
                 make_map(&X.mPhA1[0], X.PhA1.hi, 128, 64, tc::BM) && make_map(&X.mPhA1[1], X.PhA1.lo, 128, 64, tc::BM) &&
                 make_map(&X.mPhB2f[0], X.PhB2f.hi, 128, 128, tc::BN) &&
                 make_map(&X.mPhB2f[1], X.PhB2f.lo, 128, 128, tc::BN) &&
                 make_map(&X.mPhB1i[0], X.PhB1i.hi, 128, 128, tc::BN) &&
                 make_map(&X.mPhB1i[1], X.PhB1i.lo, 128, 128, tc::BN) &&
                 make_map(&X.mPhB2i[0], X.PhB2i.hi, 64, 128, tc::BN) && make_map(&X.mPhB2i[1], X.PhB2i.lo, 64, 128, tc::BN) &&
                 make_map(&X.mPhT[0], X.PhT.hi, (uint64_t)64 * Nu, 128, tc::BM) &&
                 make_map(&X.mPhT[1], X.PhT.lo, (uint64_t)64 * Nu, 128, tc::BM) &&
                 // X MN-major [(m2, ri)][(m1, i)]; V as [(i, m1, ri)][j2] (blocked MN-major A of Q2)
                 make_map(&X.mPhX[0], X.PhX.hi, 128, (uint64_t)64 * Nu, 64) &&
                 make_map(&X.mPhX[1], X.PhX.lo, 128, (uint64_t)64 * Nu, 64) &&
                 make_map(&X.mPhV[0], X.PhV.hi, (uint64_t)128 * Nu, 64, 64) &&
                 make_map(&X.mPhV[1], X.PhV.lo, (uint64_t)128 * Nu, 64, 64);
      if (!ok4) return fail(DG_ERR_CUDA, "mixed precision", "tensor map encoding failed (phi transforms at 4096)");
      XK((prepare_gemm<tc::kEpiPhiS1, false, true>()));
      XK((prepare_gemm<tc::kEpiPhiS2, false, false>()));
      XK((prepare_gemm<tc::kEpiI2ToX, false, false>()));
      XK((prepare_gemm<tc::kEpiPhiQ1, true, false>()));
      XK((prepare_gemm<tc::kEpiPhiQ2, true, false>()));
    }
    XK((prepare_gemm<tc::kEpiPhiToXin, false, false>()));
    XK((prepare_gemm<tc::kEpiTwiddleF1, false, true>()));
    XK((prepare_gemm<tc::kEpiSplitScaled, true, false>()));
    XK((prepare_gemm<tc::kEpiTwiddleI1, false, false>()));
    XK((prepare_gemm<tc::kEpiI2ToZ, false, false>()));
    XK((prepare_gemm<tc::kEpiRowScaleF32, true, false>()));
  }
  XK((prepare_gemm<tc::kEpiSplit, false, false>()));
  XK((prepare_gemm<tc::kEpiSplitScaled, false, false>()));
  XK((prepare_gemm<tc::kEpiRowScaleF32, false, false>()));
  XK(cudaStreamSynchronize(st));
  {
    const char *hk = getenv("DISKGPU_HYDRO32");
    X.hydro_kind = MixedState::kHydroPacked;
    if (hk && strcmp(hk, "warp") == 0) X.hydro_kind = MixedState::kHydroWarp;
    if (hk && strcmp(hk, "tile") == 0) X.hydro_kind = MixedState::kHydroTile;
    if (Nphi < kLd32t || Nphi % 2) X.hydro_kind = MixedState::kHydroWarp;
    if (X.hydro_kind != MixedState::kHydroWarp) {
      XK(hydro32t_prepare());
      bool okh = make_map_f32(&X.mPhi, X.dPhi, Nu, Nphi);
      for (int b = 0; b < 2; ++b)
        okh = okh && make_map_f32(&X.mSig[b], X.sig[b], Nu, Nphi) && make_map_f32(&X.mU[b], X.u[b], Nu, Nphi) &&
              make_map_f32(&X.mW[b], X.w[b], Nu, Nphi);
      if (!okh) return fail(DG_ERR_CUDA, "mixed precision", "tensor map encoding failed (hydro tiles)");
    }
  }
  {
    const char *ts = getenv("DISKGPU_TEST_ROWTILE_STALL");
    if (ts && *ts) {
      const int k = atoi(ts);
      if (k >= 0 && k < (Nu + kTileI - 1) / kTileI) X.test_stall = k;
    }
  }
  X.tables_ready = true;
  return DG_OK;
}

void dg_handle::mixed_basic(std::vector<double> *S0, std::vector<double> *V0, std::vector<double> *g0) const {
  if (!mx) {
    S0->clear(); V0->clear(); g0->clear();
    return;
  }
  *S0 = mx->S0;
  *V0 = mx->V0;
  *g0 = mx->g0;
}

void dg_handle::mixed_release() {
  if (!mx) return;
  MixedState &X = *mx;
  for (int b = 0; b < 2; ++b) {
    if (X.sig[b]) cudaFree(X.sig[b]);
    if (X.u[b]) cudaFree(X.u[b]);
    if (X.w[b]) cudaFree(X.w[b]);
  }
  SplitBuf *bufs[] = {&X.Sx, &X.X1, &X.Wt, &X.Z, &X.Fphi, &X.Cu, &X.CuT, &X.Gphi,
                      &X.Xin, &X.Tb, &X.Yk, &X.Ub, &X.RB, &X.RA, &X.RGA, &X.RGB, &X.PA, &X.PB,
                      &X.IA, &X.IB, &X.Zt, &X.PhA1, &X.PhB2f, &X.PhB1i, &X.PhB2i, &X.PhT, &X.PhX, &X.PhV};
  for (SplitBuf *b : bufs) free_split(*b);
  void *ptrs[] = {X.KW,  X.dPhi, X.rowpend, X.phiscale, X.rowbuf, X.rowtab, X.rowbufd,
                  X.KW2, X.tw,   X.khm,     X.twp,      X.twphi,  X.twph};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  delete mx;
  mx = nullptr;
}

// Basic state and its per-row tables.  S0, V0 are the phi averages of the given state
// (exactly the unperturbed profiles after dg_init_standard), g0 the phi-averaged radial
// force of the basic state's own FP64 potential.
static int build_basic(dg_handle *h, const double *Sig, const double *vp) {
  MixedState &X = *h->mx;
  const dg_params &p = h->p;
  const int Nu = p.Nu, Nphi = p.Nphi;
  X.S0.assign(Nu, 0.0);
  X.V0.assign(Nu, 0.0);
  X.g0.assign(Nu, 0.0);
  if (h->basic_from_standard) {
    X.S0 = h->std_sigma0;
    X.V0 = h->std_vphi0;
    X.g0 = h->std_gR0;
  } else {
    for (int i = 0; i < Nu; ++i) {
      double a = 0, b = 0;
      for (int j = 0; j < Nphi; ++j) { a += Sig[(size_t)i * Nphi + j]; b += vp[(size_t)i * Nphi + j]; }
      X.S0[i] = a / Nphi;
      X.V0[i] = b / Nphi;
    }
    if (p.selfgrav) {
      const size_t n = (size_t)Nu * Nphi;
      std::vector<double> axi(n), gR(n);
      for (int i = 0; i < Nu; ++i)
        for (int j = 0; j < Nphi; ++j) axi[(size_t)i * Nphi + j] = X.S0[i];
      if (cudaMemcpyAsync(h->gA, axi.data(), n * sizeof(double), cudaMemcpyHostToDevice, h->st) != cudaSuccess)
        return h->fail(DG_ERR_CUDA, "basic state", "upload");
      int rc = h->potential64(h->gA, h->dPhi);
      if (rc) return rc;
      if (launch_forces64(h->dPhi, h->gA, h->gB, h->geom, h->st) != cudaSuccess ||
          cudaMemcpyAsync(gR.data(), h->gA, n * sizeof(double), cudaMemcpyDeviceToHost, h->st) != cudaSuccess ||
          cudaStreamSynchronize(h->st) != cudaSuccess)
        return h->fail(DG_ERR_CUDA, "basic state", "gravity");
      for (int i = 0; i < Nu; ++i) {
        double s = 0;
        for (int j = 0; j < Nphi; ++j) s += gR[(size_t)i * Nphi + j];
        X.g0[i] = s / Nphi;
      }
    }
  }
  // FP64 row constants -> FP32 tables
  const std::vector<double> &R = h->R, &Rf = h->Rf, &Vol = h->Vol;
  const double K = p.Kpoly, gam = p.gamma_gas;
  std::vector<double> P0(Nu), dP0dR(Nu), a0(Nu);
  for (int i = 0; i < Nu; ++i) P0[i] = K * std::pow(X.S0[i], gam);
  for (int i = 0; i < Nu; ++i) {
    int im = i - 1 > 0 ? i - 1 : 0, ip = i + 1 < Nu - 1 ? i + 1 : Nu - 1;
    dP0dR[i] = (P0[ip] - P0[im]) / (R[ip] - R[im]);
    double gR = -p.gmstar / (R[i] * R[i]) + (p.selfgrav ? X.g0[i] : 0.0);
    a0[i] = -dP0dR[i] / X.S0[i] + gR + X.V0[i] * X.V0[i] / R[i];
  }
  const int L = Nu + 1;
  std::vector<float> rb((size_t)24 * L, 0.f);
  auto col = [&](int k) { return rb.data() + (size_t)k * L; };
  for (int i = 0; i < Nu; ++i) {
    int im = i - 1 > 0 ? i - 1 : 0, ip = i + 1 < Nu - 1 ? i + 1 : Nu - 1;
    col(0)[i] = (float)R[i];
    col(1)[i] = (float)(1.0 / R[i]);
    col(2)[i] = (float)(1.0 / (R[ip] - R[im]));
    col(3)[i] = (float)dP0dR[i];
    col(4)[i] = (float)X.S0[i];
    col(5)[i] = (float)(1.0 / X.S0[i]);
    col(6)[i] = (float)X.V0[i];
    col(7)[i] = (float)a0[i];
    col(8)[i] = (float)(Rf[i + 1] - Rf[i]);
    col(9)[i] = (float)(R[i] * h->dphi);
    col(10)[i] = (float)(Rf[i + 1] - Rf[i]);
    col(11)[i] = (float)(1.0 / Vol[i]);
    col(12)[i] = (float)h->R32[i];
    col(13)[i] = (float)P0[i];
    col(19)[i] = (float)(1.0 / (Rf[i + 1] - Rf[i]));
    col(20)[i] = (float)(1.0 / (R[i] * h->dphi));
  }
  for (int f = 0; f <= Nu; ++f) {
    col(14)[f] = (float)(Rf[f] * h->dphi);
    col(15)[f] = (f >= 1) ? (float)(Rf[f] - Rf[f - 1]) : 0.f;
    col(16)[f] = (f <= Nu - 1) ? (float)(Rf[f + 1] - Rf[f]) : 0.f;
    col(17)[f] = (f >= 1 && f <= Nu - 1) ? (float)(X.V0[f] - X.V0[f - 1]) : 0.f;
    col(18)[f] = (f >= 1 && f <= Nu - 1) ? (float)(X.S0[f] - X.S0[f - 1]) : 0.f;
    col(21)[f] = (f >= 1) ? (float)(1.0 / (Rf[f] - Rf[f - 1])) : 0.f;
    col(22)[f] = (f <= Nu - 1) ? (float)(1.0 / (Rf[f + 1] - Rf[f])) : 0.f;
  }
  std::vector<double> rd((size_t)4 * Nu);
  for (int i = 0; i < Nu; ++i) {
    rd[i] = X.S0[i];
    rd[Nu + i] = X.V0[i];
    rd[2 * Nu + i] = R[i];
    rd[3 * Nu + i] = R[i] * (Rf[i + 1] - Rf[i]) * h->dphi;
  }
  // row-major copy for k_hydro32p: row r = i + kRowTabLead, the tile kernels' row constants
  // (zero outside the grid; face arrays are defined up to i = Nu)
  static const int rt_col[tNConst] = {4, 5, 6, 7, 3, 2, 1, 0, 11, 20, 10, 12, 19, 13, 18, 17, 14, 21, 22};
  std::vector<float> rt((size_t)(Nu + kRowTabExtra) * kRowTabW, 0.f);
  for (int r = 0; r < Nu + kRowTabExtra; ++r) {
    const int i = r - kRowTabLead;
    for (int k = 0; k < tNConst; ++k) {
      const bool face = k >= tDS0;
      if (i >= 0 && (face ? i <= Nu : i < Nu)) rt[(size_t)r * kRowTabW + k] = col(rt_col[k])[i];
    }
  }
  if (cudaMemcpyAsync(X.rowbuf, rb.data(), rb.size() * sizeof(float), cudaMemcpyHostToDevice, h->st) != cudaSuccess ||
      cudaMemcpyAsync(X.rowtab, rt.data(), rt.size() * sizeof(float), cudaMemcpyHostToDevice, h->st) != cudaSuccess ||
      cudaMemcpyAsync(X.rowbufd, rd.data(), rd.size() * sizeof(double), cudaMemcpyHostToDevice, h->st) != cudaSuccess)
    return h->fail(DG_ERR_CUDA, "basic state", "row tables");
  Rows32 &g = X.rows;
  float *b = X.rowbuf;
  auto dc = [&](int k) { return (const float *)(b + (size_t)k * L); };
  g.R = dc(0); g.invR = dc(1); g.invdRc = dc(2); g.dP0dR = dc(3); g.S0 = dc(4); g.invS0 = dc(5); g.V0 = dc(6);
  g.a0 = dc(7); g.dR = dc(8); g.dl = dc(9); g.Aphi = dc(10); g.invVol = dc(11); g.R32 = dc(12); g.P0 = dc(13);
  g.Af = dc(14); g.dRl = dc(15); g.dRr = dc(16); g.dV = dc(17); g.dS0 = dc(18);
  g.invdR = dc(19); g.invdl = dc(20); g.invdRl = dc(21); g.invdRr = dc(22);
  g.rowtab = X.rowtab;
  g.S0d = X.rowbufd; g.V0d = X.rowbufd + Nu; g.Rd = X.rowbufd + 2 * Nu; g.dAd = X.rowbufd + 3 * Nu;
  g.Nu = Nu; g.Nphi = Nphi;
  g.dphi = (float)h->dphi; g.inv2dphi = (float)(1.0 / (2.0 * h->dphi));
  g.invdu = (float)(1.0 / h->du); g.inv2du = (float)(1.0 / (2.0 * h->du));
  g.Kpoly = (float)K; g.gamma = (float)gam; g.gmstar = (float)p.gmstar;
  g.gamma2 = (gam == 2.0) ? 1 : 0;
  return DG_OK;
}

static cudaError_t launch_hydro32(MixedState &X, const float *sig, const float *u, const float *w, const float *Phi,
                                  const double *gR, const double *gp, int fm, float *so, float *uo, float *wo, Ctl *ctl,
                                  cudaStream_t st, int *rowpend = nullptr, bool early_state = false,
                                  bool finalize = true);
static cudaError_t launch_finalize(const MixedState &X, Ctl *ctl, cudaStream_t st);

int dg_handle::mixed_upload_state(const double *Sig, const double *vRh, const double *vph) {
  MixedState &X = *mx;
  const size_t n = (size_t)p.Nu * p.Nphi;
  // a new basic state on dg_set_state / dg_init_standard; dg_step_host keeps the current one
  if (!in_step_host) {
    int rc = build_basic(this, Sig, vph);
    if (rc) return rc;
  }
  XK(cudaMemcpyAsync(S[0], Sig, n * sizeof(double), cudaMemcpyHostToDevice, st));
  XK(cudaMemcpyAsync(VR[0], vRh, n * sizeof(double), cudaMemcpyHostToDevice, st));
  XK(cudaMemcpyAsync(VP[0], vph, n * sizeof(double), cudaMemcpyHostToDevice, st));
  k_to_pert<<<grid_for(n), 256, 0, st>>>(S[0], VR[0], VP[0], X.sig[cur], X.u[cur], X.w[cur], X.Sx, X.rows);
  XK(cudaGetLastError());
  if (!in_step_host && !X.tuned) {
    int rc = mixed_autotune();
    if (rc) return rc;
    // the tuning launches overwrote the gravity operand: rebuild it from the uploaded state
    k_to_pert<<<grid_for(n), 256, 0, st>>>(S[0], VR[0], VP[0], X.sig[cur], X.u[cur], X.w[cur], X.Sx, X.rows);
    XK(cudaGetLastError());
  }
  // no hydro step is in flight: the row-tile counters start from zero.  This memset is the
  // upload's last operation, so the next step's phi transform (which, with the row-tile
  // hand-over, does not wait on its predecessor kernel) never directly follows the kernel
  // that wrote its input.
  XK(cudaMemsetAsync(X.rowpend, 0, (size_t)(p.Nu + kTileI - 1) / kTileI * sizeof(int), st));
  X.prev_rs = false;
  return DG_OK;
}

// ---------------------------------------------------------------------------------
// Autotuner.  At a handle's first state upload (dg_set_state, dg_init_standard, dg_load;
// never inside a stream capture) it times the step's kernel variants on the handle's own
// buffers and keeps the fastest:
//   * the pipeline depth (1, 2 or 4 stages) of every gravity product, one product at a time
//     with the others fixed, timing the whole gravity of the uploaded state;
//   * the hydro form (tiled, packed two-column, warp-marching), writing the other ping-pong
//     buffers and a scratch control block, so the handle's dt, time and records are untouched.
// A variant must beat the current choice by 2 % to replace it.  Choices are cached per
// process by (Nu, Nphi, Gamma = 2, self-gravity), so the disks of a batch that share a grid
// are tuned once.  DISKGPU_TUNE=0 keeps the defaults (packed hydro, stages by K);
// DISKGPU_HYDRO32 fixes the hydro form.
namespace {
struct TuneKey {
  int Nu, Nphi, g2, sg;
  bool operator<(const TuneKey &o) const {
    if (Nu != o.Nu) return Nu < o.Nu;
    if (Nphi != o.Nphi) return Nphi < o.Nphi;
    if (g2 != o.g2) return g2 < o.g2;
    return sg < o.sg;
  }
};
struct TuneVal {
  int hydro_kind;
  int ns[6];
  std::string info;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune_cache;
const char *kHydroNames[3] = {"warp", "tile", "packed"};
}  // namespace

int dg_handle::mixed_autotune() {
  MixedState &X = *mx;
  X.tuned = true;
  const char *env = getenv("DISKGPU_TUNE");
  if (env && strcmp(env, "0") == 0) {
    X.tune_info = "tuning off: hydro " + std::string(kHydroNames[X.hydro_kind]) + ", stages by K";
    return DG_OK;
  }
  const char *hk = getenv("DISKGPU_HYDRO32");
  // the warp form is the only one for odd or narrow grids; a user's choice stands
  const bool hydro_fixed = (hk && *hk) || X.hydro_kind == MixedState::kHydroWarp;
  // DISKGPU_STAGES=s0,s1,s2,s3,s4,s5 fixes the pipeline depth of every gravity product
  // (0 = chosen by K, else 1, 2 or 4; 8 = the persistent kernel, 16 = the same with
  // 128 x 256 tiles) and skips their tuning
  bool stages_fixed = false;
  if (const char *sv = getenv("DISKGPU_STAGES")) {
    int v[6], n = sscanf(sv, "%d,%d,%d,%d,%d,%d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5]);
    if (n != 6) return fail(DG_ERR_INVALID, "autotune", "DISKGPU_STAGES wants six comma-separated depths");
    for (int k = 0; k < 6; ++k) {
      if (v[k] != 0 && v[k] != 1 && v[k] != 2 && v[k] != 4 && v[k] != kPersist && v[k] != kPersistWide)
        return fail(DG_ERR_INVALID, "autotune",
                    "DISKGPU_STAGES: a depth is 0, 1, 2, 4, 8 (persistent) or 16 (persistent, 128 x 256 tiles)");
      X.ns[k] = v[k];
    }
    stages_fixed = true;
  }
  const TuneKey key{p.Nu, p.Nphi, X.rows.gamma2, p.selfgrav};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      if (!hydro_fixed) X.hydro_kind = it->second.hydro_kind;
      if (!stages_fixed) memcpy(X.ns, it->second.ns, sizeof(X.ns));
      X.tune_info = it->second.info + " (cached)";
      if (stages_fixed && p.selfgrav) {  // the fixed depths, not the cached ones, are in use
        std::string f = "gravity stages fixed";
        for (int k = 0; k < 6; ++k) f += " " + std::to_string(X.ns[k]);
        X.tune_info = f + "; " + X.tune_info;
      }
      return DG_OK;
    }
  }
  const bool prof_was = prof_on;
  prof_on = false;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  XK(cudaEventCreate(&e0));
  XK(cudaEventCreate(&e1));
  Ctl *sctl = nullptr;
  int rc = DG_OK;
  char buf[256];
  std::string info;
  // best of 3 timed runs after one warm-up, in microseconds
  auto time_us = [&](auto &&fn, float *best) -> cudaError_t {
    *best = 1e30f;
    for (int r = 0; r < 4; ++r) {
      cudaError_t e = fn(true);
      if (e != cudaSuccess) return e;
      if ((e = cudaEventRecord(e0, st)) != cudaSuccess) return e;
      if ((e = fn(false)) != cudaSuccess) return e;
      if ((e = cudaEventRecord(e1, st)) != cudaSuccess) return e;
      if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return e;
      float ms = 0.f;
      if ((e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) return e;
      if (r > 0 && 1e3f * ms < *best) *best = 1e3f * ms;
    }
    return cudaSuccess;
  };
  do {
    if (p.selfgrav && stages_fixed) {
      info += "gravity stages fixed";
      for (int k = 0; k < 6; ++k) {
        snprintf(buf, sizeof buf, " %d", X.ns[k]);
        info += buf;
      }
    } else if (p.selfgrav) {
      // products that run as k_gemm_split (the fused kernels have no pipeline to tune)
      const std::vector<int> slots = !X.factored ? std::vector<int>{0, 1, 2, 5}
                                     : (X.fused_phi ? std::vector<int>{}
                                        : (X.fused_u ? std::vector<int>{0, 5} : std::vector<int>{0, 1, 2, 3, 4, 5}));
      auto grav = [&](bool) -> cudaError_t { return mixed_gravity() ? cudaErrorUnknown : cudaSuccess; };
      float tbest;
      cudaError_t e = time_us(grav, &tbest);
      if (e != cudaSuccess) { rc = fail(DG_ERR_CUDA, "autotune", cudaGetErrorString(e)); break; }
      const float t0 = tbest;
      for (int sl : slots) {
        int keep = X.ns[sl];
        for (int cand : {1, 2, 4, kPersist, kPersistWide}) {
          X.ns[sl] = cand;
          float t;
          if ((e = time_us(grav, &t)) != cudaSuccess) break;
          if (t < 0.98f * tbest) {
            tbest = t;
            keep = cand;
          }
        }
        X.ns[sl] = keep;
        if (e != cudaSuccess) break;
      }
      if (e != cudaSuccess) { rc = fail(DG_ERR_CUDA, "autotune", cudaGetErrorString(e)); break; }
      snprintf(buf, sizeof buf, "gravity %.1f us (stages by K: %.1f us), stages", tbest, t0);
      info += buf;
      for (int sl : slots) {
        snprintf(buf, sizeof buf, " %d", X.ns[sl] ? X.ns[sl] : 0);
        info += buf;
      }
    }
    if (!hydro_fixed) {
      if (cudaMalloc(&sctl, sizeof(Ctl)) != cudaSuccess) { rc = fail(DG_ERR_NOMEM, "autotune", "control block"); break; }
      Ctl h0;
      memset(&h0, 0, sizeof h0);
      h0.t = 0.0; h0.tlim = 1e300; h0.cfl = 0.3; h0.dt = 1e-7; h0.tnext = 1e300; h0.dtout = 1.0; h0.mD = 1.0;
      h0.fixed_dt = 1;
      const int fm = p.selfgrav ? kForcePhi : kForceNone;
      const int c = cur, o = cur ^ 1;
      auto hyd = [&](bool) -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(sctl, &h0, sizeof(Ctl), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
        return launch_hydro32(X, X.sig[c], X.u[c], X.w[c], X.dPhi, nullptr, nullptr, fm, X.sig[o], X.u[o], X.w[o],
                              sctl, st);
      };
      // the packed form first: it is timed alone here, but inside a step its TMA-staged tile,
      // bulk-copied row constants and early control loads overlap the kernels around it, so
      // another form must beat it by the margin alone
      const int kinds[3] = {MixedState::kHydroPacked, MixedState::kHydroTile, MixedState::kHydroWarp};
      float tk[3] = {0.f, 0.f, 0.f};
      int best = MixedState::kHydroPacked;
      float tb = 1e30f;
      cudaError_t e = cudaSuccess;
      for (int q = 0; q < 3 && e == cudaSuccess; ++q) {
        X.hydro_kind = kinds[q];
        e = time_us(hyd, &tk[q]);
        if (e == cudaSuccess && (q == 0 || tk[q] < 0.98f * tb)) {
          tb = tk[q];
          best = kinds[q];
        }
      }
      X.hydro_kind = best;
      if (e != cudaSuccess) { rc = fail(DG_ERR_CUDA, "autotune", cudaGetErrorString(e)); break; }
      snprintf(buf, sizeof buf, "%shydro %s (packed %.1f us, tile %.1f us, warp %.1f us)", info.empty() ? "" : "; ",
               kHydroNames[best], tk[0], tk[1], tk[2]);
      info += buf;
    } else {
      info += std::string(info.empty() ? "" : "; ") + "hydro " + kHydroNames[X.hydro_kind] + " (fixed)";
    }
  } while (false);
  if (sctl) cudaFree(sctl);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  prof_on = prof_was;
  if (rc) return rc;
  X.tune_info = info;
  if (stages_fixed) return DG_OK;  // a forced choice is not what the grid's tuning found
  std::lock_guard<std::mutex> lk(g_tune_mu);
  TuneVal v;
  v.hydro_kind = X.hydro_kind;
  memcpy(v.ns, X.ns, sizeof(v.ns));
  v.info = info;
  g_tune_cache[key] = v;
  return DG_OK;
}

std::string dg_handle::mixed_tuning_info() const { return mx ? mx->tune_info : std::string(); }

int dg_handle::mixed_download_state(double *Sig, double *vRh, double *vph) {
  MixedState &X = *mx;
  const size_t n = (size_t)p.Nu * p.Nphi;
  k_from_pert<<<grid_for(n), 256, 0, st>>>(X.sig[cur], X.u[cur], X.w[cur], S[0], VR[0], VP[0], X.rows);
  XK(cudaGetLastError());
  XK(cudaMemcpyAsync(Sig, S[0], n * sizeof(double), cudaMemcpyDeviceToHost, st));
  XK(cudaMemcpyAsync(vRh, VR[0], n * sizeof(double), cudaMemcpyDeviceToHost, st));
  XK(cudaMemcpyAsync(vph, VP[0], n * sizeof(double), cudaMemcpyDeviceToHost, st));
  XK(cudaStreamSynchronize(st));
  return DG_OK;
}

// End of a tile hydro launch: t, dt, records and diagnostics from the sums its CTAs folded
// into the control block (step_ctl.cuh finish_launch_deferred).
__global__ void k_step_finalize(Ctl *ctl) {
  pdl_trigger();  // the next kernel's prologue may start; it waits for this one's completion
  pdl_wait();     // every CTA of the hydro launch has folded its sums
  if (threadIdx.x == 0) finalize_launch(ctl, read_step_info(ctl, true, ctl->pend_active));
}

// the same for every disk of a group (one block per disk)
__global__ void k_step_finalize_group(const HydroDisk *__restrict__ disks) {
  pdl_trigger();
  pdl_wait();
  Ctl *ctl = disks[blockIdx.x].ctl;
  if (threadIdx.x == 0) finalize_launch(ctl, read_step_info(ctl, true, ctl->pend_active));
}

// the step's finalisation after a tile hydro launch (the warp form finalises in its last CTA)
static cudaError_t launch_finalize(const MixedState &X, Ctl *ctl, cudaStream_t st) {
  if (X.hydro_kind == MixedState::kHydroWarp) return cudaSuccess;
  return launch_pdl(k_step_finalize, dim3(1), dim3(32), 0, st, ctl);
}

static cudaError_t launch_hydro32(MixedState &X, const float *sig, const float *u, const float *w, const float *Phi,
                                  const double *gR, const double *gp, int fm, float *so, float *uo, float *wo, Ctl *ctl,
                                  cudaStream_t st, int *rowpend, bool early_state, bool finalize) {
  if (X.hydro_kind == MixedState::kHydroPacked) {
    dim3 grid((X.Nphi + kTileJp - 1) / kTileJp, (X.Nu + kTileI - 1) / kTileI);
    const SplitBf16 sx{X.Sx.hi, X.Sx.lo};
    cudaError_t e = cudaSuccess;
    const int b = (sig == X.sig[1]) ? 1 : 0;  // which ping-pong buffer holds the input
    auto go = [&](auto kern) {
      e = launch_pdl(kern, grid, dim3(kThreads32t), kSmem32p, st, X.mSig[b], X.mU[b], X.mW[b], X.mPhi, sig, u, w, Phi,
                     gR, gp, so, uo, wo, sx, ctl, X.rows, rowpend, early_state ? 1 : 0);
    };
    const bool g2 = X.rows.gamma2 != 0;
    if (fm == kForcePhi) g2 ? go(k_hydro32p<true, kForcePhi>) : go(k_hydro32p<false, kForcePhi>);
    else if (fm == kForceArrays) g2 ? go(k_hydro32p<true, kForceArrays>) : go(k_hydro32p<false, kForceArrays>);
    else g2 ? go(k_hydro32p<true, kForceNone>) : go(k_hydro32p<false, kForceNone>);
    if (e == cudaSuccess && finalize) e = launch_finalize(X, ctl, st);
    return e;
  }
  if (X.hydro_kind == MixedState::kHydroTile) {
    dim3 grid((X.Nphi + kTileJ - 1) / kTileJ, (X.Nu + kTileI - 1) / kTileI);
    const SplitBf16 sx{X.Sx.hi, X.Sx.lo};
    cudaError_t e = cudaSuccess;
    auto go = [&](auto kern) {
      e = launch_pdl(kern, grid, dim3(kThreads32t), kSmem32t, st, sig, u, w, Phi, gR, gp, so, uo, wo, sx, ctl, X.rows,
                     rowpend);
    };
    const bool g2 = X.rows.gamma2 != 0;
    if (fm == kForcePhi) g2 ? go(k_hydro32t<true, kForcePhi>) : go(k_hydro32t<false, kForcePhi>);
    else if (fm == kForceArrays) g2 ? go(k_hydro32t<true, kForceArrays>) : go(k_hydro32t<false, kForceArrays>);
    else g2 ? go(k_hydro32t<true, kForceNone>) : go(k_hydro32t<false, kForceNone>);
    if (e == cudaSuccess && finalize) e = launch_finalize(X, ctl, st);
    return e;
  }
  if (rowpend) return cudaErrorInvalidValue;  // the warp form has no row-tile hand-over
  const int nstrips = (X.Nphi + kOutCols32 - 1) / kOutCols32;
  dim3 grid((nstrips + kWarps32 - 1) / kWarps32, (X.Nu + kBand32 - 1) / kBand32);
  k_hydro32w<<<grid, kWarps32 * 32, 0, st>>>(sig, u, w, Phi, gR, gp, fm, so, uo, wo, SplitBf16{X.Sx.hi, X.Sx.lo}, ctl,
                                             X.rows, nstrips);
  return cudaGetLastError();
}


// dPhi = gravity of s (the split operand in X.Sx)
int dg_handle::mixed_gravity() {
  MixedState &X = *mx;
  const int Nu = p.Nu, Nphi = p.Nphi;
  tc::GemmArgs a{};
  a.status = &ctl->status;
  if (X.factored) {
    const int A = X.fa, nm = X.nm;
    a.fa = A; a.nphi = Nphi; a.nmodes = nm; a.twiddle = X.tw;
    // G1: phi DFT, stored as the F1 operand Xin[(i2, ri)][(m, i1)]
    a.out_hi = X.Xin.hi; a.out_lo = X.Xin.lo;
    XK(prof_begin(DG_PROF_GRAV_PHI_FWD));
    if (X.fused_phi) {
      // real 32-point stage, twiddle, complex 32-point stage: 4 rows per CTA
      tc::PhiFwdArgs f{X.Sx.hi, X.Sx.lo, X.twphi, X.Xin.hi, X.Xin.lo, nm * A, Nphi, &ctl->status,
                       X.rs_wait ? X.rowpend : nullptr};
      XK(launch_pdl(tc::k_phifwd, dim3(Nu / tc::kPfRows), dim3(tc::kPfThreads), tc::kPfSmem, st, X.mPA[0], X.mPA[1],
                    X.mPB[0], X.mPB[1], f));
    } else if (X.phi4096) {
      // S1: real 64-point DFT over j1 (s read as [(i, j1)][j2]), x W_N^{j2 m1} -> T[(m1, i)][(ri, j2)]
      a.out_hi = X.PhT.hi; a.out_lo = X.PhT.lo; a.twiddle = X.twph;
      XK((gemm<tc::kEpiPhiS1, false, true>(X.mPhA1[0], X.mPhA1[1], X.mSxBlk[0], X.mSxBlk[1], 128, Nu * 64, 64, a,
                                             st, X.ns[0])));
      // S2: complex 64-point DFT over j2 -> modes m = m1 + 64 m2 <= N/2 into Xin
      a.out_hi = X.Xin.hi; a.out_lo = X.Xin.lo;
      XK(gemm<tc::kEpiPhiS2>(X.mPhT[0], X.mPhT[1], X.mPhB2f[0], X.mPhB2f[1], 64 * Nu, 128, 128, a, st, X.ns[0]));
      a.twiddle = X.tw;
    } else {
      XK(gemm<tc::kEpiPhiToXin>(X.mFphi[0], X.mFphi[1], X.mSx[0], X.mSx[1], Nphi, Nu, Nphi, a, st, X.ns[0]));
    }
    XK(prof_end(DG_PROF_GRAV_PHI_FWD));
    XK(prof_begin(DG_PROF_GRAV_U));
    if (X.fused_u) {
      // F1, F2, I1, I2 in one kernel: four modes per CTA, operands kept on chip
      tc::UconvArgs u{X.twp, X.khm, X.Z.hi, X.Z.lo, Nu, Nphi, &ctl->status,
                      X.fused_phi ? X.Zt.hi : nullptr, X.fused_phi ? X.Zt.lo : nullptr};
      XK(launch_pdl(tc::k_uconv, dim3(nm / tc::kUcModes), dim3(tc::kUcThreads), tc::kUcSmem, st, X.mRB[0], X.mRB[1],
                    X.mXin[0], X.mXin[1], X.mRA[0], X.mRA[1], X.mRGA[0], X.mRGA[1], X.mRGB[0], X.mRGB[1], u));
    } else {
      // F1: 64-point DFT over i2 (K = 32 complex), twiddle, -> Tb[(i1, ri)][(m, p2)]
      a.out_hi = X.Tb.hi; a.out_lo = X.Tb.lo;
      XK((gemm<tc::kEpiTwiddleF1, false, true>(X.mRB[0], X.mRB[1], X.mXin[0], X.mXin[1], 128, nm * A, 64, a, st,
                                                 X.ns[1])));
      // F2: A-point DFT over i1, x khat / M -> Yk[(m, p2)][(p1, ri)]
      a.out_hi = X.Yk.hi; a.out_lo = X.Yk.lo; a.ldo = 2 * A; a.table = X.KW2;
      XK((gemm<tc::kEpiSplitScaled, true, false>(X.mTb[0], X.mTb[1], X.mRA[0], X.mRA[1], nm * 64, 2 * A, 2 * A, a,
                                                   st, X.ns[2])));
      // I1: inverse A-point DFT over p1, conjugate twiddle -> Ub[(m, i1)][(p2, ri)]
      a.out_hi = X.Ub.hi; a.out_lo = X.Ub.lo; a.table = nullptr;
      XK(gemm<tc::kEpiTwiddleI1>(X.mYk[0], X.mYk[1], X.mRGA[0], X.mRGA[1], nm * 64, 2 * A, 2 * A, a, st, X.ns[3]));
      // I2: inverse 64-point DFT over p2 (the 32 physical i2) -> Z[c][i], or at Nphi = 4096
      // the full Hermitian spectrum X[(m / 64, ri)][(m % 64, i)] of the four-step inverse
      if (X.phi4096) {
        a.out_hi = X.PhX.hi; a.out_lo = X.PhX.lo;
        XK(gemm<tc::kEpiI2ToX>(X.mUb[0], X.mUb[1], X.mRGB[0], X.mRGB[1], nm * A, 64, 128, a, st, X.ns[4]));
      } else {
        a.out_hi = X.Z.hi; a.out_lo = X.Z.lo;
        XK(gemm<tc::kEpiI2ToZ>(X.mUb[0], X.mUb[1], X.mRGB[0], X.mRGB[1], nm * A, 64, 128, a, st, X.ns[4]));
      }
    }
    XK(prof_end(DG_PROF_GRAV_U));
    // G4: inverse phi DFT: the fused two-stage kernel from Zt, or a product with Z as an
    // MN-major operand; in a time step it arms the hydro's row-tile counters with the hydro
    // launch's column-tile count
    int *rp = X.rs_arm ? X.rowpend : nullptr;
    const int rp_n = (Nu + kTileI - 1) / kTileI;
    const int rp_val =
        X.hydro_kind == MixedState::kHydroPacked ? (Nphi + kTileJp - 1) / kTileJp : (Nphi + kTileJ - 1) / kTileJ;
    XK(prof_begin(DG_PROF_GRAV_PHI_INV));
    if (X.phi4096) {
      // Q1: inverse 64-point DFT over m2 (X read MN-major), x W_N^{-j2 m1} -> V[(i, m1)][(ri, j2)]
      a.out_hi = X.PhV.hi; a.out_lo = X.PhV.lo; a.twiddle = X.twph;
      XK((gemm<tc::kEpiPhiQ1, true, false>(X.mPhX[0], X.mPhX[1], X.mPhB1i[0], X.mPhB1i[1], 64 * Nu, 128, 128, a,
                                            st, X.ns[5])));
      // Q2: real part of the inverse 64-point DFT over m1, / N, x (-G du dphi / sqrt(R))
      a.out_hi = a.out_lo = nullptr; a.out_f32 = X.dPhi; a.row_scale = X.phiscale;
      XK((gemm<tc::kEpiPhiQ2, true, false>(X.mPhV[0], X.mPhV[1], X.mPhB2i[0], X.mPhB2i[1], 64 * Nu, 64, 128, a,
                                            st, X.ns[5])));
    } else if (X.fused_phi) {
      tc::PhiInvArgs f{X.Zt.hi, X.Zt.lo, X.twphi, X.phiscale, X.dPhi, Nphi, &ctl->status, rp, rp_n, rp_val};
      XK(launch_pdl(tc::k_phiinv, dim3(Nu / tc::kPiRows), dim3(tc::kPiThreads), tc::kPiSmem, st, X.mIA[0], X.mIA[1],
                    X.mIB[0], X.mIB[1], f));
    } else {
      a.out_hi = a.out_lo = nullptr; a.out_f32 = X.dPhi; a.ldo = Nphi; a.row_scale = X.phiscale;
      a.rowpend = rp; a.rp_n = rp_n; a.rp_val = rp_val;
      XK((gemm<tc::kEpiRowScaleF32, true, false>(X.mZmn[0], X.mZmn[1], X.mGphi[0], X.mGphi[1], Nu, Nphi, Nphi, a, st,
                                                 X.ns[5])));
    }
    XK(prof_end(DG_PROF_GRAV_PHI_INV));
    return DG_OK;
  }
  // G1: X1[c][i] = Fphi[c][:] . Sx[i][:]
  a.out_hi = X.X1.hi; a.out_lo = X.X1.lo; a.ldo = Nu;
  XK(prof_begin(DG_PROF_GRAV_PHI_FWD));
  XK(gemm<tc::kEpiSplit>(X.mFphi[0], X.mFphi[1], X.mSx[0], X.mSx[1], Nphi, Nu, Nphi, a, st, X.ns[0]));
  XK(prof_end(DG_PROF_GRAV_PHI_FWD));
  // G2: Wt[c][p] = KW[c][p] * X1[c][:] . Cu[p][:]
  a.out_hi = X.Wt.hi; a.out_lo = X.Wt.lo; a.ldo = 2 * Nu; a.table = X.KW;
  XK(prof_begin(DG_PROF_GRAV_U));
  XK(gemm<tc::kEpiSplitScaled>(X.mX1[0], X.mX1[1], X.mCu[0], X.mCu[1], Nphi, 2 * Nu, Nu, a, st, X.ns[1]));
  // G3: Z[i][c] = CuT[i][:] . Wt[c][:]
  a.out_hi = X.Z.hi; a.out_lo = X.Z.lo; a.ldo = Nphi; a.table = nullptr;
  XK(gemm<tc::kEpiSplit>(X.mCuT[0], X.mCuT[1], X.mWt[0], X.mWt[1], Nu, Nphi, 2 * Nu, a, st, X.ns[2]));
  XK(prof_end(DG_PROF_GRAV_U));
  // G4: dPhi[i][j] = phiscale[i] * Z[i][:] . Gphi[j][:]
  a.out_hi = a.out_lo = nullptr; a.out_f32 = X.dPhi; a.ldo = Nphi; a.row_scale = X.phiscale;
  XK(prof_begin(DG_PROF_GRAV_PHI_INV));
  XK(gemm<tc::kEpiRowScaleF32>(X.mZ[0], X.mZ[1], X.mGphi[0], X.mGphi[1], Nu, Nphi, Nphi, a, st, X.ns[5]));
  XK(prof_end(DG_PROF_GRAV_PHI_INV));
  return DG_OK;
}

// whether the last enqueued hydro counted down the row-tile counters (prev_rs)
int dg_handle::loop_flags() const { return (mx && mx->prev_rs) ? 1 : 0; }
void dg_handle::set_loop_flags(int f) {
  if (mx) mx->prev_rs = (f & 1) != 0;
}

// the tile forms end with k_step_finalize
int dg_handle::mixed_hydro_kernels() const {
  return (mx && mx->hydro_kind != MixedState::kHydroWarp) ? 2 : 1;
}

int dg_handle::mixed_gravity_kernels() const {
  if (!u_factored(p.Nu)) return 4;
  if (mx && mx->phi4096) return 8;
  return u_fused(p.Nu) ? 3 : 6;
}

int dg_handle::mixed_enqueue_step() {
  MixedState &X = *mx;
  const int c = cur, o = cur ^ 1;
  int fm = kForceNone;
  // row-tile hand-over: this step's phi transform waits for the previous step's hydro rows,
  // its inverse phi transform arms the counters this step's hydro counts down
  const bool rs = p.selfgrav && X.rowsync_ok();
  if (p.selfgrav) {
    XK(prof_begin(DG_PROF_GRAVITY));
    X.rs_arm = rs;
    X.rs_wait = rs && X.prev_rs;
    int rc = mixed_gravity();
    X.rs_arm = X.rs_wait = false;
    if (rc) return rc;
    XK(prof_end(DG_PROF_GRAVITY));
    fm = kForcePhi;
  }
  XK(prof_begin(DG_PROF_HYDRO));
  // with self-gravity the hydro's predecessor is the inverse phi transform, which writes
  // only dPhi: the packed form may fetch the state before its dependence wait
  XK(launch_hydro32(X, X.sig[c], X.u[c], X.w[c], X.dPhi, nullptr, nullptr, fm, X.sig[o], X.u[o], X.w[o], ctl, st,
                    rs ? X.rowpend : nullptr, fm == kForcePhi, false));
  X.prev_rs = rs;
  XK(prof_end(DG_PROF_HYDRO));  // the hydro kernel alone; its finalisation follows
  XK(launch_finalize(X, ctl, st));
  if (rs && X.test_stall >= 0) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    XK(cudaStreamIsCapturing(st, &cs));
    if (cs == cudaStreamCaptureStatusNone) {
      k_rowtile_stall<<<1, 1, 0, st>>>(X.rowpend + X.test_stall);
      XK(cudaGetLastError());
      X.test_stall = -1;
    }
  }
  cur = o;
  return DG_OK;
}

int dg_handle::mixed_enqueue_step_forces(const double *gRh, const double *gph) {
  MixedState &X = *mx;
  const size_t n = (size_t)p.Nu * p.Nphi;
  int fm = kForceNone;
  if (gRh) {
    // caller forces replace the self-gravity: subtract the basic-state gravity g0 from them
    std::vector<double> a(gRh, gRh + n);
    if (p.selfgrav)
      for (int i = 0; i < p.Nu; ++i)
        for (int j = 0; j < p.Nphi; ++j) a[(size_t)i * p.Nphi + j] -= X.g0[i];
    XK(cudaMemcpyAsync(gA, a.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    XK(cudaMemcpyAsync(gB, gph, n * sizeof(double), cudaMemcpyHostToDevice, st));
    XK(cudaStreamSynchronize(st));
    fm = kForceArrays;
  } else if (p.selfgrav) {
    // no forces: the basic state loses its disk gravity too
    std::vector<double> a(n);
    for (int i = 0; i < p.Nu; ++i)
      for (int j = 0; j < p.Nphi; ++j) a[(size_t)i * p.Nphi + j] = -X.g0[i];
    std::vector<double> z(n, 0.0);
    XK(cudaMemcpyAsync(gA, a.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    XK(cudaMemcpyAsync(gB, z.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    XK(cudaStreamSynchronize(st));
    fm = kForceArrays;
  }
  const int c = cur, o = cur ^ 1;
  X.prev_rs = false;
  XK(launch_hydro32(X, X.sig[c], X.u[c], X.w[c], nullptr, gA, gB, fm, X.sig[o], X.u[o], X.w[o], ctl, st));
  cur = o;
  return DG_OK;
}

int dg_handle::mixed_cfl_launch(int nmodes, int record) {
  MixedState &X = *mx;
  const size_t n = (size_t)p.Nu * p.Nphi;
  int blocks = grid_for(n);
  if (blocks > 148 * 4) blocks = 148 * 4;
  k_cfl32<<<blocks, 256, 0, st>>>(X.sig[cur], X.u[cur], X.w[cur], ctl, X.rows, nmodes, record);
  XK(cudaGetLastError());
  return DG_OK;
}

int dg_handle::mixed_modes_launch(int nmodes, double *out) {
  MixedState &X = *mx;
  const size_t n = (size_t)p.Nu * p.Nphi;
  XK(cudaMemsetAsync(out, 0, 2 * nmodes * sizeof(double), st));
  k_modes32<<<grid_for(n) < 592 ? grid_for(n) : 592, 256, 0, st>>>(X.sig[cur], X.rows, nmodes, out);
  XK(cudaGetLastError());
  return DG_OK;
}

int dg_handle::mixed_conserved_launch(double *out2) {
  MixedState &X = *mx;
  const size_t n = (size_t)p.Nu * p.Nphi;
  XK(cudaMemsetAsync(out2, 0, 2 * sizeof(double), st));
  k_conserved32<<<grid_for(n) < 592 ? grid_for(n) : 592, 256, 0, st>>>(X.sig[cur], X.w[cur], X.rows, out2);
  XK(cudaGetLastError());
  return DG_OK;
}

// dg_potential in mixed precision: the tensor-core convolution of a full field
int dg_handle::mixed_potential(const double *dSig, double *dOut) {
  MixedState &X = *mx;
  const size_t n = (size_t)p.Nu * p.Nphi;
  k_full_to_sx<<<grid_for(n), 256, 0, st>>>(dSig, X.Sx, dR32, p.Nu, p.Nphi);
  XK(cudaGetLastError());
  int rc = mixed_gravity();
  if (rc) return rc;
  k_f32_to_f64<<<grid_for(n), 256, 0, st>>>(X.dPhi, dOut, n);
  XK(cudaGetLastError());
  // restore s of the current state for the next step
  if (have_state) {
    k_sig_to_sx<<<grid_for(n), 256, 0, st>>>(X.sig[cur], X.Sx, X.rows);
    XK(cudaGetLastError());
  }
  return DG_OK;
}

// ---------------------------------------------------------------------------------
// Disk groups of a batched sweep (batch.cu): disks of one grid, Gamma class, hydro form and
// product pipeline depths advance with one launch per kernel for the whole group (the
// disk in blockIdx.z, or blockIdx.y for the fused 1024^2 transforms).  Each disk keeps its
// own state, khat table, row tables, control block and dt; the DFT tables, identical for
// one grid, are the lead disk's.  A disk's tiles run exactly the code of its lone step, so
// a grouped step equals the lone one bit for bit (the lone step's row-tile hand-over
// between the hydro sweep and the phi transforms only orders the same work differently).

struct MixedGroup {
  std::vector<dg_handle *> disks;
  dg_handle *lead = nullptr;
  int kind = MixedState::kHydroPacked;
  bool g2 = false;
  int ns[6] = {0, 0, 0, 0, 0, 0};
  bool persist = true;  // products by the persistent 128 x 128 kernel (DISKGPU_GROUP_GEMM=tile: per-tile kernel)
  int nsm = 148;
  tc::GemmDisk *gd[4] = {nullptr, nullptr, nullptr, nullptr};  // per product: one entry per disk
  HydroDisk *hd = nullptr;
  // 1024^2 disks: the fused phi transform, u convolution and inverse phi transform
  bool fused = false;
  tc::PhiFwdArgs *pf = nullptr;
  tc::UconvDisk *uc = nullptr;
  tc::PhiInvArgs *pi = nullptr;
};

std::string mixed_group_key(const dg_handle *h, bool with_fused) {
  if (!h || h->p.precision != DG_PREC_MIXED || !h->p.selfgrav || !h->mx || !h->mx->tables_ready ||
      !h->have_state)
    return std::string();
  const MixedState &X = *h->mx;
  // dense products, or the fused 1024^2 transforms (the other factored forms step alone)
  if (X.factored && (!X.fused_phi || !with_fused)) return std::string();
  if (X.hydro_kind != MixedState::kHydroPacked && X.hydro_kind != MixedState::kHydroTile) return std::string();
  char b[160];
  snprintf(b, sizeof b, "%d:%d:%d:%d:%d:%d:%d,%d,%d,%d", h->dev, X.Nu, X.Nphi, X.fused_phi ? 1 : 0, X.rows.gamma2,
           X.hydro_kind, X.ns[0], X.ns[1], X.ns[2], X.ns[5]);
  return std::string(b);
}

template <int MODE, bool A_MN, bool B_MN, bool PER_A>
static cudaError_t gemm_group(const CUtensorMap &Ch, const CUtensorMap &Cl, const tc::GemmDisk *d, int G, int M,
                              int N, int K, cudaStream_t st, int ns, bool prepare, bool persist = false,
                              int nsm = 148) {
  if (M % tc::BM || N % tc::BN || K % tc::BK) return cudaErrorInvalidValue;
  // 128 x 256 tiles where N allows (half the bytes of the shared operand per flop; two
  // pipeline stages), unless DISKGPU_GROUP_TILE=128
  static const bool wide_ok = [] {
    const char *v = getenv("DISKGPU_GROUP_TILE");
    return !(v && strcmp(v, "128") == 0);
  }();
  if (persist && N % 256 == 0 && wide_ok) {
    auto kp = tc::k_gemm_group_persist<MODE, A_MN, B_MN, PER_A, 256>;
    if (prepare) return smem_attrs((const void *)kp, tc::smem_persist(256));
    const int tn = N / 256, tm = M / tc::BM, nt = tn * tm * G;
    return launch_pdl(kp, dim3(nt < nsm ? nt : nsm), dim3(tc::threads_persist(tc::kEpiWarpsGroup)),
                      tc::smem_persist(256), st, Ch, Cl, d, tn, tm, nt);
  }
  if (persist && N % tc::BN2 == 0) {
    auto kp = tc::k_gemm_group_persist<MODE, A_MN, B_MN, PER_A>;
    if (prepare) return smem_attrs((const void *)kp, tc::kSmemP);
    const int tn = N / tc::BN2, tm = M / tc::BM, nt = tn * tm * G;
    return launch_pdl(kp, dim3(nt < nsm ? nt : nsm), dim3(tc::threads_persist(tc::kEpiWarpsGroup)), tc::kSmemP, st,
                      Ch, Cl, d, tn, tm, nt);
  }
  const int nk = K / tc::BK;
  if (ns == 0) ns = nk <= 1 ? 1 : (nk <= 2 ? 2 : tc::STAGES);
  const int NS = ns <= 1 ? 1 : (ns <= 2 ? 2 : tc::STAGES);
  auto k1 = tc::k_gemm_split_group<MODE, A_MN, B_MN, 1, PER_A>;
  auto k2 = tc::k_gemm_split_group<MODE, A_MN, B_MN, 2, PER_A>;
  auto k4 = tc::k_gemm_split_group<MODE, A_MN, B_MN, tc::STAGES, PER_A>;
  if (prepare) {
    const void *fn = NS == 1 ? (const void *)k1 : (NS == 2 ? (const void *)k2 : (const void *)k4);
    return smem_attrs(fn, tc::smem_bytes(NS));
  }
  dim3 grid(N / tc::BN, M / tc::BM, G);
  if (NS == 1) return launch_pdl(k1, grid, dim3(tc::kThreads), tc::smem_bytes(1), st, Ch, Cl, d);
  if (NS == 2) return launch_pdl(k2, grid, dim3(tc::kThreads), tc::smem_bytes(2), st, Ch, Cl, d);
  return launch_pdl(k4, grid, dim3(tc::kThreads), tc::smem_bytes(tc::STAGES), st, Ch, Cl, d);
}

// The group's kernels for one step, or (prepare) the shared-memory limits they need.
static int group_launch(MixedGroup *g, cudaStream_t st, bool prepare) {
  dg_handle *L = g->lead;
  MixedState &X = *L->mx;
  const int Nu = X.Nu, Nphi = X.Nphi, G = (int)g->disks.size();
  cudaError_t e;
  if (g->fused) {
    // phi transform -> Xin, u convolution (F1 F2 I1 I2) -> Zt, inverse phi transform -> dPhi
    if (prepare) {
      e = smem_attrs((const void *)tc::k_phifwd_group, tc::kPfSmem);
      if (e == cudaSuccess) e = smem_attrs((const void *)tc::k_uconv_group, tc::kUcSmem);
      if (e == cudaSuccess) e = smem_attrs((const void *)tc::k_phiinv_group, tc::kPiSmem);
      if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: fused transforms", cudaGetErrorString(e));
    } else {
      e = launch_pdl(tc::k_phifwd_group, dim3(Nu / tc::kPfRows, G), dim3(tc::kPfThreads), tc::kPfSmem, st,
                     X.mPA[0], X.mPA[1], X.mPB[0], X.mPB[1], (const tc::PhiFwdArgs *)g->pf);
      if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: phi transform", cudaGetErrorString(e));
      e = launch_pdl(tc::k_uconv_group, dim3(X.nm / tc::kUcModes, G), dim3(tc::kUcThreads), tc::kUcSmem, st,
                     X.mRB[0], X.mRB[1], X.mRA[0], X.mRA[1], X.mRGA[0], X.mRGA[1], X.mRGB[0], X.mRGB[1],
                     (const tc::UconvDisk *)g->uc);
      if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: u convolution", cudaGetErrorString(e));
      e = launch_pdl(tc::k_phiinv_group, dim3(Nu / tc::kPiRows, G), dim3(tc::kPiThreads), tc::kPiSmem, st,
                     X.mIA[0], X.mIA[1], X.mIB[0], X.mIB[1], (const tc::PhiInvArgs *)g->pi);
      if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: inverse phi transform", cudaGetErrorString(e));
    }
  }
  // G1: X1[c][i] = Fphi[c][:] . Sx[i][:];  G2: Wt[c][p] = KW[c][p] X1[c][:] . Cu[p][:];
  // G3: Z[i][c] = CuT[i][:] . Wt[c][:];    G4: dPhi[i][j] = phiscale[i] Z[i][:] . Gphi[j][:]
  if (!g->fused) e = gemm_group<tc::kEpiSplit, false, false, false>(X.mFphi[0], X.mFphi[1], g->gd[0], G, Nphi, Nu, Nphi, st, g->ns[0],
                                                       prepare, g->persist, g->nsm);
  if (!g->fused) {
  if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: phi DFT", cudaGetErrorString(e));
  e = gemm_group<tc::kEpiSplitScaled, false, false, true>(X.mCu[0], X.mCu[1], g->gd[1], G, Nphi, 2 * Nu, Nu, st,
                                                          g->ns[1], prepare, g->persist, g->nsm);
  if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: u DFT x khat", cudaGetErrorString(e));
  e = gemm_group<tc::kEpiSplit, false, false, false>(X.mCuT[0], X.mCuT[1], g->gd[2], G, Nu, Nphi, 2 * Nu, st,
                                                       g->ns[2], prepare, g->persist, g->nsm);
  if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: inverse u DFT", cudaGetErrorString(e));
  e = gemm_group<tc::kEpiRowScaleF32, false, false, true>(X.mGphi[0], X.mGphi[1], g->gd[3], G, Nu, Nphi, Nphi, st,
                                                          g->ns[5], prepare, g->persist, g->nsm);
  if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: inverse phi DFT", cudaGetErrorString(e));
  }
  const bool packed = g->kind == MixedState::kHydroPacked;
  auto hk = packed ? (g->g2 ? k_hydro32p_group<true> : k_hydro32p_group<false>)
                   : (g->g2 ? k_hydro32t_group<true> : k_hydro32t_group<false>);
  const size_t hsm = packed ? kSmem32p : kSmem32t;
  if (prepare) {
    e = smem_attrs((const void *)hk, hsm);
    if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: hydro", cudaGetErrorString(e));
    return DG_OK;
  }
  const int b = L->cur;
  const int tj = packed ? kTileJp : kTileJ;
  dim3 hgrid((Nphi + tj - 1) / tj, (Nu + kTileI - 1) / kTileI, G);
  e = launch_pdl(hk, hgrid, dim3(kThreads32t), hsm, st, (const HydroDisk *)g->hd, b);
  if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: hydro", cudaGetErrorString(e));
  e = launch_pdl(k_step_finalize_group, dim3(G), dim3(32), 0, st, (const HydroDisk *)g->hd);
  if (e != cudaSuccess) return L->fail(DG_ERR_CUDA, "batch group: finalisation", cudaGetErrorString(e));
  for (dg_handle *h : g->disks) h->cur ^= 1;
  return DG_OK;
}

void mixed_group_destroy(MixedGroup *g) {
  if (!g) return;
  for (tc::GemmDisk *p : g->gd)
    if (p) cudaFree(p);
  if (g->hd) cudaFree(g->hd);
  if (g->pf) cudaFree(g->pf);
  if (g->uc) cudaFree(g->uc);
  if (g->pi) cudaFree(g->pi);
  delete g;
}

template <class T>
static cudaError_t upload(T **dst, const std::vector<T> &v) {
  cudaError_t e = cudaMalloc(dst, sizeof(T) * v.size());
  return e == cudaSuccess ? cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) : e;
}

MixedGroup *mixed_group_create(const std::vector<dg_handle *> &disks, std::string *err) {
  if (disks.empty()) return nullptr;
  const std::string key = mixed_group_key(disks[0]);
  for (dg_handle *h : disks)
    if (key.empty() || mixed_group_key(h) != key || h->cur != disks[0]->cur) {
      *err = "batch group: disks differ in grid, Gamma class, hydro form or buffer parity";
      return nullptr;
    }
  MixedGroup *g = new MixedGroup();
  g->disks = disks;
  g->lead = disks[0];
  const MixedState &XL = *g->lead->mx;
  g->kind = XL.hydro_kind;
  g->g2 = XL.rows.gamma2 != 0;
  for (int k = 0; k < 6; ++k) g->ns[k] = XL.ns[k];
  {
    const char *gg = getenv("DISKGPU_GROUP_GEMM");
    g->persist = !(gg && strcmp(gg, "tile") == 0);
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, g->lead->dev) == cudaSuccess && nsm > 0)
      g->nsm = nsm;
  }
  g->fused = XL.fused_phi;
  const int G = (int)disks.size(), Nu = XL.Nu, Nphi = XL.Nphi;
  std::vector<tc::GemmDisk> gd[4];
  std::vector<HydroDisk> hd(G);
  std::vector<tc::PhiFwdArgs> pf;
  std::vector<tc::UconvDisk> uc;
  std::vector<tc::PhiInvArgs> pi;
  if (!g->fused)
    for (int q = 0; q < 4; ++q) gd[q].resize(G);
  for (int k = 0; k < G; ++k) {
    dg_handle *h = disks[k];
    MixedState &X = *h->mx;
    HydroDisk &d = hd[k];
    for (int b = 0; b < 2; ++b) {
      d.tmS[b] = X.mSig[b]; d.tmU[b] = X.mU[b]; d.tmW[b] = X.mW[b];
      d.sig[b] = X.sig[b]; d.u[b] = X.u[b]; d.w[b] = X.w[b];
    }
    d.tmP = X.mPhi;
    d.dPhi = X.dPhi;
    d.Sx = SplitBf16{X.Sx.hi, X.Sx.lo};
    d.ctl = h->ctl;
    d.g = X.rows;
    if (g->fused) {
      // the lone step's arguments without the row-tile hand-over (tables: the lead's)
      pf.push_back(tc::PhiFwdArgs{X.Sx.hi, X.Sx.lo, XL.twphi, X.Xin.hi, X.Xin.lo, X.nm * X.fa, Nphi,
                                  &h->ctl->status, nullptr});
      tc::UconvDisk u{};
      u.xh = X.mXin[0]; u.xl = X.mXin[1];
      u.a = tc::UconvArgs{XL.twp, X.khm, X.Z.hi, X.Z.lo, Nu, Nphi, &h->ctl->status, X.Zt.hi, X.Zt.lo};
      uc.push_back(u);
      pi.push_back(tc::PhiInvArgs{X.Zt.hi, X.Zt.lo, XL.twphi, X.phiscale, X.dPhi, Nphi, &h->ctl->status, nullptr,
                                  0, 0});
      continue;
    }
    tc::GemmArgs a{};
    a.status = &h->ctl->status;
    // G1: per-disk B = Sx -> X1
    a.M = Nphi; a.N = Nu; a.K = Nphi; a.out_hi = X.X1.hi; a.out_lo = X.X1.lo; a.ldo = Nu;
    gd[0][k].hi = X.mSx[0]; gd[0][k].lo = X.mSx[1]; gd[0][k].args = a;
    // G2: per-disk A = X1 -> Wt, x KW
    a.M = Nphi; a.N = 2 * Nu; a.K = Nu; a.out_hi = X.Wt.hi; a.out_lo = X.Wt.lo; a.ldo = 2 * Nu; a.table = X.KW;
    gd[1][k].hi = X.mX1[0]; gd[1][k].lo = X.mX1[1]; gd[1][k].args = a;
    // G3: per-disk B = Wt -> Z
    a.M = Nu; a.N = Nphi; a.K = 2 * Nu; a.out_hi = X.Z.hi; a.out_lo = X.Z.lo; a.ldo = Nphi; a.table = nullptr;
    gd[2][k].hi = X.mWt[0]; gd[2][k].lo = X.mWt[1]; gd[2][k].args = a;
    // G4: per-disk A = Z -> dPhi (FP32, scaled by -G du dphi / sqrt(R))
    a.M = Nu; a.N = Nphi; a.K = Nphi; a.out_hi = a.out_lo = nullptr; a.out_f32 = X.dPhi; a.ldo = Nphi;
    a.row_scale = X.phiscale;
    gd[3][k].hi = X.mZ[0]; gd[3][k].lo = X.mZ[1]; gd[3][k].args = a;
  }
  cudaError_t e = cudaSetDevice(g->lead->dev);
  if (g->fused) {
    if (e == cudaSuccess) e = upload(&g->pf, pf);
    if (e == cudaSuccess) e = upload(&g->uc, uc);
    if (e == cudaSuccess) e = upload(&g->pi, pi);
  }
  for (int q = 0; q < 4 && e == cudaSuccess && !g->fused; ++q) {
    e = cudaMalloc(&g->gd[q], sizeof(tc::GemmDisk) * G);
    if (e == cudaSuccess)
      e = cudaMemcpy(g->gd[q], gd[q].data(), sizeof(tc::GemmDisk) * G, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc(&g->hd, sizeof(HydroDisk) * G);
  if (e == cudaSuccess) e = cudaMemcpy(g->hd, hd.data(), sizeof(HydroDisk) * G, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    *err = std::string("batch group tables: ") + cudaGetErrorString(e);
    mixed_group_destroy(g);
    return nullptr;
  }
  if (group_launch(g, nullptr, true) != DG_OK) {
    *err = g->lead->err;
    mixed_group_destroy(g);
    return nullptr;
  }
  return g;
}

int mixed_group_enqueue_step(MixedGroup *g, cudaStream_t st) { return group_launch(g, st, false); }
