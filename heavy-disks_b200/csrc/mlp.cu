// Surrogate network: a small MLP (n_in -> width x depth SiLU -> n_out, linear head) with
// hand-written forward, backward and Adam kernels.  It maps sweep parameters (Q_min,
// M_d/M_*, softening/r, Gamma) to the hydro results (gamma, Omega_p, saturated |C2|/|C0|);
// it has no counterpart in the reference.
//
// Every product runs on the tensor cores through the split-BF16 tcgen05 GEMM of
// tc_gemm.cuh: weights are used in BF16 (one plane; FP32 master copies are what Adam
// updates), activations and back-propagated gradients are split into BF16 (hi, lo) pairs,
// accumulation is FP32 in TMEM.  Operands are padded with zeros to the GEMM's tiles: the
// batch to a multiple of 128 rows, the input features to 64, hidden and output features to
// multiples of 128.  The epilogues fuse the bias and SiLU (forward), the SiLU derivative
// (backward) and the bounded store of the weight gradients; per product:
//   forward   Z_l = A_{l-1} W_l^T + b_l, A_l = SiLU(Z_l)       (A_{l-1} K-major, W_l K-major)
//   dA        dZ_{l-1} = (dZ_l W_l) * SiLU'(Z_{l-1})           (dZ_l K-major, W_l MN-major)
//   dW        dW_l = dZ_l^T A_{l-1}                            (both MN-major, K = batch)
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "diskgpu.h"
#include "tc_gemm.cuh"

// mixed.cu: a K-major BF16 tensor map of a [rows][cols] matrix, 64-column boxes of box_rows rows
bool dg_bf16_tensor_map(CUtensorMap *m, const void *base, uint64_t rows, uint64_t cols, uint32_t box_rows);

namespace {

using dg::tc::GemmArgs;
namespace tc = dg::tc;

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

struct Split {
  __nv_bfloat16 *hi = nullptr, *lo = nullptr;
};

__device__ __forceinline__ void put_split(Split s, size_t k, float v) {
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  s.hi[k] = h;
  s.lo[k] = __float2bfloat16_rn(v - __bfloat162float(h));
}

// input rows -> split operand [rows][P], zero beyond n rows and n_in columns
__global__ void k_x_to_split(int n, int n_in, int P, int rows, const float *__restrict__ x, Split X) {
  const int cnt = rows * P;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    const int b = k / P, i = k - b * P;
    put_split(X, k, (b < n && i < n_in) ? x[(size_t)b * n_in + i] : 0.f);
  }
}

// dY = 2 (Y - T) / (n n_out) on [rows][P] (zero outside n x n_out), FP32 and split; loss
// partial sums of (Y - T)^2
__global__ void k_mse(int n, int n_out, int P, int rows, float inv, const float *__restrict__ Y,
                      const float *__restrict__ T, float *__restrict__ dYf, Split dY, float *__restrict__ loss) {
  __shared__ float red[256];
  float s = 0.f;
  const int cnt = rows * P;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    const int b = k / P, o = k - b * P;
    const float d = (b < n && o < n_out) ? Y[k] - T[(size_t)b * n_out + o] : 0.f;
    const float gk = 2.f * d * inv;
    dYf[k] = gk;
    put_split(dY, k, gk);
    s += d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] * inv);
}

// db[j] = sum_b dZ[b][j]  (one block per column, row stride ld)
__global__ void k_colsum(int B, int ld, const float *__restrict__ dZ, float *__restrict__ db) {
  __shared__ float red[256];
  const int j = blockIdx.x;
  float s = 0.f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) s += dZ[(size_t)b * ld + j];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[j] = red[0];
}

// Adam on the FP32 master parameters
__global__ void k_adam(int n, float lr, float b1, float b2, float c1, float c2, float eps, float *__restrict__ w,
                       const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    w[k] = w[k] - lr * (mk * c1) / (sqrtf(vk * c2) + eps);
  }
}

// the BF16 weights [Pfo][Pfi] and FP32 bias [Pfo] of one layer, zero-padded, from the master
__global__ void k_pack_layer(int fo, int fi, int Pfo, int Pfi, const float *__restrict__ w, const float *__restrict__ b,
                             __nv_bfloat16 *__restrict__ Wp, float *__restrict__ bp) {
  const int cnt = Pfo * Pfi;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    const int o = k / Pfi, i = k - o * Pfi;
    Wp[k] = __float2bfloat16_rn((o < fo && i < fi) ? w[(size_t)o * fi + i] : 0.f);
    if (i == 0) bp[o] = o < fo ? b[o] : 0.f;
  }
}

}  // namespace

struct dg_mlp {
  int n_in = 0, width = 0, depth = 0, n_out = 0, dev = -1;
  int nlayers = 0;                 // depth + 1 linear maps
  std::vector<int> fan_in, fan_out;
  std::vector<int> pin, pout;      // padded fan-in / fan-out of each layer
  std::vector<size_t> woff, boff;  // offsets into the flat parameter vector
  size_t nparams = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // FP32 master, grad, Adam moments
  // BF16 weights and FP32 biases used by the products, zero-padded, and a zero plane that
  // serves as the weights' "lo" half
  std::vector<__nv_bfloat16 *> Wp;
  std::vector<float *> bp;
  __nv_bfloat16 *zero = nullptr;
  int pz = 0;
  std::vector<CUtensorMap> mW;
  CUtensorMap mZero;
  // activations: cap rows (a multiple of 128)
  int cap = 0;
  float *Xf = nullptr, *Tt = nullptr, *Yf = nullptr, *dYf = nullptr, *loss = nullptr;
  int *status = nullptr;
  Split Xs, dYs;
  std::vector<float *> Z, dZf;
  std::vector<Split> A, dZs;
  // per split buffer: K-major maps (128-row boxes, A operands) and MN-major maps (64-row boxes)
  CUtensorMap mXk[2], mXmn[2], mdYk[2], mdYmn[2];
  std::vector<CUtensorMap> mAk, mAmn, mdZk, mdZmn;  // 2 per layer
  long long t = 0;  // Adam step
  cudaStream_t st = nullptr;
  std::string err;
  int fail(int code, const char *what, const char *why) {
    err = std::string(what) + ": " + (why ? why : "");
    return code;
  }
};

#define MK2(call)                                                                       \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) return mm->fail(DG_ERR_CUDA, #call, cudaGetErrorString(e_)); \
  } while (0)

static cudaError_t alloc_split(Split &s, size_t n) {
  cudaError_t e = cudaMalloc(&s.hi, n * sizeof(__nv_bfloat16));
  if (e == cudaSuccess) e = cudaMalloc(&s.lo, n * sizeof(__nv_bfloat16));
  if (e == cudaSuccess) e = cudaMemset(s.hi, 0, n * sizeof(__nv_bfloat16));
  if (e == cudaSuccess) e = cudaMemset(s.lo, 0, n * sizeof(__nv_bfloat16));
  return e;
}
static void free_split(Split &s) {
  if (s.hi) cudaFree(s.hi);
  if (s.lo) cudaFree(s.lo);
  s.hi = s.lo = nullptr;
}

static bool split_maps(const Split &s, int rows, int cols, CUtensorMap *k, CUtensorMap *mn) {
  return dg_bf16_tensor_map(&k[0], s.hi, rows, cols, tc::BM) && dg_bf16_tensor_map(&k[1], s.lo, rows, cols, tc::BM) &&
         dg_bf16_tensor_map(&mn[0], s.hi, rows, cols, 64) && dg_bf16_tensor_map(&mn[1], s.lo, rows, cols, 64);
}

static void free_acts(dg_mlp *mm) {
  for (float **p : {&mm->Xf, &mm->Tt, &mm->Yf, &mm->dYf})
    if (*p) {
      cudaFree(*p);
      *p = nullptr;
    }
  free_split(mm->Xs);
  free_split(mm->dYs);
  for (auto *vv : {&mm->Z, &mm->dZf})
    for (auto &p : *vv) {
      if (p) cudaFree(p);
      p = nullptr;
    }
  for (auto *vv : {&mm->A, &mm->dZs})
    for (auto &s : *vv) free_split(s);
  mm->cap = 0;
}

// activation buffers for at least n rows (rounded to the 128-row tiles)
static int ensure_cap(dg_mlp *mm, int n) {
  if (n <= mm->cap) return DG_OK;
  free_acts(mm);
  const int cap = round_up(n, tc::BM);
  const int Pin = mm->pin[0], Pw = round_up(mm->width, tc::BM), Pout = mm->pout[mm->nlayers - 1];
  MK2(cudaMalloc(&mm->Xf, sizeof(float) * cap * mm->n_in));
  MK2(cudaMalloc(&mm->Tt, sizeof(float) * cap * mm->n_out));
  MK2(cudaMalloc(&mm->Yf, sizeof(float) * cap * Pout));
  MK2(cudaMalloc(&mm->dYf, sizeof(float) * cap * Pout));
  MK2(alloc_split(mm->Xs, (size_t)cap * Pin));
  MK2(alloc_split(mm->dYs, (size_t)cap * Pout));
  bool ok = split_maps(mm->Xs, cap, Pin, mm->mXk, mm->mXmn) && split_maps(mm->dYs, cap, Pout, mm->mdYk, mm->mdYmn);
  mm->mAk.resize(2 * mm->depth); mm->mAmn.resize(2 * mm->depth);
  mm->mdZk.resize(2 * mm->depth); mm->mdZmn.resize(2 * mm->depth);
  for (int l = 0; l < mm->depth; ++l) {
    MK2(cudaMalloc(&mm->Z[l], sizeof(float) * cap * Pw));
    MK2(cudaMalloc(&mm->dZf[l], sizeof(float) * cap * Pw));
    MK2(alloc_split(mm->A[l], (size_t)cap * Pw));
    MK2(alloc_split(mm->dZs[l], (size_t)cap * Pw));
    ok = ok && split_maps(mm->A[l], cap, Pw, &mm->mAk[2 * l], &mm->mAmn[2 * l]) &&
         split_maps(mm->dZs[l], cap, Pw, &mm->mdZk[2 * l], &mm->mdZmn[2 * l]);
  }
  if (!ok) return mm->fail(DG_ERR_CUDA, "surrogate network", "tensor map encoding failed");
  mm->cap = cap;
  return DG_OK;
}

// one product of the network: D[M x N] = A[M x K] B[N x K]^T with the epilogue MODE
template <int MODE, bool A_MN, bool B_MN, int NS>
static cudaError_t product_ns(cudaStream_t st, const CUtensorMap *a2, const CUtensorMap &bh, const CUtensorMap &bl,
                              int M, int N, int K, const GemmArgs &args, bool prepare) {
  auto kern = tc::k_gemm_split<MODE, A_MN, B_MN, NS>;
  if (prepare) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::smem_bytes(NS));
  kern<<<dim3(N / tc::BN, M / tc::BM), tc::kThreads, tc::smem_bytes(NS), st>>>(a2[0], a2[1], bh, bl, args);
  return cudaGetLastError();
}

template <int MODE, bool A_MN, bool B_MN>
static cudaError_t product(cudaStream_t st, const CUtensorMap *a2, const CUtensorMap &bh, const CUtensorMap &bl, int M,
                           int N, int K, GemmArgs args, bool prepare = false) {
  if (!prepare && (M % tc::BM || N % tc::BN || K % tc::BK)) return cudaErrorInvalidValue;
  args.M = M; args.N = N; args.K = K;
  const int nk = K / tc::BK;
  if (prepare) {
    cudaError_t e = product_ns<MODE, A_MN, B_MN, 1>(st, a2, bh, bl, M, N, K, args, true);
    if (e == cudaSuccess) e = product_ns<MODE, A_MN, B_MN, 2>(st, a2, bh, bl, M, N, K, args, true);
    if (e == cudaSuccess) e = product_ns<MODE, A_MN, B_MN, tc::STAGES>(st, a2, bh, bl, M, N, K, args, true);
    return e;
  }
  if (nk <= 1) return product_ns<MODE, A_MN, B_MN, 1>(st, a2, bh, bl, M, N, K, args, false);
  if (nk <= 2) return product_ns<MODE, A_MN, B_MN, 2>(st, a2, bh, bl, M, N, K, args, false);
  return product_ns<MODE, A_MN, B_MN, tc::STAGES>(st, a2, bh, bl, M, N, K, args, false);
}

static int pack_weights(dg_mlp *mm) {
  for (int l = 0; l < mm->nlayers; ++l) {
    const int cnt = mm->pout[l] * mm->pin[l];
    k_pack_layer<<<(cnt + 255) / 256 < 512 ? (cnt + 255) / 256 : 512, 256, 0, mm->st>>>(
        mm->fan_out[l], mm->fan_in[l], mm->pout[l], mm->pin[l], mm->w + mm->woff[l], mm->w + mm->boff[l], mm->Wp[l],
        mm->bp[l]);
  }
  MK2(cudaGetLastError());
  return DG_OK;
}

// forward of n rows already in mm->Xf
static int forward(dg_mlp *mm, int n) {
  const int Bp = round_up(n, tc::BM);
  const int cnt = Bp * mm->pin[0];
  k_x_to_split<<<(cnt + 255) / 256 < 1024 ? (cnt + 255) / 256 : 1024, 256, 0, mm->st>>>(n, mm->n_in, mm->pin[0], Bp,
                                                                                          mm->Xf, mm->Xs);
  MK2(cudaGetLastError());
  const CUtensorMap *in = mm->mXk;
  for (int l = 0; l < mm->nlayers; ++l) {
    GemmArgs a{};
    a.status = mm->status;
    a.bias = mm->bp[l];
    if (l < mm->depth) {
      a.out_f32 = mm->Z[l]; a.out_hi = mm->A[l].hi; a.out_lo = mm->A[l].lo; a.ldo = mm->pout[l];
      MK2((product<tc::kEpiMlpAct, false, false>(mm->st, in, mm->mW[l], mm->mZero, Bp, mm->pout[l], mm->pin[l], a)));
      in = &mm->mAk[2 * l];
    } else {
      a.out_f32 = mm->Yf; a.ldo = mm->pout[l];
      MK2((product<tc::kEpiMlpOut, false, false>(mm->st, in, mm->mW[l], mm->mZero, Bp, mm->pout[l], mm->pin[l], a)));
    }
  }
  return DG_OK;
}

// backward from dY (FP32 and split, [Bp][Pout]): gradients into mm->g
static int backward(dg_mlp *mm, int n) {
  const int Bp = round_up(n, tc::BM);
  const CUtensorMap *dk = mm->mdYk, *dmn = mm->mdYmn;
  const float *df = mm->dYf;
  for (int l = mm->nlayers - 1; l >= 0; --l) {
    const int fo = mm->fan_out[l], fi = mm->fan_in[l];
    const CUtensorMap *inmn = (l == 0) ? mm->mXmn : &mm->mAmn[2 * (l - 1)];
    // dW[o][i] = sum_b dOut[b][o] in[b][i]
    GemmArgs a{};
    a.status = mm->status;
    a.out_f32 = mm->g + mm->woff[l]; a.ldo = fi; a.lim_m = fo; a.lim_n = fi;
    MK2((product<tc::kEpiStoreBounded, true, true>(mm->st, dmn, inmn[0], inmn[1], mm->pout[l], mm->pin[l], Bp, a)));
    k_colsum<<<fo, 256, 0, mm->st>>>(Bp, mm->pout[l], df, mm->g + mm->boff[l]);
    MK2(cudaGetLastError());
    if (l > 0) {
      // dZ_{l-1} = (dOut W_l) * SiLU'(Z_{l-1})
      GemmArgs b{};
      b.status = mm->status;
      b.out_f32 = mm->dZf[l - 1]; b.out_hi = mm->dZs[l - 1].hi; b.out_lo = mm->dZs[l - 1].lo;
      b.ldo = mm->pin[l]; b.table = mm->Z[l - 1];
      MK2((product<tc::kEpiMlpBack, false, true>(mm->st, dk, mm->mW[l], mm->mZero, Bp, mm->pin[l], mm->pout[l], b)));
      dk = &mm->mdZk[2 * (l - 1)];
      dmn = &mm->mdZmn[2 * (l - 1)];
      df = mm->dZf[l - 1];
    }
  }
  return DG_OK;
}

static int check_status(dg_mlp *mm) {
  int s = 0;
  MK2(cudaMemcpyAsync(&s, mm->status, sizeof(int), cudaMemcpyDeviceToHost, mm->st));
  MK2(cudaStreamSynchronize(mm->st));
  if (s) {
    cudaMemsetAsync(mm->status, 0, sizeof(int), mm->st);
    return mm->fail(DG_ERR_TIMEOUT, "surrogate network", "a bounded device wait gave up");
  }
  return DG_OK;
}

static int loss_and_grad(dg_mlp *mm, int n, const float *x, const float *tgt, float *loss_out) {
  int rc = ensure_cap(mm, n);
  if (rc) return rc;
  MK2(cudaMemcpyAsync(mm->Xf, x, sizeof(float) * n * mm->n_in, cudaMemcpyHostToDevice, mm->st));
  MK2(cudaMemcpyAsync(mm->Tt, tgt, sizeof(float) * n * mm->n_out, cudaMemcpyHostToDevice, mm->st));
  rc = forward(mm, n);
  if (rc) return rc;
  MK2(cudaMemsetAsync(mm->loss, 0, sizeof(float), mm->st));
  const int Bp = round_up(n, tc::BM), Pout = mm->pout[mm->nlayers - 1];
  const int cnt = Bp * Pout;
  k_mse<<<(cnt + 255) / 256 < 64 ? (cnt + 255) / 256 : 64, 256, 0, mm->st>>>(
      n, mm->n_out, Pout, Bp, 1.f / (n * mm->n_out), mm->Yf, mm->Tt, mm->dYf, mm->dYs, mm->loss);
  MK2(cudaGetLastError());
  rc = backward(mm, n);
  if (rc) return rc;
  if (loss_out) MK2(cudaMemcpyAsync(loss_out, mm->loss, sizeof(float), cudaMemcpyDeviceToHost, mm->st));
  return DG_OK;
}

extern "C" {

int dg_mlp_create(int n_in, int width, int depth, int n_out, unsigned long long seed, int device, dg_mlp **out) {
  if (!out || n_in < 1 || width < 1 || depth < 1 || n_out < 1) return DG_ERR_INVALID;
  *out = nullptr;
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return DG_ERR_CUDA;
  dg_mlp *mm = new (std::nothrow) dg_mlp();
  if (!mm) return DG_ERR_NOMEM;
  cudaGetDevice(&mm->dev);
  mm->n_in = n_in; mm->width = width; mm->depth = depth; mm->n_out = n_out;
  mm->nlayers = depth + 1;
  const int Pw = round_up(width, tc::BM);
  for (int l = 0; l < mm->nlayers; ++l) {
    mm->fan_in.push_back(l == 0 ? n_in : width);
    mm->fan_out.push_back(l == depth ? n_out : width);
    mm->pin.push_back(l == 0 ? round_up(n_in, tc::BK) : Pw);
    mm->pout.push_back(l == depth ? round_up(n_out, tc::BM) : Pw);
  }
  for (int l = 0; l < mm->nlayers; ++l) {
    mm->woff.push_back(mm->nparams);
    mm->nparams += (size_t)mm->fan_in[l] * mm->fan_out[l];
    mm->boff.push_back(mm->nparams);
    mm->nparams += mm->fan_out[l];
  }
  mm->Z.assign(depth, nullptr); mm->dZf.assign(depth, nullptr);
  mm->A.assign(depth, Split{}); mm->dZs.assign(depth, Split{});
  mm->Wp.assign(mm->nlayers, nullptr); mm->bp.assign(mm->nlayers, nullptr); mm->mW.resize(mm->nlayers);
  // He-style initialisation from a counter-based generator (splitmix64 + Box-Muller)
  std::vector<float> w(mm->nparams, 0.f);
  auto sm = [](unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
  };
  unsigned long long ctr = seed * 0x100000001B3ull;
  for (int l = 0; l < mm->nlayers; ++l) {
    const double sd = std::sqrt(2.0 / mm->fan_in[l]);
    const size_t cnt = (size_t)mm->fan_in[l] * mm->fan_out[l];
    for (size_t k = 0; k < cnt; ++k) {
      double u1 = ((sm(ctr++) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      double u2 = ((sm(ctr++) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      w[mm->woff[l] + k] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2));
    }
  }
  mm->pz = std::max(std::max(mm->pin[0], Pw), mm->pout[depth]);
  bool ok = cudaStreamCreateWithFlags(&mm->st, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&mm->w, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMalloc(&mm->g, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMalloc(&mm->m, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMalloc(&mm->v, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMalloc(&mm->loss, sizeof(float)) == cudaSuccess &&
            cudaMalloc(&mm->status, sizeof(int)) == cudaSuccess &&
            cudaMemset(mm->status, 0, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&mm->zero, sizeof(__nv_bfloat16) * mm->pz * mm->pz) == cudaSuccess &&
            cudaMemset(mm->zero, 0, sizeof(__nv_bfloat16) * mm->pz * mm->pz) == cudaSuccess &&
            dg_bf16_tensor_map(&mm->mZero, mm->zero, mm->pz, mm->pz, 64) &&
            cudaMemcpy(mm->w, w.data(), sizeof(float) * mm->nparams, cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemset(mm->m, 0, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMemset(mm->v, 0, sizeof(float) * mm->nparams) == cudaSuccess;
  for (int l = 0; ok && l < mm->nlayers; ++l)
    ok = cudaMalloc(&mm->Wp[l], sizeof(__nv_bfloat16) * mm->pout[l] * mm->pin[l]) == cudaSuccess &&
         cudaMalloc(&mm->bp[l], sizeof(float) * mm->pout[l]) == cudaSuccess &&
         dg_bf16_tensor_map(&mm->mW[l], mm->Wp[l], mm->pout[l], mm->pin[l], 64);
  // shared-memory limits of every product instantiation
  if (ok) {
    GemmArgs a{};
    CUtensorMap m2[2] = {mm->mZero, mm->mZero};
    ok = product<tc::kEpiMlpAct, false, false>(nullptr, m2, mm->mZero, mm->mZero, 0, 0, 0, a, true) == cudaSuccess &&
         product<tc::kEpiMlpOut, false, false>(nullptr, m2, mm->mZero, mm->mZero, 0, 0, 0, a, true) == cudaSuccess &&
         product<tc::kEpiMlpBack, false, true>(nullptr, m2, mm->mZero, mm->mZero, 0, 0, 0, a, true) == cudaSuccess &&
         product<tc::kEpiStoreBounded, true, true>(nullptr, m2, mm->mZero, mm->mZero, 0, 0, 0, a, true) == cudaSuccess;
  }
  if (ok) ok = pack_weights(mm) == DG_OK && cudaStreamSynchronize(mm->st) == cudaSuccess;
  if (!ok) {
    dg_mlp_destroy(mm);
    return DG_ERR_CUDA;
  }
  *out = mm;
  return DG_OK;
}

void dg_mlp_destroy(dg_mlp *mm) {
  if (!mm) return;
  cudaSetDevice(mm->dev);
  if (mm->st) cudaStreamSynchronize(mm->st);
  free_acts(mm);
  float *ps[] = {mm->w, mm->g, mm->m, mm->v, mm->loss};
  for (float *p : ps)
    if (p) cudaFree(p);
  if (mm->status) cudaFree(mm->status);
  if (mm->zero) cudaFree(mm->zero);
  for (auto *p : mm->Wp)
    if (p) cudaFree(p);
  for (auto *p : mm->bp)
    if (p) cudaFree(p);
  if (mm->st) cudaStreamDestroy(mm->st);
  delete mm;
}

const char *dg_mlp_last_error(const dg_mlp *mm) { return mm ? mm->err.c_str() : ""; }

long long dg_mlp_num_params(const dg_mlp *mm) { return mm ? (long long)mm->nparams : 0; }

int dg_mlp_get_params(dg_mlp *mm, float *params) {
  if (!mm || !params) return DG_ERR_INVALID;
  MK2(cudaSetDevice(mm->dev));
  MK2(cudaMemcpyAsync(params, mm->w, sizeof(float) * mm->nparams, cudaMemcpyDeviceToHost, mm->st));
  MK2(cudaStreamSynchronize(mm->st));
  return DG_OK;
}

int dg_mlp_set_params(dg_mlp *mm, const float *params) {
  if (!mm || !params) return DG_ERR_INVALID;
  MK2(cudaSetDevice(mm->dev));
  MK2(cudaMemcpyAsync(mm->w, params, sizeof(float) * mm->nparams, cudaMemcpyHostToDevice, mm->st));
  int rc = pack_weights(mm);
  if (rc) return rc;
  MK2(cudaMemsetAsync(mm->m, 0, sizeof(float) * mm->nparams, mm->st));
  MK2(cudaMemsetAsync(mm->v, 0, sizeof(float) * mm->nparams, mm->st));
  MK2(cudaStreamSynchronize(mm->st));
  mm->t = 0;
  return DG_OK;
}

int dg_mlp_forward(dg_mlp *mm, int n, const float *x, float *y) {
  if (!mm || n < 1 || !x || !y) return DG_ERR_INVALID;
  MK2(cudaSetDevice(mm->dev));
  int rc = ensure_cap(mm, n);
  if (rc) return rc;
  MK2(cudaMemcpyAsync(mm->Xf, x, sizeof(float) * n * mm->n_in, cudaMemcpyHostToDevice, mm->st));
  rc = forward(mm, n);
  if (rc) return rc;
  const int Pout = mm->pout[mm->nlayers - 1];
  MK2(cudaMemcpy2DAsync(y, sizeof(float) * mm->n_out, mm->Yf, sizeof(float) * Pout, sizeof(float) * mm->n_out, n,
                        cudaMemcpyDeviceToHost, mm->st));
  return check_status(mm);
}

int dg_mlp_loss_grad(dg_mlp *mm, int n, const float *x, const float *tgt, float *loss, float *grad) {
  if (!mm || n < 1 || !x || !tgt) return DG_ERR_INVALID;
  MK2(cudaSetDevice(mm->dev));
  int rc = loss_and_grad(mm, n, x, tgt, loss);
  if (rc) return rc;
  if (grad) MK2(cudaMemcpyAsync(grad, mm->g, sizeof(float) * mm->nparams, cudaMemcpyDeviceToHost, mm->st));
  return check_status(mm);
}

int dg_mlp_train_step(dg_mlp *mm, int n, const float *x, const float *tgt, float lr, float *loss) {
  if (!mm || n < 1 || !x || !tgt || !(lr > 0)) return DG_ERR_INVALID;
  MK2(cudaSetDevice(mm->dev));
  int rc = loss_and_grad(mm, n, x, tgt, loss);
  if (rc) return rc;
  mm->t += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f / (1.f - std::pow(b1, (float)mm->t)), c2 = 1.f / (1.f - std::pow(b2, (float)mm->t));
  k_adam<<<256, 256, 0, mm->st>>>((int)mm->nparams, lr, b1, b2, c1, c2, 1e-8f, mm->w, mm->g, mm->m, mm->v);
  MK2(cudaGetLastError());
  rc = pack_weights(mm);
  if (rc) return rc;
  return check_status(mm);
}

}  // extern "C"
