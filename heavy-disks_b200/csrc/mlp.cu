// Surrogate network: a small MLP (n_in -> width x depth SiLU -> n_out, linear head) with
// hand-written forward, backward and Adam kernels.  Weights are used in BF16 for every
// product (FP32 master copies are what Adam updates), activations and accumulation are
// FP32.  It maps sweep parameters (Q_min, M_d/M_*, softening/r, Gamma) to the hydro
// results (gamma, Omega_p, saturated |C2|/|C0|); it has no counterpart in the reference.
//
// One tiled kernel serves every product: C[M x N] = sum_k A(m, k) B(k, n) with A, B read
// through element strides (so X W^T, dZ W and dZ^T A are the same kernel), 64 x 64 tiles,
// 4 x 4 outputs per thread, and a fused epilogue (bias + SiLU, or plain store).
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "diskgpu.h"

namespace {

constexpr int kT = 64, kBK = 16;

enum MlpEpi : int { kEpiStore = 0, kEpiBiasSilu = 1, kEpiBias = 2 };

__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.f / (1.f + __expf(-z));
  return s * (1.f + z * (1.f - s));
}

template <typename TB> __device__ __forceinline__ float tofloat(TB x);
template <> __device__ __forceinline__ float tofloat<float>(float x) { return x; }
template <> __device__ __forceinline__ float tofloat<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }

template <typename TB, int EPI>
__global__ void __launch_bounds__(256) k_mlp_gemm(int M, int N, int K, const float *__restrict__ A, long sam, long sak,
                                                  const TB *__restrict__ B, long sbk, long sbn,
                                                  const float *__restrict__ bias, float *__restrict__ C,
                                                  float *__restrict__ C2, int ldc) {
  __shared__ float As[kBK][kT + 1], Bs[kBK][kT + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * kT, n0 = blockIdx.x * kT;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kBK) {
    for (int t = threadIdx.x; t < kBK * kT; t += 256) {
      const int kk = t / kT, mm = t % kT;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? A[m * sam + k * sak] : 0.f;
      const int n = n0 + mm;
      Bs[kk][mm] = (n < N && k < K) ? tofloat<TB>(B[k * sbk + n * sbn]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float v = acc[i][j];
      if (EPI != kEpiStore) v += bias[n];
      C[(long)m * ldc + n] = v;
      if (EPI == kEpiBiasSilu) C2[(long)m * ldc + n] = silu(v);
    }
  }
}

// dZ = dA * SiLU'(Z)
__global__ void k_silu_back(int n, const float *__restrict__ dA, const float *__restrict__ Z, float *__restrict__ dZ) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) dZ[k] = dA[k] * silu_grad(Z[k]);
}

// db[j] = sum_b dZ[b][j]  (one block per column)
__global__ void k_colsum(int B, int N, const float *__restrict__ dZ, float *__restrict__ db) {
  __shared__ float red[256];
  const int j = blockIdx.x;
  float s = 0.f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) s += dZ[(long)b * N + j];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[j] = red[0];
}

// dY = 2 (Y - T) / (B n_out); loss partial sums of (Y - T)^2
__global__ void k_mse(int n, float inv, const float *__restrict__ Y, const float *__restrict__ T, float *__restrict__ dY,
                      float *__restrict__ loss) {
  __shared__ float red[256];
  float s = 0.f;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float d = Y[k] - T[k];
    dY[k] = 2.f * d * inv;
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

// Adam on the FP32 master parameters, then refresh their BF16 copies
__global__ void k_adam(int n, float lr, float b1, float b2, float c1, float c2, float eps, float *__restrict__ w,
                       const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       __nv_bfloat16 *__restrict__ wb) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    const float wk = w[k] - lr * (mk * c1) / (sqrtf(vk * c2) + eps);
    w[k] = wk;
    wb[k] = __float2bfloat16_rn(wk);
  }
}

__global__ void k_to_bf16(int n, const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) wb[k] = __float2bfloat16_rn(w[k]);
}

}  // namespace

struct dg_mlp {
  int n_in = 0, width = 0, depth = 0, n_out = 0, dev = -1;
  int nlayers = 0;                 // depth + 1 linear maps
  std::vector<int> fan_in, fan_out;
  std::vector<size_t> woff, boff;  // offsets into the flat parameter vector
  size_t nparams = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // FP32 master, grad, Adam moments
  __nv_bfloat16 *wb = nullptr;     // BF16 weights used by every product
  // activations (capacity cap rows)
  int cap = 0;
  float *X = nullptr, *Tt = nullptr, *Y = nullptr, *dY = nullptr, *loss = nullptr;
  std::vector<float *> Z, Aact, dA, dZ;
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

static int ensure_cap(dg_mlp *mm, int n) {
  if (n <= mm->cap) return DG_OK;
  auto fr = [](float *&p) {
    if (p) cudaFree(p);
    p = nullptr;
  };
  fr(mm->X); fr(mm->Tt); fr(mm->Y); fr(mm->dY);
  for (auto *vv : {&mm->Z, &mm->Aact, &mm->dA, &mm->dZ})
    for (auto &p : *vv) fr(p);
  const int cap = n;
  MK2(cudaMalloc(&mm->X, sizeof(float) * cap * mm->n_in));
  MK2(cudaMalloc(&mm->Tt, sizeof(float) * cap * mm->n_out));
  MK2(cudaMalloc(&mm->Y, sizeof(float) * cap * mm->n_out));
  MK2(cudaMalloc(&mm->dY, sizeof(float) * cap * mm->n_out));
  for (int l = 0; l < mm->depth; ++l) {
    MK2(cudaMalloc(&mm->Z[l], sizeof(float) * cap * mm->width));
    MK2(cudaMalloc(&mm->Aact[l], sizeof(float) * cap * mm->width));
    MK2(cudaMalloc(&mm->dA[l], sizeof(float) * cap * mm->width));
    MK2(cudaMalloc(&mm->dZ[l], sizeof(float) * cap * mm->width));
  }
  mm->cap = cap;
  return DG_OK;
}

template <typename TB, int EPI>
static cudaError_t gemm(cudaStream_t st, int M, int N, int K, const float *A, long sam, long sak, const TB *B, long sbk,
                        long sbn, const float *bias, float *C, float *C2, int ldc) {
  dim3 grid((N + kT - 1) / kT, (M + kT - 1) / kT);
  k_mlp_gemm<TB, EPI><<<grid, 256, 0, st>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, C, C2, ldc);
  return cudaGetLastError();
}

// forward of n rows already in mm->X
static int forward(dg_mlp *mm, int n) {
  const float *in = mm->X;
  int fin = mm->n_in;
  for (int l = 0; l < mm->nlayers; ++l) {
    const __nv_bfloat16 *W = mm->wb + mm->woff[l];
    const float *b = mm->w + mm->boff[l];
    const int fo = mm->fan_out[l];
    if (l < mm->depth) {
      // Z = in W^T + b, A = SiLU(Z): A(m,k) = in[m*fin + k], B(k,n) = W[n*fin + k]
      MK2((gemm<__nv_bfloat16, kEpiBiasSilu>(mm->st, n, fo, fin, in, fin, 1, W, 1, fin, b, mm->Z[l], mm->Aact[l], fo)));
      in = mm->Aact[l];
      fin = fo;
    } else {
      MK2((gemm<__nv_bfloat16, kEpiBias>(mm->st, n, fo, fin, in, fin, 1, W, 1, fin, b, mm->Y, nullptr, fo)));
    }
  }
  return DG_OK;
}

// backward from mm->dY: gradients into mm->g
static int backward(dg_mlp *mm, int n) {
  const float *dOut = mm->dY;
  for (int l = mm->nlayers - 1; l >= 0; --l) {
    const int fo = mm->fan_out[l], fi = mm->fan_in[l];
    const float *inAct = (l == 0) ? mm->X : mm->Aact[l - 1];
    // dW[o][i] = sum_b dOut[b][o] in[b][i]: A(m=o, k=b) = dOut[b*fo + o], B(k=b, n=i) = in[b*fi + i]
    MK2((gemm<float, kEpiStore>(mm->st, fo, fi, n, dOut, 1, fo, inAct, fi, 1, nullptr, mm->g + mm->woff[l], nullptr, fi)));
    k_colsum<<<fo, 256, 0, mm->st>>>(n, fo, dOut, mm->g + mm->boff[l]);
    MK2(cudaGetLastError());
    if (l > 0) {
      // dA[b][i] = sum_o dOut[b][o] W[o][i]
      const __nv_bfloat16 *W = mm->wb + mm->woff[l];
      MK2((gemm<__nv_bfloat16, kEpiStore>(mm->st, n, fi, fo, dOut, fo, 1, W, fi, 1, nullptr, mm->dA[l - 1], nullptr, fi)));
      const int cnt = n * fi;
      k_silu_back<<<(cnt + 255) / 256, 256, 0, mm->st>>>(cnt, mm->dA[l - 1], mm->Z[l - 1], mm->dZ[l - 1]);
      MK2(cudaGetLastError());
      dOut = mm->dZ[l - 1];
    }
  }
  return DG_OK;
}

static int loss_and_grad(dg_mlp *mm, int n, const float *x, const float *tgt, float *loss_out) {
  int rc = ensure_cap(mm, n);
  if (rc) return rc;
  MK2(cudaMemcpyAsync(mm->X, x, sizeof(float) * n * mm->n_in, cudaMemcpyHostToDevice, mm->st));
  MK2(cudaMemcpyAsync(mm->Tt, tgt, sizeof(float) * n * mm->n_out, cudaMemcpyHostToDevice, mm->st));
  rc = forward(mm, n);
  if (rc) return rc;
  MK2(cudaMemsetAsync(mm->loss, 0, sizeof(float), mm->st));
  const int cnt = n * mm->n_out;
  k_mse<<<(cnt + 255) / 256 < 64 ? (cnt + 255) / 256 : 64, 256, 0, mm->st>>>(cnt, 1.f / cnt, mm->Y, mm->Tt, mm->dY,
                                                                               mm->loss);
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
  for (int l = 0; l < mm->nlayers; ++l) {
    mm->fan_in.push_back(l == 0 ? n_in : width);
    mm->fan_out.push_back(l == depth ? n_out : width);
  }
  for (int l = 0; l < mm->nlayers; ++l) {
    mm->woff.push_back(mm->nparams);
    mm->nparams += (size_t)mm->fan_in[l] * mm->fan_out[l];
    mm->boff.push_back(mm->nparams);
    mm->nparams += mm->fan_out[l];
  }
  mm->Z.assign(depth, nullptr); mm->Aact.assign(depth, nullptr); mm->dA.assign(depth, nullptr); mm->dZ.assign(depth, nullptr);
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
  bool ok = cudaStreamCreateWithFlags(&mm->st, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&mm->w, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMalloc(&mm->g, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMalloc(&mm->m, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMalloc(&mm->v, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMalloc(&mm->wb, sizeof(__nv_bfloat16) * mm->nparams) == cudaSuccess &&
            cudaMalloc(&mm->loss, sizeof(float)) == cudaSuccess &&
            cudaMemcpy(mm->w, w.data(), sizeof(float) * mm->nparams, cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemset(mm->m, 0, sizeof(float) * mm->nparams) == cudaSuccess &&
            cudaMemset(mm->v, 0, sizeof(float) * mm->nparams) == cudaSuccess;
  if (ok) {
    k_to_bf16<<<256, 256, 0, mm->st>>>((int)mm->nparams, mm->w, mm->wb);
    ok = cudaStreamSynchronize(mm->st) == cudaSuccess;
  }
  if (!ok) {
    delete mm;
    return DG_ERR_CUDA;
  }
  *out = mm;
  return DG_OK;
}

void dg_mlp_destroy(dg_mlp *mm) {
  if (!mm) return;
  cudaSetDevice(mm->dev);
  if (mm->st) cudaStreamSynchronize(mm->st);
  float *ps[] = {mm->w, mm->g, mm->m, mm->v, mm->loss, mm->X, mm->Tt, mm->Y, mm->dY};
  for (float *p : ps)
    if (p) cudaFree(p);
  for (auto *vv : {&mm->Z, &mm->Aact, &mm->dA, &mm->dZ})
    for (float *p : *vv)
      if (p) cudaFree(p);
  if (mm->wb) cudaFree(mm->wb);
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
  k_to_bf16<<<256, 256, 0, mm->st>>>((int)mm->nparams, mm->w, mm->wb);
  MK2(cudaGetLastError());
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
  MK2(cudaMemcpyAsync(mm->X, x, sizeof(float) * n * mm->n_in, cudaMemcpyHostToDevice, mm->st));
  rc = forward(mm, n);
  if (rc) return rc;
  MK2(cudaMemcpyAsync(y, mm->Y, sizeof(float) * n * mm->n_out, cudaMemcpyDeviceToHost, mm->st));
  MK2(cudaStreamSynchronize(mm->st));
  return DG_OK;
}

int dg_mlp_loss_grad(dg_mlp *mm, int n, const float *x, const float *tgt, float *loss, float *grad) {
  if (!mm || n < 1 || !x || !tgt) return DG_ERR_INVALID;
  MK2(cudaSetDevice(mm->dev));
  int rc = loss_and_grad(mm, n, x, tgt, loss);
  if (rc) return rc;
  if (grad) MK2(cudaMemcpyAsync(grad, mm->g, sizeof(float) * mm->nparams, cudaMemcpyDeviceToHost, mm->st));
  MK2(cudaStreamSynchronize(mm->st));
  return DG_OK;
}

int dg_mlp_train_step(dg_mlp *mm, int n, const float *x, const float *tgt, float lr, float *loss) {
  if (!mm || n < 1 || !x || !tgt || !(lr > 0)) return DG_ERR_INVALID;
  MK2(cudaSetDevice(mm->dev));
  int rc = loss_and_grad(mm, n, x, tgt, loss);
  if (rc) return rc;
  mm->t += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f / (1.f - std::pow(b1, (float)mm->t)), c2 = 1.f / (1.f - std::pow(b2, (float)mm->t));
  k_adam<<<256, 256, 0, mm->st>>>((int)mm->nparams, lr, b1, b2, c1, c2, 1e-8f, mm->w, mm->g, mm->m, mm->v, mm->wb);
  MK2(cudaGetLastError());
  MK2(cudaStreamSynchronize(mm->st));
  return DG_OK;
}

}  // extern "C"
