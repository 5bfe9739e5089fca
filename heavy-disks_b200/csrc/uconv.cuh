// Fused u-direction convolution of the factored split-BF16 gravity, Nu = 1024.
//
// For every complex phi mode m the radial direction needs
//   y[i] = sum_p W_M^{-ip} (khat[m][p] / M) sum_i' W_M^{i'p} x[i'],   M = 2 Nu = 2048,
// with x zero beyond Nu (kalnajs.hpp:48-63: zero padding, r2c, x khat, c2r).  With
// i = i1 + 32 i2 and p = p2 + 64 p1 (i1, p1 < 32; i2 < 32 physical, p2 < 64) this is
//   S1  T[i1][p2] = W_M^{i1 p2} sum_{i2} W_64^{i2 p2} x[i1 + 32 i2]       (64-point stage)
//   S2  Y[p2][p1] = (khat / M) sum_{i1} W_32^{i1 p1} T[i1][p2]            (32-point stage)
//   S3  U[i1][p2] = W_M^{-i1 p2} sum_{p1} W_32^{-i1 p1} Y[p2][p1]
//   S4  y[i1 + 32 i2] = sum_{p2} W_64^{-i2 p2} U[i1][p2],  i2 < 32.
// Each stage is one tcgen05 split-BF16 product (A_hi B_hi + A_hi B_lo + A_lo B_hi, FP32
// in TMEM) against a constant real block of the complex twiddle matrix; the epilogue of
// one stage writes the next stage's operand straight into 128-byte-swizzled shared
// memory, so a CTA takes four modes from the phi spectrum to the potential spectrum
// without touching global memory in between.  One CTA per four modes (129 CTAs at
// Nphi = 1024), 8 warps: warp w drains TMEM lanes 32 (w % 4) .. +31, column half w / 4.
#pragma once

#include "tc_gemm.cuh"

namespace dg {
namespace tc {

constexpr int kUcModes = 4;      // complex phi modes per CTA
constexpr int kUcThreads = 256;  // 8 warps
// shared-memory plan, byte offsets from a 1024-aligned base; hi tile first, lo after it
constexpr uint32_t kUcRB = 0;        // W_64 block, rows (p2, ro) x K (i2, ri): 128 x 64     hi|lo 32 KB
constexpr uint32_t kUcX = 32768;     // input slice, K (i2, ri) x N (m, i1) MN-major: 2 chunks  hi|lo 32 KB
constexpr uint32_t kUcRA = 65536;    // W_32 block, rows (p1, ro) x K (i1, ri): 64 x 64       hi|lo 16 KB
constexpr uint32_t kUcRGA = 81920;   // conj W_32 block, rows (i1, ro) x K (p1, ri)           hi|lo 16 KB
constexpr uint32_t kUcRGB = 98304;   // conj W_64 block, rows (i2, ro) x K (p2, ri): 2 K blocks hi|lo 32 KB
constexpr uint32_t kUcT = 131072;    // T, rows (m, p2) x K (i1, ri): 256 x 64                hi|lo 64 KB
constexpr uint32_t kUcY = 0;         // Y, rows (m, p2) x K (p1, ri), over RB and X (dead after S1)
constexpr uint32_t kUcU = 131072;    // U, M (m, i1) x K (p2, ri) MN-major [kb][mc], over T (dead after S2)
constexpr uint32_t kUcTw = 196608;   // twiddles W_M^{p2 i1}, [64][kUcTwLd] float2 (padded rows)
constexpr int kUcTwLd = 33;          // odd row length in float2: the 64 rows fall on different banks
constexpr uint32_t kUcTwBytes = 64 * kUcTwLd * 8;  // 16896, a multiple of 16 (one bulk copy)
constexpr size_t kUcSmem = kUcTw + kUcTwBytes + 1024;
constexpr uint32_t kUcTmemCols = 256;
// Zt rows (the fused inverse phi transform's input): modes m = 0..543 as (re, im) BF16 pairs;
// entries above Nphi / 2 = 512 stay zero
constexpr int kZtModes = 544;
constexpr int kZtLd = 2 * kZtModes;

struct UconvArgs {
  const float2 *twiddle;  // W_M^{p2 i1}, [64][kUcTwLd] (columns 32.. unused)
  const float *khm;       // khat[m][p] / M (0 for padding modes), [nmodes][M]
  __nv_bfloat16 *z_hi, *z_lo;  // Z[c][i], Nphi x Nu (dense inverse phi transform)
  int Nu, Nphi;
  int *status;
  // when set: the output goes to Zt rows instead, [Nu][kZtLd] with mode m's (re, im) at
  // columns 2m, 2m + 1 (the fused inverse phi transform's input, phiinv.cuh; modes above
  // Nphi / 2 stay zero)
  __nv_bfloat16 *zt_hi, *zt_lo;
};

// byte offset of 16-byte chunk ch of row r in a 128-byte-swizzled tile
__device__ __forceinline__ uint32_t sw128(int r, int ch) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((ch ^ (r & 7)) << 4));
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// split a complex value into its hi and lo (re, im) BF16 words
// (one packed two-value conversion per plane; the same roundings as split_bf16 on each)
__device__ __forceinline__ void split_pair(float re, float im, uint32_t &hi, uint32_t &lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);  // .x (low half) = re
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(re - hf.x, im - hf.y);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}


__device__ __forceinline__ void mma3(uint32_t d, uint64_t ah, uint64_t al, uint64_t bh, uint64_t bl, uint32_t idesc,
                                     bool first) {
  mma_bf16(d, ah, bh, idesc, first ? 0u : 1u);
  mma_bf16(d, ah, bl, idesc, 1u);
  mma_bf16(d, al, bh, idesc, 1u);
}

// generic-proxy shared stores -> visible to the tensor core; TMEM reads ordered before the
// next MMA; then a CTA barrier
__device__ __forceinline__ void uc_stage_sync() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

__device__ __forceinline__ void uconv_cta(const CUtensorMap *pRBh, const CUtensorMap *pRBl, const CUtensorMap *pXh, const CUtensorMap *pXl, const CUtensorMap *pRAh, const CUtensorMap *pRAl, const CUtensorMap *pRGAh, const CUtensorMap *pRGAl, const CUtensorMap *pRGBh, const CUtensorMap *pRGBl, const UconvArgs &a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *sm = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t bar_in0, bar_in1, bar_mma;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3, hw = warp >> 2;
  if (threadIdx.x == 0) {
    mbar_init(&bar_in0, 1);
    mbar_init(&bar_in1, 1);
    mbar_init(&bar_mma, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&tmem_slot, kUcTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16);  // this warp's TMEM lane quarter
  bool in0_seen = false, in1_seen = false;
  // E2's rows (mode ml, p2) and its 32 kernel values khat[m][p2 + 64 p1] / M, loaded now so
  // that their latency hides behind the loads and the first two stages
  const int h = hw, r = q * 32 + lane, ml = 2 * h + (r >> 6), p2 = r & 63;
  float khv[32];
  {
    const float *kh = a.khm + (size_t)(blockIdx.x * kUcModes + ml) * 2048 + p2;
#pragma unroll
    for (int p1 = 0; p1 < 32; ++p1) khv[p1] = __ldg(kh + 64 * p1);
  }
  const float2 *tws = reinterpret_cast<const float2 *>(sm + kUcTw);

  if (threadIdx.x == 0) {
    // constant tables first: they do not depend on the previous kernel
    mbar_arrive_expect_tx(&bar_in0, 65536 + kUcTwBytes);
    bulk_load(sm + kUcTw, a.twiddle, kUcTwBytes, &bar_in0);
    tma_load_2d(sm + kUcRB, pRBh, &bar_in0, 0, 0);
    tma_load_2d(sm + kUcRB + 16384, pRBl, &bar_in0, 0, 0);
    mbar_arrive_expect_tx(&bar_in1, 65536);
    tma_load_2d(sm + kUcRA, pRAh, &bar_in1, 0, 0);
    tma_load_2d(sm + kUcRA + 8192, pRAl, &bar_in1, 0, 0);
    tma_load_2d(sm + kUcRGA, pRGAh, &bar_in1, 0, 0);
    tma_load_2d(sm + kUcRGA + 8192, pRGAl, &bar_in1, 0, 0);
    tma_load_2d(sm + kUcRGB, pRGBh, &bar_in1, 0, 0);
    tma_load_2d(sm + kUcRGB + 8192, pRGBh, &bar_in1, 64, 0);
    tma_load_2d(sm + kUcRGB + 16384, pRGBl, &bar_in1, 0, 0);
    tma_load_2d(sm + kUcRGB + 24576, pRGBl, &bar_in1, 64, 0);
    // the phi spectrum is the previous kernel's output
    pdl_wait();
    const int x0 = blockIdx.x * (kUcModes * 32);
    tma_load_2d(sm + kUcX, pXh, &bar_in0, x0, 0);
    tma_load_2d(sm + kUcX + 8192, pXh, &bar_in0, x0 + 64, 0);
    tma_load_2d(sm + kUcX + 16384, pXl, &bar_in0, x0, 0);
    tma_load_2d(sm + kUcX + 24576, pXl, &bar_in0, x0 + 64, 0);
    // ---- S1: D1[(m, i1)][(p2, ro)] at TMEM columns 0..127 (the input slice is the A
    // operand, MN-major, so every TMEM lane is one (mode, i1) and its (re, im) pairs sit
    // in adjacent columns) ----
    in0_seen = mbar_wait(&bar_in0, 0, a.status);
    if (in0_seen) {
      tc_fence_after();
      const uint32_t id = idesc_bf16(128, 128, true, false);
      const uint64_t ah = sdesc_mn_sw128(sm + kUcX, 8192), al = sdesc_mn_sw128(sm + kUcX + 16384, 8192);
      const uint64_t bh = sdesc_sw128(sm + kUcRB), bl = sdesc_sw128(sm + kUcRB + 16384);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) mma3(tmem, ah + 128 * kk, al + 128 * kk, bh + 2 * kk, bl + 2 * kk, id, kk == 0);
      mma_commit(&bar_mma);
    } else {
      abort_flag = 1;
    }
  }
  __syncwarp();
  pdl_wait();  // every thread: Z is read by the kernel after this one's predecessor
  pdl_trigger();
  bool ok = mbar_wait(&bar_mma, 0, a.status);
  tc_fence_after();

  // ---- E1: twiddle W_M^{i1 p2}; T[(m, p2)][(i1, ri)] ----
  ok = ok && !abort_flag && mbar_wait(&bar_in0, 0, a.status);  // the twiddles in shared memory, for every thread
  if (__all_sync(0xffffffffu, ok && !abort_flag)) {  // warp-uniform: tcgen05.ld is .sync.aligned
    // lane (m = q, i1 = lane); columns (p2, ro) for p2 in [32 hw, 32 hw + 32)
    const int i1 = lane;
#pragma unroll 1
    for (int c = 0; c < 2; ++c) {
      uint32_t v[32];
      tmem_ld32(tl + (uint32_t)(64 * hw + 32 * c), v);
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const int p2 = 32 * hw + 16 * c + t;
        const float re = __uint_as_float(v[2 * t]), im = __uint_as_float(v[2 * t + 1]);
        const float2 w = tws[p2 * kUcTwLd + i1];
        const float tr = re * w.x - im * w.y, ti = re * w.y + im * w.x;
        uint32_t hi, lo;
        split_pair(tr, ti, hi, lo);
        // row (m, p2) of T; the warp's 32 lanes fill its 128 bytes
        const uint32_t off = sw128(q * 64 + p2, i1 >> 2) + (uint32_t)(i1 & 3) * 4;
        *reinterpret_cast<uint32_t *>(sm + kUcT + off) = hi;
        *reinterpret_cast<uint32_t *>(sm + kUcT + 32768 + off) = lo;
      }
    }
  } else {
    abort_flag = 1;
  }
  uc_stage_sync();

  // ---- S2: D2[h][(m, p2)][(p1, ro)] at TMEM columns 128 + 64 h ----
  if (threadIdx.x == 0 && !abort_flag) {
    in1_seen = mbar_wait(&bar_in1, 0, a.status);
    if (in1_seen) {
      tc_fence_after();
      const uint32_t id = idesc_bf16(128, 64);
      const uint64_t bh = sdesc_sw128(sm + kUcRA), bl = sdesc_sw128(sm + kUcRA + 8192);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint64_t ah = sdesc_sw128(sm + kUcT + h * 16384), al = sdesc_sw128(sm + kUcT + 32768 + h * 16384);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
          mma3(tmem + 128 + 64 * h, ah + 2 * kk, al + 2 * kk, bh + 2 * kk, bl + 2 * kk, id, kk == 0);
      }
      mma_commit(&bar_mma);
    } else {
      abort_flag = 1;
    }
  }
  __syncwarp();
  ok = !abort_flag && mbar_wait(&bar_mma, 1, a.status);
  tc_fence_after();

  // ---- E2: x khat / M; Y[(m, p2)][(p1, ri)] ----
  if (__all_sync(0xffffffffu, ok && !abort_flag)) {  // warp-uniform: tcgen05.ld is .sync.aligned
    const int R = 128 * h + r;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      uint32_t v[32];
      tmem_ld32(tl + (uint32_t)(128 + 64 * h + 32 * c), v);
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        uint32_t ph[4], pl[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float s = khv[16 * c + 4 * g + e];  // p1 = 16 c + 4 g + e
          split_pair(__uint_as_float(v[8 * g + 2 * e]) * s, __uint_as_float(v[8 * g + 2 * e + 1]) * s, ph[e], pl[e]);
        }
        const uint32_t off = sw128(R, 4 * c + g);
        *reinterpret_cast<uint4 *>(sm + kUcY + off) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
        *reinterpret_cast<uint4 *>(sm + kUcY + 32768 + off) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
      }
    }
  } else {
    abort_flag = 1;
  }
  uc_stage_sync();

  // ---- S3: D3[h][(m, p2)][(i1, ro)] at TMEM columns 64 h ----
  if (threadIdx.x == 0 && !abort_flag) {
    const uint32_t id = idesc_bf16(128, 64);
    const uint64_t bh = sdesc_sw128(sm + kUcRGA), bl = sdesc_sw128(sm + kUcRGA + 8192);
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const uint64_t ah = sdesc_sw128(sm + kUcY + hh * 16384), al = sdesc_sw128(sm + kUcY + 32768 + hh * 16384);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mma3(tmem + 64 * hh, ah + 2 * kk, al + 2 * kk, bh + 2 * kk, bl + 2 * kk, id, kk == 0);
    }
    mma_commit(&bar_mma);
  }
  __syncwarp();
  ok = !abort_flag && mbar_wait(&bar_mma, 0, a.status);
  tc_fence_after();

  // ---- E3: conj twiddle; U[(m, i1)][(p2, ri)] MN-major, sub-tiles [kb = p2 / 32][mc = h] ----
  if (__all_sync(0xffffffffu, ok && !abort_flag)) {  // warp-uniform: tcgen05.ld is .sync.aligned
    const float2 *twr = tws + p2 * kUcTwLd;
    uint8_t *ub = sm + kUcU + (p2 >> 5) * 16384 + h * 8192;
#pragma unroll 1
    for (int c = 0; c < 2; ++c) {
      uint32_t v[32];
      tmem_ld32(tl + (uint32_t)(64 * h + 32 * c), v);
      float ur[16], ui[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const float re = __uint_as_float(v[2 * e]), im = __uint_as_float(v[2 * e + 1]);
        const float2 w = twr[16 * c + e];
        ur[e] = re * w.x + im * w.y;
        ui[e] = im * w.x - re * w.y;
      }
#pragma unroll
      for (int ri = 0; ri < 2; ++ri) {
        const int krow = (2 * p2 + ri) & 63;
#pragma unroll
        for (int g = 0; g < 2; ++g) {
          uint32_t ph[4], pl[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float x0 = ri ? ui[8 * g + 2 * e] : ur[8 * g + 2 * e];
            const float x1 = ri ? ui[8 * g + 2 * e + 1] : ur[8 * g + 2 * e + 1];
            split_pair(x0, x1, ph[e], pl[e]);
          }
          const uint32_t off = sw128(krow, 4 * (ml & 1) + 2 * c + g);
          *reinterpret_cast<uint4 *>(ub + off) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
          *reinterpret_cast<uint4 *>(ub + 32768 + off) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
        }
      }
    }
  } else {
    abort_flag = 1;
  }
  uc_stage_sync();

  // ---- S4: D4[(m, i1)][(i2, ro)] at TMEM columns 128 ----
  if (threadIdx.x == 0 && !abort_flag) {
    const uint32_t id = idesc_bf16(128, 64, true, false);
#pragma unroll
    for (int kb = 0; kb < 2; ++kb) {
      const uint64_t ah = sdesc_mn_sw128(sm + kUcU + kb * 16384, 8192);
      const uint64_t al = sdesc_mn_sw128(sm + kUcU + 32768 + kb * 16384, 8192);
      const uint64_t bh = sdesc_sw128(sm + kUcRGB + kb * 8192), bl = sdesc_sw128(sm + kUcRGB + 16384 + kb * 8192);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mma3(tmem + 128, ah + 128 * kk, al + 128 * kk, bh + 2 * kk, bl + 2 * kk, id, kb == 0 && kk == 0);
    }
    mma_commit(&bar_mma);
  }
  __syncwarp();
  ok = !abort_flag && mbar_wait(&bar_mma, 1, a.status);
  tc_fence_after();

  if (a.zt_hi) {
    // ---- E4 (fused inverse): Zt[i][2m, 2m + 1] for the CTA's four modes.  Each (mode, row)
    // value goes to shared memory as one word per plane, (re | im << 16), at slot
    // mode ^ ((i >> 3) & 3) of the row's 16 bytes (the XOR keeps a warp's 32 rows on
    // distinct banks); then one thread per row writes the row's 16 bytes per plane.  The
    // staging area is U's (dead after S4). ----
    uint32_t *stg = reinterpret_cast<uint32_t *>(sm + kUcU);  // [Nu][4] hi, then [Nu][4] lo
    const int half = a.Nphi / 2;
    if (__all_sync(0xffffffffu, ok && !abort_flag)) {
      uint32_t v[32];
      tmem_ld32(tl + (uint32_t)(128 + 32 * hw), v);  // columns (i2, ro), i2 = 16 hw + t / 2
      const int m = blockIdx.x * kUcModes + q;
      const bool live = m <= half, has_im = live && m != 0 && m != half;
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const int ii = lane + 32 * (16 * hw + t);
        uint32_t hi, lo;
        split_pair(live ? __uint_as_float(v[2 * t]) : 0.f, has_im ? __uint_as_float(v[2 * t + 1]) : 0.f, hi, lo);
        const int slot = q ^ ((ii >> 3) & 3);
        stg[ii * 4 + slot] = hi;
        stg[4 * a.Nu + ii * 4 + slot] = lo;
      }
    }
    __syncthreads();
    if (!abort_flag) {
      const int m0 = blockIdx.x * kUcModes;
      const int s = (threadIdx.x >> 3) & 3;  // rows threadIdx.x + 256 k share (i >> 3) & 3
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int ii = threadIdx.x + kUcThreads * k;
#pragma unroll
        for (int pl = 0; pl < 2; ++pl) {
          const uint4 w = *reinterpret_cast<const uint4 *>(stg + pl * 4 * a.Nu + ii * 4);
          auto pick = [&](int idx) { return idx == 0 ? w.x : (idx == 1 ? w.y : (idx == 2 ? w.z : w.w)); };
          // modes m0 .. m0+3 in order
          __nv_bfloat16 *row = (pl ? a.zt_lo : a.zt_hi) + (size_t)ii * kZtLd;
          *reinterpret_cast<uint4 *>(row + 2 * m0) = make_uint4(pick(s), pick(1 ^ s), pick(2 ^ s), pick(3 ^ s));
        }
      }
    }
  } else if (__all_sync(0xffffffffu, ok && !abort_flag)) {  // warp-uniform: tcgen05.ld is .sync.aligned
    // ---- E4: Z[c(m, ro)][i1 + 32 i2] ----
    uint32_t v[32];
    tmem_ld32(tl + (uint32_t)(128 + 32 * hw), v);  // columns (i2, ro), i2 = 16 hw + t / 2
    const int m = blockIdx.x * kUcModes + q, i1 = lane;
    const int half = a.Nphi / 2;
    if (m <= half) {
      const int cre = (m == 0) ? 0 : (m == half ? 1 : 2 * m);
      const int cim = (m == 0 || m == half) ? -1 : 2 * m + 1;  // self-conjugate modes have no imaginary row
      const size_t Nu = (size_t)a.Nu;
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const size_t ii = (size_t)i1 + 32 * (size_t)(16 * hw + t);
        __nv_bfloat16 hh, ll;
        split_bf16(__uint_as_float(v[2 * t]), hh, ll);
        a.z_hi[(size_t)cre * Nu + ii] = hh;
        a.z_lo[(size_t)cre * Nu + ii] = ll;
        if (cim >= 0) {
          split_bf16(__uint_as_float(v[2 * t + 1]), hh, ll);
          a.z_hi[(size_t)cim * Nu + ii] = hh;
          a.z_lo[(size_t)cim * Nu + ii] = ll;
        }
      }
    }
  }
  // every issued copy must have landed before the CTA exits (bounded waits)
  if (threadIdx.x == 0) {
    if (!in0_seen) mbar_wait(&bar_in0, 0, a.status);
    if (!in1_seen) mbar_wait(&bar_in1, 0, a.status);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kUcTmemCols);
}

__global__ void __launch_bounds__(kUcThreads, 1)
    k_uconv(const __grid_constant__ CUtensorMap tRBh,
    const __grid_constant__ CUtensorMap tRBl,
    const __grid_constant__ CUtensorMap tXh,
    const __grid_constant__ CUtensorMap tXl,
    const __grid_constant__ CUtensorMap tRAh,
    const __grid_constant__ CUtensorMap tRAl,
    const __grid_constant__ CUtensorMap tRGAh,
    const __grid_constant__ CUtensorMap tRGAl,
    const __grid_constant__ CUtensorMap tRGBh,
    const __grid_constant__ CUtensorMap tRGBl, UconvArgs a) {
  uconv_cta(&tRBh, &tRBl, &tXh, &tXl, &tRAh, &tRAl, &tRGAh, &tRGAl, &tRGBh, &tRGBl, a);
}

// The same for a group of disks of one grid (batched sweeps): blockIdx.y is the disk; its
// own operand maps sit with its arguments in a device array.
struct __align__(64) UconvDisk {
  CUtensorMap xh, xl;  // the disk's input slice Xin (hi / lo)
  UconvArgs a;
};

__global__ void __launch_bounds__(kUcThreads, 1)
    k_uconv_group(const __grid_constant__ CUtensorMap tRBh,
    const __grid_constant__ CUtensorMap tRBl,
    const __grid_constant__ CUtensorMap tRAh,
    const __grid_constant__ CUtensorMap tRAl,
    const __grid_constant__ CUtensorMap tRGAh,
    const __grid_constant__ CUtensorMap tRGAl,
    const __grid_constant__ CUtensorMap tRGBh,
    const __grid_constant__ CUtensorMap tRGBl, const UconvDisk *__restrict__ disks) {
  const UconvDisk &d = disks[blockIdx.y];
  uconv_cta(&tRBh, &tRBl, &d.xh, &d.xl, &tRAh, &tRAl, &tRGAh, &tRGAl, &tRGBh, &tRGBl, d.a);
}

}  // namespace tc
}  // namespace dg
