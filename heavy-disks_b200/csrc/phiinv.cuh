// Fused inverse phi transform of the split-BF16 gravity, Nphi = 1024 (= 32 x 32), from the
// radial convolution's output (uconv.cuh, Zt rows) to the FP32 potential the hydro step
// differentiates.
//
// For every radial row i the potential is the inverse real DFT of its phi spectrum,
//   Phi[j] = s_i Re sum_{m=0}^{N-1} X'[m] W^{-jm},  W = e^{-2 pi i / N},
// with X'[m] = (w_m / N) X[m] for m <= N/2 (w = 1 at m = 0 and N/2, else 2) and 0 above
// (kalnajs.hpp:48-63, the c2r over phi; s_i = -G du dphi / sqrt(R_i)).  The weights w_m / N
// are folded into the radial kernel table, so the Zt rows already hold X'.  With
// m = m2 + 32 m1 and j = j1 + 32 j2:
//   SA  Y[m2][j1] = sum_{m1} W_32^{-j1 m1} X'[m2 + 32 m1]               (complex, 32 points)
//   SB  Phi[j1 + 32 j2] = Re sum_{m2} W_32^{-j2 m2} (W^{-j1 m2} Y[m2][j1])  (real outputs)
// Both stages are tcgen05 split-BF16 products (A_hi B_hi + A_hi B_lo + A_lo B_hi, FP32 in
// TMEM).  One CTA takes 4 rows:
//   SA: D[(i, m2)][(j1, ro)] = X'[(i, m2)][(m1, ri)] . C[(j1, ro)][(m1, ri)], M = 128, N = 64,
//       K = 64; the Zt slice is the A operand, MN-major: per row pair, 64 K rows (m1, ri) of
//       64 contiguous (i, m2) entries; 32 bytes of one Zt row (8 modes as (re, im) pairs)
//       give the 16-byte pieces of K rows (m1, 0) and (m1, 1) by byte permutes (rows
//       m1 > 16 lie above N/2 and are zero);
//   EA: each TMEM lane (i, m2) holds Y[j1] in column pairs: twiddle W^{-j1 m2} and write
//       T[(j1, i)][(m2, ri)] K-major into swizzled shared memory;
//   SB: D[(j1, i)][j2] = T . B[j2][(m2, ri)], M = 128, N = 32, K = 64;
//   EB: Phi[i][j1 + 32 j2] = s_i D, FP32.
// 256 CTAs at Nu = 1024, 8 warps, 57 KB of shared memory, 128 TMEM columns.
#pragma once

#include "uconv.cuh"

namespace dg {
namespace tc {

constexpr int kPiRows = 4;         // radial rows per CTA
constexpr int kPiThreads = 256;
constexpr uint32_t kPiC = 0;       // stage-A operand C, 64 rows (j1, ro) x 64 K (m1, ri)           hi|lo 16 KB
constexpr uint32_t kPiX = 16384;   // Zt slice, MN-major: 2 chunks of 64 K rows x 128 B               hi|lo 32 KB
constexpr uint32_t kPiB = 49152;   // stage-B operand, 32 rows j2 x 64 K (m2, ri)                    hi|lo 8 KB
constexpr uint32_t kPiT = 0;       // T, 128 rows (j1, i) x 64 K (m2, ri), over C and X (dead after SA) hi|lo 32 KB
constexpr size_t kPiSmem = 57344 + 1024;
constexpr uint32_t kPiTmemCols = 128;

struct PhiInvArgs {
  const __nv_bfloat16 *zt_hi, *zt_lo;  // X' rows, [Nu][kZtLd]
  const float2 *twiddle;               // W^{m2 j1}, [32][32] (conjugated here)
  const float *row_scale;              // s_i
  float *phi;                          // [Nu][Nphi]
  int Nphi;
  int *status;
  // row-tile counters of the hydro step that follows (dg_common.cuh rowtile_*): CTA 0 sets
  // rowpend[0 .. rp_n) = rp_val once this kernel's predecessor has completed
  int *rowpend;
  int rp_n, rp_val;
};

__device__ __forceinline__ void phiinv_cta(const CUtensorMap *pCh, const CUtensorMap *pCl, const CUtensorMap *pBh, const CUtensorMap *pBl, const PhiInvArgs &a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *sm = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t bar_in, bar_mma;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3, hw = warp >> 2;
  const int i0 = blockIdx.x * kPiRows;
  if (threadIdx.x == 0) {
    mbar_init(&bar_in, 1);
    mbar_init(&bar_mma, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&tmem_slot, kPiTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16);
  bool in_seen = false;

  // EA: TMEM lane (i = q, m2 = lane), columns j1 in [16 hw, 16 hw + 16); W^{m2 j1} is
  // symmetric in (m2, j1), so the table row j1 serves
  float2 tw[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) tw[k] = __ldg(a.twiddle + (16 * hw + k) * 32 + lane);
  const float s_out = a.row_scale[i0 + (lane & 3)];  // EB: this lane's row

  if (threadIdx.x == 0) {  // constant operands: they do not depend on the previous kernel
    mbar_arrive_expect_tx(&bar_in, 16384 + 8192);
    tma_load_2d(sm + kPiC, pCh, &bar_in, 0, 0);
    tma_load_2d(sm + kPiC + 8192, pCl, &bar_in, 0, 0);
    tma_load_2d(sm + kPiB, pBh, &bar_in, 0, 0);
    tma_load_2d(sm + kPiB + 4096, pBl, &bar_in, 0, 0);
  }
  pdl_wait();  // Zt comes from the previous kernel; the potential's last reader (the hydro
               // step of the previous time step) completed before that kernel started
  pdl_trigger();
  if (a.rowpend && blockIdx.x == 0)
    for (int r = threadIdx.x; r < a.rp_n; r += blockDim.x) a.rowpend[r] = a.rp_val;
  // Zt slice: unit t of a plane = row pair ip, m1, 16-byte chunk c of the 128-byte K rows
  // (m1, 0) and (m1, 1), holding the real and the imaginary parts of
  // X'[i0 + 2 ip + c / 4][32 m1 + 8 (c % 4) .. + 7]: two 16-byte loads of (re, im) pairs
  {
    uint4 xv[8];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int t = threadIdx.x + kPiThreads * (r & 1), ip = t >> 8, m1 = (t >> 3) & 31, c = t & 7;
      xv[2 * r] = xv[2 * r + 1] = make_uint4(0u, 0u, 0u, 0u);
      if (m1 <= 16) {
        const uint4 *src = reinterpret_cast<const uint4 *>((r < 2 ? a.zt_hi : a.zt_lo) +
                                                           (size_t)(i0 + 2 * ip + (c >> 2)) * kZtLd +
                                                           2 * (32 * m1 + 8 * (c & 3)));
        xv[2 * r] = __ldcg(src);
        xv[2 * r + 1] = __ldcg(src + 1);
      }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int t = threadIdx.x + kPiThreads * (r & 1), ip = t >> 8, m1 = (t >> 3) & 31, c = t & 7;
      const uint4 p = xv[2 * r], u = xv[2 * r + 1];  // modes 8 (c % 4) + 0..3, + 4..7 as (re | im << 16)
      const uint4 re = make_uint4(__byte_perm(p.x, p.y, 0x5410), __byte_perm(p.z, p.w, 0x5410),
                                  __byte_perm(u.x, u.y, 0x5410), __byte_perm(u.z, u.w, 0x5410));
      const uint4 im = make_uint4(__byte_perm(p.x, p.y, 0x7632), __byte_perm(p.z, p.w, 0x7632),
                                  __byte_perm(u.x, u.y, 0x7632), __byte_perm(u.z, u.w, 0x7632));
      uint8_t *dst = sm + kPiX + (r < 2 ? 0 : 16384) + ip * 8192;
      *reinterpret_cast<uint4 *>(dst + sw128(2 * m1, c)) = re;
      *reinterpret_cast<uint4 *>(dst + sw128(2 * m1 + 1, c)) = im;
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  if (threadIdx.x == 0) {
    in_seen = mbar_wait(&bar_in, 0, a.status);
    if (in_seen) {
      tc_fence_after();
      // ---- SA: D[(i, m2)][(j1, ro)], TMEM columns 0..63 ----
      const uint32_t id = idesc_bf16(128, 64, true, false);
      const uint64_t ah = sdesc_mn_sw128(sm + kPiX, 8192), al = sdesc_mn_sw128(sm + kPiX + 16384, 8192);
      const uint64_t bh = sdesc_sw128(sm + kPiC), bl = sdesc_sw128(sm + kPiC + 8192);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) mma3(tmem, ah + 128 * kk, al + 128 * kk, bh + 2 * kk, bl + 2 * kk, id, kk == 0);
      mma_commit(&bar_mma);
    } else {
      abort_flag = 1;
    }
  }
  __syncwarp();
  bool ok = mbar_wait(&bar_mma, 0, a.status);
  tc_fence_after();

  // ---- EA: twiddle W^{-j1 m2}; T[(j1, i)][(m2, ri)] (row 4 j1 + i, K-major, swizzled) ----
  if (__all_sync(0xffffffffu, ok && !abort_flag)) {  // warp-uniform: tcgen05.ld is .sync.aligned
    uint32_t v[32];
    tmem_ld32(tl + (uint32_t)(32 * hw), v);  // columns (j1, ro), j1 = 16 hw .. 16 hw + 15
    const int il = q, m2 = lane;
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const float re = __uint_as_float(v[2 * t]), im = __uint_as_float(v[2 * t + 1]);
      const float c = tw[t].x, s = -tw[t].y;  // e^{+2 pi i j1 m2 / N}
      const float tr = re * c - im * s, ti = re * s + im * c;
      uint32_t hi, lo;
      split_pair(tr, ti, hi, lo);
      const uint32_t off = sw128(4 * (16 * hw + t) + il, m2 >> 2) + (uint32_t)(m2 & 3) * 4;
      *reinterpret_cast<uint32_t *>(sm + kPiT + off) = hi;
      *reinterpret_cast<uint32_t *>(sm + kPiT + 16384 + off) = lo;
    }
  } else {
    abort_flag = 1;
  }
  uc_stage_sync();

  // ---- SB: D[(j1, i)][j2], TMEM columns 64..95 ----
  if (threadIdx.x == 0 && !abort_flag) {
    const uint32_t id = idesc_bf16(128, 32);
    const uint64_t ah = sdesc_sw128(sm + kPiT), al = sdesc_sw128(sm + kPiT + 16384);
    const uint64_t bh = sdesc_sw128(sm + kPiB), bl = sdesc_sw128(sm + kPiB + 4096);
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) mma3(tmem + 64, ah + 2 * kk, al + 2 * kk, bh + 2 * kk, bl + 2 * kk, id, kk == 0);
    mma_commit(&bar_mma);
  }
  __syncwarp();
  ok = !abort_flag && mbar_wait(&bar_mma, 1, a.status);
  tc_fence_after();

  // ---- EB: Phi[i][j1 + 32 j2] = s_i D; lanes of one row and 8 consecutive j1 fill 32 bytes ----
  if (__all_sync(0xffffffffu, ok && !abort_flag)) {
    uint32_t v[16];
    tmem_ld16(tl + (uint32_t)(64 + 16 * hw), v);  // columns j2 = 16 hw .. 16 hw + 15
    const int rb = q * 32 + lane, j1 = rb >> 2, il = rb & 3;
    float *out = a.phi + (size_t)(i0 + il) * a.Nphi + j1;
#pragma unroll
    for (int t = 0; t < 16; ++t) out[32 * (16 * hw + t)] = s_out * __uint_as_float(v[t]);
  }
  if (threadIdx.x == 0 && !in_seen) mbar_wait(&bar_in, 0, a.status);  // copies in flight land first
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kPiTmemCols);
}

__global__ void __launch_bounds__(kPiThreads, 2)
    k_phiinv(const __grid_constant__ CUtensorMap tCh,
    const __grid_constant__ CUtensorMap tCl,
    const __grid_constant__ CUtensorMap tBh,
    const __grid_constant__ CUtensorMap tBl, PhiInvArgs a) {
  phiinv_cta(&tCh, &tCl, &tBh, &tBl, a);
}

// The same for a group of disks of one grid (batched sweeps): blockIdx.y is the disk, whose
// arguments come from a device array.
__global__ void __launch_bounds__(kPiThreads, 2)
    k_phiinv_group(const __grid_constant__ CUtensorMap tCh,
    const __grid_constant__ CUtensorMap tCl,
    const __grid_constant__ CUtensorMap tBh,
    const __grid_constant__ CUtensorMap tBl, const PhiInvArgs *__restrict__ disks) {
  phiinv_cta(&tCh, &tCl, &tBh, &tBl, disks[blockIdx.y]);
}

}  // namespace tc
}  // namespace dg
