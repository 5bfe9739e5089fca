// Fused forward phi transform of the split-BF16 gravity, Nphi = 1024 (= 32 x 32), written
// straight into the operand layout of the fused radial convolution (uconv.cuh).
//
// For every radial row i the phi spectrum of the real source x[j] = R^{3/2} sigma is
//   X[m] = sum_j x[j] W^{jm},  W = e^{-2 pi i / 1024},  m = 0 .. 512
// (kalnajs.hpp:48-63, the r2c over phi).  With j = j1 + 32 j2 and m = m2 + 32 m1:
//   SA  Y[j1][m2] = sum_{j2} W_32^{j2 m2} x[j1 + 32 j2]          (real input, 32 points)
//   SB  X[m2 + 32 m1] = sum_{j1} W_32^{j1 m1} (W^{j1 m2} Y[j1][m2])   (complex, 32 points)
// Both stages are tcgen05 split-BF16 products (A_hi B_hi + A_hi B_lo + A_lo B_hi, FP32 in
// TMEM).  One CTA takes 4 rows:
//   SA: D[(i, j1)][(m2, ro)] = x[(i, j1)][j2] . C[(m2, ro)][j2], M = 128, N = 64, K = 32;
//       every thread copies 16-byte runs of x (8 consecutive j1 of one row and one j2) into
//       the swizzled MN-major layout: per row pair, 32 K rows (j2) of 64 contiguous (i, j1)
//       entries;
//   EA: each TMEM lane (i, j1) holds its complex Y[m2] in column pairs: twiddle W^{j1 m2}
//       and write T[(m2, i)][(j1, ri)] K-major into swizzled shared memory (a warp, one i,
//       fills 128 contiguous bytes of a row);
//   SB: D[(m2, i)][(m1, ro)] = T . B[(m1, ro)][(j1, ri)], M = 128, N = 64, K = 64;
//   EB: X[m][i] for m <= 512 -> Xin[(i2, ri)][(m, i1)] (i = i1 + 32 i2), BF16 hi / lo.
// 256 CTAs at Nu = 1024, 8 warps, 48 KB of shared memory, 128 TMEM columns.
#pragma once

#include "uconv.cuh"

namespace dg {
namespace tc {

constexpr int kPfRows = 4;        // radial rows per CTA
constexpr int kPfHydroRows = 16;  // rows of a hydro tile (the unit of the row-tile counters)
constexpr int kPfThreads = 256;
constexpr uint32_t kPfC = 0;      // stage-A operand C, 64 rows (m2, ro) x 64 K (j2 < 32 used) hi|lo 16 KB
constexpr uint32_t kPfX = 16384;  // x slice, MN-major: 2 chunks of 32 K rows x 128 B          hi|lo 16 KB
constexpr uint32_t kPfB = 32768;  // stage-B operand, 64 rows (m1, ro) x 64 K (j1, ri)          hi|lo 16 KB
constexpr uint32_t kPfT = 0;      // T, 128 rows (m2, i) x 64 K (j1, ri), over C and x (dead after SA) hi|lo 32 KB
constexpr size_t kPfSmem = 49152 + 1024;
constexpr uint32_t kPfTmemCols = 128;

struct PhiFwdArgs {
  const __nv_bfloat16 *sx_hi, *sx_lo;  // R^{3/2} sigma, [Nu][Nphi]
  const float2 *twiddle;  // W^{m2 j1}, [32][32]
  __nv_bfloat16 *xin_hi, *xin_lo;  // Xin[(i2, ri)][(m, i1)], row length ld
  int ld;                 // nmodes * 32
  int Nphi;
  int *status;
  // hydro row-tile counters (dg_common.cuh rowtile_*): when set, this CTA waits for the
  // 16-row tile row holding its rows instead of for the whole previous kernel
  const int *rowpend;
};

__device__ __forceinline__ void phifwd_cta(const CUtensorMap *pCh, const CUtensorMap *pCl, const CUtensorMap *pBh, const CUtensorMap *pBl, const PhiFwdArgs &a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *sm = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t bar_in, bar_mma;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3, hw = warp >> 2;
  const int i0 = blockIdx.x * kPfRows;
  if (threadIdx.x == 0) {
    mbar_init(&bar_in, 1);
    mbar_init(&bar_mma, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&tmem_slot, kPfTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16);
  bool in_seen = false;

  // EA: TMEM lane (i = q, j1 = lane), columns m2 in [16 hw, 16 hw + 16); their twiddles
  // W^{j1 m2} are loaded now
  float2 tw[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) tw[k] = __ldg(a.twiddle + (16 * hw + k) * 32 + lane);

  if (threadIdx.x == 0) {  // constant operands: they do not depend on the previous kernel
    mbar_arrive_expect_tx(&bar_in, 32768);
    tma_load_2d(sm + kPfC, pCh, &bar_in, 0, 0);
    tma_load_2d(sm + kPfC + 8192, pCl, &bar_in, 0, 0);
    tma_load_2d(sm + kPfB, pBh, &bar_in, 0, 0);
    tma_load_2d(sm + kPfB + 8192, pBl, &bar_in, 0, 0);
  }
  // the source comes from the hydro step before this kernel (Xin's last reader, the u
  // convolution of the previous step, completed before that hydro step started)
  if (a.rowpend) {
    if (threadIdx.x == 0) rowtile_wait(a.rowpend + i0 / kPfHydroRows, a.status);
    __syncthreads();
  } else {
    pdl_wait();
  }
  pdl_trigger();
  // x slice: chunk t of a plane = row pair ip, K row j2, 16-byte chunk c of the 128-byte row,
  // holding x[i0 + 2 ip + c / 4][32 j2 + 8 (c % 4) .. + 7]
  {
    uint4 xv[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int t = threadIdx.x + kPfThreads * (r & 1), ip = t >> 8, j2 = (t >> 3) & 31, c = t & 7;
      const size_t g = (size_t)(i0 + 2 * ip + (c >> 2)) * a.Nphi + 32 * j2 + 8 * (c & 3);
      xv[r] = __ldcg(reinterpret_cast<const uint4 *>((r < 2 ? a.sx_hi : a.sx_lo) + g));  // L2: fresh after the wait
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int t = threadIdx.x + kPfThreads * (r & 1), ip = t >> 8, j2 = (t >> 3) & 31, c = t & 7;
      *reinterpret_cast<uint4 *>(sm + kPfX + (r < 2 ? 0 : 8192) + ip * 4096 + sw128(j2, c)) = xv[r];
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  if (threadIdx.x == 0) {
    in_seen = mbar_wait(&bar_in, 0, a.status);
    if (in_seen) {
      tc_fence_after();
      // ---- SA: D[(i, j1)][(m2, ro)], TMEM columns 0..63 ----
      const uint32_t id = idesc_bf16(128, 64, true, false);
      const uint64_t ah = sdesc_mn_sw128(sm + kPfX, 4096), al = sdesc_mn_sw128(sm + kPfX + 8192, 4096);
      const uint64_t bh = sdesc_sw128(sm + kPfC), bl = sdesc_sw128(sm + kPfC + 8192);
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) mma3(tmem, ah + 128 * kk, al + 128 * kk, bh + 2 * kk, bl + 2 * kk, id, kk == 0);
      mma_commit(&bar_mma);
    } else {
      abort_flag = 1;
    }
  }
  __syncwarp();
  bool ok = mbar_wait(&bar_mma, 0, a.status);
  tc_fence_after();

  // ---- EA: twiddle; T[(m2, i)][(j1, ri)] (row 4 m2 + i, K-major, swizzled) ----
  if (__all_sync(0xffffffffu, ok && !abort_flag)) {  // warp-uniform: tcgen05.ld is .sync.aligned
    uint32_t v[32];
    tmem_ld32(tl + (uint32_t)(32 * hw), v);  // columns (m2, ro), m2 = 16 hw .. 16 hw + 15
    const int il = q, j1 = lane;
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const float re = __uint_as_float(v[2 * t]), im = __uint_as_float(v[2 * t + 1]);
      const float tr = re * tw[t].x - im * tw[t].y, ti = re * tw[t].y + im * tw[t].x;
      uint32_t hi, lo;
      split_pair(tr, ti, hi, lo);
      const uint32_t off = sw128(4 * (16 * hw + t) + il, j1 >> 2) + (uint32_t)(j1 & 3) * 4;
      *reinterpret_cast<uint32_t *>(sm + kPfT + off) = hi;
      *reinterpret_cast<uint32_t *>(sm + kPfT + 16384 + off) = lo;
    }
  } else {
    abort_flag = 1;
  }
  uc_stage_sync();

  // ---- SB: D[(m2, i)][(m1, ro)], TMEM columns 64..127 ----
  if (threadIdx.x == 0 && !abort_flag) {
    const uint32_t id = idesc_bf16(128, 64);
    const uint64_t ah = sdesc_sw128(sm + kPfT), al = sdesc_sw128(sm + kPfT + 16384);
    const uint64_t bh = sdesc_sw128(sm + kPfB), bl = sdesc_sw128(sm + kPfB + 8192);
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) mma3(tmem + 64, ah + 2 * kk, al + 2 * kk, bh + 2 * kk, bl + 2 * kk, id, kk == 0);
    mma_commit(&bar_mma);
  }
  __syncwarp();
  ok = !abort_flag && mbar_wait(&bar_mma, 1, a.status);
  tc_fence_after();

  // ---- EB: X[m2 + 32 m1][i] -> Xin[(i2, ri)][(m, i1)] for m <= Nphi / 2 ----
  if (__all_sync(0xffffffffu, ok && !abort_flag)) {
    uint32_t v[32];
    tmem_ld32(tl + (uint32_t)(64 + 32 * hw), v);  // columns (m1, ro), m1 = 16 hw .. 16 hw + 15
    const int rb = q * 32 + lane, m2 = rb >> 2, il = rb & 3;
    const int i = i0 + il, i1 = i & 31, i2 = i >> 5;
    const int half = a.Nphi / 2;
    const size_t rre = (size_t)(2 * i2) * a.ld, rim = rre + a.ld;
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const int m = m2 + 32 * (16 * hw + t);
      if (m <= half) {
        const size_t col = (size_t)m * 32 + i1;
        uint32_t h, l;  // (re | im << 16) per plane
        split_pair(__uint_as_float(v[2 * t]), __uint_as_float(v[2 * t + 1]), h, l);
        reinterpret_cast<uint16_t *>(a.xin_hi)[rre + col] = (uint16_t)h;
        reinterpret_cast<uint16_t *>(a.xin_lo)[rre + col] = (uint16_t)l;
        if (m != 0 && m != half) {  // self-conjugate modes have no imaginary part
          reinterpret_cast<uint16_t *>(a.xin_hi)[rim + col] = (uint16_t)(h >> 16);
          reinterpret_cast<uint16_t *>(a.xin_lo)[rim + col] = (uint16_t)(l >> 16);
        }
      }
    }
  }
  if (threadIdx.x == 0 && !in_seen) mbar_wait(&bar_in, 0, a.status);  // copies in flight land first
  // with the row-tile hand-over this kernel never waited for its predecessor (the step's
  // finalisation); waiting now makes this kernel's completion imply that one's
  if (a.rowpend) pdl_wait();
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kPfTmemCols);
}

__global__ void __launch_bounds__(kPfThreads, 2)
    k_phifwd(const __grid_constant__ CUtensorMap tCh,
    const __grid_constant__ CUtensorMap tCl,
    const __grid_constant__ CUtensorMap tBh,
    const __grid_constant__ CUtensorMap tBl, PhiFwdArgs a) {
  phifwd_cta(&tCh, &tCl, &tBh, &tBl, a);
}

// The same for a group of disks of one grid (batched sweeps): blockIdx.y is the disk, whose
// arguments come from a device array.
__global__ void __launch_bounds__(kPfThreads, 2)
    k_phifwd_group(const __grid_constant__ CUtensorMap tCh,
    const __grid_constant__ CUtensorMap tCl,
    const __grid_constant__ CUtensorMap tBh,
    const __grid_constant__ CUtensorMap tBl, const PhiFwdArgs *__restrict__ disks) {
  phifwd_cta(&tCh, &tCl, &tBh, &tBl, disks[blockIdx.y]);
}

}  // namespace tc
}  // namespace dg
