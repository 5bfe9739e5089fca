// Split-BF16 tensor-core GEMM for sm_100a (tcgen05 + TMA + TMEM).
//
//   D[M x N] (FP32) = A[M x K] . B[N x K]^T,  A = A_hi + A_lo,  B = B_hi + B_lo (BF16 pairs)
//   D ~= A_hi B_hi + A_hi B_lo + A_lo B_hi          (the A_lo B_lo term is below 2^-16 relative)
//
// Both operands are K-major (K contiguous) in global memory and are staged by TMA into
// 128-byte-swizzled shared-memory tiles.  One thread issues the MMAs (three per 16-wide
// K step, all accumulating into one FP32 TMEM accumulator); one thread drives TMA; the
// four warps then drain TMEM through tcgen05.ld and run a fused epilogue.  Every
// mbarrier wait is bounded: on timeout the kernel raises kStTimeout in the caller's
// status word, drains what it has in flight, frees its TMEM and returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "dg_common.cuh"

namespace dg {
namespace tc {

constexpr int BM = 128;      // rows of a CTA tile (TMEM lanes)
constexpr int BN = 64;       // columns of a CTA tile (TMEM columns)
constexpr int BK = 64;       // K per stage: 64 BF16 = one 128-byte swizzle row
constexpr int STAGES = 4;
constexpr int kThreads = 128;
constexpr uint32_t kTileA = BM * BK * 2;
constexpr uint32_t kTileB = BN * BK * 2;
constexpr uint32_t kStageBytes = 2 * kTileA + 2 * kTileB;
constexpr uint32_t kTmemCols = 64;  // power of two >= 32 and >= BN
constexpr size_t kSmemBytes = (size_t)STAGES * kStageBytes + 1024;
// dynamic shared memory for a pipeline of ns stages (short-K GEMMs use 1-2 stages so that
// several CTAs share an SM)
__host__ __device__ constexpr size_t smem_bytes(int ns) { return (size_t)ns * kStageBytes + 1024; }

enum EpiMode : int {
  kEpiSplit = 0,        // out_hi/out_lo[row][col] = split(D)
  kEpiSplitScaled = 1,  // out = split(D * table[row][col])
  kEpiRowScaleF32 = 2,  // out_f32[row][col] = D * row_scale[row]
  // factored u-direction convolution (mixed.cu documents the index maps)
  kEpiPhiToXin = 3,     // phi spectrum row c, column i  -> Xin[(i2, ri)][(m, i1)]
  kEpiTwiddleF1 = 4,    // rows (p2, ri), cols (m, i1): x W_M^{p2 i1} -> T[(i1, ri)][(m, p2)]
  kEpiTwiddleI1 = 5,    // rows (m, p2), cols (i1, ri): x W_M^{-p2 i1} -> U[(m, i1)][(p2, ri)]
  kEpiI2ToZ = 6,        // rows (m, i1), cols (i2, ri) -> Z[c(m, ri)][i1 + A i2]
  // surrogate network (mlp.cu); row stride ldo everywhere
  kEpiMlpAct = 7,       // z = D + bias[col] -> out_f32 (pre-activation); split(SiLU(z)) -> out_hi / out_lo
  kEpiMlpOut = 8,       // D + bias[col] -> out_f32 (linear head)
  kEpiMlpBack = 9,      // d = D * SiLU'(table[row][col]) -> out_f32 and split(d) -> out_hi / out_lo
  kEpiStoreBounded = 10,  // D -> out_f32[row][col] for row < lim_m, col < lim_n (weight gradients)
  // factored phi transforms at Nphi = 4096 = 64 x 64 (j = 64 j1 + j2, m = m1 + 64 m2;
  // mixed.cu documents the passes).  The S1 product reads its B operand (the gravity
  // operand s[i][64 j1 + j2] as the [(i, j1)][j2] matrix) in 64 x 64 blocks per row i, the
  // Q2 product its A operand (V[(i, m1)][(ri, j2)] as [(i, m1, ri)][j2]) in 128 x 64
  // blocks per row i: both MN-major with the block's rows as K.
  // Layouts chosen so that every epilogue stores contiguous runs: T and V hold the real
  // and imaginary parts as two 64-column planes of each row, X is stored MN-major.
  kEpiPhiS1 = 11,       // rows (m1, ri), cols (i, j2): x W_N^{j2 m1} -> T[(m1, i)][(ri, j2)]
  kEpiPhiS2 = 12,       // rows (m1, i), cols (m2, ri): modes m <= N/2 -> Xin[(i2, ri)][(m, i1)]
  kEpiI2ToX = 13,       // rows (m, i1), cols (i2, ri): X and its conjugate -> X[(m / 64, ri)][(m % 64, i)]
  kEpiPhiQ1 = 14,       // rows (m1, i), cols (j2, ri): x W_N^{-j2 m1} -> V[(i, m1)][(ri, j2)]
  kEpiPhiQ2 = 15,       // rows (i, j2), cols j1: x row_scale[i] -> out_f32[i][64 j1 + j2]
};

struct GemmArgs {
  int M, N, K;
  __nv_bfloat16 *out_hi, *out_lo;
  float *out_f32;
  int ldo;
  const float *table;  // kEpiSplitScaled, row stride ldo
  const float *row_scale;
  int *status;         // kSt* bits raised on a bounded-wait timeout
  // factored u-direction: A = i1 range (Nu / 32), Nphi, padded complex-mode count
  int fa, nphi, nmodes;
  const float2 *twiddle;  // W_M^{p2 i1}, [64][fa]
  // row-tile counters of the hydro step that follows (dg_common.cuh rowtile_*): CTA (0, 0)
  // sets rowpend[0 .. rp_n) = rp_val once this kernel's predecessor has completed
  int *rowpend;
  int rp_n, rp_val;
  // surrogate network epilogues
  const float *bias;   // kEpiMlpAct, kEpiMlpOut: per column, padded with zeros
  int lim_m, lim_n;    // kEpiStoreBounded
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded parity wait: gives up after ~1 s of SM clock and raises kStTimeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *status) {
  const uint32_t addr = smem_u32(bar);
  long long start = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
    if (it == 64) start = clock64();
    if (it > 64 && clock64() - start > (1ll << 31)) {
      if (status) atomicOr(status, kStTimeout);
      return false;
    }
  }
}

// one contiguous global -> shared copy completing on an mbarrier (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, uint64_t *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)tm), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t sdesc_sw128(const void *p) {
  uint64_t a = smem_u32(p);
  uint64_t d = 0;
  d |= (a >> 4) & 0x3FFFull;            // start address
  d |= 1ull << 16;                      // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;     // stride byte offset: 8 rows x 128 B
  d |= 1ull << 46;                      // descriptor version (sm_100)
  d |= 2ull << 61;                      // SWIZZLE_128B
  return d;
}

// Shared-memory matrix descriptor: MN-major, 128-byte swizzle.  The tile is stored as
// 64-element MN chunks (lbo bytes apart) of K rows of 128 bytes, 8-row groups 1024 bytes
// apart; one 16-deep K step is 16 rows = 2048 bytes.
__device__ __forceinline__ uint64_t sdesc_mn_sw128(const void *p, uint32_t lbo) {
  uint64_t a = smem_u32(p);
  uint64_t d = 0;
  d |= (a >> 4) & 0x3FFFull;
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;  // leading byte offset: next MN chunk
  d |= (uint64_t)(1024 >> 4) << 32;             // stride byte offset: next 8 K rows
  d |= 1ull << 46;
  d |= 2ull << 61;
  return d;
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, M x N; a_mn / b_mn select
// MN-major operands.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn = false, bool b_mn = false) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// Epilogues of the factored u-direction passes: 32 accumulator columns starting at col of
// one row.  Index maps (mixed.cu): i = i1 + A i2 (A = args.fa, i2 < 32), p = p2 + 64 p1,
// complex modes m in [0, nmodes), phi index c(m, ri): c = 0 -> (0, re), c = 1 ->
// (Nphi/2, re), c >= 2 -> (c / 2, c % 2).
template <int MODE>
__device__ __forceinline__ void epi_factored(const GemmArgs &a, int row, int col, const uint32_t (&r)[32], int lane) {
  const int A = a.fa;  // a multiple of 32, so a 32-column chunk never straddles A
  auto put = [&](size_t k, float x) {
    __nv_bfloat16 h, l;
    split_bf16(x, h, l);
    a.out_hi[k] = h;
    a.out_lo[k] = l;
  };
  if (MODE == kEpiPhiToXin) {
    // rows c of the phi spectrum, columns i = i1 + A i2 -> Xin[(i2, ri)][(m, i1)], ld = nmodes * A;
    // the chunk's 32 columns are 32 consecutive i1 of one i2: one contiguous 64-byte run
    const int c = row;
    const int m = (c == 0) ? 0 : (c == 1 ? a.nphi / 2 : c >> 1);
    const int ri = (c < 2) ? 0 : (c & 1);
    const int i2 = col / A, i1b = col - i2 * A;
    const size_t k0 = (size_t)(i2 * 2 + ri) * ((size_t)a.nmodes * A) + (size_t)m * A + i1b;
    uint32_t ph[16], pl[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      __nv_bfloat16 h0, l0, h1, l1;
      split_bf16(__uint_as_float(r[2 * q]), h0, l0);
      split_bf16(__uint_as_float(r[2 * q + 1]), h1, l1);
      ph[q] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
      pl[q] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
    uint4 *oh = reinterpret_cast<uint4 *>(a.out_hi + k0);
    uint4 *ol = reinterpret_cast<uint4 *>(a.out_lo + k0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      oh[q] = make_uint4(ph[4 * q], ph[4 * q + 1], ph[4 * q + 2], ph[4 * q + 3]);
      ol[q] = make_uint4(pl[4 * q], pl[4 * q + 1], pl[4 * q + 2], pl[4 * q + 3]);
    }
  } else if (MODE == kEpiTwiddleF1) {
    // rows (p2, ri) (re / im in lanes l, l^1), cols (m, i1) -> T[(i1, ri)][(m, p2)], ld = nmodes * 64
    const int p2 = row >> 1, ri = row & 1;
    const int m = col / A, i1b = col - m * A;
    const size_t ld = (size_t)a.nmodes * 64;
    const size_t base = (size_t)m * 64 + p2;
    const float2 *tw = a.twiddle + p2 * A + i1b;
#pragma unroll
    for (int q = 0; q < 32; ++q) {
      const float v = __uint_as_float(r[q]);
      const float o = __shfl_xor_sync(0xffffffffu, v, 1);
      const float re = ri ? o : v, im = ri ? v : o;
      const float2 w = __ldg(tw + q);
      const float out = ri ? (re * w.y + im * w.x) : (re * w.x - im * w.y);
      put((size_t)((i1b + q) * 2 + ri) * ld + base, out);
    }
  } else if (MODE == kEpiTwiddleI1) {
    // rows (m, p2), cols (i1, ri) pairs in-thread: x conj(W_M^{p2 i1}) -> U[(m, i1)][(p2, ri)], ld = 128
    const int m = row >> 6, p2 = row & 63;
    const int i1b = col >> 1;
    const float2 *tw = a.twiddle + p2 * A + i1b;
    const size_t base = ((size_t)m * A + i1b) * 128 + (size_t)p2 * 2;
#pragma unroll
    for (int q = 0; q < 32; q += 2) {
      const float re = __uint_as_float(r[q]), im = __uint_as_float(r[q + 1]);
      const float2 w = __ldg(tw + (q >> 1));
      const float ore = re * w.x + im * w.y, oim = im * w.x - re * w.y;
      __nv_bfloat16 h0, l0, h1, l1;
      split_bf16(ore, h0, l0);
      split_bf16(oim, h1, l1);
      const size_t k = base + (size_t)(q >> 1) * 128;
      *reinterpret_cast<uint32_t *>(a.out_hi + k) =
          (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
      *reinterpret_cast<uint32_t *>(a.out_lo + k) =
          (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
  } else if (MODE == kEpiI2ToZ) {
    // rows (m, i1), cols (i2, ri) -> Z[c(m, ri)][i1 + A i2] (MN-major operand of the inverse phi GEMM)
    const int m = row / A, i1 = row - m * A;
    const int half = a.nphi / 2;
    if (m > half) return;  // padding modes
    const size_t Nu = (size_t)A * 32;
    const int cre = (m == 0) ? 0 : (m == half ? 1 : 2 * m);
    const int cim = (m == 0 || m == half) ? -1 : 2 * m + 1;  // imaginary parts of self-conjugate modes vanish
    const int i2b = col >> 1;
#pragma unroll
    for (int q = 0; q < 32; q += 2) {
      const size_t ii = (size_t)i1 + (size_t)A * (i2b + (q >> 1));
      put((size_t)cre * Nu + ii, __uint_as_float(r[q]));
      if (cim >= 0) put((size_t)cim * Nu + ii, __uint_as_float(r[q + 1]));
    }
  }
}

// Epilogues of the surrogate network's products: 32 accumulator columns from col of one row.
__device__ __forceinline__ float silu_f(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float silu_grad_f(float z) {
  const float sg = 1.f / (1.f + __expf(-z));
  return sg * (1.f + z * (1.f - sg));
}

template <int MODE>
__device__ __forceinline__ void epi_mlp_bounded(const GemmArgs &a, int row, int col, const uint32_t (&r)[32]) {
  if (row >= a.lim_m) return;
  const size_t base = (size_t)row * a.ldo + col;
#pragma unroll
  for (int q = 0; q < 32; ++q)
    if (col + q < a.lim_n) a.out_f32[base + q] = __uint_as_float(r[q]);
}

template <int MODE>
__device__ __forceinline__ void epi_mlp(const GemmArgs &a, int row, int col, const uint32_t (&r)[32]) {
  const size_t base = (size_t)row * a.ldo + col;
  float v[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
  if (MODE == kEpiMlpAct || MODE == kEpiMlpOut) {
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] += __ldg(a.bias + col + q);
  }
  if (MODE == kEpiMlpBack) {
    const float *z = a.table + base;
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] *= silu_grad_f(z[q]);
  }
  float4 *o = reinterpret_cast<float4 *>(a.out_f32 + base);
#pragma unroll
  for (int q = 0; q < 8; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  if (MODE == kEpiMlpAct || MODE == kEpiMlpBack) {
    if (MODE == kEpiMlpAct) {
#pragma unroll
      for (int q = 0; q < 32; ++q) v[q] = silu_f(v[q]);
    }
    uint32_t ph[16], pl[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      __nv_bfloat16 h0, l0, h1, l1;
      split_bf16(v[2 * q], h0, l0);
      split_bf16(v[2 * q + 1], h1, l1);
      ph[q] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
      pl[q] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
    uint4 *oh = reinterpret_cast<uint4 *>(a.out_hi + base);
    uint4 *ol = reinterpret_cast<uint4 *>(a.out_lo + base);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      oh[q] = make_uint4(ph[4 * q], ph[4 * q + 1], ph[4 * q + 2], ph[4 * q + 3]);
      ol[q] = make_uint4(pl[4 * q], pl[4 * q + 1], pl[4 * q + 2], pl[4 * q + 3]);
    }
  }
}

// Epilogues of the factored phi transforms at Nphi = 4096 (twiddle: W_N^{m1 j2} as
// [64][64], A = Nu / 32, nmodes = padded complex-mode count of the u stage).
template <int MODE>
__device__ __forceinline__ void epi_phi4096(const GemmArgs &a, int row, int col, const uint32_t (&r)[32], int lane) {
  const int A = a.fa, Nu = 32 * A, N = a.nphi, half = N / 2;
  auto put = [&](size_t k, float x) {
    __nv_bfloat16 h, l;
    split_bf16(x, h, l);
    a.out_hi[k] = h;
    a.out_lo[k] = l;
  };
  if (MODE == kEpiPhiS1) {
    // rows (m1, ri): re / im of one m1 in lanes l, l^1; cols (i, j2), the chunk inside one i;
    // each lane stores its 32 values of one plane contiguously
    const int m1 = row >> 1, ri = row & 1;
    const int i = col >> 6, j2b = col & 63;
    const float2 *tw = a.twiddle + m1 * 64 + j2b;
    uint32_t ph[16], pl[16];
#pragma unroll
    for (int q = 0; q < 32; q += 2) {
      float out[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const float v = __uint_as_float(r[q + e]);
        const float o = __shfl_xor_sync(0xffffffffu, v, 1);
        const float re = ri ? o : v, im = ri ? v : o;
        const float2 w = __ldg(tw + q + e);
        out[e] = ri ? (re * w.y + im * w.x) : (re * w.x - im * w.y);
      }
      __nv_bfloat16 h0, l0, h1, l1;
      split_bf16(out[0], h0, l0);
      split_bf16(out[1], h1, l1);
      ph[q >> 1] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
      pl[q >> 1] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
    const size_t base = ((size_t)m1 * Nu + i) * 128 + ri * 64 + j2b;
    uint4 *oh = reinterpret_cast<uint4 *>(a.out_hi + base);
    uint4 *ol = reinterpret_cast<uint4 *>(a.out_lo + base);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      oh[q] = make_uint4(ph[4 * q], ph[4 * q + 1], ph[4 * q + 2], ph[4 * q + 3]);
      ol[q] = make_uint4(pl[4 * q], pl[4 * q + 1], pl[4 * q + 2], pl[4 * q + 3]);
    }
  } else if (MODE == kEpiPhiS2) {
    // rows (m1, i), cols (m2, ri) pairs in-thread -> the u stage's operand Xin
    const int m1 = row / Nu, i = row - m1 * Nu;
    const int i2 = i / A, i1 = i - i2 * A;
    const size_t ld = (size_t)a.nmodes * A;
#pragma unroll
    for (int q = 0; q < 32; q += 2) {
      const int m = m1 + 64 * ((col + q) >> 1);
      if (m > half) continue;
      put((size_t)(2 * i2) * ld + (size_t)m * A + i1, __uint_as_float(r[q]));
      if (m != 0 && m != half) put((size_t)(2 * i2 + 1) * ld + (size_t)m * A + i1, __uint_as_float(r[q + 1]));
    }
  } else if (MODE == kEpiI2ToX) {
    // rows (m, i1), cols (i2, ri) pairs in-thread -> the full Hermitian spectrum X
    const int m = row / A, i1 = row - m * A;
    if (m > half) return;  // padding modes
    const int i2b = col >> 1;
#pragma unroll
    for (int q = 0; q < 32; q += 2) {
      const size_t i = (size_t)i1 + (size_t)A * (i2b + (q >> 1));
      const float re = __uint_as_float(r[q]);
      const float im = (m == 0 || m == half) ? 0.f : __uint_as_float(r[q + 1]);
      // MN-major: row (m2, ri), column (m1, i): consecutive lanes (i1) store consecutive words
      const size_t ldx = (size_t)64 * Nu;
      const size_t c0 = (size_t)(m & 63) * Nu + i;
      put((size_t)(2 * (m >> 6)) * ldx + c0, re);
      put((size_t)(2 * (m >> 6) + 1) * ldx + c0, im);
      if (m != 0 && m != half) {
        const int mc = N - m;
        const size_t c1 = (size_t)(mc & 63) * Nu + i;
        put((size_t)(2 * (mc >> 6)) * ldx + c1, re);
        put((size_t)(2 * (mc >> 6) + 1) * ldx + c1, -im);
      }
    }
  } else if (MODE == kEpiPhiQ1) {
    // rows (m1, i), cols (j2, ri) pairs in-thread: x conj(W_N^{m1 j2}) -> V[(i, m1)][(ri, j2)],
    // 16 contiguous j2 per plane
    const int m1 = row / Nu, i = row - m1 * Nu;
    const int j2b = col >> 1;
    const float2 *tw = a.twiddle + m1 * 64 + j2b;
    float ore[16], oim[16];
#pragma unroll
    for (int q = 0; q < 32; q += 2) {
      const float re = __uint_as_float(r[q]), im = __uint_as_float(r[q + 1]);
      const float2 w = __ldg(tw + (q >> 1));
      ore[q >> 1] = re * w.x + im * w.y;
      oim[q >> 1] = im * w.x - re * w.y;
    }
    const size_t base = ((size_t)i * 64 + m1) * 128 + j2b;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const float *src = e ? oim : ore;
      uint32_t ph[8], pl[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        __nv_bfloat16 h0, l0, h1, l1;
        split_bf16(src[2 * q], h0, l0);
        split_bf16(src[2 * q + 1], h1, l1);
        ph[q] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
        pl[q] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
      }
      uint4 *oh = reinterpret_cast<uint4 *>(a.out_hi + base + 64 * e);
      uint4 *ol = reinterpret_cast<uint4 *>(a.out_lo + base + 64 * e);
      oh[0] = make_uint4(ph[0], ph[1], ph[2], ph[3]);
      oh[1] = make_uint4(ph[4], ph[5], ph[6], ph[7]);
      ol[0] = make_uint4(pl[0], pl[1], pl[2], pl[3]);
      ol[1] = make_uint4(pl[4], pl[5], pl[6], pl[7]);
    }
  } else if (MODE == kEpiPhiQ2) {
    // rows (i, j2), cols j1: dPhi[i][64 j1 + j2] (lanes: consecutive j2, so coalesced)
    const int i = row >> 6, j2 = row & 63;
    const float sc = a.row_scale[i];
    float *o = a.out_f32 + (size_t)i * N + j2;
#pragma unroll
    for (int q = 0; q < 32; ++q) o[64 * (col + q)] = __uint_as_float(r[q]) * sc;
  }
  (void)lane;
}

// The epilogue of one 32-column accumulator chunk of row `row`, columns col..col+31.
template <int MODE>
__device__ __forceinline__ void epi_chunk(const GemmArgs &args, int row, int col, const uint32_t (&r)[32], int lane) {
  if (MODE == kEpiStoreBounded) {
    epi_mlp_bounded<MODE>(args, row, col, r);
    return;
  }
  if (MODE >= kEpiPhiS1) {
    epi_phi4096<MODE>(args, row, col, r, lane);
    return;
  }
  if (MODE >= kEpiMlpAct) {
    epi_mlp<MODE>(args, row, col, r);
    return;
  }
  if (MODE >= kEpiPhiToXin) {
    epi_factored<MODE>(args, row, col, r, lane);
    return;
  }
  if (MODE == kEpiRowScaleF32) {
    const float sc = args.row_scale[row];
    float4 *o = reinterpret_cast<float4 *>(args.out_f32 + (size_t)row * args.ldo + col);
#pragma unroll
    for (int q = 0; q < 8; ++q)
      o[q] = make_float4(__uint_as_float(r[4 * q]) * sc, __uint_as_float(r[4 * q + 1]) * sc,
                         __uint_as_float(r[4 * q + 2]) * sc, __uint_as_float(r[4 * q + 3]) * sc);
  } else {
    float v[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
    if (MODE == kEpiSplitScaled) {
      const float4 *tb = reinterpret_cast<const float4 *>(args.table + (size_t)row * args.ldo + col);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        float4 t = tb[q];
        v[4 * q] *= t.x; v[4 * q + 1] *= t.y; v[4 * q + 2] *= t.z; v[4 * q + 3] *= t.w;
      }
    }
    uint32_t ph[16], pl[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      __nv_bfloat16 h0, l0, h1, l1;
      split_bf16(v[2 * q], h0, l0);
      split_bf16(v[2 * q + 1], h1, l1);
      ph[q] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
      pl[q] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
    uint4 *oh = reinterpret_cast<uint4 *>(args.out_hi + (size_t)row * args.ldo + col);
    uint4 *ol = reinterpret_cast<uint4 *>(args.out_lo + (size_t)row * args.ldo + col);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      oh[q] = make_uint4(ph[4 * q], ph[4 * q + 1], ph[4 * q + 2], ph[4 * q + 3]);
      ol[q] = make_uint4(pl[4 * q], pl[4 * q + 1], pl[4 * q + 2], pl[4 * q + 3]);
    }
  }
}

// The body of one CTA tile (blockIdx.x: N tile, blockIdx.y: M tile) of the split GEMM.
template <int MODE, bool A_MN, bool B_MN, int NS>
__device__ __forceinline__ void gemm_tile(const CUtensorMap *pAh, const CUtensorMap *pAl, const CUtensorMap *pBh,
                                          const CUtensorMap *pBl, const GemmArgs &args) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full_bar[NS], empty_bar[NS], done_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int nk = args.K / BK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_d = tmem_slot;
  pdl_wait();  // operands come from the previous kernel on the stream
  pdl_trigger();
  if (args.rowpend && blockIdx.x == 0 && blockIdx.y == 0)
    for (int r = threadIdx.x; r < args.rp_n; r += blockDim.x) args.rowpend[r] = args.rp_val;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ----
    int issued = 0;
    for (int kc = 0; kc < nk; ++kc) {
      const int s = kc % NS;
      if (kc >= NS && !mbar_wait(&empty_bar[s], ((kc / NS) - 1) & 1, args.status)) {
        abort_flag = 1;
        break;
      }
      if (abort_flag) break;
      uint8_t *st = smem + s * kStageBytes;
      mbar_arrive_expect_tx(&full_bar[s], kStageBytes);
      if (A_MN && MODE == kEpiPhiQ2) {  // V as [(i, m1, ri)][j2]: M chunk c = row i = m0 / 64 + c
        tma_load_2d(st, pAh, &full_bar[s], 0, (m0 / 64) * 128 + kc * BK);
        tma_load_2d(st + kTileA / 2, pAh, &full_bar[s], 0, (m0 / 64 + 1) * 128 + kc * BK);
        tma_load_2d(st + kTileA, pAl, &full_bar[s], 0, (m0 / 64) * 128 + kc * BK);
        tma_load_2d(st + kTileA + kTileA / 2, pAl, &full_bar[s], 0, (m0 / 64 + 1) * 128 + kc * BK);
      } else if (A_MN) {  // [K][M] in global: two 64-wide M chunks of 64 K rows
        tma_load_2d(st, pAh, &full_bar[s], m0, kc * BK);
        tma_load_2d(st + kTileA / 2, pAh, &full_bar[s], m0 + 64, kc * BK);
        tma_load_2d(st + kTileA, pAl, &full_bar[s], m0, kc * BK);
        tma_load_2d(st + kTileA + kTileA / 2, pAl, &full_bar[s], m0 + 64, kc * BK);
      } else {
        tma_load_2d(st, pAh, &full_bar[s], kc * BK, m0);
        tma_load_2d(st + kTileA, pAl, &full_bar[s], kc * BK, m0);
      }
      if (B_MN && MODE == kEpiPhiS1) {  // the [(i, j1)][j2] view of s: N chunk n0 = row i's 64 columns
        tma_load_2d(st + 2 * kTileA, pBh, &full_bar[s], 0, n0 + kc * BK);
        tma_load_2d(st + 2 * kTileA + kTileB, pBl, &full_bar[s], 0, n0 + kc * BK);
      } else if (B_MN) {  // [K][N] in global: one 64-wide N chunk
        tma_load_2d(st + 2 * kTileA, pBh, &full_bar[s], n0, kc * BK);
        tma_load_2d(st + 2 * kTileA + kTileB, pBl, &full_bar[s], n0, kc * BK);
      } else {
        tma_load_2d(st + 2 * kTileA, pBh, &full_bar[s], kc * BK, n0);
        tma_load_2d(st + 2 * kTileA + kTileB, pBl, &full_bar[s], kc * BK, n0);
      }
      ++issued;
    }
    // every issued copy must land before the CTA may exit
    for (int kc = issued > NS ? issued - NS : 0; kc < issued; ++kc)
      mbar_wait(&full_bar[kc % NS], (kc / NS) & 1, args.status);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    const uint32_t idesc = idesc_bf16(BM, BN, A_MN, B_MN);
    for (int kc = 0; kc < nk; ++kc) {
      const int s = kc % NS;
      if (!mbar_wait(&full_bar[s], (kc / NS) & 1, args.status)) {
        abort_flag = 1;
        break;
      }
      tc_fence_after();
      uint8_t *st = smem + s * kStageBytes;
      const uint64_t dAh = A_MN ? sdesc_mn_sw128(st, kTileA / 2) : sdesc_sw128(st);
      const uint64_t dAl = A_MN ? sdesc_mn_sw128(st + kTileA, kTileA / 2) : sdesc_sw128(st + kTileA);
      const uint64_t dBh = B_MN ? sdesc_mn_sw128(st + 2 * kTileA, 0) : sdesc_sw128(st + 2 * kTileA);
      const uint64_t dBl = B_MN ? sdesc_mn_sw128(st + 2 * kTileA + kTileB, 0) : sdesc_sw128(st + 2 * kTileA + kTileB);
      // a 16-deep K step is 32 bytes along a K-major row, or 16 rows (2048 bytes) of an MN-major tile
      const uint64_t stepA = A_MN ? (2048 >> 4) : (32 >> 4), stepB = B_MN ? (2048 >> 4) : (32 >> 4);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint64_t oa = (uint64_t)kk * stepA, ob = (uint64_t)kk * stepB;
        mma_bf16(tmem_d, dAh + oa, dBh + ob, idesc, (kc | kk) != 0);
        mma_bf16(tmem_d, dAh + oa, dBl + ob, idesc, 1u);
        mma_bf16(tmem_d, dAl + oa, dBh + ob, idesc, 1u);
      }
      mma_commit(&empty_bar[s]);
    }
    mma_commit(&done_bar);  // arrives once every MMA issued above has completed
  }
  __syncwarp();

  // ---- epilogue: TMEM lanes 32w..32w+31 belong to warp w ----
  const bool ok = mbar_wait(&done_bar, 0, args.status);
  tc_fence_after();
  if (ok && !abort_flag) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t r[32];
      tmem_ld32(tmem_d + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
      epi_chunk<MODE>(args, row, n0 + c0, r, lane);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem_d, kTmemCols);
}

template <int MODE, bool A_MN = false, bool B_MN = false, int NS = STAGES>
__global__ void __launch_bounds__(kThreads, (NS == 1 ? 4 : (NS == 2 ? 2 : 1)))
    k_gemm_split(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
                 const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBl, GemmArgs args) {
  gemm_tile<MODE, A_MN, B_MN, NS>(&tmAh, &tmAl, &tmBh, &tmBl, args);
}

// One product for a group of disks of the same grid (batched sweeps): blockIdx.z is the
// disk.  One operand is the group's shared DFT table (the grid-constant maps), the other
// is the disk's own (its tensor maps sit with its epilogue arguments in a device array;
// TMA reads a map from global memory as from a kernel parameter).  PER_A: the per-disk
// operand is A.  Each disk's tiles run exactly the single-disk kernel's code.
struct __align__(64) GemmDisk {
  CUtensorMap hi, lo;  // the disk's operand (hi / lo planes)
  GemmArgs args;       // its epilogue: outputs, khat table, row scale, status word
};

template <int MODE, bool A_MN, bool B_MN, int NS, bool PER_A>
__global__ void __launch_bounds__(kThreads, (NS == 1 ? 4 : (NS == 2 ? 2 : 1)))
    k_gemm_split_group(const __grid_constant__ CUtensorMap tmCh, const __grid_constant__ CUtensorMap tmCl,
                       const GemmDisk *__restrict__ disks) {
  const GemmDisk &d = disks[blockIdx.z];
  if (PER_A)
    gemm_tile<MODE, A_MN, B_MN, NS>(&d.hi, &d.lo, &tmCh, &tmCl, d.args);
  else
    gemm_tile<MODE, A_MN, B_MN, NS>(&tmCh, &tmCl, &d.hi, &d.lo, d.args);
}

// ---------------------------------------------------------------------------------
// Persistent form of the group product (batched sweeps).  One CTA per SM walks the tiles
// of every disk of the group (tile t = blockIdx.x + k gridDim.x; disk, M tile, N tile
// from t) with its warps specialised: warp 0 drives TMA through an NS2-deep ring of stages
// that runs ahead across tile boundaries, warp 1 issues the MMAs, the other EW warps drain
// TMEM and run the epilogue (EW / 4 warps per 32-lane TMEM quarter, each taking its share
// of the tile's columns).  Two TMEM accumulators (128 columns each) let the epilogue of
// one tile overlap the MMAs of the next.  A lone disk's products run with EW = 8: its
// four-step and factored passes, one or two K blocks per tile with heavy epilogues, are
// epilogue-bound.  The batch groups' dense products keep EW = 4, which measured about
// 5 % faster for them.  Tiles are 128 x 128: per byte loaded from L2 twice
// the MMA work of the 128 x 64 tiles above.  Each output element sees the same sequence
// of K steps and products as in k_gemm_split.  All waits are bounded as above; on a
// timeout every role stops at its next wait, in-flight copies are drained, and TMEM is
// freed.
constexpr int BN2 = 128;
constexpr int NS2 = 3;
constexpr uint32_t kTileB2 = BN2 * BK * 2;
constexpr uint32_t kStageBytes2 = 2 * kTileA + 2 * kTileB2;  // 64 KB
constexpr int kEpiWarpsLone = 8, kEpiWarpsGroup = 4;  // epilogue warps of the two entries
constexpr int threads_persist(int ew) { return 64 + 32 * ew; }
constexpr uint32_t kTmemColsP = 2 * BN2;
constexpr size_t kSmemP = (size_t)NS2 * kStageBytes2 + 1024;
// pipeline stages and dynamic shared memory of the persistent kernel for a tile width
__host__ __device__ constexpr int persist_stages(int bnt) { return bnt == 256 ? 2 : NS2; }
__host__ __device__ constexpr size_t smem_persist(int bnt) {
  return (size_t)persist_stages(bnt) * (2 * kTileA + 2 * (size_t)bnt * BK * 2) + 1024;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int MODE, bool A_MN, bool B_MN, bool PER_A, int EW, int BNT>
__device__ __forceinline__ void gemm_persist_body(const CUtensorMap *pCh, const CUtensorMap *pCl,
                                                  const GemmDisk *__restrict__ disks, int tiles_n, int tiles_m,
                                                  int ntiles) {
  // tile width BNT (128, or 256 with two stages and the whole TMEM for two accumulators)
  constexpr int NST = persist_stages(BNT);
  constexpr uint32_t kTB = (uint32_t)BNT * BK * 2, kSB = 2 * kTileA + 2 * kTB, kTC = 2 * BNT;
  constexpr uint32_t kChunkB = 64 * BK * 2;  // one 64-wide N chunk (or 64-row box) of a B plane
  static_assert(EW % 4 == 0 && BNT % (32 * (EW / 4)) == 0, "epilogue warps cover the tile");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full_bar[NST], empty_bar[NST], acc_full[2], acc_empty[2];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int q = 0; q < NST; ++q) {
      mbar_init(&full_bar[q], 1);
      mbar_init(&empty_bar[q], 1);
    }
    for (int q = 0; q < 2; ++q) {
      mbar_init(&acc_full[q], 1);
      mbar_init(&acc_empty[q], EW);  // one arrival per epilogue warp
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&tmem_slot, kTC);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  pdl_wait();  // operands come from the previous kernel on the stream
  pdl_trigger();
  if (disks[0].args.rowpend && blockIdx.x == 0)  // a lone product that arms the hydro's row tiles
    for (int r = threadIdx.x; r < disks[0].args.rp_n; r += blockDim.x) disks[0].args.rowpend[r] = disks[0].args.rp_val;
  const int per_disk = tiles_n * tiles_m;
  auto decode = [&](int t, int &z, int &m0, int &n0) {
    z = t / per_disk;
    const int r = t - z * per_disk;
    m0 = (r / tiles_n) * BM;
    n0 = (r - (r / tiles_n) * tiles_n) * BNT;
  };

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer ----
      uint32_t it = 0;
      int *st_word = nullptr;
      for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x) {
        int z, m0, n0;
        decode(t, z, m0, n0);
        const GemmDisk &d = disks[z];
        st_word = d.args.status;
        const CUtensorMap *Ah = PER_A ? &d.hi : pCh, *Al = PER_A ? &d.lo : pCl;
        const CUtensorMap *Bh = PER_A ? pCh : &d.hi, *Bl = PER_A ? pCl : &d.lo;
        const int nk = d.args.K / BK;
        for (int kc = 0; kc < nk; ++kc) {
          const uint32_t sidx = it % NST;
          if (it >= NST && !mbar_wait(&empty_bar[sidx], ((it / NST) - 1) & 1, st_word)) {
            abort_flag = 1;
            break;
          }
          if (abort_flag) break;
          uint8_t *st = smem + sidx * kSB;
          mbar_arrive_expect_tx(&full_bar[sidx], kSB);
          if (A_MN && MODE == kEpiPhiQ2) {  // V as [(i, m1, ri)][j2]: M chunk c = row i = m0 / 64 + c
            tma_load_2d(st, Ah, &full_bar[sidx], 0, (m0 / 64) * 128 + kc * BK);
            tma_load_2d(st + kTileA / 2, Ah, &full_bar[sidx], 0, (m0 / 64 + 1) * 128 + kc * BK);
            tma_load_2d(st + kTileA, Al, &full_bar[sidx], 0, (m0 / 64) * 128 + kc * BK);
            tma_load_2d(st + kTileA + kTileA / 2, Al, &full_bar[sidx], 0, (m0 / 64 + 1) * 128 + kc * BK);
          } else if (A_MN) {
            tma_load_2d(st, Ah, &full_bar[sidx], m0, kc * BK);
            tma_load_2d(st + kTileA / 2, Ah, &full_bar[sidx], m0 + 64, kc * BK);
            tma_load_2d(st + kTileA, Al, &full_bar[sidx], m0, kc * BK);
            tma_load_2d(st + kTileA + kTileA / 2, Al, &full_bar[sidx], m0 + 64, kc * BK);
          } else {
            tma_load_2d(st, Ah, &full_bar[sidx], kc * BK, m0);
            tma_load_2d(st + kTileA, Al, &full_bar[sidx], kc * BK, m0);
          }
          uint8_t *sb = st + 2 * kTileA;
#pragma unroll
          for (int c = 0; c < BNT / 64; ++c) {  // 64-wide N chunks (MN-major) or 64-row boxes (K-major)
            if (B_MN && MODE == kEpiPhiS1) {  // the [(i, j1)][j2] view of s: N chunk = row i's 64 columns
              tma_load_2d(sb + c * (kChunkB), Bh, &full_bar[sidx], 0, n0 + 64 * c + kc * BK);
              tma_load_2d(sb + kTB + c * (kChunkB), Bl, &full_bar[sidx], 0, n0 + 64 * c + kc * BK);
            } else if (B_MN) {
              tma_load_2d(sb + c * (kChunkB), Bh, &full_bar[sidx], n0 + 64 * c, kc * BK);
              tma_load_2d(sb + kTB + c * (kChunkB), Bl, &full_bar[sidx], n0 + 64 * c, kc * BK);
            } else {
              tma_load_2d(sb + c * (kChunkB), Bh, &full_bar[sidx], kc * BK, n0 + 64 * c);
              tma_load_2d(sb + kTB + c * (kChunkB), Bl, &full_bar[sidx], kc * BK, n0 + 64 * c);
            }
          }
          ++it;
        }
      }
      // every issued copy must land before the CTA may exit
      for (uint32_t j = it > NST ? it - NST : 0; j < it; ++j) mbar_wait(&full_bar[j % NST], (j / NST) & 1, st_word);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer ----
      const uint32_t idesc = idesc_bf16(BM, BNT, A_MN, B_MN);
      uint32_t it = 0;
      int lt = 0;
      for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x, ++lt) {
        int z, m0, n0;
        decode(t, z, m0, n0);
        const GemmDisk &d = disks[z];
        const int nk = d.args.K / BK;
        const int buf = lt & 1;
        if (lt >= 2 && !mbar_wait(&acc_empty[buf], ((lt >> 1) - 1) & 1, d.args.status)) {
          abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + (uint32_t)(buf * BNT);
        bool ok = true;
        for (int kc = 0; kc < nk; ++kc, ++it) {
          const uint32_t sidx = it % NST;
          if (!mbar_wait(&full_bar[sidx], (it / NST) & 1, d.args.status)) {
            abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          uint8_t *st = smem + sidx * kSB;
          const uint64_t dAh = A_MN ? sdesc_mn_sw128(st, kTileA / 2) : sdesc_sw128(st);
          const uint64_t dAl = A_MN ? sdesc_mn_sw128(st + kTileA, kTileA / 2) : sdesc_sw128(st + kTileA);
          const uint64_t dBh = B_MN ? sdesc_mn_sw128(st + 2 * kTileA, kChunkB) : sdesc_sw128(st + 2 * kTileA);
          const uint64_t dBl =
              B_MN ? sdesc_mn_sw128(st + 2 * kTileA + kTB, kChunkB) : sdesc_sw128(st + 2 * kTileA + kTB);
          const uint64_t stepA = A_MN ? (2048 >> 4) : (32 >> 4), stepB = B_MN ? (2048 >> 4) : (32 >> 4);
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
            const uint64_t oa = (uint64_t)kk * stepA, ob = (uint64_t)kk * stepB;
            mma_bf16(acc, dAh + oa, dBh + ob, idesc, (kc | kk) != 0);
            mma_bf16(acc, dAh + oa, dBl + ob, idesc, 1u);
            mma_bf16(acc, dAl + oa, dBh + ob, idesc, 1u);
          }
          mma_commit(&empty_bar[sidx]);
        }
        if (!ok) break;
        mma_commit(&acc_full[buf]);  // arrives once this tile's MMAs have completed
      }
    }
  } else {
    // ---- epilogue: warp w drains TMEM lanes 32 (w % 4) .. + 31, columns of its half ----
    const int qd = warp & 3;
    constexpr int kCols = BNT / (EW / 4);
    const int cb = ((warp - 2) / 4) * kCols;
    int lt = 0;
    for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x, ++lt) {
      int z, m0, n0;
      decode(t, z, m0, n0);
      const GemmDisk &d = disks[z];
      const int buf = lt & 1;
      if (!mbar_wait(&acc_full[buf], (lt >> 1) & 1, d.args.status)) {
        abort_flag = 1;
        break;
      }
      tc_fence_after();
      const int row = m0 + qd * 32 + lane;
#pragma unroll 1
      for (int c0 = cb; c0 < cb + kCols; c0 += 32) {
        uint32_t r[32];
        tmem_ld32(tmem + (uint32_t)(buf * BNT) + ((uint32_t)(qd * 32) << 16) + (uint32_t)c0, r);
        epi_chunk<MODE>(d.args, row, n0 + c0, r, lane);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[buf]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTC);
}

template <int MODE, bool A_MN, bool B_MN, bool PER_A, int BNT = BN2>
__global__ void __launch_bounds__(threads_persist(kEpiWarpsGroup), 1)
    k_gemm_group_persist(const __grid_constant__ CUtensorMap tmCh, const __grid_constant__ CUtensorMap tmCl,
                         const GemmDisk *__restrict__ disks, int tiles_n, int tiles_m, int ntiles) {
  gemm_persist_body<MODE, A_MN, B_MN, PER_A, kEpiWarpsGroup, BNT>(&tmCh, &tmCl, disks, tiles_n, tiles_m, ntiles);
}

// One product of a lone disk by the persistent kernel: A's maps as kernel parameters, B's
// maps and the epilogue arguments as one by-value entry (a "group" of one disk whose
// tensor maps TMA reads from the parameter space).
template <int MODE, bool A_MN, bool B_MN, int BNT = BN2>
__global__ void __launch_bounds__(threads_persist(kEpiWarpsLone), 1)
    k_gemm_persist(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
                   const __grid_constant__ GemmDisk b, int tiles_n, int tiles_m, int ntiles) {
  gemm_persist_body<MODE, A_MN, B_MN, false, kEpiWarpsLone, BNT>(&tmAh, &tmAl, &b, tiles_n, tiles_m, ntiles);
}

}  // namespace tc
}  // namespace dg
