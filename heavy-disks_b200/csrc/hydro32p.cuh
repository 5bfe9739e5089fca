// Packed form of the tiled mixed-precision hydro step: the arithmetic of hydro32t.cuh, with
// every thread advancing two adjacent columns at once in FP32x2 registers (Blackwell's
// paired FADD2 / FMUL2 / FFMA2), so one instruction, one shared-memory access and one set
// of row constants serve two zones.
//
// Stages, one warp per row (CTA barriers only where a stage reads other warps' rows):
//   S0 stage sigma, u, w, dPhi of rows i0-3 .. i0+kTileI+2        | barrier
//   S1 pressure perturbation of the staged rows                     | barrier
//   S2 source kick of rows i0-2 .. i0+kTileI+1 (hydro.hpp:73-96)    | barrier
//   S3 radial faces i0 .. i0+kTileI-1, two rows per warp            | barrier
//   S4-S6 per output row, in registers: the row's radial gather, its azimuthal faces
//      (neighbours by lane shuffles) and azimuthal gather, outputs and CFL rate; the warp
//      of the last row first computes the tile's top face i0+kTileI.
//
// Tile: kTileI rows x kTileJp = 58 output columns.  Stored columns c in [0, 64) hold the
// unwrapped columns J = j0 - 3 + c (a 3-column halo on each side); the outputs are
// c in [3, 61).  Tile bx starts at j0 = 58 bx + 1, so j0 - 3 is even and every column
// pair, and every global pair access, stays 8-byte aligned, also across the periodic
// wrap; the tiles cover J = 1 .. Nphi, column Nphi being column 0.  Lane l of a warp owns
// the pair (2l, 2l+1) of every row it visits (lanes 1 and 30 output one half); warp w
// visits rows w, w + 8, ...  Azimuthal neighbours (columns 2l - 2 .. 2l + 2) come from the
// neighbouring lanes by shuffle.  Columns whose results are never used are computed anyway
// and discarded, so shuffles run with every lane active.  With 58 columns a 1024-column
// grid takes 18 column tiles, so a 1024 x 1024 launch is 1152 CTAs: under two waves of
// four CTAs on each of the 148 SMs.
//
// Interior column tiles (no periodic wrap inside the tile) with self-gravity or no force
// stage sigma, u, w and dPhi in shared memory as one TMA box each (68 x 22 floats from the
// 16-byte-aligned column at or left of j0 - 3; rows outside the grid read as zero); the
// two edge tiles and the caller-forces path use thread loads.
#pragma once

#include "hydro32t.cuh"
#include "tc_gemm.cuh"

namespace dg {

constexpr int kTileJp = kLd32t - 6;        // output columns per CTA (58)
constexpr int kLdP = kLd32t + 4;           // floats per staged row: a TMA box from the aligned column
constexpr int kWarps32p = kThreads32t / 32;  // 8 row groups, one warp each
constexpr int kItLoadP = (kRows32t + kWarps32p - 1) / kWarps32p;
constexpr int kItSrcP = (kSrcRows32t + kWarps32p - 1) / kWarps32p;
constexpr int kItFaceP = kTileI / kWarps32p;  // S3 face rows per warp (the last face is S4's)
static_assert(kItFaceP * kWarps32p == kTileI, "face rows split evenly over the warps");
constexpr int kItOutP = (kTileI + kWarps32p - 1) / kWarps32p;
static_assert(kItOutP * kWarps32p == kTileI, "output rows split evenly over the warps");
// shared-memory plan of this kernel in floats: the five staged fields first (each one TMA
// box of kRows32t x kLdP; a TMA destination in shared memory is 128-byte aligned, so each
// field is padded to a multiple of 32 floats), then the radial fluxes and the row
// constants.  u1 / w1 (source rows i0-2 ..) overwrite the raw u / w of the same points one
// row down, in place.
constexpr int kFieldP = kRows32t * kLdP;            // 22 x 68 floats of one box
constexpr int kFieldStrideP = (kFieldP + 31) / 32 * 32;  // 1504
constexpr int kOffSgP = 0, kOffDpP = kFieldStrideP, kOffPhP = 2 * kFieldStrideP, kOffU0P = 3 * kFieldStrideP,
              kOffW0P = 4 * kFieldStrideP;
static_assert(kOffPhP % 32 == 0 && kOffU0P % 32 == 0 && kOffW0P % 32 == 0, "TMA destinations 128-byte aligned");
constexpr int kOffFP = 5 * kFieldStrideP;
// row constants: rows of the packed table Rows32::rowtab, [kRows32t][kRowTabW], one bulk copy
constexpr int kRowTabW = 20;      // floats per table row (the tNConst constants, padded to 16 bytes)
constexpr int kRowTabLead = 3;    // table row r holds row i = r - 3 (a tile's first staged row is i0 - 3)
constexpr int kRowTabExtra = 24;  // table rows beyond Nu: i = -3 .. Nu + 20
static_assert(tNConst <= kRowTabW && (kRowTabW * 4) % 16 == 0, "row table rows");
constexpr uint32_t kRcBytesP = kRows32t * kRowTabW * 4;
constexpr int kOffRcP = kOffFP + 4 * kFaceArr32t;
static_assert(kOffRcP % 4 == 0, "bulk-copy destination 16-byte aligned");
constexpr size_t kSmem32p = (size_t)(kOffRcP + kRows32t * kRowTabW) * sizeof(float) + 128;  // + alignment slack
constexpr uint32_t kFieldBytesP = kFieldP * 4;

namespace p2 {
typedef float2 F2;
__device__ __forceinline__ F2 S(float a) { return make_float2(a, a); }
__device__ __forceinline__ F2 add(F2 a, F2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ F2 mul(F2 a, F2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ F2 sub(F2 a, F2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }  // exact a - b
__device__ __forceinline__ F2 sel(bool px, bool py, F2 a, F2 b) {
  return make_float2(px ? a.x : b.x, py ? a.y : b.y);
}
__device__ __forceinline__ F2 sels(bool px, bool py, float a, float b) {
  return make_float2(px ? a : b, py ? a : b);
}
__device__ __forceinline__ F2 fdiv(F2 a, F2 b) { return make_float2(__fdividef(a.x, b.x), __fdividef(a.y, b.y)); }
// the fast divide is a * (1 / b), so several quotients by one b share one reciprocal
__device__ __forceinline__ F2 rcp(F2 b) { return make_float2(__fdividef(1.f, b.x), __fdividef(1.f, b.y)); }
// sqrt(x) for x > 0 as x rsqrt(x): one special-function operation
__device__ __forceinline__ float sqrt_pos(float x) { return x * rsqrtf(x); }
// hydro.hpp:16-18 on each half (see vanleer32)
__device__ __forceinline__ F2 vanleer(F2 a, F2 b) {
  const F2 p = mul(a, b), s = add(a, b), n = add(p, p);
  return make_float2(p.x > 0.f ? __fdividef(n.x, s.x) : 0.f, p.y > 0.f ? __fdividef(n.y, s.y) : 0.f);
}
__device__ __forceinline__ float up1(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float dn1(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }
}  // namespace p2

template <bool G2, int FM, bool IN>
__device__ __forceinline__ void hydro32p_tile(
    const float *__restrict__ sig, const float *__restrict__ uu, const float *__restrict__ ww,
    const float *__restrict__ Phi, const double *__restrict__ gRin, const double *__restrict__ gpin,
    float *__restrict__ so, float *__restrict__ uo, float *__restrict__ wo, const SplitBf16 &Sx, Ctl *ctl,
    const Rows32 &g, float *sm32t, double *red, double *bsum, double *zsum, const CUtensorMap *tmS,
    const CUtensorMap *tmU, const CUtensorMap *tmW, const CUtensorMap *tmP, uint64_t *bar_ld, uint64_t *bar_rc,
    bool early_state) {
  using namespace p2;
  float *rc = sm32t + kOffRcP;
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const int Nu = g.Nu, Nphi = g.Nphi;
  const int i0 = blockIdx.y * kTileI, j0 = blockIdx.x * kTileJp + 1;
  const int ib = i0 - 3;
  // staged fields as pairs: row r, lane l -> element r * L2 + l (+ po).  A TMA box starts at
  // the 16-byte-aligned column xa = j0 - 3 - 2 po, po = 0 or 1 (j0 - 3 is even)
  const int xs0 = j0 - 3;
  const bool use_tma = FM != kForceArrays && xs0 >= 0 && xs0 + kLd32t <= Nphi;  // CTA-uniform
  const int po = use_tma ? (xs0 & 3) >> 1 : 0;
  constexpr int L2 = kLdP / 2, LF = kLd32t / 2;  // pair strides: staged fields, face arrays
  F2 *SG = reinterpret_cast<F2 *>(sm32t + kOffSgP) + po, *DP = reinterpret_cast<F2 *>(sm32t + kOffDpP) + po;
  F2 *PH = reinterpret_cast<F2 *>(sm32t + kOffPhP) + po;
  F2 *U0 = reinterpret_cast<F2 *>(sm32t + kOffU0P) + po, *W0 = reinterpret_cast<F2 *>(sm32t + kOffW0P) + po;
  F2 *U1 = U0 + L2, *W1 = W0 + L2;  // source row rs = stored row rs + 1
  F2 *FF = reinterpret_cast<F2 *>(sm32t + kOffFP), *FR = FF + kFaceArr32t / 2, *GA = FR + kFaceArr32t / 2,
     *GB = GA + kFaceArr32t / 2;
  F2 *S3 = DP;  // new sigma for the mode sums, over the pressure perturbation (dead after S2)

  const int iend = (i0 + kTileI < Nu) ? i0 + kTileI : Nu;
  const int jc = wrap_col(xs0 + 2 * lane, Nphi);  // global column of this lane's first element (even)
  // output columns c in [3, 61) with J = xs0 + c <= Nphi: .x on lanes 2..30, .y on lanes 1..29
  const bool outx = lane >= 2 && lane <= 30 && xs0 + 2 * lane <= Nphi;
  const bool outy = lane >= 1 && lane <= 29 && xs0 + 2 * lane + 1 <= Nphi;
#define RC(k, i) rc[((i) - ib) * kRowTabW + (k)]
  // four row constants of row i in one shared-memory broadcast (rows are 80-byte aligned)
#define RC4(b, i) (*reinterpret_cast<const float4 *>(rc + ((i) - ib) * kRowTabW + 4 * (b)))
  static_assert(tS0 == 0 && tInvS0 == 1 && tV0 == 2 && tA0 == 3 && tDP0 == 4 && tInvdRc == 5 && tInvR == 6 &&
                    tR == 7 && tInvVol == 8 && tInvdl == 9 && tAphi == 10 && tR32 == 11 && tInvdR == 12 &&
                    tDS0 == 14 && tDV == 15 && tAf == 16 && tInvdRl == 17 && tInvdRr == 18,
                "the float4 groups of the row-constant loads below");
  auto row_ok = [&](int i) { return IN || (i >= 0 && i < Nu); };
  auto first_row = [&](int i) { return !IN && i == 0; };
  auto last_row = [&](int i) { return !IN && i == Nu - 1; };

  if (tid == 0) {  // the tile's row constants: constant tables, independent of the previous kernel
    tc::mbar_arrive_expect_tx(bar_rc, kRcBytesP);
    tc::bulk_load(rc, g.rowtab + (size_t)(ib + kRowTabLead) * kRowTabW, kRcBytesP, bar_rc);
  }
  if (tid < 2 * kMaxModes) {
    bsum[tid] = 0.0;
    zsum[tid] = 0.0;
  }
  // ---- S0 (interior column tiles): sigma, u, w, dPhi of rows i0-3 .. i0+kTileI+2 by TMA,
  // issued before the step info is read so that the two latencies overlap.  With
  // early_state (a time step whose previous kernel only wrote dPhi, so the state's writer
  // completed before it started) the state's boxes go out before the dependence wait. ----
  const int xa = xs0 - 2 * po;  // a multiple of 4 columns (16 bytes)
  if (use_tma && tid == 0 && early_state) {
    tc::mbar_arrive_expect_tx(bar_ld, (FM == kForcePhi ? 4u : 3u) * kFieldBytesP);
    tc::tma_load_2d(sm32t + kOffSgP, tmS, bar_ld, xa, ib);
    tc::tma_load_2d(sm32t + kOffU0P, tmU, bar_ld, xa, ib);
    tc::tma_load_2d(sm32t + kOffW0P, tmW, bar_ld, xa, ib);
  }
  pdl_wait();  // dt, the state and dPhi come from earlier kernels on the stream
  pdl_trigger();
  if (use_tma && tid == 0) {
    if (!early_state) {
      tc::mbar_arrive_expect_tx(bar_ld, (FM == kForcePhi ? 4u : 3u) * kFieldBytesP);
      tc::tma_load_2d(sm32t + kOffSgP, tmS, bar_ld, xa, ib);
      tc::tma_load_2d(sm32t + kOffU0P, tmU, bar_ld, xa, ib);
      tc::tma_load_2d(sm32t + kOffW0P, tmW, bar_ld, xa, ib);
    }
    if (FM == kForcePhi) tc::tma_load_2d(sm32t + kOffPhP, tmP, bar_ld, xa, ib);
  }
  // the step's control fields: loaded now, used once the tile has landed
  const StepRaw sraw = load_step_raw(ctl);
  float lmaxf = 0.f;
  bool bad = false;

  // ---- S0 (edge tiles, caller forces): the same rows by thread loads ----
  if (!use_tma) {
    F2 sv[kItLoadP], pv[kItLoadP], uv[kItLoadP], wv[kItLoadP];
#pragma unroll
    for (int k = 0; k < kItLoadP; ++k) {
      const int r = wp + kWarps32p * k, i = ib + r;
      sv[k] = pv[k] = uv[k] = wv[k] = S(0.f);
      if (r < kRows32t && row_ok(i)) {
        const size_t q = (size_t)i * Nphi + jc;
        sv[k] = *reinterpret_cast<const F2 *>(sig + q);
        uv[k] = *reinterpret_cast<const F2 *>(uu + q);
        wv[k] = *reinterpret_cast<const F2 *>(ww + q);
        if (FM == kForcePhi) pv[k] = *reinterpret_cast<const F2 *>(Phi + q);
      }
    }
#pragma unroll
    for (int k = 0; k < kItLoadP; ++k) {
      const int r = wp + kWarps32p * k;
      if (r < kRows32t) {
        SG[r * L2 + lane] = sv[k];
        U0[r * L2 + lane] = uv[k];
        W0[r * L2 + lane] = wv[k];
        PH[r * L2 + lane] = pv[k];
      }
    }
  }
  __syncthreads();  // thread-loaded fields staged
  {
    bool landed = tc::mbar_wait(bar_rc, 0, &ctl->status);
    if (use_tma) landed = tc::mbar_wait(bar_ld, 0, &ctl->status) && landed;
    if (!landed && tid == 0) {
      // the copies did not land in time: the step is void (status raised); wait once more
      // (bounded) so that no copy is in flight when the CTA exits, then go on with the rest
      tc::mbar_wait(bar_rc, 0, &ctl->status);
      if (use_tma) tc::mbar_wait(bar_ld, 0, &ctl->status);
    }
  }
  const StepInfo si = step_info_from(sraw, true);
  const float dt = (float)si.dt;

  if (!si.active) {
    // pass-through: copy the tile and report the CFL rate of the unchanged state
#pragma unroll
    for (int k = 0; k < kItOutP; ++k) {
      const int i = i0 + wp + kWarps32p * k;
      if (i < Nu) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (e == 0 ? outx : outy) {
            const size_t q = (size_t)i * Nphi + jc + e;
            so[q] = sig[q]; uo[q] = uu[q]; wo[q] = ww[q];
            lmaxf = fmaxf(lmaxf, cfl_rate32(g, i, sig[q], uu[q], ww[q]));
          }
        }
      }
    }
    __syncthreads();
    finish_launch_deferred<kThreads32t>(ctl, si, (double)lmaxf, tid == 0 ? bsum : zsum, red);
    return;
  }

  // ---- S1: pressure perturbation dP of the staged rows ----
#pragma unroll
  for (int k = 0; k < kItLoadP; ++k) {
    const int r = wp + kWarps32p * k, i = ib + r;
    if (r < kRows32t) {
      const F2 s = SG[r * L2 + lane];
      F2 d = S(0.f);
      if (row_ok(i)) {
        if (G2) {
          d = mul(mul(S(g.Kpoly), s), add(S(2.f * RC(tS0, i)), s));
        } else {
          const float P0 = RC(tP0, i), iS0 = RC(tInvS0, i);
          d = make_float2(P0 * expm1f(g.gamma * log1pf(s.x * iS0)), P0 * expm1f(g.gamma * log1pf(s.y * iS0)));
        }
      }
      DP[r * L2 + lane] = d;
    }
  }
  __syncthreads();

  // ---- S2: source kick of rows i0-2 .. i0+kTileI+1 (hydro.hpp:73-96) ----
#pragma unroll
  for (int k = 0; k < kItSrcP; ++k) {
    const int rs = wp + kWarps32p * k, r = rs + 1, i = ib + r;
    if (rs < kSrcRows32t) {  // warp-uniform
      const int x = r * L2 + lane;
      const F2 dc = DP[x];
      // azimuthal neighbours: column 2l-1 is the left lane's .y, 2l+2 the right lane's .x
      const float dl = up1(dc.y), dr = dn1(dc.x);
      F2 pc = S(0.f);
      float pl = 0.f, pr = 0.f;
      if (FM == kForcePhi) {
        pc = PH[x];
        pl = up1(pc.y);
        pr = dn1(pc.x);
      }
      F2 nu1 = S(0.f), nw1 = S(0.f);
      if (row_ok(i)) {
        const float4 c0 = RC4(0, i), c1 = RC4(1, i);  // S0 invS0 V0 a0 | dP0/dR invdRc invR R
        const F2 s_g = SG[x];
        const F2 s = add(S(c0.x), s_g);
        const F2 pim = first_row(i) ? dc : DP[x - L2];
        const F2 pip = last_row(i) ? dc : DP[x + L2];
        const F2 ddP = mul(sub(pip, pim), S(c1.y));
        const F2 dPdphi = mul(sub(make_float2(dc.y, dr), make_float2(dl, dc.x)), S(g.inv2dphi));
        const float iR = c1.z;
        F2 dgR = S(0.f), dgp = S(0.f);
        if (FM == kForcePhi) {
          F2 dPhidu;
          if (first_row(i)) dPhidu = mul(sub(PH[x + L2], pc), S(g.invdu));
          else if (last_row(i)) dPhidu = mul(sub(pc, PH[x - L2]), S(g.invdu));
          else dPhidu = mul(sub(PH[x + L2], PH[x - L2]), S(g.inv2du));
          dgR = mul(dPhidu, S(-iR));
          dgp = mul(mul(sub(make_float2(pc.y, pr), make_float2(pl, pc.x)), S(-g.inv2dphi)), S(iR));
        } else if (FM == kForceArrays) {
          const size_t q = (size_t)i * Nphi + jc;
          dgR = make_float2((float)gRin[q], (float)gRin[q + 1]);
          dgp = make_float2((float)gpin[q], (float)gpin[q + 1]);
        }
        const F2 uc = U0[x], wc = W0[x];  // raw u, w of the point (row r of the staged fields)
        const float V = c0.z;
        const F2 rs = rcp(s);  // one reciprocal for both accelerations
        const F2 q1 = mul(sub(mul(mul(S(c1.x), s_g), S(c0.y)), ddP), rs);
        const F2 aR = add(add(add(S(c0.w), q1), dgR), mul(mul(add(S(2.f * V), wc), wc), S(iR)));
        const F2 q2 = mul(mul(dPdphi, S(-1.f)), mul(rs, S(iR)));
        const F2 ap = sub(add(q2, dgp), mul(mul(uc, add(S(V), wc)), S(iR)));
        nu1 = fma(S(dt), aR, uc);
        nw1 = fma(S(dt), ap, wc);
      }
      U1[rs * L2 + lane] = nu1;
      W1[rs * L2 + lane] = nw1;
    }
  }
  __syncthreads();

  // radial face f (hydro.hpp:107-130): mass flux F, and the fluxes of u and of vphi seen
  // from the rows below (GA) and above (GB) the face
  struct Face { F2 F, FR, GA, GB; };
  auto radial_face = [&](int f) -> Face {
    F2 F = S(0.f), FRv = S(0.f), GAv = S(0.f), GBv = S(0.f);
    if (IN || (f >= 1 && f <= Nu - 1)) {
      const int xs = (f - 2 - ib) * L2 + lane;  // sigma rows f-2 .. f+1
      const int xu = (f - 3 - ib) * L2 + lane;  // u1 / w1 rows f-2 .. f+1
      const F2 s0 = SG[xs], s1 = SG[xs + L2], s2 = SG[xs + 2 * L2], s3 = SG[xs + 3 * L2];
      const F2 u0 = U1[xu], u1 = U1[xu + L2], u2 = U1[xu + 2 * L2], u3 = U1[xu + 3 * L2];
      const F2 w0 = W1[xu], w1 = W1[xu + L2], w2 = W1[xu + 2 * L2], w3 = W1[xu + 3 * L2];
      const F2 vf = mul(S(0.5f), add(u1, u2));
      const bool ux = vf.x > 0.f, uy = vf.y > 0.f;
      const F2 vdt = mul(vf, S(dt));
      // face constants: DS0 / DV of faces f-1, f, f+1; Af, invdRl, invdRr of face f
      const float4 cm = RC4(3, f - 1), cf = RC4(3, f), cp = RC4(3, f + 1), ca = RC4(4, f);
      const F2 hu = mul(S(0.5f), sub(S(1.f), mul(vdt, S(ca.y))));
      const F2 hd = mul(S(-0.5f), add(S(1.f), mul(vdt, S(ca.z))));
      const F2 hf = sel(ux, uy, hu, hd);
      // cells cc-1, cc, cc+1 with cc = f-1 (upwind from below) or f
      const F2 sa = sel(ux, uy, s0, s1), sb = sel(ux, uy, s1, s2), sc = sel(ux, uy, s2, s3);
      const F2 ua = sel(ux, uy, u0, u1), ub = sel(ux, uy, u1, u2), uc = sel(ux, uy, u2, u3);
      const F2 wa = sel(ux, uy, w0, w1), wb = sel(ux, uy, w1, w2), wc = sel(ux, uy, w2, w3);
      const F2 ds_c = sels(ux, uy, cm.z, cf.z), ds_c1 = sels(ux, uy, cf.z, cp.z);
      const F2 dv_c = sels(ux, uy, cm.w, cf.w), dv_c1 = sels(ux, uy, cf.w, cp.w);
      const F2 s0_c = sels(ux, uy, RC(tS0, f - 1), RC(tS0, f));
      F2 kS = vanleer(add(ds_c1, sub(sc, sb)), add(ds_c, sub(sb, sa)));
      F2 kU = vanleer(sub(uc, ub), sub(ub, ua));
      F2 kV = vanleer(add(dv_c1, sub(wc, wb)), add(dv_c, sub(wb, wa)));
      if (!IN) {  // no slope in the first and last cell (hydro.hpp:117-119)
        const int ccx = ux ? f - 1 : f, ccy = uy ? f - 1 : f;
        const bool okx = ccx > 0 && ccx < Nu - 1, oky = ccy > 0 && ccy < Nu - 1;
        kS = sel(okx, oky, kS, S(0.f));
        kU = sel(okx, oky, kU, S(0.f));
        kV = sel(okx, oky, kV, S(0.f));
      }
      const F2 Sf = fma(hf, kS, add(s0_c, sb));
      const F2 uf = fma(hf, kU, ub);
      const float dVf = cf.w;
      const F2 Df = fma(hf, kV, add(sels(ux, uy, 0.f, dVf), wb));  // vphi_f - V0(f-1)
      F = mul(mul(vf, Sf), S(ca.x));
      FRv = mul(F, uf);
      GAv = mul(F, Df);
      GBv = mul(F, sub(Df, S(dVf)));
    }
    return Face{F, FRv, GAv, GBv};
  };

  auto store_face = [&](int fr) {
    const Face fc = radial_face(i0 + fr);
    const int x = fr * LF + lane;
    FF[x] = fc.F; FR[x] = fc.FR; GA[x] = fc.GA; GB[x] = fc.GB;
  };
  // ---- S3: radial faces f = i0 .. i0+kTileI-1, two face rows per warp.  The last face,
  // i0+kTileI, is needed only by row i0+kTileI-1: the warp that gathers that row computes
  // it after the barrier, while the other warps go on (each lane reads back only its own
  // entries, so no further synchronisation is needed). ----
#pragma unroll
  for (int k = 0; k < kItFaceP; ++k) store_face(wp + kWarps32p * k);
  __syncthreads();
  if (wp == (kTileI - 1) % kWarps32p) store_face(kTileI);

  // ---- S4-S6, one output row per warp iteration: radial gather (hydro.hpp:131-139),
  // azimuthal faces 2l and 2l+1 (the left faces of the lane's columns; hydro.hpp:150-170),
  // azimuthal gather, floor (hydro.hpp:69), outputs and CFL rate.  A row's three stages read
  // only that row (neighbour columns by lane shuffles) and the radial fluxes of S3, so they
  // run back to back in registers with no CTA barrier between them. ----
#pragma unroll
  for (int k = 0; k < kItOutP; ++k) {
    const int ri = wp + kWarps32p * k, i = i0 + ri;
    if (IN || i < iend) {  // warp-uniform: every lane takes part in the shuffles below
      const int xs = (i - ib) * L2 + lane, xu = (i - ib - 1) * L2 + lane, xf = ri * LF + lane;
      const float4 c0 = RC4(0, i), c2 = RC4(2, i);  // S0 invS0 V0 a0 | invVol invdl Aphi R32
      const float S0 = c0.x, V = c0.z, iv = c2.x, idl = c2.y, A = c2.z;
      // S4: radial gather
      const F2 sgi = SG[xs], u1i = U1[xu], w1i = W1[xu];
      const F2 s = add(S(S0), sgi);
      const F2 s2 = fma(mul(S(dt), sub(FF[xf], FF[xf + LF])), S(iv), sgi);
      const F2 sn = add(S(S0), s2);
      const F2 dd = make_float2(sn.x < 1e-10f ? 1e-10f : sn.x, sn.y < 1e-10f ? 1e-10f : sn.y);
      const F2 rdd = rcp(dd);
      const F2 u2 = mul(fma(mul(S(dt), sub(FR[xf], FR[xf + LF])), S(iv), mul(s, u1i)), rdd);
      const F2 w2 = mul(fma(mul(S(dt), sub(GB[xf], GA[xf + LF])), S(iv), mul(s, w1i)), rdd);
      // S5: azimuthal faces; columns 2l-2, 2l-1 from the left lane, 2l+2 from the right lane
      F2 fm, fr, fg;
      {
        const F2 sm = s2, um = u2, wm = w2;
        const float sL0 = up1(sm.x), sL1 = up1(sm.y), sR = dn1(sm.x);
        const float uL0 = up1(um.x), uL1 = up1(um.y), uR = dn1(um.x);
        const float wL0 = up1(wm.x), wL1 = up1(wm.y), wR = dn1(wm.x);
        const F2 dv = mul(S(0.5f), add(make_float2(wL1, wm.x), make_float2(wm.x, wm.y)));
        const F2 vf = add(S(V), dv);
        const bool ux = vf.x > 0.f, uy = vf.y > 0.f;
        const F2 vdt = mul(mul(vf, S(dt)), S(idl));
        const F2 hf = sel(ux, uy, mul(S(0.5f), sub(S(1.f), vdt)), mul(S(-0.5f), add(S(1.f), vdt)));
        // face 2l: cells (2l-2, 2l-1, 2l) upwind from the left, else (2l-1, 2l, 2l+1);
        // face 2l+1: (2l-1, 2l, 2l+1) or (2l, 2l+1, 2l+2)
        const F2 sa = make_float2(ux ? sL0 : sL1, uy ? sL1 : sm.x),
                 sb = make_float2(ux ? sL1 : sm.x, uy ? sm.x : sm.y),
                 sc = make_float2(ux ? sm.x : sm.y, uy ? sm.y : sR);
        const F2 ua = make_float2(ux ? uL0 : uL1, uy ? uL1 : um.x),
                 ub = make_float2(ux ? uL1 : um.x, uy ? um.x : um.y),
                 uc = make_float2(ux ? um.x : um.y, uy ? um.y : uR);
        const F2 wa = make_float2(ux ? wL0 : wL1, uy ? wL1 : wm.x),
                 wb = make_float2(ux ? wL1 : wm.x, uy ? wm.x : wm.y),
                 wc = make_float2(ux ? wm.x : wm.y, uy ? wm.y : wR);
        const F2 sf = fma(hf, vanleer(sub(sc, sb), sub(sb, sa)), sb);
        const F2 Sf = add(S(S0), sf);
        const F2 uf = fma(hf, vanleer(sub(uc, ub), sub(ub, ua)), ub);
        const F2 wf = fma(hf, vanleer(sub(wc, wb), sub(wb, wa)), wb);
        const F2 Ffull = mul(mul(vf, Sf), S(A));
        fm = mul(S(A), fma(S(V), sf, mul(dv, Sf)));
        fr = mul(Ffull, uf);
        fg = mul(Ffull, wf);
      }
      // S6: azimuthal gather; the right face of column 2l+1 is the right lane's first face
      const F2 fm1 = make_float2(fm.y, dn1(fm.x)), fr1 = make_float2(fr.y, dn1(fr.x)), fg1 = make_float2(fg.y, dn1(fg.x));
      if (outx || outy) {
        const F2 sn2 = sn;
        F2 s3 = fma(mul(S(dt), sub(fm, fm1)), S(iv), s2);
        const F2 sn3 = add(S(S0), s3);
        const bool flx = sn3.x < 1e-10f, fly = sn3.y < 1e-10f;
        const F2 d = make_float2(flx ? 1e-10f : sn3.x, fly ? 1e-10f : sn3.y);
        const F2 rd = rcp(d);
        const F2 u3 = mul(fma(mul(S(dt), sub(fr, fr1)), S(iv), mul(sn2, u2)), rd);
        const F2 w3 = mul(fma(mul(S(dt), sub(fg, fg1)), S(iv), mul(sn2, w2)), rd);
        s3 = make_float2(flx ? 1e-10f - S0 : s3.x, fly ? 1e-10f - S0 : s3.y);
        const size_t q = (size_t)i * Nphi + jc;
        const float R32 = c2.w;
        const F2 xr = mul(S(R32), s3);
        // split-BF16 operand: one packed conversion per plane, the roundings of split_bf16
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(xr.x, xr.y);
        const float2 hf = __bfloat1622float2(h2);
        const __nv_bfloat162 l2 = __floats2bfloat162_rn(xr.x - hf.x, xr.y - hf.y);
        if (outx && outy) {
          *reinterpret_cast<F2 *>(so + q) = s3;
          *reinterpret_cast<F2 *>(uo + q) = u3;
          *reinterpret_cast<F2 *>(wo + q) = w3;
          *reinterpret_cast<__nv_bfloat162 *>(Sx.hi + q) = h2;
          *reinterpret_cast<__nv_bfloat162 *>(Sx.lo + q) = l2;
        } else if (outx) {  // one half of the pair is output (tile edges)
          so[q] = s3.x; uo[q] = u3.x; wo[q] = w3.x;
          Sx.hi[q] = h2.x;
          Sx.lo[q] = l2.x;
        } else {
          so[q + 1] = s3.y; uo[q + 1] = u3.y; wo[q + 1] = w3.y;
          Sx.hi[q + 1] = h2.y;
          Sx.lo[q + 1] = l2.y;
        }
        // CFL rate of the new state (hydro.hpp:54-57)
        const F2 scl = make_float2(flx ? 1e-10f : sn3.x, fly ? 1e-10f : sn3.y);
        const float gk = g.gamma * g.Kpoly;
        const F2 cs = G2 ? make_float2(sqrt_pos(gk * scl.x), sqrt_pos(gk * scl.y))
                         : make_float2(sqrt_pos(gk * powf(scl.x, g.gamma - 1.f)),
                                       sqrt_pos(gk * powf(scl.y, g.gamma - 1.f)));
        const float idR = RC(tInvdR, i);
        const F2 rate = fma(add(make_float2(fabsf(V + w3.x), fabsf(V + w3.y)), cs), S(idl),
                            mul(add(make_float2(fabsf(u3.x), fabsf(u3.y)), cs), S(idR)));
        if (outx) {
          bad |= !(rate.x == rate.x) || !(u3.x == u3.x) || !(w3.x == w3.x);
          lmaxf = fmaxf(lmaxf, rate.x);
        }
        if (outy) {
          bad |= !(rate.y == rate.y) || !(u3.y == u3.y) || !(w3.y == w3.y);
          lmaxf = fmaxf(lmaxf, rate.y);
        }
        S3[ri * L2 + lane] = s3;
      }
    }
  }
  // mode sums of the new state (output times and per-step diagnostics only)
  if (si.nmodes) {
    __syncthreads();
    const double phx = (jc + 0.5) * (double)g.dphi, phy = (jc + 1.5) * (double)g.dphi;
    for (int m = 0; m < si.nmodes; ++m) {
      double re = 0.0, im = 0.0;
      if (outx || outy) {
        double snx, csx, sny, csy;
        sincos(m * phx, &snx, &csx);
        sincos(m * phy, &sny, &csy);
#pragma unroll 1
        for (int k = 0; k < kItOutP; ++k) {
          const int ri = wp + kWarps32p * k, i = i0 + ri;
          if (i < iend) {
            const F2 s3 = S3[ri * L2 + lane];
            const double dA = g.dAd[i], S0d = g.S0d[i];
            if (outx) {
              const double sf = S0d + (double)s3.x;
              re += sf * csx * dA;
              im -= sf * snx * dA;
            }
            if (outy) {
              const double sf = S0d + (double)s3.y;
              re += sf * csy * dA;
              im -= sf * sny * dA;
            }
          }
        }
      }
      re = warp_sum(re);
      im = warp_sum(im);
      if (lane == 0) {
        atomicAdd(&bsum[2 * m], re);
        atomicAdd(&bsum[2 * m + 1], im);
      }
    }
  }
  __syncthreads();
  double lmax = (double)lmaxf;
  if (bad) lmax = __longlong_as_double(0x7ff8000000000000ll);
  finish_launch_deferred<kThreads32t>(ctl, si, lmax, tid == 0 ? bsum : zsum, red);
#undef RC
}

template <bool G2, int FM>
__global__ void __launch_bounds__(kThreads32t, 4) k_hydro32p(
    const __grid_constant__ CUtensorMap tmS, const __grid_constant__ CUtensorMap tmU,
    const __grid_constant__ CUtensorMap tmW, const __grid_constant__ CUtensorMap tmP,
    const float *__restrict__ sig, const float *__restrict__ uu, const float *__restrict__ ww,
    const float *__restrict__ Phi, const double *__restrict__ gRin, const double *__restrict__ gpin,
    float *__restrict__ so, float *__restrict__ uo, float *__restrict__ wo, SplitBf16 Sx, Ctl *ctl, Rows32 g,
    int *rowpend, int early_state) {
  extern __shared__ __align__(16) uint8_t sm32p_raw[];
  // TMA destinations: the field offsets are multiples of 128 bytes from a 128-aligned base
  float *sm32t = reinterpret_cast<float *>(((uintptr_t)sm32p_raw + 127) & ~(uintptr_t)127);
  __shared__ double red[kThreads32t / 32];
  __shared__ double bsum[2 * kMaxModes], zsum[2 * kMaxModes];
  __shared__ __align__(8) uint64_t bar_ld, bar_rc;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar_ld, 1);
    tc::mbar_init(&bar_rc, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // (the first CTA barrier inside the tile function orders the set-up before any wait)
  const int i0 = blockIdx.y * kTileI;
  if (i0 >= 3 && i0 + kTileI + 3 <= g.Nu)
    hydro32p_tile<G2, FM, true>(sig, uu, ww, Phi, gRin, gpin, so, uo, wo, Sx, ctl, g, sm32t, red, bsum, zsum, &tmS,
                                &tmU, &tmW, &tmP, &bar_ld, &bar_rc, early_state != 0);
  else
    hydro32p_tile<G2, FM, false>(sig, uu, ww, Phi, gRin, gpin, so, uo, wo, Sx, ctl, g, sm32t, red, bsum, zsum, &tmS,
                                 &tmU, &tmW, &tmP, &bar_ld, &bar_rc, early_state != 0);
  if (rowpend) rowtile_done(rowpend + blockIdx.y);  // this tile's outputs are written
}

// One step of a group of disks of the same grid (batched sweeps) with their own
// self-gravity: blockIdx.z is the disk.  Each disk's fields, state tensor maps and row
// tables come from a device array, and its tiles run exactly the single-disk kernel's
// code (b: the ping-pong buffer that holds the input state).  The tile form below reads
// the same entries and ignores the maps.
struct __align__(64) HydroDisk {
  CUtensorMap tmS[2], tmU[2], tmW[2], tmP;  // sigma, u, w of both ping-pong buffers; dPhi
  float *sig[2], *u[2], *w[2];
  const float *dPhi;
  SplitBf16 Sx;
  Ctl *ctl;
  Rows32 g;
};

template <bool G2>
__global__ void __launch_bounds__(kThreads32t, 4) k_hydro32p_group(const HydroDisk *__restrict__ disks, int b) {
  extern __shared__ __align__(16) uint8_t sm32p_raw[];
  float *sm32t = reinterpret_cast<float *>(((uintptr_t)sm32p_raw + 127) & ~(uintptr_t)127);
  __shared__ double red[kThreads32t / 32];
  __shared__ double bsum[2 * kMaxModes], zsum[2 * kMaxModes];
  __shared__ __align__(8) uint64_t bar_ld, bar_rc;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar_ld, 1);
    tc::mbar_init(&bar_rc, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const HydroDisk &d = disks[blockIdx.z];
  const int o = b ^ 1;
  const int i0 = blockIdx.y * kTileI;
  // the predecessor (the group's inverse phi product) writes only dPhi: early state loads
  if (i0 >= 3 && i0 + kTileI + 3 <= d.g.Nu)
    hydro32p_tile<G2, kForcePhi, true>(d.sig[b], d.u[b], d.w[b], d.dPhi, nullptr, nullptr, d.sig[o], d.u[o], d.w[o],
                                       d.Sx, d.ctl, d.g, sm32t, red, bsum, zsum, &d.tmS[b], &d.tmU[b], &d.tmW[b],
                                       &d.tmP, &bar_ld, &bar_rc, true);
  else
    hydro32p_tile<G2, kForcePhi, false>(d.sig[b], d.u[b], d.w[b], d.dPhi, nullptr, nullptr, d.sig[o], d.u[o], d.w[o],
                                        d.Sx, d.ctl, d.g, sm32t, red, bsum, zsum, &d.tmS[b], &d.tmU[b], &d.tmW[b],
                                        &d.tmP, &bar_ld, &bar_rc, true);
}

template <bool G2>
__global__ void __launch_bounds__(kThreads32t, 4) k_hydro32t_group(const HydroDisk *__restrict__ disks, int b) {
  extern __shared__ float sm32t[];
  __shared__ double red[kThreads32t / 32];
  __shared__ double bsum[2 * kMaxModes], zsum[2 * kMaxModes];
  const HydroDisk &d = disks[blockIdx.z];
  const int o = b ^ 1;
  const int i0 = blockIdx.y * kTileI;
  if (i0 >= 3 && i0 + kTileI + 3 <= d.g.Nu)
    hydro32t_tile<G2, kForcePhi, true>(d.sig[b], d.u[b], d.w[b], d.dPhi, nullptr, nullptr, d.sig[o], d.u[o], d.w[o],
                                       d.Sx, d.ctl, d.g, sm32t, red, bsum, zsum);
  else
    hydro32t_tile<G2, kForcePhi, false>(d.sig[b], d.u[b], d.w[b], d.dPhi, nullptr, nullptr, d.sig[o], d.u[o],
                                        d.w[o], d.Sx, d.ctl, d.g, sm32t, red, bsum, zsum);
}

}  // namespace dg
