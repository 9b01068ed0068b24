// Tensor-core batched step with an exactly accumulated main product (sm_100a).
//
// The block SpMM of one element row and one 64-shot tile,
//   Y[shot][r] = sum_b sum_c X_b[shot][c] * B_b[r][c],
// runs on the 5th-generation tensor cores in BF16 with FP32 accumulation in
// tensor memory. Both operands are written in fixed point with a shared
// power-of-two scale per accumulated row (per shot and element tile for the
// state, per block row for the operator):
//   x = 2^(ex-8) * (x0 + x1 + x2),  x0 = q1, x1 = q2/2^8, x2 = q3/2^16,
//   |q1| <= 256, |q2|, |q3| <= 128,
// each term exactly representable in BF16 ("slice planes" 0, 1, 2).
// The products of plane p of the state and plane q of the operator are
// summed by weight class g = p + q (g <= 3; the g = 4 term is below 2^-32 of
// the result). Class 0 (x0 * b0) is a sum of integers below 2^16 whose total
// stays below 2^24: it is exact whatever rounding the tensor core applies to
// its FP32 sums. Classes 1..3 are 2^-7 and smaller, so their rounding is
// ~2^-31 of the result. The epilogue scales each block's classes and sums the
// row's blocks in FP64: no biased rounding reaches the leap-frog recurrence.
//
// One MMA covers one state plane p against the operator planes concatenated
// along N ([b0 | b1 | b2], each GW columns), writing classes p, p+1, p+2 of
// the accumulator slot at column p*GW: K/16 x 3 MMAs per block (one more at
// the first K step, which initialises class 3 on its own).
//
// Data flow, all on-chip between HBM reads and writes:
//   * operator slices: built once (k_make_bslices) as an image of the
//     shared-memory operand layout, one contiguous image per block;
//   * state slices: written by the previous step's epilogue (or
//     k_make_xslices) as one contiguous image per element and 64-shot tile;
//   * warp 0 (one lane) streams both images of each block, and the block's
//     scales, into shared-memory rings with bulk copies completing on
//     mbarriers;
//   * warp 1 (one lane) issues the MMAs (MN-major, no swizzle) into a ring of
//     per-block accumulator slots in tensor memory and commits them to
//     mbarriers;
//   * warps 2..9 read the accumulators (tcgen05.ld) and sum the row's blocks
//     in FP64 into one of two shared-memory row-sum buffers;
//   * warps 10..17 take the previous item's row sums, run the leap-frog
//     update (state tile staged in shared memory by cp.async), the source,
//     the receivers and the energy, and write u^{k+1} and its slices for the
//     next step, while the readers work on the next item.
// Every wait is bounded: on a timeout the CTA sets the error word, stops,
// waits (bounded) for its own copies and MMAs, frees its tensor memory and
// returns.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "tsp_kernels.cuh"
#include "tsp_tcgen05.cuh"

namespace tsp {

template <int R>
struct FxCfg {
  static constexpr int NP = R / 2;
  static constexpr int M = 64;                    // shots per tile (MMA M)
  static constexpr int GW = (R + 15) & ~15;       // columns of one weight class (operator rows, padded)
  static constexpr int KPAD = (R + 15) & ~15;     // MMA K per block
  static constexpr int NPL = 3;                   // slice planes per operand
  static constexpr int LBO_A = (M / 8) * 128;     // bytes between K groups (A)
  static constexpr int APLANE = KPAD * M * 2;     // one slice plane of an element tile
  static constexpr int ABYTES = NPL * APLANE;     // element-tile image: [plane][kgroup][mgroup][8 x 16 B]
  static constexpr int BPL_KG = (GW / 8) * 128;   // one plane within a K group
  static constexpr int LBO_B = NPL * BPL_KG;      // bytes between K groups (B): [kgroup][plane][ngroup][8 x 16 B]
  static constexpr int BBYTES = (KPAD / 8) * LBO_B;
  static constexpr int STAGE = ABYTES + BBYTES;
  static constexpr int NCLS = 4;                  // weight classes 0..3
  static constexpr int SLOTW = NCLS * GW <= 64 ? 64 : NCLS * GW <= 128 ? 128 : 256;
  static constexpr int NACC = 512 / SLOTW > 4 ? 4 : 512 / SLOTW;  // accumulator slots (blocks in flight)
  static constexpr int TCOLS = NACC * SLOTW;
  static constexpr int YS = R + 1;                // FP64 row-sum stride (odd: conflict-free columns)
  static constexpr int NRD = 8;                   // reader warps: two per tensor-memory lane quadrant
  static constexpr int NUP = 8;                   // update warps
  static constexpr int NUPT = 32 * NUP;
  static constexpr int NT = 32 * (2 + NRD + NUP);
  static constexpr int NSC = 8;                   // scale ring (per block: state scales, row scales)
  static constexpr int SCW = M + GW;              // floats per scale-ring entry
  static constexpr int TILE = M * R;              // doubles of one state tile (64 shots x 2Np)
  static constexpr int NBAR_MAX = 2 * 16 + 2 * 4 + 2 * NSC + 4 + 1;
  static constexpr size_t FIXED = size_t(2) * M * YS * 8 + size_t(2) * TILE * 8 + 64 * 8 + NUP * 8 +
                                  size_t(NSC) * SCW * 4 + 64 * 4 * 2 + NBAR_MAX * 8 + 16;
  static constexpr size_t BUDGET = 227 * 1024 - 1024;
  static constexpr int NST_FIT = int((BUDGET - FIXED) / STAGE);
  static constexpr int NST = NST_FIT > 8 ? 8 : NST_FIT;
  static constexpr size_t smem_bytes() { return size_t(NST) * STAGE + FIXED; }
  static_assert(NST >= 2, "shared memory too small for two stages");
  static_assert(3 * GW <= 256, "MMA N");
  static_assert(TCOLS <= 512 && TCOLS >= 32, "tensor memory");
  static_assert(TCOLS < 512 || smem_bytes() > 116 * 1024, "512 TMEM columns need one CTA per SM");
};

__device__ __forceinline__ void fx_mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fx_mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fx_mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Bulk copy global -> this CTA's shared memory, completing on an mbarrier
// (plain load: no multicast).
__device__ __forceinline__ void fx_bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// Bounded wait that also gives up when another role has aborted; false on
// timeout or abort (a timeout raises the abort flag).
__device__ __forceinline__ bool fx_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    if (mbar_try(bar, parity)) return true;
    if (*abort_flag) return false;
    if (clock64() - t0 > (1ll << 31)) {
      *abort_flag = 1;
      return false;
    }
  }
}
template <int NTHR>
__device__ __forceinline__ void fx_epi_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(NTHR) : "memory");
}

// Shared exponent of a row whose largest magnitude is m: 2^(ex-1) <= m < 2^ex,
// read from the bits (zero, subnormal, infinite and NaN rows: kNoExp, i.e.
// the row counts as zero). A state row holding a NaN or an infinity, or a
// value of 2^1000 or more (a run that is overflowing), gets kNaNExp instead:
// its slices are zero and its scale is NaN, so every product it enters
// becomes NaN and the neighbours' rows carry the failure on, as the FP64
// recurrence would.
constexpr int kNoExp = -2147483647 - 1;
constexpr int kNaNExp = 2147483647;
__device__ __forceinline__ int fx_exponent(double m) {
  const int f = int((__double_as_longlong(m) >> 52) & 0x7FF);
  return (f == 0 || f == 0x7FF) ? kNoExp : f - 1022;
}
__device__ __forceinline__ bool fx_valid(int ex) { return ex >= -900 && ex <= 1000; }
// 2^n from its bits (n in [-1022, 1023]).
__device__ __forceinline__ double fx_pow2(int n) { return __longlong_as_double((long long)(n + 1023) << 52); }
// Factor 2^(24-ex) mapping a row into the 24-bit fixed-point grid (0 for a zero row).
__device__ __forceinline__ double fx_factor24(int ex) { return fx_valid(ex) ? fx_pow2(24 - ex) : 0.0; }
// Row scales of a block product whose class sum is counted in units of
// 2^-8: 2^(ex-8) * 2^(eb-8) * 2^-8 = fx_shot_scale(ex) * fx_row_scale(eb)
// (0 for a zero row).
__device__ __forceinline__ double fx_shot_scale(int ex) {
  return fx_valid(ex) ? fx_pow2(ex - 24) : (ex == kNaNExp ? __longlong_as_double(0x7FF8000000000000ll) : 0.0);
}
__device__ __forceinline__ double fx_row_scale(int eb) { return fx_valid(eb) ? fx_pow2(eb) : 0.0; }

// BF16 bits of q * scale for a small integer q (|q| <= 256) and a power of
// two scale: exact, so the FP32 bits truncate to BF16 without rounding.
__device__ __forceinline__ uint32_t fx_bf16_bits(int q, float scale) {
  return __float_as_uint((__int_as_float(0x4B400000 + q) - 12582912.0f) * scale) >> 16;
}
// Fixed-point slices of v with fac = 2^(24-ex): W = rint(v * fac) (one FMA
// against 1.5 * 2^52), W = q1 * 2^16 + q2 * 2^8 + q3 with |q1| <= 256 and
// |q2|, |q3| <= 128; planes q1, q2 / 2^8, q3 / 2^16 as BF16 bits.
__device__ __forceinline__ void fx_slice_bits(double v, double fac, uint32_t& b0, uint32_t& b1, uint32_t& b2) {
  // |W| < 2^25 and the low word of 1.5 * 2^52 is zero: W is the low word.
  const int w = __double2loint(fma(v, fac, 6755399441055744.0));
  const int q1 = (w + 32768) >> 16;
  const int rest = w - (q1 << 16);
  const int q2 = (rest + 128) >> 8;
  const int q3 = rest - (q2 << 8);
  b0 = fx_bf16_bits(q1, 1.0f);
  b1 = fx_bf16_bits(q2, 1.0f / 256.0f);
  b2 = fx_bf16_bits(q3, 1.0f / 65536.0f);
}
// Exact class sum of one accumulator entry in units of 2^-8, as a double:
// g0 is the exact integer main class (|g0| < 2^22), c the sum of the
// correction classes (|c| < 2^14), rounded to 2^-8.
__device__ __forceinline__ double fx_class_sum(float g0, float c) {
  const int i0 = __float_as_int(g0 + 12582912.0f) - 0x4B400000;
  const int ic = __float_as_int(fmaf(c, 256.0f, 12582912.0f)) - 0x4B400000;
  const int V = i0 * 256 + ic;  // |V| < 2^31
  return __hiloint2double(0x43300000, V ^ int(0x80000000)) - 4503601774854144.0;  // 2^52 + 2^31
}

// 16 lanes x 8 columns: thread t holds lanes t/4 and t/4 + 8, columns
// 2(t%4) and 2(t%4) + 1 ({lane t/4: col, col+1; lane t/4+8: col, col+1}).
__device__ __forceinline__ void fx_ld16x8(uint32_t addr, uint32_t* v) {
  asm volatile("tcgen05.ld.sync.aligned.16x256b.x1.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(addr));
}

template <int R>
__global__ void __launch_bounds__(FxCfg<R>::NT, 1) k_step_batched_fx(const StepParams p, int* err_flag) {
  typedef FxCfg<R> CF;
  constexpr int NP = CF::NP, GW = CF::GW, KPAD = CF::KPAD, M = CF::M, NST = CF::NST, NACC = CF::NACC;
  constexpr int YS = CF::YS, NSC = CF::NSC, SCW = CF::SCW, NUPT = CF::NUPT, TILE = CF::TILE;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* stages = smem;
  double* Ysb = reinterpret_cast<double*>(smem + size_t(NST) * CF::STAGE);  // [2][M][YS] row sums, then u^{k+1}
  double* Stu = Ysb + 2 * M * YS;                                             // [TILE] u^k of the tile
  double* Stp = Stu + TILE;                                                   // [TILE] u^{k-1} (or v^0) of the tile
  double* shfac = Stp + TILE;                                                 // [64]
  double* red = shfac + 64;                                                   // [NUP]
  int* scl = reinterpret_cast<int*>(red + CF::NUP);                           // [NSC][SCW]: state exps[64], row exps[GW]
  int* shexp = reinterpret_cast<int*>(scl + NSC * SCW);                       // [64]
  int* msrc = shexp + 64;                                                     // [64]
  uint64_t* bars = reinterpret_cast<uint64_t*>(msrc + 64);
  uint64_t* bfull = bars;          // [NST]  stage landed (loader arrival + bytes)
  uint64_t* bempty = bfull + NST;  // [NST]  stage read by the MMAs (commit)
  uint64_t* baccf = bempty + NST;  // [NACC] accumulators ready (commit)
  uint64_t* bacce = baccf + NACC;  // [NACC] accumulators read (reader warps)
  uint64_t* bscf = bacce + NACC;   // [NSC]  scales landed
  uint64_t* bsce = bscf + NSC;     // [NSC]  scales read (reader warps)
  uint64_t* byf = bsce + NSC;      // [2]    row sums written (reader warps)
  uint64_t* bye = byf + 2;         // [2]    row sums consumed (update warps)
  uint64_t* bdrain = bye + 2;
  uint32_t* tmem_s = reinterpret_cast<uint32_t*>(bdrain + 1);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_s + 1);

  // After a timed-out launch the results are void: later launches of the
  // same run return at once instead of timing out one by one.
  if (*reinterpret_cast<volatile int*>(err_flag) != 0) return;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  if (t == 0) {
    *abort_s = 0;
    for (int i = 0; i < NST; ++i) {
      fx_mbar_init(smem_u32(&bfull[i]), 1);
      fx_mbar_init(smem_u32(&bempty[i]), 1);
    }
    for (int i = 0; i < NACC; ++i) {
      fx_mbar_init(smem_u32(&baccf[i]), 1);
      fx_mbar_init(smem_u32(&bacce[i]), CF::NRD);
    }
    for (int i = 0; i < NSC; ++i) {
      fx_mbar_init(smem_u32(&bscf[i]), 1);
      fx_mbar_init(smem_u32(&bsce[i]), CF::NRD);
    }
    for (int i = 0; i < 2; ++i) {
      fx_mbar_init(smem_u32(&byf[i]), CF::NRD);
      fx_mbar_init(smem_u32(&bye[i]), CF::NUP);
    }
    fx_mbar_init(smem_u32(bdrain), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_s)),
                 "r"(CF::TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_s;

  const int S = p.S;
  const int ntile = (S + M - 1) / M;
  const long long nitems = (long long)p.ne * ntile;
  const long long G = gridDim.x;

  if (warp == 0) {
    // ---------------- loader: one lane streams the operand images and scales ----------------
    if (lane == 0) {
      const unsigned char* xsl_in = reinterpret_cast<const unsigned char*>(p.xsl_in);
      const unsigned char* bsl = reinterpret_cast<const unsigned char*>(p.bsl);
      uint32_t j = 0;
      long long item = blockIdx.x;
      // Row of the current item (loaded once here, then one item ahead).
      int rb = 0, nb = 0, cols[4] = {0, 0, 0, 0};
      if (item < nitems) {
        const int e0 = int(item / ntile);
        row_span(p, e0, rb, nb);
#pragma unroll
        for (int b = 0; b < 4; ++b) cols[b] = b < nb ? col_at(p, rb + b) : 0;
      }
      bool ok = true;
      for (; item < nitems && ok; item += G) {
        const int tile = int(item % ntile);
        const long long nxt = item + G;
        int rbn = 0, nbn = 0, coln[4] = {0, 0, 0, 0};
        if (nxt < nitems) {
          const int en = int(nxt / ntile);
          row_span(p, en, rbn, nbn);
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          if (b >= nb) break;
          const int s = int(j % NST), sc = int(j % NSC);
          const uint32_t n = j / NST, nsc = j / NSC;
          if ((n > 0 && !fx_wait(smem_u32(&bempty[s]), (n - 1) & 1, abort_s)) ||
              (nsc > 0 && !fx_wait(smem_u32(&bsce[sc]), (nsc - 1) & 1, abort_s))) {
            ok = false;
            break;
          }
          const int c = cols[b];
          const uint32_t dst = smem_u32(stages + size_t(s) * CF::STAGE);
          fx_mbar_arrive_tx(smem_u32(&bfull[s]), CF::STAGE);
          fx_bulk_g2s(dst, xsl_in + (size_t(c) * ntile + tile) * CF::ABYTES, CF::ABYTES, smem_u32(&bfull[s]));
          fx_bulk_g2s(dst + CF::ABYTES, bsl + size_t(rb + b) * CF::BBYTES, CF::BBYTES, smem_u32(&bfull[s]));
          const uint32_t sd = smem_u32(scl + sc * SCW);
          fx_mbar_arrive_tx(smem_u32(&bscf[sc]), SCW * 4);
          fx_bulk_g2s(sd, p.xex_in + (size_t(c) * ntile + tile) * M, M * 4, smem_u32(&bscf[sc]));
          fx_bulk_g2s(sd + M * 4, p.bex + size_t(rb + b) * GW, GW * 4, smem_u32(&bscf[sc]));
          ++j;
          if (b == 0 && nxt < nitems) {
#pragma unroll
            for (int bb = 0; bb < 4; ++bb) coln[bb] = bb < nbn ? col_at(p, rbn + bb) : 0;
          }
        }
        rb = rbn;
        nb = nbn;
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) cols[bb] = coln[bb];
      }
      // Every issued copy must land before the CTA ends (bounded; the
      // copies themselves always complete).
      const long long t0 = clock64();
      for (int s = 0; s < NST; ++s) {
        if (j <= uint32_t(s)) continue;
        const uint32_t uses = (j - 1 - s) / NST + 1;
        while (!mbar_try(smem_u32(&bfull[s]), (uses - 1) & 1) && clock64() - t0 < (1ll << 31)) {
        }
      }
      for (int s = 0; s < NSC; ++s) {
        if (j <= uint32_t(s)) continue;
        const uint32_t uses = (j - 1 - s) / NSC + 1;
        while (!mbar_try(smem_u32(&bscf[s]), (uses - 1) & 1) && clock64() - t0 < (1ll << 31)) {
        }
      }
      if (clock64() - t0 >= (1ll << 31)) *abort_s = 1;
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer: one lane ----------------
    if (lane == 0) {
      const uint32_t id3 = umma_idesc_bf16_mn(M, 3 * GW), id2 = umma_idesc_bf16_mn(M, 2 * GW),
                     id1 = umma_idesc_bf16_mn(M, GW);
      // Descriptors of stage 0; other stages, planes and K steps add a
      // constant to the 14-bit start-address field (no carry: < 2^18 bytes).
      const uint64_t dA0 = umma_desc(smem_u32(stages), CF::LBO_A, 128);
      const uint64_t dB0 = umma_desc(smem_u32(stages) + CF::ABYTES, CF::LBO_B, 128);
      constexpr uint32_t PA = CF::APLANE >> 4, KA = (2 * CF::LBO_A) >> 4, KB = (2 * CF::LBO_B) >> 4;
      constexpr uint32_t B2 = (2 * CF::BPL_KG) >> 4;
      uint32_t j = 0;
      long long item = blockIdx.x;
      int nb = 0;
      if (item < nitems) {
        const int e0 = int(item / ntile);
        int rb0;
        row_span(p, e0, rb0, nb);
      }
      bool ok = true;
      for (; item < nitems && ok; item += G) {
        const long long nxt = item + G;
        int rp0 = 0, rp1 = 0;
        if (nxt < nitems) {
          const int en = int(nxt / ntile);
          int nbx;
          row_span(p, en, rp0, nbx);
          rp1 = rp0 + nbx;
        }
        for (int b = 0; b < nb; ++b, ++j) {
          const int s = int(j % NST), a = int(j % NACC);
          const uint32_t na = j / NACC;
          if (!fx_wait(smem_u32(&bfull[s]), (j / NST) & 1, abort_s) ||
              (na > 0 && !fx_wait(smem_u32(&bacce[a]), (na - 1) & 1, abort_s))) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint64_t soff = uint64_t((s * CF::STAGE) >> 4);
          const uint64_t da = dA0 + soff, db = dB0 + soff;
          const uint32_t d0 = tmem + uint32_t(a * CF::SLOTW);
          // K step 0: plane 0 x [b0|b1|b2] initialises classes 0..2, plane 1
          // x [b0|b1] adds to 1..2, plane 1 x b2 initialises class 3, plane 2
          // x [b0|b1] adds to 2..3.
          umma_bf16(d0, da, db, id3, 0u);
          umma_bf16(d0 + GW, da + PA, db, id2, 1u);
          umma_bf16(d0 + 3 * GW, da + PA, db + B2, id1, 0u);
          umma_bf16(d0 + 2 * GW, da + 2 * PA, db, id2, 1u);
#pragma unroll
          for (int ks = 1; ks < KPAD / 16; ++ks) {
            umma_bf16(d0, da + ks * KA, db + ks * KB, id3, 1u);
            umma_bf16(d0 + GW, da + PA + ks * KA, db + ks * KB, id3, 1u);
            umma_bf16(d0 + 2 * GW, da + 2 * PA + ks * KA, db + ks * KB, id2, 1u);
          }
          umma_commit(smem_u32(&bempty[s]));
          umma_commit(smem_u32(&baccf[a]));
        }
        nb = rp1 - rp0;
      }
      // Drain: every issued MMA completes before the tensor memory is freed.
      umma_commit(smem_u32(bdrain));
      const long long t0 = clock64();
      while (!mbar_try(smem_u32(bdrain), 0))
        if (clock64() - t0 > (1ll << 31)) {
          *abort_s = 1;
          break;
        }
    }
  } else if (warp < 2 + CF::NRD) {
    // ---------------- readers: warps 2..9, tensor memory -> FP64 row sums ----------------
    // Warp (quadrant sp, half hf) reads 16-lane x 8-column chunks ch0..ch0+CPW-1
    // of its quadrant: thread t holds shots 16sp + t/4 and 16sp + t/4 + 8,
    // rows 8ch + 2(t%4) and 8ch + 2(t%4) + 1 of every chunk.
    const int rw = warp - 2;  // 0..7
    const int sp = warp & 3;  // tensor-memory lane quadrant of this warp
    constexpr int NCH = GW / 8, CPW = (NCH + 1) / 2;
    const int ch0 = (rw >> 2) * CPW;
    const int sha = 16 * sp + (lane >> 2), shb = sha + 8;  // the thread's two shots
    const int rc = 2 * (lane & 3);                          // its first row within a chunk
    const uint32_t lane_base = tmem + (uint32_t(32 * sp) << 16);
    uint32_t j = 0, li = 0;
    long long item = blockIdx.x;
    int rp0 = 0, rp1 = 0;
    if (item < nitems) {
      const int e0 = int(item / ntile);
      int nbx;
      row_span(p, e0, rp0, nbx);
      rp1 = rp0 + nbx;
    }
    bool ok = true;
    for (; item < nitems && ok; item += G, ++li) {
      const int nb = rp1 - rp0;
      const long long nxt = item + G;
      if (nxt < nitems) {
        const int en = int(nxt / ntile);
        int nbx;
        row_span(p, en, rp0, nbx);
        rp1 = rp0 + nbx;
      }
      // yacc[4 i + 2 v + h]: shot (v ? shb : sha), row 8(ch0 + i) + rc + h;
      // the row's blocks accumulate in registers, in FP64, in block order.
      double yacc[CPW * 4];
#pragma unroll
      for (int i = 0; i < CPW * 4; ++i) yacc[i] = 0.0;
      for (int b = 0; b < nb; ++b, ++j) {
        const int a = int(j % NACC), sc = int(j % NSC);
        const bool got = fx_wait(smem_u32(&bscf[sc]), (j / NSC) & 1, abort_s) &&
                         fx_wait(smem_u32(&baccf[a]), (j / NACC) & 1, abort_s);
        if (!__all_sync(0xffffffffu, got)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int* sv = scl + sc * SCW;
        const double ssa = fx_shot_scale(sv[sha]), ssb = fx_shot_scale(sv[shb]);
        // Chunk i+1 is loaded while chunk i is summed (two register sets).
        uint32_t g[2][4][4];  // [buffer][class][value]
        {
          const uint32_t ad = lane_base + uint32_t(a * CF::SLOTW + 8 * ch0);
#pragma unroll
          for (int cl = 0; cl < 4; ++cl) fx_ld16x8(ad + cl * GW, g[0][cl]);
        }
#pragma unroll
        for (int i = 0; i < CPW; ++i) {
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (i + 1 < CPW && ch0 + i + 1 < NCH) {
            const uint32_t ad = lane_base + uint32_t(a * CF::SLOTW + 8 * (ch0 + i + 1));
#pragma unroll
            for (int cl = 0; cl < 4; ++cl) fx_ld16x8(ad + cl * GW, g[(i + 1) & 1][cl]);
          }
          if (ch0 + i < NCH) {
            const int r0 = 8 * (ch0 + i) + rc;
            const double rs0 = fx_row_scale(sv[M + r0]), rs1 = fx_row_scale(sv[M + r0 + 1]);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int h = q & 1, v = q >> 1;
              if (r0 + h < R) {
                const uint32_t* gg = &g[i & 1][0][0];
                const float c = __uint_as_float(gg[4 + q]) + __uint_as_float(gg[8 + q]) + __uint_as_float(gg[12 + q]);
                yacc[4 * i + q] =
                    fma(fx_class_sum(__uint_as_float(gg[q]), c) * (v ? ssb : ssa), h ? rs1 : rs0, yacc[4 * i + q]);
              }
            }
          }
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        // The values are in registers: the accumulator slot and the scale
        // entry are free again.
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          fx_mbar_arrive(smem_u32(&bacce[a]));
          fx_mbar_arrive(smem_u32(&bsce[sc]));
        }
      }
      if (!ok) break;
      // Hand the row sums to the update warps through buffer li % 2.
      const int bf = int(li & 1);
      const uint32_t nuse = li >> 1;
      if (nuse > 0 && !__all_sync(0xffffffffu, fx_wait(smem_u32(&bye[bf]), (nuse - 1) & 1, abort_s))) break;
      double* Ys = Ysb + bf * M * YS;
#pragma unroll
      for (int i = 0; i < CPW; ++i) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int h = q & 1, v = q >> 1;
          const int r = 8 * (ch0 + i) + rc + h;
          if (ch0 + i < NCH && r < R) Ys[(v ? shb : sha) * YS + r] = yacc[4 * i + q];
        }
      }
      __syncwarp();
      if (lane == 0) fx_mbar_arrive(smem_u32(&byf[bf]));
    }
  } else {
    // ---------------- update warps: 10..17 ----------------
    const int uw = warp - 2 - CF::NRD;  // 0..7
    const int ut = t - 32 * (2 + CF::NRD);
    const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
    const double dt = p.dt;
    unsigned char* xsl_out = reinterpret_cast<unsigned char*>(p.xsl_out);
    // The tile's u^k and u^{k-1} (contiguous, nsv*R doubles each) are copied
    // into shared memory with cp.async during the previous item's slicing.
    auto stage_state = [&](long long it) {
      if (it >= nitems) return;
      const int e2 = int(it / ntile), t2 = int(it - (long long)e2 * ntile);
      const int s02 = t2 * M, nsv2 = min(M, S - s02);
      const double* xb = p.x + (size_t(e2) * S + s02) * R;
      const double* pb = p.uprev ? p.uprev + (size_t(e2) * S + s02) * R : nullptr;
      const int n16 = nsv2 * R / 2;
      for (int i = ut; i < n16; i += NUPT) {
        cp_async16(Stu + 2 * i, xb + 2 * i);
        if (pb) cp_async16(Stp + 2 * i, pb + 2 * i);
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // Scalars of the next item, loaded one item ahead.
    int q0_n = 0, q1_n = 0, src_n = -1;
    double mi_n = 0.0;
    auto prefetch = [&](long long it) {
      if (it >= nitems) return;
      const int e2 = int(it / ntile), t2 = int(it - (long long)e2 * ntile);
      const int s02 = t2 * M, nsv2 = min(M, S - s02);
      mi_n = p.minv[e2];
      if (p.rcv_ptr != nullptr) {
        q0_n = rcv_ptr_at(p, e2);
        q1_n = rcv_ptr_at(p, e2 + 1);
      }
      src_n = (ut < nsv2) ? src_elem_at(p, s02 + ut) : -1;
    };
    // A warp that gives up (timeout or another role's abort) keeps walking
    // the item loop without work so that every named barrier below is still
    // reached by all update warps.
    bool dead = false;
    uint32_t li = 0;
    stage_state(blockIdx.x);
    prefetch(blockIdx.x);
    for (long long item = blockIdx.x; item < nitems; item += G, ++li) {
      const int e = int(item / ntile), tile = int(item - (long long)e * ntile);
      const int s0 = tile * M;
      const int nsv = min(M, S - s0);
      const int q0 = q0_n, q1 = q1_n;
      const double mi = mi_n;
      const int bf = int(li & 1);
      double* Ys = Ysb + bf * M * YS;
      if (ut < M) {
        shexp[ut] = kNoExp;
        msrc[ut] = src_n;
      }
      if (!dead && !__all_sync(0xffffffffu, fx_wait(smem_u32(&byf[bf]), (li >> 1) & 1, abort_s))) dead = true;
      asm volatile("cp.async.wait_group 0;" ::: "memory");
      fx_epi_sync<NUPT>();
      // ---- leap-frog update; exponents by shot ----
      double en = 0.0;
      if (!dead) {
        for (int w = ut; w < nsv * NP; w += NUPT) {
          const int s2 = w / NP, q = w - s2 * NP;
          const int sh = s0 + s2, r0 = 2 * q;
          const bool is_src = (msrc[s2] == e) && (k < p.nF);
          const double2 uu = reinterpret_cast<const double2*>(Stu)[w];
          const double2 up = p.uprev ? reinterpret_cast<const double2*>(Stp)[w] : make_double2(0.0, 0.0);
          const double u[2] = {uu.x, uu.y}, upv[2] = {up.x, up.y};
          double un[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = r0 + h;
            const int cmp = r / NP, ii = r - cmp * NP;
            const double f = is_src ? p.F[(size_t(sh) * p.nF + k) * 2 + cmp] * p.src_phi[size_t(sh) * NP + ii] : 0.0;
            const double y = Ys[s2 * YS + r];
            if (p.mode == kModeStep) un[h] = (2 * u[h] - upv[h]) + mi * ((-dt * dt) * (y - f));
            else un[h] = (u[h] + dt * upv[h]) - mi * (dt * dt / 2 * (y - f));
            if (p.energy != nullptr) {
              const double d = un[h] - u[h];
              en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un[h] * y;
            }
            Ys[s2 * YS + r] = un[h];
          }
          *reinterpret_cast<double2*>(p.out + (size_t(e) * S + sh) * R + r0) = make_double2(un[0], un[1]);
          if (isfinite(un[0]) && isfinite(un[1])) {
            const double mx = fmax(fabs(un[0]), fabs(un[1]));
            if (mx > 0.0) atomicMax(&shexp[s2], fx_exponent(mx));
          } else {
            atomicMax(&shexp[s2], kNaNExp);
            if (p.nonfinite != nullptr) *p.nonfinite = 1;
          }
        }
      }
      fx_epi_sync<NUPT>();
      // The state tile is consumed: stage the next item's, and its scalars.
      if (!dead) {
        stage_state(item + G);
        prefetch(item + G);
      }
      // ---- per-shot factors and scales of u^{k+1} on this element ----
      const size_t tix = size_t(e) * ntile + tile;
      if (ut < M && !dead) {
        const int ex0 = (ut < nsv) ? shexp[ut] : kNoExp;
        const int ex = ex0 > 1000 ? kNaNExp : ex0;
        if (ex0 > 1000 && ex0 != kNaNExp && p.nonfinite != nullptr) *p.nonfinite = 1;
        shfac[ut] = fx_factor24(ex);
        p.xex_out[tix * M + ut] = (fx_valid(ex) || ex == kNaNExp) ? ex : kNoExp;
      }
      fx_epi_sync<NUPT>();
      // ---- slices of u^{k+1}: image of the shared-memory operand layout ----
      {
        unsigned char* dst = xsl_out + tix * CF::ABYTES;
        for (int w = dead ? KPAD * 8 : ut; w < KPAD * 8; w += NUPT) {
          const int kr = w & 7, mg = (w >> 3) & 7, kg = w >> 6;
          const int kk = kg * 8 + kr;
          uint32_t hh[3][4];
#pragma unroll
          for (int i = 0; i < 8; i += 2) {
            uint32_t lo[3], hi[3];
            const int s2 = 8 * mg + i;
            const double fa = shfac[s2], fb = shfac[s2 + 1];
            const double va = (kk < R && s2 < nsv && fa != 0.0) ? Ys[s2 * YS + kk] : 0.0;
            const double vb = (kk < R && s2 + 1 < nsv && fb != 0.0) ? Ys[(s2 + 1) * YS + kk] : 0.0;
            fx_slice_bits(va, fa, lo[0], lo[1], lo[2]);
            fx_slice_bits(vb, fb, hi[0], hi[1], hi[2]);
#pragma unroll
            for (int pl = 0; pl < 3; ++pl) hh[pl][i / 2] = lo[pl] | (hi[pl] << 16);
          }
#pragma unroll
          for (int pl = 0; pl < CF::NPL; ++pl)
            *reinterpret_cast<uint4*>(dst + pl * CF::APLANE + w * 16) =
                make_uint4(hh[pl][0], hh[pl][1], hh[pl][2], hh[pl][3]);
        }
      }
      // ---- receivers ----
      if (q1 > q0 && !dead) {
        const long long slot = k % p.seis_cap;
        const int nwork = (q1 - q0) * M * 2;
        for (int w = ut; w < nwork; w += NUPT) {
          const int cmp = w & 1, s2 = (w >> 1) % M, q = q0 + (w >> 1) / M;
          if (s2 >= nsv) continue;
          const int rid = rcv_id_at(p, q);
          const double* ph = p.rcv_phi + size_t(rid) * NP;
          const double* un = Ys + s2 * YS + cmp * NP;
          double v = 0.0;
          for (int ii = 0; ii < NP; ++ii) v += ph[ii] * un[ii];
          p.seis[((size_t(s0 + s2) * p.seis_cap + slot) * p.nrcv + rid) * 2 + cmp] = v;
        }
      }
      if (p.energy != nullptr) {
        const double v = warp_sum(en);
        if (lane == 0) red[uw] = v;
        fx_epi_sync<NUPT>();
        if (ut == 0 && !dead) {
          double sum = 0.0;
          for (int w = 0; w < CF::NUP; ++w) sum += red[w];
          atomicAdd(p.energy + (k % p.energy_cap), sum);
        }
      }
      fx_epi_sync<NUPT>();
      // Buffer bf may be refilled by the readers.
      if (lane == 0 && !dead) fx_mbar_arrive(smem_u32(&bye[bf]));
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (*abort_s && t == 0) atomicExch(err_flag, 1);
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CF::TCOLS));
}

// Operator slices: one thread per (block, row r). Row r of block b is
// B_b[r][c] = blocks[b][c * pitch + r] (column-major storage). The image is
// [kgroup][plane][ngroup][8 K rows x 8 rows r] and zeroed beforehand
// (padding rows and columns stay zero).
template <typename BT, int R>
__global__ void k_make_bslices(const BT* __restrict__ blocks, int pitch, long long nnzb, unsigned char* __restrict__ img,
                               int* __restrict__ bex) {
  typedef FxCfg<R> CF;
  constexpr int GW = CF::GW;
  const long long n = nnzb * GW;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / GW;
    const int r = int(i - b * GW);
    if (r >= R) {
      bex[i] = kNoExp;
      continue;
    }
    const BT* col0 = blocks + size_t(b) * R * pitch + r;
    double m = 0.0;
    for (int c = 0; c < R; ++c) m = fmax(m, fabs(double(col0[size_t(c) * pitch])));
    const int ex = fx_exponent(m);
    const double fac = fx_factor24(ex);
    bex[i] = fx_valid(ex) ? ex : kNoExp;
    unsigned char* dst = img + size_t(b) * CF::BBYTES;
    for (int c = 0; c < R; ++c) {
      uint32_t h[3];
      fx_slice_bits(fac != 0.0 ? double(col0[size_t(c) * pitch]) : 0.0, fac, h[0], h[1], h[2]);
      const size_t off = size_t(c >> 3) * CF::LBO_B + (r >> 3) * 128 + (c & 7) * 16 + (r & 7) * 2;
      for (int pl = 0; pl < CF::NPL; ++pl) *reinterpret_cast<uint16_t*>(dst + pl * CF::BPL_KG + off) = uint16_t(h[pl]);
    }
  }
}

// State slices of a whole FP64 state (before first_step and after a state
// upload): one thread per (element, tile, shot-in-tile). The image is zeroed
// beforehand.
template <int R>
__global__ void k_make_xslices(const double* __restrict__ u, int ne, int S, unsigned char* __restrict__ img,
                               int* __restrict__ xex) {
  typedef FxCfg<R> CF;
  const int ntile = (S + 63) / 64;
  const long long n = (long long)ne * ntile * 64;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int sl = int(i & 63);
    const long long tix = i >> 6;
    const int tile = int(tix % ntile);
    const long long e = tix / ntile;
    const int sh = tile * 64 + sl;
    if (sh >= S) {
      xex[i] = kNoExp;
      continue;
    }
    const double* ue = u + (size_t(e) * S + sh) * R;
    double m = 0.0;
    bool fin = true;
    for (int r = 0; r < R; ++r) {
      m = fmax(m, fabs(ue[r]));
      fin = fin && isfinite(ue[r]);
    }
    const int ex = (fin && fx_exponent(m) <= 1000) ? fx_exponent(m) : kNaNExp;
    const double fac = fx_factor24(ex);
    xex[i] = (fx_valid(ex) || ex == kNaNExp) ? ex : kNoExp;
    unsigned char* dst = img + size_t(tix) * CF::ABYTES;
    for (int r = 0; r < R; ++r) {
      uint32_t h[3];
      fx_slice_bits(fac != 0.0 ? ue[r] : 0.0, fac, h[0], h[1], h[2]);
      const size_t off = size_t(r >> 3) * CF::LBO_A + (sl >> 3) * 128 + (r & 7) * 16 + (sl & 7) * 2;
      for (int pl = 0; pl < CF::NPL; ++pl) *reinterpret_cast<uint16_t*>(dst + pl * CF::APLANE + off) = uint16_t(h[pl]);
    }
  }
}

}  // namespace tsp
