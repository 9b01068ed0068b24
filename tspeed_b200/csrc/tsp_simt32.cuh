// Batched step with an FP32 operator on the CUDA cores, warp-specialised and
// persistent (internal header of tspeed_b200).
//
// Per work item (element row e, tile of 64 shots) the block SpMM
//   Y[shot][r] = sum_b sum_k X_{col b}[shot][k] B_b[r][k]
// runs in FP32 (FP32 operator blocks, the FP32 shadow of the state, FP32
// accumulation) with register tiles large enough that the FP32 pipe, not the
// shared-memory or issue bandwidth, bounds the products: each lane owns
// 8 shots x RL rows (RL = 6 at 2Np = 42: 48 accumulators fed by two 16-byte
// loads of the state and RL/2 8-byte loads of the block per K step). The
// leap-frog update, the source, the receivers and the energy terms stay in
// FP64 (u^k, u^{k-1} and u^{k+1} in FP64); the epilogue also writes the FP32
// shadow of u^{k+1} that the next step's neighbours read.
//
// Roles: NGR pairs of an FMA group (NWG warps: the products of one item) and
// an update set (NU warps: the FP64 epilogue of that group's items), and a
// producer warp. One producer lane per pair streams, per block, two bulk
// copies into the pair's own ring of NSG stages (cp.async.bulk, completion
// on mbarriers, no multicast): the stored FP32 block (column-major, pitch
// KP = 2Np padded to 4) and the neighbour's FP32 shadow tile (2Np rows of
// 64 shots, contiguous). The FMA group writes the item's FP32 row sums into
// the pair's Y tile in shared memory and goes on with its next item; the
// update set reads them, runs the leap-frog update with coalesced FP64 loads
// and stores of the contiguous state tile (a shot tile of an element is one
// run of 64 x 2Np doubles), writes u^{k+1} back into the Y tile in FP32 and
// stores it transposed as the next step's shadow (rows of 64 shots,
// coalesced), then samples the receivers. The FMA warps never wait on global
// memory; the update sets hide their load latency behind the products.
// Every ring and the Y tile are used by one pair only, in its own item
// order, so each mbarrier wait is unambiguous (use n - 1 of a barrier is
// always one the waiter consumed itself).
//
// Lane (sg, rg) of warp w of an FMA group: shots 4 sg .. 4 sg + 3 and
// 32 + 4 sg .. 32 + 4 sg + 3 (each quarter-warp reads 128 contiguous bytes
// of a state row: conflict-free), rows w RW + rg RL .. + RL - 1 with
// RW = 4 RL. Rows at or beyond 2Np (the last warp's padding) are computed
// from in-bounds shared memory (the stage's tail) and never stored.
//
// Every wait is bounded (about a second); on a timeout the CTA raises an
// abort flag in shared memory, every role stops waiting, the update sets keep
// their named barriers balanced, the producers wait (bounded) for their
// copies in flight, and err_flag tells the host that the results are void.
#pragma once

#include <stdint.h>

#include "tsp_kernels.cuh"
#include "tsp_tcfx.cuh"
#include "tsp_tcgen05.cuh"

namespace tsp {

template <int R>
struct S32WCfg {
  static constexpr int KP = (R + 3) & ~3;  // stored block pitch of batched handles
  static constexpr int ST = 64;            // shots per tile (the FP32 shadow's tile)
  // Rows per lane (even: the FP64 epilogue works on row pairs): padding
  // rows kept small with at most two warps per item.
  static constexpr int RL = R <= 8 ? 2 : R <= 16 ? 4 : R <= 24 ? 6 : R <= 32 ? 4 : R <= 48 ? 6 : 8;
  static constexpr int RW = 4 * RL;                   // rows per warp
  static constexpr int NWG = (R + RW - 1) / RW;       // warps per group
  static constexpr int BSZ = R * KP;                  // floats: operator stage [k][r], pitch KP
  static constexpr int XSZ = R * ST;                  // floats: state stage [k][shot]
  static constexpr int STAGE = BSZ + XSZ;
  static_assert((BSZ * 4) % 16 == 0 && (STAGE * 4) % 16 == 0, "16-byte aligned stages");
  // The last warp's padding rows read at most this far into a stage.
  static_assert((R - 1) * KP + NWG * RW <= STAGE, "padding rows stay inside the stage");
};

template <int R, int NGR, int NSG, int NU>
struct S32WLayout {
  typedef S32WCfg<R> C;
  static constexpr int NF = NGR * C::NWG;              // FMA warps
  static constexpr int NUT = NU * 32;                  // threads of an update set
  static constexpr int NT = (NF + NGR * NU + 1) * 32;  // + update warps + the producer warp
  static constexpr int NST = NGR * NSG;
  static constexpr int YP = R + 1;                     // odd pitch of the Y tile [shot][YP]
  static constexpr int YSZ = C::ST * YP;               // floats of one pair's Y tile
  static_assert((YSZ * 4) % 16 == 0, "aligned barriers after the Y tiles");
  static constexpr size_t smem_bytes() {
    return size_t(NST) * C::STAGE * sizeof(float) + size_t(NGR) * YSZ * sizeof(float) +
           size_t(2 * NST + 2 * NGR) * sizeof(uint64_t) + 16;
  }
};

// Stages per pair ring (at most 6) that fit in shared memory beside the Y
// tiles; 0 if not even one does.
template <int R, int NGR, int NU>
constexpr int s32w_fit_nsg() {
  constexpr size_t budget = 227 * 1024;
  int n = 6;
  while (n > 0) {
    const size_t bytes = size_t(NGR) * n * S32WCfg<R>::STAGE * sizeof(float) +
                         size_t(NGR) * S32WLayout<R, NGR, 1, NU>::YSZ * sizeof(float) +
                         size_t(2 * NGR * n + 2 * NGR) * sizeof(uint64_t) + 16;
    if (bytes <= budget) break;
    --n;
  }
  return n;
}

// Packed FP32 FMA on pairs (Blackwell fma.rn.f32x2; one instruction per two
// FMAs leaves issue slots to the loads).
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b,
                                                    unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ unsigned long long f32x2_splat(float v) {
  unsigned long long d;
  asm("mov.b64 %0, {%1, %1};" : "=l"(d) : "f"(v));
  return d;
}
__device__ __forceinline__ void f32x2_unpack(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

// Shots of a 64-shot tile whose source lies in element e (bit sl), for steps
// that still have a force sample; the same in every lane of the warp.
__device__ __forceinline__ unsigned long long tile_source_mask(const StepParams& p, int e, int s0, int nsv,
                                                               long long k, int ln) {
  if (k >= p.nF) return 0ull;
  const bool a = ln < nsv && src_elem_at(p, s0 + ln) == e;
  const bool b = ln + 32 < nsv && src_elem_at(p, s0 + 32 + ln) == e;
  return (unsigned long long)__ballot_sync(0xffffffffu, a) | ((unsigned long long)__ballot_sync(0xffffffffu, b) << 32);
}

// FP64 epilogue of one item's state tile by an update set of NUT threads, UB
// row pairs per thread and load batch (both levels' loads of a batch first).
// Reads the FP32 row sums from the Y tile ([shot][R + 1]) and writes u^{k+1}
// back into it in FP32 for the shadow. (A software-pipelined form, the next
// batch's loads issued before the current batch is stored, needs twice the
// load registers and spilled at the 96 registers per thread of these
// kernels: slower.)
template <int R, int NUT, int UB>
__device__ __forceinline__ void s32_update_tile(const StepParams& p, float* Y, int e, int s0, int nsv, size_t base,
                                                int ut, long long k, double dt, double& en) {
  constexpr int NP = R / 2, YP = R + 1, STEP = NUT * UB;
  static_assert(S32WCfg<R>::ST == 64, "one 64-bit source mask per shot tile");
  const double mi = p.minv[e];
  const int npair = nsv * NP;
  const double2* xs = reinterpret_cast<const double2*>(p.x + base);
  const double2* ps = p.uprev ? reinterpret_cast<const double2*>(p.uprev + base) : nullptr;
  // The update warps are few and run dependent chains, so the epilogue keeps
  // per-pair work to the FP64 recurrence: the shots whose source lies in this
  // element are found once per tile (bit sl of smask, two loads per lane),
  // and a non-finite u^{k+1} is caught by one FMA per value (inf * 0 and
  // NaN * 0 are NaN) and reported once per tile.
  const unsigned long long smask = tile_source_mask(p, e, s0, nsv, k, ut & 31);
  double chk = 0.0;
  // Row pair q = pb + NUT b + ut is entry 2q of the tile: shot q / NP, rows
  // 2 (q % NP) and +1 (coalesced loads and stores).
  for (int q0 = 0; q0 < npair; q0 += STEP) {
    double2 uu[UB], up[UB];
#pragma unroll
    for (int b = 0; b < UB; ++b) {
      const int q = q0 + NUT * b + ut;
      const bool v = q < npair;
      uu[b] = v ? __ldg(xs + q) : make_double2(0.0, 0.0);
      up[b] = (v && ps) ? ps[q] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int b = 0; b < UB; ++b) {
      const int q = q0 + NUT * b + ut;
      if (q >= npair) continue;
      const int sl = q / NP, r0 = 2 * (q - sl * NP);
      const double u[2] = {uu[b].x, uu[b].y}, upr[2] = {up[b].x, up[b].y};
      double yv[2] = {double(Y[sl * YP + r0]), double(Y[sl * YP + r0 + 1])};
      if (smask != 0 && ((smask >> sl) & 1)) {
        const int sh = s0 + sl;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = r0 + h, cmp = r / NP, ii = r - cmp * NP;
          yv[h] -= p.F[(size_t(sh) * p.nF + k) * 2 + cmp] * p.src_phi[size_t(sh) * NP + ii];
        }
      }
      double un[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (p.mode == kModeStep) un[h] = (2 * u[h] - upr[h]) + mi * ((-dt * dt) * yv[h]);
        else un[h] = (u[h] + dt * upr[h]) - mi * (dt * dt / 2 * yv[h]);  // kModeFirst, uprev = v0
        chk = __fma_rn(un[h], 0.0, chk);
      }
      if (p.energy != nullptr) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const double d = un[h] - u[h];
          // y of the energy term is the product B u^k without the source.
          en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un[h] * double(Y[sl * YP + r0 + h]);
        }
      }
      Y[sl * YP + r0] = float(un[0]);
      Y[sl * YP + r0 + 1] = float(un[1]);
      *(reinterpret_cast<double2*>(p.out + base) + q) = make_double2(un[0], un[1]);
    }
  }
  if (chk != chk && p.nonfinite != nullptr) *p.nonfinite = 1;
}

// F2 selects packed pair FMAs (1) or scalar FMAs (0) for the products.
// UB: row pairs per update thread and load batch.
template <int R, int NGR, int NSG, int NU, int F2, int UB = 6>
__global__ void __launch_bounds__(S32WLayout<R, NGR, NSG, NU>::NT, 1)
    k_step_batched32w(const StepParams p, int* err_flag) {
  typedef S32WCfg<R> CF;
  typedef S32WLayout<R, NGR, NSG, NU> LY;
  constexpr int NP = R / 2, KP = CF::KP, ST = CF::ST, RL = CF::RL, RW = CF::RW, NWG = CF::NWG;
  constexpr int NST = LY::NST, NF = LY::NF, NUT = LY::NUT, YP = LY::YP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* stages = reinterpret_cast<float*>(smem_raw);
  float* ybuf = stages + size_t(NST) * CF::STAGE;                                    // [NGR][ST][YP]
  uint64_t* bfull = reinterpret_cast<uint64_t*>(ybuf + size_t(NGR) * LY::YSZ);      // [NGR][NSG] stage landed
  uint64_t* bempty = bfull + NST;                                                    // [NGR][NSG] stage consumed
  uint64_t* yfull = bempty + NST;                                                    // [NGR] Y tile written
  uint64_t* yempty = yfull + NGR;                                                    // [NGR] Y tile consumed
  volatile int* abort_s = reinterpret_cast<volatile int*>(yempty + NGR);

  if (*reinterpret_cast<volatile int*>(err_flag) != 0) return;  // an earlier launch of the run timed out
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  if (t == 0) {
    *abort_s = 0;
    for (int i = 0; i < NST; ++i) {
      fx_mbar_init(smem_u32(&bfull[i]), 1);
      fx_mbar_init(smem_u32(&bempty[i]), NWG);
    }
    for (int i = 0; i < NGR; ++i) {
      fx_mbar_init(smem_u32(&yfull[i]), NWG);
      fx_mbar_init(smem_u32(&yempty[i]), NU);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = t; i < NST * CF::STAGE + NGR * LY::YSZ; i += LY::NT) stages[i] = 0.0f;
  __syncthreads();

  const int S = p.S;
  const int ntile = (S + ST - 1) / ST;
  const long long nitems = (long long)p.ne * ntile;
  const long long G = gridDim.x;
  const float* blocks = reinterpret_cast<const float*>(p.blocks);

  if (warp == NF + NGR * NU) {
    // ---------------- producers: lane g fills ring g ----------------
    if (lane < NGR) {
      const int g = lane;
      uint64_t* gfull = bfull + g * NSG;
      uint64_t* gempty = bempty + g * NSG;
      float* gst = stages + size_t(g) * NSG * CF::STAGE;
      constexpr uint32_t bbytes = uint32_t(R) * KP * 4, xbytes = uint32_t(R) * ST * 4;
      uint32_t j = 0;
      bool ok = true;
      for (long long item = blockIdx.x + g * G; item < nitems && ok; item += NGR * G) {
        const int e = int(item / ntile), tile = int(item % ntile);
        int rb, nb;
        row_span(p, e, rb, nb);
        for (int b = 0; b < nb; ++b) {
          const int s = int(j % NSG);
          const uint32_t n = j / NSG;
          if (n > 0 && !fx_wait(smem_u32(&gempty[s]), (n - 1) & 1, abort_s)) {
            ok = false;
            break;
          }
          const int c = col_at(p, rb + b);
          const uint32_t bar = smem_u32(&gfull[s]);
          const uint32_t dB = smem_u32(gst + size_t(s) * CF::STAGE), dX = dB + CF::BSZ * 4;
          fx_mbar_arrive_tx(bar, bbytes + xbytes);
          fx_bulk_g2s(dB, blocks + size_t(rb + b) * R * KP, bbytes, bar);
          fx_bulk_g2s(dX, p.x32_in + (size_t(c) * ntile + tile) * R * ST, xbytes, bar);
          ++j;
        }
      }
      // Every issued copy lands before the CTA ends (bounded; copies
      // complete). At most one use of a stage is in flight.
      const long long t0 = clock64();
      for (int s = 0; s < NSG; ++s) {
        if (j <= uint32_t(s)) continue;
        const uint32_t uses = (j - 1 - s) / NSG + 1;
        while (!mbar_try(smem_u32(&gfull[s]), (uses - 1) & 1) && clock64() - t0 < (1ll << 31)) {
        }
      }
      if (clock64() - t0 >= (1ll << 31)) *abort_s = 1;
    }
  } else if (warp < NF) {
    // ---------------- FMA groups ----------------
    const int grp = warp / NWG, w = warp % NWG;
    const int sg = lane & 7, rg = lane >> 3;
    const int rbase = w * RW + rg * RL;  // the lane's first row
    uint64_t* gfull = bfull + grp * NSG;
    uint64_t* gempty = bempty + grp * NSG;
    const float* gst = stages + size_t(grp) * NSG * CF::STAGE;
    float* Y = ybuf + size_t(grp) * LY::YSZ;
    uint32_t j = 0, m = 0;  // ring index; uses of the Y tile
    bool dead = false;
    long long it = 0;
    for (long long item = blockIdx.x; item < nitems; item += G, ++it) {
      if (int(it % NGR) != grp) continue;  // another pair's item
      const int e = int(item / ntile);
      int rb, nb;
      row_span(p, e, rb, nb);
      float acc[RL][8];
      unsigned long long acc2[RL][4];  // F2: shots (2m, 2m + 1) of the lane's 8
#pragma unroll
      for (int i = 0; i < RL; ++i) {
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[i][q] = 0.0f;
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) acc2[i][mm] = 0ull;
      }
      for (int b = 0; b < nb; ++b) {
        const int s = int(j % NSG);
        const uint32_t n = j / NSG;
        ++j;
        if (dead) continue;
        const bool okw = fx_wait(smem_u32(&gfull[s]), n & 1, abort_s);
        if (__any_sync(0xffffffffu, !okw)) {
          dead = true;
          continue;
        }
        const float* Bs = gst + size_t(s) * CF::STAGE + rbase;
        const float* Xs = gst + size_t(s) * CF::STAGE + CF::BSZ + 4 * sg;
        // K steps unrolled by 14 at 2Np = 42 and 56 (measured: 1.13 ms per
        // step on config 3 against 1.16 at 6, 1.21 at 2 and at full unroll).
        constexpr int KU = R % 14 == 0 ? 14 : R % 10 == 0 ? 10 : R % 6 == 0 ? 6 : 2;
#pragma unroll KU
        for (int kk = 0; kk < R; ++kk) {
          float bv[RL];
#pragma unroll
          for (int i = 0; i < RL; i += 2) {
            const float2 b2 = *reinterpret_cast<const float2*>(Bs + kk * KP + i);
            bv[i] = b2.x;
            bv[i + 1] = b2.y;
          }
          if constexpr (F2) {
            const ulonglong2 xa = *reinterpret_cast<const ulonglong2*>(Xs + kk * ST);
            const ulonglong2 xb = *reinterpret_cast<const ulonglong2*>(Xs + kk * ST + 32);
            const unsigned long long xp[4] = {xa.x, xa.y, xb.x, xb.y};
#pragma unroll
            for (int i = 0; i < RL; ++i) {
              const unsigned long long bb = f32x2_splat(bv[i]);
#pragma unroll
              for (int mm = 0; mm < 4; ++mm) acc2[i][mm] = ffma2(xp[mm], bb, acc2[i][mm]);
            }
          } else {
            const float4 xa = *reinterpret_cast<const float4*>(Xs + kk * ST);
            const float4 xb = *reinterpret_cast<const float4*>(Xs + kk * ST + 32);
            const float xv[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
#pragma unroll
            for (int i = 0; i < RL; ++i)
#pragma unroll
              for (int q = 0; q < 8; ++q) acc[i][q] = fmaf(xv[q], bv[i], acc[i][q]);
          }
        }
        __syncwarp();
        if (lane == 0) fx_mbar_arrive(smem_u32(&gempty[s]));
      }
      if constexpr (F2) {
#pragma unroll
        for (int i = 0; i < RL; ++i)
#pragma unroll
          for (int mm = 0; mm < 4; ++mm) f32x2_unpack(acc2[i][mm], acc[i][2 * mm], acc[i][2 * mm + 1]);
      }
      // ---- hand the row sums to the pair's update set ----
      if (!dead && m > 0) {
        const bool okw = fx_wait(smem_u32(&yempty[grp]), (m - 1) & 1, abort_s);
        if (__any_sync(0xffffffffu, !okw)) dead = true;
      }
      ++m;
      if (dead) continue;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int sl = (q < 4 ? 0 : 32) + 4 * sg + (q & 3);
#pragma unroll
        for (int i = 0; i < RL; ++i)
          if (rbase + i < R) Y[sl * YP + rbase + i] = acc[i][q];
      }
      __syncwarp();
      if (lane == 0) fx_mbar_arrive(smem_u32(&yfull[grp]));
    }
  } else {
    // ---------------- update sets: FP64 epilogue of the pair's items ----------------
    const int ug = (warp - NF) / NU;
    const int ut = t - (NF + ug * NU) * 32;  // thread within the set
    const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
    const double dt = p.dt;
    float* Y = ybuf + size_t(ug) * LY::YSZ;
    constexpr int BATCH = UB;  // row pairs per thread and load batch
    double en = 0.0;
    uint32_t m = 0;
    bool dead = false;
    long long it = 0;
    for (long long item = blockIdx.x; item < nitems; item += G, ++it) {
      if (int(it % NGR) != ug) continue;
      const int e = int(item / ntile), tile = int(item % ntile);
      const int s0 = tile * ST, nsv = min(ST, S - s0);
      const size_t base = (size_t(e) * S + s0) * R;  // the tile: nsv * R contiguous doubles
      const size_t tix = size_t(e) * ntile + tile;
      if (!dead) {
        const bool okw = fx_wait(smem_u32(&yfull[ug]), m & 1, abort_s);
        if (!__all_sync(0xffffffffu, okw)) dead = true;
      }
      ++m;
      if (!dead) s32_update_tile<R, NUT, BATCH>(p, Y, e, s0, nsv, base, ut, k, dt, en);
      // u^{k+1} of the item (FP64 in global memory, FP32 in the Y tile) is
      // complete once the whole set passes this barrier (id 1 + pair).
      asm volatile("bar.sync %0, %1;" ::"r"(1 + ug), "n"(NUT) : "memory");
      if (!dead) {
        // FP32 shadow of u^{k+1}, transposed: rows of 64 shots (shots beyond
        // S stay zero), four shots per 16-byte store.
        for (int i4 = ut; i4 < R * (ST / 4); i4 += NUT) {
          const int r = i4 / (ST / 4), sl = (i4 - r * (ST / 4)) * 4;
          float4 v;
          v.x = sl < nsv ? Y[sl * YP + r] : 0.0f;
          v.y = sl + 1 < nsv ? Y[(sl + 1) * YP + r] : 0.0f;
          v.z = sl + 2 < nsv ? Y[(sl + 2) * YP + r] : 0.0f;
          v.w = sl + 3 < nsv ? Y[(sl + 3) * YP + r] : 0.0f;
          *reinterpret_cast<float4*>(p.x32_out + (tix * R + r) * ST + sl) = v;
        }
        // Receivers of this element.
        if (p.rcv_ptr != nullptr) {
          const int q0 = rcv_ptr_at(p, e), q1 = rcv_ptr_at(p, e + 1);
          const long long slot = k % p.seis_cap;
          for (int wk = ut; wk < (q1 - q0) * nsv * 2; wk += NUT) {
            const int cmp = wk & 1, sl = (wk >> 1) % nsv, q = q0 + (wk >> 1) / nsv;
            const int sh = s0 + sl;
            const int rid = rcv_id_at(p, q);
            const double* ph = p.rcv_phi + size_t(rid) * NP;
            const double* un = p.out + base + size_t(sl) * R + cmp * NP;
            double v = 0.0;
            for (int ii = 0; ii < NP; ++ii) v += ph[ii] * un[ii];
            p.seis[((size_t(sh) * p.seis_cap + slot) * p.nrcv + rid) * 2 + cmp] = v;
          }
        }
        __syncwarp();
        if (lane == 0) fx_mbar_arrive(smem_u32(&yempty[ug]));
      }
    }
    if (p.energy != nullptr) {
      const double v = warp_sum(en);
      if (lane == 0 && v != 0.0) atomicAdd(p.energy + (k % p.energy_cap), v);
    }
  }
  __syncthreads();
  if (t == 0 && *abort_s) atomicExch(err_flag, 1);
}

}  // namespace tsp
