// Tensor-core (tcgen05) batched step for sm_100a.
//
// Per work item (element row e, 64-shot tile) the row's block SpMM
//   Y[shot][r] = sum_b sum_c X_b[shot][c] * B_b[r][c]
// runs on the 5th-generation tensor cores: M = 64 shots, N = 2Np padded to
// 8, K = 2Np padded to 16 per block, FP32 accumulator in tensor memory.
// Operands are FP32 (blocks, and the FP32 shadow of the neighbours' state)
// split on the fly into three BF16 terms x = x1 + x2 + x3 (8 significand
// bits each); the six products of total order <= 2 (11, 12, 21, 13, 22, 31)
// recover FP32-level accuracy. Operands sit in shared memory in the
// MN-major, no-swizzle canonical layout: 8x8 core matrices of 8 K-rows by
// 16 bytes (8 consecutive M or N elements), K groups LBO apart, M/N groups
// SBO = 128 bytes apart. Two operand slots alternate so that the split of
// block b+1 overlaps the MMAs of block b. One thread issues the MMAs and
// commits them to a per-slot mbarrier; every wait is bounded and a timeout
// aborts the CTA (error flag set, tensor memory freed).
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "tsp_kernels.cuh"

namespace tsp {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor for kind::f16: BF16 x BF16 -> F32, both MN-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16_mn(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | (uint32_t(N >> 3) << 17) |
         (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait (~2 s of SM clock); false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity))
    if (clock64() - t0 > (4ll << 30)) return false;
  return true;
}

__device__ __forceinline__ void split3(float x, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c) {
  a = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(a);
  b = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(b);
  c = __float2bfloat16_rn(r2);
}

template <int R>
struct TcCfg {
  static constexpr int NP = R / 2;
  static constexpr int RP = (R + 3) & ~3;        // block column pitch in HBM (floats)
  static constexpr int NPAD = (R + 7) & ~7;      // MMA N
  static constexpr int KPAD = (R + 15) & ~15;    // MMA K per block
  static constexpr int M = 64;                   // shots per item (MMA M)
  static constexpr int LBO_A = (M / 8) * 128;    // bytes between K groups of A
  static constexpr int LBO_B = (NPAD / 8) * 128;
  static constexpr int SPLIT_A = (KPAD / 8) * LBO_A;  // bytes of one BF16 term of A
  static constexpr int SPLIT_B = (KPAD / 8) * LBO_B;
  static constexpr int SLOT = 3 * SPLIT_A + 3 * SPLIT_B;
  static constexpr int NT = 128;                 // 4 warps: one TMEM lane quadrant each
  static constexpr int TCOLS = NPAD <= 32 ? 32 : (NPAD <= 64 ? 64 : 128);
  static constexpr size_t smem_bytes() { return size_t(2) * SLOT + 64; }
};

template <int R>
__global__ void __launch_bounds__(TcCfg<R>::NT) k_step_batched_tc(const StepParams p, int* err_flag) {
  typedef TcCfg<R> CF;
  constexpr int NP = CF::NP, RP = CF::RP, NPAD = CF::NPAD, KPAD = CF::KPAD, M = CF::M;
  constexpr int NTILE_SH = 64;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* slots = smem_raw;                                   // 2 x SLOT
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + 2 * CF::SLOT);  // [2]
  uint32_t* tmem_base_s = reinterpret_cast<uint32_t*>(bars + 2);
  int* abort_s = reinterpret_cast<int*>(tmem_base_s + 1);

  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int S = p.S;
  const int ntile = (S + M - 1) / M;
  const long long nitems = (long long)p.ne * ntile;

  // ---- set-up: zero both slots (the K and N padding stays zero), barriers, TMEM ----
  for (int i = t; i < 2 * CF::SLOT / 16; i += CF::NT) reinterpret_cast<uint4*>(slots)[i] = make_uint4(0, 0, 0, 0);
  if (t == 0) {
    *abort_s = 0;
    for (int i = 0; i < 2; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bars[i])), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_base_s)),
                 "r"(CF::TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  const uint32_t tmem = *tmem_base_s;
  const uint32_t idesc = umma_idesc_bf16_mn(M, NPAD);
  const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
  const double dt = p.dt;
  const int nsh_tile = (S + NTILE_SH - 1) / NTILE_SH;

  uint32_t uses[2] = {0u, 0u};  // completed-or-issued MMA batches per slot
  bool aborted = false;
  for (long long item = blockIdx.x; item < nitems && !aborted; item += gridDim.x) {
    const int e = int(item / ntile), tile = int(item - (long long)e * ntile);
    const int s0 = tile * M;
    const int nsv = min(M, S - s0);
    const int rb = p.row_ptr[e], nb = p.row_ptr[e + 1] - rb;
    int last_slot = 0;
    for (int b = 0; b < nb; ++b) {
      const int slot = (uses[0] + uses[1]) & 1;
      last_slot = slot;
      // The slot's previous MMA batch must have finished reading it.
      if (uses[slot] > 0) {
        if (t == 0 && !mbar_wait_bounded(smem_u32(&bars[slot]), (uses[slot] - 1) & 1)) *abort_s = 1;
        __syncthreads();
        if (*abort_s) {
          aborted = true;
          break;
        }
      }
      unsigned char* sa = slots + slot * CF::SLOT;
      unsigned char* sb = sa + 3 * CF::SPLIT_A;
      // A = neighbour's FP32 shadow tile [c][shot]: task (c, shot group of 8).
      const int c = p.col[rb + b];
      const int sht = s0 / NTILE_SH, sho = s0 - sht * NTILE_SH;
      const float* gx = p.x32_in + (size_t(c) * nsh_tile + sht) * R * NTILE_SH + sho;
      for (int task = t; task < R * (M / 8); task += CF::NT) {
        const int kk = task % R, mg = task / R;
        const float4 v0 = *reinterpret_cast<const float4*>(gx + kk * NTILE_SH + 8 * mg);
        const float4 v1 = *reinterpret_cast<const float4*>(gx + kk * NTILE_SH + 8 * mg + 4);
        const float xs[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
        __align__(16) __nv_bfloat16 h[3][8];
#pragma unroll
        for (int q = 0; q < 8; ++q) split3(xs[q], h[0][q], h[1][q], h[2][q]);
        const int off = (kk >> 3) * CF::LBO_A + mg * 128 + (kk & 7) * 16;
#pragma unroll
        for (int sp = 0; sp < 3; ++sp)
          *reinterpret_cast<uint4*>(sa + sp * CF::SPLIT_A + off) = *reinterpret_cast<const uint4*>(h[sp]);
      }
      // B = block (column-major [c][r], pitch RP): task (c, row group of 8).
      const float* gb = reinterpret_cast<const float*>(p.blocks) + size_t(rb + b) * R * RP;
      for (int task = t; task < R * (NPAD / 8); task += CF::NT) {
        const int kk = task % R, ng = task / R;
        const int r0 = 8 * ng;
        float xs[8];
#pragma unroll
        for (int hq = 0; hq < 2; ++hq) {
          float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
          if (r0 + 4 * hq < RP) v = *reinterpret_cast<const float4*>(gb + kk * RP + r0 + 4 * hq);
          xs[4 * hq + 0] = v.x;
          xs[4 * hq + 1] = v.y;
          xs[4 * hq + 2] = v.z;
          xs[4 * hq + 3] = v.w;
        }
        __align__(16) __nv_bfloat16 h[3][8];
#pragma unroll
        for (int q = 0; q < 8; ++q) split3(xs[q], h[0][q], h[1][q], h[2][q]);
        const int off = (kk >> 3) * CF::LBO_B + ng * 128 + (kk & 7) * 16;
#pragma unroll
        for (int sp = 0; sp < 3; ++sp)
          *reinterpret_cast<uint4*>(sb + sp * CF::SPLIT_B + off) = *reinterpret_cast<const uint4*>(h[sp]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (t == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
        const int pairs[6][2] = {{0, 0}, {0, 1}, {1, 0}, {0, 2}, {1, 1}, {2, 0}};
#pragma unroll
        for (int ks = 0; ks < KPAD / 16; ++ks)
#pragma unroll
          for (int pq = 0; pq < 6; ++pq) {
            const uint64_t da = umma_desc(a0 + pairs[pq][0] * CF::SPLIT_A + ks * 2 * CF::LBO_A, CF::LBO_A, 128);
            const uint64_t db = umma_desc(b0 + pairs[pq][1] * CF::SPLIT_B + ks * 2 * CF::LBO_B, CF::LBO_B, 128);
            umma_bf16(tmem, da, db, idesc, (b > 0 || ks > 0 || pq > 0) ? 1u : 0u);
          }
        umma_commit(smem_u32(&bars[slot]));
      }
      uses[slot] += 1;
    }
    if (aborted) break;
    // ---- wait for the item's last MMA batch, then the epilogue ----
    if (t == 0 && !mbar_wait_bounded(smem_u32(&bars[last_slot]), (uses[last_slot] - 1) & 1)) *abort_s = 1;
    __syncthreads();
    if (*abort_s) {
      aborted = true;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // Warp w reads TMEM lanes 32w..32w+31; for M = 64, shots 16w..16w+15 are
    // in lanes 32w..32w+15, columns = output rows.
    float y[NPAD];
    const uint32_t lane_addr = tmem + (uint32_t(32 * warp) << 16);
#pragma unroll
    for (int cb = 0; cb < NPAD; cb += 8) {
      uint32_t r8[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(r8[0]), "=r"(r8[1]), "=r"(r8[2]), "=r"(r8[3]), "=r"(r8[4]), "=r"(r8[5]), "=r"(r8[6]),
                     "=r"(r8[7])
                   : "r"(lane_addr + uint32_t(cb)));
#pragma unroll
      for (int q = 0; q < 8; ++q) y[cb + q] = __uint_as_float(r8[q]);
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    const int sl = 16 * warp + lane;  // shot within the tile (lanes < 16)
    const double mi = p.minv[e];
    if (lane < 16 && sl < nsv) {
      const int sh = s0 + sl;
      const size_t me = (size_t(e) * S + sh) * R;
      const bool is_src = (p.src_elem[sh] == e) && (k < p.nF);
      double Fk[2] = {0.0, 0.0};
      if (is_src) {
        Fk[0] = p.F[(size_t(sh) * p.nF + k) * 2];
        Fk[1] = p.F[(size_t(sh) * p.nF + k) * 2 + 1];
      }
      float* gxo = p.x32_out + (size_t(e) * nsh_tile + (s0 / NTILE_SH)) * R * NTILE_SH + (s0 % NTILE_SH) + sl;
#pragma unroll
      for (int r0 = 0; r0 < R; r0 += 2) {
        const double2 uu = __ldg(reinterpret_cast<const double2*>(p.x + me + r0));
        const double2 up = p.uprev ? *reinterpret_cast<const double2*>(p.uprev + me + r0) : make_double2(0.0, 0.0);
        const double u[2] = {uu.x, uu.y}, upv[2] = {up.x, up.y};
        double un[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = r0 + h;
          const int cmp = r / NP, ii = r - cmp * NP;
          const double f = is_src ? Fk[cmp] * p.src_phi[size_t(sh) * NP + ii] : 0.0;
          const double yy = double(y[r]);
          if (p.mode == kModeStep) un[h] = (2 * u[h] - upv[h]) + mi * ((-dt * dt) * (yy - f));
          else un[h] = (u[h] + dt * upv[h]) - mi * (dt * dt / 2 * (yy - f));
          gxo[r * NTILE_SH] = float(un[h]);
        }
        *reinterpret_cast<double2*>(p.out + me + r0) = make_double2(un[0], un[1]);
      }
    }
    if (p.rcv_ptr != nullptr) {
      const int q0 = p.rcv_ptr[e], q1 = p.rcv_ptr[e + 1];
      if (q1 > q0) {
        __syncthreads();
        const long long slot = k % p.seis_cap;
        const int nwork = (q1 - q0) * M * 2;
        for (int w = t; w < nwork; w += CF::NT) {
          const int cmp = w & 1, sl2 = (w >> 1) % M, q = q0 + (w >> 1) / M;
          if (sl2 >= nsv) continue;
          const int rid = p.rcv_id[q];
          const double* ph = p.rcv_phi + size_t(rid) * NP;
          const double* un = p.out + (size_t(e) * S + s0 + sl2) * R + cmp * NP;
          double v = 0.0;
          for (int ii = 0; ii < NP; ++ii) v += ph[ii] * un[ii];
          p.seis[((size_t(s0 + sl2) * p.seis_cap + slot) * p.nrcv + rid) * 2 + cmp] = v;
        }
      }
    }
    // The next item's first MMA overwrites the accumulator.
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  if (aborted && t == 0) atomicExch(err_flag, 1);
  // Drain: the last issued batch of each slot must be complete before the
  // tensor memory is released (bounded; on timeout the error flag is set).
  if (t == 0)
    for (int sl3 = 0; sl3 < 2; ++sl3)
      if (uses[sl3] > 0 && !mbar_wait_bounded(smem_u32(&bars[sl3]), (uses[sl3] - 1) & 1)) atomicExch(err_flag, 1);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CF::TCOLS));
}

}  // namespace tsp
