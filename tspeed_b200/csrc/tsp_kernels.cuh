// Device kernels of the tspeed_b200 engine (sm_100a).
//
// Data layout in HBM
//   state   u[(e*S + s)*R + r], R = 2*Np, r = c*Np + i: element-major,
//           shot-interleaved, FP64. One element's 2Np modes of one shot are
//           contiguous (16-byte aligned since R is even).
//   blocks  block-CSR of MyMat (MyMat.cpp:128-154): per element row the
//           diagonal block first, then the face neighbours in edge order.
//           Each 2Np x 2Np block is stored COLUMN-major (entry (r, c) at
//           c*R + r), so the lanes of a team that own consecutive row pairs
//           read one contiguous, coalesced run of a column.
//   minv    1/(rho_e detJ_e) per element (Matrices_imp.hpp:187,189).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tsp {

// ---------------------------------------------------------------------------
// Shared parameter block of the step kernels.
// ---------------------------------------------------------------------------
enum StepMode : int {
  kModeStep = 0,   // u^{k+1} = 2u^k - u^{k-1} + minv*(-dt*dt*(B u^k - f))     (TimeAdvance.cpp:52)
  kModeFirst = 1,  // u^1 = u^0 + dt v^0 - minv*(dt*dt/2*(B u^0 - f))          (TimeAdvance.cpp:30)
  kModeApply = 2,  // y = B x
  kModePower = 3   // y = minv * (B x) with Rayleigh-quotient accumulators
};

struct StepParams {
  int ne;
  int S;                      // shots
  int mode;
  const int* row_ptr;         // [ne+1]
  const int* col;             // [nnzb]
  const void* blocks;         // [nnzb][R][bpitch] column-major, BT
  int bpitch;                 // column pitch of a stored block (R, or R padded to 4)
  const float* bscale;        // [nnzb] (BF16 only)
  const double* minv;         // [ne]
  const double* x;            // u^k (gathered by neighbours)
  const double* uprev;        // u^{k-1} (kModeStep) / v^0 or null (kModeFirst)
  double* out;                // u^{k+1}; may alias uprev (same thread reads then writes)
  double dt;
  double xscale;              // kModePower: x is used as xscale*x
  const long long* step_base; // device step counter (k = *step_base + rel)
  int rel;
  // sources: one point source per shot
  const int* src_elem;        // [S]
  const double* src_phi;      // [S][Np]
  const double* F;            // [S][nF][2]
  long long nF;
  // receivers, CSR over elements
  const int* rcv_ptr;         // [ne+1] or null
  const int* rcv_id;          // [nrcv] receiver ids ordered by element
  const double* rcv_phi;      // [nrcv][Np] by receiver id
  double* seis;               // [S][cap][nrcv][2]
  int nrcv;
  long long seis_cap;
  // energy monitor (null = off) and power-iteration accumulators
  double* energy;             // [cap]
  long long energy_cap;
  double* acc;                // kModePower: [3]
  // FP32 transposed shadow of the state for the batched FP32 kernel:
  // x32[((e*ntile + tile)*R + c)*64 + shot_in_tile]. x32_in is read by the
  // neighbour gathers, x32_out receives u^{k+1}.
  const float* x32_in;
  float* x32_out;
  // Multi-mesh groups (several independent meshes concatenated into one
  // block-diagonal system; null for an ordinary handle):
  const double* dt_elem;      // per-element time step (the element's mesh's dt)
  const int* src_of;          // per-element source index into src_phi/F, -1 if none
  const int* mesh_of;         // per-element mesh id (power iteration per mesh)
  const double* xscale_mesh;  // per-mesh power-iteration scale
  // Tensor-core fixed-point path: slice images of the state (per element and
  // 64-shot tile) and of the operator (per block), with the shared binary
  // exponents of their rows (per shot of a tile, per block row).
  const void* xsl_in;
  void* xsl_out;
  const int* xex_in;
  int* xex_out;
  const void* bsl;
  const int* bex;
  // Non-finite watchdog (step modes only; null otherwise): set to 1 by any
  // kernel that writes a NaN or infinite u^{k+1}.
  int* nonfinite;
  long long nnzb;             // blocks of the pattern (the checked build's row bounds)
};

// Gather indices of the step kernels -- row extents, neighbour ids, source
// elements, receiver entries -- are read through these accessors. In the
// checked build (TSP_CHECKED) each value is range-checked first: a value out
// of range is recorded in g_index_check (site in the high word, the value in
// the low word; the first failure of a launch sequence is kept) and replaced
// by one inside the range, so the kernel reads only valid memory, completes,
// and the host reports TSP_ERR_INDEX. Without TSP_CHECKED they are the plain
// loads.
enum IndexSite : int { kSiteRow = 1, kSiteCol = 2, kSiteSrcElem = 3, kSiteRcvPtr = 4, kSiteRcvId = 5, kSiteNeigh = 6 };
#ifdef TSP_CHECKED
__device__ unsigned long long g_index_check;
__device__ __forceinline__ int checked_index(int v, int lo, int hi, int site) {
  if (v >= lo && v < hi) return v;
  atomicCAS(&g_index_check, 0ull, ((unsigned long long)(unsigned)site << 32) | (unsigned)v);
  return lo;
}
#define TSP_INDEX(v, lo, hi, site) ::tsp::checked_index((v), (lo), (hi), (site))
#else
#define TSP_INDEX(v, lo, hi, site) (v)
#endif

// Block range [rb, rb + nb) of element row e: the diagonal block and at most
// three neighbours inside the pattern (checked build: a row outside that is
// recorded and clamped to a valid one).
__device__ __forceinline__ void row_span(const StepParams& p, int e, int& rb, int& nb) {
  rb = p.row_ptr[e];
  nb = p.row_ptr[e + 1] - rb;
#ifdef TSP_CHECKED
  if (p.nnzb > 0 && (rb < 0 || rb >= p.nnzb || nb < 1 || nb > 4 || rb + nb > p.nnzb)) {
    atomicCAS(&g_index_check, 0ull, ((unsigned long long)kSiteRow << 32) | (unsigned)e);
    rb = min(max(rb, 0), int(p.nnzb - 1));
    nb = min(max(nb, 1), min(4, int(p.nnzb - rb)));
  }
#endif
}
// Column (neighbour element) of block b of the pattern.
template <class P>
__device__ __forceinline__ int col_at(const P& p, long long b) {
  return TSP_INDEX(p.col[b], 0, p.ne, kSiteCol);
}
// Source element of shot s (compared with element ids only; -1 for none).
__device__ __forceinline__ int src_elem_at(const StepParams& p, int s) {
  return TSP_INDEX(p.src_elem[s], -1, p.ne, kSiteSrcElem);
}
// Receiver entries of element e: [rcv_ptr[e], rcv_ptr[e + 1]) within the nrcv ids.
__device__ __forceinline__ int rcv_ptr_at(const StepParams& p, int e) {
  return TSP_INDEX(p.rcv_ptr[e], 0, p.nrcv + 1, kSiteRcvPtr);
}
// Receiver id of entry q (indexes rcv_phi and the seismogram buffer).
__device__ __forceinline__ int rcv_id_at(const StepParams& p, int q) {
  return TSP_INDEX(p.rcv_id[q], 0, p.nrcv, kSiteRcvId);
}

// Raises the non-finite flag when a new displacement pair holds a NaN or an
// infinity (the leap-frog recurrence keeps such a value for good).
__device__ __forceinline__ void note_nonfinite(const StepParams& p, double a, double b) {
  if (!(isfinite(a) && isfinite(b)) && p.nonfinite != nullptr) *p.nonfinite = 1;
}

// ---------------------------------------------------------------------------
// Loads. Operator blocks are streamed once per step: ld.global.cs keeps them
// from displacing the state in L2. The state is read through the read-only
// path (neighbours re-read it).
// ---------------------------------------------------------------------------
template <typename BT>
struct Pair;
template <>
struct Pair<double> {
  static __device__ __forceinline__ void load(const double* p, double& a, double& b) {
    const double2 v = __ldcs(reinterpret_cast<const double2*>(p));
    a = v.x;
    b = v.y;
  }
};
template <>
struct Pair<float> {
  static __device__ __forceinline__ void load(const float* p, float& a, float& b) {
    const float2 v = __ldcs(reinterpret_cast<const float2*>(p));
    a = v.x;
    b = v.y;
  }
};
template <>
struct Pair<__nv_bfloat16> {
  static __device__ __forceinline__ void load(const __nv_bfloat16* p, float& a, float& b) {
    const unsigned int v = __ldcs(reinterpret_cast<const unsigned int*>(p));
    a = __uint_as_float(v << 16);
    b = __uint_as_float(v & 0xffff0000u);
  }
};

template <typename BT>
struct AccOf { typedef float type; };
template <>
struct AccOf<double> { typedef double type; };

// Parameters::avg_p (Parameters.cpp:37-45): harmonic mean, 0 when both are 0.
__device__ __forceinline__ double harm(double a, double b) { return (a + b == 0) ? 0.0 : 2 * a * b / (a + b); }

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// Single-shot fused leap-frog step: block-row SpMV + inverse mass + leap-frog
// update + source injection + receiver sampling (+ energy).
//
// A team of T lanes owns one element row; lane l owns row pairs
// (2q, 2q+1), q = l + T*s. For each block column the team reads R contiguous
// entries (one coalesced run), the column's x value is a shared-memory
// broadcast. Small teams are packed TPW per warp.
// ---------------------------------------------------------------------------
template <int R, typename BT>
struct RowTeam {
  static constexpr int NPAIR = R / 2;
  static constexpr int T = NPAIR <= 32 ? NPAIR : 32;
  static constexpr int PPL = (NPAIR + T - 1) / T;
  static constexpr int TPW = 32 / T;
  static constexpr int WARPS = 8;
  static constexpr int THREADS = WARPS * 32;
  static constexpr int TEAMS_PER_CTA = WARPS * TPW;
};

// Columns per unrolled step of k_step_rows' block loop: enough block loads in
// flight per lane to stream the blocks at the HBM rate. FP64 blocks: 8
// columns where 2Np is a multiple of 8, else the largest divisor of 2Np up to
// 21; 4- and 2-byte blocks: the largest divisor of 2Np up to 32 (28 at
// 2Np = 56, 21 at 42). Measured, one shot (fractions of the measured HBM
// copy bandwidth): 160,000 triangles, N = 6, FP32 blocks, 8 columns 1.629 ms
// per step (78 %), 14 columns 1.362 ms (94 %), 28 columns 1.237 ms (103 %);
// FP64 blocks 8 columns 2.394 ms (105 %), 14 columns 2.415 ms; 40,000
// triangles, N = 5, FP64 blocks, 8 columns 0.386 ms (92 %), 14 columns
// 0.351 ms (101 %), 21 columns 0.349 ms (102 %). The FMA chains keep their
// column order: the same bits either way.
// Lanes that own two row pairs (2Np > 64) hold twice the loads per column:
// the cap is halved there, which keeps 2Np = 72 at two CTAs per SM (FP32
// blocks unrolled by 24 took 136 registers, one CTA).
template <int R, typename BT>
constexpr int row_unroll() {
  if (sizeof(BT) == 8 && R % 8 == 0) return 8;
  const int ppl = (R / 2 + 31) / 32;
  const int cap = (sizeof(BT) == 8 ? 21 : 32) / ppl;
  int u = R < cap ? R : cap;
  while (R % u != 0) --u;
  return u;
}

template <int R, typename BT, bool PADDED>
__global__ void __launch_bounds__(256) k_step_rows(const StepParams p) {
  typedef RowTeam<R, BT> RT;
  typedef typename AccOf<BT>::type AT;
  constexpr int NP = R / 2;  // Np
  constexpr int T = RT::T, PPL = RT::PPL, TPW = RT::TPW, NPAIR = RT::NPAIR;
  __shared__ __align__(16) double xs[RT::WARPS][TPW][4][R];
  __shared__ double red[RT::WARPS];

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tw = lane / T;
  const int tl = lane - tw * T;
  // Team g owns (element e, shot sh); the S shots of one element row are
  // consecutive teams, so their block reads hit L2 after the first.
  const long long g = (static_cast<long long>(blockIdx.x) * RT::WARPS + warp) * TPW + tw;
  const int S = p.S;
  const int e = static_cast<int>(g / S);
  const int sh = static_cast<int>(g - static_cast<long long>(e) * S);
  const bool active = (tw < TPW) && (e < p.ne);
  const size_t me = (static_cast<size_t>(e) * S + sh) * R;  // this team's state offset

  int rb = 0, nb = 0;
  double (*xt)[R] = xs[warp][tw < TPW ? tw : 0];
  if (active) {
    row_span(p, e, rb, nb);
    // Gather x of the row's block columns: contiguous 2Np modes per element.
    for (int b = 0; b < nb; ++b) {
      const int c = col_at(p, rb + b);
      const double2* src = reinterpret_cast<const double2*>(p.x + (size_t(c) * S + sh) * R);
      const double xs = (p.mode == kModePower) ? (p.xscale_mesh ? p.xscale_mesh[p.mesh_of[e]] : p.xscale) : 1.0;
      for (int q = tl; q < NPAIR; q += T) {
        double2 v = __ldg(src + q);
        if (p.mode == kModePower) { v.x *= xs; v.y *= xs; }
        xt[b][2 * q] = v.x;
        xt[b][2 * q + 1] = v.y;
      }
    }
  }
  __syncwarp();

  AT acc[PPL][2];
#pragma unroll
  for (int s = 0; s < PPL; ++s) acc[s][0] = acc[s][1] = AT(0);

  if (active) {
    // Column pitch: 2Np for single-shot storage, rounded up to 4 when the
    // blocks are stored for the batched kernels (compile-time either way).
    constexpr int P = PADDED ? ((R + 3) & ~3) : R;
    const BT* blk = reinterpret_cast<const BT*>(p.blocks) + size_t(rb) * R * P;
    for (int b = 0; b < nb; ++b, blk += R * P) {
      AT part[PPL][2];
#pragma unroll
      for (int s = 0; s < PPL; ++s) part[s][0] = part[s][1] = AT(0);
      constexpr int CU = row_unroll<R, BT>();
#pragma unroll CU
      for (int c = 0; c < R; ++c) {
        const AT xv = AT(xt[b][c]);
#pragma unroll
        for (int s = 0; s < PPL; ++s) {
          const int q = tl + T * s;
          if (q < NPAIR) {
            AT w0, w1;
            Pair<BT>::load(blk + c * P + 2 * q, w0, w1);
            part[s][0] = fma(w0, xv, part[s][0]);
            part[s][1] = fma(w1, xv, part[s][1]);
          }
        }
      }
      if (p.bscale != nullptr) {
        const AT sc = AT(p.bscale[rb + b]);
#pragma unroll
        for (int s = 0; s < PPL; ++s) {
          acc[s][0] = fma(sc, part[s][0], acc[s][0]);
          acc[s][1] = fma(sc, part[s][1], acc[s][1]);
        }
      } else {
#pragma unroll
        for (int s = 0; s < PPL; ++s) {
          acc[s][0] += part[s][0];
          acc[s][1] += part[s][1];
        }
      }
    }
  }

  // ---- epilogue: inverse mass, leap-frog, source ----
  const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
  double unew[PPL][2];
  double en = 0.0;  // energy / Rayleigh partials
  double en2 = 0.0, en3 = 0.0;
  if (active) {
    const double mi = p.minv[e];
    // Source row: the shot's own source (one per shot), or in a multi-mesh
    // group the source of this element's mesh.
    const int srow = p.src_of ? p.src_of[e] : ((p.src_elem != nullptr && src_elem_at(p, sh) == e) ? sh : -1);
    const bool is_src = (srow >= 0) && (k < p.nF) && (p.mode == kModeStep || p.mode == kModeFirst);
    double Fk[2] = {0.0, 0.0};
    if (is_src) {
      Fk[0] = p.F[(size_t(srow) * p.nF + k) * 2];
      Fk[1] = p.F[(size_t(srow) * p.nF + k) * 2 + 1];
    }
    const double dt = p.dt_elem ? p.dt_elem[e] : p.dt;
#pragma unroll
    for (int s = 0; s < PPL; ++s) {
      const int q = tl + T * s;
      if (q >= NPAIR) continue;
      double y[2] = {double(acc[s][0]), double(acc[s][1])};
      double* o = p.out + me + 2 * q;
      double u[2] = {xt[0][2 * q], xt[0][2 * q + 1]};
      double f[2] = {0.0, 0.0};
      if (is_src) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = 2 * q + h;
          const int comp = r / NP, i = r - comp * NP;
          f[h] = Fk[comp] * p.src_phi[size_t(srow) * NP + i];
        }
      }
      if (p.mode == kModeStep) {
        const double2 up = *reinterpret_cast<const double2*>(p.uprev + me + 2 * q);
        const double upv[2] = {up.x, up.y};
#pragma unroll
        for (int h = 0; h < 2; ++h) unew[s][h] = (2 * u[h] - upv[h]) + mi * ((-dt * dt) * (y[h] - f[h]));
      } else if (p.mode == kModeFirst) {
        double v0[2] = {0.0, 0.0};
        if (p.uprev != nullptr) {
          const double2 vv = *reinterpret_cast<const double2*>(p.uprev + me + 2 * q);
          v0[0] = vv.x;
          v0[1] = vv.y;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) unew[s][h] = (u[h] + dt * v0[h]) - mi * (dt * dt / 2 * (y[h] - f[h]));
      } else if (p.mode == kModeApply) {
        unew[s][0] = y[0];
        unew[s][1] = y[1];
      } else {  // kModePower
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          unew[s][h] = mi * y[h];
          en += u[h] * y[h];
          en2 += u[h] * u[h] / mi;
          en3 += unew[s][h] * unew[s][h];
        }
      }
      *reinterpret_cast<double2*>(o) = make_double2(unew[s][0], unew[s][1]);
      note_nonfinite(p, unew[s][0], unew[s][1]);
      if (p.energy != nullptr && (p.mode == kModeStep || p.mode == kModeFirst)) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const double d = unew[s][h] - u[h];
          en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * unew[s][h] * y[h];
        }
      }
    }
  }

  // ---- receivers: sample the new level of this element ----
  if (p.rcv_ptr != nullptr && (p.mode == kModeStep || p.mode == kModeFirst)) {
    __syncwarp();
    int r0 = 0, r1 = 0;
    if (active) {
      r0 = rcv_ptr_at(p, e);
      r1 = rcv_ptr_at(p, e + 1);
      if (r1 > r0) {
#pragma unroll
        for (int s = 0; s < PPL; ++s) {
          const int q = tl + T * s;
          if (q < NPAIR) {
            xt[1][2 * q] = unew[s][0];
            xt[1][2 * q + 1] = unew[s][1];
          }
        }
      }
    }
    __syncwarp();
    if (active && r1 > r0) {
      const long long slot = k % p.seis_cap;
      for (int t = tl; t < 2 * (r1 - r0); t += T) {
        const int rid = rcv_id_at(p, r0 + t / 2);
        const int comp = t & 1;
        const double* ph = p.rcv_phi + size_t(rid) * NP;
        double v = 0.0;
        for (int i = 0; i < NP; ++i) v += ph[i] * xt[1][comp * NP + i];
        p.seis[((size_t(sh) * p.seis_cap + slot) * p.nrcv + rid) * 2 + comp] = v;
      }
    }
  }

  // ---- per-mesh power-iteration sums (multi-mesh groups) ----
  if (p.mode == kModePower && p.mesh_of != nullptr) {
    // Team-segmented sum through shared memory: teams of one warp can
    // belong to different meshes.
    __shared__ double tsum[RT::WARPS][32][3];
    tsum[warp][lane][0] = en;
    tsum[warp][lane][1] = en2;
    tsum[warp][lane][2] = en3;
    __syncwarp();
    if (active && tl == 0) {
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      for (int l2 = 0; l2 < T; ++l2) {
        a0 += tsum[warp][tw * T + l2][0];
        a1 += tsum[warp][tw * T + l2][1];
        a2 += tsum[warp][tw * T + l2][2];
      }
      double* acc3 = p.acc + 3 * size_t(p.mesh_of[e]);
      atomicAdd(acc3 + 0, a0);
      atomicAdd(acc3 + 1, a1);
      atomicAdd(acc3 + 2, a2);
    }
    return;
  }
  // ---- block reductions (energy, power iteration) ----
  if (p.mode == kModePower || p.energy != nullptr) {
    const int nred = (p.mode == kModePower) ? 3 : 1;
    for (int w = 0; w < nred; ++w) {
      double v = warp_sum(w == 0 ? en : (w == 1 ? en2 : en3));
      __syncthreads();
      if (lane == 0) red[warp] = v;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < RT::WARPS; ++i) t += red[i];
        if (p.mode == kModePower) atomicAdd(p.acc + w, t);
        else atomicAdd(p.energy + (k % p.energy_cap), t);
      }
    }
  }
}


// ---------------------------------------------------------------------------
// Batched multi-shot step: per element row a (shots x 2Np) += (shots x K) .
// (K x 2Np) GEMM over the row's blocks, K = 2Np per block, on CUDA cores in
// the accumulation type (FP32 for FP32/BF16 blocks, FP64 for FP64 blocks),
// followed by the same fused leap-frog / source / receiver epilogue.
//
// One CTA owns (element row e, 64 shots). Per block: the block (column pitch
// RP = 2Np rounded up to 4, zero padded) and the neighbour's state X (64
// shots x 2Np, FP64, converted once) are staged in shared memory; X is
// stored transposed ([c][shot]) so that each thread's 4 shots and 4 rows are
// two 16-byte shared loads per k. Thread (tx, ty) owns shots 4tx..4tx+3 and
// rows 4ty..4ty+3: 16 FMAs per k.
// ---------------------------------------------------------------------------
template <int R>
struct BatchCfg {
  static constexpr int RP = (R + 3) & ~3;
  static constexpr int ST = 64;       // shots per CTA
  static constexpr int SP = ST + 4;   // pitch of a transposed X row
  static constexpr int TY = RP / 4;
  static constexpr int THREADS = 16 * TY;
  static constexpr int NT = ((THREADS + 31) / 32) * 32;
  template <typename AT>
  static constexpr size_t smem_bytes() { return size_t(R) * (RP + SP) * sizeof(AT) + (NT / 32) * sizeof(double); }
};

template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
  static __device__ __forceinline__ void ld(const float* p, float* v) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
};
template <>
struct Vec4<double> {
  static __device__ __forceinline__ void ld(const double* p, double* v) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
};

template <typename BT, typename AT>
__device__ __forceinline__ AT to_acc(BT v) { return AT(v); }
template <>
__device__ __forceinline__ float to_acc<__nv_bfloat16, float>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <int R, typename BT>
__global__ void __launch_bounds__(BatchCfg<R>::NT) k_step_batched(const StepParams p) {
  typedef BatchCfg<R> CF;
  typedef typename AccOf<BT>::type AT;
  constexpr int NP = R / 2, RP = CF::RP, ST = CF::ST, SP = CF::SP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  AT* Bs = reinterpret_cast<AT*>(smem_raw);                 // [R][RP]
  AT* Xs = Bs + R * RP;                                      // [R][SP]
  double* red = reinterpret_cast<double*>(Xs + R * SP);      // [NT/32]

  const int e = blockIdx.x;
  const int s0 = blockIdx.y * ST;
  const int S = p.S;
  const int t = threadIdx.x;
  const int tx = t & 15, ty = t >> 4;
  const bool comp = ty < CF::TY;
  int rb, nb;
  row_span(p, e, rb, nb);
  const BT* blocks = reinterpret_cast<const BT*>(p.blocks);

  AT acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = AT(0);

  for (int b = 0; b < nb; ++b) {
    const int c = col_at(p, rb + b);
    // Stage the block (already in the padded column-major layout).
    const BT* gb = blocks + size_t(rb + b) * R * RP;
    for (int i = t; i < R * RP; i += CF::NT) Bs[i] = to_acc<BT, AT>(gb[i]);
    // Stage X^T: thread -> (shot, row pair); shots vary fastest so the
    // transposed shared stores are conflict-free.
    const double* gx = p.x + size_t(c) * S * R;
    for (int i = t; i < ST * NP; i += CF::NT) {
      const int sl = i % ST, pr = i / ST;
      const int sh = s0 + sl;
      double2 v = make_double2(0.0, 0.0);
      if (sh < S) v = __ldg(reinterpret_cast<const double2*>(gx + size_t(sh) * R) + pr);
      Xs[(2 * pr) * SP + sl] = AT(v.x);
      Xs[(2 * pr + 1) * SP + sl] = AT(v.y);
    }
    __syncthreads();
    if (comp) {
#pragma unroll 6
      for (int cc = 0; cc < R; ++cc) {
        AT xv[4], bv[4];
        Vec4<AT>::ld(&Xs[cc * SP + 4 * tx], xv);
        Vec4<AT>::ld(&Bs[cc * RP + 4 * ty], bv);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fma(xv[i], bv[j], acc[i][j]);
      }
    }
    __syncthreads();
  }

  // ---- epilogue ----
  const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
  const double mi = p.minv[e];
  const double dt = p.dt;
  double en = 0.0;
  if (comp) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int sh = s0 + 4 * tx + i;
      if (sh >= S) continue;
      const size_t me = (size_t(e) * S + sh) * R;
      const bool is_src = (src_elem_at(p, sh) == e) && (k < p.nF);
      double Fk[2] = {0.0, 0.0};
      if (is_src) {
        Fk[0] = p.F[(size_t(sh) * p.nF + k) * 2];
        Fk[1] = p.F[(size_t(sh) * p.nF + k) * 2 + 1];
      }
#pragma unroll
      for (int jp = 0; jp < 2; ++jp) {
        const int r0 = 4 * ty + 2 * jp;
        if (r0 >= R) continue;  // rows come in pairs (R is even)
        const double2 uu = __ldg(reinterpret_cast<const double2*>(p.x + me + r0));
        // kModeStep: u^{k-1}; kModeFirst: v^0 (absent means zero).
        const double2 up = p.uprev ? *reinterpret_cast<const double2*>(p.uprev + me + r0) : make_double2(0.0, 0.0);
        const double u[2] = {uu.x, uu.y}, upv[2] = {up.x, up.y};
        double un[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = r0 + h;
          const int cmp = r / NP, ii = r - cmp * NP;
          const double f = is_src ? Fk[cmp] * p.src_phi[size_t(sh) * NP + ii] : 0.0;
          const double y = double(acc[i][2 * jp + h]);
          if (p.mode == kModeStep) un[h] = (2 * u[h] - upv[h]) + mi * ((-dt * dt) * (y - f));
          else un[h] = (u[h] + dt * upv[h]) - mi * (dt * dt / 2 * (y - f));  // kModeFirst, uprev = v0
          if (p.energy != nullptr) {
            const double d = un[h] - u[h];
            en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un[h] * y;
          }
        }
        *reinterpret_cast<double2*>(p.out + me + r0) = make_double2(un[0], un[1]);
        note_nonfinite(p, un[0], un[1]);
      }
    }
  }

  // ---- receivers ----
  if (p.rcv_ptr != nullptr) {
    const int q0 = rcv_ptr_at(p, e), q1 = rcv_ptr_at(p, e + 1);
    if (q1 > q0) {
      __syncthreads();  // this CTA's writes of u^{k+1} are visible after the barrier
      const long long slot = k % p.seis_cap;
      const int nwork = (q1 - q0) * ST * 2;
      for (int w = t; w < nwork; w += CF::NT) {
        const int cmp = w & 1, sl = (w >> 1) % ST, q = q0 + (w >> 1) / ST;
        const int sh = s0 + sl;
        if (sh >= S) continue;
        const int rid = rcv_id_at(p, q);
        const double* ph = p.rcv_phi + size_t(rid) * NP;
        const double* un = p.out + (size_t(e) * S + sh) * R + cmp * NP;
        double v = 0.0;
        for (int ii = 0; ii < NP; ++ii) v += ph[ii] * un[ii];
        p.seis[((size_t(sh) * p.seis_cap + slot) * p.nrcv + rid) * 2 + cmp] = v;
      }
    }
  }

  // ---- energy ----
  if (p.energy != nullptr) {
    const double v = warp_sum(en);
    if ((t & 31) == 0) red[t >> 5] = v;
    __syncthreads();
    if (t == 0) {
      double sum = 0.0;
      for (int w = 0; w < CF::NT / 32; ++w) sum += red[w];
      atomicAdd(p.energy + (k % p.energy_cap), sum);
    }
  }
}


__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Batched FP64 step on the FP64 tensor cores (DMMA, mma.sync m8n8k4 .f64).
// Exact FP64 products and FP64 accumulation, so the result is the plain
// FP64 step's up to summation order. Per CTA: one element row and a tile of
// ST shots; per block of the row, Y[shot][r] += X_c[shot][k] B[r][k] as a
// (ST x KP) . (KP x 8*NTL) product, KP = R padded to the MMA's k = 4.
// The WM x WN warps split it: warp (wm, wn) owns MTW m-tiles of 8 shots
// and NTW n-tiles of 8 operator rows. Blocks and the neighbours' state tiles
// are staged global->shared with 16-byte cp.async into a two-stage ring
// (block b+1 copies while block b multiplies). Shared pitches PS satisfy
// PS mod 16 in {4, 12}, which makes both fragment loads conflict-free.
// The K padding (columns R..KP-1 of X and of B) is zeroed once; C columns
// n >= R read operator entries of the next column and are discarded.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int d64_pitch(int kp) { return (kp % 16 == 4 || kp % 16 == 12) ? kp : d64_pitch(kp + 2); }

template <int R>
struct D64Cfg {
  static constexpr int KP = (R + 3) & ~3;
  static constexpr int NTL = (R + 7) / 8;
  static constexpr int PS = d64_pitch(KP);
  static constexpr int ST = R <= 42 ? 64 : 32;     // shots per CTA
  static constexpr int WM = 4, WN = 2, WARPS = WM * WN;
  static constexpr int MTW = ST / (8 * WM);        // m-tiles per warp
  static constexpr int NTW = (NTL + WN - 1) / WN;  // n-tiles per warp
  static constexpr int NT = WARPS * 32;
  static constexpr int BSZ = KP * PS;              // doubles: B stage [k][n]
  static constexpr int XSZ = ST * PS;              // doubles: X stage [shot][k]
  static constexpr int STAGE = BSZ + XSZ;
  static constexpr size_t smem_bytes() { return size_t(2) * STAGE * sizeof(double) + WARPS * sizeof(double); }
};

__device__ __forceinline__ void dmma_m8n8k4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// FP64 tensor-core throughput probe for the benchmark's roofline: every warp
// runs 8 independent DMMA accumulation chains on register operands, nothing
// is read from memory; the result is written only under a condition that
// never holds, so the loop is not removed.
__global__ void k_fp64_tensor_peak(double* sink, int iters) {
  double c[8][2];
#pragma unroll
  for (int j = 0; j < 8; ++j) c[j][0] = c[j][1] = 0.0;
  const double a = 1e-3 * (threadIdx.x + 1), b = 1.0 + 1e-9 * blockIdx.x;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) dmma_m8n8k4(c[j][0], c[j][1], a, b);
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += c[j][0] + c[j][1];
  if (s == -1.0) *sink = s;
}

template <int R>
__global__ void __launch_bounds__(D64Cfg<R>::NT, 3) k_step_batched64d(const StepParams p) {
  typedef D64Cfg<R> CF;
  constexpr int NP = R / 2, KP = CF::KP, PS = CF::PS, ST = CF::ST, NTL = CF::NTL, MTW = CF::MTW, NTW = CF::NTW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* stage0 = reinterpret_cast<double*>(smem_raw);
  double* red = stage0 + 2 * CF::STAGE;

  const int e = blockIdx.x;
  const int s0 = blockIdx.y * ST;
  const int S = p.S;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int wm = w % CF::WM, wn = w / CF::WM;
  const int g = lane >> 2, tg = lane & 3;
  int rb, nb;
  row_span(p, e, rb, nb);
  const double* blocks = reinterpret_cast<const double*>(p.blocks);
  const int nsh = min(ST, S - s0);  // shots of this tile

  // Zero what cp.async never writes: K padding of B and X, and the X rows of
  // shots beyond S, in both stages.
  for (int st = 0; st < 2; ++st) {
    double* B = stage0 + st * CF::STAGE;
    double* X = B + CF::BSZ;
    for (int i = t; i < (KP - R) * PS; i += CF::NT) B[R * PS + i] = 0.0;
    if constexpr (PS > R) {
      for (int i = t; i < ST * (PS - R); i += CF::NT) {
        const int r = i / (PS - R), c = R + i % (PS - R);
        X[r * PS + c] = 0.0;
      }
    }
    for (int i = t; i < (ST - nsh) * R; i += CF::NT) {
      const int r = nsh + i / R, c = i % R;
      X[r * PS + c] = 0.0;
    }
  }

  auto issue = [&](int b, int st) {
    double* B = stage0 + st * CF::STAGE;
    double* X = B + CF::BSZ;
    const double* gb = blocks + size_t(rb + b) * R * p.bpitch;
    for (int i = t; i < R * NP; i += CF::NT) {  // column k, 16-byte chunk j
      const int k = i / NP, j = i - k * NP;
      cp_async16(B + k * PS + 2 * j, gb + size_t(k) * p.bpitch + 2 * j);
    }
    const int c = col_at(p, rb + b);
    const double* gx = p.x + (size_t(c) * S + s0) * R;
    for (int i = t; i < nsh * NP; i += CF::NT) {
      const int r = i / NP, j = i - r * NP;
      cp_async16(X + r * PS + 2 * j, gx + size_t(r) * R + 2 * j);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };

  double acc[MTW][NTW][2];
#pragma unroll
  for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
    for (int q = 0; q < NTW; ++q) acc[mt][q][0] = acc[mt][q][1] = 0.0;
  // n-tiles of this warp that exist (warp-uniform).
  const int nt0 = wn * NTW, ntn = min(NTW, NTL - nt0);

  issue(0, 0);
  for (int b = 0; b < nb; ++b) {
    if (b + 1 < nb) {
      issue(b + 1, (b + 1) & 1);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();
    const double* B = stage0 + (b & 1) * CF::STAGE;
    const double* X = B + CF::BSZ + (wm * MTW * 8 + g) * PS + tg;
    const double* Bt = B + tg * PS + nt0 * 8 + g;
#pragma unroll 1
    for (int k0 = 0; k0 < KP; k0 += 4) {
      double a[MTW], bb[NTW];
#pragma unroll
      for (int mt = 0; mt < MTW; ++mt) a[mt] = X[mt * 8 * PS + k0];
#pragma unroll
      for (int q = 0; q < NTW; ++q) bb[q] = (q < ntn) ? Bt[k0 * PS + q * 8] : 0.0;
#pragma unroll
      for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
        for (int q = 0; q < NTW; ++q)
          if (q < ntn) dmma_m8n8k4(acc[mt][q][0], acc[mt][q][1], a[mt], bb[q]);
    }
    __syncthreads();
  }

  // ---- epilogue: thread holds rows (8(nt0+q) + 2tg, +1) of shots 8(wm*MTW + mt) + g ----
  const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
  const double mi = p.minv[e];
  const double dt = p.dt;
  double en = 0.0;
#pragma unroll
  for (int mt = 0; mt < MTW; ++mt) {
    const int sh = s0 + (wm * MTW + mt) * 8 + g;
    if (sh >= S) continue;
    const size_t me = (size_t(e) * S + sh) * R;
    const bool is_src = (src_elem_at(p, sh) == e) && (k < p.nF);
    double Fk[2] = {0.0, 0.0};
    if (is_src) {
      Fk[0] = p.F[(size_t(sh) * p.nF + k) * 2];
      Fk[1] = p.F[(size_t(sh) * p.nF + k) * 2 + 1];
    }
#pragma unroll
    for (int q = 0; q < NTW; ++q) {
      const int r0 = (nt0 + q) * 8 + 2 * tg;
      if (q >= ntn || r0 >= R) continue;  // rows come in pairs (R is even)
      const double2 uu = __ldg(reinterpret_cast<const double2*>(p.x + me + r0));
      const double2 up = p.uprev ? *reinterpret_cast<const double2*>(p.uprev + me + r0) : make_double2(0.0, 0.0);
      const double u[2] = {uu.x, uu.y}, upv[2] = {up.x, up.y};
      double un[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = r0 + h;
        const int cmp = r / NP, ii = r - cmp * NP;
        const double f = is_src ? Fk[cmp] * p.src_phi[size_t(sh) * NP + ii] : 0.0;
        const double y = acc[mt][q][h];
        if (p.mode == kModeStep) un[h] = (2 * u[h] - upv[h]) + mi * ((-dt * dt) * (y - f));
        else un[h] = (u[h] + dt * upv[h]) - mi * (dt * dt / 2 * (y - f));  // kModeFirst, uprev = v0
        if (p.energy != nullptr) {
          const double d = un[h] - u[h];
          en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un[h] * y;
        }
      }
      *reinterpret_cast<double2*>(p.out + me + r0) = make_double2(un[0], un[1]);
      note_nonfinite(p, un[0], un[1]);
    }
  }

  // ---- receivers ----
  if (p.rcv_ptr != nullptr) {
    const int q0 = rcv_ptr_at(p, e), q1 = rcv_ptr_at(p, e + 1);
    if (q1 > q0) {
      __syncthreads();  // this CTA's writes of u^{k+1} are visible after the barrier
      const long long slot = k % p.seis_cap;
      const int nwork = (q1 - q0) * ST * 2;
      for (int wk = t; wk < nwork; wk += CF::NT) {
        const int cmp = wk & 1, sl = (wk >> 1) % ST, q = q0 + (wk >> 1) / ST;
        const int sh = s0 + sl;
        if (sh >= S) continue;
        const int rid = rcv_id_at(p, q);
        const double* ph = p.rcv_phi + size_t(rid) * NP;
        const double* un = p.out + (size_t(e) * S + sh) * R + cmp * NP;
        double v = 0.0;
        for (int ii = 0; ii < NP; ++ii) v += ph[ii] * un[ii];
        p.seis[((size_t(sh) * p.seis_cap + slot) * p.nrcv + rid) * 2 + cmp] = v;
      }
    }
  }

  // ---- energy ----
  if (p.energy != nullptr) {
    const double v = warp_sum(en);
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (t == 0) {
      double sum = 0.0;
      for (int i = 0; i < CF::WARPS; ++i) sum += red[i];
      atomicAdd(p.energy + (k % p.energy_cap), sum);
    }
  }
}

// ---------------------------------------------------------------------------
// Batched FP32 step with asynchronous staging. Same GEMM as k_step_batched,
// but the neighbours' states come from the FP32 transposed shadow written by
// the previous step's epilogue, so the blocks and the state tiles of all the
// row's blocks are copied global->shared with cp.async (no register staging,
// no conversion) behind a single barrier. The epilogue writes u^{k+1} in FP64
// and its FP32 shadow (one 16-byte store per thread and row).
// ---------------------------------------------------------------------------
template <int R>
struct Batch32Cfg {
  static constexpr int RP = (R + 3) & ~3;
  static constexpr int ST = 64;
  static constexpr int SP = ST + 4;
  static constexpr int TY = RP / 4;
  static constexpr int NT = ((16 * TY + 31) / 32) * 32;
  static constexpr size_t smem_bytes() {
    return size_t(4) * R * (RP + SP) * sizeof(float) + (NT / 32) * sizeof(double);
  }
};


template <int R>
__global__ void __launch_bounds__(Batch32Cfg<R>::NT) k_step_batched32(const StepParams p) {
  typedef Batch32Cfg<R> CF;
  constexpr int NP = R / 2, RP = CF::RP, ST = CF::ST, SP = CF::SP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* Bs = reinterpret_cast<float*>(smem_raw);        // [4][R][RP]
  float* Xs = Bs + 4 * R * RP;                            // [4][R][SP]
  double* red = reinterpret_cast<double*>(Xs + 4 * R * SP);

  const int e = blockIdx.x;
  const int tile = blockIdx.y, ntile = gridDim.y;
  const int s0 = tile * ST;
  const int S = p.S;
  const int t = threadIdx.x;
  const int tx = t & 15, ty = t >> 4;
  const bool comp = ty < CF::TY;
  int rb, nb;
  row_span(p, e, rb, nb);

  // ---- stage every block of the row and every neighbour tile ----
  {
    const float* gb = reinterpret_cast<const float*>(p.blocks) + size_t(rb) * R * RP;
    const int nbc = nb * R * RP / 4;  // 16-byte chunks, blocks contiguous in HBM
    for (int i = t; i < nbc; i += CF::NT) cp_async16(Bs + 4 * i, gb + 4 * i);
    for (int b = 0; b < nb; ++b) {
      const int c = col_at(p, rb + b);
      const float* gx = p.x32_in + (size_t(c) * ntile + tile) * R * ST;
      float* sx = Xs + b * R * SP;
      for (int i = t; i < R * (ST / 4); i += CF::NT) {
        const int row = i / (ST / 4), ch = i - row * (ST / 4);
        cp_async16(sx + row * SP + 4 * ch, gx + row * ST + 4 * ch);
      }
    }
    cp_async_wait_all();
    __syncthreads();
  }

  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  if (comp) {
    for (int b = 0; b < nb; ++b) {
      const float* xb = Xs + b * R * SP + 4 * tx;
      const float* bb = Bs + b * R * RP + 4 * ty;
#pragma unroll 6
      for (int cc = 0; cc < R; ++cc) {
        const float4 xv = *reinterpret_cast<const float4*>(xb + cc * SP);
        const float4 bv = *reinterpret_cast<const float4*>(bb + cc * RP);
        const float xa[4] = {xv.x, xv.y, xv.z, xv.w}, ba[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(xa[i], ba[j], acc[i][j]);
      }
    }
  }

  // ---- epilogue: leap-frog in FP64, FP64 state + FP32 shadow out ----
  const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
  const double mi = p.minv[e];
  const double dt = p.dt;
  double en = 0.0;
  if (comp) {
    float sh32[4][4];  // [row j][shot i]
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) sh32[j][i] = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int sh = s0 + 4 * tx + i;
      if (sh >= S) continue;
      const size_t me = (size_t(e) * S + sh) * R;
      const bool is_src = (src_elem_at(p, sh) == e) && (k < p.nF);
      double Fk[2] = {0.0, 0.0};
      if (is_src) {
        Fk[0] = p.F[(size_t(sh) * p.nF + k) * 2];
        Fk[1] = p.F[(size_t(sh) * p.nF + k) * 2 + 1];
      }
#pragma unroll
      for (int jp = 0; jp < 2; ++jp) {
        const int r0 = 4 * ty + 2 * jp;
        if (r0 >= R) continue;
        const double2 uu = __ldg(reinterpret_cast<const double2*>(p.x + me + r0));
        const double2 up = p.uprev ? *reinterpret_cast<const double2*>(p.uprev + me + r0) : make_double2(0.0, 0.0);
        const double u[2] = {uu.x, uu.y}, upv[2] = {up.x, up.y};
        double un[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = r0 + h;
          const int cmp = r / NP, ii = r - cmp * NP;
          const double f = is_src ? Fk[cmp] * p.src_phi[size_t(sh) * NP + ii] : 0.0;
          const double y = double(acc[i][2 * jp + h]);
          if (p.mode == kModeStep) un[h] = (2 * u[h] - upv[h]) + mi * ((-dt * dt) * (y - f));
          else un[h] = (u[h] + dt * upv[h]) - mi * (dt * dt / 2 * (y - f));
          if (p.energy != nullptr) {
            const double d = un[h] - u[h];
            en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un[h] * y;
          }
          sh32[2 * jp + h][i] = float(un[h]);
        }
        *reinterpret_cast<double2*>(p.out + me + r0) = make_double2(un[0], un[1]);
        note_nonfinite(p, un[0], un[1]);
      }
    }
    float* gx = p.x32_out + (size_t(e) * ntile + tile) * R * ST + 4 * tx;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = 4 * ty + j;
      if (r < R) *reinterpret_cast<float4*>(gx + r * ST) = make_float4(sh32[j][0], sh32[j][1], sh32[j][2], sh32[j][3]);
    }
  }

  // ---- receivers ----
  if (p.rcv_ptr != nullptr) {
    const int q0 = rcv_ptr_at(p, e), q1 = rcv_ptr_at(p, e + 1);
    if (q1 > q0) {
      __syncthreads();
      const long long slot = k % p.seis_cap;
      const int nwork = (q1 - q0) * ST * 2;
      for (int w = t; w < nwork; w += CF::NT) {
        const int cmp = w & 1, sl = (w >> 1) % ST, q = q0 + (w >> 1) / ST;
        const int sh = s0 + sl;
        if (sh >= S) continue;
        const int rid = rcv_id_at(p, q);
        const double* ph = p.rcv_phi + size_t(rid) * NP;
        const double* un = p.out + (size_t(e) * S + sh) * R + cmp * NP;
        double v = 0.0;
        for (int ii = 0; ii < NP; ++ii) v += ph[ii] * un[ii];
        p.seis[((size_t(sh) * p.seis_cap + slot) * p.nrcv + rid) * 2 + cmp] = v;
      }
    }
  }

  if (p.energy != nullptr) {
    const double v = warp_sum(en);
    if ((t & 31) == 0) red[t >> 5] = v;
    __syncthreads();
    if (t == 0) {
      double sum = 0.0;
      for (int w = 0; w < CF::NT / 32; ++w) sum += red[w];
      atomicAdd(p.energy + (k % p.energy_cap), sum);
    }
  }
}

// ---------------------------------------------------------------------------
// Persistent, software-pipelined batched FP32 step (the production form of
// k_step_batched32). One CTA per SM walks the work items (element row,
// shot tile) round-robin. Per item i:
//   - cp.async group T_i: the item's FP64 state tiles u^k and u^{k-1}
//     (needed only by the epilogue, so their latency hides behind the GEMM);
//   - cp.async group G_{i+1}: the next item's blocks and neighbour FP32 tiles
//     into the other stage buffer;
//   - wait G_i, GEMM from shared memory, wait T_i, fused epilogue.
// Thread (tx, ty) owns shots 4tx..4tx+3 and rows TR*ty..TR*ty+TR-1.
// ---------------------------------------------------------------------------
template <int R, int ST, int TR>
struct PipeCfg {
  static constexpr int RP = (R + 3) & ~3;   // block column pitch (floats)
  static constexpr int UP = R + 2;          // state tile pitch (doubles)
  static constexpr int YP = R + 1;          // accumulator tile pitch (floats, odd: 2-way at most)
  static constexpr int HP = ST + 1;         // shadow staging pitch (floats)
  static constexpr int TX = ST / 4;
  static constexpr int TY = RP / TR;
  static constexpr int NT = ((TX * TY + 31) / 32) * 32;
  static constexpr int STAGE = 4 * R * RP + 4 * R * ST;  // floats per stage
  static constexpr size_t smem_bytes() {
    return size_t(2) * STAGE * sizeof(float) + size_t(2) * ST * UP * sizeof(double) +
           size_t(ST) * YP * sizeof(float) + size_t(R) * HP * sizeof(float) + (NT / 32) * sizeof(double) + 16;
  }
};

template <int TR>
struct RowVec;
template <>
struct RowVec<4> {
  static __device__ __forceinline__ void ld(const float* p, float* v) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
};
template <>
struct RowVec<2> {
  static __device__ __forceinline__ void ld(const float* p, float* v) {
    const float2 a = *reinterpret_cast<const float2*>(p);
    v[0] = a.x; v[1] = a.y;
  }
};

// GEMM of one block: acc[i][j] += X[cc][4tx+i] * B[cc][TR*ty+j] over cc, with
// the next column's operands loaded while the current one is consumed.
template <int R, int ST, int RP, int TR>
__device__ __forceinline__ void block_gemm(const float* __restrict__ xb, const float* __restrict__ bb,
                                           float (&acc)[4][TR]) {
  float4 xv = *reinterpret_cast<const float4*>(xb);
  float bv[TR];
  RowVec<TR>::ld(bb, bv);
#pragma unroll
  for (int cc = 0; cc < R; ++cc) {
    float4 xn = xv;
    float bn[TR];
#pragma unroll
    for (int j = 0; j < TR; ++j) bn[j] = bv[j];
    if (cc + 1 < R) {
      xn = *reinterpret_cast<const float4*>(xb + (cc + 1) * ST);
      RowVec<TR>::ld(bb + (cc + 1) * RP, bn);
    }
    const float xa[4] = {xv.x, xv.y, xv.z, xv.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < TR; ++j) acc[i][j] = fmaf(xa[i], bv[j], acc[i][j]);
    xv = xn;
#pragma unroll
    for (int j = 0; j < TR; ++j) bv[j] = bn[j];
  }
}

template <int R, int ST, int TR>
__global__ void __launch_bounds__(PipeCfg<R, ST, TR>::NT, 1) k_step_batched32p(const StepParams p) {
  typedef PipeCfg<R, ST, TR> CF;
  constexpr int NP = R / 2, RP = CF::RP, UP = CF::UP, YP = CF::YP, HP = CF::HP, TX = CF::TX, TY = CF::TY;
  constexpr int NPAIR = R / 2;
  constexpr int NTILE_SH = 64;  // shots per tile of the FP32 shadow layout
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* stage0 = reinterpret_cast<float*>(smem_raw);
  double* Uk = reinterpret_cast<double*>(stage0 + 2 * CF::STAGE);  // [ST][UP]
  double* Up = Uk + ST * UP;                                          // [ST][UP]
  float* Ys = reinterpret_cast<float*>(Up + ST * UP);                // [ST][YP]
  float* Hs = Ys + ST * YP;                                          // [R][HP]
  double* red = reinterpret_cast<double*>(reinterpret_cast<uintptr_t>(Hs + R * HP + 3) & ~uintptr_t(7));

  const int S = p.S;
  const int ntile = (S + ST - 1) / ST;
  const int nsh_tile = (S + NTILE_SH - 1) / NTILE_SH;
  const long long nitems = (long long)p.ne * ntile;
  const int t = threadIdx.x;
  const int tx = t % TX, ty = t / TX;
  const bool comp = ty < TY;
  const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
  const double dt = p.dt;

  auto issue_operands = [&](long long item, float* st) {
    const int e = int(item / ntile), tile = int(item - (long long)e * ntile);
    const int s0 = tile * ST;
    int rb, nb;
    row_span(p, e, rb, nb);
    float* Bs = st;
    float* Xs = st + 4 * R * RP;
    const float* gb = reinterpret_cast<const float*>(p.blocks) + size_t(rb) * R * RP;
    const int nbc = nb * R * RP / 4;
    for (int i = t; i < nbc; i += CF::NT) cp_async16(Bs + 4 * i, gb + 4 * i);
    const int sht = s0 / NTILE_SH, sho = s0 - sht * NTILE_SH;
    for (int b = 0; b < nb; ++b) {
      const int c = col_at(p, rb + b);
      const float* gx = p.x32_in + (size_t(c) * nsh_tile + sht) * R * NTILE_SH + sho;
      float* sx = Xs + b * R * ST;
      for (int i = t; i < R * (ST / 4); i += CF::NT) {
        const int row = i / (ST / 4), ch = i - row * (ST / 4);
        cp_async16(sx + row * ST + 4 * ch, gx + row * NTILE_SH + 4 * ch);
      }
    }
  };
  auto issue_state = [&](long long item) {
    const int e = int(item / ntile), tile = int(item - (long long)e * ntile);
    const int s0 = tile * ST;
    const int nsv = min(ST, S - s0);
    const double* gk = p.x + (size_t(e) * S + s0) * R;
    const double* gp = p.uprev ? p.uprev + (size_t(e) * S + s0) * R : nullptr;
    for (int i = t; i < nsv * NPAIR; i += CF::NT) {
      const int sl = i / NPAIR, ch = i - sl * NPAIR;
      cp_async16(Uk + sl * UP + 2 * ch, gk + size_t(sl) * R + 2 * ch);
      if (gp) cp_async16(Up + sl * UP + 2 * ch, gp + size_t(sl) * R + 2 * ch);
    }
  };

  long long item = blockIdx.x;
  int buf = 0;
  if (item < nitems) issue_operands(item, stage0);
  asm volatile("cp.async.commit_group;\n" ::: "memory");

  for (; item < nitems; item += gridDim.x, buf ^= 1) {
    const int e = int(item / ntile), tile = int(item - (long long)e * ntile);
    const int s0 = tile * ST;
    const int nsv = min(ST, S - s0);
    int rb, nb;
    row_span(p, e, rb, nb);
    float* st = stage0 + buf * CF::STAGE;
    issue_state(item);
    asm volatile("cp.async.commit_group;\n" ::: "memory");  // T_i
    const long long nxt = item + gridDim.x;
    if (nxt < nitems) issue_operands(nxt, stage0 + (buf ^ 1) * CF::STAGE);
    asm volatile("cp.async.commit_group;\n" ::: "memory");  // G_{i+1}
    asm volatile("cp.async.wait_group 2;\n" ::: "memory");  // G_i landed
    __syncthreads();

    float acc[4][TR];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < TR; ++j) acc[i][j] = 0.0f;
    if (comp) {
      const float* Bs = st;
      const float* Xs = st + 4 * R * RP;
      for (int b = 0; b < nb; ++b)
        block_gemm<R, ST, RP, TR>(Xs + b * R * ST + 4 * tx, Bs + b * R * RP + TR * ty, acc);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < TR; ++j)
          if (TR * ty + j < R) Ys[(4 * tx + i) * YP + TR * ty + j] = acc[i][j];
    }
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // T_i landed
    __syncthreads();

    // ---- epilogue, row-major mapping: thread -> (shot, row pair) ----
    const double mi = p.minv[e];
    double en = 0.0;
    for (int w = t; w < nsv * NPAIR; w += CF::NT) {
      const int sl = w / NPAIR, q = w - sl * NPAIR;
      const int sh = s0 + sl, r0 = 2 * q;
      const bool is_src = (src_elem_at(p, sh) == e) && (k < p.nF);
      const double2 uu = *reinterpret_cast<const double2*>(Uk + sl * UP + r0);
      const double2 up = p.uprev ? *reinterpret_cast<const double2*>(Up + sl * UP + r0) : make_double2(0.0, 0.0);
      const double u[2] = {uu.x, uu.y}, upv[2] = {up.x, up.y};
      double un[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = r0 + h;
        const int cmp = r / NP, ii = r - cmp * NP;
        const double f = is_src ? p.F[(size_t(sh) * p.nF + k) * 2 + cmp] * p.src_phi[size_t(sh) * NP + ii] : 0.0;
        const double y = double(Ys[sl * YP + r]);
        if (p.mode == kModeStep) un[h] = (2 * u[h] - upv[h]) + mi * ((-dt * dt) * (y - f));
        else un[h] = (u[h] + dt * upv[h]) - mi * (dt * dt / 2 * (y - f));
        if (p.energy != nullptr) {
          const double d = un[h] - u[h];
          en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un[h] * y;
        }
        Hs[r * HP + sl] = float(un[h]);
      }
      *reinterpret_cast<double2*>(p.out + (size_t(e) * S + sh) * R + r0) = make_double2(un[0], un[1]);
      note_nonfinite(p, un[0], un[1]);
    }
    __syncthreads();
    {
      // FP32 shadow of u^{k+1}: rows of the 64-shot layout, 16-byte stores.
      const int sht = s0 / NTILE_SH, sho = s0 - sht * NTILE_SH;
      float* gx = p.x32_out + (size_t(e) * nsh_tile + sht) * R * NTILE_SH + sho;
      for (int w = t; w < R * (ST / 4); w += CF::NT) {
        const int r = w / (ST / 4), c4 = w - r * (ST / 4);
        const float* hr = Hs + r * HP + 4 * c4;
        float4 v = make_float4(hr[0], hr[1], hr[2], hr[3]);
        if (4 * c4 + 3 >= nsv) {  // shots past S stay zero
          if (4 * c4 + 0 >= nsv) v.x = 0.f;
          if (4 * c4 + 1 >= nsv) v.y = 0.f;
          if (4 * c4 + 2 >= nsv) v.z = 0.f;
          if (4 * c4 + 3 >= nsv) v.w = 0.f;
        }
        *reinterpret_cast<float4*>(gx + r * NTILE_SH + 4 * c4) = v;
      }
    }

    if (p.rcv_ptr != nullptr) {
      const int q0 = rcv_ptr_at(p, e), q1 = rcv_ptr_at(p, e + 1);
      if (q1 > q0) {
        const long long slot = k % p.seis_cap;
        const int nwork = (q1 - q0) * ST * 2;
        for (int w = t; w < nwork; w += CF::NT) {
          const int cmp = w & 1, sl = (w >> 1) % ST, q = q0 + (w >> 1) / ST;
          if (sl >= nsv) continue;
          const int rid = rcv_id_at(p, q);
          const double* ph = p.rcv_phi + size_t(rid) * NP;
          // u^{k+1} of this item was written to global by the whole CTA
          // before the barrier above.
          const double* un = p.out + (size_t(e) * S + s0 + sl) * R + cmp * NP;
          double v = 0.0;
          for (int ii = 0; ii < NP; ++ii) v += ph[ii] * un[ii];
          p.seis[((size_t(s0 + sl) * p.seis_cap + slot) * p.nrcv + rid) * 2 + cmp] = v;
        }
      }
    }
    if (p.energy != nullptr) {
      const double v = warp_sum(en);
      if ((t & 31) == 0) red[t >> 5] = v;
      __syncthreads();
      if (t == 0) {
        double sum = 0.0;
        for (int w = 0; w < CF::NT / 32; ++w) sum += red[w];
        atomicAdd(p.energy + (k % p.energy_cap), sum);
      }
    }
    __syncthreads();  // stage buf, state tiles, Ys and Hs are reused
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Batched FP32 step, K split across warp groups (production kernel for
// 2Np <= 42). Four warp groups share a persistent CTA; group g multiplies
// block g of the current item's row (the row has at most 4 blocks), so the
// CTA runs 4x the warps of a single-tile GEMM. Partial tiles are reduced in
// shared memory by the epilogue. Operands for item i+1 are copied with
// cp.async into the other stage buffer while item i is computed; the FP64
// state is read directly by the epilogue with coalesced loads.
// ---------------------------------------------------------------------------
template <int R>
struct KsplitCfg {
  static constexpr int RP = (R + 3) & ~3;
  static constexpr int ST = 64;
  static constexpr int YP = R + 1;
  static constexpr int HP = ST + 1;
  static constexpr int TX = ST / 4;
  static constexpr int TY = RP / 4;
  static constexpr int GT = TX * TY;              // threads per warp group (multiple of 16)
  static constexpr int GTW = ((GT + 31) / 32) * 32;
  static constexpr int NT = 4 * GTW;
  static constexpr int STAGE = 4 * R * RP + 4 * R * ST;
  static constexpr size_t smem_bytes() {
    return size_t(2) * STAGE * sizeof(float) + size_t(4) * ST * YP * sizeof(float) + size_t(R) * HP * sizeof(float) +
           (NT / 32) * sizeof(double) + 16;
  }
};

template <int R>
__global__ void __launch_bounds__(KsplitCfg<R>::NT, 1) k_step_batched32k(const StepParams p) {
  typedef KsplitCfg<R> CF;
  constexpr int NP = R / 2, RP = CF::RP, ST = CF::ST, YP = CF::YP, HP = CF::HP, TX = CF::TX;
  constexpr int NPAIR = R / 2;
  constexpr int NTILE_SH = 64;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* stage0 = reinterpret_cast<float*>(smem_raw);
  float* Yp = stage0 + 2 * CF::STAGE;  // [4][ST][YP] partial products
  float* Hs = Yp + 4 * ST * YP;        // [R][HP] FP32 shadow staging
  double* red = reinterpret_cast<double*>(reinterpret_cast<uintptr_t>(Hs + R * HP + 3) & ~uintptr_t(7));

  const int S = p.S;
  const int ntile = (S + ST - 1) / ST;
  const int nsh_tile = (S + NTILE_SH - 1) / NTILE_SH;
  const long long nitems = (long long)p.ne * ntile;
  const int t = threadIdx.x;
  const int grp = t / CF::GTW, gt = t - grp * CF::GTW;
  const int tx = gt % TX, ty = gt / TX;
  const bool comp = gt < CF::GT;
  const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
  const double dt = p.dt;

  auto issue_operands = [&](long long item, float* st) {
    const int e = int(item / ntile), tile = int(item - (long long)e * ntile);
    const int s0 = tile * ST;
    int rb, nb;
    row_span(p, e, rb, nb);
    float* Bs = st;
    float* Xs = st + 4 * R * RP;
    const float* gb = reinterpret_cast<const float*>(p.blocks) + size_t(rb) * R * RP;
    const int nbc = nb * R * RP / 4;
    for (int i = t; i < nbc; i += CF::NT) cp_async16(Bs + 4 * i, gb + 4 * i);
    const int sht = s0 / NTILE_SH, sho = s0 - sht * NTILE_SH;
    for (int b = 0; b < nb; ++b) {
      const int c = col_at(p, rb + b);
      const float* gx = p.x32_in + (size_t(c) * nsh_tile + sht) * R * NTILE_SH + sho;
      float* sx = Xs + b * R * ST;
      for (int i = t; i < R * (ST / 4); i += CF::NT) {
        const int row = i / (ST / 4), ch = i - row * (ST / 4);
        cp_async16(sx + row * ST + 4 * ch, gx + row * NTILE_SH + 4 * ch);
      }
    }
  };

  long long item = blockIdx.x;
  int buf = 0;
  if (item < nitems) issue_operands(item, stage0);
  asm volatile("cp.async.commit_group;\n" ::: "memory");

  for (; item < nitems; item += gridDim.x, buf ^= 1) {
    const int e = int(item / ntile), tile = int(item - (long long)e * ntile);
    const int s0 = tile * ST;
    const int nsv = min(ST, S - s0);
    int rb, nb;
    row_span(p, e, rb, nb);
    float* st = stage0 + buf * CF::STAGE;
    const long long nxt = item + gridDim.x;
    if (nxt < nitems) issue_operands(nxt, stage0 + (buf ^ 1) * CF::STAGE);
    asm volatile("cp.async.commit_group;\n" ::: "memory");  // G_{i+1}
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // G_i landed
    __syncthreads();

    if (comp && grp < nb) {
      float acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
      block_gemm<R, ST, RP, 4>(st + 4 * R * RP + grp * R * ST + 4 * tx, st + grp * R * RP + 4 * ty, acc);
      float* yp = Yp + grp * ST * YP;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (4 * ty + j < R) yp[(4 * tx + i) * YP + 4 * ty + j] = acc[i][j];
    }
    __syncthreads();

    // ---- epilogue, row-major mapping: thread -> (shot, row pair) ----
    const double mi = p.minv[e];
    double en = 0.0;
    for (int w = t; w < nsv * NPAIR; w += CF::NT) {
      const int sl = w / NPAIR, q = w - sl * NPAIR;
      const int sh = s0 + sl, r0 = 2 * q;
      const size_t me = (size_t(e) * S + sh) * R + r0;
      const bool is_src = (src_elem_at(p, sh) == e) && (k < p.nF);
      const double2 uu = __ldg(reinterpret_cast<const double2*>(p.x + me));
      const double2 up = p.uprev ? *reinterpret_cast<const double2*>(p.uprev + me) : make_double2(0.0, 0.0);
      const double u[2] = {uu.x, uu.y}, upv[2] = {up.x, up.y};
      double un[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = r0 + h;
        const int cmp = r / NP, ii = r - cmp * NP;
        const double f = is_src ? p.F[(size_t(sh) * p.nF + k) * 2 + cmp] * p.src_phi[size_t(sh) * NP + ii] : 0.0;
        float ys = 0.0f;
        for (int g = 0; g < nb; ++g) ys += Yp[(g * ST + sl) * YP + r];
        const double y = double(ys);
        if (p.mode == kModeStep) un[h] = (2 * u[h] - upv[h]) + mi * ((-dt * dt) * (y - f));
        else un[h] = (u[h] + dt * upv[h]) - mi * (dt * dt / 2 * (y - f));
        if (p.energy != nullptr) {
          const double d = un[h] - u[h];
          en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un[h] * y;
        }
        Hs[r * HP + sl] = float(un[h]);
      }
      *reinterpret_cast<double2*>(p.out + me) = make_double2(un[0], un[1]);
      note_nonfinite(p, un[0], un[1]);
    }
    __syncthreads();
    {
      const int sht = s0 / NTILE_SH, sho = s0 - sht * NTILE_SH;
      float* gx = p.x32_out + (size_t(e) * nsh_tile + sht) * R * NTILE_SH + sho;
      for (int w = t; w < R * (ST / 4); w += CF::NT) {
        const int r = w / (ST / 4), c4 = w - r * (ST / 4);
        const float* hr = Hs + r * HP + 4 * c4;
        float4 v = make_float4(hr[0], hr[1], hr[2], hr[3]);
        if (4 * c4 + 3 >= nsv) {
          if (4 * c4 + 0 >= nsv) v.x = 0.f;
          if (4 * c4 + 1 >= nsv) v.y = 0.f;
          if (4 * c4 + 2 >= nsv) v.z = 0.f;
          if (4 * c4 + 3 >= nsv) v.w = 0.f;
        }
        *reinterpret_cast<float4*>(gx + r * NTILE_SH + 4 * c4) = v;
      }
    }
    if (p.rcv_ptr != nullptr) {
      const int q0 = rcv_ptr_at(p, e), q1 = rcv_ptr_at(p, e + 1);
      if (q1 > q0) {
        const long long slot = k % p.seis_cap;
        const int nwork = (q1 - q0) * ST * 2;
        for (int w = t; w < nwork; w += CF::NT) {
          const int cmp = w & 1, sl = (w >> 1) % ST, q = q0 + (w >> 1) / ST;
          if (sl >= nsv) continue;
          const int rid = rcv_id_at(p, q);
          const double* ph = p.rcv_phi + size_t(rid) * NP;
          const double* un = p.out + (size_t(e) * S + s0 + sl) * R + cmp * NP;
          double v = 0.0;
          for (int ii = 0; ii < NP; ++ii) v += ph[ii] * un[ii];
          p.seis[((size_t(s0 + sl) * p.seis_cap + slot) * p.nrcv + rid) * 2 + cmp] = v;
        }
      }
    }
    if (p.energy != nullptr) {
      const double v = warp_sum(en);
      if ((t & 31) == 0) red[t >> 5] = v;
      __syncthreads();
      if (t == 0) {
        double sum = 0.0;
        for (int w = 0; w < CF::NT / 32; ++w) sum += red[w];
        atomicAdd(p.energy + (k % p.energy_cap), sum);
      }
    }
    __syncthreads();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Shots [s0, s0+ns) of a device state u[(e*S + s)*2Np + c*Np + i] in the
// reference's vector layout out[s - s0][c*ne*Np + e*Np + i]
// (FESpace_imp.hpp:152-153): one thread per output value, coalesced writes.
// Tinv (optional, [Np][Np] row-major): the state holds w = L^T u per element
// and component; out = L^-T w, i.e. out_i = sum_j Tinv[j][i] w_j with
// Tinv = L^-1.
__global__ void k_state_to_ref(const double* __restrict__ u, int ne, int S, int Np, int s0, int ns,
                               double* __restrict__ out, const double* __restrict__ Tinv) {
  const long long per = 2ll * ne * Np;
  const long long n = per * ns;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const long long sl = o / per, rem = o - sl * per;
    const long long c = rem / ((long long)ne * Np), rem2 = rem - c * ne * Np;
    const long long e = rem2 / Np, i = rem2 - e * Np;
    const double* w = u + (e * S + s0 + sl) * 2 * Np + c * Np;
    if (Tinv) {
      double v = 0.0;
      for (int j = int(i); j < Np; ++j) v = fma(Tinv[j * Np + i], w[j], v);  // L^-1 is lower triangular
      out[o] = v;
    } else {
      out[o] = w[i];
    }
  }
}

// FP32 transposed shadow of a whole FP64 state (before first_step and after
// tsp_set_state): one thread per (element, tile, row, shot-in-tile).
__global__ void k_make_shadow(const double* __restrict__ u, float* __restrict__ x32, int ne, int S, int R,
                              int ntile) {
  const long long n = (long long)ne * ntile * R * 64;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int sl = int(i & 63);
    long long rest = i >> 6;
    const int r = int(rest % R);
    rest /= R;
    const int tile = int(rest % ntile);
    const long long e = rest / ntile;
    const int sh = tile * 64 + sl;
    x32[i] = (sh < S) ? float(u[(e * S + sh) * R + r]) : 0.0f;
  }
}


// ---------------------------------------------------------------------------
// Matrix-free step (FP64): the action of B on u^k is computed from the
// factorised reference-element tables and per-element geometry/materials
// instead of stored blocks. Same terms as the assembled operator
// (Matrices_imp.hpp:22-215 with I <- I + I^T and B = pen N^2 S + I + A),
// evaluated at quadrature points:
//   volume   y^m += |detJ| sum_ab K^{ab} (sum_n alpha^{mn}_ab x^n)
//   face l   with J^n(k) = u_e^n(k) - u_nb^n(Q-1-k) (jump at edge point k),
//            T_e^m(k) = sum_{n,a} beta^{nm}_a(e) g_e^n_a(k) (traction of u_e),
//            T_nb^m   = same on the neighbour's side with its own beta:
//     y^m_i += sum_k w_k b_i(k) [pen N^2 sum_n c_mn J^n - L/2 (T_e^m - T_nb^m)]
//            + sum_k w_k sum_a g^a_i(k) [-L/2 sum_n beta^{mn}_a(e) J^n]
// One warp per element; persistent CTAs keep the tables in shared memory.
// ---------------------------------------------------------------------------
struct MatFreeParams {
  const double* tables;  // packed KT | TRT | TR | w1 (see matfree_table_doubles)
  const double* invJ;    // [ne][4]
  const double* detJ;    // [ne]
  const double* lam;     // [ne]
  const double* mu;      // [ne]
  const double* elen;    // [ne][3]
  const double* enrm;    // [ne][3][2]
  const int* neigh;      // [ne][3]
  const int* nedge;      // [ne][3]
  double pen_n2;
};

template <int N>
struct MFCfg {
  static constexpr int NP = (N + 1) * (N + 2) / 2;
  static constexpr int Q = N + 1;
  static constexpr int R = 2 * NP;
  static constexpr int WARPS = 8;
  static constexpr int KT = 4 * NP * NP;       // KT[ab][j][i]
  static constexpr int TRT = 3 * NP * 3 * Q;   // TRT[l][j][r]
  static constexpr int TR = 3 * 3 * Q * NP;    // TR[l][r][i]
  static constexpr int TABLES = KT + TRT + TR + Q;
  static constexpr int WS = 2 * NP + 2 * NP + 8 * NP + 2 * 3 * Q + 2 * 3 * Q + 6 * Q;  // per-warp scratch
  static constexpr size_t smem_bytes() { return size_t(TABLES + WARPS * WS) * sizeof(double) + WARPS * sizeof(double); }
};

__device__ __forceinline__ void mf_beta(const MatFreeParams& q, int e, int l, double* beta /*[m][n][a]*/) {
  const double lam = q.lam[e], mu = q.mu[e];
  const double n0 = q.enrm[6 * size_t(e) + 2 * l], n1 = q.enrm[6 * size_t(e) + 2 * l + 1];
  const double* iJ = q.invJ + 4 * size_t(e);
  const double tau[4][2] = {{(lam + 2 * mu) * n0, mu * n1}, {lam * n1, mu * n0}, {mu * n1, lam * n0},
                            {mu * n0, (lam + 2 * mu) * n1}};
#pragma unroll
  for (int mn = 0; mn < 4; ++mn)
#pragma unroll
    for (int a = 0; a < 2; ++a) beta[mn * 2 + a] = tau[mn][0] * iJ[a] + tau[mn][1] * iJ[a + 2];
}

template <int N>
__global__ void __launch_bounds__(MFCfg<N>::WARPS * 32) k_step_matfree(const StepParams p, const MatFreeParams q) {
  typedef MFCfg<N> CF;
  constexpr int NP = CF::NP, Q = CF::Q, R = CF::R, Q3 = 3 * Q;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* tab = reinterpret_cast<double*>(smem_raw);
  const double* KT = tab;
  const double* TRT = KT + CF::KT;
  const double* TR = TRT + CF::TRT;
  const double* W1 = TR + CF::TR;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* ws = tab + CF::TABLES + warp * CF::WS;
  double* xe = ws;              // [2][NP]
  double* xn = xe + 2 * NP;     // [2][NP]
  double* zz = xn + 2 * NP;     // [8][NP]  z^{ab,m}, index (m*4 + ab)
  double* TE = zz + 8 * NP;     // [2][3Q]
  double* TN = TE + 2 * Q3;     // [2][3Q]
  double* FH = TN + 2 * Q3;     // [6][Q]: F^0, F^1, H^0_0, H^0_1, H^1_0, H^1_1
  double* red = tab + CF::TABLES + CF::WARPS * CF::WS;

  for (int i = threadIdx.x; i < CF::TABLES; i += blockDim.x) tab[i] = q.tables[i];
  __syncthreads();

  const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
  double en = 0.0, pw1 = 0.0, pw2 = 0.0;  // energy / power-iteration partials
  const int gw = blockIdx.x * CF::WARPS + warp, nw = gridDim.x * CF::WARPS;
  for (int e = gw; e < p.ne; e += nw) {
    const double* xg = p.x + size_t(e) * R;
    const double xsc = (p.mode == kModePower) ? (p.xscale_mesh ? p.xscale_mesh[p.mesh_of[e]] : p.xscale) : 1.0;
    for (int t = lane; t < R; t += 32) {
      double v = __ldg(xg + t);
      if (p.mode == kModePower) v *= xsc;
      xe[t] = v;
    }
    // alpha^{mn}_{ab} and z^{ab,m}_j = sum_n alpha^{mn}_ab x^n_j
    {
      const double lam = q.lam[e], mu = q.mu[e];
      const double* iJ = q.invJ + 4 * size_t(e);
      const double C[4][4] = {{lam + 2 * mu, 0, 0, mu}, {0, lam, mu, 0}, {0, mu, lam, 0}, {mu, 0, 0, lam + 2 * mu}};
      double al[16];
#pragma unroll
      for (int mn = 0; mn < 4; ++mn)
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            double s = 0.0;
#pragma unroll
            for (int kk = 0; kk < 2; ++kk)
#pragma unroll
              for (int ll = 0; ll < 2; ++ll) s += C[mn][kk * 2 + ll] * iJ[a + 2 * kk] * iJ[b + 2 * ll];
            al[mn * 4 + a * 2 + b] = s;
          }
      __syncwarp();
      for (int j = lane; j < NP; j += 32) {
        const double x0 = xe[j], x1 = xe[NP + j];
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
          for (int ab = 0; ab < 4; ++ab) zz[(m * 4 + ab) * NP + j] = al[(m * 2 + 0) * 4 + ab] * x0 + al[(m * 2 + 1) * 4 + ab] * x1;
      }
    }
    __syncwarp();
    constexpr int RS = (NP + 31) / 32;  // row slots per lane
    double acc[RS][2];
#pragma unroll
    for (int s = 0; s < RS; ++s) acc[s][0] = acc[s][1] = 0.0;
    // ---- volume ----
#pragma unroll
    for (int s = 0; s < RS; ++s) {
      const int i = lane + 32 * s;
      if (i < NP) {
        double a0 = 0.0, a1 = 0.0;
        for (int j = 0; j < NP; ++j) {
#pragma unroll
          for (int ab = 0; ab < 4; ++ab) {
            const double kv = KT[(ab * NP + j) * NP + i];
            a0 = fma(kv, zz[(0 * 4 + ab) * NP + j], a0);
            a1 = fma(kv, zz[(1 * 4 + ab) * NP + j], a1);
          }
        }
        const double adet = fabs(q.detJ[e]);
        acc[s][0] = adet * a0;
        acc[s][1] = adet * a1;
      }
    }
    // ---- faces ----
#pragma unroll 1
    for (int l = 0; l < 3; ++l) {
      const int nb = TSP_INDEX(q.neigh[3 * size_t(e) + l], -1, p.ne, kSiteNeigh);
      if (nb < 0) continue;
      const int lp = TSP_INDEX(q.nedge[3 * size_t(e) + l], 0, 3, kSiteNeigh);
      const double* xgn = p.x + size_t(nb) * R;
      for (int t = lane; t < R; t += 32) {
        double v = __ldg(xgn + t);
        if (p.mode == kModePower) v *= xsc;  // neighbours belong to the same mesh
        xn[t] = v;
      }
      __syncwarp();
      // Traces: values and reference gradients at the edge points, both sides.
      for (int task = lane; task < 2 * Q3; task += 32) {
        const bool self = task < Q3;
        const int r = self ? task : task - Q3;
        const double* T = TRT + (self ? l : lp) * NP * Q3;
        const double* xv = self ? xe : xn;
        double v0 = 0.0, v1 = 0.0;
        for (int j = 0; j < NP; ++j) {
          const double tv = T[j * Q3 + r];
          v0 = fma(tv, xv[j], v0);
          v1 = fma(tv, xv[NP + j], v1);
        }
        double* out = self ? TE : TN;
        out[r] = v0;
        out[Q3 + r] = v1;
      }
      __syncwarp();
      if (lane < Q) {
        const int kq = lane, kk = Q - 1 - lane;
        double be[8], bn[8];
        mf_beta(q, e, l, be);
        mf_beta(q, nb, lp, bn);
        const double al_ = harm(q.lam[e], q.lam[nb]), am_ = harm(q.mu[e], q.mu[nb]);
        const double n0 = q.enrm[6 * size_t(e) + 2 * l], n1 = q.enrm[6 * size_t(e) + 2 * l + 1];
        const double c00 = (al_ + 2 * am_) * n0 * n0 + 2 * am_ * n1 * n1;
        const double c11 = (al_ + 2 * am_) * n1 * n1 + 2 * am_ * n0 * n0;
        const double c01 = al_ * n0 * n1;
        const double L = q.elen[3 * size_t(e) + l];
        const double w = W1[kq];
        const double J0 = TE[kq] - TN[kk], J1 = TE[Q3 + kq] - TN[Q3 + kk];
        double Te[2], Tn[2];
#pragma unroll
        for (int m = 0; m < 2; ++m) {
          double se = 0.0, sn = 0.0;
#pragma unroll
          for (int n = 0; n < 2; ++n)
#pragma unroll
            for (int a = 0; a < 2; ++a) {
              se += be[(n * 2 + m) * 2 + a] * TE[n * Q3 + (1 + a) * Q + kq];
              sn += bn[(n * 2 + m) * 2 + a] * TN[n * Q3 + (1 + a) * Q + kk];
            }
          Te[m] = se;
          Tn[m] = sn;
        }
        FH[0 * Q + kq] = w * (q.pen_n2 * (c00 * J0 + c01 * J1) - 0.5 * L * (Te[0] - Tn[0]));
        FH[1 * Q + kq] = w * (q.pen_n2 * (c01 * J0 + c11 * J1) - 0.5 * L * (Te[1] - Tn[1]));
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
          for (int a = 0; a < 2; ++a)
            FH[(2 + m * 2 + a) * Q + kq] =
                -0.5 * L * w * (be[(m * 2 + 0) * 2 + a] * J0 + be[(m * 2 + 1) * 2 + a] * J1);
      }
      __syncwarp();
      const double* T = TR + l * Q3 * NP;
#pragma unroll
      for (int s = 0; s < RS; ++s) {
        const int i = lane + 32 * s;
        if (i < NP) {
          double a0 = 0.0, a1 = 0.0;
#pragma unroll
          for (int kq = 0; kq < Q; ++kq) {
            const double bv = T[kq * NP + i], g0 = T[(Q + kq) * NP + i], g1 = T[(2 * Q + kq) * NP + i];
            a0 += bv * FH[0 * Q + kq] + g0 * FH[2 * Q + kq] + g1 * FH[3 * Q + kq];
            a1 += bv * FH[1 * Q + kq] + g0 * FH[4 * Q + kq] + g1 * FH[5 * Q + kq];
          }
          acc[s][0] += a0;
          acc[s][1] += a1;
        }
      }
      __syncwarp();
    }
    // ---- epilogue (rows i: component 0 at i, component 1 at NP + i) ----
    const double mi = p.minv[e];
    const int srow = p.src_of ? p.src_of[e] : ((p.src_elem != nullptr && src_elem_at(p, 0) == e) ? 0 : -1);
    const bool is_src = (srow >= 0) && (k < p.nF) && (p.mode == kModeStep || p.mode == kModeFirst);
    const double dt = p.dt_elem ? p.dt_elem[e] : p.dt;
    double* og = p.out + size_t(e) * R;
    double ew = 0.0, pe0 = 0.0, pe1 = 0.0, pe2 = 0.0;  // this element's power-iteration sums
#pragma unroll
    for (int s = 0; s < RS; ++s) {
      const int i = lane + 32 * s;
      if (i >= NP) continue;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int r = c * NP + i;
        const double y = acc[s][c];
        const double u = xe[r];
        double un;
        if (p.mode == kModeStep || p.mode == kModeFirst) {
          const double f = is_src ? p.F[(size_t(srow) * p.nF + k) * 2 + c] * p.src_phi[size_t(srow) * NP + i] : 0.0;
          if (p.mode == kModeStep) un = (2 * u - p.uprev[size_t(e) * R + r]) + mi * ((-dt * dt) * (y - f));
          else un = (u + dt * (p.uprev ? p.uprev[size_t(e) * R + r] : 0.0)) - mi * (dt * dt / 2 * (y - f));
          if (p.energy != nullptr) {
            const double d = un - u;
            en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un * y;
          }
        } else if (p.mode == kModeApply) {
          un = y;
        } else {  // kModePower
          un = mi * y;
          pe0 += u * y;
          pe1 += u * u / mi;
          pe2 += un * un;
        }
        og[r] = un;
        note_nonfinite(p, un, 0.0);
      }
    }
    (void)ew;
    if (p.mode == kModePower) {
      if (p.mesh_of != nullptr) {
        const double v0 = warp_sum(pe0), v1 = warp_sum(pe1), v2 = warp_sum(pe2);
        if (lane == 0) {
          double* acc3 = p.acc + 3 * size_t(p.mesh_of[e]);
          atomicAdd(acc3 + 0, v0);
          atomicAdd(acc3 + 1, v1);
          atomicAdd(acc3 + 2, v2);
        }
      } else {
        en += pe0;
        pw1 += pe1;
        pw2 += pe2;
      }
    }
    // receivers of this element
    if (p.rcv_ptr != nullptr && (p.mode == kModeStep || p.mode == kModeFirst)) {
      const int r0 = rcv_ptr_at(p, e), r1 = rcv_ptr_at(p, e + 1);
      if (r1 > r0) {
        __syncwarp();  // og written by the whole warp
        const long long slot = k % p.seis_cap;
        for (int t = lane; t < 2 * (r1 - r0); t += 32) {
          const int rid = rcv_id_at(p, r0 + t / 2), c = t & 1;
          const double* ph = p.rcv_phi + size_t(rid) * NP;
          double v = 0.0;
          for (int i = 0; i < NP; ++i) v += ph[i] * og[c * NP + i];
          p.seis[(size_t(slot) * p.nrcv + rid) * 2 + c] = v;
        }
      }
    }
    __syncwarp();
  }
  if (p.mode == kModePower && p.mesh_of == nullptr) {
    const double v0 = warp_sum(en), v1 = warp_sum(pw1), v2 = warp_sum(pw2);
    if (lane == 0) {
      atomicAdd(p.acc + 0, v0);
      atomicAdd(p.acc + 1, v1);
      atomicAdd(p.acc + 2, v2);
    }
  } else if (p.energy != nullptr && (p.mode == kModeStep || p.mode == kModeFirst)) {
    const double v = warp_sum(en);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double sum = 0.0;
      for (int w = 0; w < CF::WARPS; ++w) sum += red[w];
      atomicAdd(p.energy + (k % p.energy_cap), sum);
    }
  }
}

__global__ void k_advance(long long* step, long long n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *step += n;
}

// ---------------------------------------------------------------------------
// Operator assembly on the device from the factorised reference tables.
//
// For block b of row e and column c (entries r = m*Np+i, c' = n*Np+j):
//   diagonal (c == e):
//     |detJ| sum_ab alpha^{mn}_ab K^{ab}_ij                                   (A)
//     + sum_faces [ pen*N^2 c_mn(face) Ws_l[i][j]                            (S)
//                   - L/2 sum_a (beta^{mn}_a Ds^a_l[i][j] + beta^{nm}_a Ds^a_l[j][i]) ]   (I + I^T)
//   off-diagonal (c = neighbour across face l of e, l' its face):
//     - pen*N^2 c_mn Wx_{ll'}[i][j]
//     + L/2 sum_a beta^{mn}_a(e,l) Dx^a_{ll'}[i][j] + L'/2 sum_a beta^{nm}_a(c,l') Dx^a_{l'l}[j][i]
// with
//   alpha^{mn}_ab = sum_kl C^{mn}_kl invJ[a][k] invJ[b][l]   (Hooke tensor of
//     CTensorProduct/mat_dot, TimeAdvance.cpp:60-66, in stress_loc,
//     Matrices_imp.hpp:73-94);
//   beta^{mn}_a = sum_p tau^{mn}_p invJ[a][p], tau = traction of
//     sigma(phi e_m) on n, row n (interelement, Matrices_imp.hpp:95-141);
//   c_00 = (l+2m)n0^2 + 2m n1^2, c_11 = (l+2m)n1^2 + 2m n0^2, c_01 = c_10 = l n0 n1
//     with harmonic means (stability, Matrices_imp.hpp:142-182;
//     Parameters::avg_p, Parameters.cpp:37-45). The reference's factor
//     h_scaled * ds = (1/L)(L w_k) is applied as w_k.
// ---------------------------------------------------------------------------
struct AssembleParams {
  int ne, N, Np;
  double pen_n2;             // penalty * N * N
  const int* row_ptr;
  const int* col;
  const signed char* bface;  // face of the row element for each block, -1 diagonal
  const int* neigh;          // [ne][3]
  const int* nedge;          // [ne][3]
  const double* invJ;        // [ne][4] (00,10,01,11)
  const double* detJ;        // [ne]
  const double* elen;        // [ne][3]
  const double* enrm;        // [ne][3][2]
  const double* lam;         // [ne]
  const double* mu;          // [ne]
  const double* K;           // [4][Np][Np]
  const double* Ws;          // [3][Np][Np]
  const double* Wx;          // [9][Np][Np]
  const double* Ds;          // [6][Np][Np]
  const double* Dx;          // [18][Np][Np]
  int prec;                  // 0 fp64, 1 fp32, 2 bf16+scale
  int pitch;                 // column pitch of a stored block (>= 2Np; padding pre-zeroed)
  void* out;                 // blocks, column-major per block
  float* scale;              // [nnzb] (bf16)
};


// beta^{mn}_a for element e, face l: out[(m*2+n)*2 + a]
__device__ __forceinline__ void face_beta(const AssembleParams& p, int e, int l, double* beta) {
  const double lam = p.lam[e], mu = p.mu[e];
  const double n0 = p.enrm[6 * size_t(e) + 2 * l], n1 = p.enrm[6 * size_t(e) + 2 * l + 1];
  const double* iJ = p.invJ + 4 * size_t(e);  // iJ[a + 2*k] = invJ(a, k)
  double tau[4][2];
  tau[0][0] = (lam + 2 * mu) * n0; tau[0][1] = mu * n1;   // (0,0)
  tau[1][0] = lam * n1;            tau[1][1] = mu * n0;   // (0,1)
  tau[2][0] = mu * n1;             tau[2][1] = lam * n0;  // (1,0)
  tau[3][0] = mu * n0;             tau[3][1] = (lam + 2 * mu) * n1;  // (1,1)
  for (int mn = 0; mn < 4; ++mn)
    for (int a = 0; a < 2; ++a) beta[mn * 2 + a] = tau[mn][0] * iJ[a] + tau[mn][1] * iJ[a + 2];
}

__device__ __forceinline__ double block_entry(const AssembleParams& p, int e, int c, int face, int r, int cc,
                                              const double* alpha, const double* betas /*[3][8]*/,
                                              const double* cmn /*[3][4]*/, const double* betan /*[8]*/) {
  const int Np = p.Np;
  const size_t P2 = size_t(Np) * Np;
  const int m = r / Np, i = r - m * Np, n = cc / Np, j = cc - n * Np;
  const int mn = m * 2 + n, nm = n * 2 + m;
  double v = 0.0;
  if (face < 0) {
    const double adet = fabs(p.detJ[e]);
    double a = 0.0;
    for (int ab = 0; ab < 4; ++ab) a += alpha[mn * 4 + ab] * p.K[ab * P2 + size_t(i) * Np + j];
    v = adet * a;
    for (int l = 0; l < 3; ++l) {
      if (p.neigh[3 * size_t(e) + l] < 0) continue;
      const double L = p.elen[3 * size_t(e) + l];
      v += p.pen_n2 * cmn[l * 4 + mn] * p.Ws[l * P2 + size_t(i) * Np + j];
      double t = 0.0;
      for (int a = 0; a < 2; ++a) {
        const double* D = p.Ds + (a * 3 + l) * P2;
        t += betas[l * 8 + mn * 2 + a] * D[size_t(i) * Np + j] + betas[l * 8 + nm * 2 + a] * D[size_t(j) * Np + i];
      }
      v -= 0.5 * L * t;
    }
  } else {
    const int l = face, lp = p.nedge[3 * size_t(e) + l];
    const double L = p.elen[3 * size_t(e) + l], Lp = p.elen[3 * size_t(c) + lp];
    v = -p.pen_n2 * cmn[l * 4 + mn] * p.Wx[(l * 3 + lp) * P2 + size_t(i) * Np + j];
    double t1 = 0.0, t2 = 0.0;
    for (int a = 0; a < 2; ++a) {
      t1 += betas[l * 8 + mn * 2 + a] * p.Dx[((a * 3 + l) * 3 + lp) * P2 + size_t(i) * Np + j];
      t2 += betan[nm * 2 + a] * p.Dx[((a * 3 + lp) * 3 + l) * P2 + size_t(j) * Np + i];
    }
    v += 0.5 * L * t1 + 0.5 * Lp * t2;
  }
  return v;
}

// One CTA per element row: the row's set-up (the elastic tensor in the
// element's frame, the face terms of its three faces and of the neighbours'
// matching faces) is shared by the row's blocks and computed by seven
// threads at once; then the row's blocks are written entry by entry.
__global__ void __launch_bounds__(256) k_assemble(const AssembleParams p) {
  const int e = blockIdx.x;
  __shared__ double alpha[16], betas[24], cmn[12], betan[4][8];
  __shared__ float s_max[8];
  const int rb = p.row_ptr[e], nb = min(4, p.row_ptr[e + 1] - rb);
  const int t = threadIdx.x;
  if (t == 0) {
    const double lam = p.lam[e], mu = p.mu[e];
    const double* iJ = p.invJ + 4 * size_t(e);
    // C^{mn}_{kl} (k,l index physical derivatives), row-major [mn][k*2+l].
    double C[4][4] = {{lam + 2 * mu, 0, 0, mu}, {0, lam, mu, 0}, {0, mu, lam, 0}, {mu, 0, 0, lam + 2 * mu}};
    for (int mn = 0; mn < 4; ++mn)
      for (int a = 0; a < 2; ++a)
        for (int bb = 0; bb < 2; ++bb) {
          double sum = 0.0;
          for (int kk = 0; kk < 2; ++kk)
            for (int ll = 0; ll < 2; ++ll) sum += C[mn][kk * 2 + ll] * iJ[a + 2 * kk] * iJ[bb + 2 * ll];
          alpha[mn * 4 + a * 2 + bb] = sum;
        }
  } else if (t <= 3) {
    const int l = t - 1;
    const int nbr = p.neigh[3 * size_t(e) + l];
    if (nbr < 0) {
      for (int q = 0; q < 8; ++q) betas[l * 8 + q] = 0.0;
      for (int q = 0; q < 4; ++q) cmn[l * 4 + q] = 0.0;
    } else {
      face_beta(p, e, l, betas + l * 8);
      const double al = harm(p.lam[e], p.lam[nbr]), am = harm(p.mu[e], p.mu[nbr]);
      const double n0 = p.enrm[6 * size_t(e) + 2 * l], n1 = p.enrm[6 * size_t(e) + 2 * l + 1];
      cmn[l * 4 + 0] = (al + 2 * am) * n0 * n0 + 2 * am * n1 * n1;
      cmn[l * 4 + 3] = (al + 2 * am) * n1 * n1 + 2 * am * n0 * n0;
      cmn[l * 4 + 1] = al * n0 * n1;
      cmn[l * 4 + 2] = al * n0 * n1;
    }
  } else if (t <= 7 && t - 4 < nb) {
    const int q = t - 4, face = p.bface[rb + q];
    if (face >= 0) face_beta(p, col_at(p, rb + q), p.nedge[3 * size_t(e) + face], betan[q]);
  }
  __syncthreads();
  const int R = 2 * p.Np;
  const int RR = R * R;
  for (int q = 0; q < nb; ++q) {
    const int b = rb + q, c = col_at(p, b), face = p.bface[b];
    float inv_sc = 1.0f;
    if (p.prec == 2) {
      float amax = 0.0f;
      for (int i = t; i < RR; i += blockDim.x) {
        const int cc = i / R, r = i - cc * R;
        amax = fmaxf(amax, float(fabs(block_entry(p, e, c, face, r, cc, alpha, betas, cmn, betan[q]))));
      }
      for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
      if ((t & 31) == 0) s_max[t >> 5] = amax;
      __syncthreads();
      if (t == 0) {
        float m = 0.0f;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) m = fmaxf(m, s_max[w]);
        // Power-of-two scale: values land in [-1, 1] and scaling is exact.
        const float sc = (m > 0.0f) ? exp2f(ceilf(log2f(m))) : 1.0f;
        s_max[0] = sc;
        p.scale[b] = sc;
      }
      __syncthreads();
      inv_sc = 1.0f / s_max[0];
      __syncthreads();  // s_max is reused by the next block
    }
    for (int i = t; i < RR; i += blockDim.x) {
      const int cc = i / R, r = i - cc * R;  // column-major storage: (r, cc) at cc*pitch + r
      const double v = block_entry(p, e, c, face, r, cc, alpha, betas, cmn, betan[q]);
      const size_t o = size_t(b) * R * p.pitch + size_t(cc) * p.pitch + r;
      if (p.prec == 0) reinterpret_cast<double*>(p.out)[o] = v;
      else if (p.prec == 1) reinterpret_cast<float*>(p.out)[o] = float(v);
      else reinterpret_cast<__nv_bfloat16*>(p.out)[o] = __float2bfloat16_rn(float(v) * inv_sc);
    }
  }
}

// Applies A (Np x Np, row-major) to every Np-segment of the rows (side 0:
// B <- diag(A, A) B) or of the columns (side 1: B <- B diag(A, A)^T) of each
// 2Np x 2Np block, in FP64, and stores the result in the storage type.
// With A = L^-1, L the Cholesky factor of the reference mass of a
// non-orthonormal basis, the two sides give L^-1 B L^-T, the operator in the
// orthonormalised coordinates w = L^T u, where the per-element mass is again
// rho_e detJ_e times the identity. in: FP64 blocks, column-major with column
// pitch pin. Working in place (in == out, FP64, pout == pin) is allowed: each
// chunk of columns (side 0) or rows (side 1) is read completely into shared
// memory before any of it is written.
constexpr int kFoldMaxNp = 45;  // Np of N = 8
constexpr int kFoldVecs = 16;
__global__ void __launch_bounds__(256) k_fold_basis(const double* in, int pin, int Np, const double* __restrict__ A,
                                                    int side, int prec, int pout, void* out, float* scale) {
  __shared__ double sA[kFoldMaxNp * kFoldMaxNp];
  __shared__ double sv[2 * kFoldMaxNp * kFoldVecs];
  __shared__ float s_max[8];
  const int b = blockIdx.x, R = 2 * Np;
  for (int t = threadIdx.x; t < Np * Np; t += blockDim.x) sA[t] = A[t];
  const double* blk = in + size_t(b) * R * pin;
  float amax = 0.0f, inv_sc = 1.0f;
  for (int pass = (prec == 2 ? 0 : 1); pass < 2; ++pass) {
    for (int v0 = 0; v0 < R; v0 += kFoldVecs) {
      const int nv = min(kFoldVecs, R - v0);
      __syncthreads();
      // sv[vv][k]: entry k of vector v0 + vv (a column for side 0, a row for
      // side 1); consecutive threads read consecutive addresses.
      for (int t = threadIdx.x; t < nv * R; t += blockDim.x) {
        if (side == 0) {
          const int vv = t / R, k = t - vv * R;
          sv[vv * R + k] = blk[size_t(v0 + vv) * pin + k];
        } else {
          const int k = t / nv, vv = t - k * nv;
          sv[vv * R + k] = blk[size_t(k) * pin + v0 + vv];
        }
      }
      __syncthreads();
      for (int t = threadIdx.x; t < nv * R; t += blockDim.x) {
        const int vv = t / R, k = t - vv * R;
        const int comp = k >= Np ? 1 : 0, i = k - comp * Np;
        const double* vec = sv + vv * R + comp * Np;
        double v = 0.0;
        for (int j = 0; j < Np; ++j) v = fma(sA[i * Np + j], vec[j], v);
        if (pass == 0) {
          amax = fmaxf(amax, float(fabs(v)));
        } else {
          const int row = side == 0 ? k : v0 + vv, col = side == 0 ? v0 + vv : k;
          const size_t o = size_t(b) * R * pout + size_t(col) * pout + row;
          if (prec == 0) reinterpret_cast<double*>(out)[o] = v;
          else if (prec == 1) reinterpret_cast<float*>(out)[o] = float(v);
          else reinterpret_cast<__nv_bfloat16*>(out)[o] = __float2bfloat16_rn(float(v) * inv_sc);
        }
      }
    }
    if (pass == 0) {
      for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
      if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = amax;
      __syncthreads();
      if (threadIdx.x == 0) {
        float m = 0.0f;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) m = fmaxf(m, s_max[w]);
        const float scv = (m > 0.0f) ? exp2f(ceilf(log2f(m))) : 1.0f;  // as k_assemble
        s_max[0] = scv;
        scale[b] = scv;
      }
      __syncthreads();
      inv_sc = 1.0f / s_max[0];
    }
  }
}

// The expansion of one shot's state at npt reference points of every
// element: out[(e*npt + q)*2 + c] = sum_j T[q][j] u[(e*S + shot)*2Np + c*Np + j]
// (T = basis values at the points, in the device's coordinates).
__global__ void k_eval_points(const double* __restrict__ u, int ne, int S, int Np, int shot,
                              const double* __restrict__ T, int npt, double* __restrict__ out) {
  const long long n = 2ll * ne * npt;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const long long e = o / (2 * npt);
    const int q = int((o / 2) % npt), c = int(o & 1);
    const double* w = u + (e * S + shot) * 2 * Np + c * Np;
    const double* t = T + size_t(q) * Np;
    double v = 0.0;
    for (int j = 0; j < Np; ++j) v = fma(t[j], w[j], v);
    out[o] = v;
  }
}

// Per-element terms of FESpace::L2error (FESpace_imp.hpp:107-133):
// out[e] = detJ_e * sum_q w_q ((u_h,x(x_q) - ex_q,x)^2 + (u_h,y(x_q) - ex_q,y)^2),
// points in order; the host adds the terms in element order.
__global__ void k_l2_local(const double* __restrict__ u, int ne, int S, int Np, int shot,
                           const double* __restrict__ T, const double* __restrict__ wq, int nq,
                           const double* __restrict__ detJ, const double* __restrict__ exact,
                           double* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    const double* ux = u + ((long long)e * S + shot) * 2 * Np;
    const double* uy = ux + Np;
    const double* ex = exact + (long long)e * nq * 2;
    double loc = 0.0;
    for (int q = 0; q < nq; ++q) {
      const double* t = T + size_t(q) * Np;
      double ax = 0.0, ay = 0.0;
      for (int j = 0; j < Np; ++j) {
        ax = fma(t[j], ux[j], ax);
        ay = fma(t[j], uy[j], ay);
      }
      const double dx = ax - ex[2 * q], dy = ay - ex[2 * q + 1];
      loc += (dx * dx + dy * dy) * wq[q];
    }
    out[e] = loc * detJ[e];
  }
}

// FESpace::transform (FESpace_imp.hpp:136-179) on the device, written into
// one shot's slot of a state buffer: for element e, component c and mode i,
// u[(e*S + shot)*2Np + c*Np + i] = 1/detJ_e * sum_q T[q][i] f[e][q][c] |detJ_e| w_q,
// with T the basis at the volume points in the device's coordinates
// (L^-1 phi for a non-orthonormal basis, where w = L^T u = L^-1 rhs / detJ).
// vals == nullptr writes zeros.
__global__ void k_project_points(double* __restrict__ u, int ne, int S, int Np, int shot,
                                 const double* __restrict__ T, const double* __restrict__ wq, int nq,
                                 const double* __restrict__ detJ, const double* __restrict__ vals) {
  const long long n = 2ll * ne * Np;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const long long e = o / (2 * Np);
    const int r = int(o - e * 2 * Np), c = r >= Np ? 1 : 0, i = r - c * Np;
    double v = 0.0;
    if (vals) {
      const double dJ = detJ[e], adJ = fabs(dJ);
      const double* f = vals + e * nq * 2 + c;
      double rhs = 0.0;
      for (int q = 0; q < nq; ++q) rhs = fma(f[2 * q] * adJ * wq[q], T[size_t(q) * Np + i], rhs);
      v = 1. / dJ * rhs;
    }
    u[(e * S + shot) * 2 * Np + r] = v;
  }
}

}  // namespace tsp
