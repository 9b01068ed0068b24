// Batched FP64 step on the FP64 tensor cores, warp-specialised and
// persistent (internal header of tspeed_b200).
//
// The same product as k_step_batched64d -- per work item (element row e,
// tile of ST shots) Y[shot][r] = sum_b sum_k X_{col b}[shot][k] B_b[r][k]
// with mma.sync m8n8k4 .f64 (exact FP64 products, FP64 accumulation) -- but
// the operands stream through shared-memory rings (NSG stages per consumer
// group) filled by producer lanes with bulk copies (cp.async.bulk, completion
// on mbarriers, no multicast), so the consumer warps never wait on their own
// copies and the next item's blocks arrive while the current item's epilogue
// runs.
//
// Roles: NG groups of NCW consumer warps (WM x WN warps, each MTW m-tiles
// of 8 shots x NTW n-tiles of 8 operator rows; accumulators in registers;
// they also run the leap-frog epilogue, receivers and energy); the groups
// take the CTA's items in turn, so one group's epilogue overlaps the other's
// products. The last warp produces: its lane g fills group g's ring.
// The epilogue reads u^k from the diagonal block's state stage (the
// element's own tile, already in shared memory) and u^{k-1} through loads
// issued before the item's products, so it waits on no global load.
// Per block the producer issues two bulk copies: the operator block as it is
// stored (column-major, pitch KP = R padded to 4, padding rows zero) and the
// state tile of the neighbour (ST shot rows of R doubles, contiguous in the
// state layout). Many small copies would be limited by the copy engine's
// request rate; two large ones are not. The K padding of the operator
// (columns R..KP-1) is zeroed once and never written, so the state's K
// padding (the next shot row's first entries, or zeroed slack) multiplies
// zeros; outputs of padded rows and of shots beyond S are discarded. The
// stages are zeroed once so that no entry ever read is uninitialised.
//
// Every wait is bounded (about a second); on a timeout the CTA raises an
// abort flag in shared memory, every role stops waiting, the consumer warps
// keep their named barriers balanced, the producer waits (bounded) for its
// copies in flight, and err_flag tells the host that the results are void.
#pragma once

#include <stdint.h>

#include "tsp_kernels.cuh"
#include "tsp_tcfx.cuh"
#include "tsp_tcgen05.cuh"

namespace tsp {

template <int R, int NSG_, int NG_, int WM_ = 4, int WN_ = 2>
struct D64WCfg {
  static constexpr int KP = (R + 3) & ~3;  // also the stored block pitch of batched handles
  static constexpr int NTL = (R + 7) / 8;
  static constexpr int ST = R <= 42 ? 64 : 32;
  static constexpr int WM = WM_, WN = WN_, NCW = WM * WN, NG = NG_;
  static constexpr int MTW = ST / (8 * WM);
  static constexpr int NTW = (NTL + WN - 1) / WN;
  static constexpr int NT = (NG * NCW + 1) * 32;
  // Each consumer group has a ring of its own (NSG stages), filled by its own
  // producer lane in the group's block order. A consumer waits on its ring
  // index j with the parity of use j / NSG: index j - NSG of the same ring is
  // the group's own block, consumed (hence landed) before, and use j + NSG
  // cannot be issued before this group releases j, so the barrier has
  // completed either j / NSG or j / NSG + 1 uses and the parity names the
  // right one -- whatever the row lengths and the ring length. (A ring shared
  // by the groups does not have this property: a group's index j - NST may
  // belong to another group's copy that is still in flight, and bulk copies
  // complete in any order.)
  static constexpr int NSG = NSG_;
  static constexpr int NST = NG * NSG;     // stages in total
  static_assert(NSG_ >= 1 && NG_ >= 1, "ring");
  static constexpr int BSZ = KP * KP;      // doubles: operator stage [k][n], pitch KP
  static constexpr int XSZ = ST * R + 4;   // doubles: state stage [shot][k], pitch R, zero slack
  static constexpr int STAGE = BSZ + XSZ;
  static_assert(BSZ % 2 == 0 && STAGE % 2 == 0, "16-byte aligned stages");
  static constexpr size_t smem_bytes() {
    return size_t(NST) * STAGE * sizeof(double) + size_t(2 * NST) * sizeof(uint64_t) + 16;
  }
};

// Stages per group ring that fit in shared memory (at most CAP).
template <int R, int NG, int WM, int WN, int CAP>
constexpr int d64w_fit_nsg() {
  constexpr size_t one = D64WCfg<R, 1, NG, WM, WN>::smem_bytes();
  constexpr size_t budget = 227 * 1024;
  return int(budget / one) >= CAP ? CAP : int(budget / one);
}

// The decoupled epilogue (EPI = 2): each consumer group hands its FP64 row
// sums to an update set of NU warps through a Y tile in shared memory
// ([shot][2Np + 1], odd pitch) and goes on with its next item, so the DMMA
// warps never wait on global memory; the update set runs the leap-frog
// update with coalesced loads and stores of the contiguous state tile, the
// sources, the energy terms and the receivers.
template <int R, int NSG, int NG, int WM, int WN, int NU>
struct D64WUpd {
  typedef D64WCfg<R, NSG, NG, WM, WN> CF;
  static constexpr int YP = R + 1;
  static constexpr int YSZ = CF::ST * YP;  // doubles of one group's Y tile
  static constexpr int NT = CF::NT + NG * NU * 32;
  static constexpr size_t smem_bytes() {
    return CF::smem_bytes() + (NU > 0 ? size_t(NG) * YSZ * sizeof(double) + size_t(2 * NG) * sizeof(uint64_t) : 0);
  }
};

// Stages per group ring that fit beside the Y tiles (at most CAP).
template <int R, int NG, int WM, int WN, int NU, int CAP>
constexpr int d64w_fit_nsg_upd() {
  constexpr size_t one = D64WUpd<R, 1, NG, WM, WN, NU>::smem_bytes();
  constexpr size_t stage = size_t(NG) * (D64WCfg<R, 1, NG, WM, WN>::STAGE * sizeof(double) + 2 * sizeof(uint64_t));
  constexpr size_t budget = 227 * 1024;
  return int((budget - one) / stage) + 1 >= CAP ? CAP : int((budget - one) / stage) + 1;
}

// Threads of the kernel: with a register split (RA > 0) the producer warp is
// padded to a whole warpgroup, so that every warpgroup is all consumers or
// the producer's.
template <int R, int NSG, int NG, int WM, int WN, int NU, int RA>
constexpr int d64w_nt() {
  constexpr int nt = D64WUpd<R, NSG, NG, WM, WN, NU>::NT;
  return RA > 0 ? ((nt / 32 + 3) / 4) * 128 : nt;
}
// Registers per thread of the producer warpgroup under a register split.
constexpr int kD64ProducerRegs = 24;

// EPI selects where the epilogue gets u^k and u^{k-1}: 0 global loads issued
// by the epilogue (fewest registers: the two consumer groups hide the
// latency behind each other's products); 1 u^k from the diagonal block's
// state stage and u^{k-1} requested before the products (no load latency in
// the epilogue; 24 more registers per thread at 2Np = 42 with all rows per
// warp, so it suits warp tiles of half the rows and a single group); 2 the
// decoupled epilogue of NU update warps per group (D64WUpd); 3 u^{k-1} requested
// before the products as in 1 and u^k loaded by the epilogue (an L2 hit: the
// diagonal block's state copy brought the element's tile there), half the
// extra registers of 1.
// RA > 0: register split -- the consumer warpgroups raise their registers to
// RA per thread (setmaxnreg), the producer warpgroup lowers its own to
// kD64ProducerRegs; the launch must hold at least NCONS * 32 * RA +
// (threads - NCONS * 32) * kD64ProducerRegs registers (the host checks the
// compiled register count before launching), so that the raise never waits.
// It gives EPI = 1 (latency-free epilogue) room with two consumer groups.
template <int R, int NSG, int NG, int MINB = 1, int WM = 4, int WN = 2, int EPI = 0, int NU = 0, int RA = 0>
__global__ void __launch_bounds__(d64w_nt<R, NSG, NG, WM, WN, NU, RA>(), MINB)
    k_step_batched64w(const StepParams p, int* err_flag) {
  typedef D64WCfg<R, NSG, NG, WM, WN> CF;
  typedef D64WUpd<R, NSG, NG, WM, WN, NU> UF;
  static_assert((EPI == 2) == (NU > 0), "update warps exist exactly for the decoupled epilogue");
  constexpr int NP = R / 2, KP = CF::KP, ST = CF::ST, NTL = CF::NTL, MTW = CF::MTW, NTW = CF::NTW;
  constexpr int NST = CF::NST, YP = UF::YP, NTT = d64w_nt<R, NSG, NG, WM, WN, NU, RA>();
  constexpr int NCONS = NG * CF::NCW;    // DMMA warps
  constexpr int PW = NCONS + NG * NU;    // the producer warp
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* stages = reinterpret_cast<double*>(smem_raw);
  double* ytiles = stages + size_t(NST) * CF::STAGE;                                    // [NG][ST][YP] (EPI = 2)
  uint64_t* bfull = reinterpret_cast<uint64_t*>(ytiles + (NU > 0 ? size_t(NG) * UF::YSZ : 0));  // [NG][NSG]
  uint64_t* bempty = bfull + NST;                                                       // [NG][NSG] stage consumed
  uint64_t* yfull = bempty + NST;                                                       // [NG] Y tile written (EPI = 2)
  uint64_t* yempty = yfull + (NU > 0 ? NG : 0);                                         // [NG] Y tile consumed
  volatile int* abort_s = reinterpret_cast<volatile int*>(yempty + (NU > 0 ? NG : 0));

  if (*reinterpret_cast<volatile int*>(err_flag) != 0) return;  // an earlier launch of the run timed out
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  if (t == 0) {
    *abort_s = 0;
    for (int i = 0; i < NST; ++i) {
      fx_mbar_init(smem_u32(&bfull[i]), 1);
      fx_mbar_init(smem_u32(&bempty[i]), CF::NCW);
    }
    for (int i = 0; i < (NU > 0 ? NG : 0); ++i) {
      fx_mbar_init(smem_u32(&yfull[i]), CF::NCW);
      fx_mbar_init(smem_u32(&yempty[i]), NU > 0 ? NU : 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = t; i < NST * CF::STAGE + (NU > 0 ? NG * UF::YSZ : 0); i += NTT) stages[i] = 0.0;
  __syncthreads();

  const int S = p.S;
  const int ntile = (S + ST - 1) / ST;
  const long long nitems = (long long)p.ne * ntile;
  const long long G = gridDim.x;
  const double* blocks = reinterpret_cast<const double*>(p.blocks);
  if constexpr (RA > 0) {
    static_assert(NU == 0 && NCONS % 4 == 0 && RA % 8 == 0 && RA <= 256, "register split: consumer warpgroups");
    if (warp < NCONS) asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(RA));
    else asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kD64ProducerRegs));
  }

  if (warp == PW) {
    // ---------------- producers: lane g fills ring g ----------------
    if (lane < NG) {
      const int g = lane;
      uint64_t* gfull = bfull + g * NSG;
      uint64_t* gempty = bempty + g * NSG;
      double* gst = stages + size_t(g) * NSG * CF::STAGE;
      uint32_t j = 0;
      bool ok = true;
      for (long long item = blockIdx.x + g * G; item < nitems && ok; item += NG * G) {
        const int e = int(item / ntile), tile = int(item % ntile);
        const int s0 = tile * ST, nsh = min(ST, S - s0);
        int rb, nb;
        row_span(p, e, rb, nb);
        const uint32_t bbytes = uint32_t(R) * KP * 8, xbytes = uint32_t(nsh) * R * 8;
        for (int b = 0; b < nb; ++b) {
          const int s = int(j % NSG);
          const uint32_t n = j / NSG;
          if (n > 0 && !fx_wait(smem_u32(&gempty[s]), (n - 1) & 1, abort_s)) {
            ok = false;
            break;
          }
          const int c = col_at(p, rb + b);
          const uint32_t bar = smem_u32(&gfull[s]);
          const uint32_t dB = smem_u32(gst + size_t(s) * CF::STAGE), dX = dB + CF::BSZ * 8;
          fx_mbar_arrive_tx(bar, bbytes + xbytes);
          fx_bulk_g2s(dB, blocks + size_t(rb + b) * R * KP, bbytes, bar);
          fx_bulk_g2s(dX, p.x + (size_t(c) * S + s0) * R, xbytes, bar);
          ++j;
        }
      }
      // Every issued copy lands before the CTA ends (bounded; copies
      // complete). At most one use of a stage is in flight: use u is issued
      // only after use u - 1 was consumed.
      const long long t0 = clock64();
      for (int s = 0; s < NSG; ++s) {
        if (j <= uint32_t(s)) continue;
        const uint32_t uses = (j - 1 - s) / NSG + 1;
        while (!mbar_try(smem_u32(&gfull[s]), (uses - 1) & 1) && clock64() - t0 < (1ll << 31)) {
        }
      }
      if (clock64() - t0 >= (1ll << 31)) *abort_s = 1;
    }
  } else if (warp < NCONS) {
    // ---------------- consumers ----------------
    const int grp = warp / CF::NCW, wl = warp % CF::NCW, tl = t - grp * CF::NCW * 32;
    const int wm = wl % CF::WM, wn = wl / CF::WM;
    const int g = lane >> 2, tg = lane & 3;
    // Fragment row g holds shot 8 mt + gs: rows 0..3 take the even shots and
    // 4..7 the odd ones: with the state's shot pitch of R doubles, rows two
    // shots apart are 4R words apart (168 = 8 mod 32 for 2Np = 42), so each
    // half-warp's A loads fall in distinct banks.
    const int gs = ((g & 3) << 1) | (g >> 2);
    const int nt0 = wn * NTW, ntn = min(NTW, NTL - nt0);
    const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
    const double dt = p.dt;
    uint64_t* gfull = bfull + grp * NSG;
    uint64_t* gempty = bempty + grp * NSG;
    const double* gst = stages + size_t(grp) * NSG * CF::STAGE;
    double en = 0.0;
    double chk = 0.0;  // NaN once a non-finite u^{k+1} was written (inf * 0 and NaN * 0 are NaN)
    uint32_t j = 0;  // index into this group's ring
    uint32_t m = 0;  // uses of this group's Y tile (EPI = 2)
    bool dead = false;
    long long it = 0;
    for (long long item = blockIdx.x; item < nitems; item += G, ++it) {
      if (int(it % NG) != grp) continue;  // another group's item (its own ring)
      const int e = int(item / ntile), tile = int(item % ntile);
      const int s0 = tile * ST;
      int rb, nb;
      row_span(p, e, rb, nb);
      // The epilogue's scalar inputs, requested now so that they arrive during
      // the products: the element's inverse-mass factor and, per m-tile,
      // whether the shot's source lies in this element.
      const double mi_e = p.minv[e];
      int src_e[MTW];
#pragma unroll
      for (int mt = 0; mt < MTW; ++mt) {
        const int sh = s0 + (wm * MTW + mt) * 8 + gs;
        src_e[mt] = (sh < S) ? src_elem_at(p, sh) : -1;
      }
      // u^{k-1} of this warp's outputs, requested now and used by the
      // epilogue: the loads overlap the products. u^k comes from the
      // diagonal block's state stage (the element's own tile) when the row
      // starts with its diagonal block, else from global memory.
      double2 upv[MTW][NTW], uk[MTW][NTW];
#pragma unroll
      for (int mt = 0; mt < MTW; ++mt) {
        if constexpr (EPI == 0) break;
        const int sh = s0 + (wm * MTW + mt) * 8 + gs;
        const size_t me = (size_t(e) * S + (sh < S ? sh : 0)) * R;
#pragma unroll
        for (int q = 0; q < NTW; ++q) {
          const int r0 = (nt0 + q) * 8 + 2 * tg;
          const bool valid = sh < S && q < ntn && r0 < R;
          upv[mt][q] = (valid && p.uprev) ? *reinterpret_cast<const double2*>(p.uprev + me + r0) : make_double2(0.0, 0.0);
          uk[mt][q] = make_double2(0.0, 0.0);
        }
      }
      const bool diag_first = EPI == 1 && col_at(p, rb) == e;
      double acc[MTW][NTW][2];
#pragma unroll
      for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
        for (int q = 0; q < NTW; ++q) acc[mt][q][0] = acc[mt][q][1] = 0.0;
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
        const double* B = gst + size_t(s) * CF::STAGE;
        const double* X = B + CF::BSZ + (wm * MTW * 8 + gs) * R + tg;
        const double* Bt = B + tg * KP + nt0 * 8 + g;
#pragma unroll
        for (int k0 = 0; k0 < KP; k0 += 4) {
          double a[MTW], bb[NTW];
#pragma unroll
          for (int mt = 0; mt < MTW; ++mt) a[mt] = X[mt * 8 * R + k0];
#pragma unroll
          for (int q = 0; q < NTW; ++q) bb[q] = (NTL % CF::WN == 0 || q < ntn) ? Bt[k0 * KP + q * 8] : 0.0;
#pragma unroll
          for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
            for (int q = 0; q < NTW; ++q)
              if (NTL % CF::WN == 0 || q < ntn) dmma_m8n8k4(acc[mt][q][0], acc[mt][q][1], a[mt], bb[q]);
        }
        if (b == 0 && diag_first) {
          const double* Xs = B + CF::BSZ;
#pragma unroll
          for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
            for (int q = 0; q < NTW; ++q) {
              const int r0 = (nt0 + q) * 8 + 2 * tg;
              if (q < ntn && r0 < R)
                uk[mt][q] = *reinterpret_cast<const double2*>(Xs + ((wm * MTW + mt) * 8 + gs) * R + r0);
            }
        }
        __syncwarp();
        if (lane == 0) fx_mbar_arrive(smem_u32(&gempty[s]));
      }
      if constexpr (EPI == 2) {
        // ---- hand the row sums to the group's update set ----
        if (!dead && m > 0) {
          const bool okw = fx_wait(smem_u32(&yempty[grp]), (m - 1) & 1, abort_s);
          if (__any_sync(0xffffffffu, !okw)) dead = true;
        }
        ++m;
        if (dead) continue;
        double* Y = ytiles + size_t(grp) * UF::YSZ;
#pragma unroll
        for (int mt = 0; mt < MTW; ++mt) {
          const int sl = (wm * MTW + mt) * 8 + gs;
#pragma unroll
          for (int q = 0; q < NTW; ++q) {
            const int r0 = (nt0 + q) * 8 + 2 * tg;
            if (q < ntn && r0 < R) {
              Y[sl * YP + r0] = acc[mt][q][0];
              Y[sl * YP + r0 + 1] = acc[mt][q][1];
            }
          }
        }
        __syncwarp();
        if (lane == 0) fx_mbar_arrive(smem_u32(&yfull[grp]));
        continue;
      }
      // ---- epilogue (leap-frog, source, energy terms) ----
      if (!dead) {
        const double mi = mi_e;
#pragma unroll
        for (int mt = 0; mt < MTW; ++mt) {
          const int sh = s0 + (wm * MTW + mt) * 8 + gs;
          if (sh >= S) continue;
          const size_t me = (size_t(e) * S + sh) * R;
          const bool is_src = (src_e[mt] == e) && (k < p.nF);
          double Fk[2] = {0.0, 0.0};
          if (is_src) {
            Fk[0] = p.F[(size_t(sh) * p.nF + k) * 2];
            Fk[1] = p.F[(size_t(sh) * p.nF + k) * 2 + 1];
          }
#pragma unroll
          for (int q = 0; q < NTW; ++q) {
            const int r0 = (nt0 + q) * 8 + 2 * tg;
            if (q >= ntn || r0 >= R) continue;  // rows come in pairs (R is even)
            const double2 uu = diag_first ? uk[mt][q] : __ldg(reinterpret_cast<const double2*>(p.x + me + r0));
            const double2 up =
                EPI != 0 ? upv[mt][q]
                         : (p.uprev ? *reinterpret_cast<const double2*>(p.uprev + me + r0) : make_double2(0.0, 0.0));
            const double u[2] = {uu.x, uu.y}, upr[2] = {up.x, up.y};
            double un[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int r = r0 + h;
              const int cmp = r / NP, ii = r - cmp * NP;
              const double f = is_src ? Fk[cmp] * p.src_phi[size_t(sh) * NP + ii] : 0.0;
              const double y = acc[mt][q][h];
              if (p.mode == kModeStep) un[h] = (2 * u[h] - upr[h]) + mi * ((-dt * dt) * (y - f));
              else un[h] = (u[h] + dt * upr[h]) - mi * (dt * dt / 2 * (y - f));  // kModeFirst, uprev = v0
              if (p.energy != nullptr) {
                const double d = un[h] - u[h];
                en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un[h] * y;
              }
            }
            *reinterpret_cast<double2*>(p.out + me + r0) = make_double2(un[0], un[1]);
            chk = __fma_rn(un[0], 0.0, __fma_rn(un[1], 0.0, chk));
          }
        }
      }
      // ---- receivers (the condition is the same for every consumer warp) ----
      if (p.rcv_ptr != nullptr) {
        const int q0 = rcv_ptr_at(p, e), q1 = rcv_ptr_at(p, e + 1);
        if (q1 > q0) {
          // u^{k+1} of this item is visible to the whole group (barrier 1 + grp).
          asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "n"(CF::NCW * 32) : "memory");
          if (!dead) {
            const long long slot = k % p.seis_cap;
            const int nwork = (q1 - q0) * ST * 2;
            for (int wk = tl; wk < nwork; wk += CF::NCW * 32) {
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
      }
    }
    if (chk != chk && p.nonfinite != nullptr) *p.nonfinite = 1;
    if (p.energy != nullptr) {
      const double v = warp_sum(en);
      if (lane == 0 && v != 0.0) atomicAdd(p.energy + (k % p.energy_cap), v);
    }
  } else {
    if constexpr (EPI == 2) {
      // ---------------- update sets: FP64 epilogue of the group's items ----------------
      constexpr int NUT = (NU > 0 ? NU : 1) * 32;
      const int ug = (warp - NCONS) / (NU > 0 ? NU : 1);
      const int ut = t - (NCONS + ug * NU) * 32;  // thread within the set
      const long long k = (p.step_base ? *p.step_base : 0) + p.rel;
      const double dt = p.dt;
      const double* Y = ytiles + size_t(ug) * UF::YSZ;
      constexpr int BATCH = 6;  // row pairs per thread and load batch
      double en = 0.0;
      double chk = 0.0;
      uint32_t m = 0;
      bool dead = false;
      long long it = 0;
      for (long long item = blockIdx.x; item < nitems; item += G, ++it) {
        if (int(it % NG) != ug) continue;
        const int e = int(item / ntile), tile = int(item % ntile);
        const int s0 = tile * ST, nsv = min(ST, S - s0);
        const size_t base = (size_t(e) * S + s0) * R;  // the tile: nsv * R contiguous doubles
        if (!dead) {
          const bool okw = fx_wait(smem_u32(&yfull[ug]), m & 1, abort_s);
          if (!__all_sync(0xffffffffu, okw)) dead = true;
        }
        ++m;
        if (!dead) {
          const double mi = p.minv[e];
          const int npair = nsv * NP;
          for (int pb = 0; pb < npair; pb += NUT * BATCH) {
            // Row pair q = pb + NUT b + ut is entry 2q of the tile: shot
            // q / NP, rows 2 (q % NP) and +1. Both levels' loads first.
            double2 uu[BATCH], up[BATCH];
#pragma unroll
            for (int b = 0; b < BATCH; ++b) {
              const int q = pb + NUT * b + ut;
              const bool v = q < npair;
              uu[b] = v ? __ldg(reinterpret_cast<const double2*>(p.x + base) + q) : make_double2(0.0, 0.0);
              up[b] = (v && p.uprev) ? *(reinterpret_cast<const double2*>(p.uprev + base) + q) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int b = 0; b < BATCH; ++b) {
              const int q = pb + NUT * b + ut;
              if (q >= npair) continue;
              const int sl = q / NP, r0 = 2 * (q - sl * NP);
              const int sh = s0 + sl;
              const bool is_src = (src_elem_at(p, sh) == e) && (k < p.nF);
              const double u[2] = {uu[b].x, uu[b].y}, upr[2] = {up[b].x, up[b].y};
              double un[2];
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const int r = r0 + h;
                const int cmp = r / NP, ii = r - cmp * NP;
                const double f =
                    is_src ? p.F[(size_t(sh) * p.nF + k) * 2 + cmp] * p.src_phi[size_t(sh) * NP + ii] : 0.0;
                const double y = Y[sl * YP + r];
                if (p.mode == kModeStep) un[h] = (2 * u[h] - upr[h]) + mi * ((-dt * dt) * (y - f));
                else un[h] = (u[h] + dt * upr[h]) - mi * (dt * dt / 2 * (y - f));  // kModeFirst, uprev = v0
                if (p.energy != nullptr) {
                  const double d = un[h] - u[h];
                  en += 0.5 * (d * d) / (mi * dt * dt) + 0.5 * un[h] * y;
                }
              }
              *(reinterpret_cast<double2*>(p.out + base) + q) = make_double2(un[0], un[1]);
              chk = __fma_rn(un[0], 0.0, __fma_rn(un[1], 0.0, chk));
            }
          }
        }
        // u^{k+1} of the item is complete once the set passes this barrier
        // (id 1 + group).
        asm volatile("bar.sync %0, %1;" ::"r"(1 + ug), "n"(NUT) : "memory");
        if (!dead) {
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
      if (chk != chk && p.nonfinite != nullptr) *p.nonfinite = 1;
      if (p.energy != nullptr) {
        const double v = warp_sum(en);
        if (lane == 0 && v != 0.0) atomicAdd(p.energy + (k % p.energy_cap), v);
      }
    }
  }
  __syncthreads();
  if (t == 0 && *abort_s) atomicExch(err_flag, 1);
}

// Self-test of the bounded mbarrier wait that every warp-specialised kernel
// here relies on: one thread waits on a phase that nothing completes. The
// wait must give up after its limit (about a second), raise the abort flag
// and let the kernel end normally, leaving the context usable.
__global__ void k_selftest_bounded_wait(int* out) {
  __shared__ uint64_t bar;
  __shared__ int abort_s;
  if (threadIdx.x == 0) {
    abort_s = 0;
    fx_mbar_init(smem_u32(&bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const long long t0 = clock64();
    const bool ok = fx_wait(smem_u32(&bar), 0, &abort_s);
    out[0] = ok ? 1 : 0;
    out[1] = abort_s;
    out[2] = int((clock64() - t0) >> 20);  // waited cycles / 2^20
  }
}

}  // namespace tsp
