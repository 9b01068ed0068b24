// C-ABI of the tspeed_b200 engine (include/tspeed_b200.h).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <tuple>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/tspeed_b200.h"
#include "tsp_host.h"
#include "tsp_kernels.cuh"
#include "tsp_tcgen05.cuh"
#include "tsp_tcfx.cuh"
#include "tsp_dmma.cuh"
#include "tsp_simt32.cuh"

namespace {

thread_local std::string g_create_error = "no error";

}  // namespace

struct tsp_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  int ne = 0, N = 0, Np = 0, R = 0, S = 1, nrcv = 0;
  long long nnzb = 0;
  int prec = TSP_PREC_FP64, op_kind = TSP_OP_EXPLICIT;
  int bpitch = 0;  // column pitch of stored blocks: 2Np (one shot) or 2Np rounded up to 4 (batched)
  // Non-orthonormal basis (BoundaryAdapted): M_ref = L L^T (Cholesky). The
  // device works in the orthonormalised coordinates w = L^T u of every
  // element and component: blocks L^-1 B L^-T, source and receiver values
  // L^-1 phi, per-element mass rho detJ I as for Dubiner, so every kernel
  // (the energy monitor included) runs unchanged. Host vectors stay in the
  // reference's coefficients u; the maps are applied at the boundary.
  // Empty for the orthonormal Dubiner basis. [Np][Np] row-major.
  int basis = tsp::kDubiner;
  std::vector<double> minv_ref, lref, lref_inv;
  double* d_lref_inv = nullptr;
  // Signed element determinants (handles built from a mesh; empty for
  // tsp_create_from_blocks), for tsp_l2_error.
  std::vector<double> detJ;
  // operator
  int* d_row_ptr = nullptr;
  int* d_col = nullptr;
  void* d_blocks = nullptr;
  float* d_bscale = nullptr;
  double* d_minv = nullptr;
  // matrix-free operator: packed reference tables and per-element data
  tsp::MatFreeParams mf = {};
  // multi-mesh group (set by tsp_batch_create; null for ordinary handles)
  double* d_dt_elem = nullptr;
  int* d_src_of = nullptr;
  int* d_mesh_of = nullptr;
  double* d_xscale_mesh = nullptr;
  int nmesh = 0;
  // state
  double* d_U[2] = {nullptr, nullptr};
  int cur = 0;  // d_U[cur] holds u^k, d_U[1-cur] holds u^{k-1}
  double* d_v0 = nullptr;
  float* d_X32[2] = {nullptr, nullptr};  // FP32 transposed shadows of d_U (batched FP32 kernel)
  bool shadow = false;
  // FP32 batched step variant: 0 K split over warp groups (2Np <= 42) or the
  // pipelined single group (2Np = 56); 1 pipelined single group; 2 the
  // non-persistent cp.async kernel; 4 the tensor-core fixed-point kernel.
  // -1 until the autotuner has chosen; TSP_BATCHED_VARIANT forces one.
  int kernel_variant = -1;
  // Tensor-core fixed-point step (variant 4): operator slice images and row
  // scales, built once; state slice images and shot scales, one pair per
  // state level like the FP32 shadow.
  bool fx = false;
  unsigned char* d_Bsl = nullptr;
  int* d_Bex = nullptr;
  unsigned char* d_Xsl[2] = {nullptr, nullptr};
  int* d_Xex[2] = {nullptr, nullptr};
  // [0] set by a kernel whose bounded wait gave up; [1] set by a step kernel
  // that wrote a NaN or infinite displacement (cleared by new initial values
  // or a resumed state).
  int* d_err = nullptr;
  int num_sms = 148;
  long long* d_step = nullptr;
  // sources / receivers
  int* d_src_elem = nullptr;
  double* d_src_phi = nullptr;
  double* d_F = nullptr;
  long long nF = 0;
  int* d_rcv_ptr = nullptr;
  int* d_rcv_id = nullptr;
  double* d_rcv_phi = nullptr;
  double* d_seis = nullptr;
  long long seis_cap = 0;
  double* d_energy = nullptr;
  long long energy_cap = 0;
  bool energy_on = false;
  double* d_acc = nullptr;
  // host mirrors
  std::vector<int> src_elem, rcv_elem;
  std::vector<double> src_phi, rcv_phi, Fhost;
  double dt = 0.0;
  bool dt_set = false;
  long long steps_done = 0;
  double last_time = 0.0;
  std::string err = "no error";
  std::map<std::pair<long long, int>, cudaGraphExec_t> graphs;  // (steps, parity) -> tsp_run piece
  std::vector<void*> owned;  // device allocations, freed at destroy
};

namespace {

// NVTX range over a scope: set-up, uploads, the step loop and read-backs show
// up by name in a profiler's timeline (header-only NVTX; a no-op without a
// tool attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

int fail(tsp_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  else g_create_error = msg;
  return code;
}

#define TSP_CUDA(h, call)                                                                          \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail((h), e_ == cudaErrorMemoryAllocation ? TSP_ERR_NOMEM : TSP_ERR_CUDA,             \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                             \
  } while (0)

// Device memory of every handle comes from one stream-ordered pool per
// device that keeps freed memory for the process (release threshold
// unlimited): a program that creates and destroys simulations one after the
// other (shot batches, parameter sweeps) pays cudaMalloc/cudaFree of the
// multi-GB operator and state buffers once, not per simulation.
// tsp_release_cached_memory returns the cached memory to the driver.
constexpr int kMaxDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[kMaxDevices] = {};

cudaError_t device_pool(int dev, cudaMemPool_t* out) {
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mutex);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = ~uint64_t(0);
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return e;
    }
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return cudaSuccess;
}

// Allocation on the handle's stream, completed before returning so that the
// memory may be used from any stream or by synchronous copies.
cudaError_t pool_alloc(tsp_handle* h, void** p, size_t bytes) {
  cudaMemPool_t pool = nullptr;
  cudaError_t e = device_pool(h->device, &pool);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes, pool, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return e;
}

template <typename T>
int dalloc(tsp_handle* h, T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  void* q = nullptr;
  cudaError_t e = pool_alloc(h, &q, n * sizeof(T));
  if (e != cudaSuccess)
    return fail(h, TSP_ERR_NOMEM, std::string("device allocation of ") + std::to_string(n * sizeof(T)) + " bytes: " +
                                      cudaGetErrorString(e));
  *p = static_cast<T*>(q);
  h->owned.push_back(q);
  return TSP_OK;
}

// A copy ordered on the handle's stream and complete on return. Plain
// cudaMemcpy runs on the legacy default stream, which does not order against
// the handles' non-blocking streams, and from pageable host memory it may
// return before the data has reached the device.
cudaError_t copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

// Stream-ordered release: work already queued on the handle's stream that
// reads p completes first.
void dfree(tsp_handle* h, void* p) {
  if (!p) return;
  auto it = std::find(h->owned.begin(), h->owned.end(), p);
  if (it != h->owned.end()) h->owned.erase(it);
  cudaFreeAsync(p, h->stream);
}

template <typename T>
int upload(tsp_handle* h, T** d, const T* src, size_t n) {
  int rc = dalloc(h, d, n);
  if (rc) return rc;
  if (n) TSP_CUDA(h, cudaMemcpyAsync(*d, src, n * sizeof(T), cudaMemcpyHostToDevice, h->stream));
  return TSP_OK;
}

// v <- A v (trans = false) or A^T v (trans = true) for nvec consecutive
// Np-vectors, A [Np][Np] row-major.
void map_vectors(const std::vector<double>& A, bool trans, int Np, double* v, long long nvec) {
  double t[tsp::kFoldMaxNp];
  for (long long r = 0; r < nvec; ++r) {
    double* x = v + size_t(r) * Np;
    for (int i = 0; i < Np; ++i) {
      double a = 0.0;
      for (int j = 0; j < Np; ++j) a += (trans ? A[size_t(j) * Np + i] : A[size_t(i) * Np + j]) * x[j];
      t[i] = a;
    }
    std::memcpy(x, t, Np * sizeof(double));
  }
}
// Reference coefficients u -> device coordinates w = L^T u, and back
// u = L^-T w, for nvec Np-vectors in place. No-ops for Dubiner.
void to_dev_coords(const tsp_handle* h, double* v, long long nvec) {
  if (!h->lref.empty()) map_vectors(h->lref, true, h->Np, v, nvec);
}
void to_ref_coords(const tsp_handle* h, double* v, long long nvec) {
  if (!h->lref_inv.empty()) map_vectors(h->lref_inv, true, h->Np, v, nvec);
}

// Longest graph tsp_run captures (steps); longer runs replay it.
constexpr long long kRunChunk = 256;

void clear_graphs(tsp_handle* h) {
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
}

// Receivers sorted by element into a CSR over elements.
int build_receiver_csr(tsp_handle* h) {
  if (h->nrcv == 0) return TSP_OK;
  std::vector<int> ptr(size_t(h->ne) + 1, 0), ids(h->nrcv);
  for (int r = 0; r < h->nrcv; ++r) ptr[h->rcv_elem[r] + 1]++;
  for (int e = 0; e < h->ne; ++e) ptr[e + 1] += ptr[e];
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int r = 0; r < h->nrcv; ++r) ids[fill[h->rcv_elem[r]]++] = r;
  int rc;
  if ((rc = upload(h, &h->d_rcv_ptr, ptr.data(), ptr.size()))) return rc;
  if ((rc = upload(h, &h->d_rcv_id, ids.data(), ids.size()))) return rc;
  std::vector<double> rphi(h->rcv_phi);
  if (!h->lref_inv.empty()) map_vectors(h->lref_inv, false, h->Np, rphi.data(), h->nrcv);
  if ((rc = upload(h, &h->d_rcv_phi, rphi.data(), rphi.size()))) return rc;
  return TSP_OK;
}

int alloc_seis(tsp_handle* h, long long cap) {
  dfree(h, h->d_seis);
  h->d_seis = nullptr;
  h->seis_cap = cap;
  if (h->nrcv == 0) return TSP_OK;
  int rc = dalloc(h, &h->d_seis, size_t(h->S) * size_t(cap) * h->nrcv * 2);
  if (rc) return rc;
  TSP_CUDA(h, cudaMemsetAsync(h->d_seis, 0, size_t(h->S) * size_t(cap) * h->nrcv * 2 * sizeof(double), h->stream));
  clear_graphs(h);
  return TSP_OK;
}

template <int R>
using FxDefault = tsp::FxCfg<R>;

// State slices of level i from its FP64 values (padding stays zero).
template <int R>
int fx_refresh_R(tsp_handle* h, int i) {
  tsp::k_make_xslices<R><<<1184, 128, 0, h->stream>>>(h->d_U[i], h->ne, h->S, h->d_Xsl[i], h->d_Xex[i]);
  TSP_CUDA(h, cudaGetLastError());
  return TSP_OK;
}

// Operator slice images from the stored FP32 blocks, state slice buffers.
template <int R>
int fx_setup_R(tsp_handle* h) {
  typedef FxDefault<R> CF;
  int rc;
  const size_t bbytes = size_t(h->nnzb) * CF::BBYTES;
  if ((rc = dalloc(h, &h->d_Bsl, bbytes)) || (rc = dalloc(h, &h->d_Bex, size_t(h->nnzb) * CF::GW))) return rc;
  TSP_CUDA(h, cudaMemsetAsync(h->d_Bsl, 0, bbytes, h->stream));
  tsp::k_make_bslices<float, R><<<1184, 128, 0, h->stream>>>(
      reinterpret_cast<const float*>(h->d_blocks), h->bpitch, h->nnzb, h->d_Bsl, h->d_Bex);
  TSP_CUDA(h, cudaGetLastError());
  const size_t ntile = size_t((h->S + 63) / 64);
  const size_t xbytes = size_t(h->ne) * ntile * CF::ABYTES;
  for (int i = 0; i < 2; ++i) {
    if ((rc = dalloc(h, &h->d_Xsl[i], xbytes)) || (rc = dalloc(h, &h->d_Xex[i], size_t(h->ne) * ntile * 64)))
      return rc;
    TSP_CUDA(h, cudaMemsetAsync(h->d_Xsl[i], 0, xbytes, h->stream));
    TSP_CUDA(h, cudaMemsetAsync(h->d_Xex[i], 0x80, size_t(h->ne) * ntile * 64 * sizeof(int), h->stream));
  }
  return TSP_OK;
}

int fx_dispatch(tsp_handle* h, bool setup, int i) {
  switch (h->R) {
    case 6: return setup ? fx_setup_R<6>(h) : fx_refresh_R<6>(h, i);
    case 12: return setup ? fx_setup_R<12>(h) : fx_refresh_R<12>(h, i);
    case 20: return setup ? fx_setup_R<20>(h) : fx_refresh_R<20>(h, i);
    case 30: return setup ? fx_setup_R<30>(h) : fx_refresh_R<30>(h, i);
    case 42: return setup ? fx_setup_R<42>(h) : fx_refresh_R<42>(h, i);
    case 56: return setup ? fx_setup_R<56>(h) : fx_refresh_R<56>(h, i);
    default: return fail(h, TSP_ERR_UNSUPPORTED, "no tensor-core step for 2Np = " + std::to_string(h->R));
  }
}

int launch_step(tsp_handle* h, int mode, const double* x, const double* uprev, double* out, int rel,
                double xscale, cudaStream_t st);
int check_device_error(tsp_handle* h);

// Autotuner of the batched step kernels: each applicable kernel variant
// (tile shape, shots per CTA, ring depth, CUDA cores or tensor cores) runs a
// few steps on the zero initial state of the handle -- no sources are set
// yet, so every output stays zero and nothing needs restoring -- timed with
// CUDA events on the handle's stream, twice per candidate; the fastest is
// kept. FP32 operator
// (with its FP32 state shadow): 7 and 8 warp-specialised with bulk-copy rings
// and 8 shots x several rows per lane (6 or 8 FMA warps per SM), 0 K
// split over warp groups, 1 pipelined
// single group, 2 non-persistent, 4 tensor-core fixed point. FP64 operator: 5 and 6
// warp-specialised DMMA (two consumer groups of 8 warps, or one group of 16
// warps with a latency-free epilogue), 3 single-role DMMA, 2 CUDA cores. TSP_BATCHED_VARIANT skips
// the trials. Choices are kept per process for handles of the same shape
// (device, precision, 2Np, shots, elements): a second handle of the same
// problem skips the trials.
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int, int, int>, int> g_tune_cache;

// The autotuner's earlier choice for a handle of this shape, or -1.
int tune_cached(const tsp_handle* h) {
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  auto it = g_tune_cache.find(std::make_tuple(h->device, h->prec, h->R, h->S, h->ne));
  return it == g_tune_cache.end() ? -1 : it->second;
}

int autotune(tsp_handle* h) {
  NvtxRange nvtx_("autotune");
  const bool fx_ok = h->fx;
  const bool fp64_batched = h->S > 1 && h->prec == TSP_PREC_FP64 && h->op_kind == TSP_OP_EXPLICIT;
  if (fp64_batched) {
    if (h->kernel_variant >= 0) {
      const int v = h->kernel_variant;
      if (v != 2 && v != 3 && v != 6 && v != 9 && v != 10 && v != 13) h->kernel_variant = 5;
      return TSP_OK;
    }
  } else if (h->kernel_variant >= 0 || !h->shadow) {
    if (h->kernel_variant < 0) h->kernel_variant = 0;
    return TSP_OK;
  }
  const auto key = std::make_tuple(h->device, h->prec, h->R, h->S, h->ne);
  int cached = -1;
  {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) cached = it->second;
  }
  std::vector<int> cands;
  if (fp64_batched) cands = {5, 13, 9, 10, 6, 3, 2};
  else if (h->R <= 42) cands = {7, 8, 0, 1, 2};
  else if (h->R <= 56) cands = {7, 8, 0, 2};
  else cands = {2};
  if (fx_ok) cands.push_back(4);
  if (cached >= 0 && (cached != 4 || fx_ok)) cands = {cached};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  TSP_CUDA(h, cudaEventCreate(&e0));
  TSP_CUDA(h, cudaEventCreate(&e1));
  // Two rounds over the candidates, each candidate's faster round counts:
  // a single short trial let run-to-run noise pick between near-equal
  // variants.
  std::vector<float> best(cands.size(), 0.0f);
  int bestv = cands[0], rc = TSP_OK;
  for (int round = 0; round < 2 && cands.size() > 1 && !rc; ++round)
    for (size_t ci = 0; ci < cands.size(); ++ci) {
      const int v = cands[ci];
      h->kernel_variant = v;
      h->fx = (v == 4);
      for (int w = 0; w < 2 && !rc; ++w) rc = launch_step(h, tsp::kModeStep, h->d_U[1], h->d_U[0], h->d_U[0], 0, 1.0, h->stream);
      if (!rc) rc = cudaEventRecord(e0, h->stream) == cudaSuccess ? TSP_OK : TSP_ERR_CUDA;
      for (int w = 0; w < 5 && !rc; ++w) rc = launch_step(h, tsp::kModeStep, h->d_U[1], h->d_U[0], h->d_U[0], 0, 1.0, h->stream);
      if (!rc) rc = cudaEventRecord(e1, h->stream) == cudaSuccess ? TSP_OK : TSP_ERR_CUDA;
      float ms = 0.0f;
      if (!rc) rc = (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
                        ? TSP_OK
                        : TSP_ERR_CUDA;
      if (rc) break;
      if (round == 0 || ms < best[ci]) best[ci] = ms;
    }
  if (!rc && cands.size() > 1) {
    size_t bi = 0;
    for (size_t ci = 1; ci < cands.size(); ++ci)
      if (best[ci] < best[bi]) bi = ci;
    bestv = cands[bi];
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc == TSP_ERR_CUDA ? fail(h, TSP_ERR_CUDA, "autotuner launch failed") : rc;
  if ((rc = check_device_error(h))) return rc;
  h->kernel_variant = bestv;
  h->fx = (bestv == 4);
  {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tune_cache[key] = bestv;
  }
  if (fx_ok && !h->fx) {
    dfree(h, h->d_Bsl);
    dfree(h, h->d_Bex);
    h->d_Bsl = nullptr;
    h->d_Bex = nullptr;
    for (int i = 0; i < 2; ++i) {
      dfree(h, h->d_Xsl[i]);
      dfree(h, h->d_Xex[i]);
      h->d_Xsl[i] = nullptr;
      h->d_Xex[i] = nullptr;
    }
  }
  return TSP_OK;
}

// Common tail of both constructors: state, step counter, sources, receivers.
// Sets up a non-orthonormal basis from its reference mass M_ref.
int set_basis_mass(tsp_handle* h, int basis, const std::vector<double>& mass, const std::vector<double>& minv) {
  h->basis = basis;
  h->minv_ref = minv;
  if (!tsp::cholesky(h->Np, mass, &h->lref, &h->lref_inv))
    return fail(h, TSP_ERR_ARG, "reference mass is not symmetric positive definite");
  return upload(h, &h->d_lref_inv, h->lref_inv.data(), h->lref_inv.size());
}

// Turns FP64 blocks B on the device (column-major, pitch pin; overwritten)
// into L^-1 B L^-T in the handle's storage type at h->d_blocks.
int fold_blocks(tsp_handle* h, double* d_in, int pin) {
  tsp::k_fold_basis<<<unsigned(h->nnzb), 256, 0, h->stream>>>(d_in, pin, h->Np, h->d_lref_inv, 0, TSP_PREC_FP64, pin,
                                                             d_in, nullptr);
  tsp::k_fold_basis<<<unsigned(h->nnzb), 256, 0, h->stream>>>(d_in, pin, h->Np, h->d_lref_inv, 1, h->prec, h->bpitch,
                                                             h->d_blocks, h->d_bscale);
  cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
  if (ce != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("basis fold: ") + cudaGetErrorString(ce));
  return TSP_OK;
}

int finish_create(tsp_handle* h) {
  int rc;
  const size_t nstate = size_t(h->ne) * h->S * h->R;
  for (int i = 0; i < 2; ++i) {
    if ((rc = dalloc(h, &h->d_U[i], nstate))) return rc;
    TSP_CUDA(h, cudaMemsetAsync(h->d_U[i], 0, nstate * sizeof(double), h->stream));
  }
  // The FP32 batched kernel (FP32 blocks, several shots, 2Np <= 72) keeps an
  // FP32 transposed shadow of each state level.
  h->shadow = (h->S > 1 && h->prec == TSP_PREC_FP32 && h->R <= 72);
  if (h->shadow) {
    const int ntile = (h->S + 63) / 64;
    const size_t nsh = size_t(h->ne) * ntile * h->R * 64;
    for (int i = 0; i < 2; ++i) {
      if ((rc = dalloc(h, &h->d_X32[i], nsh))) return rc;
      TSP_CUDA(h, cudaMemsetAsync(h->d_X32[i], 0, nsh * sizeof(float), h->stream));
    }
  }
  // The tensor-core kernel's slice buffers exist when it is forced or is a
  // candidate of the autotuner.
  // (Not when the autotuner already chose another kernel for this shape.)
  const bool fx_ok = h->shadow && h->op_kind == TSP_OP_EXPLICIT && h->R <= 56;
  const int cached = h->kernel_variant < 0 ? tune_cached(h) : -1;
  h->fx = fx_ok && (h->kernel_variant == 4 || (h->kernel_variant < 0 && (cached < 0 || cached == 4)));
  if (h->fx && (rc = fx_dispatch(h, true, 0))) return rc;
  if ((rc = dalloc(h, &h->d_step, 1))) return rc;
  TSP_CUDA(h, cudaMemsetAsync(h->d_step, 0, sizeof(long long), h->stream));
  if ((rc = dalloc(h, &h->d_err, 2))) return rc;
  TSP_CUDA(h, cudaMemsetAsync(h->d_err, 0, 2 * sizeof(int), h->stream));
  if ((rc = dalloc(h, &h->d_acc, 3))) return rc;
  if ((rc = upload(h, &h->d_src_elem, h->src_elem.data(), h->src_elem.size()))) return rc;
  {
    // Device coordinates: the force vector L^-1 f and the receiver functional
    // u -> phi^T u = (L^-1 phi)^T w both take L^-1 phi.
    std::vector<double> sphi(h->src_phi);
    if (!h->lref_inv.empty()) map_vectors(h->lref_inv, false, h->Np, sphi.data(), h->S);
    if ((rc = upload(h, &h->d_src_phi, sphi.data(), sphi.size()))) return rc;
  }
  if ((rc = build_receiver_csr(h))) return rc;
  long long cap = 4096;
  if (h->nrcv > 0) {
    const long long per = (long long)h->S * h->nrcv * 16;
    cap = std::max<long long>(1, std::min<long long>(4096, (256ll << 20) / per));
  }
  if ((rc = alloc_seis(h, cap))) return rc;
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  return autotune(h);
}

template <int R, typename BT>
int launch_batched(tsp_handle* h, const tsp::StepParams& p, dim3 grid, cudaStream_t st) {
  typedef tsp::BatchCfg<R> CF;
  typedef typename tsp::AccOf<BT>::type AT;
  const size_t smem = CF::template smem_bytes<AT>();
  static unsigned long long configured = 0;  // per instantiation, one bit per device
  const unsigned long long bit = 1ull << (h->device & 63);
  if (!(configured & bit)) {
    cudaError_t e = cudaFuncSetAttribute(tsp::k_step_batched<R, BT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(smem));
    if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("batched kernel smem: ") + cudaGetErrorString(e));
    configured |= bit;
  }
  tsp::k_step_batched<R, BT><<<grid, CF::NT, smem, st>>>(p);
  return TSP_OK;
}

template <int R>
int launch_d64(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  typedef tsp::D64Cfg<R> CF;
  const size_t smem = CF::smem_bytes();
  static unsigned long long configured = 0;  // one bit per device
  const unsigned long long bit = 1ull << (h->device & 63);
  if (!(configured & bit)) {
    cudaError_t e = cudaFuncSetAttribute(tsp::k_step_batched64d<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(smem));
    if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("FP64 batched kernel smem: ") + cudaGetErrorString(e));
    configured |= bit;
  }
  const dim3 grid(unsigned(h->ne), unsigned((h->S + CF::ST - 1) / CF::ST));
  tsp::k_step_batched64d<R><<<grid, CF::NT, smem, st>>>(p);
  return TSP_OK;
}

// FP64 warp-specialised DMMA step, two configurations (autotuner
// candidates): V = 5, two consumer groups of 8 warps alternating items (one
// group's epilogue, with its global loads, overlaps the other's products),
// each warp one m-tile of 8 shots x every operator row, a ring of its own per
// group (2Np <= 56; one group for 2Np = 72 and 90, whose stages fit fewer
// times); V = 6, one group of 16 warps, each 8 shots x half the rows, whose
// epilogue reads u^k from shared memory and u^{k-1} from loads requested
// before the products, so it has no latency to hide.
template <int R, int V>
int launch_d64w(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  constexpr bool two = V == 5 || V == 13;
  constexpr int NG = (two && R <= 56) ? 2 : 1;
  constexpr int ST = tsp::D64WCfg<R, 1, NG>::ST;
  constexpr int NCW = two ? 8 : 16;
  constexpr int WM = ST / 8, WN = NCW / WM;
  constexpr int EPI = (V == 5) ? 0 : (V == 13) ? 3 : 1;
  // V = 13: variant 5's tiles, u^{k-1} requested before the products and u^k
  // loaded by the epilogue (EPI = 3); the 24 registers that takes come from a
  // warpgroup register split (two consumer groups only; else as 5).
  constexpr int RA = (V == 13 && NG == 2) ? 112 : 0;
  constexpr int NSG = tsp::d64w_fit_nsg<R, NG, WM, WN, (NG == 1 ? 6 : 4)>();
  static_assert(NSG >= 2, "FP64 DMMA ring: two stages per group must fit");
  typedef tsp::D64WCfg<R, NSG, NG, WM, WN> CF;
  constexpr int NT = tsp::d64w_nt<R, NSG, NG, WM, WN, 0, RA>();
  const size_t smem = CF::smem_bytes();
  static unsigned long long configured = 0;  // one bit per device
  static unsigned long long split_ok = 0;    // one bit per device: the register split fits the launch
  const unsigned long long bit = 1ull << (h->device & 63);
  if (!(configured & bit)) {
    auto kern = tsp::k_step_batched64w<R, NSG, NG, 1, WM, WN, EPI, 0, RA>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("FP64 batched kernel smem: ") + cudaGetErrorString(e));
    if constexpr (RA > 0) {
      // setmaxnreg.inc waits until the CTA's pool (threads x registers at
      // launch) has the registers: launch only if the split fits.
      cudaFuncAttributes fa;
      if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess)
        return fail(h, TSP_ERR_CUDA, "FP64 batched kernel attributes");
      const long long pool = (long long)fa.numRegs * NT;
      const long long need = (long long)CF::NCW * NG * 32 * RA + (long long)(NT - CF::NCW * NG * 32) * tsp::kD64ProducerRegs;
      if (pool >= need && fa.numRegs <= RA) split_ok |= bit;
    }
    configured |= bit;
  }
  if constexpr (RA > 0) {
    if (!(split_ok & bit)) return launch_d64w<R, 5>(h, p, st);  // the same product and results
  } else if constexpr (V == 13) {
    return launch_d64w<R, 5>(h, p, st);  // one consumer group: no split, variant 5's form
  }
  // Persistent: one CTA per SM.
  const long long items = (long long)h->ne * ((h->S + CF::ST - 1) / CF::ST);
  const unsigned grid = unsigned(std::min<long long>(items, h->num_sms));
  tsp::k_step_batched64w<R, NSG, NG, 1, WM, WN, EPI, 0, RA><<<grid, NT, smem, st>>>(p, h->d_err);
  return TSP_OK;
}

// FP64 warp-specialised DMMA step with the decoupled epilogue (EPI = 2):
// V = 9, two groups of 8 DMMA warps (8 shots x all rows per warp), one
// update warp and a 2-stage ring per group; V = 10, one group of 16 DMMA
// warps (8 shots x half the rows), two update warps and a 5-stage ring.
// The DMMA warps hand their FP64 row sums to the update warps through a Y
// tile in shared memory and never wait on global memory.
template <int R, int V>
int launch_d64u(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  constexpr int NG = (V == 9 && R <= 56) ? 2 : 1;
  constexpr int ST = tsp::D64WCfg<R, 1, NG>::ST;
  constexpr int NCW = (V == 9) ? 8 : 16;
  constexpr int WM = ST / 8, WN = NCW / WM;
  constexpr int NU = (V == 9) ? 1 : 2;
  constexpr int NSG = tsp::d64w_fit_nsg_upd<R, NG, WM, WN, NU, (NG == 1 ? 6 : 4)>();
  static_assert(NSG >= 2, "FP64 DMMA ring: two stages per group must fit");
  typedef tsp::D64WUpd<R, NSG, NG, WM, WN, NU> UF;
  const size_t smem = UF::smem_bytes();
  static unsigned long long configured = 0;  // one bit per device
  const unsigned long long bit = 1ull << (h->device & 63);
  if (!(configured & bit)) {
    cudaError_t e = cudaFuncSetAttribute(tsp::k_step_batched64w<R, NSG, NG, 1, WM, WN, 2, NU>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("FP64 batched kernel smem: ") + cudaGetErrorString(e));
    configured |= bit;
  }
  const long long items = (long long)h->ne * ((h->S + ST - 1) / ST);
  const unsigned grid = unsigned(std::min<long long>(items, h->num_sms));
  tsp::k_step_batched64w<R, NSG, NG, 1, WM, WN, 2, NU><<<grid, UF::NT, smem, st>>>(p, h->d_err);
  return TSP_OK;
}

template <int N>
int launch_matfree_N(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  typedef tsp::MFCfg<N> CF;
  const size_t smem = CF::smem_bytes();
  static unsigned long long configured = 0;
  const unsigned long long bit = 1ull << (h->device & 63);
  if (!(configured & bit)) {
    cudaError_t e = cudaFuncSetAttribute(tsp::k_step_matfree<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("matrix-free kernel smem: ") + cudaGetErrorString(e));
    configured |= bit;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tsp::k_step_matfree<N>, CF::WARPS * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const long long want = (h->ne + CF::WARPS - 1) / CF::WARPS;
  const unsigned grid = unsigned(std::min<long long>(want, (long long)per_sm * h->num_sms));
  tsp::k_step_matfree<N><<<grid, CF::WARPS * 32, smem, st>>>(p, h->mf);
  return TSP_OK;
}

int launch_matfree(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  switch (h->N) {
    case 1: return launch_matfree_N<1>(h, p, st);
    case 2: return launch_matfree_N<2>(h, p, st);
    case 3: return launch_matfree_N<3>(h, p, st);
    case 4: return launch_matfree_N<4>(h, p, st);
    case 5: return launch_matfree_N<5>(h, p, st);
    case 6: return launch_matfree_N<6>(h, p, st);
    case 7: return launch_matfree_N<7>(h, p, st);
    case 8: return launch_matfree_N<8>(h, p, st);
    default: return fail(h, TSP_ERR_UNSUPPORTED, "matrix-free kernel: N must be in 1..8");
  }
}

template <int R, int ST, int TR>
int launch_pipe(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  typedef tsp::PipeCfg<R, ST, TR> CF;
  const size_t smem = CF::smem_bytes();
  static unsigned long long configured = 0;
  const unsigned long long bit = 1ull << (h->device & 63);
  if (!(configured & bit)) {
    cudaError_t e = cudaFuncSetAttribute(tsp::k_step_batched32p<R, ST, TR>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("pipelined kernel smem: ") + cudaGetErrorString(e));
    configured |= bit;
  }
  const long long items = (long long)h->ne * ((h->S + ST - 1) / ST);
  const unsigned grid = unsigned(std::min<long long>(items, h->num_sms));
  tsp::k_step_batched32p<R, ST, TR><<<grid, CF::NT, smem, st>>>(p);
  return TSP_OK;
}

template <int R>
int launch_fx(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  typedef FxDefault<R> CF;
  const size_t smem = CF::smem_bytes();
  static unsigned long long configured = 0;
  const unsigned long long bit = 1ull << (h->device & 63);
  if (!(configured & bit)) {
    cudaError_t e =
        cudaFuncSetAttribute(tsp::k_step_batched_fx<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("tensor-core kernel smem: ") + cudaGetErrorString(e));
    configured |= bit;
  }
  // Persistent: one CTA per SM (its shared memory and tensor memory admit no
  // second one).
  const long long items = (long long)h->ne * ((h->S + CF::M - 1) / CF::M);
  const unsigned grid = unsigned(std::min<long long>(items, h->num_sms));
  tsp::k_step_batched_fx<R><<<grid, CF::NT, smem, st>>>(p, h->d_err);
  return TSP_OK;
}

// FP32-operator step on the CUDA cores with warp-specialised bulk-copy rings
// and packed pair FMAs: pairs of an FMA group (NWG warps per item) and an
// update set of 2 warps (the FP64 epilogue), a ring and a Y tile per pair.
// V = 7: 6 FMA warps (3 pairs at 2Np = 42), 3-stage rings, 128 registers per
// thread; V = 8: 8 FMA warps (4 pairs), 2-stage rings, 96 registers, smaller
// update load batches.
template <int R, int V>
int launch_s32w(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  constexpr int NWG = tsp::S32WCfg<R>::NWG;
  // 2Np = 56: four pairs' rings no longer fit twice; variant 8 keeps three.
  constexpr int NGR = V == 7 ? (NWG == 1 ? 4 : 3) : (NWG == 1 ? 6 : R <= 48 ? 4 : 3);
  constexpr int NU = 2, UB = V == 7 ? 6 : 3;
  constexpr int NSG = tsp::s32w_fit_nsg<R, NGR, NU>();
  static_assert(NSG >= 2, "FP32 ring: two stages per pair must fit");
  typedef tsp::S32WLayout<R, NGR, NSG, NU> LY;
  const size_t smem = LY::smem_bytes();
  static_assert(LY::smem_bytes() <= 227 * 1024, "FP32 ring kernel shared memory");
  static unsigned long long configured = 0;
  const unsigned long long bit = 1ull << (h->device & 63);
  if (!(configured & bit)) {
    cudaError_t e = cudaFuncSetAttribute(tsp::k_step_batched32w<R, NGR, NSG, NU, 1, UB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("FP32 ring kernel smem: ") + cudaGetErrorString(e));
    configured |= bit;
  }
  const long long items = (long long)h->ne * ((h->S + 63) / 64);
  const unsigned grid = unsigned(std::min<long long>(items, h->num_sms));
  tsp::k_step_batched32w<R, NGR, NSG, NU, 1, UB><<<grid, LY::NT, smem, st>>>(p, h->d_err);
  return TSP_OK;
}

template <int R>
int launch_ksplit(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  typedef tsp::KsplitCfg<R> CF;
  const size_t smem = CF::smem_bytes();
  static unsigned long long configured = 0;
  const unsigned long long bit = 1ull << (h->device & 63);
  if (!(configured & bit)) {
    cudaError_t e =
        cudaFuncSetAttribute(tsp::k_step_batched32k<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("k-split kernel smem: ") + cudaGetErrorString(e));
    configured |= bit;
  }
  const long long items = (long long)h->ne * ((h->S + CF::ST - 1) / CF::ST);
  const unsigned grid = unsigned(std::min<long long>(items, h->num_sms));
  tsp::k_step_batched32k<R><<<grid, CF::NT, smem, st>>>(p);
  return TSP_OK;
}

template <int R>
int launch_R(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  if constexpr (R <= 56) {
    if (h->fx && (p.mode == tsp::kModeStep || p.mode == tsp::kModeFirst)) return launch_fx<R>(h, p, st);
  }
  if (h->shadow && (p.mode == tsp::kModeStep || p.mode == tsp::kModeFirst) &&
      (h->kernel_variant == 7 || h->kernel_variant == 8)) {
    if constexpr (R <= 56) return h->kernel_variant == 7 ? launch_s32w<R, 7>(h, p, st) : launch_s32w<R, 8>(h, p, st);
  }
  if (h->shadow && (p.mode == tsp::kModeStep || p.mode == tsp::kModeFirst) && h->kernel_variant != 2) {
    if constexpr (R <= 42) {
      if (h->kernel_variant <= 0) return launch_ksplit<R>(h, p, st);
      return launch_pipe<R, 64, 4>(h, p, st);
    } else if constexpr (R <= 56) {
      return launch_pipe<R, 32, 2>(h, p, st);
    }
  }
  if (h->shadow && (p.mode == tsp::kModeStep || p.mode == tsp::kModeFirst)) {
    typedef tsp::Batch32Cfg<R> CF;
    const size_t smem = CF::smem_bytes();
    static unsigned long long configured = 0;
    const unsigned long long bit = 1ull << (h->device & 63);
    if (!(configured & bit)) {
      cudaError_t e = cudaFuncSetAttribute(tsp::k_step_batched32<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(smem));
      if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("batched32 kernel smem: ") + cudaGetErrorString(e));
      configured |= bit;
    }
    const dim3 grid(unsigned(h->ne), unsigned((h->S + CF::ST - 1) / CF::ST));
    tsp::k_step_batched32<R><<<grid, CF::NT, smem, st>>>(p);
    return TSP_OK;
  }
  // FP64 with several shots: the FP64 tensor-core (DMMA) kernels, chosen by
  // the autotuner or TSP_BATCHED_VARIANT: 5 and 6 the warp-specialised
  // persistent kernel (two warp tiles), 3 the single-role DMMA kernel, 2 the
  // register-staged CUDA-core kernel.
  if (h->S > 1 && h->prec == TSP_PREC_FP64 && h->kernel_variant != 2 &&
      (p.mode == tsp::kModeStep || p.mode == tsp::kModeFirst))
    return h->kernel_variant == 3    ? launch_d64<R>(h, p, st)
           : h->kernel_variant == 6  ? launch_d64w<R, 6>(h, p, st)
           : h->kernel_variant == 13 ? launch_d64w<R, 13>(h, p, st)
           : h->kernel_variant == 9  ? launch_d64u<R, 9>(h, p, st)
           : h->kernel_variant == 10 ? launch_d64u<R, 10>(h, p, st)
                                     : launch_d64w<R, 5>(h, p, st);
  if (h->S > 1 && (p.mode == tsp::kModeStep || p.mode == tsp::kModeFirst)) {
    typedef tsp::BatchCfg<R> CF;
    const dim3 grid(unsigned(h->ne), unsigned((h->S + CF::ST - 1) / CF::ST));
    switch (h->prec) {
      case TSP_PREC_FP64: return launch_batched<R, double>(h, p, grid, st);
      case TSP_PREC_FP32: return launch_batched<R, float>(h, p, grid, st);
      default: return launch_batched<R, __nv_bfloat16>(h, p, grid, st);
    }
  }
  typedef tsp::RowTeam<R, double> RT;
  const long long teams = (long long)h->ne * p.S;
  const unsigned grid = unsigned((teams + RT::TEAMS_PER_CTA - 1) / RT::TEAMS_PER_CTA);
  const bool padded = p.bpitch != R;
  switch (h->prec) {
    case TSP_PREC_FP64:
      if (padded) tsp::k_step_rows<R, double, true><<<grid, RT::THREADS, 0, st>>>(p);
      else tsp::k_step_rows<R, double, false><<<grid, RT::THREADS, 0, st>>>(p);
      break;
    case TSP_PREC_FP32:
      if (padded) tsp::k_step_rows<R, float, true><<<grid, RT::THREADS, 0, st>>>(p);
      else tsp::k_step_rows<R, float, false><<<grid, RT::THREADS, 0, st>>>(p);
      break;
    default:
      if (padded) tsp::k_step_rows<R, __nv_bfloat16, true><<<grid, RT::THREADS, 0, st>>>(p);
      else tsp::k_step_rows<R, __nv_bfloat16, false><<<grid, RT::THREADS, 0, st>>>(p);
      break;
  }
  return TSP_OK;
}

int launch_step(tsp_handle* h, int mode, const double* x, const double* uprev, double* out, int rel,
                double xscale, cudaStream_t st) {
  tsp::StepParams p;
  std::memset(&p, 0, sizeof(p));
  p.ne = h->ne;
  p.S = h->S;
  p.mode = mode;
  p.row_ptr = h->d_row_ptr;
  p.col = h->d_col;
  p.blocks = h->d_blocks;
  p.bpitch = h->bpitch;
  p.bscale = (h->prec == TSP_PREC_BF16) ? h->d_bscale : nullptr;
  p.minv = h->d_minv;
  p.x = x;
  p.uprev = uprev;
  p.out = out;
  p.dt = h->dt;
  p.xscale = xscale;
  p.step_base = h->d_step;
  p.rel = rel;
  p.src_elem = h->d_src_elem;
  p.src_phi = h->d_src_phi;
  p.F = h->d_F;
  p.nF = h->d_F ? h->nF : 0;
  const bool sample = (mode == tsp::kModeStep || mode == tsp::kModeFirst);
  p.rcv_ptr = (sample && h->nrcv > 0) ? h->d_rcv_ptr : nullptr;
  p.rcv_id = h->d_rcv_id;
  p.rcv_phi = h->d_rcv_phi;
  p.seis = h->d_seis;
  p.nrcv = h->nrcv;
  p.seis_cap = h->seis_cap;
  p.energy = (sample && h->energy_on) ? h->d_energy : nullptr;
  p.nonfinite = sample ? h->d_err + 1 : nullptr;
  p.nnzb = h->nnzb;
  p.energy_cap = h->energy_cap;
  p.acc = h->d_acc;
  p.x32_in = nullptr;
  p.x32_out = nullptr;
  if (h->shadow) {
    // The shadow pair follows the FP64 pair: x reads d_U[i] <-> d_X32[i].
    const int ix = (x == h->d_U[0]) ? 0 : 1;
    p.x32_in = h->d_X32[ix];
    p.x32_out = h->d_X32[1 - ix];
    if (h->fx) {
      p.xsl_in = h->d_Xsl[ix];
      p.xsl_out = h->d_Xsl[1 - ix];
      p.xex_in = h->d_Xex[ix];
      p.xex_out = h->d_Xex[1 - ix];
      p.bsl = h->d_Bsl;
      p.bex = h->d_Bex;
    }
  }
  if (mode == tsp::kModeApply || mode == tsp::kModePower) p.S = 1;  // single-vector products
  p.dt_elem = h->d_dt_elem;
  p.src_of = h->d_src_of;
  p.mesh_of = (mode == tsp::kModePower) ? h->d_mesh_of : nullptr;
  p.xscale_mesh = (mode == tsp::kModePower) ? h->d_xscale_mesh : nullptr;
  if (h->op_kind == TSP_OP_MATRIX_FREE) return launch_matfree(h, p, st);
  switch (h->R) {
    case 6: return launch_R<6>(h, p, st);
    case 12: return launch_R<12>(h, p, st);
    case 20: return launch_R<20>(h, p, st);
    case 30: return launch_R<30>(h, p, st);
    case 42: return launch_R<42>(h, p, st);
    case 56: return launch_R<56>(h, p, st);
    case 72: return launch_R<72>(h, p, st);
    case 90: return launch_R<90>(h, p, st);
    default: return fail(h, TSP_ERR_UNSUPPORTED, "no kernel for 2Np = " + std::to_string(h->R));
  }
}

// Rebuilds the FP32 shadow of state level i from its FP64 values.
int refresh_shadow(tsp_handle* h, int i) {
  if (!h->shadow) return TSP_OK;
  const int ntile = (h->S + 63) / 64;
  tsp::k_make_shadow<<<1184, 256, 0, h->stream>>>(h->d_U[i], h->d_X32[i], h->ne, h->S, h->R, ntile);
  TSP_CUDA(h, cudaGetLastError());
  if (h->fx) return fx_dispatch(h, false, i);
  return TSP_OK;
}

// The single-shot row kernel reads columns of exactly 2Np entries; the
// batched kernel reads four rows at a time and wants the column pitch
// rounded up to 4 (zero padded).
int block_pitch(int R, int S) { return S > 1 ? ((R + 3) & ~3) : R; }

// Launches the step kernel family with fully prepared parameters.
int launch_step_params(tsp_handle* h, const tsp::StepParams& p, cudaStream_t st) {
  if (h->op_kind == TSP_OP_MATRIX_FREE) return launch_matfree(h, p, st);
  switch (h->R) {
    case 6: return launch_R<6>(h, p, st);
    case 12: return launch_R<12>(h, p, st);
    case 20: return launch_R<20>(h, p, st);
    case 30: return launch_R<30>(h, p, st);
    case 42: return launch_R<42>(h, p, st);
    case 56: return launch_R<56>(h, p, st);
    case 72: return launch_R<72>(h, p, st);
    case 90: return launch_R<90>(h, p, st);
    default: return fail(h, TSP_ERR_UNSUPPORTED, "no kernel for 2Np = " + std::to_string(h->R));
  }
}

// Reference layout u[c*ne*Np + e*Np + i] <-> device layout [(e*S+s)*R + c*Np + i].
// The device holds w = L^T u (u itself for Dubiner).
void ref_to_dev(const tsp_handle* h, int shot, const double* src, double* dst_all) {
  const int ne = h->ne, Np = h->Np, R = h->R, S = h->S;
  for (int e = 0; e < ne; ++e) {
    double* d = dst_all + (size_t(e) * S + shot) * R;
    for (int c = 0; c < 2; ++c)
      std::memcpy(d + size_t(c) * Np, src + size_t(c) * ne * Np + size_t(e) * Np, Np * sizeof(double));
    to_dev_coords(h, d, 2);
  }
}
void dev_to_ref(const tsp_handle* h, int shot, const double* src_all, double* dst) {
  const int ne = h->ne, Np = h->Np, R = h->R, S = h->S;
  double t[2 * tsp::kFoldMaxNp];
  for (int e = 0; e < ne; ++e) {
    std::memcpy(t, src_all + (size_t(e) * S + shot) * R, R * sizeof(double));
    to_ref_coords(h, t, 2);
    for (int c = 0; c < 2; ++c) std::memcpy(dst + size_t(c) * ne * Np + size_t(e) * Np, t + c * Np, Np * sizeof(double));
  }
}


// Reports a bounded device-side wait that gave up (after a synchronisation).
int check_device_error(tsp_handle* h) {
#ifdef TSP_CHECKED
  // Checked build: the first gather index a kernel found out of range since
  // the last check (site, value); the kernels clamped it, the results are void.
  {
    unsigned long long w = 0;
    TSP_CUDA(h, cudaMemcpyFromSymbolAsync(&w, tsp::g_index_check, sizeof(w), 0, cudaMemcpyDeviceToHost, h->stream));
    TSP_CUDA(h, cudaStreamSynchronize(h->stream));
    if (w != 0) {
      const unsigned long long zero = 0;
      TSP_CUDA(h, cudaMemcpyToSymbolAsync(tsp::g_index_check, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, h->stream));
      TSP_CUDA(h, cudaStreamSynchronize(h->stream));
      static const char* const kSites[] = {"?", "row extent of element", "neighbour id", "source element",
                                           "receiver range", "receiver id", "mesh neighbour"};
      const unsigned site = unsigned(w >> 32);
      return fail(h, TSP_ERR_INDEX,
                  std::string("device index check: ") + kSites[site < 7 ? site : 0] + " out of range (value " +
                      std::to_string(int(unsigned(w & 0xffffffffu))) + "); results invalid");
    }
  }
#endif
  if (!h->d_err) return TSP_OK;
  int v = 0;
  TSP_CUDA(h, copy_sync(&v, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if (v) return fail(h, TSP_ERR_TIMEOUT, "a tensor-core step kernel timed out waiting for its MMAs; results invalid");
  return TSP_OK;
}

// Reads the non-finite flag of the step kernels (synchronises the stream).
int read_nonfinite(tsp_handle* h, int* v) {
  *v = 0;
  if (!h->d_err) return TSP_OK;
  TSP_CUDA(h, copy_sync(v, h->d_err + 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  return TSP_OK;
}
int check_nonfinite(tsp_handle* h) {
  int v = 0, rc = read_nonfinite(h, &v);
  if (rc) return rc;
  if (v)
    return fail(h, TSP_ERR_NONFINITE,
                "a step produced a NaN or infinite displacement (dt above the stability limit, or bad inputs)");
  return TSP_OK;
}
int reset_nonfinite(tsp_handle* h) {
  if (h->d_err) TSP_CUDA(h, cudaMemsetAsync(h->d_err + 1, 0, sizeof(int), h->stream));
  return TSP_OK;
}

// One shot's slice of a device state buffer (ne runs of R doubles with a
// stride of S*R) to/from a reference-layout host vector (NULL: zeros).
int get_shot(tsp_handle* h, const double* dsrc, int shot, double* out) {
  const int ne = h->ne, R = h->R;
  std::vector<double> slice(size_t(ne) * R);
  TSP_CUDA(h, cudaMemcpy2DAsync(slice.data(), size_t(R) * sizeof(double), dsrc + size_t(shot) * R,
                                size_t(h->S) * R * sizeof(double), size_t(R) * sizeof(double), ne,
                                cudaMemcpyDeviceToHost, h->stream));
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  to_ref_coords(h, slice.data(), 2ll * ne);
  for (int e = 0; e < ne; ++e)
    for (int c = 0; c < 2; ++c)
      std::memcpy(out + size_t(c) * ne * h->Np + size_t(e) * h->Np, &slice[size_t(e) * R + size_t(c) * h->Np],
                  h->Np * sizeof(double));
  return TSP_OK;
}
int put_shot(tsp_handle* h, double* ddst, int shot, const double* in) {
  const int ne = h->ne, R = h->R;
  std::vector<double> slice(size_t(ne) * R, 0.0);
  if (in)
    for (int e = 0; e < ne; ++e)
      for (int c = 0; c < 2; ++c)
        std::memcpy(&slice[size_t(e) * R + size_t(c) * h->Np], in + size_t(c) * ne * h->Np + size_t(e) * h->Np,
                    h->Np * sizeof(double));
  to_dev_coords(h, slice.data(), 2ll * ne);
  TSP_CUDA(h, cudaMemcpy2DAsync(ddst + size_t(shot) * R, size_t(h->S) * R * sizeof(double), slice.data(),
                                size_t(R) * sizeof(double), size_t(R) * sizeof(double), ne, cudaMemcpyHostToDevice,
                                h->stream));
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  return TSP_OK;
}

int begin(tsp_handle* h) {
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  return TSP_OK;
}

int make_handle(int device, tsp_handle** out) {
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(nullptr, TSP_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= ndev) return fail(nullptr, TSP_ERR_ARG, "device ordinal out of range");
  tsp_handle* h = new tsp_handle();
  h->device = device;
  if (const char* v = std::getenv("TSP_BATCHED_VARIANT")) h->kernel_variant = std::atoi(v);
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete h;
    return fail(nullptr, TSP_ERR_CUDA, std::string("stream creation: ") + cudaGetErrorString(e));
  }
  *out = h;
  return TSP_OK;
}

int create_error_from(tsp_handle* h, int rc) {
  g_create_error = h->err;
  tsp_destroy(h);
  return rc;
}

}  // namespace

extern "C" {

const char* tsp_version(void) { return "tspeed_b200 0.1 sm_100a"; }

const char* tsp_last_error(const tsp_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int tsp_create(const tsp_problem* P, tsp_handle** out) {
  NvtxRange nvtx_("tsp_create");
  if (!P || !out) return fail(nullptr, TSP_ERR_ARG, "null argument");
  *out = nullptr;
  if (P->N < 1 || P->N > tsp::kMaxN) return fail(nullptr, TSP_ERR_UNSUPPORTED, "degree N must be in 1..8");
  if (P->ne <= 0 || P->nverts <= 0 || !P->xy || !P->tri || !P->lambda || !P->mu || !P->rho)
    return fail(nullptr, TSP_ERR_ARG, "mesh or material arrays missing");
  if (P->nshots < 1 || !P->src_xy) return fail(nullptr, TSP_ERR_ARG, "need nshots >= 1 and src_xy");
  if (P->nrcv < 0 || (P->nrcv > 0 && !P->rcv_xy)) return fail(nullptr, TSP_ERR_ARG, "bad receivers");
  if (P->precision < TSP_PREC_FP64 || P->precision > TSP_PREC_BF16) return fail(nullptr, TSP_ERR_ARG, "bad precision");
  if (P->op_kind != TSP_OP_EXPLICIT && P->op_kind != TSP_OP_MATRIX_FREE)
    return fail(nullptr, TSP_ERR_ARG, "bad operator kind");
  if (P->op_kind == TSP_OP_MATRIX_FREE && (P->precision != TSP_PREC_FP64 || P->nshots != 1))
    return fail(nullptr, TSP_ERR_UNSUPPORTED, "the matrix-free operator runs FP64 with one shot per handle");
  if (P->basis != TSP_BASIS_DUBINER && P->basis != TSP_BASIS_BOUNDARY_ADAPTED)
    return fail(nullptr, TSP_ERR_ARG, "bad basis");
  if (P->basis != TSP_BASIS_DUBINER && P->op_kind == TSP_OP_MATRIX_FREE)
    return fail(nullptr, TSP_ERR_UNSUPPORTED, "the matrix-free operator is built for the orthonormal Dubiner basis");
  for (int32_t i = 0; i < 3 * P->ne; ++i)
    if (P->tri[i] < 0 || P->tri[i] >= P->nverts) return fail(nullptr, TSP_ERR_MESH, "vertex id out of range");
  for (int32_t i = 0; i < 2 * P->nverts; ++i)
    if (!std::isfinite(P->xy[i])) return fail(nullptr, TSP_ERR_MESH, "vertex coordinates must be finite");
  for (int32_t e = 0; e < P->ne; ++e)
    if (!(P->rho[e] > 0) || !(P->mu[e] >= 0) || !std::isfinite(P->lambda[e]))
      return fail(nullptr, TSP_ERR_ARG, "material values must be finite with rho > 0, mu >= 0");

  tsp_handle* h = nullptr;
  int rc = make_handle(P->device, &h);
  if (rc) return rc;
  h->ne = P->ne;
  h->N = P->N;
  h->Np = tsp::np_of(P->N);
  h->R = 2 * h->Np;
  h->S = P->nshots;
  h->nrcv = P->nrcv;
  h->prec = P->precision;
  h->op_kind = P->op_kind;
  h->basis = P->basis;

  // ---- host setup: geometry, neighbours, pattern, tables ----
  tsp::Geometry g = tsp::make_geometry(P->ne, P->xy, P->tri);
  for (int32_t e = 0; e < P->ne; ++e)
    if (!(g.detJ[e] > 0)) {
      fail(h, TSP_ERR_MESH, "element " + std::to_string(e) +
                                " is clockwise or degenerate (detJ <= 0); the signed-detJ mass of "
                                "Matrices_imp.hpp:186-189 would be non-positive");
      return create_error_from(h, TSP_ERR_MESH);
    }
  h->detJ = g.detJ;
  std::vector<int32_t> neigh(size_t(P->ne) * 3), nedge(size_t(P->ne) * 3);
  std::string err;
  if (!tsp::build_neighbours(P->ne, P->tri, neigh.data(), nedge.data(), &err)) {
    fail(h, TSP_ERR_MESH, err);
    return create_error_from(h, TSP_ERR_MESH);
  }
  std::vector<int32_t> row_ptr, col;
  std::vector<int8_t> bface;
  tsp::bsr_pattern(P->ne, neigh.data(), &row_ptr, &col, &bface);
  h->nnzb = (long long)col.size();
  tsp::RefTables T = tsp::make_tables(P->N, P->basis);
  if (P->basis != TSP_BASIS_DUBINER && (rc = set_basis_mass(h, P->basis, T.M, T.Minv))) return create_error_from(h, rc);

  // ---- sources and receivers (one point-location pass for both) ----
  {
    const int np_all = h->S + h->nrcv;
    std::vector<double> pts(2 * size_t(np_all)), phi(size_t(np_all) * h->Np);
    std::vector<int32_t> el(np_all);
    std::copy(P->src_xy, P->src_xy + 2 * size_t(h->S), pts.begin());
    if (h->nrcv) std::copy(P->rcv_xy, P->rcv_xy + 2 * size_t(h->nrcv), pts.begin() + 2 * size_t(h->S));
    tsp::locate_points(P->N, P->ne, P->xy, P->tri, g, np_all, pts.data(), el.data(), phi.data(), P->basis);
    for (int k = 0; k < np_all; ++k)
      if (el[k] < 0) {
        const bool src = k < h->S;
        fail(h, TSP_ERR_NOT_FOUND, std::string(src ? "source" : "receiver") + " point " +
                                       std::to_string(src ? k : k - h->S) + " not found in the mesh");
        return create_error_from(h, TSP_ERR_NOT_FOUND);
      }
    h->src_elem.assign(el.begin(), el.begin() + h->S);
    h->rcv_elem.assign(el.begin() + h->S, el.end());
    h->src_phi.assign(phi.begin(), phi.begin() + size_t(h->S) * h->Np);
    h->rcv_phi.assign(phi.begin() + size_t(h->S) * h->Np, phi.end());
  }

  // ---- device upload + assembly ----
  std::vector<double> minv(P->ne);
  for (int32_t e = 0; e < P->ne; ++e) minv[e] = (1. / P->rho[e]) / g.detJ[e];  // Matrices_imp.hpp:187
  int* d_neigh = nullptr;
  int* d_nedge = nullptr;
  signed char* d_bface = nullptr;
  double *d_invJ = nullptr, *d_detJ = nullptr, *d_elen = nullptr, *d_enrm = nullptr, *d_lam = nullptr,
         *d_mu = nullptr, *d_K = nullptr, *d_Ws = nullptr, *d_Wx = nullptr, *d_Ds = nullptr, *d_Dx = nullptr;
  if ((rc = upload(h, &h->d_row_ptr, row_ptr.data(), row_ptr.size())) ||
      (rc = upload(h, &h->d_col, col.data(), col.size())) || (rc = upload(h, &h->d_minv, minv.data(), minv.size())) ||
      (rc = upload(h, &d_neigh, neigh.data(), neigh.size())) ||
      (rc = upload(h, &d_nedge, nedge.data(), nedge.size())) ||
      (rc = upload(h, &d_bface, reinterpret_cast<const signed char*>(bface.data()), bface.size())) ||
      (rc = upload(h, &d_invJ, g.invJ.data(), g.invJ.size())) ||
      (rc = upload(h, &d_detJ, g.detJ.data(), g.detJ.size())) ||
      (rc = upload(h, &d_elen, g.elen.data(), g.elen.size())) ||
      (rc = upload(h, &d_enrm, g.enrm.data(), g.enrm.size())) || (rc = upload(h, &d_lam, P->lambda, size_t(P->ne))) ||
      (rc = upload(h, &d_mu, P->mu, size_t(P->ne))) || (rc = upload(h, &d_K, T.K.data(), T.K.size())) ||
      (rc = upload(h, &d_Ws, T.Ws.data(), T.Ws.size())) || (rc = upload(h, &d_Wx, T.Wx.data(), T.Wx.size())) ||
      (rc = upload(h, &d_Ds, T.Ds.data(), T.Ds.size())) || (rc = upload(h, &d_Dx, T.Dx.data(), T.Dx.size())))
    return create_error_from(h, rc);
  h->bpitch = block_pitch(h->R, h->S);
  if (h->op_kind == TSP_OP_MATRIX_FREE) {
    // Packed tables in the kernel's shared-memory layout: KT[ab][j][i],
    // TRT[l][j][r], TR[l][r][i] (r < Q: basis, Q <= r < 3Q: gradient a = r/Q-1), w1.
    const int Np = h->Np, Q = T.Q, Q3 = 3 * Q;
    const size_t P2 = size_t(Np) * Np;
    std::vector<double> pk(4 * P2 + 2 * size_t(3) * Np * Q3 + Q);
    double* KT = pk.data();
    double* TRT = KT + 4 * P2;
    double* TR = TRT + size_t(3) * Np * Q3;
    double* W1 = TR + size_t(3) * Q3 * Np;
    for (int ab = 0; ab < 4; ++ab)
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) KT[(size_t(ab) * Np + j) * Np + i] = T.K[ab * P2 + size_t(i) * Np + j];
    for (int l = 0; l < 3; ++l)
      for (int r = 0; r < Q3; ++r)
        for (int j = 0; j < Np; ++j) {
          const int kq = r % Q, part = r / Q;
          const double v = part == 0 ? T.Be[(size_t(l) * Q + kq) * Np + j]
                                     : T.Ge[((size_t(l) * 2 + (part - 1)) * Q + kq) * Np + j];
          TRT[(size_t(l) * Np + j) * Q3 + r] = v;
          TR[(size_t(l) * Q3 + r) * Np + j] = v;
        }
    for (int kq = 0; kq < Q; ++kq) W1[kq] = T.w1[kq];
    double* d_tab = nullptr;
    if ((rc = upload(h, &d_tab, pk.data(), pk.size()))) return create_error_from(h, rc);
    h->mf.tables = d_tab;
    h->mf.invJ = d_invJ;
    h->mf.detJ = d_detJ;
    h->mf.lam = d_lam;
    h->mf.mu = d_mu;
    h->mf.elen = d_elen;
    h->mf.enrm = d_enrm;
    h->mf.neigh = d_neigh;
    h->mf.nedge = d_nedge;
    h->mf.pen_n2 = P->penalty * h->N * h->N;
    for (void* q : {(void*)d_bface, (void*)d_K, (void*)d_Ws, (void*)d_Wx, (void*)d_Ds, (void*)d_Dx}) dfree(h, q);
    if ((rc = finish_create(h))) return create_error_from(h, rc);
    *out = h;
    return TSP_OK;
  }
  const size_t RRp = size_t(h->R) * h->bpitch;
  const size_t esz = h->prec == TSP_PREC_FP64 ? 8 : (h->prec == TSP_PREC_FP32 ? 4 : 2);
  {
    void* blk = nullptr;
    cudaError_t ce = pool_alloc(h, &blk, size_t(h->nnzb) * RRp * esz);
    if (ce != cudaSuccess) {
      fail(h, TSP_ERR_NOMEM, "operator blocks (" + std::to_string(size_t(h->nnzb) * RRp * esz) +
                                 " bytes) do not fit: " + cudaGetErrorString(ce));
      return create_error_from(h, TSP_ERR_NOMEM);
    }
    h->owned.push_back(blk);
    h->d_blocks = blk;
    if (h->bpitch != h->R) TSP_CUDA(h, cudaMemsetAsync(blk, 0, size_t(h->nnzb) * RRp * esz, h->stream));
  }
  if (h->prec == TSP_PREC_BF16 && (rc = dalloc(h, &h->d_bscale, size_t(h->nnzb)))) return create_error_from(h, rc);
  tsp::AssembleParams ap;
  ap.ne = h->ne;
  ap.N = h->N;
  ap.Np = h->Np;
  ap.pen_n2 = P->penalty * h->N * h->N;
  ap.row_ptr = h->d_row_ptr;
  ap.col = h->d_col;
  ap.bface = d_bface;
  ap.neigh = d_neigh;
  ap.nedge = d_nedge;
  ap.invJ = d_invJ;
  ap.detJ = d_detJ;
  ap.elen = d_elen;
  ap.enrm = d_enrm;
  ap.lam = d_lam;
  ap.mu = d_mu;
  ap.K = d_K;
  ap.Ws = d_Ws;
  ap.Wx = d_Wx;
  ap.Ds = d_Ds;
  ap.Dx = d_Dx;
  ap.prec = h->prec;
  ap.pitch = h->bpitch;
  ap.out = h->d_blocks;
  ap.scale = h->d_bscale;
  // Non-orthonormal basis: assemble B in FP64 (in place for FP64 storage,
  // else in a temporary at pitch 2Np), then map it to L^-1 B L^-T.
  double* d_tmp = nullptr;
  if (!h->lref.empty()) {
    ap.prec = TSP_PREC_FP64;
    if (h->prec != TSP_PREC_FP64) {
      if ((rc = dalloc(h, &d_tmp, size_t(h->nnzb) * h->R * h->R))) return create_error_from(h, rc);
      ap.out = d_tmp;
      ap.pitch = h->R;
    }
  }
  // Large meshes exceed the 2^31-1 grid limit only beyond 2 G blocks.
  tsp::k_assemble<<<unsigned(h->ne), 256, 0, h->stream>>>(ap);
  {
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
    if (ce != cudaSuccess) {
      fail(h, TSP_ERR_CUDA, std::string("assembly kernel: ") + cudaGetErrorString(ce));
      return create_error_from(h, TSP_ERR_CUDA);
    }
  }
  if (!h->lref.empty()) {
    rc = fold_blocks(h, d_tmp ? d_tmp : reinterpret_cast<double*>(h->d_blocks), ap.pitch);
    if (d_tmp) dfree(h, d_tmp);
    if (rc) return create_error_from(h, rc);
  }
  for (void* q : {(void*)d_neigh, (void*)d_nedge, (void*)d_bface, (void*)d_invJ, (void*)d_detJ, (void*)d_elen,
                  (void*)d_enrm, (void*)d_lam, (void*)d_mu, (void*)d_K, (void*)d_Ws, (void*)d_Wx, (void*)d_Ds,
                  (void*)d_Dx})
    dfree(h, q);
  if ((rc = finish_create(h))) return create_error_from(h, rc);
  *out = h;
  return TSP_OK;
}

int tsp_create_from_blocks(const tsp_block_problem* P, tsp_handle** out) {
  NvtxRange nvtx_("tsp_create_from_blocks");
  if (!P || !out) return fail(nullptr, TSP_ERR_ARG, "null argument");
  *out = nullptr;
  if (P->ne <= 0 || P->Np <= 0 || P->nnzb < P->ne || !P->row_ptr || !P->col || !P->blocks || !P->minv)
    return fail(nullptr, TSP_ERR_ARG, "operator arrays missing");
  if (P->nshots < 1 || !P->src_elem || !P->src_phi) return fail(nullptr, TSP_ERR_ARG, "need nshots >= 1 sources");
  if (P->nrcv < 0 || (P->nrcv > 0 && (!P->rcv_elem || !P->rcv_phi))) return fail(nullptr, TSP_ERR_ARG, "bad receivers");
  if (P->precision < TSP_PREC_FP64 || P->precision > TSP_PREC_BF16) return fail(nullptr, TSP_ERR_ARG, "bad precision");
  int N = -1;
  for (int n = 1; n <= tsp::kMaxN; ++n)
    if (tsp::np_of(n) == P->Np) N = n;
  if (N < 0) return fail(nullptr, TSP_ERR_UNSUPPORTED, "Np must be (N+1)(N+2)/2 for N in 1..8");
  if (P->row_ptr[0] != 0 || P->row_ptr[P->ne] != P->nnzb) return fail(nullptr, TSP_ERR_ARG, "row_ptr inconsistent");
  for (int e = 0; e < P->ne; ++e) {
    const int n = P->row_ptr[e + 1] - P->row_ptr[e];
    if (n < 1 || n > 4) return fail(nullptr, TSP_ERR_ARG, "each block row needs 1..4 blocks");
  }
  for (int b = 0; b < P->nnzb; ++b)
    if (P->col[b] < 0 || P->col[b] >= P->ne) return fail(nullptr, TSP_ERR_ARG, "block column out of range");
  for (int s = 0; s < P->nshots; ++s)
    if (P->src_elem[s] < 0 || P->src_elem[s] >= P->ne) return fail(nullptr, TSP_ERR_ARG, "source element out of range");
  for (int r = 0; r < P->nrcv; ++r)
    if (P->rcv_elem[r] < 0 || P->rcv_elem[r] >= P->ne) return fail(nullptr, TSP_ERR_ARG, "receiver element out of range");
  std::vector<double> mref, mi;
  if (P->ref_invmass) {
    mi.assign(P->ref_invmass, P->ref_invmass + size_t(P->Np) * P->Np);
    if (!tsp::spd_inverse(P->Np, mi, &mref))
      return fail(nullptr, TSP_ERR_ARG, "ref_invmass is not symmetric positive definite");
  }

  tsp_handle* h = nullptr;
  int rc = make_handle(P->device, &h);
  if (rc) return rc;
  h->ne = P->ne;
  h->N = N;
  h->Np = P->Np;
  h->R = 2 * P->Np;
  h->S = P->nshots;
  h->nrcv = P->nrcv;
  h->prec = P->precision;
  h->nnzb = P->nnzb;
  if (P->ref_invmass && (rc = set_basis_mass(h, TSP_BASIS_BOUNDARY_ADAPTED, mref, mi))) return create_error_from(h, rc);
  h->src_elem.assign(P->src_elem, P->src_elem + h->S);
  h->src_phi.assign(P->src_phi, P->src_phi + size_t(h->S) * h->Np);
  h->rcv_elem.assign(P->rcv_elem, P->rcv_elem + h->nrcv);
  h->rcv_phi.assign(P->rcv_phi, P->rcv_phi + size_t(h->nrcv) * h->Np);
  if ((rc = upload(h, &h->d_row_ptr, P->row_ptr, size_t(P->ne) + 1)) || (rc = upload(h, &h->d_col, P->col, size_t(P->nnzb))) ||
      (rc = upload(h, &h->d_minv, P->minv, size_t(P->ne))))
    return create_error_from(h, rc);
  // Transpose every block to column-major and convert to the storage type.
  const int R = h->R;
  const size_t RR = size_t(R) * R;
  h->bpitch = block_pitch(R, h->S);
  const int BP = h->bpitch;
  if (!h->lref.empty()) {
    // FP64 column-major copy on the device, mapped to L^-1 B L^-T there.
    std::vector<double> cm(size_t(P->nnzb) * RR);
    for (int b = 0; b < P->nnzb; ++b)
      for (int r = 0; r < R; ++r)
        for (int c = 0; c < R; ++c) cm[size_t(b) * RR + size_t(c) * R + r] = P->blocks[size_t(b) * RR + size_t(r) * R + c];
    double* d_tmp = nullptr;
    const size_t esz = h->prec == TSP_PREC_FP64 ? 8 : (h->prec == TSP_PREC_FP32 ? 4 : 2);
    if ((rc = upload(h, &d_tmp, cm.data(), cm.size()))) return create_error_from(h, rc);
    std::vector<double>().swap(cm);
    unsigned char* dblk = nullptr;
    if ((rc = dalloc(h, &dblk, size_t(P->nnzb) * R * BP * esz))) return create_error_from(h, rc);
    h->d_blocks = dblk;
    TSP_CUDA(h, cudaMemsetAsync(h->d_blocks, 0, size_t(P->nnzb) * R * BP * esz, h->stream));
    if (h->prec == TSP_PREC_BF16 && (rc = dalloc(h, &h->d_bscale, size_t(P->nnzb)))) return create_error_from(h, rc);
    rc = fold_blocks(h, d_tmp, R);
    dfree(h, d_tmp);
    if (rc) return create_error_from(h, rc);
    if ((rc = finish_create(h))) return create_error_from(h, rc);
    *out = h;
    return TSP_OK;
  }
  const size_t esz = h->prec == TSP_PREC_FP64 ? 8 : (h->prec == TSP_PREC_FP32 ? 4 : 2);
  std::vector<unsigned char> host(size_t(P->nnzb) * R * BP * esz, 0);
  std::vector<float> scales(h->prec == TSP_PREC_BF16 ? size_t(P->nnzb) : 0);
  for (int b = 0; b < P->nnzb; ++b) {
    const double* src = P->blocks + size_t(b) * RR;
    float sc = 1.0f;
    if (h->prec == TSP_PREC_BF16) {
      float m = 0.0f;
      for (size_t t = 0; t < RR; ++t) m = std::max(m, float(std::fabs(src[t])));
      sc = m > 0 ? std::exp2(std::ceil(std::log2(m))) : 1.0f;
      scales[b] = sc;
    }
    for (int r = 0; r < R; ++r)
      for (int c = 0; c < R; ++c) {
        const double v = src[size_t(r) * R + c];
        const size_t o = size_t(b) * R * BP + size_t(c) * BP + r;
        if (h->prec == TSP_PREC_FP64) reinterpret_cast<double*>(host.data())[o] = v;
        else if (h->prec == TSP_PREC_FP32) reinterpret_cast<float*>(host.data())[o] = float(v);
        else reinterpret_cast<__nv_bfloat16*>(host.data())[o] = __float2bfloat16_rn(float(v) / sc);
      }
  }
  {
    unsigned char* d = nullptr;
    if ((rc = upload(h, &d, host.data(), host.size()))) return create_error_from(h, rc);
    h->d_blocks = d;
  }
  if (h->prec == TSP_PREC_BF16 && (rc = upload(h, &h->d_bscale, scales.data(), scales.size())))
    return create_error_from(h, rc);
  if ((rc = finish_create(h))) return create_error_from(h, rc);
  *out = h;
  return TSP_OK;
}

int tsp_destroy(tsp_handle* h) {
  if (!h) return TSP_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  clear_graphs(h);
  for (void* p : h->owned) cudaFreeAsync(p, h->stream);
  if (h->stream) {
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
  }
  delete h;
  return TSP_OK;
}

int tsp_release_cached_memory(int32_t device) {
  if (device < 0 || device >= kMaxDevices) return fail(nullptr, TSP_ERR_ARG, "device ordinal out of range");
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_pool_mutex);
    pool = g_pools[device];
  }
  if (!pool) return TSP_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
  cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(nullptr, TSP_ERR_CUDA, std::string("pool trim: ") + cudaGetErrorString(e));
  return TSP_OK;
}

int tsp_get_sizes(const tsp_handle* h, int32_t* ne, int32_t* Np, int32_t* nshots, int32_t* nrcv, int64_t* nnzb) {
  if (!h) return TSP_ERR_ARG;
  if (ne) *ne = h->ne;
  if (Np) *Np = h->Np;
  if (nshots) *nshots = h->S;
  if (nrcv) *nrcv = h->nrcv;
  if (nnzb) *nnzb = h->nnzb;
  return TSP_OK;
}

int tsp_set_dt(tsp_handle* h, double dt) {
  if (!h) return TSP_ERR_ARG;
  if (!(dt > 0) || !std::isfinite(dt)) return fail(h, TSP_ERR_ARG, "dt must be positive and finite");
  h->dt = dt;
  h->dt_set = true;
  clear_graphs(h);
  return TSP_OK;
}

int tsp_force_times(double dt, int64_t n, double* out) {
  if (n < 0 || (n > 0 && !out)) return TSP_ERR_ARG;
  tsp::force_times(dt, n, out);
  return TSP_OK;
}

int tsp_set_force_table(tsp_handle* h, int32_t shot, const double* F, int64_t n) {
  NvtxRange nvtx_("tsp_set_force_table");
  if (!h) return TSP_ERR_ARG;
  if (shot < 0 || shot >= h->S || n < 0 || (n > 0 && !F)) return fail(h, TSP_ERR_ARG, "bad force table");
  int rc;
  if ((rc = begin(h))) return rc;
  if (n > h->nF) {
    // Grow the [S][nF][2] table, keeping the other shots' entries.
    std::vector<double> grown(size_t(h->S) * n * 2, 0.0);
    for (int s = 0; s < h->S; ++s)
      if (h->nF)
        std::memcpy(&grown[size_t(s) * n * 2], &h->Fhost[size_t(s) * h->nF * 2], size_t(h->nF) * 2 * sizeof(double));
    h->Fhost.swap(grown);
    h->nF = n;
  }
  std::fill(h->Fhost.begin() + size_t(shot) * h->nF * 2, h->Fhost.begin() + size_t(shot + 1) * h->nF * 2, 0.0);
  std::memcpy(&h->Fhost[size_t(shot) * h->nF * 2], F, size_t(n) * 2 * sizeof(double));
  // Re-upload the whole table (setup-time call).
  if (h->d_F) {
    TSP_CUDA(h, cudaStreamSynchronize(h->stream));
    dfree(h, h->d_F);
    h->d_F = nullptr;
  }
  if ((rc = upload(h, &h->d_F, h->Fhost.data(), h->Fhost.size()))) return rc;
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  clear_graphs(h);
  return TSP_OK;
}

int tsp_set_ricker(tsp_handle* h, int32_t shot, double f0, double t0, double amp, int32_t direction, int64_t n) {
  if (!h) return TSP_ERR_ARG;
  if (!h->dt_set) return fail(h, TSP_ERR_STATE, "tsp_set_ricker needs tsp_set_dt first");
  if (direction != 0 && direction != 1) return fail(h, TSP_ERR_ARG, "direction must be 0 or 1");
  if (n < 0) return fail(h, TSP_ERR_ARG, "negative length");
  std::vector<double> t(static_cast<size_t>(n)), F(static_cast<size_t>(n) * 2, 0.0);
  tsp::force_times(h->dt, n, t.data());
  for (int64_t k = 0; k < n; ++k) F[size_t(k) * 2 + direction] = tsp::ricker(t[k], f0, t0, amp);
  return tsp_set_force_table(h, shot, F.data(), n);
}

int tsp_set_initial(tsp_handle* h, int32_t shot, const double* u0, const double* v0) {
  NvtxRange nvtx_("tsp_set_initial");
  if (!h) return TSP_ERR_ARG;
  if (shot < 0 || shot >= h->S) return fail(h, TSP_ERR_ARG, "shot out of range");
  int rc;
  if ((rc = begin(h))) return rc;
  const size_t nstate = size_t(h->ne) * h->S * h->R;
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  // Level u^0 lives in d_U[0] before first_step.
  h->cur = 0;
  if ((rc = put_shot(h, h->d_U[0], shot, u0))) return rc;
  if (v0 || h->d_v0) {
    if (!h->d_v0) {
      if ((rc = dalloc(h, &h->d_v0, nstate))) return rc;
      TSP_CUDA(h, cudaMemsetAsync(h->d_v0, 0, nstate * sizeof(double), h->stream));
    }
    if ((rc = put_shot(h, h->d_v0, shot, v0))) return rc;
  }
  h->steps_done = 0;
  h->last_time = 0.0;
  TSP_CUDA(h, cudaMemsetAsync(h->d_step, 0, sizeof(long long), h->stream));
  if ((rc = reset_nonfinite(h))) return rc;
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  clear_graphs(h);
  return TSP_OK;
}

int tsp_first_step(tsp_handle* h) {
  NvtxRange nvtx_("tsp_first_step");
  if (!h) return TSP_ERR_ARG;
  if (!h->dt_set) return fail(h, TSP_ERR_STATE, "first_step needs dt (tsp_set_dt)");
  int rc;
  if ((rc = begin(h))) return rc;
  if (h->steps_done != 0) {
    // The reference only warns here (TimeAdvance.cpp:26-27); restart from u^0 is not possible.
    return fail(h, TSP_ERR_STATE, "first_step after other steps");
  }
  if (h->energy_on) TSP_CUDA(h, cudaMemsetAsync(h->d_energy, 0, size_t(h->energy_cap) * sizeof(double), h->stream));
  // u^0 is in d_U[0]; write u^1 into d_U[1].
  if ((rc = refresh_shadow(h, 0))) return rc;
  if ((rc = launch_step(h, tsp::kModeFirst, h->d_U[0], h->d_v0, h->d_U[1], 0, 1.0, h->stream))) return rc;
  tsp::k_advance<<<1, 1, 0, h->stream>>>(h->d_step, 1);
  TSP_CUDA(h, cudaGetLastError());
  h->cur = 1;
  h->steps_done = 1;
  h->last_time = h->dt;  // TimeAdvance.cpp:31
  return TSP_OK;
}

int tsp_step(tsp_handle* h) {
  NvtxRange nvtx_("tsp_step");
  if (!h) return TSP_ERR_ARG;
  if (h->steps_done < 1) return fail(h, TSP_ERR_STATE, "step before first_step");
  int rc;
  if ((rc = begin(h))) return rc;
  double* x = h->d_U[h->cur];
  double* prev = h->d_U[1 - h->cur];
  if ((rc = launch_step(h, tsp::kModeStep, x, prev, prev, 0, 1.0, h->stream))) return rc;
  tsp::k_advance<<<1, 1, 0, h->stream>>>(h->d_step, 1);
  TSP_CUDA(h, cudaGetLastError());
  h->cur = 1 - h->cur;
  h->steps_done += 1;
  h->last_time = h->last_time + h->dt;  // TimeAdvance.cpp:46, 230
  return TSP_OK;
}

int tsp_run(tsp_handle* h, int64_t nsteps) {
  NvtxRange nvtx_("tsp_run");
  if (!h) return TSP_ERR_ARG;
  if (nsteps < 0) return fail(h, TSP_ERR_ARG, "negative step count");
  if (nsteps == 0) return TSP_OK;
  if (h->steps_done < 1) return fail(h, TSP_ERR_STATE, "run before first_step");
  int rc;
  if ((rc = begin(h))) return rc;
  // The run is a sequence of pieces, each a replay of a cached graph of
  // kRunChunk steps or of a power of two below it (the binary digits of the
  // remainder): at most 2 x (1 + log2 kRunChunk) graphs per handle, keyed by
  // length and the parity of the current level, whatever step counts the
  // caller asks for. Steps of a piece read the device step counter plus their
  // offset, and the piece advances the counter, so pieces replay anywhere in
  // time.
  int c = h->cur;
  for (int64_t left = nsteps; left > 0;) {
    long long len = kRunChunk;
    if (left < kRunChunk) {
      len = 1;
      while (len * 2 <= left) len *= 2;
    }
    const auto key = std::make_pair(len, c);
    auto it = h->graphs.find(key);
    if (it == h->graphs.end()) {
      cudaGraph_t graph;
      TSP_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      int cc = c;
      int lrc = TSP_OK;
      for (long long i = 0; i < len && lrc == TSP_OK; ++i) {
        lrc = launch_step(h, tsp::kModeStep, h->d_U[cc], h->d_U[1 - cc], h->d_U[1 - cc], int(i), 1.0, h->stream);
        cc = 1 - cc;
      }
      tsp::k_advance<<<1, 1, 0, h->stream>>>(h->d_step, len);
      cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
      if (lrc) return lrc;
      if (ce != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      cudaGraphExec_t exec;
      ce = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
      it = h->graphs.emplace(key, exec).first;
    }
    TSP_CUDA(h, cudaGraphLaunch(it->second, h->stream));
    if (len & 1) c = 1 - c;
    left -= len;
  }
  h->cur = c;
  h->steps_done += nsteps;
  for (int64_t i = 0; i < nsteps; ++i) h->last_time = h->last_time + h->dt;
  return TSP_OK;
}

int tsp_run_timed(tsp_handle* h, int64_t nsteps, double* ms) {
  NvtxRange nvtx_("tsp_run_timed");
  if (!h || !ms) return TSP_ERR_ARG;
  int rc;
  if ((rc = begin(h))) return rc;
  cudaEvent_t a, b;
  TSP_CUDA(h, cudaEventCreate(&a));
  TSP_CUDA(h, cudaEventCreate(&b));
  TSP_CUDA(h, cudaEventRecord(a, h->stream));
  rc = tsp_run(h, nsteps);
  if (rc == TSP_OK) {
    float f = 0.0f;
    cudaError_t e = cudaEventRecord(b, h->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&f, a, b);
    if (e != cudaSuccess) rc = fail(h, TSP_ERR_CUDA, std::string("timing events: ") + cudaGetErrorString(e));
    *ms = f;
    if (rc == TSP_OK) rc = check_device_error(h);
    if (rc == TSP_OK) rc = check_nonfinite(h);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

int tsp_get_kernel_variant(const tsp_handle* h, int32_t* variant) {
  if (!h || !variant) return TSP_ERR_ARG;
  // FP64 with several shots: 2 CUDA-core, 3 single-role DMMA, 5 and 6 the
  // warp-specialised DMMA kernel (two warp tiles); set by the autotuner.
  *variant = h->kernel_variant;
  return TSP_OK;
}

int tsp_checked_build(void) {
#ifdef TSP_CHECKED
  return 1;
#else
  return 0;
#endif
}

int tsp_get_progress(const tsp_handle* h, int64_t* steps_done, double* last_time) {
  if (!h) return TSP_ERR_ARG;
  if (steps_done) *steps_done = h->steps_done;
  if (last_time) *last_time = h->last_time;
  return TSP_OK;
}

int tsp_get_u(tsp_handle* h, int32_t shot, double* out) {
  NvtxRange nvtx_("tsp_get_u");
  if (!h || !out) return TSP_ERR_ARG;
  if (shot < 0 || shot >= h->S) return fail(h, TSP_ERR_ARG, "shot out of range");
  int rc;
  if ((rc = begin(h))) return rc;
  if ((rc = get_shot(h, h->d_U[h->cur], shot, out))) return rc;
  return check_device_error(h);
}

int tsp_get_u_all(tsp_handle* h, double* out) {
  NvtxRange nvtx_("tsp_get_u_all");
  if (!h || !out) return TSP_ERR_ARG;
  int rc;
  if ((rc = begin(h))) return rc;
  // The state is transposed to the reference layout on the device, a chunk
  // of shots at a time, and each chunk is copied back in one transfer.
  const size_t nref = size_t(2) * h->ne * h->Np;
  const int chunk = int(std::max<size_t>(1, std::min<size_t>(size_t(h->S), (size_t(256) << 20) / (nref * 8))));
  double* tmp = nullptr;
  if ((rc = dalloc(h, &tmp, nref * chunk))) return rc;
  for (int s0 = 0; s0 < h->S && rc == TSP_OK; s0 += chunk) {
    const int ns = std::min(chunk, h->S - s0);
    tsp::k_state_to_ref<<<1184, 256, 0, h->stream>>>(h->d_U[h->cur], h->ne, h->S, h->Np, s0, ns, tmp,
                                                     h->d_lref_inv);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out + size_t(s0) * nref, tmp, nref * ns * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = fail(h, TSP_ERR_CUDA, std::string("state read-back: ") + cudaGetErrorString(e));
  }
  dfree(h, tmp);
  if (rc) return rc;
  return check_device_error(h);
}

int tsp_set_seismogram_capacity(tsp_handle* h, int64_t nsteps) {
  if (!h) return TSP_ERR_ARG;
  if (nsteps < 1) return fail(h, TSP_ERR_ARG, "capacity must be >= 1");
  int rc;
  if ((rc = begin(h))) return rc;
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  if ((rc = alloc_seis(h, nsteps))) return rc;
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  return TSP_OK;
}

int tsp_get_seismograms(tsp_handle* h, int64_t k0, int64_t nk, double* out) {
  NvtxRange nvtx_("tsp_get_seismograms");
  if (!h) return TSP_ERR_ARG;
  if (k0 < 0 || nk < 0 || (nk > 0 && !out)) return fail(h, TSP_ERR_ARG, "bad range");
  if (nk > h->seis_cap) return fail(h, TSP_ERR_ARG, "range longer than the seismogram capacity");
  if (h->nrcv == 0 || nk == 0) return TSP_OK;
  int rc;
  if ((rc = begin(h))) return rc;
  const size_t per = size_t(h->nrcv) * 2;
  for (int s = 0; s < h->S; ++s)
    for (int64_t k = 0; k < nk;) {
      // Contiguous run inside the ring buffer.
      const long long slot = (k0 + k) % h->seis_cap;
      const long long run = std::min<long long>(nk - k, h->seis_cap - slot);
      TSP_CUDA(h, cudaMemcpyAsync(out + (size_t(s) * nk + k) * per, h->d_seis + (size_t(s) * h->seis_cap + slot) * per,
                                  size_t(run) * per * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      k += run;
    }
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
#ifdef TSP_CHECKED
  return check_device_error(h);  // the samples are void after an index failure
#else
  return TSP_OK;
#endif
}

int tsp_enable_energy(tsp_handle* h, int32_t on) {
  if (!h) return TSP_ERR_ARG;
  int rc;
  if ((rc = begin(h))) return rc;
  if (on && !h->d_energy) {
    h->energy_cap = std::max<long long>(h->seis_cap, 4096);
    if ((rc = dalloc(h, &h->d_energy, size_t(h->energy_cap)))) return rc;
    TSP_CUDA(h, cudaMemsetAsync(h->d_energy, 0, size_t(h->energy_cap) * sizeof(double), h->stream));
  }
  h->energy_on = on != 0;
  clear_graphs(h);
  return TSP_OK;
}

int tsp_get_energy(tsp_handle* h, int64_t k0, int64_t nk, double* out) {
  if (!h) return TSP_ERR_ARG;
  if (!h->d_energy) return fail(h, TSP_ERR_STATE, "energy monitor not enabled");
  if (k0 < 0 || nk < 0 || nk > h->energy_cap || (nk > 0 && !out)) return fail(h, TSP_ERR_ARG, "bad range");
  int rc;
  if ((rc = begin(h))) return rc;
  for (int64_t k = 0; k < nk;) {
    const long long slot = (k0 + k) % h->energy_cap;
    const long long run = std::min<long long>(nk - k, h->energy_cap - slot);
    TSP_CUDA(h, cudaMemcpyAsync(out + k, h->d_energy + slot, size_t(run) * sizeof(double), cudaMemcpyDeviceToHost,
                                h->stream));
    k += run;
  }
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  return TSP_OK;
}

int tsp_get_state(tsp_handle* h, double* u_prev, double* u_cur, int64_t* steps_done, double* last_time) {
  NvtxRange nvtx_("tsp_get_state");
  if (!h) return TSP_ERR_ARG;
  int rc;
  if ((rc = begin(h))) return rc;
  const size_t nstate = size_t(h->ne) * h->S * h->R, nref = size_t(2) * h->ne * h->Np;
  std::vector<double> all(nstate);
  for (int lvl = 0; lvl < 2; ++lvl) {
    double* dst = lvl == 0 ? u_prev : u_cur;
    if (!dst) continue;
    const double* src = lvl == 0 ? h->d_U[1 - h->cur] : h->d_U[h->cur];
    TSP_CUDA(h, cudaMemcpyAsync(all.data(), src, nstate * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TSP_CUDA(h, cudaStreamSynchronize(h->stream));
    for (int s = 0; s < h->S; ++s) dev_to_ref(h, s, all.data(), dst + size_t(s) * nref);
  }
  if (steps_done) *steps_done = h->steps_done;
  if (last_time) *last_time = h->last_time;
  return TSP_OK;
}

int tsp_set_state(tsp_handle* h, const double* u_prev, const double* u_cur, int64_t steps_done, double last_time) {
  NvtxRange nvtx_("tsp_set_state");
  if (!h || !u_prev || !u_cur) return TSP_ERR_ARG;
  if (steps_done < 1) return fail(h, TSP_ERR_ARG, "a resumable state has at least one step done");
  int rc;
  if ((rc = begin(h))) return rc;
  const size_t nstate = size_t(h->ne) * h->S * h->R, nref = size_t(2) * h->ne * h->Np;
  std::vector<double> all(nstate);
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  h->cur = 1;
  for (int lvl = 0; lvl < 2; ++lvl) {
    const double* src = lvl == 0 ? u_prev : u_cur;
    for (int s = 0; s < h->S; ++s) ref_to_dev(h, s, src + size_t(s) * nref, all.data());
    TSP_CUDA(h, copy_sync(lvl == 0 ? h->d_U[0] : h->d_U[1], all.data(), nstate * sizeof(double),
                          cudaMemcpyHostToDevice, h->stream));
  }
  if ((rc = refresh_shadow(h, 1))) return rc;
  h->steps_done = steps_done;
  h->last_time = last_time;
  if ((rc = reset_nonfinite(h))) return rc;
  long long sd = steps_done;
  TSP_CUDA(h, copy_sync(h->d_step, &sd, sizeof(sd), cudaMemcpyHostToDevice, h->stream));
  clear_graphs(h);
  return TSP_OK;
}

int tsp_check_finite(tsp_handle* h, int32_t* bad) {
  if (!h || !bad) return TSP_ERR_ARG;
  int rc;
  if ((rc = begin(h))) return rc;
  const size_t nstate = size_t(h->ne) * h->S * h->R;
  std::vector<double> all(nstate);
  TSP_CUDA(h, cudaMemcpyAsync(all.data(), h->d_U[h->cur], nstate * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  // The step kernels' flag (any non-finite value written since the initial
  // values were set), or a non-finite value in the current level.
  int flag = 0;
  if ((rc = read_nonfinite(h, &flag))) return rc;
  *bad = flag ? 1 : 0;
  for (size_t i = 0; i < all.size() && !*bad; ++i)
    if (!std::isfinite(all[i])) *bad = 1;
  return TSP_OK;
}

int tsp_apply(tsp_handle* h, const double* x, double* y) {
  if (!h || !x || !y) return TSP_ERR_ARG;
  int rc;
  if ((rc = begin(h))) return rc;
  // Single-vector product: temporary vectors in the one-shot layout [e][R].
  const size_t n1 = size_t(h->ne) * h->R;
  double *dx = nullptr, *dy = nullptr;
  if ((rc = dalloc(h, &dx, n1)) || (rc = dalloc(h, &dy, n1))) return rc;
  std::vector<double> v(n1, 0.0);
  for (int e = 0; e < h->ne; ++e)
    for (int c = 0; c < 2; ++c)
      std::memcpy(&v[size_t(e) * h->R + size_t(c) * h->Np], x + size_t(c) * h->ne * h->Np + size_t(e) * h->Np,
                  h->Np * sizeof(double));
  to_dev_coords(h, v.data(), 2ll * h->ne);  // B x = L (L^-1 B L^-T) (L^T x)
  TSP_CUDA(h, copy_sync(dx, v.data(), n1 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if ((rc = launch_step(h, tsp::kModeApply, dx, nullptr, dy, 0, 1.0, h->stream))) return rc;
  TSP_CUDA(h, cudaGetLastError());
  TSP_CUDA(h, cudaMemcpyAsync(v.data(), dy, n1 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (!h->lref.empty()) map_vectors(h->lref, false, h->Np, v.data(), 2ll * h->ne);
  for (int e = 0; e < h->ne; ++e)
    for (int c = 0; c < 2; ++c)
      std::memcpy(y + size_t(c) * h->ne * h->Np + size_t(e) * h->Np, &v[size_t(e) * h->R + size_t(c) * h->Np],
                  h->Np * sizeof(double));
  dfree(h, dx);
  dfree(h, dy);
  return TSP_OK;
}

int tsp_estimate_lmax(tsp_handle* h, int32_t iters, double* lmax) {
  NvtxRange nvtx_("tsp_estimate_lmax");
  if (!h || !lmax || iters < 1) return TSP_ERR_ARG;
  int rc;
  if ((rc = begin(h))) return rc;
  const size_t nstate = size_t(h->ne) * h->R;  // one vector, layout [e][R]
  double *da = nullptr, *db = nullptr;
  if ((rc = dalloc(h, &da, nstate)) || (rc = dalloc(h, &db, nstate))) return rc;
  // Deterministic start vector with all modes excited.
  std::vector<double> x0(nstate);
  uint64_t st = 0x9E3779B97F4A7C15ull;
  for (size_t i = 0; i < nstate; ++i) {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    x0[i] = double(st >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  }
  TSP_CUDA(h, copy_sync(da, x0.data(), nstate * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  double scale = 1.0, lam = 0.0;
  double acc[3];
  for (int it = 0; it < iters; ++it) {
    TSP_CUDA(h, cudaMemsetAsync(h->d_acc, 0, 3 * sizeof(double), h->stream));
    if ((rc = launch_step(h, tsp::kModePower, da, nullptr, db, 0, scale, h->stream))) return rc;
    TSP_CUDA(h, cudaMemcpyAsync(acc, h->d_acc, sizeof(acc), cudaMemcpyDeviceToHost, h->stream));
    TSP_CUDA(h, cudaStreamSynchronize(h->stream));
    lam = acc[0] / acc[1];  // Rayleigh quotient x^T B x / x^T M x
    scale = acc[2] > 0 ? 1.0 / std::sqrt(acc[2]) : 1.0;
    std::swap(da, db);
  }
  *lmax = lam;
  dfree(h, da);
  dfree(h, db);
  return TSP_OK;
}

int tsp_export_operator(tsp_handle* h, int32_t* row_ptr, int32_t* col, double* blocks, double* minv) {
  if (!h) return TSP_ERR_ARG;
  if (h->op_kind == TSP_OP_MATRIX_FREE && blocks)
    return fail(h, TSP_ERR_UNSUPPORTED, "a matrix-free handle stores no blocks");
  int rc;
  if ((rc = begin(h))) return rc;
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (row_ptr) TSP_CUDA(h, copy_sync(row_ptr, h->d_row_ptr, (size_t(h->ne) + 1) * 4, cudaMemcpyDeviceToHost, h->stream));
  if (col) TSP_CUDA(h, copy_sync(col, h->d_col, size_t(h->nnzb) * 4, cudaMemcpyDeviceToHost, h->stream));
  if (minv) TSP_CUDA(h, copy_sync(minv, h->d_minv, size_t(h->ne) * 8, cudaMemcpyDeviceToHost, h->stream));
  if (blocks) {
    const size_t RR = size_t(h->R) * h->R;
    const int BP = h->bpitch;
    const size_t esz = h->prec == TSP_PREC_FP64 ? 8 : (h->prec == TSP_PREC_FP32 ? 4 : 2);
    std::vector<unsigned char> raw(size_t(h->nnzb) * h->R * BP * esz);
    std::vector<float> sc;
    TSP_CUDA(h, copy_sync(raw.data(), h->d_blocks, raw.size(), cudaMemcpyDeviceToHost, h->stream));
    if (h->prec == TSP_PREC_BF16) {
      sc.resize(size_t(h->nnzb));
      TSP_CUDA(h, copy_sync(sc.data(), h->d_bscale, sc.size() * 4, cudaMemcpyDeviceToHost, h->stream));
    }
    for (long long b = 0; b < h->nnzb; ++b)
      for (int c = 0; c < h->R; ++c)
        for (int r = 0; r < h->R; ++r) {
          const size_t i = size_t(b) * h->R * BP + size_t(c) * BP + r;
          double v;
          if (h->prec == TSP_PREC_FP64) v = reinterpret_cast<double*>(raw.data())[i];
          else if (h->prec == TSP_PREC_FP32) v = reinterpret_cast<float*>(raw.data())[i];
          else v = double(__bfloat162float(reinterpret_cast<__nv_bfloat16*>(raw.data())[i])) * sc[b];
          blocks[size_t(b) * RR + size_t(r) * h->R + c] = v;
        }
    if (!h->lref.empty()) {
      // Stored: L^-1 B L^-T; exported: B = L (L^-1 B L^-T) L^T, applied to
      // the Np-segments of every row (right factor) and column (left factor).
      const int Np = h->Np, R = h->R;
      std::vector<double> col(Np);
      for (long long b = 0; b < h->nnzb; ++b) {
        double* blk = blocks + size_t(b) * RR;
        for (int r = 0; r < R; ++r) map_vectors(h->lref, false, Np, blk + size_t(r) * R, 2);
        for (int c = 0; c < R; ++c)
          for (int comp = 0; comp < 2; ++comp) {
            for (int j = 0; j < Np; ++j) col[j] = blk[size_t(comp * Np + j) * R + c];
            map_vectors(h->lref, false, Np, col.data(), 1);
            for (int j = 0; j < Np; ++j) blk[size_t(comp * Np + j) * R + c] = col[j];
          }
      }
    }
  }
  return TSP_OK;
}

int tsp_export_points(tsp_handle* h, int32_t* src_elem, double* src_phi, int32_t* rcv_elem, double* rcv_phi) {
  if (!h) return TSP_ERR_ARG;
  if (src_elem) std::copy(h->src_elem.begin(), h->src_elem.end(), src_elem);
  if (src_phi) std::copy(h->src_phi.begin(), h->src_phi.end(), src_phi);
  if (rcv_elem) std::copy(h->rcv_elem.begin(), h->rcv_elem.end(), rcv_elem);
  if (rcv_phi) std::copy(h->rcv_phi.begin(), h->rcv_phi.end(), rcv_phi);
  return TSP_OK;
}

int tsp_gmsh_read(const char* path, int32_t* nverts, double* xy, int32_t* ne, int32_t* tri, int32_t* region) {
  if (!path || !nverts || !ne) return fail(nullptr, TSP_ERR_ARG, "null argument");
  std::vector<double> vxy;
  std::vector<int32_t> vtri, vreg;
  std::string err;
  if (!tsp::gmsh_read(path, &vxy, &vtri, &vreg, &err)) return fail(nullptr, TSP_ERR_MESH, err);
  const int32_t nv = int32_t(vxy.size() / 2), nt = int32_t(vtri.size() / 3);
  if (xy && *nverts < nv) return fail(nullptr, TSP_ERR_ARG, "xy buffer too small");
  if (tri && *ne < nt) return fail(nullptr, TSP_ERR_ARG, "tri buffer too small");
  *nverts = nv;
  *ne = nt;
  if (xy) std::copy(vxy.begin(), vxy.end(), xy);
  if (tri) std::copy(vtri.begin(), vtri.end(), tri);
  if (region) std::copy(vreg.begin(), vreg.end(), region);
  return TSP_OK;
}

int tsp_quadrature_points(int32_t N, int32_t nverts, const double* xy, int32_t ne, const int32_t* tri, double* pts) {
  if (N < 1 || N > tsp::kMaxN || nverts <= 0 || ne <= 0 || !xy || !tri || !pts)
    return fail(nullptr, TSP_ERR_ARG, "bad arguments to tsp_quadrature_points");
  for (int32_t i = 0; i < 3 * ne; ++i)
    if (tri[i] < 0 || tri[i] >= nverts) return fail(nullptr, TSP_ERR_MESH, "vertex id out of range");
  tsp::quadrature_points(N, ne, xy, tri, pts);
  return TSP_OK;
}

int tsp_project_basis(int32_t N, int32_t basis, int32_t nverts, const double* xy, int32_t ne, const int32_t* tri,
                      const double* fvals, double* out) {
  if (N < 1 || N > tsp::kMaxN || nverts <= 0 || ne <= 0 || !xy || !tri || !fvals || !out)
    return fail(nullptr, TSP_ERR_ARG, "bad arguments to tsp_project");
  if (basis != TSP_BASIS_DUBINER && basis != TSP_BASIS_BOUNDARY_ADAPTED) return fail(nullptr, TSP_ERR_ARG, "bad basis");
  for (int32_t i = 0; i < 3 * ne; ++i)
    if (tri[i] < 0 || tri[i] >= nverts) return fail(nullptr, TSP_ERR_MESH, "vertex id out of range");
  tsp::project(N, ne, xy, tri, fvals, out, basis);
  return TSP_OK;
}

int tsp_project(int32_t N, int32_t nverts, const double* xy, int32_t ne, const int32_t* tri, const double* fvals,
                double* out) {
  return tsp_project_basis(N, TSP_BASIS_DUBINER, nverts, xy, ne, tri, fvals, out);
}

namespace {

// Basis values at reference points in the device's coordinates: T[q][j] =
// phi_j(r_q) for Dubiner, (L^-1 phi(r_q))_j for a non-orthonormal basis
// (u_h = phi^T u = (L^-1 phi)^T w).
std::vector<double> device_basis_table(const tsp_handle* h, int npt, const double* rc, const double* re) {
  std::vector<double> T(size_t(npt) * h->Np);
  for (int q = 0; q < npt; ++q) tsp::basis_phi(h->basis, h->N, rc[q], re[q], &T[size_t(q) * h->Np]);
  if (!h->lref_inv.empty()) map_vectors(h->lref_inv, false, h->Np, T.data(), npt);
  return T;
}

int field_values(tsp_handle* h, int shot, std::vector<double>* vals) {
  double rc[4], re[4];
  for (int q = 0; q < 4; ++q) {
    rc[q] = tsp::kFieldPoints[q][0];
    re[q] = tsp::kFieldPoints[q][1];
  }
  const std::vector<double> T = device_basis_table(h, 4, rc, re);
  int rc_ = TSP_OK;
  double *dT = nullptr, *dout = nullptr;
  const size_t n = size_t(h->ne) * 8;
  if ((rc_ = upload(h, &dT, T.data(), T.size())) || (rc_ = dalloc(h, &dout, n))) return rc_;
  tsp::k_eval_points<<<1184, 256, 0, h->stream>>>(h->d_U[h->cur], h->ne, h->S, h->Np, shot, dT, 4, dout);
  vals->resize(n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(vals->data(), dout, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  dfree(h, dT);
  dfree(h, dout);
  if (e != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("field values: ") + cudaGetErrorString(e));
  return TSP_OK;
}

}  // namespace

int tsp_field_values(tsp_handle* h, int32_t shot, double* out) {
  if (!h || !out) return TSP_ERR_ARG;
  if (shot < 0 || shot >= h->S) return fail(h, TSP_ERR_ARG, "shot out of range");
  int rc;
  if ((rc = begin(h))) return rc;
  std::vector<double> v;
  if ((rc = field_values(h, shot, &v))) return rc;
  std::copy(v.begin(), v.end(), out);
  return check_device_error(h);
}

int tsp_write_field(tsp_handle* h, int32_t shot, const char* fname, int64_t step) {
  if (!h || !fname || step < 0) return TSP_ERR_ARG;
  if (shot < 0 || shot >= h->S) return fail(h, TSP_ERR_ARG, "shot out of range");
  int rc;
  if ((rc = begin(h))) return rc;
  std::vector<double> v;
  if ((rc = field_values(h, shot, &v))) return rc;
  if ((rc = check_device_error(h))) return rc;
  // The file name and line format of FESpace::field_out (FESpace_imp.hpp:89-103).
  const std::string path = std::string(fname) + "u_" + std::to_string(step) + ".field";
  std::ofstream f(path);
  if (!f.is_open()) return fail(h, TSP_ERR_ARG, "cannot open " + path);
  for (size_t i = 0; i < v.size(); i += 2) f << v[i] << " " << v[i + 1] << std::endl;
  if (!f.good()) return fail(h, TSP_ERR_ARG, "write failed: " + path);
  return TSP_OK;
}

int tsp_l2_error(tsp_handle* h, int32_t shot, const double* exact, double* err) {
  if (!h || !exact || !err) return TSP_ERR_ARG;
  if (shot < 0 || shot >= h->S) return fail(h, TSP_ERR_ARG, "shot out of range");
  if (h->detJ.empty()) return fail(h, TSP_ERR_UNSUPPORTED, "the L2 error needs the mesh (handle built from blocks)");
  int rc;
  if ((rc = begin(h))) return rc;
  std::vector<double> c, e, w;
  tsp::volume_rule(h->N, &c, &e, &w);
  const int nq = int(w.size());
  const std::vector<double> T = device_basis_table(h, nq, c.data(), e.data());
  double *dT = nullptr, *dw = nullptr, *dJ = nullptr, *dex = nullptr, *dout = nullptr;
  if ((rc = upload(h, &dT, T.data(), T.size())) || (rc = upload(h, &dw, w.data(), w.size())) ||
      (rc = upload(h, &dJ, h->detJ.data(), h->detJ.size())) ||
      (rc = upload(h, &dex, exact, size_t(h->ne) * nq * 2)) || (rc = dalloc(h, &dout, size_t(h->ne)))) {
    for (void* q : {(void*)dT, (void*)dw, (void*)dJ, (void*)dex, (void*)dout}) dfree(h, q);
    return rc;
  }
  tsp::k_l2_local<<<(h->ne + 255) / 256, 256, 0, h->stream>>>(h->d_U[h->cur], h->ne, h->S, h->Np, shot, dT, dw, nq, dJ,
                                                               dex, dout);
  std::vector<double> loc(h->ne);
  cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(loc.data(), dout, loc.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
  for (void* q : {(void*)dT, (void*)dw, (void*)dJ, (void*)dex, (void*)dout}) dfree(h, q);
  if (ce != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("L2 error: ") + cudaGetErrorString(ce));
  double s = 0.0;
  for (double v : loc) s += v;
  *err = std::sqrt(s);
  return check_device_error(h);
}

int tsp_set_initial_values(tsp_handle* h, int32_t shot, const double* u_vals, const double* v_vals) {
  NvtxRange nvtx_("tsp_set_initial_values");
  if (!h) return TSP_ERR_ARG;
  if (shot < 0 || shot >= h->S) return fail(h, TSP_ERR_ARG, "shot out of range");
  if (h->detJ.empty()) return fail(h, TSP_ERR_UNSUPPORTED, "the projection needs the mesh (handle built from blocks)");
  int rc;
  if ((rc = begin(h))) return rc;
  const size_t nstate = size_t(h->ne) * h->S * h->R;
  std::vector<double> c, e, w;
  tsp::volume_rule(h->N, &c, &e, &w);
  const int nq = int(w.size());
  const std::vector<double> T = device_basis_table(h, nq, c.data(), e.data());
  const size_t nv = size_t(h->ne) * nq * 2;
  double *dT = nullptr, *dw = nullptr, *dJ = nullptr, *dval = nullptr;
  auto cleanup = [&]() {
    for (void* q : {(void*)dT, (void*)dw, (void*)dJ, (void*)dval}) dfree(h, q);
  };
  if ((rc = upload(h, &dT, T.data(), T.size())) || (rc = upload(h, &dw, w.data(), w.size())) ||
      (rc = upload(h, &dJ, h->detJ.data(), h->detJ.size())) || (rc = dalloc(h, &dval, nv))) {
    cleanup();
    return rc;
  }
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (v_vals && !h->d_v0) {
    if ((rc = dalloc(h, &h->d_v0, nstate))) {
      cleanup();
      return rc;
    }
    TSP_CUDA(h, cudaMemsetAsync(h->d_v0, 0, nstate * sizeof(double), h->stream));
  }
  // Level u^0 lives in d_U[0] before first_step (as tsp_set_initial).
  h->cur = 0;
  cudaError_t ce = cudaSuccess;
  for (int lvl = 0; lvl < 2 && ce == cudaSuccess; ++lvl) {
    const double* vals = lvl == 0 ? u_vals : v_vals;
    double* dst = lvl == 0 ? h->d_U[0] : h->d_v0;
    if (!dst) continue;
    if (vals) ce = cudaMemcpyAsync(dval, vals, nv * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (ce == cudaSuccess) {
      tsp::k_project_points<<<1184, 256, 0, h->stream>>>(dst, h->ne, h->S, h->Np, shot, dT, dw, nq, dJ,
                                                         vals ? dval : nullptr);
      ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
  }
  cleanup();
  if (ce != cudaSuccess) return fail(h, TSP_ERR_CUDA, std::string("projection: ") + cudaGetErrorString(ce));
  h->steps_done = 0;
  h->last_time = 0.0;
  TSP_CUDA(h, cudaMemsetAsync(h->d_step, 0, sizeof(long long), h->stream));
  if ((rc = reset_nonfinite(h))) return rc;
  TSP_CUDA(h, cudaStreamSynchronize(h->stream));
  clear_graphs(h);
  return TSP_OK;
}

int tsp_points_out(int32_t nverts, const double* xy, int32_t ne, const int32_t* tri, const char* fname) {
  if (nverts <= 0 || ne <= 0 || !xy || !tri || !fname) return fail(nullptr, TSP_ERR_ARG, "bad arguments to tsp_points_out");
  for (int32_t i = 0; i < 3 * ne; ++i)
    if (tri[i] < 0 || tri[i] >= nverts) return fail(nullptr, TSP_ERR_MESH, "vertex id out of range");
  std::ofstream f(fname);
  if (!f.is_open()) return fail(nullptr, TSP_ERR_ARG, std::string("cannot open ") + fname);
  // Triangle::map(p) = p0 + J p (Geometry.cpp:203-207), J = [p1 - p0 | p2 - p0].
  for (int32_t el = 0; el < ne; ++el) {
    const double* p0 = xy + 2 * size_t(tri[3 * size_t(el)]);
    const double* p1 = xy + 2 * size_t(tri[3 * size_t(el) + 1]);
    const double* p2 = xy + 2 * size_t(tri[3 * size_t(el) + 2]);
    for (int q = 0; q < 4; ++q) {
      const double a = tsp::kFieldPoints[q][0], b = tsp::kFieldPoints[q][1];
      f << p0[0] + ((p1[0] - p0[0]) * a + (p2[0] - p0[0]) * b) << " "
        << p0[1] + ((p1[1] - p0[1]) * a + (p2[1] - p0[1]) * b) << std::endl;
    }
  }
  if (!f.good()) return fail(nullptr, TSP_ERR_ARG, std::string("write failed: ") + fname);
  return TSP_OK;
}

int tsp_locate_points(int32_t N, int32_t basis, int32_t nverts, const double* xy, int32_t ne, const int32_t* tri,
                      int32_t npts, const double* pts, int32_t* elem, double* phi) {
  if (N < 1 || N > tsp::kMaxN || nverts <= 0 || ne <= 0 || !xy || !tri || npts < 0 ||
      (npts > 0 && (!pts || !elem || !phi)))
    return fail(nullptr, TSP_ERR_ARG, "bad arguments to tsp_locate_points");
  if (basis != TSP_BASIS_DUBINER && basis != TSP_BASIS_BOUNDARY_ADAPTED) return fail(nullptr, TSP_ERR_ARG, "bad basis");
  for (int32_t i = 0; i < 3 * ne; ++i)
    if (tri[i] < 0 || tri[i] >= nverts) return fail(nullptr, TSP_ERR_MESH, "vertex id out of range");
  for (int32_t i = 0; i < 2 * nverts; ++i)
    if (!std::isfinite(xy[i])) return fail(nullptr, TSP_ERR_MESH, "vertex coordinates must be finite");
  const tsp::Geometry g = tsp::make_geometry(ne, xy, tri);
  tsp::locate_points(N, ne, xy, tri, g, npts, pts, elem, phi, basis);
  return TSP_OK;
}

int tsp_eval_basis(int32_t N, int32_t basis, int32_t npts, const double* rpts, double* phi) {
  if (N < 1 || N > tsp::kMaxN || npts < 0 || (npts > 0 && (!rpts || !phi)))
    return fail(nullptr, TSP_ERR_ARG, "bad arguments to tsp_eval_basis");
  if (basis != TSP_BASIS_DUBINER && basis != TSP_BASIS_BOUNDARY_ADAPTED) return fail(nullptr, TSP_ERR_ARG, "bad basis");
  const int Np = tsp::np_of(N);
  for (int32_t q = 0; q < npts; ++q) tsp::basis_phi(basis, N, rpts[2 * q], rpts[2 * q + 1], phi + size_t(q) * Np);
  return TSP_OK;
}

int tsp_quadrature_rule(int32_t N, double* rpts, double* w) {
  if (N < 1 || N > tsp::kMaxN) return fail(nullptr, TSP_ERR_ARG, "degree N must be in 1..8");
  std::vector<double> c, e, wq;
  tsp::volume_rule(N, &c, &e, &wq);
  for (size_t q = 0; q < wq.size(); ++q) {
    if (rpts) {
      rpts[2 * q] = c[q];
      rpts[2 * q + 1] = e[q];
    }
    if (w) w[q] = wq[q];
  }
  return TSP_OK;
}

namespace {
__device__ double g_peak_sink;
}  // namespace

int tsp_selftest_bounded_wait(int32_t device, int32_t* completed, int32_t* abort_raised) {
  if (!completed || !abort_raised) return fail(nullptr, TSP_ERR_ARG, "null argument");
  int prev = 0;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(device);
  cudaStream_t st = nullptr;
  int* d = nullptr;
  int h[3] = {-1, -1, -1};
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&d), 3 * sizeof(int), st);
  if (e == cudaSuccess) {
    tsp::k_selftest_bounded_wait<<<1, 32, 0, st>>>(d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (d) cudaFreeAsync(d, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (st) cudaStreamDestroy(st);
  cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(nullptr, TSP_ERR_CUDA, std::string("bounded-wait self-test: ") + cudaGetErrorString(e));
  *completed = h[0];
  *abort_raised = h[1];
  return TSP_OK;
}

int tsp_fp64_tensor_peak(int32_t device, double* tflops) {
  if (!tflops) return fail(nullptr, TSP_ERR_ARG, "null argument");
  int prev = 0, sms = 0;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  double* sink = nullptr;
  if (e == cudaSuccess) e = cudaGetSymbolAddress(reinterpret_cast<void**>(&sink), g_peak_sink);
  float ms = 0.0f;
  const int grid = 4 * sms, threads = 512, iters = 1024;
  if (e == cudaSuccess) {
    tsp::k_fp64_tensor_peak<<<grid, threads, 0, st>>>(sink, 16);  // warm-up
    e = cudaEventRecord(e0, st);
    tsp::k_fp64_tensor_peak<<<grid, threads, 0, st>>>(sink, iters);
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(nullptr, TSP_ERR_CUDA, std::string("FP64 tensor probe: ") + cudaGetErrorString(e));
  // 8 DMMAs of 8 x 8 x 4 multiply-adds per warp and iteration.
  const double flops = 2.0 * 256.0 * 8.0 * iters * double(grid) * (threads / 32);
  *tflops = flops / (double(ms) * 1e-3) / 1e12;
  return TSP_OK;
}

int tsp_get_ref_invmass(const tsp_handle* h, int32_t* basis, double* out) {
  if (!h) return TSP_ERR_ARG;
  if (basis) *basis = h->basis;
  if (out) {
    const size_t n = size_t(h->Np) * h->Np;
    if (h->minv_ref.empty())
      for (size_t i = 0; i < n; ++i) out[i] = (i % (size_t(h->Np) + 1) == 0) ? 1.0 : 0.0;
    else
      std::copy(h->minv_ref.begin(), h->minv_ref.end(), out);
  }
  return TSP_OK;
}

int tsp_mesh_neighbours(int32_t ne, const int32_t* tri, int32_t* neigh, int32_t* neighedge) {
  if (ne <= 0 || !tri || !neigh || !neighedge) return fail(nullptr, TSP_ERR_ARG, "null argument");
  std::string err;
  if (!tsp::build_neighbours(ne, tri, neigh, neighedge, &err)) return fail(nullptr, TSP_ERR_MESH, err);
  return TSP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free power iteration.
//
// For callers that may not allocate device memory at the time they need a
// CFL estimate: code running under a caching allocator or memory pool that
// forbids raw cudaMalloc, real-time loops where an allocation's implicit
// synchronisation is unacceptable, or applications that own all device memory
// and cap what libraries may take. The two iteration vectors and the three
// accumulators live in this file-scope array instead of cudaMalloc'd buffers;
// every GPU that loads the library holds it until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchDoubles = size_t(4) << 20;  // 4 Mi doubles = 32 MiB
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

__global__ void k_noalloc_start_vector(double* x, size_t n) {
  // Deterministic start vector with all modes excited (splitmix64 of the index).
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    unsigned long long z = (unsigned long long)i + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    x[i] = double(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  }
}

}  // namespace

extern "C" int tsp_estimate_lmax_noalloc(tsp_handle* h, int32_t iters, double* lmax) {
  if (!h || !lmax || iters < 1) return TSP_ERR_ARG;
  int rc;
  if ((rc = begin(h))) return rc;
  if (h->nmesh > 0)
    return fail(h, TSP_ERR_UNSUPPORTED,
                "tsp_estimate_lmax_noalloc: multi-mesh groups estimate per mesh (tsp_batch_estimate_lmax)");
  const size_t n1 = size_t(h->ne) * h->R;  // one vector, layout [e][R]
  if (2 * n1 + 3 > kNoAllocScratchDoubles)
    return fail(h, TSP_ERR_ARG,
                "tsp_estimate_lmax_noalloc: 2*ne*2Np + 3 = " + std::to_string(2 * n1 + 3) +
                    " doubles exceed the fixed scratch of " + std::to_string(kNoAllocScratchDoubles) +
                    " doubles (32 MiB); use tsp_estimate_lmax");
  // Device address of the array in the current context (begin() made the
  // handle's device current). Looked up on every call -- a cheap host query
  // -- so that no address outlives a context reset and concurrent callers
  // share no host state. Host code cannot use the symbol itself as a device
  // pointer.
  void* ptr = nullptr;
  cudaError_t ge = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (ge != cudaSuccess)
    return fail(h, TSP_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(ge));
  double* da = static_cast<double*>(ptr);
  double* db = da + n1;
  double* dacc = db + n1;
  k_noalloc_start_vector<<<592, 256, 0, h->stream>>>(da, n1);
  TSP_CUDA(h, cudaGetLastError());
  tsp::StepParams p;
  std::memset(&p, 0, sizeof(p));
  p.ne = h->ne;
  p.S = 1;
  p.mode = tsp::kModePower;
  p.row_ptr = h->d_row_ptr;
  p.col = h->d_col;
  p.blocks = h->d_blocks;
  p.bpitch = h->bpitch;
  p.bscale = (h->prec == TSP_PREC_BF16) ? h->d_bscale : nullptr;
  p.minv = h->d_minv;
  p.acc = dacc;
  p.nnzb = h->nnzb;
  double scale = 1.0, lam = 0.0;
  double acc[3];
  for (int it = 0; it < iters; ++it) {
    // The accumulators keep the previous call's values: clear them.
    TSP_CUDA(h, cudaMemsetAsync(dacc, 0, 3 * sizeof(double), h->stream));
    p.x = da;
    p.out = db;
    p.xscale = scale;
    if ((rc = launch_step_params(h, p, h->stream))) return rc;
    TSP_CUDA(h, cudaGetLastError());
    TSP_CUDA(h, cudaMemcpyAsync(acc, dacc, sizeof(acc), cudaMemcpyDeviceToHost, h->stream));
    TSP_CUDA(h, cudaStreamSynchronize(h->stream));
    lam = acc[0] / acc[1];
    scale = acc[2] > 0 ? 1.0 / std::sqrt(acc[2]) : 1.0;
    std::swap(da, db);
  }
  *lmax = lam;
  return TSP_OK;
}


// ---------------------------------------------------------------------------
// Multi-mesh batch: independent meshes of uneven size and degree advanced
// together. Meshes of one degree are concatenated into one group handle (a
// block-diagonal-by-mesh system with per-element dt, per-element source
// index and per-element mesh id); every step of every group is captured in
// one CUDA graph.
// ---------------------------------------------------------------------------
struct tsp_batch {
  int nmesh = 0;
  std::vector<tsp_handle*> groups;     // one per degree present
  std::vector<int> mesh_group;         // mesh -> group
  std::vector<int> mesh_first;         // mesh -> first element in its group
  std::vector<int> mesh_ne, mesh_Np;   // per mesh
  std::vector<int> mesh_rcv0, mesh_nrcv;  // mesh -> first receiver id in its group, count
  std::vector<int> group_first_mesh;   // group -> mesh ids in order
  std::vector<std::vector<int>> group_meshes;
  cudaStream_t stream = nullptr;
  int device = 0;
  std::map<long long, cudaGraphExec_t> graphs;
  std::string err = "no error";
};

namespace {
int bfail(tsp_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  else g_create_error = msg;
  return code;
}
void batch_clear_graphs(tsp_batch* b) {
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
}
}  // namespace

extern "C" {

int tsp_batch_destroy(tsp_batch* b) {
  if (!b) return TSP_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_clear_graphs(b);
  for (tsp_handle* h : b->groups) tsp_destroy(h);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return TSP_OK;
}

const char* tsp_batch_last_error(const tsp_batch* b) { return b ? b->err.c_str() : g_create_error.c_str(); }

int tsp_batch_create(const tsp_problem* meshes, int32_t nmesh, tsp_batch** out) {
  NvtxRange nvtx_("tsp_batch_create");
  if (!meshes || !out || nmesh < 1) return bfail(nullptr, TSP_ERR_ARG, "need nmesh >= 1 problems");
  *out = nullptr;
  const int prec = meshes[0].precision, op = meshes[0].op_kind, dev = meshes[0].device;
  for (int m = 0; m < nmesh; ++m) {
    const tsp_problem& P = meshes[m];
    if (P.nshots != 1 || !P.src_xy) return bfail(nullptr, TSP_ERR_ARG, "each mesh of a batch has exactly one source");
    if (P.precision != prec || P.op_kind != op || P.device != dev)
      return bfail(nullptr, TSP_ERR_ARG, "all meshes of a batch share precision, operator kind and device");
    if (P.basis != TSP_BASIS_DUBINER)
      return bfail(nullptr, TSP_ERR_UNSUPPORTED, "multi-mesh batches are built for the Dubiner basis");
    if (P.N < 1 || P.N > tsp::kMaxN || P.ne <= 0 || P.nverts <= 0 || !P.xy || !P.tri || !P.lambda || !P.mu || !P.rho)
      return bfail(nullptr, TSP_ERR_ARG, "mesh " + std::to_string(m) + ": bad problem");
    if (P.nrcv < 0 || (P.nrcv > 0 && !P.rcv_xy)) return bfail(nullptr, TSP_ERR_ARG, "bad receivers");
  }
  tsp_batch* b = new tsp_batch();
  b->nmesh = nmesh;
  b->device = dev;
  b->mesh_group.assign(nmesh, -1);
  b->mesh_first.assign(nmesh, 0);
  b->mesh_ne.assign(nmesh, 0);
  b->mesh_Np.assign(nmesh, 0);
  b->mesh_rcv0.assign(nmesh, 0);
  b->mesh_nrcv.assign(nmesh, 0);
  if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return bfail(nullptr, TSP_ERR_CUDA, "batch stream creation failed");
  }
  for (int N = 1; N <= tsp::kMaxN; ++N) {
    std::vector<int> ms;
    for (int m = 0; m < nmesh; ++m)
      if (meshes[m].N == N) ms.push_back(m);
    if (ms.empty()) continue;
    const int g = int(b->groups.size());
    const int Np = tsp::np_of(N);
    // Concatenate the group's meshes (vertex ids offset, no shared vertices).
    std::vector<double> xy, lam, mu, rho, src_phi, rcv_phi;
    std::vector<int32_t> tri, src_of, mesh_of, rcv_elem;
    std::vector<double> rcv_xy_dummy;
    int vbase = 0, ebase = 0, rbase = 0;
    for (size_t q = 0; q < ms.size(); ++q) {
      const tsp_problem& P = meshes[ms[q]];
      xy.insert(xy.end(), P.xy, P.xy + 2 * size_t(P.nverts));
      for (int i = 0; i < 3 * P.ne; ++i) tri.push_back(P.tri[i] + vbase);
      lam.insert(lam.end(), P.lambda, P.lambda + P.ne);
      mu.insert(mu.end(), P.mu, P.mu + P.ne);
      rho.insert(rho.end(), P.rho, P.rho + P.ne);
      // Point location within the mesh only (meshes may overlap in space).
      tsp::Geometry gq = tsp::make_geometry(P.ne, P.xy, P.tri);
      std::vector<double> ph(Np);
      const int se = tsp::locate_point(N, P.ne, P.xy, P.tri, gq, P.src_xy[0], P.src_xy[1], ph.data());
      if (se < 0) {
        tsp_batch_destroy(b);
        return bfail(nullptr, TSP_ERR_NOT_FOUND, "mesh " + std::to_string(ms[q]) + ": source point not found");
      }
      src_of.resize(size_t(ebase) + P.ne, -1);
      src_of[size_t(ebase) + se] = int(q);
      src_phi.insert(src_phi.end(), ph.begin(), ph.end());
      for (int r = 0; r < P.nrcv; ++r) {
        const int re = tsp::locate_point(N, P.ne, P.xy, P.tri, gq, P.rcv_xy[2 * r], P.rcv_xy[2 * r + 1], ph.data());
        if (re < 0) {
          tsp_batch_destroy(b);
          return bfail(nullptr, TSP_ERR_NOT_FOUND, "mesh " + std::to_string(ms[q]) + ": receiver not found");
        }
        rcv_elem.push_back(ebase + re);
        rcv_phi.insert(rcv_phi.end(), ph.begin(), ph.end());
      }
      for (int e = 0; e < P.ne; ++e) mesh_of.push_back(int(q));
      b->mesh_group[ms[q]] = g;
      b->mesh_first[ms[q]] = ebase;
      b->mesh_ne[ms[q]] = P.ne;
      b->mesh_Np[ms[q]] = Np;
      b->mesh_rcv0[ms[q]] = rbase;
      b->mesh_nrcv[ms[q]] = P.nrcv;
      vbase += P.nverts;
      ebase += P.ne;
      rbase += P.nrcv;
    }
    // Group handle from the concatenated mesh. Its own source/receiver search
    // is replaced below by the per-mesh results.
    const tsp_problem& P0 = meshes[ms[0]];
    std::vector<double> sxy;
    {
      // A point inside element 0 of the group (its centroid) as placeholder source.
      const double* a = &xy[2 * size_t(tri[0])];
      const double* c1 = &xy[2 * size_t(tri[1])];
      const double* c2 = &xy[2 * size_t(tri[2])];
      sxy = {(a[0] + c1[0] + c2[0]) / 3.0, (a[1] + c1[1] + c2[1]) / 3.0};
    }
    tsp_problem G = {};
    G.nverts = vbase;
    G.xy = xy.data();
    G.ne = ebase;
    G.tri = tri.data();
    G.N = N;
    G.lambda = lam.data();
    G.mu = mu.data();
    G.rho = rho.data();
    G.penalty = P0.penalty;
    G.precision = prec;
    G.op_kind = op;
    G.nshots = 1;
    G.src_xy = sxy.data();
    G.nrcv = 0;
    G.rcv_xy = nullptr;
    G.device = dev;
    tsp_handle* h = nullptr;
    int rc = tsp_create(&G, &h);
    if (rc) {
      const std::string msg = std::string("group N=") + std::to_string(N) + ": " + tsp_last_error(nullptr);
      tsp_batch_destroy(b);
      return bfail(nullptr, rc, msg);
    }
    b->groups.push_back(h);
    b->group_meshes.push_back(ms);
    // Per-mesh sources and receivers, mesh ids, per-mesh power scales.
    h->nmesh = int(ms.size());
    h->src_elem.assign(1, -1);
    h->src_phi = src_phi;  // [nmesh][Np], row = source index
    h->rcv_elem = rcv_elem;
    h->rcv_phi = rcv_phi;
    h->nrcv = rbase;
    dfree(h, h->d_src_phi);
    dfree(h, h->d_rcv_ptr);
    dfree(h, h->d_rcv_id);
    dfree(h, h->d_rcv_phi);
    h->d_rcv_ptr = nullptr;
    h->d_rcv_id = nullptr;
    h->d_rcv_phi = nullptr;
    std::vector<double> ones(ms.size(), 1.0);
    if ((rc = upload(h, &h->d_src_phi, src_phi.data(), src_phi.size())) ||
        (rc = upload(h, &h->d_src_of, src_of.data(), src_of.size())) ||
        (rc = upload(h, &h->d_mesh_of, mesh_of.data(), mesh_of.size())) ||
        (rc = upload(h, &h->d_xscale_mesh, ones.data(), ones.size())) || (rc = build_receiver_csr(h)) ||
        (rc = alloc_seis(h, h->seis_cap)) || (rc = dalloc(h, &h->d_dt_elem, size_t(ebase)))) {
      const std::string msg = h->err;
      tsp_batch_destroy(b);
      return bfail(nullptr, rc, msg);
    }
    dfree(h, h->d_acc);
    if ((rc = dalloc(h, &h->d_acc, 3 * ms.size()))) {
      const std::string msg = h->err;
      tsp_batch_destroy(b);
      return bfail(nullptr, rc, msg);
    }
    cudaStreamSynchronize(h->stream);
  }
  *out = b;
  return TSP_OK;
}

int tsp_batch_info(const tsp_batch* b, int32_t* ngroups, int64_t* total_dofs) {
  if (!b) return TSP_ERR_ARG;
  if (ngroups) *ngroups = int32_t(b->groups.size());
  if (total_dofs) {
    int64_t t = 0;
    for (int m = 0; m < b->nmesh; ++m) t += 2 * int64_t(b->mesh_ne[m]) * b->mesh_Np[m];
    *total_dofs = t;
  }
  return TSP_OK;
}

int tsp_batch_estimate_lmax(tsp_batch* b, int32_t iters, double* lmax) {
  if (!b || !lmax || iters < 1) return TSP_ERR_ARG;
  cudaSetDevice(b->device);
  for (size_t g = 0; g < b->groups.size(); ++g) {
    tsp_handle* h = b->groups[g];
    const int nm = h->nmesh;
    const size_t n1 = size_t(h->ne) * h->R;
    double *da = nullptr, *db = nullptr;
    int rc;
    if ((rc = dalloc(h, &da, n1)) || (rc = dalloc(h, &db, n1))) return bfail(b, rc, h->err);
    std::vector<double> x0(n1);
    uint64_t st = 0x9E3779B97F4A7C15ull;
    for (size_t i = 0; i < n1; ++i) {
      st ^= st << 13;
      st ^= st >> 7;
      st ^= st << 17;
      x0[i] = double(st >> 11) * (1.0 / 9007199254740992.0) - 0.5;
    }
    if (copy_sync(da, x0.data(), n1 * sizeof(double), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
      return bfail(b, TSP_ERR_CUDA, "upload of the start vector failed");
    std::vector<double> scale(nm, 1.0), acc(3 * size_t(nm)), lam(nm, 0.0);
    for (int it = 0; it < iters; ++it) {
      if (cudaMemcpyAsync(h->d_xscale_mesh, scale.data(), nm * sizeof(double), cudaMemcpyHostToDevice, h->stream) !=
              cudaSuccess ||
          cudaMemsetAsync(h->d_acc, 0, 3 * size_t(nm) * sizeof(double), h->stream) != cudaSuccess)
        return bfail(b, TSP_ERR_CUDA, "power iteration setup failed");
      if ((rc = launch_step(h, tsp::kModePower, da, nullptr, db, 0, 1.0, h->stream))) return bfail(b, rc, h->err);
      if (cudaMemcpyAsync(acc.data(), h->d_acc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream) !=
              cudaSuccess ||
          cudaStreamSynchronize(h->stream) != cudaSuccess)
        return bfail(b, TSP_ERR_CUDA, std::string("power iteration: ") + cudaGetErrorString(cudaGetLastError()));
      for (int q = 0; q < nm; ++q) {
        lam[q] = acc[3 * q] / acc[3 * q + 1];
        scale[q] = acc[3 * q + 2] > 0 ? 1.0 / std::sqrt(acc[3 * q + 2]) : 1.0;
      }
      std::swap(da, db);
    }
    for (int q = 0; q < nm; ++q) lmax[b->group_meshes[g][q]] = lam[q];
    dfree(h, da);
    dfree(h, db);
  }
  return TSP_OK;
}

int tsp_batch_set_dt(tsp_batch* b, const double* dt) {
  if (!b || !dt) return TSP_ERR_ARG;
  for (int m = 0; m < b->nmesh; ++m)
    if (!(dt[m] > 0) || !std::isfinite(dt[m])) return bfail(b, TSP_ERR_ARG, "dt must be positive and finite");
  cudaSetDevice(b->device);
  for (size_t g = 0; g < b->groups.size(); ++g) {
    tsp_handle* h = b->groups[g];
    std::vector<double> de(h->ne);
    for (int q = 0; q < h->nmesh; ++q) {
      const int m = b->group_meshes[g][q];
      for (int e = 0; e < b->mesh_ne[m]; ++e) de[b->mesh_first[m] + e] = dt[m];
    }
    if (copy_sync(h->d_dt_elem, de.data(), de.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
      return bfail(b, TSP_ERR_CUDA, "dt upload failed");
    h->dt = dt[b->group_meshes[g][0]];  // the handle's own dt is unused by its kernels
    h->dt_set = true;
    clear_graphs(h);
  }
  batch_clear_graphs(b);
  return TSP_OK;
}

int tsp_batch_set_ricker(tsp_batch* b, const double* dt, const double* f0, const double* t0, const double* amp,
                         const int32_t* dir, int64_t n) {
  if (!b || !dt || !f0 || !t0 || !amp || !dir || n < 1) return TSP_ERR_ARG;
  cudaSetDevice(b->device);
  for (size_t g = 0; g < b->groups.size(); ++g) {
    tsp_handle* h = b->groups[g];
    // Source rows are the group's meshes in order: a [nmesh][n][2] table.
    std::vector<double> F(size_t(h->nmesh) * n * 2, 0.0), ts(n);
    for (int q = 0; q < h->nmesh; ++q) {
      const int m = b->group_meshes[g][q];
      if (dir[m] != 0 && dir[m] != 1) return bfail(b, TSP_ERR_ARG, "direction must be 0 or 1");
      tsp::force_times(dt[m], n, ts.data());
      for (int64_t k = 0; k < n; ++k) F[(size_t(q) * n + k) * 2 + dir[m]] = tsp::ricker(ts[k], f0[m], t0[m], amp[m]);
    }
    dfree(h, h->d_F);
    h->d_F = nullptr;
    h->nF = n;
    h->Fhost = F;
    int rc;
    if ((rc = upload(h, &h->d_F, F.data(), F.size()))) return bfail(b, rc, h->err);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bfail(b, TSP_ERR_CUDA, "force upload failed");
    clear_graphs(h);
  }
  batch_clear_graphs(b);
  return TSP_OK;
}

int tsp_batch_set_seismogram_capacity(tsp_batch* b, int64_t nsteps) {
  if (!b || nsteps < 1) return TSP_ERR_ARG;
  for (tsp_handle* h : b->groups) {
    int rc = tsp_set_seismogram_capacity(h, nsteps);
    if (rc) return bfail(b, rc, h->err);
  }
  batch_clear_graphs(b);
  return TSP_OK;
}

int tsp_batch_first_step(tsp_batch* b) {
  if (!b) return TSP_ERR_ARG;
  for (tsp_handle* h : b->groups) {
    int rc;
    if ((rc = tsp_set_initial(h, 0, nullptr, nullptr))) return bfail(b, rc, h->err);
    if ((rc = tsp_first_step(h))) return bfail(b, rc, h->err);
  }
  for (tsp_handle* h : b->groups)
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bfail(b, TSP_ERR_CUDA, "first step failed");
  return TSP_OK;
}

// All groups' steps in one graph, replayed on the batch stream.
int tsp_batch_run(tsp_batch* b, int64_t nsteps) {
  NvtxRange nvtx_("tsp_batch_run");
  if (!b || nsteps < 0) return TSP_ERR_ARG;
  if (nsteps == 0) return TSP_OK;
  cudaSetDevice(b->device);
  for (tsp_handle* h : b->groups) {
    if (h->steps_done < 1) return bfail(b, TSP_ERR_STATE, "run before first_step");
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bfail(b, TSP_ERR_CUDA, "group stream failed");
  }
  // Key: step count and the parity of every group's current level.
  long long key = nsteps * 2 + b->groups[0]->cur;
  auto it = b->graphs.find(key);
  if (it == b->graphs.end()) {
    cudaGraph_t graph;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return bfail(b, TSP_ERR_CUDA, "batch graph capture failed to start");
    int lrc = TSP_OK;
    for (int64_t i = 0; i < nsteps && lrc == TSP_OK; ++i)
      for (tsp_handle* h : b->groups) {
        const int c = (h->cur + int(i & 1)) & 1;
        lrc = launch_step(h, tsp::kModeStep, h->d_U[c], h->d_U[1 - c], h->d_U[1 - c], int(i), 1.0, b->stream);
        if (lrc) break;
      }
    for (tsp_handle* h : b->groups) tsp::k_advance<<<1, 1, 0, b->stream>>>(h->d_step, nsteps);
    cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
    if (lrc) return bfail(b, lrc, "batch capture: kernel launch failed");
    if (ce != cudaSuccess) return bfail(b, TSP_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(ce));
    cudaGraphExec_t exec;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return bfail(b, TSP_ERR_CUDA, std::string("batch instantiate: ") + cudaGetErrorString(ce));
    it = b->graphs.emplace(key, exec).first;
  }
  if (cudaGraphLaunch(it->second, b->stream) != cudaSuccess) return bfail(b, TSP_ERR_CUDA, "batch graph launch failed");
  for (tsp_handle* h : b->groups) {
    if (nsteps & 1) h->cur = 1 - h->cur;
    h->steps_done += nsteps;
  }
  return TSP_OK;
}

int tsp_batch_run_timed(tsp_batch* b, int64_t nsteps, double* ms) {
  if (!b || !ms) return TSP_ERR_ARG;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, b->stream);
  int rc = tsp_batch_run(b, nsteps);
  float f = 0.f;
  if (rc == TSP_OK) {
    cudaEventRecord(e1, b->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&f, e0, e1) != cudaSuccess)
      rc = bfail(b, TSP_ERR_CUDA, "batch timing failed");
  }
  *ms = f;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

int tsp_batch_get_u(tsp_batch* b, int32_t mesh, double* out) {
  if (!b || !out || mesh < 0 || mesh >= b->nmesh) return TSP_ERR_ARG;
  tsp_handle* h = b->groups[b->mesh_group[mesh]];
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  const int Np = h->Np, R = h->R, ne = b->mesh_ne[mesh];
  std::vector<double> v(size_t(ne) * R);
  if (copy_sync(v.data(), h->d_U[h->cur] + size_t(b->mesh_first[mesh]) * R, v.size() * sizeof(double),
                cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
    return bfail(b, TSP_ERR_CUDA, "state read-back failed");
  for (int e = 0; e < ne; ++e)
    for (int c = 0; c < 2; ++c)
      std::memcpy(out + size_t(c) * ne * Np + size_t(e) * Np, &v[size_t(e) * R + size_t(c) * Np], Np * sizeof(double));
  return TSP_OK;
}

int tsp_batch_get_seismograms(tsp_batch* b, int32_t mesh, int64_t k0, int64_t nk, double* out) {
  if (!b || mesh < 0 || mesh >= b->nmesh || k0 < 0 || nk < 0 || (nk > 0 && !out)) return TSP_ERR_ARG;
  tsp_handle* h = b->groups[b->mesh_group[mesh]];
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  const int nr = b->mesh_nrcv[mesh], r0 = b->mesh_rcv0[mesh];
  if (nr == 0 || nk == 0) return TSP_OK;
  if (nk > h->seis_cap) return bfail(b, TSP_ERR_ARG, "range longer than the seismogram capacity");
  std::vector<double> all(size_t(nk) * h->nrcv * 2);
  int rc = tsp_get_seismograms(h, k0, nk, all.data());
  if (rc) return bfail(b, rc, h->err);
  for (int64_t k = 0; k < nk; ++k)
    std::memcpy(out + size_t(k) * nr * 2, &all[(size_t(k) * h->nrcv + r0) * 2], size_t(nr) * 2 * sizeof(double));
  return TSP_OK;
}

}  // extern "C"
