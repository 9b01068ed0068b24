/*
 * tspeed_b200 C-ABI: B200 (sm_100a) engine for tspeed's explicit leap-frog
 * time loop.
 *
 * The reference (carlomr/tspeed) exposes this path only as the header-only
 * C++ class LeapFrog : TimeAdvance (lib/include/TimeAdvance.hpp:123-256),
 * built from a Mesh, an FESpace<N>, Parameters, Receivers and a Force. This
 * library is the thin, exception-free, plain-pointer boundary under a C++
 * class of the same surface (include/tspeed_gpu.hpp). Each entry point below
 * names the reference member it replaces.
 *
 * Conventions
 *   - Every function returns an int status (tsp_status); 0 is success. Errors
 *     never exit the process (the reference calls exit(), e.g. Mesh.cpp:184,
 *     MyMat.cpp:40, Receivers_imp.hpp:50); the message of the last failure is
 *     available from tsp_last_error().
 *   - Host arrays are caller-owned and copied at call time. Device memory is
 *     library-owned. One handle = one CUDA stream on one device; a handle is
 *     not thread-safe (the reference is single-threaded).
 *   - Displacement vectors on the host use the reference's layout
 *     u[c*ne*Np + e*Np + i] (component c in {0,1}, element e, mode i;
 *     FESpace_imp.hpp:152-153). On the device the library keeps an
 *     element-major, shot-interleaved layout.
 *   - tsp_first_step, tsp_step and tsp_run allocate no device memory;
 *     tsp_run splits a run into pieces of 256 steps and the powers of two of
 *     the remainder, each a CUDA graph instantiated the first time its length
 *     (per parity of the current level) is met and replayed afterwards: at
 *     most 18 graphs per handle, whatever step counts are asked for.
 */
#ifndef TSPEED_B200_H
#define TSPEED_B200_H 1

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TSP_ABI_VERSION 1

typedef struct tsp_handle tsp_handle;

typedef enum {
  TSP_OK = 0,
  TSP_ERR_ARG = -1,         /* invalid argument */
  TSP_ERR_CUDA = -2,        /* CUDA runtime error */
  TSP_ERR_NOMEM = -3,       /* device or host allocation failed */
  TSP_ERR_STATE = -4,       /* call out of order (e.g. step before first_step) */
  TSP_ERR_NOT_FOUND = -5,   /* source/receiver point outside the mesh */
  TSP_ERR_MESH = -6,        /* malformed mesh (clockwise triangle, non-manifold edge, bad file) */
  TSP_ERR_NONFINITE = -7,   /* NaN/Inf detected in the state */
  TSP_ERR_TIMEOUT = -8,     /* a bounded device-side wait gave up */
  TSP_ERR_UNSUPPORTED = -9, /* option not built for this degree/precision */
  TSP_ERR_INDEX = -10       /* checked build: a kernel read a gather index out of range */
} tsp_status;

/* Storage of the operator blocks. The state, the recurrence, M^-1 and the
 * receivers always stay in FP64. */
typedef enum {
  TSP_PREC_FP64 = 0,  /* plain drop-in: FP64 blocks, FP64 accumulation */
  TSP_PREC_FP32 = 1,  /* FP32 blocks, FP32 accumulation */
  TSP_PREC_BF16 = 2   /* BF16 blocks with one FP32 scale per block, FP32 accumulation */
} tsp_precision;

typedef enum {
  TSP_OP_EXPLICIT = 0,    /* assembled 2Np x 2Np blocks in HBM */
  TSP_OP_MATRIX_FREE = 1  /* blocks rebuilt on the fly from reference-element matrices */
} tsp_operator_kind;

/* Modal basis of the space (ShapeFunctions.hpp): the orthonormal Dubiner<N>
 * (FESpace<N> default) or the non-orthonormal BoundaryAdapted<N>
 * (FESpace<N, Dunavant<2N>, BoundaryAdapted<N>>, Examples/src/Lamb.cpp:26),
 * whose reference mass M_ref = L L^T is dense; the per-element inverse mass
 * is then M_ref^-1 / (rho_e detJ_e) (Matrices_imp.hpp:187-189). The device
 * advances w = L^T u with the operator L^-1 B L^-T, where the mass is again
 * diagonal, so every kernel and precision runs unchanged; every host vector
 * in and out of the library stays in the reference's coefficients u. Both
 * bases span P_N. */
typedef enum {
  TSP_BASIS_DUBINER = 0,
  TSP_BASIS_BOUNDARY_ADAPTED = 1
} tsp_basis;

/*
 * A simulation set up as the reference does it: mesh (Mesh.hpp:47), degree N
 * of FESpace<N> with the default Gauss<N+1> rule and Dubiner<N> basis
 * (FESpace.hpp:37), per-element Lame parameters and density (Parameters,
 * FESpace.hpp:194-247), one point source per shot (PointWiseForce,
 * Force.hpp:56-86) and receivers shared by all shots (Receivers,
 * Receivers.hpp:77-121). The operator B = penalty*N^2*S + I + A
 * (TimeAdvance_imp.hpp:32) is assembled on the device.
 */
typedef struct {
  int32_t nverts;
  const double* xy;       /* [nverts][2] */
  int32_t ne;
  const int32_t* tri;     /* [ne][3] 0-based vertex ids, counter-clockwise */
  int32_t N;              /* polynomial degree, 1..8 */
  const double* lambda;   /* [ne] */
  const double* mu;       /* [ne] */
  const double* rho;      /* [ne] */
  double penalty;         /* c of the c*N^2*S penalty term (reference default 2) */
  int32_t precision;      /* tsp_precision */
  int32_t op_kind;        /* tsp_operator_kind */
  int32_t nshots;         /* >= 1 */
  const double* src_xy;   /* [nshots][2] source points */
  int32_t nrcv;           /* >= 0 */
  const double* rcv_xy;   /* [nrcv][2] receiver points */
  int32_t device;         /* CUDA device ordinal */
  int32_t basis;          /* tsp_basis; 0 (Dubiner) when zero-initialised.
                             BoundaryAdapted: explicit operator only (no
                             matrix-free operator, no multi-mesh batches) */
} tsp_problem;

/*
 * A simulation whose operator was assembled elsewhere (e.g. by the
 * reference's Matrices, TimeAdvance.hpp:56-119): block-CSR pattern of MyMat
 * (MyMat.cpp:128-154, diagonal block first), FP64 blocks in merged component
 * layout blocks[b][m*Np+i][n*Np+j] = B^{mn}(row, col[b])_{ij}, and the
 * inverse-mass scalars minv[e] = 1/(rho_e detJ_e) (Matrices_imp.hpp:187,189).
 */
typedef struct {
  int32_t ne;
  int32_t Np;
  int32_t nnzb;
  const int32_t* row_ptr;  /* [ne+1] */
  const int32_t* col;      /* [nnzb] */
  const double* blocks;    /* [nnzb][2Np][2Np] row-major */
  const double* minv;      /* [ne] */
  int32_t precision;       /* tsp_precision */
  int32_t nshots;
  const int32_t* src_elem; /* [nshots] */
  const double* src_phi;   /* [nshots][Np] basis values at the source point */
  int32_t nrcv;
  const int32_t* rcv_elem; /* [nrcv] */
  const double* rcv_phi;   /* [nrcv][Np] */
  int32_t device;
  /* NULL for an orthonormal basis. Else the reference inverse mass
   * M_ref^-1 [Np][Np] (FESpace::base_invmass, FESpace.hpp:163): the inverse
   * mass of element e is minv[e] * M_ref^-1 (Matrices_imp.hpp:187-189). */
  const double* ref_invmass;
} tsp_block_problem;

/* Library version and build information ("tspeed_b200 <ver> sm_100a"). */
const char* tsp_version(void);

/* Constructor: replaces LeapFrog(Xh, p, r) (TimeAdvance_imp.hpp:29-33) plus
 * the Receivers / PointWiseForce constructors. Locates sources and receivers
 * (first containing element, Receivers_imp.hpp:34-51) and assembles B. */
int tsp_create(const tsp_problem* prob, tsp_handle** out);

/* Constructor from an externally assembled operator. */
int tsp_create_from_blocks(const tsp_block_problem* prob, tsp_handle** out);

/* Releases every resource of the handle. NULL is accepted. */
int tsp_destroy(tsp_handle* h);

/* Self-test of the bounded wait used by the warp-specialised kernels (no
 * counterpart in the reference): a kernel waits on a barrier phase that
 * nothing completes; the wait gives up after about a second, raises the
 * kernel's abort flag and the kernel ends normally. Expected: *completed = 0,
 * *abort_raised = 1, TSP_OK, and the device stays usable. */
int tsp_selftest_bounded_wait(int32_t device, int32_t* completed, int32_t* abort_raised);

/* FP64 tensor-core (DMMA) throughput of a device in TFLOP/s, measured by a
 * register-only loop of a few milliseconds: the FP64 roofline denominator
 * that bench.py reports (no counterpart in the reference). */
int tsp_fp64_tensor_peak(int32_t device, double* tflops);

/* Device memory of all handles comes from one stream-ordered pool per
 * device that keeps freed memory cached for the process, so creating a
 * simulation after destroying another does not pay for multi-GB device
 * allocations again. This returns the cached memory of a device to the
 * driver (after a device synchronisation). */
int tsp_release_cached_memory(int32_t device);

/* Message of the last failing call on this handle (or of the last failing
 * create, when h is NULL). Never NULL. */
const char* tsp_last_error(const tsp_handle* h);

/* Problem sizes: ne, Np, nshots, nrcv, nnzb (NULL pointers are skipped). */
int tsp_get_sizes(const tsp_handle* h, int32_t* ne, int32_t* Np, int32_t* nshots, int32_t* nrcv, int64_t* nnzb);

/* TimeAdvance::set_dt (TimeAdvance.hpp:153). */
int tsp_set_dt(tsp_handle* h, double dt);

/* Force of one shot as a table over leap-frog steps: F[k] = (Fx, Fy) at the
 * time step k evaluates (k = 0: first_step at t = 0, TimeAdvance.cpp:28;
 * k >= 1: t = t_{k-1} + dt accumulated in double, TimeAdvance.cpp:46). Steps
 * past n use a zero force. Replaces add_force (TimeAdvance.hpp:171) with a
 * PointWiseForce of the given time function (Force.cpp:22-30). */
int tsp_set_force_table(tsp_handle* h, int32_t shot, const double* F, int64_t n);

/* Convenience: the same table for a Ricker wavelet
 * F_dir(t) = amp*(1 - 2 pi^2 f0^2 (t-t0)^2) exp(-pi^2 f0^2 (t-t0)^2)
 * (Examples/src/Lamb.cpp:37), direction 0 (x) or 1 (y), n steps. Requires dt. */
int tsp_set_ricker(tsp_handle* h, int32_t shot, double f0, double t0, double amp, int32_t direction, int64_t n);

/* Force evaluation times of steps 0..n-1 for a given dt (see above). */
int tsp_force_times(double dt, int64_t n, double* out);

/* set_initial_u / set_initial_v (TimeAdvance.hpp:179-188): modal
 * coefficients of u0 and v0 for one shot, reference layout; NULL = zero.
 * Resets the step counter. */
int tsp_set_initial(tsp_handle* h, int32_t shot, const double* u0, const double* v0);

/* LeapFrog::first_step (TimeAdvance.cpp:24-39). */
int tsp_first_step(tsp_handle* h);

/* LeapFrog::step (TimeAdvance.cpp:41-59), once. */
int tsp_step(tsp_handle* h);

/* nsteps calls of LeapFrog::step, replayed from cached CUDA graphs (pieces
 * of at most 256 steps). Asynchronous: returns once the work is queued on the
 * handle's stream. */
int tsp_run(tsp_handle* h, int64_t nsteps);

/* tsp_run with CUDA events recorded on the handle's stream around the graph
 * replay; synchronises and returns the device time in milliseconds. Returns
 * TSP_ERR_NONFINITE if any step since the initial values (or the resumed
 * state) were set wrote a NaN or infinite displacement: every step kernel
 * raises a device flag then (the reference has no such check; its Eigen loop
 * carries NaNs on silently). */
int tsp_run_timed(tsp_handle* h, int64_t nsteps, double* ms);

/* Kernel variant of the batched step chosen for this handle by the
 * autotuner at creation (or forced by TSP_BATCHED_VARIANT). FP32 operator:
 * 7 and 8 warp-specialised CUDA-core kernel with bulk-copy rings and
 * 8-shot register tiles (6 or 8 FMA warps per SM), 0 K-split /
 * pipelined CUDA-core kernel, 1 pipelined CUDA-core kernel, 2 non-persistent
 * CUDA-core kernel, 4 tensor-core fixed-point kernel. FP64
 * operator with several shots: 5 warp-specialised FP64 tensor-core (DMMA)
 * kernel with two consumer groups of 8 warps (8 shots x all rows per warp),
 * 13 the same tiles with u^{k-1} requested before the products (a
 * warpgroup register split gives the registers), 6 the same kernel with one
 * group of 16 warps (8 shots x half the rows) and an epilogue without load
 * latency, 9 and 10 the epilogue in update warps, 3 single-role DMMA kernel,
 * 2 CUDA-core kernel.
 * No counterpart in the reference (its step is a single CPU path). */
int tsp_get_kernel_variant(const tsp_handle* h, int32_t* variant);

/* 1 if this library is the checked build (libtspeed_b200_checked.so,
 * compiled with TSP_CHECKED), else 0. In the checked build every gather
 * index the step kernels read -- row extents of the block pattern,
 * neighbour ids, source elements, receiver ranges and ids, mesh neighbours
 * of the matrix-free kernel -- is range-checked on the device; an index out
 * of range is replaced by a valid one (no out-of-bounds access) and
 * recorded, and the next read-back or timed run (tsp_run_timed, tsp_get_u,
 * tsp_get_u_all, tsp_get_seismograms, tsp_field_values, tsp_write_field,
 * tsp_l2_error) returns TSP_ERR_INDEX naming the index kind and value. Results are then void. No counterpart
 * in the reference (it has no device code; its host checks call exit()). */
int tsp_checked_build(void);

/* Number of leap-frog steps done (first_step counts as 1) and the
 * reference's M_last_time. */
int tsp_get_progress(const tsp_handle* h, int64_t* steps_done, double* last_time);

/* TimeAdvance::u() (TimeAdvance.hpp:202-203) of one shot, reference layout,
 * length 2*ne*Np. Synchronises the handle's stream. */
int tsp_get_u(tsp_handle* h, int32_t shot, double* out);

/* TimeAdvance::u() of every shot at once: out[nshots][2*ne*Np], reference
 * layout (the state is transposed on the device and read back in large
 * transfers; a temporary device buffer of at most 256 MiB is used).
 * Synchronises the handle's stream. */
int tsp_get_u_all(tsp_handle* h, double* out);

/* Receiver samples, taken after every step on the device (the arithmetic of
 * TimeAdvance::eval_receivers, TimeAdvance.cpp:68-79): out[shot][k][r][2]
 * for steps k in [k0, k0+nk). k = 0 is the sample after first_step. */
int tsp_get_seismograms(tsp_handle* h, int64_t k0, int64_t nk, double* out);

/* Capacity of the on-device seismogram buffer, in steps (default 4096);
 * samples of later steps wrap around modulo the capacity. */
int tsp_set_seismogram_capacity(tsp_handle* h, int64_t nsteps);

/* Enables the discrete-energy monitor E^{k} = 1/2|u^{k}-u^{k-1}|_M^2/dt^2 +
 * 1/2 (u^{k})^T B u^{k-1}, summed over shots, recorded per step in FP64. */
int tsp_enable_energy(tsp_handle* h, int32_t on);
int tsp_get_energy(tsp_handle* h, int64_t k0, int64_t nk, double* out);

/* Checkpoint / resume: both leap-frog levels (u^{k-1}, u^{k}) of every
 * shot, reference layout, [nshots][2*ne*Np] each, plus the step counter. */
int tsp_get_state(tsp_handle* h, double* u_prev, double* u_cur, int64_t* steps_done, double* last_time);
int tsp_set_state(tsp_handle* h, const double* u_prev, const double* u_cur, int64_t steps_done, double last_time);

/* NaN/Inf watchdog: sets *bad to 1 if a step kernel has written a non-finite
 * displacement since the initial values were set, or if any value of the
 * current level is not finite. Synchronises the handle's stream. */
int tsp_check_finite(tsp_handle* h, int32_t* bad);

/* One product y = B x with the handle's operator (MyMatMultiDim::vecMult,
 * MyMat.hpp:311-319), reference layout, shot 0. */
int tsp_apply(tsp_handle* h, const double* x, double* y);

/* Largest eigenvalue of M^-1 B by power iteration on the device (the
 * reference has no CFL estimate; dt is a user setting). dt_cfl = 2/sqrt(lmax). */
int tsp_estimate_lmax(tsp_handle* h, int32_t iters, double* lmax);

/* Allocation-free variant of tsp_estimate_lmax. No counterpart in the
 * reference (which has no CFL estimate). For callers that must not allocate
 * device memory when they ask for the estimate (memory pools that forbid raw
 * cudaMalloc, real-time loops, hosts that cap library allocations): the two
 * iteration vectors and the accumulators live in a fixed 32 MiB file-scope
 * device array (4 Mi doubles) that every GPU loading the library holds until
 * exit, so 2*ne*2Np + 3 must not exceed 4,194,304 (TSP_ERR_ARG otherwise).
 * Every call looks up that array's device address in the current context (a
 * host query, so a context reset leaves no stale address behind); the first
 * call on a device may load the library's device code, so make it before any
 * stream capture. All calls share the array and each re-initialises it:
 * calls that overlap on the GPU (several handles, threads or streams at once)
 * race. Multi-mesh groups are rejected (TSP_ERR_UNSUPPORTED). Calls no
 * cudaMalloc/cudaFree. */
int tsp_estimate_lmax_noalloc(tsp_handle* h, int32_t iters, double* lmax);

/* Exports of the assembled operator (explicit handles):
 * row_ptr[ne+1], col[nnzb], blocks[nnzb][2Np][2Np] row-major, minv[ne].
 * Blocks are B as the reference assembles it; for BoundaryAdapted they are
 * recovered as L (L^-1 B L^-T) L^T from the stored operator. */
int tsp_export_operator(tsp_handle* h, int32_t* row_ptr, int32_t* col, double* blocks, double* minv);

/* Basis of the handle (tsp_basis) and its reference inverse mass M_ref^-1
 * [Np][Np] (FESpace::base_invmass; the identity for Dubiner). Either output
 * may be NULL. */
int tsp_get_ref_invmass(const tsp_handle* h, int32_t* basis, double* out);

/* Source and receiver location: elements and basis values. */
int tsp_export_points(tsp_handle* h, int32_t* src_elem, double* src_phi, int32_t* rcv_elem, double* rcv_phi);

/* ---- Multi-mesh batch --------------------------------------------------
 * Many independent simulations of uneven size and degree advanced together
 * (no counterpart in the reference, which runs one LeapFrog per process).
 * Each problem has one source (nshots = 1); all share precision, operator
 * kind and device. Meshes of one degree form one group (a concatenated,
 * block-diagonal-by-mesh system with per-mesh dt and source); every step of
 * every group is replayed from one CUDA graph by tsp_batch_run. */
typedef struct tsp_batch tsp_batch;
int tsp_batch_create(const tsp_problem* meshes, int32_t nmesh, tsp_batch** out);
int tsp_batch_destroy(tsp_batch* b);
const char* tsp_batch_last_error(const tsp_batch* b);
/* Number of degree groups and the total DOFs over all meshes. */
int tsp_batch_info(const tsp_batch* b, int32_t* ngroups, int64_t* total_dofs);
/* Largest eigenvalue of M^-1 B of every mesh (power iteration per mesh). */
int tsp_batch_estimate_lmax(tsp_batch* b, int32_t iters, double* lmax);
/* Per-mesh dt[nmesh] and Ricker sources (arrays of nmesh; see tsp_set_ricker). */
int tsp_batch_set_dt(tsp_batch* b, const double* dt);
int tsp_batch_set_ricker(tsp_batch* b, const double* dt, const double* f0, const double* t0, const double* amp,
                         const int32_t* direction, int64_t n);
int tsp_batch_set_seismogram_capacity(tsp_batch* b, int64_t nsteps);
/* Zero initial state, then LeapFrog::first_step on every mesh. */
int tsp_batch_first_step(tsp_batch* b);
int tsp_batch_run(tsp_batch* b, int64_t nsteps);
int tsp_batch_run_timed(tsp_batch* b, int64_t nsteps, double* ms);
/* One mesh's displacement (reference layout) and seismograms [k][rcv][2]. */
int tsp_batch_get_u(tsp_batch* b, int32_t mesh, double* out);
int tsp_batch_get_seismograms(tsp_batch* b, int32_t mesh, int64_t k0, int64_t nk, double* out);

/* Host-side projection of initial data (FESpace::transform,
 * FESpace_imp.hpp:136-179): the caller evaluates its field at the physical
 * volume quadrature points (collapsed Gauss<N+1> rule, (N+1)^2 points per
 * element) and gets the modal coefficients in the reference layout.
 * pts/fvals are [ne][(N+1)^2][2]; out has 2*ne*Np entries. */
int tsp_quadrature_points(int32_t N, int32_t nverts, const double* xy, int32_t ne, const int32_t* tri, double* pts);
int tsp_project(int32_t N, int32_t nverts, const double* xy, int32_t ne, const int32_t* tri, const double* fvals,
                double* out);
/* The same for a given basis (tsp_basis): uh = M_ref^-1 rhs / detJ
 * (FESpace_imp.hpp:152-153). tsp_project is this with TSP_BASIS_DUBINER. */
int tsp_project_basis(int32_t N, int32_t basis, int32_t nverts, const double* xy, int32_t ne, const int32_t* tri,
                      const double* fvals, double* out);

/* ---- Field output and error norms (FESpace_imp.hpp:70-133) ------------- */
/* FESpace::field_out values of one shot's current displacement: the
 * expansion at the reference points (0.2,0.2), (0.8,0.2), (0.2,0.8),
 * (0.5,0.5) of every element, out[ne][4][2], evaluated on the device. */
int tsp_field_values(tsp_handle* h, int32_t shot, double* out);
/* Writes them as FESpace::field_out(fname, u, step) does: file
 * fname + "u_" + step + ".field", one "valx valy" line per element and point,
 * default iostream number formatting. */
int tsp_write_field(tsp_handle* h, int32_t shot, const char* fname, int64_t step);
/* FESpace::L2error(uex, u) of one shot's current displacement: exact values
 * at the volume quadrature points (tsp_quadrature_points order),
 * exact[ne][(N+1)^2][2]; per-element terms on the device, summed in element
 * order on the host. The rule is the collapsed Gauss<N+1> of FESpace<N>
 * (for BoundaryAdapted the reference integrates with Dunavant<2N>; both are
 * exact for |u_h|^2 but differ for a non-polynomial uex). Needs a handle
 * built from a mesh (TSP_ERR_UNSUPPORTED for tsp_create_from_blocks). */
int tsp_l2_error(tsp_handle* h, int32_t shot, const double* exact, double* err);
/* TimeAdvance::set_initial_u / set_initial_v (TimeAdvance_imp.hpp:42-51) with
 * FESpace::transform on the device: field values at the volume quadrature
 * points (tsp_quadrature_points order), [ne][(N+1)^2][2] each, projected
 * into one shot's initial state (NULL: zero). Resets the step counter like
 * tsp_set_initial. Needs a handle built from a mesh. */
int tsp_set_initial_values(tsp_handle* h, int32_t shot, const double* u_vals, const double* v_vals);
/* FESpace::points_out(fname): the physical positions of the field_out
 * points, one "x y" line per element and point. */
int tsp_points_out(int32_t nverts, const double* xy, int32_t ne, const int32_t* tri, const char* fname);
/* PointWiseEntity::M_add (Receivers_imp.hpp:34-51) for many points: the
 * first (lowest-id) element passing Triangle::intriangle (Geometry.cpp:112-118)
 * and the basis values at the point, elem[npts] (-1: outside the mesh),
 * phi[npts][Np]. tsp_create locates sources and receivers with it. */
int tsp_locate_points(int32_t N, int32_t basis, int32_t nverts, const double* xy, int32_t ne, const int32_t* tri,
                      int32_t npts, const double* pts, int32_t* elem, double* phi);
/* Basis values at reference points (for callers holding u on the host):
 * rpts[npts][2] -> phi[npts][Np] (ShapeFunctions_imp.hpp). */
int tsp_eval_basis(int32_t N, int32_t basis, int32_t npts, const double* rpts, double* phi);
/* The volume rule on the reference triangle (collapsed Gauss<N+1>,
 * QuadratureRule_imp.hpp:101-113): rpts[(N+1)^2][2], w[(N+1)^2]; either may
 * be NULL. */
int tsp_quadrature_rule(int32_t N, double* rpts, double* w);

/* Host-side mesh services (Mesh.cpp). */
/* Gmsh 2.2 ASCII reader (Mesh::Mesh, Mesh.cpp:174-257): counts first
 * (xy/tri/region NULL), then data. region = elementary tag. */
int tsp_gmsh_read(const char* path, int32_t* nverts, double* xy, int32_t* ne, int32_t* tri, int32_t* region);
/* Neighbour tables (Mesh::M_neighbors, Mesh.cpp:33-128) in O(ne):
 * neigh[ne][3] (-1 on the boundary), neighedge[ne][3]. */
int tsp_mesh_neighbours(int32_t ne, const int32_t* tri, int32_t* neigh, int32_t* neighedge);

#ifdef __cplusplus
}
#endif

#endif /* TSPEED_B200_H */
