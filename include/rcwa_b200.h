/*
 * rcwa_b200.h -- C ABI of the B200-native RCWA solve path.
 *
 * The reference (rcwa3d/include/rcwa.hpp, rcwa3d/src/rcwa.cpp) exposes its
 * solver as Eigen-typed C++ free functions sequenced by main()
 * (rcwa3d/src/main.cpp:111-191).  This header replaces that surface with an
 * Eigen-free C ABI: plain pointers and sizes, complex128 as {re, im} pairs
 * (layout-compatible with std::complex<double>), column-major matrices as in
 * Eigen's default (rcwa.hpp:13), and integer return codes instead of abort()
 * (rcwa.cpp:300) or std::out_of_range.
 *
 * Every entry point returns RCWA_OK (0) or a negative RCWA_ERR_* code; the
 * message of the last failure on the calling thread is rcwa_last_error().
 * Numerical trouble inside a solve (singular pivot, eigensolver cap reached,
 * non-finite output, Kz = 0 at a Rayleigh/Wood anomaly) never aborts: it is
 * reported in a per-solve status word and the values are left as computed
 * (Inf/NaN, exactly where the reference would produce them).
 *
 * Host-pointer entry points copy inputs to the GPU and results back; the
 * *_device entry points take device pointers and leave results on the GPU.
 * A context owns one CUDA stream and its workspace; calls on one context are
 * serialised, distinct contexts may be used from distinct threads.
 */
#ifndef RCWA_B200_H
#define RCWA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ------------------------------------------------------- */
#define RCWA_OK 0
#define RCWA_ERR_INVALID (-1)   /* bad argument (null pointer, size, order) */
#define RCWA_ERR_CUDA (-2)      /* CUDA runtime error, see rcwa_last_error() */
#define RCWA_ERR_NOMEM (-3)     /* device allocation failed / over budget */
#define RCWA_ERR_NUMERIC (-4)   /* at least one per-solve status bit is set */
#define RCWA_ERR_BUSY (-5)      /* server queue full (back-pressure) */
#define RCWA_ERR_NOTFOUND (-6)  /* unknown server ticket */

/* ---- per-solve status bits ---------------------------------------------- */
#define RCWA_STATUS_SINGULAR 1u      /* zero pivot in an LU (rcwa.cpp .lu()) */
#define RCWA_STATUS_EIG_NOCONV 2u    /* QR iteration cap hit (rcwa.cpp:300 aborts) */
#define RCWA_STATUS_NONFINITE 4u     /* non-finite R/T */
#define RCWA_STATUS_WOOD_ANOMALY 8u  /* some Kz == 0: division at rcwa.cpp:225,541,560 */
#define RCWA_STATUS_REFINE_SLOW 16u  /* mixed precision: an LU solve's last FP64 refinement
                                        correction stayed above 1e-4 of |X| */

/* ---- precision modes ---------------------------------------------------- */
#define RCWA_PREC_FP64 0   /* all-FP64 (parity form, reproduces the reference) */
#define RCWA_PREC_MIXED 1  /* the stages of rcwa_context_set_mixed (default: the two GEMM stages)
                              in reduced precision; FP64 Omega^2, eig, sqrt, exp and sums */

/* Stages that RCWA_PREC_MIXED runs in reduced precision.  GEMM stages use the
 * int8-sliced tensor-core GEMM for products with m, n, k >= 256 (each row of
 * A and column of B scaled by a power of two and cut into signed 7-bit
 * digits, 5 by default (4 to 6 via rcwa_context_set_mixed), digit products
 * accumulated exactly in int32 by tcgen05 kind::i8, combined in FP64: about
 * 36 bits of every product with 5 digits; smaller products stay on the FP64
 * kernels), or with RCWA_MIXED_GEMM_TF32 the split-TF32
 * GEMM (each FP64 operand split into TF32 hi + lo, three tcgen05 kind::tf32
 * products accumulated in the tensor core's FP32).  LU stages factor and
 * solve in FP32 (complex64) and refine the solution with FP64 residuals
 * R = B - A X computed on the FP64 tensor cores. */
#define RCWA_MIXED_LAYER_GEMM 1u  /* V = Q W / lambda and the layer-assembly products (rcwa.cpp:326-348) */
#define RCWA_MIXED_STAR_GEMM 2u   /* star-product and global-column products (rcwa.cpp:602-611) */
#define RCWA_MIXED_LAYER_LU 4u    /* W^-1, V^-1, A^-1 and D^-1 solves of a layer (rcwa.cpp:335-348) */
#define RCWA_MIXED_STAR_LU 8u     /* star-product and global-column solves (rcwa.cpp:605-611) */
#define RCWA_MIXED_ALL 15u
#define RCWA_MIXED_GEMM_TF32 16u  /* GEMM stages on split-TF32 instead of int8 slices */
#define RCWA_MIXED_REFINE_INT8 32u  /* LU refinement residuals on the int8-slice GEMM instead of FP64 */

typedef struct rcwa_complex {
  double re, im;
} rcwa_complex;

/* Device (rcwa.hpp:48-78).  er/ur are flat [layer][iy][ix] row-major grids
 * (rcwa.hpp:56-60, rcwa.cpp:18), t[layer] the thicknesses. */
typedef struct rcwa_stack {
  int nx, ny, num_layers;
  double lx, ly;
  const rcwa_complex* er;
  const rcwa_complex* ur;
  const double* t;
} rcwa_stack;

/* Source (rcwa.hpp:81-95); k0 = 2*pi/lambda0 is derived (rcwa.hpp:92). */
typedef struct rcwa_source {
  double lambda0, theta, phi, pte, ptm;
} rcwa_source;

/* RCWAParams (rcwa.hpp:98-112).  P = 2*nx_harmonics+1, Q = 2*ny_harmonics+1
 * (rcwa.cpp:56-58); mode index m = ix*Q + iy (rcwa.cpp:63-64). */
typedef struct rcwa_params {
  int nx_harmonics, ny_harmonics;
  rcwa_complex er_ref, ur_ref, er_trn, ur_trn;
} rcwa_params;

/* Results (rcwa.hpp:116-128).  R and T are caller-owned Q x P column-major
 * arrays (Eigen reshaped(Q, P), rcwa.cpp:576, 582). */
typedef struct rcwa_result {
  double* R;
  double* T;
  double R_tot, T_tot;
  uint32_t status;
} rcwa_result;

typedef struct rcwa_context rcwa_context;
typedef struct rcwa_geometry rcwa_geometry;
typedef struct rcwa_server rcwa_server;

/* Layer descriptions for the device-side rasterisers (the reference fills
 * host grids in main.cpp:48-91).  Coordinates are relative to the cell
 * centre; shapes are painted in order over the background, cells sampled at
 * their centres (i + 0.5) L / n. */
#define RCWA_SHAPE_CIRCLE 1    /* disc of radius a centred at (cx, cy) */
#define RCWA_SHAPE_RECT 2      /* a x b rectangle centred at (cx, cy) */
#define RCWA_SHAPE_LINES 3     /* lines along y, width a, centred at x = cx */
#define RCWA_SHAPE_TRIANGLE 4  /* the reference demo's triangle (main.cpp:51-71): apex up, base = height = a */
typedef struct rcwa_shape {
  int kind;
  double cx, cy, a, b;
  rcwa_complex eps, mu;
} rcwa_shape;
typedef struct rcwa_layer_shapes {
  rcwa_complex eps_bg, mu_bg;
  double t;
  int n_shapes;
  const rcwa_shape* shapes;
} rcwa_layer_shapes;

/* ---- context ------------------------------------------------------------ */
const char* rcwa_last_error(void);
int rcwa_version(void);
int rcwa_context_create(int device, rcwa_context** out);
int rcwa_context_destroy(rcwa_context* ctx);
/* Use an external cudaStream_t (NULL restores the context's own stream). */
int rcwa_context_set_stream(rcwa_context* ctx, void* cuda_stream);
int rcwa_context_synchronize(rcwa_context* ctx);
/* Kernels launched by this context since creation (instrumentation). */
int rcwa_context_kernel_launches(rcwa_context* ctx, uint64_t* count);
/* Mixed-precision set-up of this context (no reference counterpart: the
 * reference is FP64 only): the RCWA_MIXED_* stages that RCWA_PREC_MIXED runs
 * in reduced precision (default RCWA_MIXED_LAYER_GEMM | RCWA_MIXED_STAR_GEMM:
 * on B200 the FP32 LU with an FP64 residual per sweep costs more than the FP64
 * LU it replaces; 0 makes RCWA_PREC_MIXED an FP64 solve), the FP64
 * refinement sweeps of its LU solves (1..4, default 1)
 * and the 7-bit digits per operand of the int8-slice GEMM (4, 5 or 6,
 * default 5: about 29, 36 or 43 bits of each product).  Sweeps and batches
 * run through the context use it. */
int rcwa_context_set_mixed(rcwa_context* ctx, unsigned stages, int refine_sweeps, int gemm_digits);

/* ---- instrumentation (no reference counterpart: the reference only prints
 * to stdout, rcwa.cpp:92-156).  When enabled, the hot kernel families
 * ("zgemm", "hess", "formq", "schur", "trevc", "lu_panel") are bracketed by
 * CUDA events on their launching stream; query returns summed device time,
 * launch count and the algorithmic flops of those launches. */
int rcwa_profile_enable(int on);
int rcwa_profile_reset(void);
int rcwa_profile_query(const char* name, double* total_ms, uint64_t* launches, double* flops);

/* ---- end-to-end solve (main.cpp:111-191) -------------------------------- */
/* One source. */
int rcwa_solve(rcwa_context* ctx, const rcwa_stack* stack, const rcwa_source* source,
               const rcwa_params* params, int precision, rcwa_result* out);
/* Many sources on one stack (wavelength / angle / polarisation sweep), batched
 * on the GPU.  out[i] receives source i. */
int rcwa_solve_sweep(rcwa_context* ctx, const rcwa_stack* stack, const rcwa_source* sources,
                     int n_sources, const rcwa_params* params, int precision,
                     rcwa_result* out);

/* Geometry handle: the per-layer convolution matrices (main.cpp:125-138,
 * rcwa.cpp:6-82) built once on the device and reused by every source.  With
 * stack_on_device != 0 the stack's er/ur/t pointers are device pointers.
 * Its device memory comes from the stream-ordered pool on the context's
 * stream: use a geometry only with the context that created it. */
int rcwa_geometry_create(rcwa_context* ctx, const rcwa_stack* stack, const rcwa_params* params,
                         int stack_on_device, rcwa_geometry** out);
/* rcwa_geometry_create with option flags (0 = rcwa_geometry_create).
 * RCWA_GEOM_LI_RULE: Li's factorization rule for crossed gratings (J. Opt.
 * Soc. Am. A 14, 2758 (1997)) in place of the reference's Laurent rule where
 * eps / mu multiply the in-plane field components (Q_i: E_x, E_y; P_i: H_x,
 * H_y of rcwa.cpp:273-285): eps_xx = [[ [[eps]]_x ]]_y, the inverse of the 1-D
 * Toeplitz matrix of 1/eps along every grid row, convolved along y, and
 * eps_yy with the axes swapped.  erc^-1 / urc^-1 (rcwa.cpp:267-281) keep the
 * Laurent rule.  Converges much faster for TM light on high-contrast and
 * metallic lamellar gratings; the reference has no such option, so its
 * results differ by the truncation error.  Returns RCWA_ERR_NUMERIC if a grid
 * value is 0 or a line's 1/eps Toeplitz matrix is singular. */
#define RCWA_GEOM_LI_RULE 1u
int rcwa_geometry_create_ex(rcwa_context* ctx, const rcwa_stack* stack, const rcwa_params* params,
                            int stack_on_device, unsigned flags, rcwa_geometry** out);
/* Releases the geometry in stream order on its context's stream (work already
 * enqueued that reads it completes first); does not block the host. */
int rcwa_geometry_destroy(rcwa_geometry* geom);
/* Sweep on a prepared geometry.  sources: host array.  R_dev/T_dev: device
 * arrays [n_sources][Q*P]; tot_dev: device [n_sources][2] (R_tot, T_tot);
 * status_dev: device uint32 [n_sources].  Asynchronous on the context stream. */
int rcwa_solve_sweep_device(rcwa_context* ctx, const rcwa_geometry* geom,
                            const rcwa_source* sources, int n_sources, int precision,
                            double* R_dev, double* T_dev, double* tot_dev,
                            uint32_t* status_dev);

/* Device-side rasterisers.  rcwa_rasterize writes the er/ur grids of nl
 * layers ([layer][iy][ix], device pointers) and, if t_dev is not NULL, the
 * thicknesses; asynchronous on the context stream.  The grids equal the
 * host builders' of rcwa_b200.configs bit for bit.
 * rcwa_geometry_create_shapes rasterises into temporary device grids and
 * builds the geometry from them (no host grids at all). */
int rcwa_rasterize(rcwa_context* ctx, int nx, int ny, double lx, double ly, int nl,
                   const rcwa_layer_shapes* layers, rcwa_complex* er_dev, rcwa_complex* ur_dev,
                   double* t_dev);
int rcwa_geometry_create_shapes(rcwa_context* ctx, int nx, int ny, double lx, double ly, int nl,
                                const rcwa_layer_shapes* layers, const rcwa_params* params,
                                rcwa_geometry** out);

/* ---- batches and serving ------------------------------------------------
 * The reference solves one problem per call (main.cpp:111-191); these run
 * many unrelated problems together.  Problems of equal shape (harmonic
 * orders, layer count, grid size, port media, which layers are uniform) are
 * solved as one batched GPU solve. */
/* n problems: stacks[i], sources[i], params[i]; out[i] receives problem i.
 * Returns RCWA_ERR_NUMERIC when any out[i].status is nonzero. */
int rcwa_solve_batch(rcwa_context* ctx, int n, const rcwa_stack* stacks,
                     const rcwa_source* sources, const rcwa_params* params, int precision,
                     rcwa_result* out);
/* Serving loop (continuous batching): `lanes` worker threads on `device`,
 * each with its own context (stream and workspace).  A free lane admits
 * queued requests in arrival order -- up to max_batch, up to its share of the
 * device-memory budget (hbm_budget_bytes / lanes), and only while all
 * requests in flight stay within the budget -- and solves them as one
 * batched solve (rcwa_solve_batch) on its stream, so batches of different
 * lanes overlap on the GPU and a request arriving during a long batch starts
 * on the next free lane.  A request that does not fit waits (later, smaller
 * ones may pass it during up to 8 admission rounds); one larger than the
 * whole budget runs alone.  At most max_queue requests wait at a time (RCWA_ERR_BUSY beyond). */
typedef struct rcwa_server_config {
  int max_batch;              /* requests per batched solve of a lane (> 0) */
  int max_queue;              /* waiting requests before RCWA_ERR_BUSY (> 0) */
  int precision;              /* RCWA_PREC_FP64 or RCWA_PREC_MIXED */
  int lanes;                  /* concurrent batches, 1..16 (0: 2) */
  uint64_t hbm_budget_bytes;  /* in-flight footprint limit (0: min(180 GB, 85 % of free memory)) */
  unsigned mixed_stages;      /* as rcwa_context_set_mixed (0: its defaults) */
  int refine_sweeps;
  int gemm_digits;
} rcwa_server_config;
int rcwa_server_create_ex(int device, const rcwa_server_config* cfg, rcwa_server** out);
/* rcwa_server_create_ex with lanes, budget and mixed settings at their defaults. */
int rcwa_server_create(int device, int max_batch, int max_queue, int precision,
                       rcwa_server** out);
/* Queues one request; the stack's arrays are copied (the caller may free them
 * on return).  RCWA_ERR_BUSY when max_queue requests are waiting. */
int rcwa_server_submit(rcwa_server* srv, const rcwa_stack* stack, const rcwa_source* source,
                       const rcwa_params* params, uint64_t* ticket);
/* *done = 1 once the request finished (wait != 0 blocks until then); out
 * (optional; R/T caller arrays of Q*P doubles, each may be NULL) receives the
 * result and the ticket is released.  Returns the request's own code once
 * done; RCWA_ERR_NOTFOUND for an unknown or already collected ticket. */
int rcwa_server_poll(rcwa_server* srv, uint64_t ticket, int wait, rcwa_result* out, int* done);
/* Completed requests and their submit-to-completion latency p50 / p99 (ms,
 * over the last 65536 completions). */
int rcwa_server_stats(rcwa_server* srv, uint64_t* completed, double* p50_ms, double* p99_ms);
typedef struct rcwa_server_info {
  uint64_t completed, queued, in_flight, rejected;  /* rejected: RCWA_ERR_BUSY submissions */
  double p50_ms, p99_ms;
  uint64_t admitted_bytes, peak_admitted_bytes, budget_bytes;
  int lanes;
} rcwa_server_info;
int rcwa_server_info_get(rcwa_server* srv, rcwa_server_info* out);
/* Finishes the queued requests, stops the worker, releases the context. */
int rcwa_server_destroy(rcwa_server* srv);

/* ---- step-level entry points (host pointers; one per reference function) */
/* ConvMat, rcwa.cpp:6-82: out is PQ x PQ column-major. */
int rcwa_convmat(rcwa_context* ctx, const rcwa_complex* field, int layer, int nx, int ny,
                 int nx_harmonics, int ny_harmonics, rcwa_complex* out);
/* ComputeWaveVectors, rcwa.cpp:85-160: k_inc[3], Kx/Ky/Kz_ref/Kz_trn[PQ]. */
int rcwa_wave_vectors(rcwa_context* ctx, double lx, double ly, const rcwa_source* source,
                      const rcwa_params* params, rcwa_complex* k_inc, rcwa_complex* Kx,
                      rcwa_complex* Ky, rcwa_complex* Kz_ref, rcwa_complex* Kz_trn);
/* GapMedium, rcwa.cpp:163-234: W0, V0 are 2PQ x 2PQ. */
int rcwa_gap_medium(rcwa_context* ctx, int pq, const rcwa_complex* Kx, const rcwa_complex* Ky,
                    rcwa_complex* W0, rcwa_complex* V0);
/* SMatrixLayer, rcwa.cpp:254-352 (S21 = S12, S22 = S11, rcwa.cpp:351). */
int rcwa_smatrix_layer(rcwa_context* ctx, int pq, const rcwa_complex* erc, const rcwa_complex* urc,
                       const rcwa_complex* Kx, const rcwa_complex* Ky, const rcwa_complex* V0,
                       double k0, double thickness, rcwa_complex* S11, rcwa_complex* S12,
                       uint32_t* status);
/* SMatrixReflection / SMatrixTransmission, rcwa.cpp:354-466 (W_ref = W_trn = I). */
int rcwa_smatrix_reflection(rcwa_context* ctx, const rcwa_params* params, const rcwa_complex* Kx,
                            const rcwa_complex* Ky, const rcwa_complex* Kz_ref,
                            const rcwa_complex* V0, rcwa_complex* S11, rcwa_complex* S12,
                            rcwa_complex* S21, rcwa_complex* S22);
int rcwa_smatrix_transmission(rcwa_context* ctx, const rcwa_params* params, const rcwa_complex* Kx,
                              const rcwa_complex* Ky, const rcwa_complex* Kz_trn,
                              const rcwa_complex* V0, rcwa_complex* S11, rcwa_complex* S12,
                              rcwa_complex* S21, rcwa_complex* S22);
/* RedhefferProduct, rcwa.cpp:588-615: S = A (x) B, all n x n. */
int rcwa_redheffer(rcwa_context* ctx, int n, const rcwa_complex* const A[4],
                   const rcwa_complex* const B[4], rcwa_complex* const S[4], uint32_t* status);
/* ComputeSourceModeCoeff + ComputeReflectedField + ComputeTransmittedField +
 * ComputeDiffractionEfficiencies, rcwa.cpp:469-585, from S_global's S11/S21. */
int rcwa_efficiencies(rcwa_context* ctx, const rcwa_source* source, const rcwa_params* params,
                      const rcwa_complex* k_inc, const rcwa_complex* Kx, const rcwa_complex* Ky,
                      const rcwa_complex* Kz_ref, const rcwa_complex* Kz_trn,
                      const rcwa_complex* S11, const rcwa_complex* S21, rcwa_result* out);

/* ---- dense building blocks (batched, host pointers) ---------------------- */
/* ComplexEigenSolver replacement (rcwa.cpp:298-306): for each of `batch`
 * n x n matrices A, eigenvalues lam[batch][n] and unit-2-norm eigenvectors
 * W[batch][n x n].  status[batch] gets RCWA_STATUS_EIG_NOCONV on failure. */
int rcwa_eig(rcwa_context* ctx, int n, int batch, const rcwa_complex* A, rcwa_complex* lam,
             rcwa_complex* W, uint32_t* status);
/* Allocation-free eigensolver.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory -- code recording a CUDA
 * graph, latency-critical loops that must keep away from the allocator, or
 * hosts that give this library a fixed memory budget -- this runs the same
 * eigensolver as rcwa_eig with no cudaMalloc/cudaFree and no allocating
 * library call.  All pointers are DEVICE pointers: A_dev (batch packed n x n,
 * column-major, left unchanged), lam_dev (batch x n), W_dev (batch packed
 * n x n), status_dev (batch uint32, cleared by the call).  Work is queued on
 * cuda_stream (NULL = legacy default stream); the call does not synchronise.
 *
 * Scratch lives in one fixed device array of RCWA_EIG_NOALLOC_SCRATCH_BYTES
 * compiled into the library, which every GPU that loads the library holds
 * until the process exits.  Limits: n <= RCWA_EIG_NOALLOC_MAX_N and
 *   bytes(n, batch) = r256(batch n^2 16) + batch (2 n^2 + n) 16
 *                     + batch (128 n + (ceil(n/32) + 1) 1024) 16 + 256
 * (input copy; Schur vectors, triangular eigenvectors and reflector scalars;
 * blocked-Hessenberg panels; r256 rounds up to a multiple of 256) at most
 * RCWA_EIG_NOALLOC_SCRATCH_BYTES -- the largest batch is 56 at n = 32, 22 at
 * n = 64, 11 at n = 98 and 7 at n = 128 -- otherwise RCWA_ERR_INVALID with
 * the bytes needed in rcwa_last_error().  The first
 * call on a device looks up the array's device address once (with that
 * device current); make that first call before any stream capture.  All calls
 * share the one array, which keeps the last call's contents: calls whose GPU
 * work overlaps (different streams, or several host threads) race on it and
 * must be serialised by the caller. */
#define RCWA_EIG_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)
#define RCWA_EIG_NOALLOC_MAX_N 128
int rcwa_eig_noalloc(int n, int batch, const rcwa_complex* A_dev, rcwa_complex* lam_dev,
                     rcwa_complex* W_dev, uint32_t* status_dev, void* cuda_stream);
/* Host-side fault injection for the eigensolver's bounded QR iteration (the
 * reference abort()s when ComplexEigenSolver fails, rcwa.cpp:300): the QR
 * sweeps allowed per eigensolve, in units of max(n, 10), for every later
 * solve in the process (-1 restores the default 100; 0 makes every matrix
 * with an undeflated block stop at once with RCWA_STATUS_EIG_NOCONV and NaN
 * eigenvalues).  Process-wide: not for use while other threads solve. */
int rcwa_eig_set_sweep_cap(int sweeps_per_n);
/* CTAs that share one matrix in the eigensolver's QR iteration (no
 * reference counterpart): 0 (default) chooses per launch -- for n >= 400 in
 * launches of few matrices, a thread-block cluster of up to 8 CTAs whose
 * helpers share the far updates of each multishift sweep -- while 1, 2, 4 or
 * 8 forces that many (if the device can hold such clusters).  Process-wide. */
int rcwa_eig_set_cluster_size(int ctas_per_matrix);
/* Test hook for the int8-slice GEMM's bounded waits (no reference
 * counterpart): while on (1), its launches leave out their first operand
 * copy, so the wait for it gives up after about a second, the CTA records the
 * failure, frees its tensor memory and returns, and the calling entry point
 * reports RCWA_ERR_CUDA; 0 turns it off.  Process-wide. */
int rcwa_debug_gemm_inject_timeout(int on);
/* PartialPivLU solve (the .lu().solve calls of rcwa.cpp): X = A^-1 B, batched. */
int rcwa_lu_solve(rcwa_context* ctx, int n, int nrhs, int batch, const rcwa_complex* A,
                  const rcwa_complex* B, rcwa_complex* X, uint32_t* status);
/* The same with a precision: RCWA_PREC_FP64 is rcwa_lu_solve; RCWA_PREC_MIXED
 * factors and solves in FP32 and runs refine_sweeps (1..4) FP64 residual
 * refinement sweeps (status may carry RCWA_STATUS_REFINE_SLOW). */
int rcwa_lu_solve_ex(rcwa_context* ctx, int n, int nrhs, int batch, const rcwa_complex* A,
                     const rcwa_complex* B, rcwa_complex* X, uint32_t* status, int precision,
                     int refine_sweeps);
/* C = A * B (m x k times k x n, column-major host arrays), batched; precision
 * selects FP64 or the context's mixed-precision GEMM -- int8 slices, or
 * split-TF32 with RCWA_MIXED_GEMM_TF32 (the Eigen operator* products of
 * rcwa.cpp). */
int rcwa_gemm(rcwa_context* ctx, int m, int n, int k, int batch, const rcwa_complex* A,
              const rcwa_complex* B, rcwa_complex* C, int precision);
/* C = alpha A B + beta C on device arrays (batch-packed, column-major),
 * asynchronous on the context's stream; the mixed-precision GEMM's workspace
 * comes from the context's workspace. */
int rcwa_gemm_device(rcwa_context* ctx, int m, int n, int k, int batch, rcwa_complex alpha,
                     const rcwa_complex* A_dev, const rcwa_complex* B_dev, rcwa_complex beta,
                     rcwa_complex* C_dev, int precision);
/* FP64 GEMM kernel per shape bucket (no reference counterpart), usually the
 * table written by the project's tuner (rcwa_b200/tune.py): choice[5 kb + sb]
 * for k bucket kb (k <= 16, <= 32, <= 64, <= 128, larger) and size bucket sb
 * (min(m, n) <= 64, <= 128, <= 256, <= 512, larger); 0 = the FP64 tensor-core
 * (DMMA) kernel fed by cp.async, 1 = the CUDA-core kernel, 2 = the DMMA kernel
 * fed by the tensor memory accelerator (TMA; products of operands as stored,
 * others fall back to 0), 3 = the cp.async-fed DMMA kernel with 32 x 64
 * tiles, -1 = the built-in rule (DMMA for k > 64).  NULL restores the
 * built-in rule.  Process-wide. */
int rcwa_set_gemm_table(const int* choice);
/* C = alpha op(A) op(B) + beta C, batched, column-major host arrays; op = 1
 * takes the conjugate transpose (A stored k x m, B stored n x k), C is read
 * when beta != 0.  FP64 only. */
int rcwa_gemm_ex(rcwa_context* ctx, int opa, int opb, int m, int n, int k, int batch,
                 rcwa_complex alpha, const rcwa_complex* A, const rcwa_complex* B, rcwa_complex beta,
                 rcwa_complex* C);

#ifdef __cplusplus
}
#endif

#endif /* RCWA_B200_H */
