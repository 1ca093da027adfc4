// Batched complex128 nonsymmetric eigensolver with eigenvectors.
//
// Replaces Eigen::ComplexEigenSolver (rcwa.cpp:298-306) for the per-layer
// Omega^2 = P Q problem.  The algorithm is the textbook one (Golub & Van Loan
// ch. 7; LAPACK zgehrd/zunghr/zlahqr/ztrevc), written for one CTA per matrix
// so a batch of wavelengths / layers / requests runs concurrently:
//
//  1-2. hess_blocked (zhess.cu): blocked Householder reduction A = Q H Q^H
//                   and Q accumulated backwards into Z, panel kernels plus
//                   batched GEMMs.
//  3. schur_kernel  (zschur.cu) complex QR -- multishift sweeps on large
//                   active blocks, single-shift on small ones -- until H = T is
//                   upper triangular; Z <- Z * (all reflectors) = Schur vectors.
//                   The number of sweeps is capped; a matrix that does not
//                   converge gets RCWA_STATUS_EIG_NOCONV (the reference aborts,
//                   rcwa.cpp:300) and NaN eigenvalues.
//  4. trevc_kernel  eigenvectors of T by back substitution, one warp per
//                   eigenvector, with (T_ii - T_kk) perturbed to
//                   max(ulp*|T_kk|, smlnum) when smaller (ztrevc's rule).
//  5. W = Z * X by the batched GEMM, then every column scaled to unit 2-norm.
//
// Non-finite input is detected up front and reported as NONFINITE|EIG_NOCONV
// without iterating.
#include <cfloat>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {

constexpr int TREVC_WARPS = 4;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

template <int NT>
__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (lane < NT / 32) t = red[lane];
  t = warp_sum(t);
  return t;
}

// ---------------------------------------------------------------------------
// 4. Eigenvectors of the upper-triangular T: X[:, k] solves
//    (T[0:k,0:k] - T_kk I) x = -T[0:k, k], x_k = 1.  One warp per k; the
//    right-hand side lives in shared memory.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TREVC_WARPS * 32)
trevc_kernel(const double2* __restrict__ Tg, int ld, long long stride, int n,
             double2* __restrict__ Xg) {
  extern __shared__ __align__(16) double2 sm[];
  const int b = blockIdx.y;
  const double2* T = Tg + (long long)b * stride;
  double2* X = Xg + (long long)b * stride;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int k = blockIdx.x * TREVC_WARPS + wid;
  if (k >= n) return;
  double2* xs = sm + (long long)wid * n;
  const double ulp = DBL_EPSILON;
  const double smlnum = DBL_MIN * ((double)n / ulp);
  const double2 tkk = T[(long long)k * ld + k];
  const double smin = fmax(ulp * cabs1(tkk), smlnum);
  const double2* tk = T + (long long)k * ld;
  for (int r = lane; r < k; r += 32) xs[r] = cneg(tk[r]);
  __syncwarp();
  for (int ii = k - 1; ii >= 0; --ii) {
    double2 d = csub(T[(long long)ii * ld + ii], tkk);
    if (cabs1(d) < smin) d = cmk(smin, 0.0);
    const double2 xi = cdiv(xs[ii], d);
    __syncwarp();
    if (lane == 0) xs[ii] = xi;
    const double2* ti = T + (long long)ii * ld;
    for (int r = lane; r < ii; r += 32) {
      double2 v = xs[r];
      double2 tt = ti[r];
      v.x -= xi.x * tt.x - xi.y * tt.y;
      v.y -= xi.x * tt.y + xi.y * tt.x;
      xs[r] = v;
    }
    __syncwarp();
  }
  double2* xk = X + (long long)k * ld;
  for (int r = lane; r < n; r += 32) xk[r] = (r < k) ? xs[r] : cmk(r == k ? 1.0 : 0.0, 0.0);
}

// 5b. unit 2-norm columns (Eigen normalises the eigenvectors).
__global__ void normalize_cols_kernel(double2* __restrict__ Wg, int ld, long long stride, int n) {
  const int b = blockIdx.y;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int k = blockIdx.x * (blockDim.x / 32) + wid;
  if (k >= n) return;
  double2* w = Wg + (long long)b * stride + (long long)k * ld;
  double s = 0.0;
  for (int r = lane; r < n; r += 32) s += cabs2(w[r]);
  s = warp_sum(s);
  if (s > 0.0 && isfinite(s)) {
    double inv = 1.0 / sqrt(s);
    for (int r = lane; r < n; r += 32) w[r] = cscale(w[r], inv);
  }
}

}  // namespace

size_t zeig_workspace_bytes(int n, int batch) {
  // Z, X (n x n each) and tau (n), all per matrix, plus the blocked
  // Hessenberg workspace (X also holds the dense reflectors meanwhile)
  return (size_t)batch * ((size_t)2 * n * n + n) * sizeof(double2) + hess_ws_bytes(n, batch) + 256;
}

int zeig(cudaStream_t s, int n, int batch, double2* A, int ld, long long sA, double2* W,
         long long sW, double2* lam, long long slam, uint32_t* status, void* ws) {
  if (n <= 0 || batch <= 0) return RCWA_OK;
  if (ld != n) {
    set_last_error("zeig: ld must equal n");
    return RCWA_ERR_INVALID;
  }
  double2* Z = (double2*)ws;
  double2* X = Z + (size_t)batch * n * n;
  double2* tau = X + (size_t)batch * n * n;
  const long long sZ = (long long)n * n;
  if (sA != sZ) {
    set_last_error("zeig: matrices must be packed (stride n*n)");
    return RCWA_ERR_INVALID;
  }
  const size_t trevc_shm = (size_t)TREVC_WARPS * n * sizeof(double2);
  if (trevc_shm > 200 * 1024) {
    set_last_error("zeig: n=%d too large", n);
    return RCWA_ERR_INVALID;
  }
  if (trevc_shm > 48 * 1024) {
    // per function and device, shared by all threads: set the bound once, not
    // this call's size (a concurrent call with a smaller n would undercut it)
    static bool set[64] = {};
    int dev = 0;
    RCWA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !set[dev]) {
      RCWA_CUDA_TRY(cudaFuncSetAttribute(trevc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024));
      if (dev < 64) set[dev] = true;
    }
  }
  void* tok = nullptr;
  (void)tau;
  {
    // blocked Householder reduction + backward Q accumulation (zhess.cu);
    // the dense reflectors live in X until trevc overwrites it
    void* hws = (void*)(((uintptr_t)(tau + (size_t)batch * n) + 255) & ~(uintptr_t)255);
    tok = prof_begin(s);
    int rc = hess_blocked(s, n, batch, A, Z, X, hws);
    prof_end(s, tok, "hess");
    // Householder reduction (40/3) n^3 + Q accumulation (16/3) n^3 real flops per matrix
    if (tok) prof_add_flops("hess", 56.0 / 3.0 * n * (double)n * n * batch);
    if (rc) return rc;
  }
  {
    int rc = schur_launch(s, A, ld, sA, n, Z, lam, slam, status, batch);
    if (rc) return rc;
  }
  {
    dim3 g(cdiv_up(n, TREVC_WARPS), batch);
    tok = prof_begin(s);
    trevc_kernel<<<g, TREVC_WARPS * 32, (size_t)TREVC_WARPS * n * sizeof(double2), s>>>(A, ld, sA,
                                                                                          n, X);
    prof_end(s, tok, "trevc");
    if (tok) prof_add_flops("trevc", 4.0 / 3.0 * n * (double)n * n * batch);
    count_launch();
    RCWA_LAUNCH_CHECK();
  }
  {
    ZGemm g;
    g.m = n;
    g.n = n;
    g.k = n;
    g.A = Z;
    g.lda = n;
    g.sA = sZ;
    g.B = X;
    g.ldb = n;
    g.sB = sZ;
    g.C = W;
    g.ldc = n;
    g.sC = sW;
    g.batch = batch;
    int rc = zgemm(s, g);
    if (rc) return rc;
  }
  {
    dim3 g(cdiv_up(n, 8), batch);
    normalize_cols_kernel<<<g, 256, 0, s>>>(W, n, sW, n);
    count_launch();
    RCWA_LAUNCH_CHECK();
  }
  return RCWA_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free eigensolver entry point.
//
// Some callers cannot allocate device memory: code running inside a CUDA
// graph that is being captured, real-time loops that must not touch the
// allocator, and hosts that hand this library a fixed memory budget up front.
// For them rcwa_eig_noalloc runs the same eigensolver as rcwa_eig, but its
// scratch (a copy of the input, the Schur vectors Z, the triangular
// eigenvectors X and the Householder scalars) lives in the file-scope device
// array below instead of a cudaMalloc'd workspace.  The array is part of the
// library image: every GPU that loads the library holds its
// RCWA_EIG_NOALLOC_SCRATCH_BYTES until the process exits.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_eig_noalloc_scratch[RCWA_EIG_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};
}  // namespace

// Device address of the scratch array on the current device, looked up once
// per device (cudaGetSymbolAddress with that device current).
static int noalloc_scratch(void** out) {
  int dev = 0;
  RCWA_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_last_error("rcwa_eig_noalloc: device %d out of range", dev);
    return RCWA_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_eig_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_last_error("rcwa_eig_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return RCWA_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return RCWA_OK;
}

size_t eig_noalloc_bytes(int n, int batch) {
  const size_t copy = (size_t)batch * n * n * sizeof(double2);
  return ((copy + 255) & ~(size_t)255) + zeig_workspace_bytes(n, batch);
}

}  // namespace rcwa

extern "C" int rcwa_eig_noalloc(int n, int batch, const rcwa_complex* A_dev, rcwa_complex* lam_dev,
                                rcwa_complex* W_dev, uint32_t* status_dev, void* cuda_stream) {
  using namespace rcwa;
  if (n <= 0 || batch <= 0 || !A_dev || !lam_dev || !W_dev || !status_dev) {
    set_last_error("rcwa_eig_noalloc: bad argument");
    return RCWA_ERR_INVALID;
  }
  if (n > RCWA_EIG_NOALLOC_MAX_N || eig_noalloc_bytes(n, batch) > RCWA_EIG_NOALLOC_SCRATCH_BYTES) {
    set_last_error("rcwa_eig_noalloc: n=%d batch=%d needs %zu scratch bytes; the fixed scratch holds "
                   "%zu bytes and n may not exceed %d",
                   n, batch, eig_noalloc_bytes(n, batch), (size_t)RCWA_EIG_NOALLOC_SCRATCH_BYTES,
                   RCWA_EIG_NOALLOC_MAX_N);
    return RCWA_ERR_INVALID;
  }
  void* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)cuda_stream;
  const size_t nn = (size_t)n * n;
  double2* Acopy = (double2*)base;
  void* ws = (char*)base + ((batch * nn * sizeof(double2) + 255) & ~(size_t)255);
  // the kernels OR status bits into status_dev: it must start at zero
  RCWA_CUDA_TRY(cudaMemsetAsync(status_dev, 0, (size_t)batch * sizeof(uint32_t), s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(Acopy, A_dev, batch * nn * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  prof_suspend(true);
  rc = zeig(s, n, batch, Acopy, n, (long long)nn, (double2*)W_dev, (long long)nn, (double2*)lam_dev, n,
            status_dev, ws);
  prof_suspend(false);
  return rc;
}
