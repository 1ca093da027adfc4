// Batched complex128 linear solve X = A^-1 B by LU with partial pivoting.
//
// This replaces every Eigen ``.lu().solve(...)`` (PartialPivLU) of the
// reference (rcwa.cpp:267, 270, 280, 281, 335, 336, 345-348, 392-408,
// 453-462, 520, 605-611).  The system is stored as one augmented column-major
// block M = [A | B] (n rows, n + nrhs columns); on return the A part holds U
// (and the L multipliers) and the B part holds the solution.
//
// 1. P A = L U by blocked right-looking elimination over the A columns, with
//    panel width NB:
//      panel  : one CTA per matrix factors the n-j x NB panel (pivot search,
//               row swaps inside the panel, scaling, rank-1 updates);
//      swap+L : one thread per trailing column applies the panel's row swaps
//               and the unit-lower NB x NB forward substitution;
//      update : the trailing block A22 -= L21 U12 as a batched GEMM.
//    Each panel's interchanges are applied to the columns on both sides, so
//    the stored multipliers form L of P A = L U (LAPACK's convention).
// 2. the right-hand sides get all row swaps at once (B <- P B): the swaps
//    are composed into gather indices (piv is overwritten with them) and each
//    column is permuted through shared memory;
// 3. L Y = P B and U X = Y by recursive halving: each off-diagonal block is
//    one GEMM with k up to n/2, only NB x NB diagonal blocks are solved by the
//    column kernels.  With many right-hand sides (the [A | I] and [D | R | R']
//    systems of the S-matrix algebra) this moves most of the flops from
//    rank-NB updates onto large-k GEMMs.
#include <algorithm>
#include <functional>

#include "common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {

constexpr int NB = 32;
constexpr int PANEL_NT = 256;
constexpr int COL_NT = 64;

__device__ __forceinline__ void argmax_reduce(double& v, int& idx) {
  // warp-level: keep the larger value, ties -> smaller index
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    double ov = __shfl_down_sync(0xffffffffu, v, off);
    int oi = __shfl_down_sync(0xffffffffu, idx, off);
    if (ov > v || (ov == v && oi < idx)) {
      v = ov;
      idx = oi;
    }
  }
}

__global__ void __launch_bounds__(PANEL_NT)
lu_panel_kernel(double2* __restrict__ Mg, int ld, long long stride, int n, int j, int jb,
                int* __restrict__ pivg, uint32_t* __restrict__ status) {
  const int b = blockIdx.x;
  double2* M = Mg + (long long)b * stride;
  int* piv = pivg + (long long)b * n;
  __shared__ double s_val[PANEL_NT / 32];
  __shared__ int s_idx[PANEL_NT / 32];
  __shared__ double2 s_urow[NB];
  __shared__ int s_p;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

  for (int c = 0; c < jb; ++c) {
    const int col = j + c;
    double2* Mc = M + (long long)col * ld;
    // 1. pivot search over rows col..n-1 (|re|+|im|, first maximum wins)
    double best = -1.0;
    int bi = n;
    for (int r = col + tid; r < n; r += PANEL_NT) {
      double v = cabs1(Mc[r]);
      if (v > best) { best = v; bi = r; }
    }
    argmax_reduce(best, bi);
    if (lane == 0) { s_val[wid] = best; s_idx[wid] = bi; }
    __syncthreads();
    if (wid == 0) {
      best = lane < PANEL_NT / 32 ? s_val[lane] : -1.0;
      bi = lane < PANEL_NT / 32 ? s_idx[lane] : n;
      argmax_reduce(best, bi);
      if (lane == 0) {
        if (bi >= n) bi = col;
        s_p = bi;
        piv[col] = bi;
      }
    }
    __syncthreads();
    const int p = s_p;
    // 2. swap rows col <-> p inside the panel
    if (p != col) {
      for (int cc = tid; cc < jb; cc += PANEL_NT) {
        double2* q = M + (long long)(j + cc) * ld;
        double2 t = q[col];
        q[col] = q[p];
        q[p] = t;
      }
    }
    __syncthreads();
    // 3. pivot row of the remaining panel columns -> smem
    for (int cc = c + 1 + tid; cc < jb; cc += PANEL_NT) s_urow[cc] = M[(long long)(j + cc) * ld + col];
    const double2 pv = Mc[col];
    if (tid == 0 && pv.x == 0.0 && pv.y == 0.0) atomicOr(status + b, (unsigned)ST_SINGULAR);
    __syncthreads();
    const double2 inv = crcp(pv);
    // 4. scale the column below the pivot and rank-1 update the panel
    for (int r = col + 1 + tid; r < n; r += PANEL_NT) {
      double2 l = cmul(Mc[r], inv);
      Mc[r] = l;
      for (int cc = c + 1; cc < jb; ++cc) {
        double2* q = M + (long long)(j + cc) * ld + r;
        double2 u = s_urow[cc];
        double2 v = *q;
        v.x -= l.x * u.x - l.y * u.y;
        v.y -= l.x * u.y + l.y * u.x;
        *q = v;
      }
    }
    __syncthreads();
  }
}

// Row swaps of panel j plus forward substitution with the unit-lower L11 for
// columns [c_begin, c_end) of the augmented matrix.
__global__ void __launch_bounds__(COL_NT)
lu_swap_lsolve_kernel(double2* __restrict__ Mg, int ld, long long stride, int n, int j, int jb,
                      int c_begin, int c_end, const int* __restrict__ pivg, int swap) {
  const int b = blockIdx.y;
  double2* M = Mg + (long long)b * stride;
  const int* piv = pivg + (long long)b * n;
  __shared__ double2 L[NB][NB + 1];  // L[r][c]
  __shared__ int sp[NB];
  const int tid = threadIdx.x;
  for (int e = tid; e < jb * jb; e += COL_NT) {
    int r = e % jb, c = e / jb;
    L[r][c] = M[(long long)(j + c) * ld + j + r];
  }
  if (swap)
    for (int e = tid; e < jb; e += COL_NT) sp[e] = piv[j + e];
  __syncthreads();
  const int col = c_begin + blockIdx.x * COL_NT + tid;
  if (col >= c_end) return;
  double2* q = M + (long long)col * ld;
  if (swap)
    for (int c = 0; c < jb; ++c) {
      int p = sp[c];
      if (p != j + c) {
        double2 t = q[j + c];
        q[j + c] = q[p];
        q[p] = t;
      }
    }
  double2 x[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) x[c] = (c < jb) ? q[j + c] : cmk(0.0, 0.0);
#pragma unroll
  for (int c = 0; c < NB; ++c) {
#pragma unroll
    for (int r = c + 1; r < NB; ++r) {
      if (r < jb) {
        double2 l = L[r][c];
        x[r].x -= l.x * x[c].x - l.y * x[c].y;
        x[r].y -= l.x * x[c].y + l.y * x[c].x;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < NB; ++c)
    if (c < jb) q[j + c] = x[c];
}

// Row interchanges piv[r_begin..r_end) (in order) applied to columns
// [c_begin, c_end): the multipliers left of a panel, and the right-hand sides
// (B <- P B).
__global__ void __launch_bounds__(COL_NT)
lu_rowswap_kernel(double2* __restrict__ Mg, int ld, long long stride, int n, int r_begin, int r_end,
                  int c_begin, int c_end, const int* __restrict__ pivg) {
  const int b = blockIdx.y;
  double2* M = Mg + (long long)b * stride;
  const int* piv = pivg + (long long)b * n;
  const int col = c_begin + blockIdx.x * COL_NT + threadIdx.x;
  if (col >= c_end) return;
  double2* q = M + (long long)col * ld;
  for (int r = r_begin; r < r_end; ++r) {
    const int p = piv[r];
    if (p != r) {
      const double2 t = q[r];
      q[r] = q[p];
      q[p] = t;
    }
  }
}

// The interchanges piv[0..n) composed into one gather: idx[r] = the row of
// the original right-hand side that ends up in row r (one thread per matrix,
// indices built in shared memory, then written over piv).
__global__ void lu_perm_kernel(int* __restrict__ pivg, int n) {
  extern __shared__ int idx[];
  int* piv = pivg + (long long)blockIdx.x * n;
  for (int r = threadIdx.x; r < n; r += blockDim.x) idx[r] = r;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int r = 0; r < n; ++r) {
      const int p = piv[r];
      if (p != r) {
        const int t = idx[r];
        idx[r] = idx[p];
        idx[p] = t;
      }
    }
  __syncthreads();
  for (int r = threadIdx.x; r < n; r += blockDim.x) piv[r] = idx[r];
}

// B <- P B as a gather with the composed indices: each warp stages one
// column in shared memory (coalesced read) and writes it back permuted
// (coalesced write); PERM_CPW columns per warp.
constexpr int PERM_WARPS = 8, PERM_CPW = 4;
__global__ void __launch_bounds__(PERM_WARPS * 32)
lu_gather_kernel(double2* __restrict__ Mg, int ld, long long stride, int n, int c_begin, int c_end,
                 const int* __restrict__ idxg) {
  extern __shared__ double2 col_sh[];
  const int nw = blockDim.x >> 5;   // warps (fewer for large n: n doubles2 of shared memory each)
  const int b = blockIdx.y, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double2* M = Mg + (long long)b * stride;
  const int* idx = idxg + (long long)b * n;
  double2* sh = col_sh + (size_t)w * n;
  for (int t = 0; t < PERM_CPW; ++t) {
    const int col = c_begin + (blockIdx.x * nw + w) * PERM_CPW + t;
    if (col >= c_end) break;   // warp-uniform
    double2* q = M + (long long)col * ld;
    for (int r = lane; r < n; r += 32) sh[r] = q[r];
    __syncwarp();
    for (int r = lane; r < n; r += 32) q[r] = sh[idx[r]];
    __syncwarp();
  }
}

// Upper-triangular solve X = U11^-1 X for rows j..j+jb-1 of the right-hand
// side columns [c_begin, c_end).
__global__ void __launch_bounds__(COL_NT)
lu_usolve_kernel(double2* __restrict__ Mg, int ld, long long stride, int j, int jb, int c_begin,
                 int c_end) {
  const int b = blockIdx.y;
  double2* M = Mg + (long long)b * stride;
  __shared__ double2 U[NB][NB + 1];
  __shared__ double2 dinv[NB];
  const int tid = threadIdx.x;
  for (int e = tid; e < jb * jb; e += COL_NT) {
    int r = e % jb, c = e / jb;
    U[r][c] = M[(long long)(j + c) * ld + j + r];
  }
  __syncthreads();
  for (int e = tid; e < jb; e += COL_NT) dinv[e] = crcp(U[e][e]);
  __syncthreads();
  const int col = c_begin + blockIdx.x * COL_NT + tid;
  if (col >= c_end) return;
  double2* q = M + (long long)col * ld;
  double2 x[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) x[c] = (c < jb) ? q[j + c] : cmk(0.0, 0.0);
#pragma unroll
  for (int c = NB - 1; c >= 0; --c) {
    if (c < jb) {
      x[c] = cmul(x[c], dinv[c]);
#pragma unroll
      for (int r = 0; r < c; ++r) {
        double2 u = U[r][c];
        x[r].x -= u.x * x[c].x - u.y * x[c].y;
        x[r].y -= u.x * x[c].y + u.y * x[c].x;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < NB; ++c)
    if (c < jb) q[j + c] = x[c];
}

}  // namespace

int zgesv(cudaStream_t s, int n, int nrhs, double2* M, int ld, long long stride, int batch,
          int* piv, uint32_t* status, int tc) {
  if (n <= 0 || batch <= 0) return RCWA_OK;
  const int ncols = n + nrhs;
  auto gemm = [&](int m, int nc, int k, const double2* A, const double2* Bm, double2* C) {
    ZGemm gm;
    gm.m = m;
    gm.n = nc;
    gm.k = k;
    gm.alpha = cmk(-1.0, 0.0);
    gm.beta = cmk(1.0, 0.0);
    gm.A = A;
    gm.lda = ld;
    gm.sA = stride;
    gm.B = Bm;
    gm.ldb = ld;
    gm.sB = stride;
    gm.C = C;
    gm.ldc = ld;
    gm.sC = stride;
    gm.batch = batch;
    gm.tc = tc;
    return zgemm(s, gm);
  };
  // 1. P A = L U, right-looking over the A columns only
  for (int j = 0; j < n; j += NB) {
    const int jb = (n - j < NB) ? (n - j) : NB;
    void* tok = prof_begin(s);
    lu_panel_kernel<<<batch, PANEL_NT, 0, s>>>(M, ld, stride, n, j, jb, piv, status);
    prof_end(s, tok, "lu_panel");
    count_launch();
    RCWA_LAUNCH_CHECK();
    if (j > 0) {   // the earlier multipliers follow this panel's interchanges (P A = L U)
      dim3 g(cdiv_up(j, COL_NT), batch);
      lu_rowswap_kernel<<<g, COL_NT, 0, s>>>(M, ld, stride, n, j, j + jb, 0, j, piv);
      count_launch();
      RCWA_LAUNCH_CHECK();
    }
    const int cb = j + jb;
    if (cb < n) {
      dim3 g(cdiv_up(n - cb, COL_NT), batch);
      lu_swap_lsolve_kernel<<<g, COL_NT, 0, s>>>(M, ld, stride, n, j, jb, cb, n, piv, 1);
      count_launch();
      RCWA_LAUNCH_CHECK();
      int rc = gemm(n - cb, n - cb, jb, M + (long long)j * ld + cb, M + (long long)cb * ld + j,
                    M + (long long)cb * ld + cb);
      if (rc) return rc;
    }
  }
  if (nrhs <= 0) return RCWA_OK;
  // 2. B <- P B
  double2* Bc = M + (long long)n * ld;   // right-hand sides, rows 0..n-1
  {
    const size_t pshm = (size_t)n * sizeof(int);
    const int pw = (int)std::min<size_t>(PERM_WARPS, (200 * 1024) / ((size_t)n * sizeof(double2)));
    if (pw < 1) {
      set_last_error("zgesv: n=%d too large", n);
      return RCWA_ERR_INVALID;
    }
    const size_t gshm = (size_t)pw * n * sizeof(double2);
    static bool set[64] = {};   // per device: allow the bound once
    int dev = 0;
    RCWA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !set[dev]) {
      RCWA_CUDA_TRY(cudaFuncSetAttribute(lu_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
      RCWA_CUDA_TRY(cudaFuncSetAttribute(lu_gather_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
      if (dev < 64) set[dev] = true;
    }
    lu_perm_kernel<<<batch, 128, pshm, s>>>(piv, n);   // piv now holds the gather indices
    count_launch();
    RCWA_LAUNCH_CHECK();
    dim3 g(cdiv_up(nrhs, pw * PERM_CPW), batch);
    lu_gather_kernel<<<g, pw * 32, gshm, s>>>(M, ld, stride, n, n, ncols, piv);
    count_launch();
    RCWA_LAUNCH_CHECK();
  }
  // 3./4. L Y = P B, then U X = Y, by recursive halving: the off-diagonal
  // blocks become GEMMs with k up to n/2 (tensor-core sized), only the
  // diagonal NB x NB blocks are solved by the column kernels
  auto split = [](int r0, int r1) { return r0 + NB * (((r1 - r0 + NB - 1) / NB) / 2); };
  int rc = RCWA_OK;
  std::function<int(int, int)> lower = [&](int r0, int r1) -> int {
    if (r1 - r0 <= NB) {
      dim3 g(cdiv_up(nrhs, COL_NT), batch);
      lu_swap_lsolve_kernel<<<g, COL_NT, 0, s>>>(M, ld, stride, n, r0, r1 - r0, n, ncols, piv, 0);
      count_launch();
      RCWA_LAUNCH_CHECK();
      return RCWA_OK;
    }
    const int mid = split(r0, r1);
    int r = lower(r0, mid);
    if (r) return r;
    r = gemm(r1 - mid, nrhs, mid - r0, M + (long long)r0 * ld + mid, Bc + r0, Bc + mid);
    if (r) return r;
    return lower(mid, r1);
  };
  std::function<int(int, int)> upper = [&](int r0, int r1) -> int {
    if (r1 - r0 <= NB) {
      dim3 g(cdiv_up(nrhs, COL_NT), batch);
      lu_usolve_kernel<<<g, COL_NT, 0, s>>>(M, ld, stride, r0, r1 - r0, n, ncols);
      count_launch();
      RCWA_LAUNCH_CHECK();
      return RCWA_OK;
    }
    const int mid = split(r0, r1);
    int r = upper(mid, r1);
    if (r) return r;
    r = gemm(mid - r0, nrhs, r1 - mid, M + (long long)mid * ld + r0, Bc + mid, Bc + r0);
    if (r) return r;
    return upper(r0, mid);
  };
  if ((rc = lower(0, n))) return rc;
  return upper(0, n);
}

}  // namespace rcwa
