// Batched complex linear solve X = A^-1 B by LU with partial pivoting.
//
// This replaces every Eigen ``.lu().solve(...)`` (PartialPivLU) of the
// reference (rcwa.cpp:267, 270, 280, 281, 335, 336, 345-348, 392-408,
// 453-462, 520, 605-611).  The system is stored as one augmented column-major
// block M = [A | B] (n rows, n + nrhs columns); on return the B part holds
// the solution.
//
// FP64 form (zgesv):
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
// On return the A part holds U and the L multipliers.
//
// Mixed-precision form (zgesv_ir): the same factorisation and solves run on
// a complex64 copy of [A | B] (the kernels below are templates over the
// element type; the FP32 GEMM updates run on CUDA cores), giving X0.  Then
// each refinement sweep computes the residual R = B - A X in FP64 on the
// FP64 tensor cores (the DMMA GEMM, A read from the untouched FP64 A part),
// solves L U dX = P R with the FP32 factors and adds dX to X in FP64.  A
// solve whose last correction stays above 1e-4 of |X| is flagged
// RCWA_STATUS_REFINE_SLOW (the FP32 factors were too inaccurate for the
// sweeps run).  The A part is left unchanged.
#include <algorithm>
#include <functional>

#include "common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {

constexpr int NB = 32;
constexpr int PANEL_NT = 256;
constexpr int PANEL_NT_WIDE = 1024;   // large n, few matrices: more rows in flight per column step
constexpr int COL_NT = 64;
constexpr int PCHUNK = 8;   // panel update: entries of a row in flight at once

template <class T>
struct Cx;
template <>
struct Cx<double2> {
  using R = double;
  __host__ __device__ static double2 mk(double r, double i) { return make_double2(r, i); }
};
template <>
struct Cx<float2> {
  using R = float;
  __host__ __device__ static float2 mk(float r, float i) { return make_float2(r, i); }
};

template <class R>
__device__ __forceinline__ void argmax_reduce(R& v, int& idx) {
  // warp-level: keep the larger value, ties -> smaller index
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    R ov = __shfl_down_sync(0xffffffffu, v, off);
    int oi = __shfl_down_sync(0xffffffffu, idx, off);
    if (ov > v || (ov == v && oi < idx)) {
      v = ov;
      idx = oi;
    }
  }
}

template <class T, int PNT>
__global__ void __launch_bounds__(PNT)
lu_panel_kernel(T* __restrict__ Mg, int ld, long long stride, int n, int j, int jb,
                int* __restrict__ pivg, uint32_t* __restrict__ status) {
  using R = typename Cx<T>::R;
  const int b = blockIdx.x;
  T* M = Mg + (long long)b * stride;
  int* piv = pivg + (long long)b * n;
  __shared__ R s_val[PNT / 32];
  __shared__ int s_idx[PNT / 32];
  __shared__ T s_urow[NB];
  __shared__ int s_p;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

  for (int c = 0; c < jb; ++c) {
    const int col = j + c;
    T* Mc = M + (long long)col * ld;
    // 1. pivot search over rows col..n-1 (|re|+|im|, first maximum wins)
    R best = -1;
    int bi = n;
    for (int r = col + tid; r < n; r += PNT) {
      R v = cabs1(Mc[r]);
      if (v > best) { best = v; bi = r; }
    }
    argmax_reduce(best, bi);
    if (lane == 0) { s_val[wid] = best; s_idx[wid] = bi; }
    __syncthreads();
    if (wid == 0) {
      best = lane < PNT / 32 ? s_val[lane] : R(-1);
      bi = lane < PNT / 32 ? s_idx[lane] : n;
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
      for (int cc = tid; cc < jb; cc += PNT) {
        T* q = M + (long long)(j + cc) * ld;
        T t = q[col];
        q[col] = q[p];
        q[p] = t;
      }
    }
    __syncthreads();
    // 3. pivot row of the remaining panel columns -> smem
    for (int cc = c + 1 + tid; cc < jb; cc += PNT) s_urow[cc] = M[(long long)(j + cc) * ld + col];
    const T pv = Mc[col];
    if (tid == 0 && pv.x == R(0) && pv.y == R(0)) atomicOr(status + b, (unsigned)ST_SINGULAR);
    __syncthreads();
    const T inv = crcp(pv);
    // 4. scale the column below the pivot and rank-1 update the panel; the
    // row's entries of the remaining columns are loaded PC at a time before
    // any is stored, so their load latencies overlap (fewer at a time with
    // 1024 threads, whose register budget is 64)
    constexpr int PC = PNT > 256 ? 4 : PCHUNK;
    for (int r = col + 1 + tid; r < n; r += PNT) {
      T l = cmul(Mc[r], inv);
      Mc[r] = l;
      for (int c0 = c + 1; c0 < jb; c0 += PC) {
        T v[PC];
#pragma unroll
        for (int u = 0; u < PC; ++u)
          if (c0 + u < jb) v[u] = M[(long long)(j + c0 + u) * ld + r];
#pragma unroll
        for (int u = 0; u < PC; ++u)
          if (c0 + u < jb) {
            const T w = s_urow[c0 + u];
            v[u].x -= l.x * w.x - l.y * w.y;
            v[u].y -= l.x * w.y + l.y * w.x;
            M[(long long)(j + c0 + u) * ld + r] = v[u];
          }
      }
    }
    __syncthreads();
  }
}

// Triangular solve with the NB x NB diagonal block at rows j..j+jb-1 for the
// right-hand-side columns [c_begin, c_end): X = L11^-1 X (unit lower, UPPER
// = false) or X = U11^-1 X (UPPER = true).  COL_NT columns per CTA are
// staged through shared memory: each warp moves whole column segments with
// one coalesced access per column (lane = row), eight columns in flight at a
// time; then each thread solves one column in registers (the column kernels'
// arithmetic, in the same order), and the tile goes back the same way.
// Dynamic shared memory: trsm_smem<T>() bytes.
template <class T>
constexpr size_t trsm_smem() {
  return sizeof(T) * ((size_t)(NB + COL_NT) * (NB + 1) + NB);
}
template <class T, bool UPPER>
__global__ void __launch_bounds__(COL_NT)
lu_trsm_tile_kernel(T* __restrict__ Mg, int ld, long long stride, int j, int jb, int c_begin, int c_end) {
  extern __shared__ __align__(16) unsigned char tsm[];
  T (*D)[NB + 1] = reinterpret_cast<T (*)[NB + 1]>(tsm);                                   // D[r][c]
  T (*Xs)[NB + 1] = reinterpret_cast<T (*)[NB + 1]>(tsm + sizeof(T) * NB * (NB + 1));     // Xs[col][r]
  T* dinv = reinterpret_cast<T*>(tsm + sizeof(T) * (NB + COL_NT) * (NB + 1));
  constexpr int NWP = COL_NT / 32;
  const int b = blockIdx.y;
  T* M = Mg + (long long)b * stride;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int cbase = c_begin + blockIdx.x * COL_NT;
  const int ncol = min(COL_NT, c_end - cbase);
  for (int e = tid; e < jb * jb; e += COL_NT) {
    const int r = e % jb, c = e / jb;
    D[r][c] = M[(long long)(j + c) * ld + j + r];
  }
  const T* src = M + (long long)cbase * ld + j + lane;
  for (int c0 = wid; c0 < ncol; c0 += NWP * 8) {
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int cc = c0 + u * NWP;
      v[u] = (cc < ncol && lane < jb) ? src[(long long)cc * ld] : Cx<T>::mk(0, 0);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int cc = c0 + u * NWP;
      if (cc < ncol && lane < jb) Xs[cc][lane] = v[u];
    }
  }
  __syncthreads();
  if (UPPER) {
    for (int e = tid; e < jb; e += COL_NT) dinv[e] = crcp(D[e][e]);
    __syncthreads();
  }
  if (tid < ncol) {
    T x[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) x[c] = (c < jb) ? Xs[tid][c] : Cx<T>::mk(0, 0);
    if (!UPPER) {
#pragma unroll
      for (int c = 0; c < NB; ++c) {
#pragma unroll
        for (int r = c + 1; r < NB; ++r) {
          if (r < jb) {
            T l = D[r][c];
            x[r].x -= l.x * x[c].x - l.y * x[c].y;
            x[r].y -= l.x * x[c].y + l.y * x[c].x;
          }
        }
      }
    } else {
#pragma unroll
      for (int c = NB - 1; c >= 0; --c) {
        if (c < jb) {
          x[c] = cmul(x[c], dinv[c]);
#pragma unroll
          for (int r = 0; r < c; ++r) {
            T u = D[r][c];
            x[r].x -= u.x * x[c].x - u.y * x[c].y;
            x[r].y -= u.x * x[c].y + u.y * x[c].x;
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NB; ++c)
      if (c < jb) Xs[tid][c] = x[c];
  }
  __syncthreads();
  T* dst = M + (long long)cbase * ld + j + lane;
  for (int c0 = wid; c0 < ncol; c0 += NWP * 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int cc = c0 + u * NWP;
      if (cc < ncol && lane < jb) dst[(long long)cc * ld] = Xs[cc][lane];
    }
  }
}

// Row interchanges piv[r_begin..r_end) (in order) applied to columns
// [c_begin, c_end): the multipliers left of a panel.
template <class T>
__global__ void __launch_bounds__(COL_NT)
lu_rowswap_kernel(T* __restrict__ Mg, int ld, long long stride, int n, int r_begin, int r_end,
                  int c_begin, int c_end, const int* __restrict__ pivg) {
  const int b = blockIdx.y;
  T* M = Mg + (long long)b * stride;
  const int* piv = pivg + (long long)b * n;
  const int col = c_begin + blockIdx.x * COL_NT + threadIdx.x;
  if (col >= c_end) return;
  T* q = M + (long long)col * ld;
  for (int r = r_begin; r < r_end; ++r) {
    const int p = piv[r];
    if (p != r) {
      const T t = q[r];
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
constexpr int GATHER_SMEM = 200 * 1024;
template <class T>
__global__ void __launch_bounds__(PERM_WARPS * 32)
lu_gather_kernel(T* __restrict__ Mg, int ld, long long stride, int n, int c_begin, int c_end,
                 const int* __restrict__ idxg) {
  extern __shared__ __align__(16) unsigned char gather_raw[];
  T* col_sh = reinterpret_cast<T*>(gather_raw);
  const int nw = blockDim.x >> 5;   // warps (fewer for large n: n elements of shared memory each)
  const int b = blockIdx.y, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T* M = Mg + (long long)b * stride;
  const int* idx = idxg + (long long)b * n;
  T* sh = col_sh + (size_t)w * n;
  for (int t = 0; t < PERM_CPW; ++t) {
    const int col = c_begin + (blockIdx.x * nw + w) * PERM_CPW + t;
    if (col >= c_end) break;   // warp-uniform
    T* q = M + (long long)col * ld;
    for (int r = lane; r < n; r += 32) sh[r] = q[r];
    __syncwarp();
    for (int r = lane; r < n; r += 32) q[r] = sh[idx[r]];
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// complex64 update C -= A B on CUDA cores (the FP32 factorisation's trailing
// updates and triangular-solve blocks).  64 x 64 C tile, K step 16, 256
// threads as 16 x 16, each a 4 x 4 complex micro-tile; the next K tile is
// fetched into registers while the current one is consumed from shared
// memory.
// ---------------------------------------------------------------------------
constexpr int CT = 64, CK = 16, CNT = 256;

__global__ void __launch_bounds__(CNT)
cgemm_sub_kernel(int m, int n, int k, const float2* __restrict__ A, int lda, long long sA,
                 const float2* __restrict__ B, int ldb, long long sB, float2* __restrict__ C, int ldc,
                 long long sC) {
  __shared__ float2 As[2][CK][CT];
  __shared__ float2 Bs[2][CK][CT + 1];
  const int bz = blockIdx.z;
  A += (long long)bz * sA;
  B += (long long)bz * sB;
  C += (long long)bz * sC;
  const int m0 = blockIdx.y * CT, n0 = blockIdx.x * CT;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  float2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  float2 ra[4], rb[4];
  auto gload = [&](int k0) {
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int e = tid + h * CNT, r = e & (CT - 1), kk = e >> 6;
      const int gr = m0 + r, gk = k0 + kk;
      ra[h] = (gr < m && gk < k) ? A[(long long)gk * lda + gr] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int e = tid + h * CNT, kk = e & (CK - 1), c = e >> 4;
      const int gk = k0 + kk, gc = n0 + c;
      rb[h] = (gk < k && gc < n) ? B[(long long)gc * ldb + gk] : make_float2(0.f, 0.f);
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int e = tid + h * CNT;
      As[buf][e >> 6][e & (CT - 1)] = ra[h];
      Bs[buf][e & (CK - 1)][e >> 4] = rb[h];
    }
  };
  const int kt = (k + CK - 1) / CK;
  if (kt > 0) {
    gload(0);
    sstore(0);
  }
  __syncthreads();
  for (int t = 0; t < kt; ++t) {
    const int buf = t & 1;
    if (t + 1 < kt) gload((t + 1) * CK);
#pragma unroll
    for (int kk = 0; kk < CK; ++kk) {
      float2 a[4], bb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[buf][kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bb[j] = Bs[buf][kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fmaf(a[i].x, bb[j].x, fmaf(-a[i].y, bb[j].y, acc[i][j].x));
          acc[i][j].y = fmaf(a[i].x, bb[j].y, fmaf(a[i].y, bb[j].x, acc[i][j].y));
        }
    }
    if (t + 1 < kt) sstore(buf ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int col = n0 + ty + 16 * j;
    if (col >= n) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = m0 + tx + 16 * i;
      if (row >= m) continue;
      float2* cp = C + (long long)col * ldc + row;
      float2 v = *cp;
      v.x -= acc[i][j].x;
      v.y -= acc[i][j].y;
      *cp = v;
    }
  }
}

// C -= A B, batched (FP64: the DMMA / CUDA-core ZGEMM; FP32: cgemm_sub_kernel)
int gemm_sub(cudaStream_t s, int m, int nc, int k, const double2* A, int ld, long long stride,
             const double2* Bm, double2* C, int batch) {
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
  return zgemm(s, gm);
}
int gemm_sub(cudaStream_t s, int m, int nc, int k, const float2* A, int ld, long long stride,
             const float2* Bm, float2* C, int batch) {
  if (m <= 0 || nc <= 0 || batch <= 0) return RCWA_OK;
  dim3 g(cdiv_up(nc, CT), cdiv_up(m, CT), batch);
  void* tok = prof_begin(s);
  cgemm_sub_kernel<<<g, CNT, 0, s>>>(m, nc, k, A, ld, stride, Bm, ld, stride, C, ld, stride);
  prof_end(s, tok, "cgemm_f32");
  if (tok) prof_add_flops("cgemm_f32", 8.0 * m * (double)nc * (double)k * batch);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

// Dynamic shared-memory limits of the permutation kernels, set once per
// device to their bound (concurrent callers with different n never lower it).
int perm_attrs() {
  static bool set[64] = {};
  int dev = 0;
  RCWA_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 64 || !set[dev]) {
    RCWA_CUDA_TRY(cudaFuncSetAttribute(lu_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    RCWA_CUDA_TRY(cudaFuncSetAttribute(lu_gather_kernel<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       GATHER_SMEM));
    RCWA_CUDA_TRY(cudaFuncSetAttribute(lu_gather_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       GATHER_SMEM));
    if (dev < 64) set[dev] = true;
  }
  return RCWA_OK;
}

// Dynamic shared-memory limits of the triangular tile kernels (above the
// 48 KB default for complex128), set once per device.
int trsm_attrs() {
  static bool set[64] = {};
  int dev = 0;
  RCWA_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 64 || !set[dev]) {
    RCWA_CUDA_TRY(cudaFuncSetAttribute(lu_trsm_tile_kernel<double2, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem<double2>()));
    RCWA_CUDA_TRY(cudaFuncSetAttribute(lu_trsm_tile_kernel<double2, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem<double2>()));
    RCWA_CUDA_TRY(cudaFuncSetAttribute(lu_trsm_tile_kernel<float2, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem<float2>()));
    RCWA_CUDA_TRY(cudaFuncSetAttribute(lu_trsm_tile_kernel<float2, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem<float2>()));
    if (dev < 64) set[dev] = true;
  }
  return RCWA_OK;
}

int panel_sms() {
  static int sms[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
  if (!sms[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    sms[dev] = v > 0 ? v : 1;
  }
  return sms[dev];
}

// 1. P A = L U on the A part of the augmented M, right-looking over the A
// columns only (piv receives the interchanges).
template <class T>
int lu_factor(cudaStream_t s, int n, T* M, int ld, long long stride, int batch, int* piv,
              uint32_t* status) {
  // the panel is latency-bound (one CTA per matrix, column by column): with
  // few large matrices, four times the threads per column step
  const bool wide = n >= 512 && batch < panel_sms();
  for (int j = 0; j < n; j += NB) {
    const int jb = (n - j < NB) ? (n - j) : NB;
    void* tok = prof_begin(s);
    if (wide)
      lu_panel_kernel<T, PANEL_NT_WIDE><<<batch, PANEL_NT_WIDE, 0, s>>>(M, ld, stride, n, j, jb, piv, status);
    else
      lu_panel_kernel<T, PANEL_NT><<<batch, PANEL_NT, 0, s>>>(M, ld, stride, n, j, jb, piv, status);
    prof_end(s, tok, "lu_panel");
    count_launch();
    RCWA_LAUNCH_CHECK();
    if (j > 0) {   // the earlier multipliers follow this panel's interchanges (P A = L U)
      dim3 g(cdiv_up(j, COL_NT), batch);
      lu_rowswap_kernel<T><<<g, COL_NT, 0, s>>>(M, ld, stride, n, j, j + jb, 0, j, piv);
      count_launch();
      RCWA_LAUNCH_CHECK();
    }
    const int cb = j + jb;
    if (cb < n) {
      // the panel's interchanges on the trailing columns as a pass of its
      // own (one thread per column, little register use: many columns in
      // flight to cover the sequential swaps' latency), then L11^-1
      dim3 g(cdiv_up(n - cb, COL_NT), batch);
      lu_rowswap_kernel<T><<<g, COL_NT, 0, s>>>(M, ld, stride, n, j, j + jb, cb, n, piv);
      count_launch();
      RCWA_LAUNCH_CHECK();
      if (int rc = trsm_attrs()) return rc;
      lu_trsm_tile_kernel<T, false><<<g, COL_NT, trsm_smem<T>(), s>>>(M, ld, stride, j, jb, cb, n);
      count_launch();
      RCWA_LAUNCH_CHECK();
      int rc = gemm_sub(s, n - cb, n - cb, jb, M + (long long)j * ld + cb, ld, stride,
                        M + (long long)cb * ld + j, M + (long long)cb * ld + cb, batch);
      if (rc) return rc;
    }
  }
  return RCWA_OK;
}

// The interchanges in piv composed into gather indices (overwrites piv).
int lu_compose(cudaStream_t s, int n, int* piv, int batch) {
  int rc = perm_attrs();
  if (rc) return rc;
  lu_perm_kernel<<<batch, 128, (size_t)n * sizeof(int), s>>>(piv, n);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

// 2.-4. X = U^-1 L^-1 P B for the nrhs columns that follow the A part of M,
// with the gather indices of lu_compose.
template <class T>
int lu_solve(cudaStream_t s, int n, int nrhs, T* M, int ld, long long stride, int batch, const int* idx) {
  if (nrhs <= 0) return RCWA_OK;
  if (int rc = trsm_attrs()) return rc;
  const int ncols = n + nrhs;
  T* Bc = M + (long long)n * ld;   // right-hand sides, rows 0..n-1
  {
    const int pw = (int)std::min<size_t>(PERM_WARPS, GATHER_SMEM / ((size_t)n * sizeof(T)));
    if (pw < 1) {
      set_last_error("zgesv: n=%d too large", n);
      return RCWA_ERR_INVALID;
    }
    int rc = perm_attrs();
    if (rc) return rc;
    const size_t gshm = (size_t)pw * n * sizeof(T);
    dim3 g(cdiv_up(nrhs, pw * PERM_CPW), batch);
    lu_gather_kernel<T><<<g, pw * 32, gshm, s>>>(M, ld, stride, n, n, ncols, idx);
    count_launch();
    RCWA_LAUNCH_CHECK();
  }
  // L Y = P B, then U X = Y, by recursive halving: the off-diagonal blocks
  // become GEMMs with k up to n/2, only the diagonal NB x NB blocks are
  // solved by the column kernels
  auto split = [](int r0, int r1) { return r0 + NB * (((r1 - r0 + NB - 1) / NB) / 2); };
  std::function<int(int, int)> lower = [&](int r0, int r1) -> int {
    if (r1 - r0 <= NB) {
      dim3 g(cdiv_up(nrhs, COL_NT), batch);
      lu_trsm_tile_kernel<T, false><<<g, COL_NT, trsm_smem<T>(), s>>>(M, ld, stride, r0, r1 - r0, n, ncols);
      count_launch();
      RCWA_LAUNCH_CHECK();
      return RCWA_OK;
    }
    const int mid = split(r0, r1);
    int r = lower(r0, mid);
    if (r) return r;
    r = gemm_sub(s, r1 - mid, nrhs, mid - r0, M + (long long)r0 * ld + mid, ld, stride, Bc + r0, Bc + mid,
                 batch);
    if (r) return r;
    return lower(mid, r1);
  };
  std::function<int(int, int)> upper = [&](int r0, int r1) -> int {
    if (r1 - r0 <= NB) {
      dim3 g(cdiv_up(nrhs, COL_NT), batch);
      lu_trsm_tile_kernel<T, true><<<g, COL_NT, trsm_smem<T>(), s>>>(M, ld, stride, r0, r1 - r0, n, ncols);
      count_launch();
      RCWA_LAUNCH_CHECK();
      return RCWA_OK;
    }
    const int mid = split(r0, r1);
    int r = upper(mid, r1);
    if (r) return r;
    r = gemm_sub(s, mid - r0, nrhs, r1 - mid, M + (long long)mid * ld + r0, ld, stride, Bc + mid, Bc + r0,
                 batch);
    if (r) return r;
    return upper(r0, mid);
  };
  int rc = lower(0, n);
  if (rc) return rc;
  return upper(0, n);
}

// ---------------------------------------------------------------------------
// refinement kernels (one grid row per system, grid-stride over its entries)
// ---------------------------------------------------------------------------
constexpr int IR_NT = 256;

// Mf[:, 0:ncols] = (complex64) M[:, 0:ncols]  (Mf: ld n, stride sf)
__global__ void ir_to_f32_kernel(const double2* __restrict__ Mg, int ld, long long stride,
                                 float2* __restrict__ Mf, long long sf, int n, int ncols) {
  const int b = blockIdx.y;
  const double2* M = Mg + (long long)b * stride;
  float2* F = Mf + (long long)b * sf;
  const long long total = (long long)n * ncols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / n), r = (int)(e - (long long)c * n);
    const double2 v = M[(long long)c * ld + r];
    F[e] = make_float2((float)v.x, (float)v.y);
  }
}

// X0 from the FP32 solve: R = B (FP64 right-hand sides of M), B <- (FP64) Xf
__global__ void ir_take_x0_kernel(double2* __restrict__ Mg, int ld, long long stride,
                                  double2* __restrict__ Rg, const float2* __restrict__ Xf, long long sf,
                                  int n, int nrhs) {
  const int b = blockIdx.y;
  double2* Bm = Mg + (long long)b * stride + (long long)n * ld;
  double2* R = Rg + (long long)b * n * nrhs;
  const float2* X = Xf + (long long)b * sf;
  const long long total = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / n), r = (int)(e - (long long)c * n);
    double2* bp = Bm + (long long)c * ld + r;
    R[e] = *bp;
    const float2 x = X[e];
    *bp = make_double2((double)x.x, (double)x.y);
  }
}

// Xf = (complex64) R
__global__ void ir_residual_f32_kernel(const double2* __restrict__ Rg, float2* __restrict__ Xf, long long sf,
                                       int n, int nrhs) {
  const int b = blockIdx.y;
  const double2* R = Rg + (long long)b * n * nrhs;
  float2* X = Xf + (long long)b * sf;
  const long long total = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const double2 v = R[e];
    X[e] = make_float2((float)v.x, (float)v.y);
  }
}

// B <- B + (FP64) dXf; D (optional) <- (FP64) dXf; nrm[b] = (max |dX|, max |X|)
// as order-preserving bits of non-negative floats
__global__ void __launch_bounds__(IR_NT)
ir_update_kernel(double2* __restrict__ Mg, int ld, long long stride, const float2* __restrict__ Xf,
                 long long sf, double2* __restrict__ Dg, int n, int nrhs, unsigned* __restrict__ nrm) {
  const int b = blockIdx.y;
  double2* Bm = Mg + (long long)b * stride + (long long)n * ld;
  const float2* X = Xf + (long long)b * sf;
  double2* D = Dg ? Dg + (long long)b * n * nrhs : nullptr;
  const long long total = (long long)n * nrhs;
  float mdx = 0.f, mx = 0.f;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / n), r = (int)(e - (long long)c * n);
    const float2 d = X[e];
    double2* bp = Bm + (long long)c * ld + r;
    double2 v = *bp;
    v.x += (double)d.x;
    v.y += (double)d.y;
    *bp = v;
    if (D) D[e] = make_double2((double)d.x, (double)d.y);
    mdx = fmaxf(mdx, fabsf(d.x) + fabsf(d.y));
    mx = fmaxf(mx, (float)(fabs(v.x) + fabs(v.y)));
  }
  // NaN never wins fmaxf; a non-finite solve is caught by the efficiency checks
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    mdx = fmaxf(mdx, __shfl_down_sync(0xffffffffu, mdx, off));
    mx = fmaxf(mx, __shfl_down_sync(0xffffffffu, mx, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(nrm + 2 * b, __float_as_uint(mdx));
    atomicMax(nrm + 2 * b + 1, __float_as_uint(mx));
  }
}

__global__ void ir_flag_kernel(const unsigned* __restrict__ nrm, uint32_t* __restrict__ status, int batch,
                               float tol) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  const float dx = __uint_as_float(nrm[2 * b]), x = __uint_as_float(nrm[2 * b + 1]);
  if (dx > tol * x) status[b] |= RCWA_STATUS_REFINE_SLOW;
}

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

unsigned ir_grid_x(long long per_system) {
  const long long g = (per_system + IR_NT - 1) / IR_NT;
  return (unsigned)std::min<long long>(std::max<long long>(g, 1), 64);
}

}  // namespace

int zgesv(cudaStream_t s, int n, int nrhs, double2* M, int ld, long long stride, int batch, int* piv,
          uint32_t* status) {
  if (n <= 0 || batch <= 0) return RCWA_OK;
  int rc = lu_factor<double2>(s, n, M, ld, stride, batch, piv, status);
  if (rc || nrhs <= 0) return rc;
  if ((rc = lu_compose(s, n, piv, batch))) return rc;   // piv now holds the gather indices
  return lu_solve<double2>(s, n, nrhs, M, ld, stride, batch, piv);
}

size_t zgesv_ir_ws_bytes(int n, int nrhs, int batch, int sweeps, int resid_int8) {
  if (n <= 0 || batch <= 0) return 0;
  const size_t sys = (size_t)batch * n;
  size_t b = al256(sys * (size_t)(n + nrhs) * sizeof(float2));    // complex64 [A | B]
  b += al256(sys * (size_t)nrhs * sizeof(double2));                // FP64 residual
  if (sweeps > 1) b += al256(sys * (size_t)nrhs * sizeof(double2));  // FP64 correction
  b += al256((size_t)batch * 2 * sizeof(unsigned));
  if (resid_int8) b += al256(zgemm_oz_ws_bytes(n, nrhs, n, batch, 6));
  return b + 256;
}

int zgesv_ir(cudaStream_t s, int n, int nrhs, double2* M, int ld, long long stride, int batch, int* piv,
             uint32_t* status, void* ws, int sweeps, int resid_int8) {
  if (n <= 0 || batch <= 0) return RCWA_OK;
  if (sweeps < 1) sweeps = 1;
  const long long sf = (long long)n * (n + nrhs);
  const long long sr = (long long)n * nrhs;
  char* w = (char*)(((uintptr_t)ws + 255) & ~(uintptr_t)255);
  float2* Mf = (float2*)w;
  w += al256((size_t)batch * sf * sizeof(float2));
  double2* R = (double2*)w;
  w += al256((size_t)batch * sr * sizeof(double2));
  double2* D = nullptr;
  if (sweeps > 1) {
    D = (double2*)w;
    w += al256((size_t)batch * sr * sizeof(double2));
  }
  unsigned* nrm = (unsigned*)w;
  w += al256((size_t)batch * 2 * sizeof(unsigned));
  void* ozws = resid_int8 ? (void*)w : nullptr;
  const size_t ozb = resid_int8 ? zgemm_oz_ws_bytes(n, nrhs, n, batch, 6) : 0;
  int* oz_err = nullptr;
  if (resid_int8 && !(oz_err = tc_error_flag())) {
    set_last_error("zgesv_ir: tensor-core error flag unavailable");
    return RCWA_ERR_CUDA;
  }
  int rc;
  // FP32 factorisation and first solve on the complex64 copy
  {
    dim3 g(ir_grid_x((long long)n * (n + nrhs)), batch);
    ir_to_f32_kernel<<<g, IR_NT, 0, s>>>(M, ld, stride, Mf, sf, n, n + nrhs);
    count_launch();
    RCWA_LAUNCH_CHECK();
  }
  if ((rc = lu_factor<float2>(s, n, Mf, n, sf, batch, piv, status))) return rc;
  if (nrhs <= 0) return RCWA_OK;
  if ((rc = lu_compose(s, n, piv, batch))) return rc;
  if ((rc = lu_solve<float2>(s, n, nrhs, Mf, n, sf, batch, piv))) return rc;
  const dim3 gr(ir_grid_x(sr), batch);
  float2* Xf = Mf + (long long)n * n;   // right-hand-side part of the complex64 system
  ir_take_x0_kernel<<<gr, IR_NT, 0, s>>>(M, ld, stride, R, Xf, sf, n, nrhs);
  count_launch();
  RCWA_LAUNCH_CHECK();
  // R = B - A X0 in FP64 (DMMA); A is the untouched FP64 A part of M
  auto residual = [&](const double2* X, int ldx, long long sx) {
    ZGemm gm;
    gm.m = n;
    gm.n = nrhs;
    gm.k = n;
    gm.alpha = cmk(-1.0, 0.0);
    gm.beta = cmk(1.0, 0.0);
    gm.A = M;
    gm.lda = ld;
    gm.sA = stride;
    gm.B = X;
    gm.ldb = ldx;
    gm.sB = sx;
    gm.C = R;
    gm.ldc = n;
    gm.sC = sr;
    gm.batch = batch;
    if (resid_int8) {   // residuals on the int8-slice GEMM with six digits (~43 bits)
      gm.tc = TC_INT8;
      gm.digits = 6;
      gm.ws = ozws;
      gm.ws_bytes = ozb;
      return zgemm_oz(s, gm, oz_err);
    }
    return zgemm(s, gm);
  };
  if ((rc = residual(M + (long long)n * ld, ld, stride))) return rc;
  for (int it = 0; it < sweeps; ++it) {
    const bool last = it + 1 == sweeps;
    ir_residual_f32_kernel<<<gr, IR_NT, 0, s>>>(R, Xf, sf, n, nrhs);
    count_launch();
    RCWA_LAUNCH_CHECK();
    if ((rc = lu_solve<float2>(s, n, nrhs, Mf, n, sf, batch, piv))) return rc;
    if (last) RCWA_CUDA_TRY(cudaMemsetAsync(nrm, 0, (size_t)batch * 2 * sizeof(unsigned), s));
    ir_update_kernel<<<gr, IR_NT, 0, s>>>(M, ld, stride, Xf, sf, last ? nullptr : D, n, nrhs, nrm);
    count_launch();
    RCWA_LAUNCH_CHECK();
    // R <- R - A dX: the residual of the corrected X without a copy of B
    if (!last && (rc = residual(D, n, sr))) return rc;
  }
  ir_flag_kernel<<<cdiv_up(batch, 128), 128, 0, s>>>(nrm, status, batch, 1e-4f);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

}  // namespace rcwa
