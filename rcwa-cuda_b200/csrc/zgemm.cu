// Batched complex128 GEMM.
//
//   C[b] = alpha * diag(dl[b]) * A[b] * B[b] * diag(dr[b]) + beta * C[b]
//
// Column-major, arbitrary m/n/k/ld/batch strides.  This is the dense
// contraction behind every Eigen operator* of the reference's S-matrix algebra
// (rcwa.cpp:288, 326, 346-348, 602-611).  The optional diagonal scalings fold
// the reference's asDiagonal() products (rcwa.cpp:273-285, 329, 339) into the
// epilogue so no dense diagonal matrix is ever materialised.
//
// FP64 kernels chosen per shape bucket by a measured table
// (rcwa_set_gemm_table): the FP64 tensor-core (DMMA) kernel with tiles staged
// by cp.async (16-byte copies, zero-filled outside the matrix; 64 x 64 or
// 32 x 64 complex tiles), the same DMMA
// tiling fed by the tensor memory accelerator (products of operands as
// stored), and a CUDA-core kernel (64x64 C tile, K step 8, 256 threads as
// 16x16, each a 4x4 complex micro-tile).  tcgen05 has no FP64 kind, so FP64
// tensor work on sm_100a is mma.sync DMMA.
#include <atomic>
#include <cstring>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {

constexpr int BM = 64, BN = 64, BK = 8, NT = 256;
// DMMA kernel shape: WM warps along M (CTA tile 32 WM x 64), ST pipeline stages
#ifndef RCWA_DMMA_WM
#define RCWA_DMMA_WM 2
#endif
#ifndef RCWA_DMMA_ST
#define RCWA_DMMA_ST 4
#endif
#ifndef RCWA_DMMA_TMA_ST
#define RCWA_DMMA_TMA_ST 4
#endif

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
  int src_bytes = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(gmem),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// OPA / OPB: 0 = the operand as stored, 1 = its conjugate transpose.
// MI = complex rows per thread: the CTA tile is (16 MI) x 64.
template <int OPA, int OPB, int MI>
__global__ void __launch_bounds__(NT, (MI > 4 ? 1 : 2))
zgemm_kernel(int m, int n, int k, double2 alpha, const double2* __restrict__ A, int lda,
             long long sA, const double2* __restrict__ B, int ldb, long long sB, double2 beta,
             double2* __restrict__ C, int ldc, long long sC, const double2* __restrict__ dl,
             long long sdl, const double2* __restrict__ dr, long long sdr) {
  constexpr int TM = 16 * MI;
  __shared__ __align__(16) double2 As[2][BK][TM];
  __shared__ __align__(16) double2 Bs[2][BK][BN];

  const int b = blockIdx.z;
  A += (long long)b * sA;
  B += (long long)b * sB;
  C += (long long)b * sC;
  const int m0 = blockIdx.y * TM;
  const int n0 = blockIdx.x * BN;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;

  // C += +-A B (alpha = +-1, no diagonal scalings, beta != 0: the LU and
  // Hessenberg rank-k updates): the accumulators start from +-beta C, read
  // before the k loop so that the read overlaps the first tile loads instead
  // of stalling the epilogue; the result is then sgn * acc.
  const bool pre = !dl && !dr && (beta.x != 0.0 || beta.y != 0.0) && alpha.y == 0.0 &&
                   (alpha.x == 1.0 || alpha.x == -1.0);
  const double sgn = pre ? alpha.x : 1.0;
  double2 acc[MI][4];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      acc[i][j] = cmk(0.0, 0.0);
      const int row = m0 + tx + 16 * i, col = n0 + ty + 16 * j;
      if (pre && row < m && col < n) {
        const double2 c0 = cmul(beta, C[(long long)col * ldc + row]);
        acc[i][j] = cmk(sgn * c0.x, sgn * c0.y);
      }
    }

  auto load_tile = [&](int buf, int k0) {
    // A tile: TM rows x 8 k (consecutive threads walk the contiguous index)
#pragma unroll
    for (int h = 0; h < TM * BK / NT; ++h) {
      const int e = tid + h * NT;
      const int r = OPA ? (e >> 3) : (e % TM), kk = OPA ? (e & 7) : (e / TM);
      const int gr = m0 + r, gk = k0 + kk;
      const bool pa = (gr < m) && (gk < k);
      const double2* srcA = pa ? (OPA ? A + (long long)gr * lda + gk : A + (long long)gk * lda + gr) : A;
      cp_async16(&As[buf][kk][r], srcA, pa);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int e = tid + h * NT;
      // B tile: 8 k x 64 cols
      {
        const int kb = OPB ? (e >> 6) : (e & 7), c = OPB ? (e & 63) : (e >> 3);
        const int gk2 = k0 + kb, gc = n0 + c;
        const bool pb = (gk2 < k) && (gc < n);
        const double2* srcB = pb ? (OPB ? B + (long long)gk2 * ldb + gc : B + (long long)gc * ldb + gk2) : B;
        cp_async16(&Bs[buf][kb][c], srcB, pb);
      }
    }
    cp_async_commit();
  };

  const int ktiles = (k + BK - 1) / BK;
  if (ktiles > 0) load_tile(0, 0);
  for (int t = 0; t < ktiles; ++t) {
    const int buf = t & 1;
    if (t + 1 < ktiles) {
      load_tile(buf ^ 1, (t + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double2 a[MI], bb[4];
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        a[i] = As[buf][kk][tx + 16 * i];
        if (OPA) a[i].y = -a[i].y;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        bb[j] = Bs[buf][kk][ty + 16 * j];
        if (OPB) bb[j].y = -bb[j].y;
      }
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cfma(acc[i][j], a[i], bb[j]);
    }
    __syncthreads();
  }

  const bool use_beta = (beta.x != 0.0 || beta.y != 0.0);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int col = n0 + ty + 16 * j;
    if (col >= n) continue;
    double2 sr = dr ? dr[(long long)b * sdr + col] : cmk(1.0, 0.0);
#pragma unroll
    for (int i = 0; i < MI; ++i) {
      int row = m0 + tx + 16 * i;
      if (row >= m) continue;
      double2* cp = C + (long long)col * ldc + row;
      if (pre) {
        *cp = cmk(sgn * acc[i][j].x, sgn * acc[i][j].y);
        continue;
      }
      double2 v = cmul(alpha, acc[i][j]);
      if (dl) v = cmul(dl[(long long)b * sdl + row], v);
      if (dr) v = cmul(v, sr);
      if (use_beta) v = cadd(v, cmul(beta, *cp));
      *cp = v;
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core kernel: mma.sync m8n8k4 f64 (DMMA).  64x64 CTA tile, K step
// 8, a 4-stage cp.async pipeline; 4 warps in a 2x2 grid, each computing a 32x32
// complex tile as 4x4 blocks of 8x8.  A complex 8x8x4 block product is four
// real DMMAs:  Cr += Ar Br + (-Ai) Bi,  Ci += Ar Bi + Ai Br.
// Fragment layout of m8n8k4.f64: A(row = lane/4, k = lane%4),
// B(k = lane%4, col = lane/4), C(row = lane/4, cols 2*(lane%4) + {0,1}).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c[0]), "+d"(c[1])
      : "d"(a), "d"(b));
}

// Thin strips: when m (or n) is a little above a multiple of the 64-wide
// tile (n = 450 = 7 * 64 + 2), a last row of 64-wide tiles would hold only a
// few live rows and still cost nearly a full tile (its loads and pipeline do
// not shrink).  The DMMA launch then tiles the 64-aligned part and gives the
// last rows (ROWS = 1, all n columns) and columns (ROWS = 0, the aligned
// rows), at most 16 of each, to extra CTAs of the same grid, which run this
// GEMV-like pass alongside the tensor-core tiles.  One call: the output
// block rows [r0, r1) x cols [c0, c1), at most 64 along the long side and 16
// along the short one; k staged through shared memory (sm: 16 x 65 + 16 x 17
// double2) in steps of 16, loads coalesced along whichever index is
// contiguous in memory; thread t owns long index t % 64 and short indices
// SPT (t / 64) + {0..SPT-1}.  A, B, C, dl, dr point at this batch item.
template <int OPA, int OPB, int ROWS, int NTH>
__device__ __forceinline__ void thin_tile(int r0, int r1, int c0, int c1, int k, double2 alpha,
                                          const double2* __restrict__ A, int lda,
                                          const double2* __restrict__ B, int ldb, double2 beta,
                                          double2* __restrict__ C, int ldc,
                                          const double2* __restrict__ dl,
                                          const double2* __restrict__ dr, double2* sm) {
  constexpr int TK = 16, TL = 64, TS = 16, SPT = TS / (NTH / TL);
  double2 (*Ls)[TL + 1] = reinterpret_cast<double2 (*)[TL + 1]>(sm);                 // [k][long]
  double2 (*Ss)[TS + 1] = reinterpret_cast<double2 (*)[TS + 1]>(sm + TK * (TL + 1));  // [k][short]
  const int nl = ROWS ? c1 - c0 : r1 - r0, ns = ROWS ? r1 - r0 : c1 - c0;
  const int tid = threadIdx.x, li = tid % TL, sg = tid / TL;
  // A(i, kk) and B(kk, j) with the operand ops applied, 0 outside the block
  auto a_at = [&](int i, int kk) -> double2 {
    if (i >= r1 || kk >= k) return cmk(0.0, 0.0);
    return OPA ? cconj(A[(long long)i * lda + kk]) : A[(long long)kk * lda + i];
  };
  auto b_at = [&](int kk, int j) -> double2 {
    if (kk >= k || j >= c1) return cmk(0.0, 0.0);
    return OPB ? cconj(B[(long long)kk * ldb + j]) : B[(long long)j * ldb + kk];
  };
  double2 acc[SPT];
#pragma unroll
  for (int q = 0; q < SPT; ++q) acc[q] = cmk(0.0, 0.0);
  for (int k0 = 0; k0 < k; k0 += TK) {
#pragma unroll
    for (int h = 0; h < TK * TL / NTH; ++h) {   // long operand, 64 x 16
      const int e = tid + NTH * h;
      if (ROWS) {
        const bool kfast = !OPB;   // B(kk, j) runs along kk in memory unless transposed
        const int kk = kfast ? e % TK : e / TL, l = kfast ? e / TK : e % TL;
        Ls[kk][l] = b_at(k0 + kk, c0 + l);
      } else {
        const bool kfast = OPA;    // A(i, kk) runs along i in memory unless transposed
        const int kk = kfast ? e % TK : e / TL, l = kfast ? e / TK : e % TL;
        Ls[kk][l] = a_at(r0 + l, k0 + kk);
      }
    }
#pragma unroll
    for (int h = 0; h < TK * TS / NTH; ++h) {   // short operand, 16 x 16
      const int e = tid + NTH * h;
      if (ROWS) {
        const bool kfast = OPA;
        const int kk = kfast ? e % TK : e / TS, q = kfast ? e / TK : e % TS;
        Ss[kk][q] = a_at(r0 + q, k0 + kk);
      } else {
        const bool kfast = !OPB;
        const int kk = kfast ? e % TK : e / TS, q = kfast ? e / TK : e % TS;
        Ss[kk][q] = b_at(k0 + kk, c0 + q);
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      const double2 lv = Ls[kk][li];
#pragma unroll
      for (int q = 0; q < SPT; ++q) {
        const double2 sv = Ss[kk][sg * SPT + q];
        acc[q].x = fma(lv.x, sv.x, fma(-lv.y, sv.y, acc[q].x));
        acc[q].y = fma(lv.x, sv.y, fma(lv.y, sv.x, acc[q].y));
      }
    }
    __syncthreads();
  }
  if (li >= nl) return;
  const bool use_beta = (beta.x != 0.0 || beta.y != 0.0);
#pragma unroll
  for (int q = 0; q < SPT; ++q) {
    const int sidx = sg * SPT + q;
    if (sidx >= ns) continue;
    const int row = ROWS ? r0 + sidx : r0 + li, col = ROWS ? c0 + li : c0 + sidx;
    double2 v = cmul(alpha, acc[q]);
    if (dl) v = cmul(dl[row], v);
    if (dr) v = cmul(v, dr[col]);
    double2* cp = C + (long long)col * ldc + row;
    if (use_beta) v = cadd(v, cmul(beta, *cp));
    *cp = v;
  }
}

// WM warps along M x 2 along N, each a 32x32 complex tile: CTA tile
// (32 WM) x 64, 64 WM threads.  The tiles cover rows [0, m) x cols [0, n);
// with mf > m or nf > n, the first thin_rows rows of the grid are thin-strip
// CTAs for rows [m, mf) x cols [0, nf) and rows [0, m) x cols [n, nf).
template <int OPA, int OPB, int WM, int ST>
__global__ void __launch_bounds__(64 * WM, (WM > 2 ? 1 : 2))
zgemm_dmma_kernel(int m, int n, int k, double2 alpha, const double2* __restrict__ A, int lda,
                  long long sA, const double2* __restrict__ B, int ldb, long long sB, double2 beta,
                  double2* __restrict__ C, int ldc, long long sC, const double2* __restrict__ dl,
                  long long sdl, const double2* __restrict__ dr, long long sdr, int mf, int nf,
                  int thin_rows) {
  constexpr int DT = 64 * WM, TM = 32 * WM;
  // rows padded by two elements: the fragment loads (4 k x 8 rows per
  // quarter-warp pattern) then hit distinct shared-memory banks
  constexpr int TMP = TM + 2, BNP = BN + 2;
  extern __shared__ __align__(16) double2 dsm[];
  double2 (*As)[BK][TMP] = reinterpret_cast<double2 (*)[BK][TMP]>(dsm);
  double2 (*Bs)[BK][BNP] = reinterpret_cast<double2 (*)[BK][BNP]>(dsm + ST * BK * TMP);
  const int b = blockIdx.z;
  A += (long long)b * sA;
  B += (long long)b * sB;
  C += (long long)b * sC;
  if ((int)blockIdx.y < thin_rows) {   // thin-strip CTA (the whole CTA takes this branch)
    const int t = blockIdx.y * gridDim.x + blockIdx.x;
    const int nrow = mf > m ? (nf + 63) / 64 : 0, ncol = nf > n ? (m + 63) / 64 : 0;
    const double2* dlb = dl ? dl + (long long)b * sdl : nullptr;
    const double2* drb = dr ? dr + (long long)b * sdr : nullptr;
    if (t < nrow)
      thin_tile<OPA, OPB, 1, DT>(m, mf, t * 64, min(nf, t * 64 + 64), k, alpha, A, lda, B, ldb, beta, C, ldc,
                                 dlb, drb, dsm);
    else if (t < nrow + ncol)
      thin_tile<OPA, OPB, 0, DT>((t - nrow) * 64, min(m, (t - nrow) * 64 + 64), n, nf, k, alpha, A, lda, B,
                                 ldb, beta, C, ldc, dlb, drb, dsm);
    return;
  }
  const int m0 = (blockIdx.y - thin_rows) * TM, n0 = blockIdx.x * BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WM, wn = warp / WM;
  const int lr = lane >> 2, lk = lane & 3;
  // 8x8 blocks of this warp that hold any row < m / column < n (warp-uniform):
  // edge tiles skip the products of blocks entirely outside the matrix
  int live_i = 0, live_j = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    live_i |= (m0 + wm * 32 + q * 8 < m) ? (1 << q) : 0;
    live_j |= (n0 + wn * 32 + q * 8 < n) ? (1 << q) : 0;
  }

  // C += +-A B (alpha = +-1, no diagonal scalings, beta != 0: the LU and
  // Hessenberg rank-k updates): the accumulators start from +-beta C, read
  // before the k loop so that the read overlaps the first tile loads; the
  // result is then sgn * acc
  const bool pre = !dl && !dr && (beta.x != 0.0 || beta.y != 0.0) && alpha.y == 0.0 &&
                   (alpha.x == 1.0 || alpha.x == -1.0);
  const double sgn = pre ? alpha.x : 1.0;
  double cr[4][4][2], ci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        cr[i][j][q] = ci[i][j][q] = 0.0;
        const int row = m0 + wm * 32 + i * 8 + lr, col = n0 + wn * 32 + j * 8 + lk * 2 + q;
        if (pre && row < m && col < n) {
          const double2 c0 = cmul(beta, C[(long long)col * ldc + row]);
          cr[i][j][q] = sgn * c0.x;
          ci[i][j][q] = sgn * c0.y;
        }
      }

  auto load_tile = [&](int buf, int k0) {
#pragma unroll
    for (int h = 0; h < TM * BK / DT; ++h) {
      const int e = tid + h * DT;
      const int r = OPA ? (e >> 3) : (e % TM), kk = OPA ? (e & 7) : (e / TM);
      const int gr = m0 + r, gk = k0 + kk;
      const bool pa = (gr < m) && (gk < k);
      const double2* srcA = pa ? (OPA ? A + (long long)gr * lda + gk : A + (long long)gk * lda + gr) : A;
      cp_async16(&As[buf][kk][r], srcA, pa);
    }
#pragma unroll
    for (int h = 0; h < BN * BK / DT; ++h) {
      const int e = tid + h * DT;
      const int kb = OPB ? (e >> 6) : (e & 7), c = OPB ? (e & 63) : (e >> 3);
      const int gk2 = k0 + kb, gc = n0 + c;
      const bool pb = (gk2 < k) && (gc < n);
      const double2* srcB = pb ? (OPB ? B + (long long)gk2 * ldb + gc : B + (long long)gc * ldb + gk2) : B;
      cp_async16(&Bs[buf][kb][c], srcB, pb);
    }
    cp_async_commit();
  };

  // ST-stage cp.async pipeline: tiles t+1 .. t+ST-1 are in flight while
  // tile t is consumed (an empty group is committed past the end so the
  // wait count stays fixed)
  const int ktiles = (k + BK - 1) / BK;
#pragma unroll
  for (int p = 0; p < ST - 1; ++p) {
    if (p < ktiles) load_tile(p, p * BK);
    else cp_async_commit();
  }
  for (int t = 0; t < ktiles; ++t) {
    const int buf = t % ST;
    cp_async_wait<ST - 2>();
    __syncthreads();
    {
      const int tn = t + ST - 1;   // refills the buffer consumed at t-1
      if (tn < ktiles) load_tile(tn % ST, tn * BK);
      else cp_async_commit();
    }
#pragma unroll
    for (int kq = 0; kq < BK / 4; ++kq) {
      double ar[4], ai[4], nai[4], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 v = As[buf][kq * 4 + lk][wm * 32 + i * 8 + lr];
        ar[i] = v.x;
        ai[i] = OPA ? -v.y : v.y;
        nai[i] = -ai[i];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 v = Bs[buf][kq * 4 + lk][wn * 32 + j * 8 + lr];
        br[j] = v.x;
        bi[j] = OPB ? -v.y : v.y;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (!((live_i >> i) & (live_j >> j) & 1)) continue;   // block beyond m or n
          dmma(cr[i][j], ar[i], br[j]);
          dmma(cr[i][j], nai[i], bi[j]);
          dmma(ci[i][j], ar[i], bi[j]);
          dmma(ci[i][j], ai[i], br[j]);
        }
    }
  }

  const bool use_beta = (beta.x != 0.0 || beta.y != 0.0);
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int col = n0 + wn * 32 + j * 8 + lk * 2 + q;
      if (col >= n) continue;
      const double2 sr = dr ? dr[(long long)b * sdr + col] : cmk(1.0, 0.0);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int row = m0 + wm * 32 + i * 8 + lr;
        if (row >= m) continue;
        double2* cpre = C + (long long)col * ldc + row;
        if (pre) {
          *cpre = cmk(sgn * cr[i][j][q], sgn * ci[i][j][q]);
          continue;
        }
        double2 v = cmul(alpha, cmk(cr[i][j][q], ci[i][j][q]));
        if (dl) v = cmul(dl[(long long)b * sdl + row], v);
        if (dr) v = cmul(v, sr);
        double2* cp = C + (long long)col * ldc + row;
        if (use_beta) v = cadd(v, cmul(beta, *cp));
        *cp = v;
      }
    }
}

// ---------------------------------------------------------------------------
// TMA-fed DMMA kernel (C = A B with both operands as stored, the form of
// every S-matrix product and of the LU / Hessenberg rank-k updates).  Same
// warp tiling and DMMA sequence as zgemm_dmma_kernel; the operand tiles come
// from the tensor memory accelerator (cp.async.bulk.tensor.3d, 128-byte
// swizzle, zero fill outside the matrix) into an ST-stage ring guarded by
// mbarriers: "full" completes when a stage's bytes have landed, "empty" when
// every warp has read it.  Lane 0 of each warp issues its share of every
// stage (A boxes g = warp, warp + NW, ...; a 64 / NW-column slice of B): the
// first ST stages up front, then, after the warp's k-tile t, the refill of
// the stage of k-tile t-1 once every warp has released it.  No CTA-wide
// barrier sits in the k loop and the copy issue is spread over the warps.
//
// Stage layout (k-tile of BK = 8):
//   A: TM / 8 boxes of 8 rows x 8 k, 1 KB each; box row kk (one k) is 128
//      bytes = 8 complex rows, its 16-byte chunk r stored at chunk r ^ kk;
//   B: 64 columns x 8 k, column c is a 128-byte row, chunk kk at kk ^ (c & 7).
// A DMMA k-step kq (0, 1) takes k = 2 lk + kq for lane k-index lk: the eight
// lanes of a quarter warp (two rows or columns x four k) then read eight
// distinct 16-byte chunks, free of bank conflicts.  The permutation of k is
// the same for A and B, so the products sum the same terms.
//
// Every mbarrier wait is bounded (about a second); if one runs out, each
// warp waits (bounded) for its copies still in flight, the CTA sets the
// device error flag and writes NaN over its tile of C, so both precisions
// report the failure (error flag, non-finite status) and the context stays
// usable.
// ---------------------------------------------------------------------------
constexpr long long DMMA_WAIT_CYCLES = 2000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init_n(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive1(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > DMMA_WAIT_CYCLES) return false;
  }
}
// one box of a 3-D tensor map (x innermost, in FP64 elements) into shared memory
__device__ __forceinline__ void tma_load3(void* sdst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(sdst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

template <int WM, int ST>
struct TmaCfg {
  static constexpr int TM = 32 * WM, NW = 2 * WM;
  static constexpr int A_BYTES = TM * BK * 16, B_BYTES = BN * BK * 16, STAGE = A_BYTES + B_BYTES;
  static constexpr int B_COLS = BN / NW;            // B columns per warp's copy
  static constexpr int SMEM = ST * STAGE + 1024;   // + slack to align the ring to 1024 bytes
};

// tmA: (2 m doubles, k, batch or 1) with box (16, 8, 1); tmB: (2 k doubles,
// n, batch or 1) with box (16, 64 / NW, 1); za / zb: 1 when the operand has
// a batch stride (else every item reads z = 0).
template <int WM, int ST>
__global__ void __launch_bounds__(64 * WM, (WM > 2 ? 1 : 2))
zgemm_dmma_tma_kernel(int m, int n, int k, double2 alpha, const __grid_constant__ CUtensorMap tmA,
                      const __grid_constant__ CUtensorMap tmB, int za, int zb,
                      const double2* __restrict__ A, int lda, long long sA, const double2* __restrict__ B,
                      int ldb, long long sB, double2 beta, double2* __restrict__ C, int ldc, long long sC,
                      const double2* __restrict__ dl, long long sdl, const double2* __restrict__ dr,
                      long long sdr, int mf, int nf, int thin_rows, int* __restrict__ err,
                      int skip_first_copy) {
  using Cfg = TmaCfg<WM, ST>;
  constexpr int TM = Cfg::TM, NW = Cfg::NW;
  extern __shared__ __align__(16) uint8_t dsm_raw[];
  __shared__ __align__(8) uint64_t full[ST], empty[ST];
  uint8_t* ring = (uint8_t*)(((uintptr_t)dsm_raw + 1023) & ~(uintptr_t)1023);
  const int b = blockIdx.z;
  A += (long long)b * sA;
  B += (long long)b * sB;
  C += (long long)b * sC;
  if ((int)blockIdx.y < thin_rows) {   // thin-strip CTA, as in zgemm_dmma_kernel
    const int t = blockIdx.y * gridDim.x + blockIdx.x;
    const int nrow = mf > m ? (nf + 63) / 64 : 0, ncol = nf > n ? (m + 63) / 64 : 0;
    const double2* dlb = dl ? dl + (long long)b * sdl : nullptr;
    const double2* drb = dr ? dr + (long long)b * sdr : nullptr;
    double2* scratch = reinterpret_cast<double2*>(ring);
    if (t < nrow)
      thin_tile<0, 0, 1, 64 * WM>(m, mf, t * 64, min(nf, t * 64 + 64), k, alpha, A, lda, B, ldb, beta, C, ldc,
                                  dlb, drb, scratch);
    else if (t < nrow + ncol)
      thin_tile<0, 0, 0, 64 * WM>((t - nrow) * 64, min(m, (t - nrow) * 64 + 64), n, nf, k, alpha, A, lda, B,
                                  ldb, beta, C, ldc, dlb, drb, scratch);
    return;
  }
  const int m0 = (blockIdx.y - thin_rows) * TM, n0 = blockIdx.x * BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WM, wn = warp / WM;
  const int lr = lane >> 2, lk = lane & 3;
  int live_i = 0, live_j = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    live_i |= (m0 + wm * 32 + q * 8 < m) ? (1 << q) : 0;
    live_j |= (n0 + wn * 32 + q * 8 < n) ? (1 << q) : 0;
  }
  // A boxes (8-row groups) of this tile that hold any row < m; this warp
  // copies boxes warp, warp + NW, ... of them and its slice of B
  const int nbox = min(TM / 8, (m - m0 + 7) / 8);
  // (boxes wholly outside the matrix are not copied: the DMMAs of their
  // 8 x 8 blocks are skipped through live_i / live_j)
  const int my_boxes = nbox > warp ? (nbox - warp + NW - 1) / NW : 0;
  const bool my_b = n0 + warp * Cfg::B_COLS < n;
  const uint32_t warp_tx = (uint32_t)(my_boxes * 1024 + (my_b ? Cfg::B_BYTES / NW : 0));
  const int ktiles = (k + BK - 1) / BK;
  const int az = za ? b : 0, bzc = zb ? b : 0;

  if (tid == 0) {
    for (int st = 0; st < ST; ++st) {
      mbar_init_n(&full[st], NW);
      mbar_init_n(&empty[st], NW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  __syncthreads();

  int pending[ST];   // lane 0: per stage, the k-tile whose copies are in flight and not yet waited for, or -1
#pragma unroll
  for (int st = 0; st < ST; ++st) pending[st] = -1;
  auto issue = [&](int t) {   // lane 0 only
    const int st = t % ST;
    if (t == 0 && skip_first_copy) return;   // test hook: k-tile 0 never arrives
    uint8_t* sa = ring + st * Cfg::STAGE;
    mbar_expect_tx(&full[st], warp_tx);
    for (int g = warp; g < nbox; g += NW) tma_load3(sa + g * 1024, &tmA, 2 * (m0 + 8 * g), t * BK, az, &full[st]);
    if (my_b)
      tma_load3(sa + Cfg::A_BYTES + warp * Cfg::B_COLS * 128, &tmB, 2 * t * BK, n0 + warp * Cfg::B_COLS, bzc,
                &full[st]);
    pending[st] = t;
  };
  if (lane == 0)
    for (int p = 0; p < ST && p < ktiles; ++p) issue(p);

  // C += +-A B: accumulators start from +-beta C (as in zgemm_dmma_kernel)
  const bool pre = !dl && !dr && (beta.x != 0.0 || beta.y != 0.0) && alpha.y == 0.0 &&
                   (alpha.x == 1.0 || alpha.x == -1.0);
  const double sgn = pre ? alpha.x : 1.0;
  double cr[4][4][2], ci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        cr[i][j][q] = ci[i][j][q] = 0.0;
        const int row = m0 + wm * 32 + i * 8 + lr, col = n0 + wn * 32 + j * 8 + lk * 2 + q;
        if (pre && row < m && col < n) {
          const double2 c0 = cmul(beta, C[(long long)col * ldc + row]);
          cr[i][j][q] = sgn * c0.x;
          ci[i][j][q] = sgn * c0.y;
        }
      }

  bool ok = true;
  for (int t = 0; t < ktiles; ++t) {
    const int st = t % ST;
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full[st], (uint32_t)((t / ST) & 1)))) {
      ok = false;
      break;
    }
    if (lane == 0) pending[st] = -1;
    const uint8_t* sa = ring + st * Cfg::STAGE;
    const uint8_t* sb = sa + Cfg::A_BYTES;
#pragma unroll
    for (int kq = 0; kq < BK / 4; ++kq) {
      const int kk = 2 * lk + kq;
      double ar[4], ai[4], nai[4], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 v =
            *reinterpret_cast<const double2*>(sa + (wm * 4 + i) * 1024 + kk * 128 + ((lr ^ kk) << 4));
        ar[i] = v.x;
        ai[i] = v.y;
        nai[i] = -v.y;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 v = *reinterpret_cast<const double2*>(sb + (wn * 32 + j * 8 + lr) * 128 + ((kk ^ lr) << 4));
        br[j] = v.x;
        bi[j] = v.y;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (!((live_i >> i) & (live_j >> j) & 1)) continue;
          dmma(cr[i][j], ar[i], br[j]);
          dmma(cr[i][j], nai[i], bi[j]);
          dmma(ci[i][j], ar[i], bi[j]);
          dmma(ci[i][j], ai[i], br[j]);
        }
    }
    __syncwarp();
    bool pok = true;
    if (lane == 0) {
      mbar_arrive1(&empty[st]);
      if (t >= 1 && t - 1 + ST < ktiles) {
        if (mbar_wait_bounded(&empty[(t - 1) % ST], (uint32_t)(((t - 1) / ST) & 1))) issue(t - 1 + ST);
        else pok = false;
      }
    }
    if (!__shfl_sync(0xffffffffu, (int)pok, 0)) {
      ok = false;
      break;
    }
  }
  ok = __syncthreads_and(ok);
  if (!ok) {
    if (lane == 0) {
      for (int st = 0; st < ST; ++st)
        if (pending[st] >= 0) mbar_wait_bounded(&full[st], (uint32_t)((pending[st] / ST) & 1));
      if (warp == 0) atomicOr(err, 1);
    }
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int row = m0 + wm * 32 + i * 8 + lr, col = n0 + wn * 32 + j * 8 + lk * 2 + q;
          if (row < m && col < n) C[(long long)col * ldc + row] = cmk(nan, nan);
        }
    return;
  }

  const bool use_beta = (beta.x != 0.0 || beta.y != 0.0);
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int col = n0 + wn * 32 + j * 8 + lk * 2 + q;
      if (col >= n) continue;
      const double2 sr = dr ? dr[(long long)b * sdr + col] : cmk(1.0, 0.0);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int row = m0 + wm * 32 + i * 8 + lr;
        if (row >= m) continue;
        double2* cp = C + (long long)col * ldc + row;
        if (pre) {
          *cp = cmk(sgn * cr[i][j][q], sgn * ci[i][j][q]);
          continue;
        }
        double2 v = cmul(alpha, cmk(cr[i][j][q], ci[i][j][q]));
        if (dl) v = cmul(dl[(long long)b * sdl + row], v);
        if (dr) v = cmul(v, sr);
        if (use_beta) v = cadd(v, cmul(beta, *cp));
        *cp = v;
      }
    }
}

// Rows / columns past the last multiple of 64 that go to thin-strip CTAs
// (0: the tensor-core tiles cover them).  RCWA_ZGEMM_THIN=0 (read once)
// keeps whole 64-wide tiles everywhere.
int thin_cut(int extent) {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("RCWA_ZGEMM_THIN");
    on = (e && strcmp(e, "0") == 0) ? 0 : 1;
  }
  const int r = extent % 64;
  return (on && extent > 64 && r != 0 && r <= 16) ? r : 0;
}

// Kernel choice per shape bucket: k in (<=16, <=32, <=64, <=128, more) by
// min(m, n) in (<=64, <=128, <=256, <=512, more); entry 0 = DMMA kernel fed
// by cp.async (64 x 64 tiles), 1 = CUDA-core kernel, 2 = DMMA kernel fed by
// TMA (products with both operands as stored; the others take entry 0's
// kernel), 3 = DMMA kernel fed by cp.async with 32 x 64 tiles (two warps),
// -1 = the built-in rule (DMMA for k > 64, CUDA cores for the rank-k
// updates).  A measured table comes from the tuner (rcwa_set_gemm_table);
// RCWA_ZGEMM=ffma, =dmma, =tma or =dmma32 (read once) forces one kernel for
// every shape.
std::atomic<int> g_gemm_table[25];
std::atomic<bool> g_gemm_table_init{false};

int gemm_bucket_k(int k) { return k <= 16 ? 0 : k <= 32 ? 1 : k <= 64 ? 2 : k <= 128 ? 3 : 4; }
int gemm_bucket_mn(int m, int n) {
  const int s = m < n ? m : n;
  return s <= 64 ? 0 : s <= 128 ? 1 : s <= 256 ? 2 : s <= 512 ? 3 : 4;
}

int gemm_impl(int m, int n, int k) {
  static int forced = -2;
  if (forced == -2) {
    const char* e = getenv("RCWA_ZGEMM");
    forced = !e                           ? -1
             : strcmp(e, "ffma") == 0     ? 1
             : strcmp(e, "dmma") == 0     ? 0
             : strcmp(e, "tma") == 0      ? 2
             : strcmp(e, "dmma32") == 0   ? 3
                                          : -1;
  }
  if (forced >= 0) return forced;
  if (g_gemm_table_init.load()) {
    const int c = g_gemm_table[gemm_bucket_k(k) * 5 + gemm_bucket_mn(m, n)].load();
    if (c >= 0 && c <= 3) return c;
  }
  return k > 64 ? 0 : 1;
}

// cuTensorMapEncodeTiled from the driver, through the runtime's entry-point
// query (the library links only the runtime); null when unavailable.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// 3-D FP64 tensor map (d0 innermost) with a (b0, b1, 1) box and the 128-byte
// swizzle; false when the driver rejects it (the caller then uses cp.async).
bool make_tensor_map(CUtensorMap* map, const void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t s1,
                     uint64_t s2, uint32_t b0, uint32_t b1) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)base & 15) || (s1 & 15) || (s2 & 15) || s1 >= (1ull << 40) || s2 >= (1ull << 40))
    return false;
  const cuuint64_t dims[3] = {d0, d1, d2};
  const cuuint64_t strides[2] = {s1, s2};
  const cuuint32_t box[3] = {b0, b1, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Launches the TMA-fed kernel; *launched stays false (nothing queued) when a
// tensor map cannot be made or the device flag is unavailable.
template <int WM, int ST>
int launch_dmma_tma(cudaStream_t s, const ZGemm& g, dim3 grid, int mm, int nm, int kk, int thin_rows,
                    bool* launched) {
  using Cfg = TmaCfg<WM, ST>;
  *launched = false;
  int* err = tc_error_flag();
  if (!err) return RCWA_OK;
  const bool za = g.batch > 1 && g.sA != 0, zb = g.batch > 1 && g.sB != 0;
  const uint64_t k1 = kk > 0 ? (uint64_t)kk : 1;
  alignas(64) CUtensorMap tmA, tmB;
  if (!make_tensor_map(&tmA, g.A, 2ull * mm, k1, za ? (uint64_t)g.batch : 1, (uint64_t)g.lda * 16,
                       za ? (uint64_t)g.sA * 16 : (uint64_t)g.lda * 16 * k1, 16, BK))
    return RCWA_OK;
  if (!make_tensor_map(&tmB, g.B, 2 * k1, (uint64_t)nm, zb ? (uint64_t)g.batch : 1, (uint64_t)g.ldb * 16,
                       zb ? (uint64_t)g.sB * 16 : (uint64_t)g.ldb * 16 * nm, 2 * BK, Cfg::B_COLS))
    return RCWA_OK;
  static bool attr[64] = {};   // per device
  int dev = 0;
  RCWA_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 64 || !attr[dev]) {
    RCWA_CUDA_TRY(cudaFuncSetAttribute(zgemm_dmma_tma_kernel<WM, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       Cfg::SMEM));
    if (dev < 64) attr[dev] = true;
  }
  zgemm_dmma_tma_kernel<WM, ST><<<grid, 64 * WM, Cfg::SMEM, s>>>(
      mm, nm, kk, g.alpha, tmA, tmB, za ? 1 : 0, zb ? 1 : 0, g.A, g.lda, g.sA, g.B, g.ldb, g.sB, g.beta, g.C,
      g.ldc, g.sC, g.dl, g.sdl, g.dr, g.sdr, g.m, g.n, thin_rows, err, gemm_inject_timeout() ? 1 : 0);
  *launched = true;
  return RCWA_OK;
}

template <int WM, int ST>
int launch_dmma(cudaStream_t s, const ZGemm& g, dim3 grid, int cm = 0, int cn = 0, bool tma = false) {
  constexpr int smem = ST * BK * (32 * WM + 2 + BN + 2) * (int)sizeof(double2);
  static bool attr[64] = {};   // per device
  int dev = 0;
  RCWA_CUDA_TRY(cudaGetDevice(&dev));
  if (smem > 48 * 1024 && (dev >= 64 || !attr[dev])) {
    RCWA_CUDA_TRY(cudaFuncSetAttribute(zgemm_dmma_kernel<0, 0, WM, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    RCWA_CUDA_TRY(cudaFuncSetAttribute(zgemm_dmma_kernel<1, 0, WM, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    RCWA_CUDA_TRY(cudaFuncSetAttribute(zgemm_dmma_kernel<0, 1, WM, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    RCWA_CUDA_TRY(cudaFuncSetAttribute(zgemm_dmma_kernel<1, 1, WM, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    if (dev < 64) attr[dev] = true;
  }
  // tiles over rows [0, m - cm) x cols [0, n - cn); the thin-strip CTAs
  // come first in the grid so that they start with the first tiles
  const int mm = g.m - cm, nm = g.n - cn;
  grid.x = cdiv_up(nm, BN);
  const int thin = (cm ? cdiv_up(g.n, 64) : 0) + (cn ? cdiv_up(mm, 64) : 0);
  const int thin_rows = cdiv_up(thin, (int)grid.x);
  grid.y = cdiv_up(mm, 32 * WM) + thin_rows;
  const int kk = g.k < 0 ? 0 : g.k;
  if constexpr (WM == RCWA_DMMA_WM) {   // the TMA feed exists for the default tile only
    if (tma && g.opA == 0 && g.opB == 0) {
      bool launched = false;
      const int rc = launch_dmma_tma<WM, RCWA_DMMA_TMA_ST>(s, g, grid, mm, nm, kk, thin_rows, &launched);
      if (rc || launched) return rc;
    }
  }
#define RCWA_DMMA_ARGS                                                                           \
  mm, nm, kk, g.alpha, g.A, g.lda, g.sA, g.B, g.ldb, g.sB, g.beta, g.C, g.ldc, g.sC, g.dl, g.sdl, \
      g.dr, g.sdr, g.m, g.n, thin_rows
  if (g.opA == 0 && g.opB == 0) zgemm_dmma_kernel<0, 0, WM, ST><<<grid, 64 * WM, smem, s>>>(RCWA_DMMA_ARGS);
  else if (g.opA == 1 && g.opB == 0) zgemm_dmma_kernel<1, 0, WM, ST><<<grid, 64 * WM, smem, s>>>(RCWA_DMMA_ARGS);
  else if (g.opA == 0 && g.opB == 1) zgemm_dmma_kernel<0, 1, WM, ST><<<grid, 64 * WM, smem, s>>>(RCWA_DMMA_ARGS);
  else zgemm_dmma_kernel<1, 1, WM, ST><<<grid, 64 * WM, smem, s>>>(RCWA_DMMA_ARGS);
#undef RCWA_DMMA_ARGS
  return RCWA_OK;
}

}  // namespace

int zgemm(cudaStream_t s, const ZGemm& g) {
  if (g.m <= 0 || g.n <= 0 || g.batch <= 0) return RCWA_OK;
  if (g.tc && !g.opA && !g.opB) {
    int* err = tc_error_flag();
    if (!err) {
      set_last_error("tensor-core GEMM: device flag unavailable");
      return RCWA_ERR_CUDA;
    }
    return g.tc == TC_INT8 ? zgemm_oz(s, g, err) : zgemm_tc(s, g, err);
  }
  // k <= 0 gives C = beta*C (the accumulators stay 0)
  dim3 grid(cdiv_up(g.n, BN), cdiv_up(g.m, BM), g.batch);
  void* tok = prof_begin(s);
  const int kk = g.k < 0 ? 0 : g.k;
  int rc = RCWA_OK;
#define RCWA_ZGEMM_ARGS                                                                          \
  g.m, g.n, kk, g.alpha, g.A, g.lda, g.sA, g.B, g.ldb, g.sB, g.beta, g.C, g.ldc, g.sC, g.dl, g.sdl, \
      g.dr, g.sdr
  const int impl = gemm_impl(g.m, g.n, kk);
  if (impl == 3) {   // 32 x 64 DMMA tiles (two warps): more CTAs for small products
    if ((rc = launch_dmma<1, RCWA_DMMA_ST>(s, g, grid, thin_cut(g.m), thin_cut(g.n)))) return rc;
  } else if (impl != 1) {
    if ((rc = launch_dmma<RCWA_DMMA_WM, RCWA_DMMA_ST>(s, g, grid, thin_cut(g.m), thin_cut(g.n), impl == 2)))
      return rc;
  } else {
    if (g.opA == 0 && g.opB == 0) zgemm_kernel<0, 0, 4><<<grid, NT, 0, s>>>(RCWA_ZGEMM_ARGS);
    else if (g.opA == 1 && g.opB == 0) zgemm_kernel<1, 0, 4><<<grid, NT, 0, s>>>(RCWA_ZGEMM_ARGS);
    else if (g.opA == 0 && g.opB == 1) zgemm_kernel<0, 1, 4><<<grid, NT, 0, s>>>(RCWA_ZGEMM_ARGS);
    else zgemm_kernel<1, 1, 4><<<grid, NT, 0, s>>>(RCWA_ZGEMM_ARGS);
  }
#undef RCWA_ZGEMM_ARGS
  // rank-k updates (k <= 64: the LU panel updates) are a family of their own
  const char* fam = kk <= 64 ? "zgemm_rank" : "zgemm";
  prof_end(s, tok, fam);
  if (tok) {
    // algorithmic flops of this launch, for the roofline (8 m n k per matrix)
    prof_add_flops(fam, 8.0 * g.m * (double)g.n * (double)kk * g.batch);
  }
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

}  // namespace rcwa

extern "C" int rcwa_set_gemm_table(const int* choice) {
  for (int i = 0; i < 25; ++i) {
    const int c = choice ? choice[i] : -1;
    if (c < -1 || c > 3) {
      rcwa::set_last_error("gemm table entries must be -1, 0, 1, 2 or 3");
      return RCWA_ERR_INVALID;
    }
  }
  for (int i = 0; i < 25; ++i) rcwa::g_gemm_table[i].store(choice ? choice[i] : -1);
  rcwa::g_gemm_table_init.store(choice != nullptr);
  return RCWA_OK;
}
