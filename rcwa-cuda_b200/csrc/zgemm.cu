// Batched complex128 GEMM on FP64 CUDA cores.
//
//   C[b] = alpha * diag(dl[b]) * A[b] * B[b] * diag(dr[b]) + beta * C[b]
//
// Column-major, arbitrary m/n/k/ld/batch strides.  This is the dense
// contraction behind every Eigen operator* of the reference's S-matrix algebra
// (rcwa.cpp:288, 326, 346-348, 602-611).  The optional diagonal scalings fold
// the reference's asDiagonal() products (rcwa.cpp:273-285, 329, 339) into the
// epilogue so no dense diagonal matrix is ever materialised.
//
// Tiling: 64x64 C tile per CTA, K step 8, 256 threads as 16x16, each thread a
// 4x4 complex micro-tile (rows tx+16i, cols ty+16j so that warp stores are
// coalesced along the column).  A and B tiles are staged into shared memory
// with cp.async (16-byte copies, zero-filled outside the matrix) and double
// buffered.
#include "common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {

constexpr int BM = 64, BN = 64, BK = 8, NT = 256;

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
template <int OPA, int OPB>
__global__ void __launch_bounds__(NT, 2)
zgemm_kernel(int m, int n, int k, double2 alpha, const double2* __restrict__ A, int lda,
             long long sA, const double2* __restrict__ B, int ldb, long long sB, double2 beta,
             double2* __restrict__ C, int ldc, long long sC, const double2* __restrict__ dl,
             long long sdl, const double2* __restrict__ dr, long long sdr) {
  __shared__ __align__(16) double2 As[2][BK][BM];
  __shared__ __align__(16) double2 Bs[2][BK][BN];

  const int b = blockIdx.z;
  A += (long long)b * sA;
  B += (long long)b * sB;
  C += (long long)b * sC;
  const int m0 = blockIdx.y * BM;
  const int n0 = blockIdx.x * BN;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;

  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = cmk(0.0, 0.0);

  auto load_tile = [&](int buf, int k0) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int e = tid + h * NT;
      // A tile: 64 rows x 8 k (consecutive threads walk the contiguous index)
      {
        const int r = OPA ? (e >> 3) : (e & 63), kk = OPA ? (e & 7) : (e >> 6);
        const int gr = m0 + r, gk = k0 + kk;
        const bool pa = (gr < m) && (gk < k);
        const double2* srcA = pa ? (OPA ? A + (long long)gr * lda + gk : A + (long long)gk * lda + gr) : A;
        cp_async16(&As[buf][kk][r], srcA, pa);
      }
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
      double2 a[4], bb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = As[buf][kk][tx + 16 * i];
        if (OPA) a[i].y = -a[i].y;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        bb[j] = Bs[buf][kk][ty + 16 * j];
        if (OPB) bb[j].y = -bb[j].y;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
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
    for (int i = 0; i < 4; ++i) {
      int row = m0 + tx + 16 * i;
      if (row >= m) continue;
      double2 v = cmul(alpha, acc[i][j]);
      if (dl) v = cmul(dl[(long long)b * sdl + row], v);
      if (dr) v = cmul(v, sr);
      double2* cp = C + (long long)col * ldc + row;
      if (use_beta) v = cadd(v, cmul(beta, *cp));
      *cp = v;
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core variant: mma.sync m8n8k4 f64 (DMMA).  Same 64x64 CTA tile,
// K step 8 and cp.async staging; 4 warps in a 2x2 grid, each computing a 32x32
// complex tile as 4x4 blocks of 8x8.  A complex 8x8x4 block product is four
// real DMMAs:  Cr += Ar Br + (-Ai) Bi,  Ci += Ar Bi + Ai Br.
// Fragment layout of m8n8k4.f64: A(row = lane/4, k = lane%4),
// B(k = lane%4, col = lane/4), C(row = lane/4, cols 2*(lane%4) + {0,1}).
// ---------------------------------------------------------------------------
constexpr int DNT = 128;

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c[0]), "+d"(c[1])
      : "d"(a), "d"(b));
}

template <int OPA, int OPB>
__global__ void __launch_bounds__(DNT, 2)
zgemm_dmma_kernel(int m, int n, int k, double2 alpha, const double2* __restrict__ A, int lda,
                  long long sA, const double2* __restrict__ B, int ldb, long long sB, double2 beta,
                  double2* __restrict__ C, int ldc, long long sC, const double2* __restrict__ dl,
                  long long sdl, const double2* __restrict__ dr, long long sdr) {
  __shared__ __align__(16) double2 As[2][BK][BM];
  __shared__ __align__(16) double2 Bs[2][BK][BN];
  const int b = blockIdx.z;
  A += (long long)b * sA;
  B += (long long)b * sB;
  C += (long long)b * sC;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int lr = lane >> 2, lk = lane & 3;

  double cr[4][4][2], ci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      cr[i][j][0] = cr[i][j][1] = 0.0;
      ci[i][j][0] = ci[i][j][1] = 0.0;
    }

  auto load_tile = [&](int buf, int k0) {
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int e = tid + h * DNT;
      {
        const int r = OPA ? (e >> 3) : (e & 63), kk = OPA ? (e & 7) : (e >> 6);
        const int gr = m0 + r, gk = k0 + kk;
        const bool pa = (gr < m) && (gk < k);
        const double2* srcA = pa ? (OPA ? A + (long long)gr * lda + gk : A + (long long)gk * lda + gr) : A;
        cp_async16(&As[buf][kk][r], srcA, pa);
      }
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
          dmma(cr[i][j], ar[i], br[j]);
          dmma(cr[i][j], nai[i], bi[j]);
          dmma(ci[i][j], ar[i], bi[j]);
          dmma(ci[i][j], ai[i], br[j]);
        }
    }
    __syncthreads();
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
        double2 v = cmul(alpha, cmk(cr[i][j][q], ci[i][j][q]));
        if (dl) v = cmul(dl[(long long)b * sdl + row], v);
        if (dr) v = cmul(v, sr);
        double2* cp = C + (long long)col * ldc + row;
        if (use_beta) v = cadd(v, cmul(beta, *cp));
        *cp = v;
      }
    }
}

// Implementation switch (read once): RCWA_ZGEMM=dmma selects the DMMA kernel,
// the default is the CUDA-core kernel (on the solve's GEMM mix it measured
// 13.8 TFLOP/s against 12.3 for the DMMA kernel on B200).
int gemm_impl() {
  static int impl = -1;
  if (impl < 0) {
    const char* e = getenv("RCWA_ZGEMM");
    impl = (e && e[0] == 'd') ? 1 : 0;
  }
  return impl;
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
    return zgemm_tc(s, g, err);
  }
  // k <= 0 gives C = beta*C (the accumulators stay 0)
  dim3 grid(cdiv_up(g.n, BN), cdiv_up(g.m, BM), g.batch);
  void* tok = prof_begin(s);
  const int kk = g.k < 0 ? 0 : g.k;
#define RCWA_ZGEMM_ARGS                                                                          \
  g.m, g.n, kk, g.alpha, g.A, g.lda, g.sA, g.B, g.ldb, g.sB, g.beta, g.C, g.ldc, g.sC, g.dl, g.sdl, \
      g.dr, g.sdr
  if (gemm_impl() == 1) {
    if (g.opA == 0 && g.opB == 0) zgemm_dmma_kernel<0, 0><<<grid, DNT, 0, s>>>(RCWA_ZGEMM_ARGS);
    else if (g.opA == 1 && g.opB == 0) zgemm_dmma_kernel<1, 0><<<grid, DNT, 0, s>>>(RCWA_ZGEMM_ARGS);
    else if (g.opA == 0 && g.opB == 1) zgemm_dmma_kernel<0, 1><<<grid, DNT, 0, s>>>(RCWA_ZGEMM_ARGS);
    else zgemm_dmma_kernel<1, 1><<<grid, DNT, 0, s>>>(RCWA_ZGEMM_ARGS);
  } else {
    if (g.opA == 0 && g.opB == 0) zgemm_kernel<0, 0><<<grid, NT, 0, s>>>(RCWA_ZGEMM_ARGS);
    else if (g.opA == 1 && g.opB == 0) zgemm_kernel<1, 0><<<grid, NT, 0, s>>>(RCWA_ZGEMM_ARGS);
    else if (g.opA == 0 && g.opB == 1) zgemm_kernel<0, 1><<<grid, NT, 0, s>>>(RCWA_ZGEMM_ARGS);
    else zgemm_kernel<1, 1><<<grid, NT, 0, s>>>(RCWA_ZGEMM_ARGS);
  }
#undef RCWA_ZGEMM_ARGS
  prof_end(s, tok, "zgemm");
  if (tok) {
    // algorithmic flops of this launch, for the roofline (8 m n k per matrix)
    prof_add_flops("zgemm", 8.0 * g.m * (double)g.n * (double)(g.k < 0 ? 0 : g.k) * g.batch);
  }
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

}  // namespace rcwa
