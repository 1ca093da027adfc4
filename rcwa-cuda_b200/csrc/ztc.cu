// Complex GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32) with
// the split-TF32 ("3xTF32") scheme, for the mixed-precision solve mode.
//
//   C = alpha * diag(dl) * A * B * diag(dr) + beta * C       (complex128 I/O)
//
// Real formulation: [Cr; Ci] = [[Ar, -Ai], [Ai, Ar]] [Br; Bi], so one
// 128 x 128 UMMA tile computes a 64 x 128 complex tile of C.  Each FP64
// operand x is split into TF32 x_hi + x_lo while it is staged into shared
// memory, and D = A_hi B_hi + A_hi B_lo + A_lo B_hi is accumulated in FP32 in
// tensor memory (error ~1e-7 relative per product).
//
// Per CTA (128 threads): TMEM holds the 128 x 128 FP32 accumulator; shared
// memory holds two stages of {A_hi, A_lo, B_hi, B_lo}, each 128 rows x 32 TF32
// in the K-major, no-swizzle canonical layout (8-row x 16-byte core matrices;
// 16-byte chunks along K are 2048 B apart, 8-row groups 128 B apart).  All
// threads convert and stage k-tile t+1 while the tensor core runs k-tile t;
// one elected thread issues the 12 MMAs of a k-tile (3 products x 4 K=8
// steps) and commits them to the stage's mbarrier.  Every mbarrier wait is
// bounded: on time-out the kernel records RCWA_STATUS_NONFINITE-free error
// flag in *err, skips the epilogue, frees its TMEM and returns.
#include <cstdint>

#include "common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {

constexpr int TNT = 128;        // threads per CTA
constexpr int TBM = 64;         // complex rows per CTA (128 real rows)
constexpr int TBN = 128;        // complex columns per CTA
constexpr int TBK = 16;         // complex k per k-tile (32 real k)
constexpr int TILE_BYTES = 128 * 32 * 4;           // one operand tile: 16 KB
constexpr int STAGE_BYTES = 4 * TILE_BYTES;        // A_hi, A_lo, B_hi, B_lo
constexpr int TC_SMEM = 2 * STAGE_BYTES + 1024;    // two stages + alignment slack
constexpr uint32_t TMEM_COLS = 128;
constexpr long long WAIT_CAP = 1LL << 26;

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// byte offset of element (row, k) in a 128 x 32 K-major canonical tile
__device__ __forceinline__ uint32_t tile_off(int row, int k) {
  return (uint32_t)((k >> 2) * 2048 + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// v = hi + lo + O(2^-22 |v|): hi = tf32(v), lo = tf32(v - hi) with the
// remainder taken from the double itself
__device__ __forceinline__ void put_split(uint8_t* hi_tile, uint8_t* lo_tile, int row, int k, double v) {
  const uint32_t h = to_tf32((float)v);
  const uint32_t l = to_tf32((float)(v - (double)__uint_as_float(h)));
  const uint32_t o = tile_off(row, k);
  *reinterpret_cast<uint32_t*>(hi_tile + o) = h;
  *reinterpret_cast<uint32_t*>(lo_tile + o) = l;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
  d |= (uint64_t)((2048u >> 4) & 0x3FFF) << 16;    // leading byte offset: next 16 B along K
  d |= (uint64_t)((128u >> 4) & 0x3FFF) << 32;     // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
  return d;                                        // base offset 0, no swizzle
}

// kind::tf32, FP32 accumulate, A and B K-major, M = 128, N = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(IDESC), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bar)));
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
  for (long long it = 0; it < WAIT_CAP; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(su32(bar)), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__global__ void __launch_bounds__(TNT, 1)
zgemm_tc_kernel(int m, int n, int k, double2 alpha, const double2* __restrict__ A, int lda,
                long long sA, const double2* __restrict__ B, int ldb, long long sB, double2 beta,
                double2* __restrict__ C, int ldc, long long sC, const double2* __restrict__ dl,
                long long sdl, const double2* __restrict__ dr, long long sdr, int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_slot;
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int bz = blockIdx.z;
  A += (long long)bz * sA;
  B += (long long)bz * sB;
  C += (long long)bz * sC;
  const int m0 = blockIdx.y * TBM, n0 = blockIdx.x * TBN;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&mbar[0]);
    mbar_init(&mbar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_slot;

  const int ktiles = (k + TBK - 1) / TBK;
  uint32_t phase[2] = {0u, 0u};
  bool ok = true;
  for (int t = 0; t < ktiles; ++t) {
    const int st = t & 1;
    uint8_t* base = smem + st * STAGE_BYTES;
    uint8_t *Ahi = base, *Alo = base + TILE_BYTES, *Bhi = base + 2 * TILE_BYTES, *Blo = base + 3 * TILE_BYTES;
    if (t >= 2) {  // the MMAs of k-tile t-2 read this stage
      if (!mbar_wait(&mbar[st], phase[st])) ok = false;
      phase[st] ^= 1u;
    }
    if (!__syncthreads_and(ok)) break;
    const int k0 = t * TBK;
    // A: 64 complex rows x 16 complex k -> real rows i (Ar | -Ai) and 64+i (Ai | Ar)
    for (int e = tid; e < TBM * TBK; e += TNT) {
      const int i = e & (TBM - 1), kk = e >> 6;
      const int gi = m0 + i, gk = k0 + kk;
      double2 a = cmk(0.0, 0.0);
      if (gi < m && gk < k) a = A[(long long)gk * lda + gi];
      put_split(Ahi, Alo, i, kk, a.x);
      put_split(Ahi, Alo, i, TBK + kk, -a.y);
      put_split(Ahi, Alo, TBM + i, kk, a.y);
      put_split(Ahi, Alo, TBM + i, TBK + kk, a.x);
    }
    // B: 16 complex k x 128 complex cols -> real (col j, k) = Br, (col j, 16+k) = Bi
    for (int e = tid; e < TBK * TBN; e += TNT) {
      const int kk = e & (TBK - 1), j = e >> 4;
      const int gk = k0 + kk, gj = n0 + j;
      double2 bv = cmk(0.0, 0.0);
      if (gk < k && gj < n) bv = B[(long long)gj * ldb + gk];
      put_split(Bhi, Blo, j, kk, bv.x);
      put_split(Bhi, Blo, j, TBK + kk, bv.y);
    }
    asm volatile("fence.proxy.async.shared::cta;");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t aH = su32(Ahi), aL = su32(Alo), bH = su32(Bhi), bL = su32(Blo);
#pragma unroll
      for (int q = 0; q < 4; ++q) {   // K = 8 per MMA: chunks 2q, 2q+1
        const uint32_t off = (uint32_t)(2 * q) * 2048u;
        mma_tf32(tmem, smem_desc(aH + off), smem_desc(bH + off), (t > 0 || q > 0) ? 1u : 0u);
        mma_tf32(tmem, smem_desc(aH + off), smem_desc(bL + off), 1u);
        mma_tf32(tmem, smem_desc(aL + off), smem_desc(bH + off), 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          su32(&mbar[st])));
    }
  }
  // the last commit tracks every MMA issued before it
  if (ok && ktiles > 0) {
    const int st = (ktiles - 1) & 1;
    if (!mbar_wait(&mbar[st], phase[st])) ok = false;
  }
  ok = __syncthreads_and(ok);
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (ok) {
    // TMEM -> shared (fp32 128 x 128, row-major) -> complex epilogue
    float* stage = reinterpret_cast<float*>(smem);
    for (int c0 = 0; c0 < 128; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
          "%12, %13, %14, %15}, [%16];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
            "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;");
      const int row = warp * 32 + lane;
#pragma unroll
      for (int q = 0; q < 16; ++q) stage[row * 129 + c0 + q] = __uint_as_float(r[q]);
    }
    __syncthreads();
    const bool use_beta = (beta.x != 0.0 || beta.y != 0.0);
    for (int e = tid; e < TBM * TBN; e += TNT) {
      const int i = e & (TBM - 1), j = e >> 6;
      const int gi = m0 + i, gj = n0 + j;
      if (gi >= m || gj >= n) continue;
      double2 v = cmul(alpha, cmk((double)stage[i * 129 + j], (double)stage[(TBM + i) * 129 + j]));
      if (dl) v = cmul(dl[(long long)bz * sdl + gi], v);
      if (dr) v = cmul(v, dr[(long long)bz * sdr + gj]);
      double2* cp = C + (long long)gj * ldc + gi;
      if (use_beta) v = cadd(v, cmul(beta, *cp));
      *cp = v;
    }
  } else if (tid == 0) {
    atomicOr(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

__device__ int g_tc_err;   // time-out flag of the bounded mbarrier waits

}  // namespace

int* tc_error_flag() {
  static int* ptr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tc_err) != cudaSuccess) return nullptr;
    ptr[dev] = (int*)p;
  }
  return ptr[dev];
}

int zgemm_tc(cudaStream_t s, const ZGemm& g, int* err) {
  if (g.m <= 0 || g.n <= 0 || g.batch <= 0) return RCWA_OK;
  if (g.opA || g.opB) {
    set_last_error("zgemm_tc: transposed operands are not supported");
    return RCWA_ERR_INVALID;
  }
  static bool attr[64] = {};   // the attribute is per device
  int dev = 0;
  RCWA_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 64 || !attr[dev]) {
    RCWA_CUDA_TRY(cudaFuncSetAttribute(zgemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    if (dev < 64) attr[dev] = true;
  }
  dim3 grid(cdiv_up(g.n, TBN), cdiv_up(g.m, TBM), g.batch);
  void* tok = prof_begin(s);
  zgemm_tc_kernel<<<grid, TNT, TC_SMEM, s>>>(g.m, g.n, g.k < 0 ? 0 : g.k, g.alpha, g.A, g.lda, g.sA, g.B,
                                             g.ldb, g.sB, g.beta, g.C, g.ldc, g.sC, g.dl, g.sdl, g.dr,
                                             g.sdr, err);
  prof_end(s, tok, "zgemm_tc");
  if (tok) prof_add_flops("zgemm_tc", 8.0 * g.m * (double)g.n * (double)(g.k < 0 ? 0 : g.k) * g.batch);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

}  // namespace rcwa
