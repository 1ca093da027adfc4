// Complex Schur form T = Z^H H Z of batched upper Hessenberg matrices, with
// the Schur vectors accumulated into Z (on entry Z holds the Hessenberg Q).
// One CTA per matrix.  This is step 3 of the eigensolver that replaces
// Eigen::ComplexEigenSolver (rcwa.cpp:298-306).
//
// Iteration (Golub & Van Loan 7.5; LAPACK zlahqr / zlaqr5 rules):
//  * deflation: the largest k in (l, i] whose subdiagonal passes the
//    Ahues-Tisseur test is zeroed; an eigenvalue converges when l == i;
//  * active blocks of MS_MIN rows or more get multishift sweeps: NS shifts
//    (eigenvalues of the trailing NS x NS block, from a small QR run by one
//    warp; zlaqr0's exceptional shifts every sixth sweep without deflation)
//    are chased as NS single-shift bulges two positions apart.  Reflectors of
//    different bulges in one chase step act on disjoint index pairs, so they
//    commute: their parameters are computed in parallel (one lane per bulge),
//    then all left applications run (disjoint rows), then all right
//    applications (disjoint columns).  This is exactly NS consecutive
//    single-shift sweeps, with NS times fewer serial steps;
//  * smaller active blocks get single-shift sweeps (Wilkinson shift,
//    exceptional shifts every 10th/20th iteration).
// Both sweeps are processed window by window: one warp chases inside a
// diagonal window held in shared memory and logs the reflectors; then the
// CTA applies the logged reflectors to the rows right of the window, the
// columns above it and to Z, each thread streaming one row or column through
// registers (register indices are compile-time, the loops are unrolled).
#include "common.cuh"
#include "eig_common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {
using namespace eig;

constexpr int NT = 128;                      // 2 CTAs/SM at <= 255 registers, no spills
constexpr int SW = 16;                      // single-shift reflectors per chunk
constexpr int SWIN = SW + 3;
constexpr int NS = 8;                        // bulges per multishift sweep
constexpr int MW = 8;                        // chase steps per chunk
constexpr int NR = MW + 2 * (NS - 1) + 1;    // rows/cols a chunk's reflectors touch
constexpr int MWIN = NR + 3;
constexpr int MS_MIN = 3 * NS;
constexpr int WINMAX = MWIN > SWIN ? MWIN : SWIN;
static_assert(WINMAX <= 32, "one lane per window column");

struct Smem {
  double2 Hw[WINMAX][WINMAX + 1];  // window, Hw[col][row]
  double2 rtau[MW][NS];
  double2 rv[MW][NS];
  double rbeta[MW][NS];
  int ract[MW][NS];
  double2 stau[SW];
  double2 sv[SW];
  double2 Hs[NS][NS + 1];          // trailing block for the shifts, Hs[col][row]
  double2 shifts[NS];
  int red[NT / 32];
  int l;
  int flag;
  double2 shift;
};

// Shared-memory loads the compiler may not hoist out of the per-row loops of
// the deferred updates (hoisting all logged reflectors would spill registers).
__device__ __forceinline__ double2 lds2(const double2* p) {
  double2 v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ int lds1(const int* p) {
  int v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}

// Eigenvalues of the m x m upper Hessenberg Hs by single-shift QR (one warp,
// eigenvalues only).  Writes sm.shifts[0..m); false if the cap is reached.
__device__ bool small_eig(Smem& sm, int m, int lane) {
  const double ulp = DBL_EPSILON;
  int ii = m - 1, its = 0, total = 0;
  while (ii > 0) {
    bool neg = false;
    if (lane >= 1 && lane <= ii) {
      const double ah = cabs1(sm.Hs[lane - 1][lane]);
      neg = ah <= ulp * (cabs1(sm.Hs[lane - 1][lane - 1]) + cabs1(sm.Hs[lane][lane])) || ah < DBL_MIN;
    }
    const unsigned msk = __ballot_sync(0xffffffffu, neg);
    const int ll = msk ? 31 - __clz(msk) : 0;
    if (ll == ii) {
      if (lane == 0) sm.shifts[ii] = sm.Hs[ii][ii];
      __syncwarp();
      --ii;
      its = 0;
      continue;
    }
    if (++total > 40 * NS * NS) return false;
    ++its;
    double2 mu;
    if (its % 10 == 0)
      mu = cadd(sm.Hs[ii][ii], cmk(0.75 * fabs(sm.Hs[ii - 1][ii].x), 0.0));
    else
      mu = wilkinson_shift(sm.Hs[ii - 1][ii - 1], sm.Hs[ii][ii - 1], sm.Hs[ii - 1][ii], sm.Hs[ii][ii]);
    if (!cfinite(mu)) return false;
    for (int k = ll; k < ii; ++k) {
      double2 alpha, x;
      if (k == ll) {
        alpha = csub(sm.Hs[k][k], mu);
        x = sm.Hs[k][k + 1];
      } else {
        alpha = sm.Hs[k - 1][k];
        x = sm.Hs[k - 1][k + 1];
      }
      double beta;
      double2 tau, v2;
      larfg2(alpha, x, beta, tau, v2);
      __syncwarp();
      if (k > ll && lane == 0) {
        sm.Hs[k - 1][k] = cmk(beta, 0.0);
        sm.Hs[k - 1][k + 1] = cmk(0.0, 0.0);
      }
      if (lane >= k && lane <= ii) refl_left(sm.Hs[lane][k], sm.Hs[lane][k + 1], tau, v2);
      __syncwarp();
      if (lane >= ll && lane <= min(k + 2, ii)) refl_right(sm.Hs[k][lane], sm.Hs[k + 1][lane], tau, v2);
      __syncwarp();
    }
  }
  if (lane == 0) sm.shifts[0] = sm.Hs[0][0];
  __syncwarp();
  return true;
}

// ---- window load / store ----------------------------------------------------
__device__ __forceinline__ void load_window(Smem& sm, const double2* H, int ld, int j0, int nw) {
  for (int e = threadIdx.x; e < nw * nw; e += NT) {
    const int r = e % nw, c = e / nw;
    sm.Hw[c][r] = H[(long long)(j0 + c) * ld + j0 + r];
  }
}
__device__ __forceinline__ void store_window(const Smem& sm, double2* H, int ld, int j0, int nw) {
  for (int e = threadIdx.x; e < nw * nw; e += NT) {
    const int r = e % nw, c = e / nw;
    H[(long long)(j0 + c) * ld + j0 + r] = sm.Hw[c][r];
  }
}

// ---- single-shift sweep over [l, i] ------------------------------------------
__device__ void single_sweep(Smem& sm, double2* H, double2* Z, int ld, int n, int l, int i,
                             double2 shift) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int k0 = l; k0 < i; k0 += SW) {
    const int k1 = min(k0 + SW, i);
    const int nrot = k1 - k0;
    const int j0 = max(l, k0 - 1), j1 = min(i, k1 + 1);
    const int nw = j1 - j0 + 1;
    load_window(sm, H, ld, j0, nw);
    __syncthreads();
    if (wid == 0) {
      for (int k = k0; k < k1; ++k) {
        const int kk = k - j0;
        double2 alpha, x;
        if (k == l) {
          alpha = csub(sm.Hw[kk][kk], shift);
          x = sm.Hw[kk][kk + 1];
        } else {
          alpha = sm.Hw[kk - 1][kk];
          x = sm.Hw[kk - 1][kk + 1];
        }
        double beta;
        double2 tau, v2;
        larfg2(alpha, x, beta, tau, v2);
        __syncwarp();
        if (k > l && lane == 0) {
          sm.Hw[kk - 1][kk] = cmk(beta, 0.0);
          sm.Hw[kk - 1][kk + 1] = cmk(0.0, 0.0);
        }
        if (lane >= kk && lane < nw) refl_left(sm.Hw[lane][kk], sm.Hw[lane][kk + 1], tau, v2);
        __syncwarp();
        if (lane <= min(k + 2, i) - j0) refl_right(sm.Hw[kk][lane], sm.Hw[kk + 1][lane], tau, v2);
        __syncwarp();
        if (lane == 0) {
          sm.stau[k - k0] = tau;
          sm.sv[k - k0] = v2;
        }
      }
    }
    __syncthreads();
    store_window(sm, H, ld, j0, nw);
    const int nA = n - 1 - j1, nB = j0, nC = n;
    for (int it = tid; it < nA + nB + nC; it += NT) {
      double2 x[SW + 1];
      if (it < nA) {
        double2* col = H + (long long)(j1 + 1 + it) * ld + k0;
#pragma unroll
        for (int r = 0; r <= SW; ++r)
          if (r <= nrot) x[r] = col[r];
#pragma unroll
        for (int r = 0; r < SW; ++r)
          if (r < nrot) refl_left(x[r], x[r + 1], lds2(&sm.stau[r]), lds2(&sm.sv[r]));
#pragma unroll
        for (int r = 0; r <= SW; ++r)
          if (r <= nrot) col[r] = x[r];
      } else {
        double2* p = (it < nA + nB) ? H + (long long)k0 * ld + (it - nA)
                                    : Z + (long long)k0 * ld + (it - nA - nB);
#pragma unroll
        for (int r = 0; r <= SW; ++r)
          if (r <= nrot) x[r] = p[(long long)r * ld];
#pragma unroll
        for (int r = 0; r < SW; ++r)
          if (r < nrot) refl_right(x[r], x[r + 1], lds2(&sm.stau[r]), lds2(&sm.sv[r]));
#pragma unroll
        for (int r = 0; r <= SW; ++r)
          if (r <= nrot) p[(long long)r * ld] = x[r];
      }
    }
    __syncthreads();
  }
}

// ---- multishift sweep over [l, i] with NS bulges (shifts in sm.shifts) --------
// Bulge b enters at step 2b; at step t it sits at k = l + t - 2b.
__device__ void multi_sweep(Smem& sm, double2* H, double2* Z, int ld, int n, int l, int i) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int T = (i - l) + 2 * (NS - 1);
  for (int t0 = 0; t0 < T; t0 += MW) {
    const int kbase = l + t0 - 2 * (NS - 1);   // register row 0 of this chunk
    const int j0 = max(l, kbase - 1), j1 = min(i, kbase + NR + 1);
    const int nw = j1 - j0 + 1;
    load_window(sm, H, ld, j0, nw);
    __syncthreads();
    if (wid == 0) {
      for (int s = 0; s < MW; ++s) {
        const int t = t0 + s;
        if (lane < NS) {
          const int b = lane, k = l + t - 2 * b;
          const bool act = (t < T) && k >= l && k <= i - 1;
          double beta = 0.0;
          double2 tau = cmk(0.0, 0.0), v2 = cmk(0.0, 0.0);
          if (act) {
            const int kk = k - j0;
            double2 alpha, x;
            if (k == l) {
              alpha = csub(sm.Hw[kk][kk], sm.shifts[b]);
              x = sm.Hw[kk][kk + 1];
            } else {
              alpha = sm.Hw[kk - 1][kk];
              x = sm.Hw[kk - 1][kk + 1];
            }
            larfg2(alpha, x, beta, tau, v2);
          }
          sm.rtau[s][b] = tau;
          sm.rv[s][b] = v2;
          sm.rbeta[s][b] = beta;
          sm.ract[s][b] = act ? 1 : 0;
        }
        __syncwarp();
        // all left applications (rows of distinct bulges are disjoint)
        for (int it = lane; it < NS * nw; it += 32) {
          const int b = it / nw, c = it - b * nw;
          if (!sm.ract[s][b]) continue;
          const int k = l + t - 2 * b, kk = k - j0;
          if (c >= kk) {
            refl_left(sm.Hw[c][kk], sm.Hw[c][kk + 1], sm.rtau[s][b], sm.rv[s][b]);
          } else if (c == kk - 1 && k > l) {
            sm.Hw[c][kk] = cmk(sm.rbeta[s][b], 0.0);
            sm.Hw[c][kk + 1] = cmk(0.0, 0.0);
          }
        }
        __syncwarp();
        // all right applications (columns of distinct bulges are disjoint)
        for (int it = lane; it < NS * nw; it += 32) {
          const int b = it / nw, r = it - b * nw;
          if (!sm.ract[s][b]) continue;
          const int k = l + t - 2 * b, kk = k - j0;
          if (r <= min(k + 2, i) - j0) refl_right(sm.Hw[kk][r], sm.Hw[kk + 1][r], sm.rtau[s][b], sm.rv[s][b]);
        }
        __syncwarp();
      }
    }
    __syncthreads();
    store_window(sm, H, ld, j0, nw);
    // deferred: rows [kbase, kbase+NR) of the columns right of the window,
    // columns [kbase, kbase+NR) of the rows above it and of Z
    const int lo = max(l, kbase), hi = min(i, kbase + NR - 1);
    const int nA = n - 1 - j1, nB = j0, nC = n;
    for (int it = tid; it < nA + nB + nC; it += NT) {
      double2 x[NR];
      if (it < nA) {
        double2* col = H + (long long)(j1 + 1 + it) * ld;
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const int row = kbase + r;
          x[r] = (row >= lo && row <= hi) ? col[row] : cmk(0.0, 0.0);
        }
#pragma unroll
        for (int s = 0; s < MW; ++s)
#pragma unroll
          for (int b = 0; b < NS; ++b)
            if (lds1(&sm.ract[s][b]))
              refl_left(x[s + 2 * (NS - 1 - b)], x[s + 2 * (NS - 1 - b) + 1], lds2(&sm.rtau[s][b]),
                        lds2(&sm.rv[s][b]));
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const int row = kbase + r;
          if (row >= lo && row <= hi) col[row] = x[r];
        }
      } else {
        double2* p = (it < nA + nB) ? H + (it - nA) : Z + (it - nA - nB);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const int c = kbase + r;
          x[r] = (c >= lo && c <= hi) ? p[(long long)c * ld] : cmk(0.0, 0.0);
        }
#pragma unroll
        for (int s = 0; s < MW; ++s)
#pragma unroll
          for (int b = 0; b < NS; ++b)
            if (lds1(&sm.ract[s][b]))
              refl_right(x[s + 2 * (NS - 1 - b)], x[s + 2 * (NS - 1 - b) + 1], lds2(&sm.rtau[s][b]),
                         lds2(&sm.rv[s][b]));
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const int c = kbase + r;
          if (c >= lo && c <= hi) p[(long long)c * ld] = x[r];
        }
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(NT, 2)
schur_kernel(double2* __restrict__ Hg, int ld, long long stride, int n, double2* __restrict__ Zg,
             double2* __restrict__ lamg, long long slam, uint32_t* __restrict__ status,
             int max_sweeps_per_n) {
  __shared__ Smem sm;
  const int b = blockIdx.x;
  double2* H = Hg + (long long)b * stride;
  double2* Z = Zg + (long long)b * stride;
  double2* lam = lamg + (long long)b * slam;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const double ulp = DBL_EPSILON;
  const double smlnum = DBL_MIN * ((double)n / ulp);

  {  // non-finite input -> fail fast
    int bad = 0;
    for (long long e = tid; e < (long long)n * n; e += NT) {
      const int r = (int)(e % n), c = (int)(e / n);
      if (r <= c + 1 && !cfinite(H[(long long)c * ld + r])) bad = 1;
    }
    if (__syncthreads_or(bad)) {
      if (tid == 0) atomicOr(status + b, (unsigned)(ST_NONFINITE | ST_EIG_NOCONV));
      for (int r = tid; r < n; r += NT) lam[r] = cmk(nan(""), nan(""));
      return;
    }
  }

  const int itmax = 30 * (n > 10 ? n : 10);
  const long long sweep_cap = (long long)max_sweeps_per_n * (n > 10 ? n : 10);
  long long total = 0;
  bool failed = false;
  int i = n - 1;
  while (i >= 0) {
    int l = 0, kdefl = 0;
    bool conv = false;
    for (int its = 0; its <= itmax; ++its) {
      // deflation: largest k in (l, i] with a negligible H[k, k-1]
      int cand = l;
      for (int k = l + 1 + tid; k <= i; k += NT)
        if (k > cand && negligible(H, ld, n, k, ulp, smlnum)) cand = k;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) cand = max(cand, __shfl_xor_sync(0xffffffffu, cand, off));
      if (lane == 0) sm.red[wid] = cand;
      __syncthreads();
      if (tid == 0) {
        int c = l;
        for (int w = 0; w < NT / 32; ++w) c = max(c, sm.red[w]);
        sm.l = c;
        if (c > 0) H[(long long)(c - 1) * ld + c] = cmk(0.0, 0.0);
      }
      __syncthreads();
      l = sm.l;
      if (l >= i) {
        conv = true;
        break;
      }
      ++kdefl;
      if (++total > sweep_cap) break;
      const int m = i - l + 1;
      if (m >= MS_MIN) {
        // NS shifts: eigenvalues of the trailing NS x NS block, or exceptional
        bool exc = (kdefl % 6 == 0);
        if (!exc) {
          const int q0 = i - NS + 1;
          for (int e = tid; e < NS * NS; e += NT) {
            const int r = e % NS, c = e / NS;
            sm.Hs[c][r] = (r <= c + 1) ? H[(long long)(q0 + c) * ld + q0 + r] : cmk(0.0, 0.0);
          }
          __syncthreads();
          if (wid == 0) {
            const bool ok = small_eig(sm, NS, lane);
            if (lane == 0) sm.flag = ok ? 0 : 1;
          }
          __syncthreads();
          exc = sm.flag != 0;
          if (!exc && tid < NS && !cfinite(sm.shifts[tid])) sm.flag = 1;
          __syncthreads();
          exc = sm.flag != 0;
        }
        if (exc) {
          if (tid < NS) {   // zlaqr0: H(k,k) + 0.75 |H(k,k-1)| down the trailing diagonal
            const int k = i - tid;
            sm.shifts[tid] = cadd(H[(long long)k * ld + k], cmk(0.75 * cabs1(H[(long long)(k - 1) * ld + k]), 0.0));
          }
          __syncthreads();
        }
        multi_sweep(sm, H, Z, ld, n, l, i);
      } else {
        if (tid == 0) {
          double2 t;
          if (kdefl % 20 == 0) {
            t = cadd(cmk(0.75 * fabs(H[(long long)(i - 1) * ld + i].x), 0.0), H[(long long)i * ld + i]);
          } else if (kdefl % 10 == 0) {
            t = cadd(cmk(0.75 * fabs(H[(long long)l * ld + l + 1].x), 0.0), H[(long long)l * ld + l]);
          } else {
            t = wilkinson_shift(H[(long long)(i - 1) * ld + i - 1], H[(long long)i * ld + i - 1],
                                H[(long long)(i - 1) * ld + i], H[(long long)i * ld + i]);
          }
          sm.shift = t;
          sm.flag = cfinite(t) ? 0 : 1;
        }
        __syncthreads();
        if (sm.flag) break;
        single_sweep(sm, H, Z, ld, n, l, i, sm.shift);
      }
    }
    if (!conv) {
      failed = true;
      break;
    }
    if (tid == 0) lam[i] = H[(long long)i * ld + i];
    i = l - 1;
  }
  __syncthreads();
  if (failed) {
    if (tid == 0) atomicOr(status + b, (unsigned)ST_EIG_NOCONV);
    for (int r = tid; r <= i; r += NT) lam[r] = cmk(nan(""), nan(""));
  }
}

}  // namespace

int schur_launch(cudaStream_t s, double2* H, int ld, long long sH, int n, double2* Z, double2* lam,
                 long long slam, uint32_t* status, int batch) {
  void* tok = prof_begin(s);
  schur_kernel<<<batch, NT, 0, s>>>(H, ld, sH, n, Z, lam, slam, status, 100);
  prof_end(s, tok, "schur");
  // work convention: eig with vectors = 100 n^3 real flops per complex matrix,
  // of which Hessenberg (40/3), Q (16/3), triangular vectors (4/3) and the
  // back-transform GEMM (8) are counted by their own kernels; the QR
  // iteration is charged the remaining 72 n^3.
  if (tok) prof_add_flops("schur", 72.0 * n * (double)n * n * batch);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

}  // namespace rcwa
