// Batched complex128 nonsymmetric eigensolver with eigenvectors.
//
// Replaces Eigen::ComplexEigenSolver (rcwa.cpp:298-306) for the per-layer
// Omega^2 = P Q problem.  The algorithm is the textbook one (Golub & Van Loan
// ch. 7; LAPACK zgehrd/zunghr/zlahqr/ztrevc), written for one CTA per matrix
// so a batch of wavelengths / layers / requests runs concurrently:
//
//  1. hess_kernel   Householder reduction A = Q H Q^H (reflectors kept below
//                   the subdiagonal, tau in a side array).
//  2. formq_kernel  Q accumulated backwards (cheapest order) into Z.
//  3. schur_kernel  single-shift complex QR with deflation by the
//                   Ahues-Tisseur criterion, Wilkinson shifts and the
//                   exceptional shifts of zlahqr, until H = T is upper
//                   triangular; Z <- Z * (all rotations) = Schur vectors.
//                   The bulge is chased window by window: one warp applies a
//                   chunk of W 2x2 reflectors to a (W+3)^2 diagonal window held
//                   in shared memory, then the whole CTA applies the chunk to
//                   the rows right of the window, the columns above it and to
//                   Z, each thread streaming one row/column through registers.
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

constexpr int HESS_NT = 512;
constexpr int SCHUR_NT = 256;
constexpr int SCHUR_W = 16;           // reflectors per window chunk
constexpr int WIN = SCHUR_W + 3;      // window side
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
// 1. Householder reduction to upper Hessenberg form.
//    For k = 0..n-3: reflector G_k = I - tau v v^H with v = [1, v2..] acting on
//    rows/cols k+1..n-1 such that G_k^H x = beta e1 (x = A[k+1:, k]); then
//    A <- G_k^H A G_k.  v (without the leading 1) overwrites A[k+2:, k].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(HESS_NT)
hess_kernel(double2* __restrict__ Ag, int ld, long long stride, int n, double2* __restrict__ taug) {
  extern __shared__ __align__(16) double2 sm[];
  double2* vs = sm;          // [n]
  double2* ws = sm + n;      // [n]
  __shared__ double red[HESS_NT / 32];
  __shared__ double2 s_tau;
  const int b = blockIdx.x;
  double2* A = Ag + (long long)b * stride;
  double2* tau = taug + (long long)b * n;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int NW = HESS_NT / 32;

  for (int k = 0; k + 2 < n; ++k) {
    double2* ak = A + (long long)k * ld;
    const int m = n - k - 1;  // length of x
    // ||x[1:]||^2
    double part = 0.0;
    for (int i = k + 2 + tid; i < n; i += HESS_NT) part += cabs2(ak[i]);
    double xn2 = block_sum<HESS_NT>(part, red);
    if (tid == 0) {
      double2 alpha = ak[k + 1];
      double2 t = cmk(0.0, 0.0);
      double2 scale = cmk(0.0, 0.0);
      double beta = alpha.x;
      if (!(xn2 == 0.0 && alpha.y == 0.0)) {
        double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
        beta = -copysign(nrm, alpha.x);
        t = cmk((beta - alpha.x) / beta, -alpha.y / beta);
        scale = crcp(cmk(alpha.x - beta, alpha.y));
      }
      s_tau = t;
      tau[k] = t;
      ws[0] = scale;  // temporary broadcast
      ak[k + 1] = cmk(beta, 0.0);
    }
    __syncthreads();
    const double2 t = s_tau;
    const double2 scale = ws[0];
    __syncthreads();
    // v (index 0 <-> row k+1)
    for (int i = tid; i < m; i += HESS_NT) {
      double2 v;
      if (i == 0) {
        v = cmk(1.0, 0.0);
      } else {
        v = cmul(ak[k + 1 + i], scale);
        ak[k + 1 + i] = v;
      }
      vs[i] = v;
    }
    __syncthreads();
    if (t.x == 0.0 && t.y == 0.0) continue;
    // left: w_j = sum_i conj(v_i) A[k+1+i, j], j = k+1..n-1  (warp per column)
    for (int jj = wid; jj < m; jj += NW) {
      const double2* col = A + (long long)(k + 1 + jj) * ld + k + 1;
      double sr = 0.0, si = 0.0;
      for (int i = lane; i < m; i += 32) {
        double2 v = vs[i], a = col[i];
        sr += v.x * a.x + v.y * a.y;
        si += v.x * a.y - v.y * a.x;
      }
      sr = warp_sum(sr);
      si = warp_sum(si);
      if (lane == 0) ws[jj] = cmk(sr, si);
    }
    __syncthreads();
    // A[k+1+i, k+1+jj] -= conj(t) v_i w_jj
    {
      const double2 tc = cconj(t);
      for (int jj = wid; jj < m; jj += NW) {
        double2* col = A + (long long)(k + 1 + jj) * ld + k + 1;
        const double2 tw = cmul(tc, ws[jj]);
        for (int i = lane; i < m; i += 32) {
          double2 v = vs[i];
          double2 a = col[i];
          a.x -= v.x * tw.x - v.y * tw.y;
          a.y -= v.x * tw.y + v.y * tw.x;
          col[i] = a;
        }
      }
    }
    __syncthreads();
    // right: y_i = sum_j A[i, k+1+j] v_j, i = 0..n-1 (thread per row)
    for (int i = tid; i < n; i += HESS_NT) {
      double2 y = cmk(0.0, 0.0);
      for (int jj = 0; jj < m; ++jj) cfma(y, A[(long long)(k + 1 + jj) * ld + i], vs[jj]);
      ws[i] = cmul(t, y);  // tau * y
    }
    __syncthreads();
    // A[i, k+1+jj] -= (tau y_i) conj(v_jj)
    for (int jj = wid; jj < m; jj += NW) {
      double2* col = A + (long long)(k + 1 + jj) * ld;
      const double2 vc = cconj(vs[jj]);
      for (int i = lane; i < n; i += 32) {
        double2 ty = ws[i];
        double2 a = col[i];
        a.x -= ty.x * vc.x - ty.y * vc.y;
        a.y -= ty.x * vc.y + ty.y * vc.x;
        col[i] = a;
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    for (int k = (n >= 2 ? n - 2 : 0); k < n; ++k) tau[k] = cmk(0.0, 0.0);
  }
}

// ---------------------------------------------------------------------------
// 2. Z = Q = G_0 G_1 ... G_{n-3}, accumulated backwards; clears the
//    reflector storage below the subdiagonal of A (leaving H).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(HESS_NT)
formq_kernel(double2* __restrict__ Ag, int ld, long long stride, int n,
             const double2* __restrict__ taug, double2* __restrict__ Zg) {
  extern __shared__ __align__(16) double2 sm[];
  double2* vs = sm;
  double2* ws = sm + n;
  const int b = blockIdx.x;
  double2* A = Ag + (long long)b * stride;
  double2* Z = Zg + (long long)b * stride;
  const double2* tau = taug + (long long)b * n;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int NW = HESS_NT / 32;
  for (long long e = tid; e < (long long)n * n; e += HESS_NT) {
    int i = (int)(e % n), j = (int)(e / n);
    Z[(long long)j * ld + i] = cmk(i == j ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  for (int k = n - 3; k >= 0; --k) {
    const double2 t = tau[k];
    const int m = n - k - 1;
    for (int i = tid; i < m; i += HESS_NT) vs[i] = (i == 0) ? cmk(1.0, 0.0) : A[(long long)k * ld + k + 1 + i];
    __syncthreads();
    if (!(t.x == 0.0 && t.y == 0.0)) {
      for (int jj = wid; jj < m; jj += NW) {
        const double2* col = Z + (long long)(k + 1 + jj) * ld + k + 1;
        double sr = 0.0, si = 0.0;
        for (int i = lane; i < m; i += 32) {
          double2 v = vs[i], a = col[i];
          sr += v.x * a.x + v.y * a.y;
          si += v.x * a.y - v.y * a.x;
        }
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (lane == 0) ws[jj] = cmul(t, cmk(sr, si));
      }
      __syncthreads();
      for (int jj = wid; jj < m; jj += NW) {
        double2* col = Z + (long long)(k + 1 + jj) * ld + k + 1;
        const double2 tw = ws[jj];
        for (int i = lane; i < m; i += 32) {
          double2 v = vs[i];
          double2 a = col[i];
          a.x -= v.x * tw.x - v.y * tw.y;
          a.y -= v.x * tw.y + v.y * tw.x;
          col[i] = a;
        }
      }
    }
    __syncthreads();
  }
  // clear reflectors (below the subdiagonal)
  for (long long e = tid; e < (long long)n * n; e += HESS_NT) {
    int i = (int)(e % n), j = (int)(e / n);
    if (i > j + 1) A[(long long)j * ld + i] = cmk(0.0, 0.0);
  }
}

// 2x2 Householder (zlarfg with n = 2): returns beta (real), tau, v2 with
// (I - tau [1 v2]^T [1 v2]^* )^H [alpha; x] = [beta; 0].
__device__ __forceinline__ void larfg2(double2 alpha, double2 x, double& beta, double2& tau,
                                       double2& v2) {
  double xn = hypot(x.x, x.y);
  if (xn == 0.0 && alpha.y == 0.0) {
    tau = cmk(0.0, 0.0);
    v2 = cmk(0.0, 0.0);
    beta = alpha.x;
    return;
  }
  double mx = fmax(fmax(fabs(alpha.x), fabs(alpha.y)), xn);
  double a = alpha.x / mx, c = alpha.y / mx, d = xn / mx;
  double nrm = mx * sqrt(a * a + c * c + d * d);
  beta = -copysign(nrm, alpha.x);
  tau = cmk((beta - alpha.x) / beta, -alpha.y / beta);
  v2 = cmul(x, crcp(cmk(alpha.x - beta, alpha.y)));
}

// Deflation test of zlahqr (Ahues & Tisseur) for subdiagonal entry (k, k-1).
__device__ __forceinline__ bool negligible(const double2* H, int ld, int n, int k, double ulp,
                                           double smlnum) {
  double2 h = H[(long long)(k - 1) * ld + k];
  double ah = cabs1(h);
  if (ah <= smlnum) return true;
  double2 hkk = H[(long long)k * ld + k];
  double2 hk1 = H[(long long)(k - 1) * ld + k - 1];
  double tst = cabs1(hk1) + cabs1(hkk);
  if (tst == 0.0) {
    if (k - 2 >= 0) tst += cabs1(H[(long long)(k - 2) * ld + k - 1]);
    if (k + 1 <= n - 1) tst += cabs1(H[(long long)k * ld + k + 1]);
  }
  if (ah <= ulp * tst) {
    double2 hup = H[(long long)k * ld + k - 1];
    double ab = fmax(ah, cabs1(hup)), ba = fmin(ah, cabs1(hup));
    double2 dd = csub(hk1, hkk);
    double aa = fmax(cabs1(hkk), cabs1(dd)), bb = fmin(cabs1(hkk), cabs1(dd));
    double s = aa + ab;
    if (ba * (ab / s) <= fmax(smlnum, ulp * (bb * (aa / s)))) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// 3. Complex Schur form by windowed single-shift QR.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(SCHUR_NT, 2)
schur_kernel(double2* __restrict__ Hg, int ld, long long stride, int n,
             double2* __restrict__ Zg, double2* __restrict__ lamg, long long slam,
             uint32_t* __restrict__ status, int max_sweeps_per_n) {
  __shared__ double2 Hw[WIN][WIN + 1];  // Hw[c][r]: column-major window
  __shared__ double2 rtau[SCHUR_W], rv[SCHUR_W];
  __shared__ int s_l, s_flag;
  __shared__ double2 s_shift;
  __shared__ int s_red[SCHUR_NT / 32];

  const int b = blockIdx.x;
  double2* H = Hg + (long long)b * stride;
  double2* Z = Zg + (long long)b * stride;
  double2* lam = lamg + (long long)b * slam;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const double ulp = DBL_EPSILON;
  const double safmin = DBL_MIN;
  const double smlnum = safmin * ((double)n / ulp);

  // non-finite input -> fail fast
  {
    int bad = 0;
    for (long long e = tid; e < (long long)n * n; e += SCHUR_NT) {
      int i = (int)(e % n), j = (int)(e / n);
      if (i <= j + 1 && !cfinite(H[(long long)j * ld + i])) bad = 1;
    }
    bad = __syncthreads_or(bad);
    if (bad) {
      if (tid == 0) atomicOr(status + b, (unsigned)(ST_NONFINITE | ST_EIG_NOCONV));
      for (int i = tid; i < n; i += SCHUR_NT) lam[i] = cmk(nan(""), nan(""));
      return;
    }
  }

  const int itmax = 30 * (n > 10 ? n : 10);
  const long long sweep_cap = (long long)max_sweeps_per_n * (n > 10 ? n : 10);
  long long total = 0;
  bool failed = false;
  int i = n - 1;
  while (i >= 0) {
    int l = 0;
    int kdefl = 0;
    bool conv = false;
    for (int its = 0; its <= itmax; ++its) {
      // --- deflation: largest k in (l, i] with negligible H[k, k-1]
      int cand = l;
      for (int k = l + 1 + tid; k <= i; k += SCHUR_NT)
        if (negligible(H, ld, n, k, ulp, smlnum) && k > cand) cand = k;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) cand = max(cand, __shfl_xor_sync(0xffffffffu, cand, off));
      if (lane == 0) s_red[wid] = cand;
      __syncthreads();
      if (tid == 0) {
        int c = l;
        for (int w = 0; w < SCHUR_NT / 32; ++w) c = max(c, s_red[w]);
        s_l = c;
        if (c > 0) H[(long long)(c - 1) * ld + c] = cmk(0.0, 0.0);
      }
      __syncthreads();
      l = s_l;
      if (l >= i) {
        conv = true;
        break;
      }
      ++kdefl;
      ++total;
      if (total > sweep_cap) break;
      // --- shift (zlahqr)
      if (tid == 0) {
        double2 t;
        const double dat1 = 0.75;
        if (kdefl % 20 == 0) {
          double s = dat1 * fabs(H[(long long)(i - 1) * ld + i].x);
          t = cadd(cmk(s, 0.0), H[(long long)i * ld + i]);
        } else if (kdefl % 10 == 0) {
          double s = dat1 * fabs(H[(long long)l * ld + l + 1].x);
          t = cadd(cmk(s, 0.0), H[(long long)l * ld + l]);
        } else {
          t = H[(long long)i * ld + i];
          double2 h_im1_i = H[(long long)i * ld + i - 1];
          double2 h_i_im1 = H[(long long)(i - 1) * ld + i];
          double2 u = cmul(csqrt_principal(h_im1_i), csqrt_principal(h_i_im1));
          double s = cabs1(u);
          if (s != 0.0) {
            double2 x = cscale(csub(H[(long long)(i - 1) * ld + i - 1], t), 0.5);
            double sx = cabs1(x);
            s = fmax(s, sx);
            double2 xs = cscale(x, 1.0 / s), us = cscale(u, 1.0 / s);
            double2 y = cscale(csqrt_principal(cadd(cmul(xs, xs), cmul(us, us))), s);
            if (sx > 0.0) {
              double2 xx = cscale(x, 1.0 / sx);
              if (xx.x * y.x + xx.y * y.y < 0.0) y = cneg(y);
            }
            t = csub(t, cmul(u, cdiv(u, cadd(x, y))));
          }
        }
        s_shift = t;
        s_flag = cfinite(t) ? 0 : 1;
      }
      __syncthreads();
      if (s_flag) break;
      const double2 shift = s_shift;
      // --- one implicit single-shift sweep, rotations k = l .. i-1
      for (int k0 = l; k0 < i; k0 += SCHUR_W) {
        const int k1 = min(k0 + SCHUR_W, i);          // rotations [k0, k1)
        const int nrot = k1 - k0;
        const int j0 = max(l, k0 - 1), j1 = min(i, k1 + 1);
        const int nw = j1 - j0 + 1;
        for (int e = tid; e < nw * nw; e += SCHUR_NT) {
          int r = e % nw, c = e / nw;
          Hw[c][r] = H[(long long)(j0 + c) * ld + j0 + r];
        }
        __syncthreads();
        if (wid == 0) {
          for (int k = k0; k < k1; ++k) {
            const int kk = k - j0;
            double2 alpha, x;
            if (k == l) {
              alpha = csub(Hw[kk][kk], shift);
              x = Hw[kk][kk + 1];
            } else {
              alpha = Hw[kk - 1][kk];
              x = Hw[kk - 1][kk + 1];
            }
            double beta;
            double2 tau, v2;
            larfg2(alpha, x, beta, tau, v2);
            __syncwarp();
            if (k > l && lane == 0) {
              Hw[kk - 1][kk] = cmk(beta, 0.0);
              Hw[kk - 1][kk + 1] = cmk(0.0, 0.0);
            }
            // left: rows kk, kk+1 of window columns >= kk
            if (lane >= kk && lane < nw) {
              double2 a = Hw[lane][kk], q = Hw[lane][kk + 1];
              double2 sum = cmulc(tau, cadd(a, cmulc(v2, q)));
              Hw[lane][kk] = csub(a, sum);
              Hw[lane][kk + 1] = csub(q, cmul(sum, v2));
            }
            __syncwarp();
            // right: cols kk, kk+1 of window rows <= min(k+2, i)
            const int rmax = min(k + 2, i) - j0;
            if (lane <= rmax) {
              double2 a = Hw[kk][lane], q = Hw[kk + 1][lane];
              double2 sum = cmul(tau, cadd(a, cmul(q, v2)));
              Hw[kk][lane] = csub(a, sum);
              Hw[kk + 1][lane] = csub(q, cmulc(v2, sum));
            }
            __syncwarp();
            if (lane == 0) {
              rtau[k - k0] = tau;
              rv[k - k0] = v2;
            }
          }
        }
        __syncthreads();
        for (int e = tid; e < nw * nw; e += SCHUR_NT) {
          int r = e % nw, c = e / nw;
          H[(long long)(j0 + c) * ld + j0 + r] = Hw[c][r];
        }
        // deferred updates of this chunk
        const int nA = n - 1 - j1;   // columns j1+1..n-1, rows k0..k1 (left)
        const int nB = j0;           // rows 0..j0-1, columns k0..k1 (right)
        const int nC = n;            // Z rows 0..n-1, columns k0..k1 (right)
        for (int it = tid; it < nA + nB + nC; it += SCHUR_NT) {
          double2 x[SCHUR_W + 1];
          if (it < nA) {
            double2* col = H + (long long)(j1 + 1 + it) * ld + k0;
#pragma unroll
            for (int r = 0; r <= SCHUR_W; ++r)
              if (r <= nrot) x[r] = col[r];
#pragma unroll
            for (int r = 0; r < SCHUR_W; ++r) {
              if (r < nrot) {
                double2 tau = rtau[r], v2 = rv[r];
                double2 sum = cmulc(tau, cadd(x[r], cmulc(v2, x[r + 1])));
                x[r] = csub(x[r], sum);
                x[r + 1] = csub(x[r + 1], cmul(sum, v2));
              }
            }
#pragma unroll
            for (int r = 0; r <= SCHUR_W; ++r)
              if (r <= nrot) col[r] = x[r];
          } else {
            double2* base;
            int row;
            if (it < nA + nB) {
              base = H;
              row = it - nA;
            } else {
              base = Z;
              row = it - nA - nB;
            }
            double2* p = base + (long long)k0 * ld + row;
#pragma unroll
            for (int r = 0; r <= SCHUR_W; ++r)
              if (r <= nrot) x[r] = p[(long long)r * ld];
#pragma unroll
            for (int r = 0; r < SCHUR_W; ++r) {
              if (r < nrot) {
                double2 tau = rtau[r], v2 = rv[r];
                double2 sum = cmul(tau, cadd(x[r], cmul(x[r + 1], v2)));
                x[r] = csub(x[r], sum);
                x[r + 1] = csub(x[r + 1], cmulc(v2, sum));
              }
            }
#pragma unroll
            for (int r = 0; r <= SCHUR_W; ++r)
              if (r <= nrot) p[(long long)r * ld] = x[r];
          }
        }
        __syncthreads();
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
    for (int r = tid; r <= i; r += SCHUR_NT) lam[r] = cmk(nan(""), nan(""));
  }
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
  // Z, X (n x n each) and tau (n), all per matrix
  return (size_t)batch * ((size_t)2 * n * n + n) * sizeof(double2);
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
  const size_t shm2 = (size_t)2 * n * sizeof(double2);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(hess_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(formq_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(trevc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  if (shm2 > 200 * 1024 || (size_t)TREVC_WARPS * n * sizeof(double2) > 200 * 1024) {
    set_last_error("zeig: n=%d too large", n);
    return RCWA_ERR_INVALID;
  }
  void* tok = prof_begin(s);
  hess_kernel<<<batch, HESS_NT, shm2, s>>>(A, ld, sA, n, tau);
  prof_end(s, tok, "hess");
  // Householder reduction: (40/3) n^3 real flops per complex matrix
  if (tok) prof_add_flops("hess", 40.0 / 3.0 * n * (double)n * n * batch);
  count_launch();
  RCWA_LAUNCH_CHECK();
  tok = prof_begin(s);
  formq_kernel<<<batch, HESS_NT, shm2, s>>>(A, ld, sA, n, tau, Z);
  prof_end(s, tok, "formq");
  count_launch();
  RCWA_LAUNCH_CHECK();
  tok = prof_begin(s);
  schur_kernel<<<batch, SCHUR_NT, 0, s>>>(A, ld, sA, n, Z, lam, slam, status, 100);
  prof_end(s, tok, "schur");
  count_launch();
  RCWA_LAUNCH_CHECK();
  {
    dim3 g(cdiv_up(n, TREVC_WARPS), batch);
    tok = prof_begin(s);
    trevc_kernel<<<g, TREVC_WARPS * 32, (size_t)TREVC_WARPS * n * sizeof(double2), s>>>(A, ld, sA,
                                                                                          n, X);
    prof_end(s, tok, "trevc");
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
