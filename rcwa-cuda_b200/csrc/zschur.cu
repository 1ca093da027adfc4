// Complex Schur form T = Z^H H Z of batched upper Hessenberg matrices, with
// the Schur vectors accumulated into Z (on entry Z holds the Hessenberg Q).
// One CTA per matrix.  This is step 3 of the eigensolver that replaces
// Eigen::ComplexEigenSolver (rcwa.cpp:298-306).
//
// Iteration (Golub & Van Loan 7.5; LAPACK zlahqr / zlaqr5 rules):
//  * deflation: the largest k in (l, i] whose subdiagonal passes the
//    Ahues-Tisseur test is zeroed; an eigenvalue converges when l == i;
//  * active blocks of AED_MIN rows or more first get aggressive early
//    deflation (zlaqr3): the trailing NWIN x NWIN window is brought to Schur
//    form, eigenvalues with a negligible spike entry deflate, the rest of the
//    window is returned to Hessenberg form and its eigenvalues become shifts;
//  * active blocks of MS_MIN rows or more get multishift sweeps: NS shifts
//    (from the early deflation, else the eigenvalues of the trailing NS x NS
//    block from a small QR run by one warp; zlaqr0's exceptional shifts every
//    sixth sweep without deflation) are chased as NS single-shift bulges two
//    positions apart.  Reflectors of
//    different bulges in one chase step act on disjoint index pairs, so they
//    commute: their parameters are computed in parallel (one lane per bulge),
//    then all left applications run (disjoint rows), then all right
//    applications (disjoint columns).  This is exactly NS consecutive
//    single-shift sweeps, with NS times fewer serial steps;
//  * smaller active blocks get single-shift sweeps (Wilkinson shift,
//    exceptional shifts every 10th/20th iteration).
// Both sweeps are processed window by window: one warp chases inside a
// diagonal window held in shared memory and logs the reflectors; the other
// warps apply the logged reflectors to the columns right of the window, the
// rows above it and to Z, each thread streaming one row or column through
// registers.
#include <atomic>

#include <cooperative_groups.h>

#include "common.cuh"
#include "eig_common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {
using namespace eig;

constexpr int NT = 256;                      // 8 warps: the chase warp + 7 update warps, 1 CTA/SM
constexpr int SW = 16;                      // single-shift reflectors per chunk
constexpr int SWIN = SW + 3;
constexpr int NS = 8;                        // bulges per multishift sweep
constexpr int MW = 8;                        // chase steps per chunk
constexpr int NR = MW + 2 * (NS - 1) + 1;    // rows/cols a chunk's reflectors touch
constexpr int MWIN = NR + 3;
static_assert(MWIN <= 32, "the chase warp moves a window row per lane");
constexpr int MS_MIN = 3 * NS;
constexpr int WINMAX = MWIN > SWIN ? MWIN : SWIN;
static_assert(WINMAX <= 32, "one lane per window column");

// Optional per-launch counters of matrix 0 (compile with -DRCWA_SCHUR_STATS):
// [0] multishift sweeps [1] single sweeps [2] cycles in multishift sweeps
// [3] cycles in single sweeps [4] cycles computing shifts [5] exceptional
// shifts [6] total cycles [7] deflation scans
#ifdef RCWA_SCHUR_STATS
__device__ unsigned long long g_schur_stats[16];
#define SCHUR_STAT(i, v) \
  do { if (blockIdx.x == 0 && threadIdx.x == 0) g_schur_stats[i] += (unsigned long long)(v); } while (0)
#define SCHUR_STAT_T(t, i, v) \
  do { if (blockIdx.x == 0 && threadIdx.x == (t)) g_schur_stats[i] += (unsigned long long)(v); } while (0)
#else
#define SCHUR_STAT(i, v) do { } while (0)
#define SCHUR_STAT_T(t, i, v) do { } while (0)
#endif

struct Smem {
  double2 Hw[WINMAX][WINMAX + 1];  // window, Hw[col][row]
  // multishift reflector log of a chunk, double buffered (chase of chunk c+1
  // runs while chunk c is applied): tau, v2 (inactive reflectors logged as
  // zeros, the identity)
  double2 rtau[2][MW][NS];
  double2 rv[2][MW][NS];
  double2 stau[SW];
  double2 sv[SW];
  double2 Hs[NS][NS + 1];          // trailing block for the shifts, Hs[col][row]
  double2 shifts[NS];
  int red[NT / 32];
  int l;
  int flag;
  double2 shift;
  // cluster mode: the command the leader CTA posts to its helpers before a
  // barrier (1 = multishift sweep over [cmd_l, cmd_i], 0 = done)
  int cmd, cmd_l, cmd_i;
};

// Barrier of the CTAs that share one matrix.  One CTA: __syncthreads.  A
// cluster of CL CTAs: a cluster barrier, with device-scope fences on both
// sides so that the global-memory updates of H and Z made by one CTA are
// seen by the others after it.
template <int CL>
__device__ __forceinline__ void mat_sync() {
  if constexpr (CL > 1) {
    __threadfence();
    cooperative_groups::this_cluster().sync();
    __threadfence();
  } else {
    __syncthreads();
  }
}
// Update warps of a matrix: the leader's 7 (its warp 0 chases) plus 8 per
// helper CTA.
template <int CL>
constexpr int update_warps() { return NT / 32 - 1 + (NT / 32) * (CL - 1); }

// Shared-memory loads the compiler may not hoist out of the per-row loops of
// the deferred updates (hoisting all logged reflectors would spill registers).
__device__ __forceinline__ double2 lds2(const double2* p) {
  double2 v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
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
// Bulge b enters at step 2b; at step t it sits at k = l + t - 2b.  Chunk c
// covers steps [c*MW, c*MW + MW); its reflectors touch rows/columns
// [kbase, kbase + NR) with kbase = l + c*MW - 2(NS-1).

// Chase of one chunk by one warp inside the shared window; logs to buffer buf.
// At step t bulge b acts on window rows/columns (kk_b, kk_b + 1) with
// kk_b = base + 2 (NS - 1 - b): the NS pairs tile [base, base + 2 NS).  The
// left applications run with one lane per window column, the right ones with
// one lane per window row; each lane holds its 2 NS entries in registers and
// applies all bulges branch-free (a reflector that does not reach the lane's
// column or row, or belongs to an inactive bulge, gets tau = 0: the identity).
__device__ void ms_chase(Smem& sm, int buf, int l, int i, int T, int t0, int j0, int nw, int lane) {
#pragma unroll 1
  for (int s = 0; s < MW; ++s) {
    const int t = t0 + s;
    // lane b < NS computes bulge b's reflector and logs it for the far
    // updates; the window updates below take it from lane b by shuffles
    // (register broadcasts, all independent: no shared-memory round trip
    // per reflector on this serial path)
    double beta = 0.0;
    double2 tau = cmk(0.0, 0.0), v2 = cmk(0.0, 0.0);
    bool act = false;
    if (lane < NS) {
      const int b = lane, k = l + t - 2 * b;
      act = (t < T) && k >= l && k <= i - 1;
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
      sm.rtau[buf][s][b] = tau;
      sm.rv[buf][s][b] = v2;
    }
    const unsigned amask = __ballot_sync(0xffffffffu, act);
    __syncwarp();
    const int base = l + t - j0 - 2 * (NS - 1);
    double2 tb[NS], vb[NS];
#pragma unroll
    for (int b = 0; b < NS; ++b) {
      tb[b] = cmk(__shfl_sync(0xffffffffu, tau.x, b), __shfl_sync(0xffffffffu, tau.y, b));
      vb[b] = cmk(__shfl_sync(0xffffffffu, v2.x, b), __shfl_sync(0xffffffffu, v2.y, b));
    }
    double2 x[2 * NS];
    {  // left: lane = window column c
      const int c = lane;
#pragma unroll
      for (int r = 0; r < 2 * NS; ++r) {
        const int row = base + r;
        x[r] = (c < nw && row >= 0 && row < nw) ? sm.Hw[c][row] : cmk(0.0, 0.0);
      }
#pragma unroll
      for (int b = 0; b < NS; ++b) {
        const int p = 2 * (NS - 1 - b), kk = base + p;
        const bool actb = (amask >> b) & 1u;
        const double bt = __shfl_sync(0xffffffffu, beta, b);
        refl_left(x[p], x[p + 1], (actb && c >= kk) ? tb[b] : cmk(0.0, 0.0), vb[b]);
        if (actb && c == kk - 1 && kk + j0 > l) {
          x[p] = cmk(bt, 0.0);
          x[p + 1] = cmk(0.0, 0.0);
        }
      }
#pragma unroll
      for (int r = 0; r < 2 * NS; ++r) {
        const int row = base + r;
        if (c < nw && row >= 0 && row < nw) sm.Hw[c][row] = x[r];
      }
    }
    __syncwarp();
    {  // right: lane = window row r
      const int r = lane;
#pragma unroll
      for (int q = 0; q < 2 * NS; ++q) {
        const int col = base + q;
        x[q] = (r < nw && col >= 0 && col < nw) ? sm.Hw[col][r] : cmk(0.0, 0.0);
      }
#pragma unroll
      for (int b = 0; b < NS; ++b) {
        const int p = 2 * (NS - 1 - b), kk = base + p;
        const bool actb = (amask >> b) & 1u;
        refl_right(x[p], x[p + 1], (actb && r <= min(kk + j0 + 2, i) - j0) ? tb[b] : cmk(0.0, 0.0), vb[b]);
      }
#pragma unroll
      for (int q = 0; q < 2 * NS; ++q) {
        const int col = base + q;
        if (r < nw && col >= 0 && col < nw) sm.Hw[col][r] = x[q];
      }
    }
    __syncwarp();
  }
}

// Applies the logged reflectors of one chunk (buffer buf) to one item: the
// NR entries p[r * stride], r in [0, NR) (rows kbase + r of a column, or
// columns kbase + r of a row); entries outside [rlo, rhi] are not read (zero)
// nor written.  Step t's reflector of bulge b acts on entries
// (t + 2 (NS-1-b), +1), so after step t entry t is final: the register
// window y slides down by two entries every two steps (y[j] = x[t + j]) and
// the rotations use fixed register indices inside a rolled loop, which keeps
// the hot loop small enough for the instruction cache.  Inactive reflectors
// are logged as tau = v2 = 0, the identity, so no rotation is branched.
template <bool LEFT>
__device__ __forceinline__ void ms_rotate_item(const Smem& sm, int buf, double2* p, long long stride,
                                               int rlo, int rhi) {
  double2 y[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) y[r] = (r >= rlo && r <= rhi) ? p[r * stride] : cmk(0.0, 0.0);
#pragma unroll 1
  for (int t = 0; t < MW; t += 2) {
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int b = 0; b < NS; ++b) {
        const int q = h + 2 * (NS - 1 - b);
        const double2 tau = lds2(&sm.rtau[buf][t + h][b]), v2 = lds2(&sm.rv[buf][t + h][b]);
        if (LEFT)
          refl_left(y[q], y[q + 1], tau, v2);
        else
          refl_right(y[q], y[q + 1], tau, v2);
      }
    if (t >= rlo && t <= rhi) p[t * stride] = y[0];
    if (t + 1 >= rlo && t + 1 <= rhi) p[(t + 1) * stride] = y[1];
#pragma unroll
    for (int j = 0; j + 2 < NR; ++j) y[j] = y[j + 2];
  }
#pragma unroll
  for (int r = 0; r + MW < NR; ++r)
    if (r + MW >= rlo && r + MW <= rhi) p[(r + MW) * stride] = y[r];
}

// Left application to H columns [c0, c1), rows [lo, hi], by warp group
// member g of ng.  A column segment is contiguous in memory, so the warp
// moves 32 columns at a time through its staging tile st[32][NR] with
// coalesced loads and stores (one lane per row), and each lane rotates one
// column in registers.
__device__ __noinline__ void ms_apply_cols(const Smem& sm, int buf, double2* H, int ld, int kbase, int lo,
                                           int hi, int c0, int c1, double2* st, int g, int ng, int lane) {
  const int row = kbase + lane;
  const bool rok = lane < NR && row >= lo && row <= hi;
  for (int t0 = c0 + 32 * g; t0 < c1; t0 += 32 * ng) {
    const int ncol = min(32, c1 - t0);
    const double2* src = H + (long long)t0 * ld + row;
    // all loads of a batch are issued before any staging store (the stores
    // could alias the global source as far as the compiler knows)
#pragma unroll
    for (int cb = 0; cb < 32; cb += 16) {
      double2 v[16];
#pragma unroll
      for (int u = 0; u < 16; ++u)
        v[u] = (cb + u < ncol && rok) ? src[(long long)(cb + u) * ld] : cmk(0.0, 0.0);
#pragma unroll
      for (int u = 0; u < 16; ++u)
        if (cb + u < ncol && lane < NR) st[(cb + u) * NR + lane] = v[u];
    }
    __syncwarp();
    if (lane < ncol) ms_rotate_item<true>(sm, buf, st + lane * NR, 1, 0, NR - 1);
    __syncwarp();
    double2* dst = H + (long long)t0 * ld + row;
#pragma unroll
    for (int cb = 0; cb < 32; cb += 16) {
      double2 v[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) v[u] = st[(cb + u) * NR + (lane < NR ? lane : 0)];
#pragma unroll
      for (int u = 0; u < 16; ++u)
        if (cb + u < ncol && rok) dst[(long long)(cb + u) * ld] = v[u];
    }
    __syncwarp();
  }
}

// Right application to H rows [0, nB) and all n rows of Z at columns
// [lo, hi]; one row per thread (lanes take consecutive rows: coalesced).
__device__ __noinline__ void ms_apply_rows(const Smem& sm, int buf, double2* H, double2* Z, int ld, int n,
                                           int kbase, int lo, int hi, int nB, int first, int stride) {
  for (int it = first; it < nB + n; it += stride) {
    double2* p = (it < nB) ? H + it : Z + (it - nB);
    ms_rotate_item<false>(sm, buf, p + (long long)kbase * ld, ld, lo - kbase, hi - kbase);
  }
}

// Pipelined sweep: while warp 0 brings window c+1 up to date (chunk c's
// reflectors on its new columns), chases it and writes it back, warps 1..
// apply chunk c's reflectors to the remaining far columns, the rows above
// window c and Z.  Window c+1 never overlaps what warps 1.. touch in that
// iteration: their columns lie right of window c+1, their rows above
// window c.
//
// With CL > 1 CTAs per matrix (a thread-block cluster) the far updates are
// shared: the leader CTA (this function) posts the sweep to its helpers
// (schur_helper) and every chunk ends with a cluster barrier instead of a
// CTA barrier; update warp g of NG = update_warps<CL>() takes columns and rows
// g, g + NG, ...
template <int CL>
__device__ void multi_sweep(Smem& sm, double2* stage, double2* H, double2* Z, int ld, int n, int l, int i) {
  constexpr int NG = update_warps<CL>();
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int T = (i - l) + 2 * (NS - 1);
  const int C = (T + MW - 1) / MW;
  auto geom = [&](int c, int& kbase, int& j0, int& j1) {
    kbase = l + c * MW - 2 * (NS - 1);
    j0 = max(l, kbase - 1);
    j1 = min(i, kbase + NR + 1);
  };
  {
    int kb, j0, j1;
    geom(0, kb, j0, j1);
    load_window(sm, H, ld, j0, j1 - j0 + 1);
    __syncthreads();
    if (wid == 0) ms_chase(sm, 0, l, i, T, 0, j0, j1 - j0 + 1, lane);
    __syncthreads();
    store_window(sm, H, ld, j0, j1 - j0 + 1);
    __syncthreads();
  }
  if constexpr (CL > 1) {   // post the sweep; chunk 0's log is ready for the helpers
    if (tid == 0) {
      sm.cmd = 1;
      sm.cmd_l = l;
      sm.cmd_i = i;
    }
    mat_sync<CL>();
  }
  for (int c = 0; c < C; ++c) {
    const int buf = c & 1;
    int kb, j0, j1;
    geom(c, kb, j0, j1);
    const int lo = max(l, kb), hi = min(i, kb + NR - 1);
    const bool next = c + 1 < C;
    int kbn = 0, j0n = 0, j1n = j1;
    if (next) geom(c + 1, kbn, j0n, j1n);
    const long long cc0 = clock64();
    if (wid == 0) {
      if (next) {
        // window c+1's new columns (j1, j1n] still lack chunk c's reflectors
        ms_apply_cols(sm, buf, H, ld, kb, lo, hi, j1 + 1, j1n + 1, stage, 0, 1, lane);
        __syncwarp();
        SCHUR_STAT_T(0, 9, clock64() - cc0);
        // window c+1 (nw <= MWIN <= 32 rows: lane = row) into shared memory,
        // eight columns' loads in flight per lane before any is stored
        const int nw = j1n - j0n + 1;
        const double2* hw = H + (long long)j0n * ld + j0n + lane;
        for (int c0 = 0; c0 < nw; c0 += 8) {
          double2 v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u)
            v[u] = (lane < nw && c0 + u < nw) ? hw[(long long)(c0 + u) * ld] : cmk(0.0, 0.0);
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (lane < nw && c0 + u < nw) sm.Hw[c0 + u][lane] = v[u];
        }
        __syncwarp();
        ms_chase(sm, buf ^ 1, l, i, T, (c + 1) * MW, j0n, nw, lane);
        if (lane < nw) {
          double2* hwo = H + (long long)j0n * ld + j0n + lane;
          for (int cc = 0; cc < nw; ++cc) hwo[(long long)cc * ld] = sm.Hw[cc][lane];
        }
      }
      SCHUR_STAT_T(0, 8, clock64() - cc0);
    } else {
      ms_apply_cols(sm, buf, H, ld, kb, lo, hi, j1n + 1, n, stage + (size_t)wid * 32 * NR, wid - 1, NG, lane);
      ms_apply_rows(sm, buf, H, Z, ld, n, kb, lo, hi, j0, tid - 32, NG * 32);
      SCHUR_STAT_T(32, 10, clock64() - cc0);
    }
    if constexpr (CL > 1)
      mat_sync<CL>();
    else
      __syncthreads();
    SCHUR_STAT(11, clock64() - cc0);
    SCHUR_STAT(12, 1);
  }
}

// Helper CTA `rank` (>= 1) of a cluster: follows the leader's posted sweeps
// and applies each chunk's logged reflectors (copied from the leader's
// shared memory) to its share of the far columns and rows, in lock step with
// the leader's per-chunk cluster barriers; returns when the leader posts 0.
// The barrier sequence mirrors multi_sweep<CL> exactly: one after the post,
// one per chunk; a last one keeps the leader's shared memory alive until
// every helper has read the final command.
template <int CL>
__device__ void schur_helper(Smem& sm, double2* stage, double2* H, double2* Z, int ld, int n, int rank) {
  constexpr int NG = update_warps<CL>();
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int g = NT / 32 - 1 + (NT / 32) * (rank - 1) + wid;
  const Smem* L = cooperative_groups::this_cluster().map_shared_rank(&sm, 0);
  for (;;) {
    mat_sync<CL>();
    if (L->cmd != 1) break;
    const int l = L->cmd_l, i = L->cmd_i;
    const int T = (i - l) + 2 * (NS - 1);
    const int C = (T + MW - 1) / MW;
    for (int c = 0; c < C; ++c) {
      const int buf = c & 1;
      for (int e = tid; e < MW * NS; e += NT) {
        const int st = e / NS, bb = e % NS;
        sm.rtau[buf][st][bb] = L->rtau[buf][st][bb];
        sm.rv[buf][st][bb] = L->rv[buf][st][bb];
      }
      __syncthreads();
      const int kb = l + c * MW - 2 * (NS - 1);
      const int j0 = max(l, kb - 1), j1 = min(i, kb + NR + 1);
      const int lo = max(l, kb), hi = min(i, kb + NR - 1);
      const int j1n = (c + 1 < C) ? min(i, kb + MW + NR + 1) : j1;
      ms_apply_cols(sm, buf, H, ld, kb, lo, hi, j1n + 1, n, stage + (size_t)wid * 32 * NR, g, NG, lane);
      ms_apply_rows(sm, buf, H, Z, ld, n, kb, lo, hi, j0, g * 32 + lane, NG * 32);
      mat_sync<CL>();
    }
  }
  mat_sync<CL>();
}

// ---- aggressive early deflation (zlaqr3 rules) ---------------------------------
// The trailing NWIN x NWIN window of the active block [l, i] is brought to
// Schur form T = V^H H_w V by one warp (single-shift QR with full T and V).
// With s = H(kw, kw-1) the coupling entry, the window's coupling column
// becomes the spike s conj(V(0, :)); eigenvalue j of T is deflatable when
// |s| |V(0, j)| <= max(smlnum, ulp |T(j, j)|) (tested upward from the
// bottom, stopping at the first failure).  If nd > 0 of them deflate, the
// spike of the k = NWIN - nd others is folded into its first entry by one
// reflector, T(0:k, 0:k) is reduced back to Hessenberg form, and V is applied
// to the rest of H (rows above, columns to the right) and to Z.  The k
// undeflated eigenvalues serve as the next sweep's shifts.
constexpr int NWIN = 14;                     // AED window
constexpr int LDW = NWIN + 1;                // column stride of the window arrays
constexpr int AED_MIN = NWIN + 16;           // smallest active block that gets AED

struct AedBuf {      // carved from the dynamic staging area (not used meanwhile)
  double2* T;        // [NWIN][LDW] window, T[col * LDW + row]
  double2* V;        // [NWIN][LDW] Schur vectors
  double2* v;        // [32] current reflector
  double2* sp;       // [32] spike
};
__device__ __forceinline__ AedBuf aed_buf(double2* stage) {
  AedBuf a;
  a.T = stage;
  a.V = stage + NWIN * LDW;
  a.v = stage + 2 * NWIN * LDW;
  a.sp = a.v + 32;
  return a;
}

// Warp-level reflector for x[0..len) held as x = lane < len ? xi : 0:
// H^H x = beta e1 with H = I - tau v v^H, v[0] = 1 (zlarfg).  Writes v to vs.
__device__ __forceinline__ void warp_larfg(double2 xi, int len, int lane, double2* vs, double2& tau,
                                           double& beta) {
  double2 a0;   // alpha = x[0]
  a0.x = __shfl_sync(0xffffffffu, xi.x, 0);
  a0.y = __shfl_sync(0xffffffffu, xi.y, 0);
  const double xn2 = warp_sum((lane >= 1 && lane < len) ? xi.x * xi.x + xi.y * xi.y : 0.0);
  if (xn2 == 0.0 && a0.y == 0.0) {
    tau = cmk(0.0, 0.0);
    beta = a0.x;
    if (lane < len) vs[lane] = lane == 0 ? cmk(1.0, 0.0) : cmk(0.0, 0.0);
    __syncwarp();
    return;
  }
  // scaled norm against overflow (values here are O(|H|))
  const double nrm = sqrt(a0.x * a0.x + a0.y * a0.y + xn2);
  beta = -copysign(nrm, a0.x);
  tau = cmk((beta - a0.x) / beta, -a0.y / beta);
  const double2 sc = crcp(cmk(a0.x - beta, a0.y));
  if (lane < len) vs[lane] = lane == 0 ? cmk(1.0, 0.0) : cmul(xi, sc);
  __syncwarp();
}

// Left application of H^H to rows [r0, r0+len) of window columns [c0, NWIN)
// (one lane per column).
__device__ __forceinline__ void warp_left(double2* T, const double2* v, double2 tau, int r0, int len,
                                          int c0, int lane) {
  const int c = lane;
  if (c >= c0 && c < NWIN) {
    double2* col = T + c * LDW + r0;
    double2 w = cmk(0.0, 0.0);
    for (int j = 0; j < len; ++j) w = cadd(w, cmulc(v[j], col[j]));
    const double2 sw = cmulc(tau, w);
    for (int j = 0; j < len; ++j) col[j] = csub(col[j], cmul(v[j], sw));
  }
  __syncwarp();
}
// Right application of H to columns [c0, c0+len) of rows [0, rmax) of A
// (one lane per row).
__device__ __forceinline__ void warp_right(double2* A, const double2* v, double2 tau, int c0, int len,
                                           int rmax, int lane) {
  const int r = lane;
  if (r < rmax) {
    double2 w = cmk(0.0, 0.0);
    for (int j = 0; j < len; ++j) w = cadd(w, cmul(A[(c0 + j) * LDW + r], v[j]));
    const double2 sw = cmul(tau, w);
    for (int j = 0; j < len; ++j) {
      double2& a = A[(c0 + j) * LDW + r];
      a = csub(a, cmulc(v[j], sw));
    }
  }
  __syncwarp();
}

// Schur form of the NWIN x NWIN Hessenberg window (full T, V accumulated),
// one warp.  False when the iteration cap is reached or a shift is not finite.
__device__ bool win_schur(double2* T, double2* V, int lane) {
  const double ulp = DBL_EPSILON;
  int ii = NWIN - 1, its = 0, total = 0;
  auto t = [&](int r, int c) -> double2& { return T[c * LDW + r]; };
  while (ii > 0) {
    bool neg = false;
    if (lane >= 1 && lane <= ii) {
      const double ah = cabs1(t(lane, lane - 1));
      neg = ah <= ulp * (cabs1(t(lane - 1, lane - 1)) + cabs1(t(lane, lane))) || ah < DBL_MIN;
    }
    const unsigned msk = __ballot_sync(0xffffffffu, neg);
    const int ll = msk ? 31 - __clz(msk) : 0;
    if (ll == ii) {
      if (lane == 0) t(ii, ii - 1) = cmk(0.0, 0.0);
      __syncwarp();
      --ii;
      its = 0;
      continue;
    }
    if (ll > 0 && lane == 0) t(ll, ll - 1) = cmk(0.0, 0.0);
    if (++total > 30 * NWIN * 4) return false;
    ++its;
    double2 mu;
    if (its % 10 == 0)
      mu = cadd(t(ii, ii), cmk(0.75 * fabs(t(ii, ii - 1).x), 0.0));
    else
      mu = wilkinson_shift(t(ii - 1, ii - 1), t(ii - 1, ii), t(ii, ii - 1), t(ii, ii));
    if (!cfinite(mu)) return false;
    __syncwarp();
    for (int k = ll; k < ii; ++k) {
      double2 alpha, x;
      if (k == ll) {
        alpha = csub(t(k, k), mu);
        x = t(k + 1, k);
      } else {
        alpha = t(k, k - 1);
        x = t(k + 1, k - 1);
      }
      double beta;
      double2 tau, v2;
      larfg2(alpha, x, beta, tau, v2);
      __syncwarp();
      if (k > ll && lane == 0) {
        t(k, k - 1) = cmk(beta, 0.0);
        t(k + 1, k - 1) = cmk(0.0, 0.0);
      }
      if (lane >= k && lane < NWIN) refl_left(T[lane * LDW + k], T[lane * LDW + k + 1], tau, v2);
      __syncwarp();
      if (lane <= min(k + 2, ii)) refl_right(T[k * LDW + lane], T[(k + 1) * LDW + lane], tau, v2);
      if (lane < NWIN) refl_right(V[k * LDW + lane], V[(k + 1) * LDW + lane], tau, v2);
      __syncwarp();
    }
  }
  return true;
}

// Y[0:len) <- Y V (row vector times the window's V), Y strided by ys.
__device__ __forceinline__ void row_times_v(double2* Y, long long ys, const double2* V) {
  double2 y[NWIN];
#pragma unroll
  for (int j = 0; j < NWIN; ++j) y[j] = Y[j * ys];
#pragma unroll 1
  for (int q = 0; q < NWIN; ++q) {
    double2 acc = cmk(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < NWIN; ++j) cfma(acc, y[j], V[q * LDW + j]);
    Y[q * ys] = acc;
  }
}
// Y[0:len) <- V^H Y (column vector), Y strided by ys.
__device__ __forceinline__ void vh_times_col(double2* Y, long long ys, const double2* V) {
  double2 y[NWIN];
#pragma unroll
  for (int j = 0; j < NWIN; ++j) y[j] = Y[j * ys];
#pragma unroll 1
  for (int q = 0; q < NWIN; ++q) {
    double2 acc = cmk(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < NWIN; ++j) acc = cadd(acc, cmulc(V[q * LDW + j], y[j]));
    Y[q * ys] = acc;
  }
}

// V applied outside the window: H rows [0, kw), H columns (i, n), Z rows.
__device__ __noinline__ void aed_apply(const double2* V, double2* H, double2* Z, int ld, int n, int kw,
                                       int i) {
  const int nA = kw, nB = n - 1 - i, total = nA + nB + n;
  for (int it = threadIdx.x; it < total; it += NT) {
    if (it < nA)
      row_times_v(H + (long long)kw * ld + it, ld, V);
    else if (it < nA + nB)
      vh_times_col(H + (long long)(i + 1 + it - nA) * ld + kw, 1, V);
    else
      row_times_v(Z + (long long)kw * ld + (it - nA - nB), ld, V);
  }
}

// AED on the active block [l, i] (i - l + 1 >= AED_MIN).  Returns the number
// of deflated eigenvalues (-1 when the window QR failed: H unchanged).  When
// at least NS eigenvalues stay undeflated, the bottom NS of them are written
// to sm.shifts and sm.flag is set to 2.
__device__ int aed(Smem& sm, double2* stage, double2* H, double2* Z, int ld, int n, int l, int i,
                   double smlnum) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const double ulp = DBL_EPSILON;
  const AedBuf A = aed_buf(stage);
  const int kw = i - NWIN + 1;
  for (int e = tid; e < NWIN * NWIN; e += NT) {
    const int r = e % NWIN, c = e / NWIN;
    A.T[c * LDW + r] = (r <= c + 1) ? H[(long long)(kw + c) * ld + kw + r] : cmk(0.0, 0.0);
    A.V[c * LDW + r] = cmk(r == c ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  if (wid == 0) {
    if (lane == 0) sm.flag = 0;
    __syncwarp();
    const bool ok = win_schur(A.T, A.V, lane);
    int nd = -1;
    if (ok) {
      const double2 sp = (kw > l) ? H[(long long)(kw - 1) * ld + kw] : cmk(0.0, 0.0);
      // deflation test upward from the bottom
      bool defl = false;
      if (lane < NWIN) {
        double foo = cabs1(A.T[lane * LDW + lane]);
        if (foo == 0.0) foo = cabs1(sp);
        defl = cabs1(sp) * cabs1(A.V[lane * LDW + 0]) <= fmax(smlnum, ulp * foo);
      }
      const unsigned dm = __ballot_sync(0xffffffffu, defl) & ((1u << NWIN) - 1);
      // trailing run of deflatable eigenvalues: lanes NWIN-1 downward
      const unsigned inv = (~dm) & ((1u << NWIN) - 1);
      nd = inv ? (NWIN - 1 - (31 - __clz(inv))) : NWIN;
      const int k = NWIN - nd;
      if (lane < NS && k >= NS) sm.shifts[lane] = A.T[(k - NS + lane) * LDW + (k - NS + lane)];
      if (lane == 0) sm.flag = (k >= NS) ? 2 : 0;
      if (nd > 0) {
        // spike of the undeflated part, s conj(V(0, j)), j < k
        const double2 spj = (lane < k) ? cmul(sp, cconj(A.V[lane * LDW + 0])) : cmk(0.0, 0.0);
        if (k > 1 && (sp.x != 0.0 || sp.y != 0.0)) {
          double2 tau;
          double beta;
          warp_larfg(spj, k, lane, A.v, tau, beta);
          warp_left(A.T, A.v, tau, 0, k, 0, lane);
          warp_right(A.T, A.v, tau, 0, k, k, lane);
          warp_right(A.V, A.v, tau, 0, k, NWIN, lane);
          if (lane < NWIN) A.sp[lane] = lane == 0 ? cmk(beta, 0.0) : cmk(0.0, 0.0);
          __syncwarp();
          // back to Hessenberg form: T(0:k, 0:k)
          for (int c = 0; c + 2 < k; ++c) {
            const int len = k - c - 1;
            const double2 xi = (lane < len) ? A.T[c * LDW + c + 1 + lane] : cmk(0.0, 0.0);
            double2 tg;
            double bg;
            warp_larfg(xi, len, lane, A.v, tg, bg);
            warp_left(A.T, A.v, tg, c + 1, len, c + 1, lane);
            if (lane < len) A.T[c * LDW + c + 1 + lane] = lane == 0 ? cmk(bg, 0.0) : cmk(0.0, 0.0);
            __syncwarp();
            warp_right(A.T, A.v, tg, c + 1, len, k, lane);
            warp_right(A.V, A.v, tg, c + 1, len, NWIN, lane);
          }
        } else {
          if (lane < NWIN) A.sp[lane] = (lane < k) ? spj : cmk(0.0, 0.0);
          __syncwarp();
        }
      }
    }
    if (lane == 0) sm.l = nd;   // broadcast (sm.l is rewritten by the next scan)
  }
  __syncthreads();
  const int nd = sm.l;
  if (nd <= 0) return nd;
  // write back the window (zero below the subdiagonal) and the spike column
  for (int e = tid; e < NWIN * NWIN; e += NT) {
    const int r = e % NWIN, c = e / NWIN;
    H[(long long)(kw + c) * ld + kw + r] = (r <= c + 1) ? A.T[c * LDW + r] : cmk(0.0, 0.0);
  }
  if (kw > l)
    for (int r = tid; r < NWIN; r += NT) H[(long long)(kw - 1) * ld + kw + r] = A.sp[r];
  aed_apply(A.V, H, Z, ld, n, kw, i);
  __syncthreads();
  return nd;
}

// One matrix per CTA (CL = 1), or per cluster of CL CTAs: the leader (rank
// 0) runs the iteration, helpers share the far updates of its multishift
// sweeps (schur_helper).
template <int CL>
__global__ void __launch_bounds__(NT, 1)
schur_kernel(double2* __restrict__ Hg, int ld, long long stride, int n, double2* __restrict__ Zg,
             double2* __restrict__ lamg, long long slam, uint32_t* __restrict__ status,
             int max_sweeps_per_n) {
  __shared__ Smem sm;
  extern __shared__ double2 stage[];   // [NT/32][32][NR] column staging tiles
  const int b = blockIdx.x / CL;
  int rank = 0;
  if constexpr (CL > 1) rank = (int)cooperative_groups::this_cluster().block_rank();
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
    bad = __syncthreads_or(bad);
    // every CTA of a cluster has read the untouched H before the leader
    // changes it, so all of them take the same branch
    if constexpr (CL > 1) mat_sync<CL>();
    if (bad) {
      if (rank == 0) {
        if (tid == 0) atomicOr(status + b, (unsigned)(ST_NONFINITE | ST_EIG_NOCONV));
        for (int r = tid; r < n; r += NT) lam[r] = cmk(nan(""), nan(""));
      }
      return;
    }
  }
  if constexpr (CL > 1) {
    if (rank != 0) {
      schur_helper<CL>(sm, stage, H, Z, ld, n, rank);
      return;
    }
  }

  const int itmax = 30 * (n > 10 ? n : 10);
  const long long sweep_cap = (long long)max_sweeps_per_n * (n > 10 ? n : 10);
  const long long c_start = clock64();
  long long total = 0;
  bool failed = false;
  int i = n - 1;
  while (i >= 0) {
    int l = 0, kdefl = 0;
    bool conv = false;
    for (int its = 0; its <= itmax; ++its) {
      // deflation: largest k in (l, i] with a negligible H[k, k-1]
      SCHUR_STAT(7, 1);
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
        // aggressive early deflation first (large blocks)
        int ib = i;             // bottom of the block the sweep chases
        bool aed_shifts = false;
        if (m >= AED_MIN) {
          const long long c4 = clock64();
          const int nd = aed(sm, stage, H, Z, ld, n, l, i, smlnum);
          SCHUR_STAT(13, 1);
          SCHUR_STAT(15, clock64() - c4);
          if (nd > 0) {
            SCHUR_STAT(14, nd);
            kdefl = 0;
            // many deflations, or too little left: rescan before sweeping
            if (nd * 100 > NWIN * 14 || (i - nd) - l + 1 < MS_MIN) continue;
            ib = i - nd;
          }
          aed_shifts = nd >= 0 && sm.flag == 2;
          __syncthreads();
        }
        // NS shifts: the window's undeflated eigenvalues, else the eigenvalues
        // of the trailing NS x NS block, or exceptional ones
        bool exc = (kdefl % 6 == 0);
        if (!exc && !aed_shifts) {
          const int q0 = ib - NS + 1;
          for (int e = tid; e < NS * NS; e += NT) {
            const int r = e % NS, c = e / NS;
            sm.Hs[c][r] = (r <= c + 1) ? H[(long long)(q0 + c) * ld + q0 + r] : cmk(0.0, 0.0);
          }
          __syncthreads();
          if (wid == 0) {
            const long long c3 = clock64();
            const bool ok = small_eig(sm, NS, lane);
            SCHUR_STAT(4, clock64() - c3);
            if (lane == 0) sm.flag = ok ? 0 : 1;
          }
          __syncthreads();
          exc = sm.flag != 0;
          if (!exc && tid < NS && !cfinite(sm.shifts[tid])) sm.flag = 1;
          __syncthreads();
          exc = sm.flag != 0;
        }
        if (exc) {
          SCHUR_STAT(5, 1);
          if (tid < NS) {   // zlaqr0: H(k,k) + 0.75 |H(k,k-1)| down the trailing diagonal
            const int k = ib - tid;
            sm.shifts[tid] = cadd(H[(long long)k * ld + k], cmk(0.75 * cabs1(H[(long long)(k - 1) * ld + k]), 0.0));
          }
          __syncthreads();
        }
        const long long c1 = clock64();
        multi_sweep<CL>(sm, stage, H, Z, ld, n, l, ib);
        SCHUR_STAT(0, 1);
        SCHUR_STAT(2, clock64() - c1);
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
        const long long c2 = clock64();
        single_sweep(sm, H, Z, ld, n, l, i, sm.shift);
        SCHUR_STAT(1, 1);
        SCHUR_STAT(3, clock64() - c2);
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
  if constexpr (CL > 1) {   // release the helpers (schur_helper's last two barriers)
    if (tid == 0) sm.cmd = 0;
    mat_sync<CL>();
    mat_sync<CL>();
  }
  SCHUR_STAT(6, clock64() - c_start);
  (void)c_start;
}

}  // namespace

#ifdef RCWA_SCHUR_STATS
extern "C" int rcwa_debug_schur_stats(unsigned long long* out, int reset) {
  cudaDeviceSynchronize();
  cudaMemcpyFromSymbol(out, g_schur_stats, sizeof(unsigned long long) * 16);
  if (reset) {
    unsigned long long z[16] = {};
    cudaMemcpyToSymbol(g_schur_stats, z, sizeof(z));
  }
  return 0;
}
#endif

// QR sweeps allowed per eigensolve, in units of max(n, 10): 100 unless a
// caller lowers it (rcwa_eig_set_sweep_cap, host-side fault injection)
static std::atomic<int> g_sweeps_per_n{100};

// CTAs per matrix: 0 = chosen per launch (schur_cluster), else forced
// (rcwa_eig_set_cluster_size: 1, 2, 4 or 8)
static std::atomic<int> g_cluster_force{0};

namespace {

constexpr size_t kStageBytes = sizeof(double2) * (NT / 32) * 32 * NR;
constexpr int kClusterMinN = 400;   // below this the chase, not the far updates, bounds a sweep

template <int CL>
int launch_cl(cudaStream_t s, double2* H, int ld, long long sH, int n, double2* Z, double2* lam, long long slam,
              uint32_t* status, int batch, int cap) {
  static bool attr_set[64] = {};   // the attributes are per device
  int dev = 0;
  RCWA_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 64 || !attr_set[dev]) {
    RCWA_CUDA_TRY(cudaFuncSetAttribute(schur_kernel<CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kStageBytes));
    if (dev < 64) attr_set[dev] = true;
  }
  if constexpr (CL == 1) {
    schur_kernel<1><<<batch, NT, kStageBytes, s>>>(H, ld, sH, n, Z, lam, slam, status, cap);
  } else {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)batch * CL);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = kStageBytes;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    RCWA_CUDA_TRY(cudaLaunchKernelEx(&cfg, schur_kernel<CL>, H, ld, sH, n, Z, lam, slam, status, cap));
  }
  return RCWA_OK;
}

// Whether clusters of CL of these CTAs (one SM each) can be resident at all
// on this device (cached per device).
template <int CL>
bool cluster_fits() {
  static int ok[64];   // 0 unknown, 1 yes, 2 no
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  if (!ok[dev]) {
    cudaFuncSetAttribute(schur_kernel<CL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageBytes);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CL);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = kStageBytes;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nc = 0;
    const cudaError_t e = cudaOccupancyMaxActiveClusters(&nc, schur_kernel<CL>, &cfg);
    cudaGetLastError();
    ok[dev] = (e == cudaSuccess && nc > 0) ? 1 : 2;
  }
  return ok[dev] == 1;
}

// CTAs per matrix: several only for large matrices in launches that leave
// SMs idle -- the largest power of two (<= 8) with batch * CL <= SMs (a
// sweep's far updates then run on CL SMs; as many matrices as SMs already
// fill the device one CTA each).
int schur_cluster(int n, int batch) {
  const int f = g_cluster_force.load();
  if (f > 0) return f;
  if (n < kClusterMinN) return 1;
  static int sms[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
  if (!sms[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    sms[dev] = v > 0 ? v : 1;
  }
  int cl = 1;
  while (cl < 8 && (long long)batch * (cl * 2) <= sms[dev]) cl *= 2;
  return cl;
}

}  // namespace

int schur_launch(cudaStream_t s, double2* H, int ld, long long sH, int n, double2* Z, double2* lam,
                 long long slam, uint32_t* status, int batch) {
  void* tok = prof_begin(s);
  const int cap = g_sweeps_per_n.load();
  int cl = schur_cluster(n, batch);
  if (cl >= 8 && !cluster_fits<8>()) cl = 4;
  if (cl >= 4 && !cluster_fits<4>()) cl = 2;
  if (cl >= 2 && !cluster_fits<2>()) cl = 1;
  int rc;
  switch (cl) {
    case 8: rc = launch_cl<8>(s, H, ld, sH, n, Z, lam, slam, status, batch, cap); break;
    case 4: rc = launch_cl<4>(s, H, ld, sH, n, Z, lam, slam, status, batch, cap); break;
    case 2: rc = launch_cl<2>(s, H, ld, sH, n, Z, lam, slam, status, batch, cap); break;
    default: rc = launch_cl<1>(s, H, ld, sH, n, Z, lam, slam, status, batch, cap); break;
  }
  if (rc) return rc;
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

extern "C" int rcwa_eig_set_cluster_size(int ctas_per_matrix) {
  if (ctas_per_matrix != 0 && ctas_per_matrix != 1 && ctas_per_matrix != 2 && ctas_per_matrix != 4 &&
      ctas_per_matrix != 8) {
    rcwa::set_last_error("ctas_per_matrix must be 0 (automatic), 1, 2, 4 or 8");
    return RCWA_ERR_INVALID;
  }
  rcwa::g_cluster_force.store(ctas_per_matrix);
  return RCWA_OK;
}

extern "C" int rcwa_eig_set_sweep_cap(int sweeps_per_n) {
  if (sweeps_per_n < -1) {
    rcwa::set_last_error("sweeps_per_n must be -1 (default) or >= 0");
    return RCWA_ERR_INVALID;
  }
  rcwa::g_sweeps_per_n.store(sweeps_per_n < 0 ? 100 : sweeps_per_n);
  return RCWA_OK;
}
