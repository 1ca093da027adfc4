// RCWA-specific kernels: Fourier convolution matrices, wave vectors, P/Q
// assembly, per-mode (2x2-block) S-matrices of uniform layers and of the
// reflection / transmission half-spaces, and the final field/efficiency
// extraction.  Every formula cites the reference line it restates.
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {

constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Non-fused complex helpers: the reference's host build contracts nothing, and
// Kz = 0 exactly at a Rayleigh anomaly must stay exactly 0 here too.
__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b) {
  return cmk(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
             __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 csub_rn(double2 a, double2 b) {
  return cmk(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}

// ---------------------------------------------------------------------------
// K1: convolution matrices (rcwa.cpp:6-82) without a full 2-D FFT.
// The Toeplitz gather only reads Fourier coefficients with
// |kx| <= 2*nxh, |ky| <= 2*nyh, so those (2P-1)(2Q-1) coefficients are
// computed as separable DFT sums (row pass then column pass).  A coefficient
// whose shifted index falls outside [0, Nx) x [0, Ny) is 0, as at rcwa.cpp:73;
// inside, the DFT at frequency k equals the FFT bin k mod N that the
// fftshift of rcwa.cpp:44-53 moves to index k + N/2.
// ---------------------------------------------------------------------------
__global__ void twiddle_kernel(double2* tw, int N) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  double s, c;
  sincospi(2.0 * (double)j / (double)N, &s, &c);
  tw[j] = cmk(c, -s);  // exp(-2 pi i j / N)
}

// Row pass: Fx[l][iy][u] = sum_ix f[l][iy][ix] w_nx^(kx ix), kx = u - (P-1).
__global__ void __launch_bounds__(256)
convmat_row_kernel(const double2* __restrict__ grids, int nx, int ny, int P,
                   const double2* __restrict__ twx, double2* __restrict__ Fx) {
  extern __shared__ __align__(16) double2 sm[];
  double2* row = sm;        // [nx]
  double2* tw = sm + nx;    // [nx]
  const int iy = blockIdx.x, l = blockIdx.y;
  const double2* src = grids + ((long long)l * ny + iy) * nx;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    row[i] = src[i];        // 16-byte coalesced loads
    tw[i] = twx[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nu = 2 * P - 1;
  for (int u = wid; u < nu; u += nw) {
    const int kx = u - (P - 1);
    const int km = ((kx % nx) + nx) % nx;
    int idx = (int)(((long long)km * lane) % nx);
    const int step = (int)(((long long)km * 32) % nx);
    double sr = 0.0, si = 0.0;
    for (int ix = lane; ix < nx; ix += 32) {
      double2 f = row[ix], w = tw[idx];
      sr = fma(f.x, w.x, fma(-f.y, w.y, sr));
      si = fma(f.x, w.y, fma(f.y, w.x, si));
      idx += step;
      if (idx >= nx) idx -= nx;
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if (lane == 0) Fx[((long long)l * ny + iy) * nu + u] = cmk(sr, si);
  }
}

// Column pass: Cg[l][v][u] = (1/(nx ny)) sum_iy Fx[l][iy][u] w_ny^(ky iy),
// zeroed where the shifted index is outside the grid.
__global__ void __launch_bounds__(256)
convmat_col_kernel(const double2* __restrict__ Fx, int nx, int ny, int P, int Q,
                   const double2* __restrict__ twy, double2* __restrict__ Cg) {
  const int l = blockIdx.y;
  const int nu = 2 * P - 1, nv = 2 * Q - 1;
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (gw >= nu * nv) return;
  const int u = gw % nu, v = gw / nu;
  const int kx = u - (P - 1), ky = v - (Q - 1);
  const bool ok = (kx + nx / 2 >= 0) && (kx + nx / 2 < nx) && (ky + ny / 2 >= 0) && (ky + ny / 2 < ny);
  double2 out = cmk(0.0, 0.0);
  if (ok) {
    const int km = ((ky % ny) + ny) % ny;
    int idx = (int)(((long long)km * lane) % ny);
    const int step = (int)(((long long)km * 32) % ny);
    double sr = 0.0, si = 0.0;
    const double2* F = Fx + (long long)l * ny * nu + u;
    for (int iy = lane; iy < ny; iy += 32) {
      double2 f = F[(long long)iy * nu], w = twy[idx];
      sr = fma(f.x, w.x, fma(-f.y, w.y, sr));
      si = fma(f.x, w.y, fma(f.y, w.x, si));
      idx += step;
      if (idx >= ny) idx -= ny;
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    const double nrm = (double)nx * (double)ny;   // F /= Nx*Ny, rcwa.cpp:41
    out = cmk(sr / nrm, si / nrm);
  }
  if (lane == 0) Cg[(long long)l * nu * nv + v * nu + u] = out;
}

// Toeplitz gather (rcwa.cpp:61-78): C(m, n) = F(py_m - py_n, px_m - px_n).
__global__ void convmat_gather_kernel(const double2* __restrict__ Cg, int P, int Q,
                                      double2* __restrict__ out) {
  const int N = P * Q;
  const int l = blockIdx.y;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)N * N) return;
  const int m = (int)(e % N), n = (int)(e / N);
  const int dkx = m / Q - n / Q, dky = m % Q - n % Q;
  const int nu = 2 * P - 1;
  out[(long long)l * N * N + e] = Cg[(long long)l * nu * (2 * Q - 1) + (dky + Q - 1) * nu + (dkx + P - 1)];
}

// ---------------------------------------------------------------------------
// Li's factorization rule (L. Li, J. Opt. Soc. Am. A 14, 2758 (1997)), an
// option beside the reference's Laurent rule: eps_aa = [[ [[eps]]_a ]]_b.
// Along every grid line of axis a (fixed coordinate ib on the other axis b)
// the Pa x Pa Toeplitz matrix of 1/eps is formed and inverted; the inverses
// are then convolved along b and gathered into the N x N mode matrix
// (m = p*Q + q).  Axis a = x: lines are grid rows (stride 1); a = y: grid
// columns (stride nx).  The DFT coefficients follow the ConvMat conventions
// above: 1/n normalisation and 0 where k + n/2 falls outside [0, n).
// ---------------------------------------------------------------------------

// One CTA per (line ib, layer l): the line's reciprocals and the twiddles in
// shared memory, one warp per coefficient k = u - (Pa-1), then the augmented
// system [T | I] (Pa x 2Pa, column-major) with T(p, p') = a(p - p').
__global__ void __launch_bounds__(256)
li_line_kernel(const double2* __restrict__ grids, int na, int nb, long long sa, long long sb,
               long long sl, int Pa, const double2* __restrict__ tw_a, double2* __restrict__ aug,
               int* __restrict__ bad) {
  extern __shared__ __align__(16) double2 sm[];
  double2* line = sm;          // [na]
  double2* tw = sm + na;       // [na]
  double2* coef = tw + na;     // [2Pa-1]
  const int ib = blockIdx.x, l = blockIdx.y;
  const double2* src = grids + l * sl + ib * sb;
  bool nonfinite = false;
  for (int i = threadIdx.x; i < na; i += blockDim.x) {
    const double2 r = crcp(src[i * sa]);
    nonfinite |= !(isfinite(r.x) && isfinite(r.y));
    line[i] = r;
    tw[i] = tw_a[i];
  }
  if (__syncthreads_or(nonfinite) && threadIdx.x == 0) atomicOr(bad, 1);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nu = 2 * Pa - 1;
  for (int u = wid; u < nu; u += nw) {
    const int k = u - (Pa - 1);
    double sr = 0.0, si = 0.0;
    if (k + na / 2 >= 0 && k + na / 2 < na) {
      const int km = ((k % na) + na) % na;
      int idx = (int)(((long long)km * lane) % na);
      const int step = (int)(((long long)km * 32) % na);
      for (int i = lane; i < na; i += 32) {
        const double2 f = line[i], w = tw[idx];
        sr = fma(f.x, w.x, fma(-f.y, w.y, sr));
        si = fma(f.x, w.y, fma(f.y, w.x, si));
        idx += step;
        if (idx >= na) idx -= na;
      }
      sr = warp_sum(sr) / (double)na;
      si = warp_sum(si) / (double)na;
    }
    if (lane == 0) coef[u] = cmk(sr, si);
  }
  __syncthreads();
  double2* A = aug + ((long long)l * nb + ib) * 2 * Pa * Pa;
  for (int e = threadIdx.x; e < 2 * Pa * Pa; e += blockDim.x) {
    const int r = e % Pa, c = e / Pa;
    A[e] = c < Pa ? coef[r - c + Pa - 1] : cmk(r == c - Pa ? 1.0 : 0.0, 0.0);
  }
}

// Laurent pass along b: Cg[l][v][p'][p] = (1/nb) sum_ib M_ib(p, p') w_nb^(kb ib),
// kb = v - (Pb-1), M_ib the inverse in the right half of line ib's system.
// One warp per (p, p', v).
__global__ void __launch_bounds__(256)
li_cross_kernel(const double2* __restrict__ aug, int nb, int Pa, int Pb,
                const double2* __restrict__ tw_b, double2* __restrict__ Cg) {
  const int l = blockIdx.y;
  const int nv = 2 * Pb - 1, PP = Pa * Pa;
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (gw >= PP * nv) return;
  const int e = gw % PP, v = gw / PP;      // e = p' * Pa + p (column-major element)
  const int kb = v - (Pb - 1);
  double2 out = cmk(0.0, 0.0);
  if (kb + nb / 2 >= 0 && kb + nb / 2 < nb) {
    const int km = ((kb % nb) + nb) % nb;
    int idx = (int)(((long long)km * lane) % nb);
    const int step = (int)(((long long)km * 32) % nb);
    double sr = 0.0, si = 0.0;
    const double2* M = aug + (long long)l * nb * 2 * PP + PP + e;
    for (int ib = lane; ib < nb; ib += 32) {
      const double2 f = M[(long long)ib * 2 * PP], w = tw_b[idx];
      sr = fma(f.x, w.x, fma(-f.y, w.y, sr));
      si = fma(f.x, w.y, fma(f.y, w.x, si));
      idx += step;
      if (idx >= nb) idx -= nb;
    }
    out = cmk(warp_sum(sr) / (double)nb, warp_sum(si) / (double)nb);
  }
  if (lane == 0) Cg[((long long)l * nv + v) * PP + e] = out;
}

// bad |= 2 when any line's Toeplitz system reported a zero pivot
__global__ void li_any_kernel(const uint32_t* __restrict__ st, long long n, int* bad) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (__syncthreads_or(i < n && st[i] != 0) && threadIdx.x == 0) atomicOr(bad, 2);
}

// out(m, n) = Cg[v = b_m - b_n + Pb - 1][a_n][a_m], (a, b) = (p, q) for axis
// x and (q, p) for axis y.
__global__ void li_gather_kernel(const double2* __restrict__ Cg, int P, int Q, int axis_y,
                                 double2* __restrict__ out) {
  const int N = P * Q;
  const int l = blockIdx.y;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)N * N) return;
  const int m = (int)(e % N), n = (int)(e / N);
  const int Pa = axis_y ? Q : P, Pb = axis_y ? P : Q;
  const int am = axis_y ? m % Q : m / Q, bm = axis_y ? m / Q : m % Q;
  const int an = axis_y ? n % Q : n / Q, bn = axis_y ? n / Q : n % Q;
  const long long PP = (long long)Pa * Pa;
  out[(long long)l * N * N + e] = Cg[((long long)l * (2 * Pb - 1) + (bm - bn + Pb - 1)) * PP + an * Pa + am];
}

// ---------------------------------------------------------------------------
// K2: wave vectors (rcwa.cpp:85-160) and gap modes (rcwa.cpp:163-234).
// ---------------------------------------------------------------------------
__global__ void wavevec_kernel(const SourceDev* __restrict__ srcs, int nxh,
                               int nyh, int Q, int N, double2 er_ref, double2 ur_ref,
                               double2 er_trn, double2 ur_trn, WaveVecs w,
                               uint32_t* __restrict__ status) {
  const int b = blockIdx.x;
  const SourceDev sv = srcs[b];
  const double2 n_inc = csqrt_principal(cmul_rn(er_ref, ur_ref));   // std::sqrt, :91
  const double st = sin(sv.theta), ct = cos(sv.theta);
  const double sp = sin(sv.phi), cp = cos(sv.phi);
  const double2 k0x = cscale(cscale(n_inc, st), cp);                 // :99
  const double2 k0y = cscale(cscale(n_inc, st), sp);                 // :102
  const double2 k0z = cscale(n_inc, ct);                             // :103
  if (threadIdx.x == 0) {
    double2* ki = w.kinc + (long long)b * 4;
    ki[0] = k0x;
    ki[1] = k0y;
    ki[2] = k0z;
    ki[3] = cmk(2.0 * kPi / sv.lambda0, 0.0);                        // k0, rcwa.hpp:92
  }
  const double cx = -(sv.lambda0 / sv.lx), cy = -(sv.lambda0 / sv.ly);    // :110, :113
  const double2 a_ref = cmul_rn(cconj(ur_ref), cconj(er_ref));
  const double2 a_trn = cmul_rn(cconj(ur_trn), cconj(er_trn));
  bool wood = false;
  for (int m = threadIdx.x; m < N; m += blockDim.x) {
    const int p = m / Q - nxh, q = m % Q - nyh;                      // m = p*Q + q
    const double2 kx = cmk(__dadd_rn(__dmul_rn((double)p, cx), k0x.x), __dadd_rn(__dmul_rn(0.0, cx), k0x.y));
    const double2 ky = cmk(__dadd_rn(__dmul_rn((double)q, cy), k0y.x), __dadd_rn(__dmul_rn(0.0, cy), k0y.y));
    const double2 kx2 = cmul_rn(kx, kx), ky2 = cmul_rn(ky, ky);
    const double2 kzr = cneg(cconj(usqrt(csub_rn(csub_rn(a_ref, kx2), ky2))));   // :134
    const double2 kzt = cconj(usqrt(csub_rn(csub_rn(a_trn, kx2), ky2)));         // :135
    const double2 kz0 = cconj(usqrt(csub_rn(csub_rn(cmk(1.0, 0.0), kx2), ky2))); // :179
    const long long o = (long long)b * N + m;
    w.Kx[o] = kx;
    w.Ky[o] = ky;
    w.Kzr[o] = kzr;
    w.Kzt[o] = kzt;
    // gap V0 = Q0 / lambda0, lambda0 = [i Kz0; i Kz0] (:186-226)
    const double2 lam0 = cmul_rn(cmk(0.0, 1.0), kz0);
    const double2 kxky = cmul_rn(kx, ky);
    double2* v0 = w.V0 + (long long)b * 4 * N;
    v0[m] = cdiv(kxky, lam0);                                         // (i, i)
    v0[N + m] = cdiv(csub_rn(cmk(1.0, 0.0), kx2), lam0);              // (i, i+N)
    v0[2 * N + m] = cdiv(csub_rn(ky2, cmk(1.0, 0.0)), lam0);          // (i+N, i)
    v0[3 * N + m] = cdiv(cneg(kxky), lam0);                           // (i+N, i+N)
    if ((kz0.x == 0.0 && kz0.y == 0.0) || (kzr.x == 0.0 && kzr.y == 0.0) ||
        (kzt.x == 0.0 && kzt.y == 0.0))
      wood = true;
  }
  if (__syncthreads_or(wood) && threadIdx.x == 0) atomicOr(status + b, (unsigned)ST_WOOD);
}

// ---------------------------------------------------------------------------
// P_i and Q_i of a patterned layer (rcwa.cpp:262-286); Kx/Ky diagonal, so
// erc^-1 diag(K) is a column scaling of erc^-1.  exx/eyy/mxx/myy are the
// in-plane permittivity / permeability matrices (all erc / urc under the
// reference's Laurent rule).
// ---------------------------------------------------------------------------
__global__ void assemble_pq_kernel(int N, const double2* __restrict__ exx,
                                   const double2* __restrict__ eyy,
                                   const double2* __restrict__ mxx,
                                   const double2* __restrict__ myy,
                                   const double2* __restrict__ einv,
                                   const double2* __restrict__ uinv, long long s_item,
                                   const double2* __restrict__ Kxg,
                                   const double2* __restrict__ Kyg, double2* __restrict__ P,
                                   double2* __restrict__ Qm) {
  const int b = blockIdx.y;
  const int n = 2 * N;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * n) return;
  const int i = (int)(e % n), j = (int)(e / n);
  const int bi = i >= N, bj = j >= N;
  const int ii = i - bi * N, jj = j - bj * N;
  const double2* Kx = Kxg + (long long)b * N;
  const double2* Ky = Kyg + (long long)b * N;
  const long long o = (long long)b * s_item + (long long)jj * N + ii;
  const double2 ei = einv[o], ui = uinv[o];
  double2 p, q;
  if (!bi && !bj) {
    p = cmul(Kx[ii], cmul(ei, Ky[jj]));                   // :273
    q = cmul(Kx[ii], cmul(ui, Ky[jj]));                   // :282
  } else if (!bi && bj) {
    p = csub(myy[o], cmul(Kx[ii], cmul(ei, Kx[jj])));     // :274
    q = csub(eyy[o], cmul(Kx[ii], cmul(ui, Kx[jj])));     // :283
  } else if (bi && !bj) {
    p = csub(cmul(Ky[ii], cmul(ei, Ky[jj])), mxx[o]);     // :275
    q = csub(cmul(Ky[ii], cmul(ui, Ky[jj])), exx[o]);     // :284
  } else {
    p = cmul(cneg(Ky[ii]), cmul(ei, Kx[jj]));             // :276
    q = cmul(cneg(Ky[ii]), cmul(ui, Kx[jj]));             // :285
  }
  const long long ob = (long long)b * n * n + e;
  P[ob] = p;
  Qm[ob] = q;
}

__global__ void layer_modes_kernel(int n, const double2* __restrict__ lam2,
                                   const double2* __restrict__ kinc, double t,
                                   const double* __restrict__ t_item, int t_stride,
                                   double2* __restrict__ lam, double2* __restrict__ ilam,
                                   double2* __restrict__ X) {
  const int b = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  if (t_item) t = t_item[(long long)b * t_stride];
  const long long o = (long long)b * n + j;
  const double k0 = kinc[(long long)b * 4 + 3].x;
  const double2 l = usqrt(lam2[o]);                       // :317
  lam[o] = l;
  ilam[o] = crcp(l);                                      // V columns / lambda, :329
  X[o] = cexp(cscale(l, -k0 * t));                        // :339
}

__global__ void assemble_ab_kernel(int N, const double2* __restrict__ Wi, long long sWi,
                                   const double2* __restrict__ Vi, long long sVi,
                                   const double2* __restrict__ V0g, double2* __restrict__ A,
                                   double2* __restrict__ Bm) {
  const int b = blockIdx.y;
  const int n = 2 * N;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * n) return;
  const int i = (int)(e % n), j = (int)(e / n);
  const double2* vi = Vi + (long long)b * sVi;
  const double2* V0 = V0g + (long long)b * 4 * N;
  double2 vv;
  if (j < N) {
    vv = cadd(cmul(vi[(long long)j * n + i], V0[j]), cmul(vi[(long long)(j + N) * n + i], V0[2 * N + j]));
  } else {
    const int jj = j - N;
    vv = cadd(cmul(vi[(long long)jj * n + i], V0[N + jj]), cmul(vi[(long long)j * n + i], V0[3 * N + jj]));
  }
  const double2 wi = Wi[(long long)b * sWi + e];
  A[(long long)b * n * n + e] = cadd(wi, vv);             // :337
  Bm[(long long)b * n * n + e] = csub(wi, vv);            // :338
}

// ---- 2x2 complex helpers for the per-mode block algebra --------------------
struct C22 {
  double2 a, b, c, d;  // [[a, b], [c, d]]
};
__device__ __forceinline__ C22 m22(double2 a, double2 b, double2 c, double2 d) { return {a, b, c, d}; }
__device__ __forceinline__ C22 mmul(const C22& x, const C22& y) {
  return {cadd(cmul(x.a, y.a), cmul(x.b, y.c)), cadd(cmul(x.a, y.b), cmul(x.b, y.d)),
          cadd(cmul(x.c, y.a), cmul(x.d, y.c)), cadd(cmul(x.c, y.b), cmul(x.d, y.d))};
}
__device__ __forceinline__ C22 madd(const C22& x, const C22& y) {
  return {cadd(x.a, y.a), cadd(x.b, y.b), cadd(x.c, y.c), cadd(x.d, y.d)};
}
__device__ __forceinline__ C22 msub(const C22& x, const C22& y) {
  return {csub(x.a, y.a), csub(x.b, y.b), csub(x.c, y.c), csub(x.d, y.d)};
}
__device__ __forceinline__ C22 mscale(const C22& x, double2 s) {
  return {cmul(x.a, s), cmul(x.b, s), cmul(x.c, s), cmul(x.d, s)};
}
__device__ __forceinline__ C22 minv(const C22& x) {
  // partial-pivoting 2x2 inverse (same pivot rule as the LU it replaces)
  double2 det;
  if (cabs1(x.a) >= cabs1(x.c)) {
    double2 l = cdiv(x.c, x.a);
    double2 u22 = csub(x.d, cmul(l, x.b));
    det = cmul(x.a, u22);
  } else {
    double2 l = cdiv(x.a, x.c);
    double2 u22 = csub(x.b, cmul(l, x.d));
    det = cneg(cmul(x.c, u22));
  }
  double2 id = crcp(det);
  return {cmul(x.d, id), cneg(cmul(x.b, id)), cneg(cmul(x.c, id)), cmul(x.a, id)};
}
__device__ __forceinline__ C22 meye() { return {cmk(1, 0), cmk(0, 0), cmk(0, 0), cmk(1, 0)}; }

__device__ __forceinline__ void store22(double2* M, int n, int N, int i, const C22& x) {
  M[(long long)i * n + i] = x.a;
  M[(long long)(i + N) * n + i] = x.b;
  M[(long long)i * n + i + N] = x.c;
  M[(long long)(i + N) * n + i + N] = x.d;
}

// "BD" storage of a 2x2-block-diagonal n x n block X: four diagonals
// [X(i,i), X(i,i+N), X(i+N,i), X(i+N,i+N)], each of length N.
__device__ __forceinline__ void store22x(double2* M, int n, int N, int i, const C22& x, bool bd) {
  if (bd) {
    M[i] = x.a;
    M[N + i] = x.b;
    M[2 * N + i] = x.c;
    M[3 * N + i] = x.d;
  } else {
    store22(M, n, N, i, x);
  }
}

__device__ __forceinline__ C22 gap_v0(const double2* V0, int N, int i) {
  return m22(V0[i], V0[N + i], V0[2 * N + i], V0[3 * N + i]);
}

// Uniform layer: erc = eps I, urc = mu I, so P, Q, Omega^2 and every matrix
// of rcwa.cpp:262-351 is 2x2-block diagonal over the (i, i+N) pairs and
// Omega^2 = (kx^2 + ky^2 - mu eps) I.  The eigenbasis W = I is used; S is
// invariant to the choice of basis inside the degenerate pairs.
__global__ void uniform_layer_kernel(int N, double2 eps, double2 mu, double t,
                                     const double2* __restrict__ eps_item,
                                     const double2* __restrict__ mu_item,
                                     const double* __restrict__ t_item, int stride, WaveVecs w,
                                     double2* __restrict__ S11g, double2* __restrict__ S12g,
                                     long long sS, int bd) {
  const int b = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  if (eps_item) eps = eps_item[(long long)b * stride];
  if (mu_item) mu = mu_item[(long long)b * stride];
  if (t_item) t = t_item[(long long)b * stride];
  const int n = 2 * N;
  const long long o = (long long)b * N + i;
  const double2 kx = w.Kx[o], ky = w.Ky[o];
  const double k0 = w.kinc[(long long)b * 4 + 3].x;
  const double2 imu = crcp(mu);
  // Q_i (rcwa.cpp:280-285) with urc^-1 = 1/mu
  const C22 Qm = m22(cmul(kx, cmul(imu, ky)), csub(eps, cmul(kx, cmul(imu, kx))),
                     csub(cmul(ky, cmul(imu, ky)), eps), cmul(cneg(ky), cmul(imu, kx)));
  const double2 lam2 = csub(cadd(cmul(kx, kx), cmul(ky, ky)), cmul(mu, eps));
  const double2 lam = usqrt(lam2);
  const double2 il = crcp(lam);
  const C22 V = mscale(Qm, il);                          // V = Q W lambda^-1, W = I
  const C22 ViV0 = mmul(minv(V), gap_v0(w.V0 + (long long)b * 4 * N, N, i));
  const C22 A = madd(meye(), ViV0);                      // W^-1 W0 = I
  const C22 B = msub(meye(), ViV0);
  const double2 x = cexp(cscale(lam, -k0 * t));
  const C22 Ai = minv(A);
  const C22 BAi = mmul(B, Ai);
  const double2 x2 = cmul(x, x);
  const C22 D = msub(A, mscale(mmul(BAi, B), x2));       // A - X B A^-1 X B
  const C22 Di = minv(D);
  const C22 S11 = mmul(Di, msub(mscale(mmul(BAi, A), x2), B));          // :347
  const C22 S12 = mscale(mmul(Di, msub(A, mmul(BAi, B))), x);           // :348
  store22x(S11g + (long long)b * sS, n, N, i, S11, bd);
  store22x(S12g + (long long)b * sS, n, N, i, S12, bd);
}

// Reflection (side 0, rcwa.cpp:354-411) / transmission (side 1, :414-466).
__global__ void port_smatrix_kernel(int N, int side, double2 er, double2 ur, WaveVecs w,
                                    double2* __restrict__ S11g, double2* __restrict__ S12g,
                                    double2* __restrict__ S21g, double2* __restrict__ S22g,
                                    long long sS, int bd) {
  const int b = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int n = 2 * N;
  const long long o = (long long)b * N + i;
  const double2 kx = w.Kx[o], ky = w.Ky[o];
  const double2 kz = side == 0 ? w.Kzr[o] : w.Kzt[o];
  const double2 ue = cmul(ur, er);
  const double2 kxky = cmul(kx, ky);
  C22 Qp = m22(kxky, csub(ue, cmul(kx, kx)), csub(cmul(ky, ky), ue), cneg(kxky));
  Qp = m22(cdiv(Qp.a, ur), cdiv(Qp.b, ur), cdiv(Qp.c, ur), cdiv(Qp.d, ur));   // Q /= ur
  const double2 lam = side == 0 ? cmul(cmk(-0.0, -1.0), kz) : cmul(cmk(0.0, 1.0), kz);  // :377 / :437
  const C22 Vp = m22(cdiv(Qp.a, lam), cdiv(Qp.b, lam), cdiv(Qp.c, lam), cdiv(Qp.d, lam));
  const C22 V0iVp = mmul(minv(gap_v0(w.V0 + (long long)b * 4 * N, N, i)), Vp);
  const C22 A = madd(meye(), V0iVp);                     // W0^-1 W_p = I
  const C22 B = msub(meye(), V0iVp);
  const C22 Ai = minv(A);
  const C22 AiB = mmul(Ai, B);
  const C22 half = mscale(msub(A, mmul(B, AiB)), cmk(0.5, 0.0));
  const C22 two = mscale(Ai, cmk(2.0, 0.0));
  const C22 BAi = mmul(B, Ai);
  const C22 mAiB = mscale(AiB, cmk(-1.0, 0.0));
  const long long ob = (long long)b * sS;
  if (side == 0) {   // :405-408
    store22x(S11g + ob, n, N, i, mAiB, bd);
    store22x(S12g + ob, n, N, i, two, bd);
    store22x(S21g + ob, n, N, i, half, bd);
    store22x(S22g + ob, n, N, i, BAi, bd);
  } else {           // :460-463
    store22x(S11g + ob, n, N, i, BAi, bd);
    store22x(S12g + ob, n, N, i, half, bd);
    store22x(S21g + ob, n, N, i, two, bd);
    store22x(S22g + ob, n, N, i, mAiB, bd);
  }
}

// ---- products with BD blocks (O(n^2) instead of a dense GEMM) --------------
// C = beta C + alpha (X M) [side 0]  or  beta C + alpha (M X) [side 1], plus I
// when addI; X is BD, M and C dense (column-major, rows x cols).
__global__ void bd_apply_kernel(int side, int N, int rows, int cols, const double2* __restrict__ Xg,
                                long long sX, const double2* __restrict__ Mg, int ldm, long long sM,
                                double2* __restrict__ Cg, int ldc, long long sC, double2 alpha,
                                double2 beta, int addI) {
  const int b = blockIdx.y;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)rows * cols) return;
  const int i = (int)(e % rows), j = (int)(e / rows);
  const double2* X = Xg + (long long)b * sX;
  const double2* M = Mg + (long long)b * sM;
  double2 v;
  if (side == 0) {
    const int ii = i < N ? i : i - N;
    const double2 m0 = M[(long long)j * ldm + ii], m1 = M[(long long)j * ldm + ii + N];
    v = i < N ? cadd(cmul(X[ii], m0), cmul(X[N + ii], m1))
              : cadd(cmul(X[2 * N + ii], m0), cmul(X[3 * N + ii], m1));
  } else {
    const int jj = j < N ? j : j - N;
    const double2 m0 = M[(long long)jj * ldm + i], m1 = M[(long long)(jj + N) * ldm + i];
    v = j < N ? cadd(cmul(m0, X[jj]), cmul(m1, X[2 * N + jj]))
              : cadd(cmul(m0, X[N + jj]), cmul(m1, X[3 * N + jj]));
  }
  v = cmul(alpha, v);
  if (addI && i == j) v.x += 1.0;
  double2* c = Cg + (long long)b * sC + (long long)j * ldc + i;
  if (beta.x != 0.0 || beta.y != 0.0) v = cadd(v, cmul(beta, *c));
  *c = v;
}

// C[:, 0:2] = beta C + alpha X[:, (a, a+N)] for a BD block X (dense n x 2 out).
__global__ void bd_cols_kernel(int N, int a, const double2* __restrict__ Xg, long long sX,
                               double2* __restrict__ Cg, int ldc, long long sC, double2 alpha,
                               double2 beta) {
  const int b = blockIdx.y;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = 2 * N;
  if (e >= 2 * n) return;
  const int i = e % n, j = e / n;
  const double2* X = Xg + (long long)b * sX;
  double2 v = cmk(0.0, 0.0);
  if (i == a) v = j == 0 ? X[a] : X[N + a];
  else if (i == a + N) v = j == 0 ? X[2 * N + a] : X[3 * N + a];
  v = cmul(alpha, v);
  double2* c = Cg + (long long)b * sC + (long long)j * ldc + i;
  if (beta.x != 0.0 || beta.y != 0.0) v = cadd(v, cmul(beta, *c));
  *c = v;
}

// C (dense n x n) = beta C + X (BD): only the four diagonals are touched when
// beta == 1; with beta == 0 the whole block is written.
__global__ void bd_dense_kernel(int N, const double2* __restrict__ Xg, long long sX,
                                double2* __restrict__ Cg, long long sC, int accumulate) {
  const int b = blockIdx.y;
  const int n = 2 * N;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * n) return;
  const int i = (int)(e % n), j = (int)(e / n);
  const double2* X = Xg + (long long)b * sX;
  const int ii = i < N ? i : i - N, jj = j < N ? j : j - N;
  double2 v = cmk(0.0, 0.0);
  if (ii == jj) v = X[(i >= N ? 2 : 0) * N + (j >= N ? N : 0) + ii];
  double2* c = Cg + (long long)b * sC + e;
  if (accumulate) {
    if (ii == jj) *c = cadd(*c, v);
  } else {
    *c = v;
  }
}

// ---------------------------------------------------------------------------
// K8: source (rcwa.cpp:469-523), fields (:526-561), efficiencies (:564-585).
// ---------------------------------------------------------------------------
__device__ void normalize3(double2 v[3]) {
  double s = cabs2(v[0]) + cabs2(v[1]) + cabs2(v[2]);
  double nrm = sqrt(s);
  if (nrm > 0.0)
    for (int k = 0; k < 3; ++k) v[k] = cmk(v[k].x / nrm, v[k].y / nrm);
}

// Block e computes the efficiencies of source record srcs[e] from the
// S-matrix columns and wave vectors of solve u = map[e] (map null: u = e) and
// writes them to row o = oidx[e] of the outputs (oidx null: o = e).  With
// ustatus, status[o] = ustatus[u] | flags (sources that share one solve);
// otherwise the flags are ORed into status[o].
__global__ void efficiencies_kernel(int N, const SourceDev* __restrict__ srcs, double2 ur_ref,
                                    double2 ur_trn, WaveVecs w, const double2* __restrict__ S11g,
                                    const double2* __restrict__ S21g, long long sS, int compact,
                                    const int* __restrict__ map, const int* __restrict__ oidx,
                                    const uint32_t* __restrict__ ustatus, double* __restrict__ Rg,
                                    double* __restrict__ Tg, double* __restrict__ tot,
                                    uint32_t* __restrict__ status) {
  const int e = blockIdx.x;
  const int b = map ? map[e] : e;         // the solve whose S-matrix and wave vectors are used
  const long long ob = oidx ? oidx[e] : e; // the output row
  const int n = 2 * N;
  __shared__ double2 s_pol[2];
  __shared__ double red[2][32];
  const double2* ki = w.kinc + (long long)b * 4;
  if (threadIdx.x == 0) {
    const SourceDev sv = srcs[e];
    double2 k[3] = {ki[0], ki[1], ki[2]};
    double2 te[3], tm[3], pol[3];
    if (fabs(sv.theta) < 1e-6) {                       // :483-486
      te[0] = cmk(0, 0); te[1] = cmk(1, 0); te[2] = cmk(0, 0);
    } else {
      te[0] = cneg(k[1]); te[1] = k[0]; te[2] = cmk(0, 0);
    }
    normalize3(te);
    tm[0] = csub(cmul(k[1], te[2]), cmul(k[2], te[1]));   // :491
    tm[1] = csub(cmul(k[2], te[0]), cmul(k[0], te[2]));
    tm[2] = csub(cmul(k[0], te[1]), cmul(k[1], te[0]));
    normalize3(tm);
    for (int c = 0; c < 3; ++c) pol[c] = cadd(cscale(te[c], sv.pte), cscale(tm[c], sv.ptm));
    normalize3(pol);                                    // :495-498
    s_pol[0] = pol[0];
    s_pol[1] = pol[1];
  }
  __syncthreads();
  const double2 c1 = s_pol[0], c2 = s_pol[1];          // esrc at PQ/2 and PQ/2+PQ; csrc = esrc (W_ref = I)
  // columns PQ/2 and PQ/2+PQ of S11/S21, or columns 0/1 when only those two
  // columns were formed (compact n x 2 storage)
  const int src0 = compact ? 0 : N / 2, src1 = compact ? 1 : N / 2 + N;
  const double2* S11 = S11g + (long long)b * sS;
  const double2* S21 = S21g + (long long)b * sS;
  const double den = cdiv(ki[2], ur_ref).x;
  double rsum = 0.0, tsum = 0.0;
  bool bad = false;
  for (int m = threadIdx.x; m < N; m += blockDim.x) {
    const long long o = (long long)b * N + m;
    const long long oo = ob * N + m;
    const double2 kx = w.Kx[o], ky = w.Ky[o];
    // r = S11 csrc (:535), r_z (:541)
    double2 rx = cadd(cmul(S11[(long long)src0 * n + m], c1), cmul(S11[(long long)src1 * n + m], c2));
    double2 ry = cadd(cmul(S11[(long long)src0 * n + m + N], c1), cmul(S11[(long long)src1 * n + m + N], c2));
    double2 rz = cdiv(cneg(cadd(cmul(kx, rx), cmul(ky, ry))), w.Kzr[o]);
    double2 tx = cadd(cmul(S21[(long long)src0 * n + m], c1), cmul(S21[(long long)src1 * n + m], c2));
    double2 ty = cadd(cmul(S21[(long long)src0 * n + m + N], c1), cmul(S21[(long long)src1 * n + m + N], c2));
    double2 tz = cdiv(cneg(cadd(cmul(kx, tx), cmul(ky, ty))), w.Kzt[o]);
    const double rr = cabs2(rx) + cabs2(ry) + cabs2(rz);
    const double tt = cabs2(tx) + cabs2(ty) + cabs2(tz);
    const double R = (cdiv(cneg(w.Kzr[o]), ur_ref).x / den) * rr;      // :576
    const double T = (cdiv(w.Kzt[o], ur_trn).x / den) * tt;             // :582
    Rg[oo] = R;   // column-major Q x P: index p*Q + q == m
    Tg[oo] = T;
    rsum += R;
    tsum += T;
    if (!isfinite(R) || !isfinite(T)) bad = true;
  }
  rsum = warp_sum(rsum);
  tsum = warp_sum(tsum);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wid] = rsum;
    red[1][wid] = tsum;
  }
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) {
    double a = 0.0, c = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      a += red[0][k];
      c += red[1][k];
    }
    tot[ob * 2] = a;
    tot[ob * 2 + 1] = c;
    if (ustatus)
      status[ob] = ustatus[b] | (bad ? (uint32_t)ST_NONFINITE : 0u);
    else if (bad)
      atomicOr(status + ob, (unsigned)ST_NONFINITE);
  }
}

// Gap V0 from given Kx, Ky (rcwa.cpp:179-226), 4 diagonals.
__global__ void gap_v0_kernel(int N, const double2* __restrict__ Kx, const double2* __restrict__ Ky,
                              double2* __restrict__ V0) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= N) return;
  const double2 kx = Kx[m], ky = Ky[m];
  const double2 kx2 = cmul_rn(kx, kx), ky2 = cmul_rn(ky, ky);
  const double2 kz0 = cconj(usqrt(csub_rn(csub_rn(cmk(1.0, 0.0), kx2), ky2)));
  const double2 lam0 = cmul_rn(cmk(0.0, 1.0), kz0);
  const double2 kxky = cmul_rn(kx, ky);
  V0[m] = cdiv(kxky, lam0);
  V0[N + m] = cdiv(csub_rn(cmk(1.0, 0.0), kx2), lam0);
  V0[2 * N + m] = cdiv(csub_rn(ky2, cmk(1.0, 0.0)), lam0);
  V0[3 * N + m] = cdiv(cneg(kxky), lam0);
}

__global__ void set_identity_kernel(double2* M, int n, int ld, long long stride, int col0,
                                    double2 diag) {
  const int b = blockIdx.y;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * n) return;
  const int i = (int)(e % n), j = (int)(e / n);
  M[(long long)b * stride + (long long)(col0 + j) * ld + i] = (i == j) ? diag : cmk(0.0, 0.0);
}

__global__ void scale_rows_kernel(double2* M, int n, int ncols, int ld, long long stride,
                                  const double2* d, long long sd) {
  const int b = blockIdx.y;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * ncols) return;
  const int i = (int)(e % n), j = (int)(e / n);
  double2* p = M + (long long)b * stride + (long long)j * ld + i;
  *p = cmul(d[(long long)b * sd + i], *p);
}

__global__ void nonuniform_kernel(const double2* g, size_t count, int* flag) {
  const double2 g0 = g[0];
  bool diff = false;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < count;
       e += (size_t)gridDim.x * blockDim.x) {
    double2 v = g[e];
    if (v.x != g0.x || v.y != g0.y) diff = true;
  }
  if (__syncthreads_or(diff) && threadIdx.x == 0) atomicOr(flag, 1);
}

}  // namespace

// ============================================================================
size_t convmat_scratch_bytes(int nl, int nx, int ny, const ModeDims& d) {
  const size_t nu = 2 * d.P - 1, nv = 2 * d.Q - 1;
  return ((size_t)nx + ny + (size_t)nl * ny * nu + (size_t)nl * nu * nv) * sizeof(double2);
}

int convmat(cudaStream_t s, const double2* grids, int nl, int nx, int ny, const ModeDims& d,
            double2* out, double2* scratch) {
  if (nl <= 0) return RCWA_OK;
  const int nu = 2 * d.P - 1, nv = 2 * d.Q - 1;
  double2* twx = scratch;
  double2* twy = twx + nx;
  double2* Fx = twy + ny;
  double2* Cg = Fx + (size_t)nl * ny * nu;
  twiddle_kernel<<<cdiv_up(nx, 256), 256, 0, s>>>(twx, nx);
  count_launch();
  twiddle_kernel<<<cdiv_up(ny, 256), 256, 0, s>>>(twy, ny);
  count_launch();
  RCWA_LAUNCH_CHECK();
  const size_t shm = (size_t)2 * nx * sizeof(double2);
  if (shm > 48 * 1024) {
    static bool set[64] = {};   // the attribute is per device
    int dev = 0;
    RCWA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !set[dev]) {
      RCWA_CUDA_TRY(cudaFuncSetAttribute(convmat_row_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024));
      if (dev < 64) set[dev] = true;
    }
    if (shm > 200 * 1024) {
      set_last_error("convmat: nx=%d too large", nx);
      return RCWA_ERR_INVALID;
    }
  }
  convmat_row_kernel<<<dim3(ny, nl), 256, shm, s>>>(grids, nx, ny, d.P, twx, Fx);
  count_launch();
  RCWA_LAUNCH_CHECK();
  convmat_col_kernel<<<dim3(cdiv_up((long long)nu * nv, 8), nl), 256, 0, s>>>(Fx, nx, ny, d.P, d.Q, twy, Cg);
  count_launch();
  RCWA_LAUNCH_CHECK();
  const long long NN = (long long)d.N * d.N;
  convmat_gather_kernel<<<dim3(cdiv_up(NN, 256), nl), 256, 0, s>>>(Cg, d.P, d.Q, out);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

static size_t li_axis_bytes(int nl, int na, int nb, int Pa, int Pb) {
  const size_t PP = (size_t)Pa * Pa, lines = (size_t)nl * nb;
  return ((size_t)na + nb + lines * 2 * PP + (size_t)nl * (2 * Pb - 1) * PP) * sizeof(double2) +
         lines * (Pa * sizeof(int) + sizeof(uint32_t)) + 1024;
}

size_t li_convmat_scratch_bytes(int nl, int nx, int ny, const ModeDims& d) {
  const size_t a = li_axis_bytes(nl, nx, ny, d.P, d.Q), b = li_axis_bytes(nl, ny, nx, d.Q, d.P);
  return a > b ? a : b;
}

int li_convmat(cudaStream_t s, const double2* grids, int nl, int nx, int ny, const ModeDims& d,
               int axis_y, double2* out, void* scratch, int* bad) {
  if (nl <= 0) return RCWA_OK;
  const int na = axis_y ? ny : nx, nb = axis_y ? nx : ny;
  const int Pa = axis_y ? d.Q : d.P, Pb = axis_y ? d.P : d.Q;
  const long long sa = axis_y ? nx : 1, sb = axis_y ? 1 : nx, sl = (long long)nx * ny;
  const size_t PP = (size_t)Pa * Pa, lines = (size_t)nl * nb;
  double2* tw_a = (double2*)scratch;
  double2* tw_b = tw_a + na;
  double2* aug = tw_b + nb;
  double2* Cg = aug + lines * 2 * PP;
  int* piv = (int*)(Cg + (size_t)nl * (2 * Pb - 1) * PP);
  uint32_t* st = (uint32_t*)(piv + lines * Pa);
  twiddle_kernel<<<cdiv_up(na, 256), 256, 0, s>>>(tw_a, na);
  count_launch();
  twiddle_kernel<<<cdiv_up(nb, 256), 256, 0, s>>>(tw_b, nb);
  count_launch();
  RCWA_LAUNCH_CHECK();
  const size_t shm = ((size_t)2 * na + 2 * Pa - 1) * sizeof(double2);
  if (shm > 200 * 1024) {
    set_last_error("Li rule: %d grid points along a line is too many", na);
    return RCWA_ERR_INVALID;
  }
  if (shm > 48 * 1024) {
    static bool set[64] = {};   // the attribute is per device
    int dev = 0;
    RCWA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !set[dev]) {
      RCWA_CUDA_TRY(cudaFuncSetAttribute(li_line_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024));
      if (dev < 64) set[dev] = true;
    }
  }
  li_line_kernel<<<dim3(nb, nl), 256, shm, s>>>(grids, na, nb, sa, sb, sl, Pa, tw_a, aug, bad);
  count_launch();
  RCWA_LAUNCH_CHECK();
  RCWA_CUDA_TRY(cudaMemsetAsync(st, 0, lines * sizeof(uint32_t), s));
  int rc = zgesv(s, Pa, Pa, aug, Pa, 2 * (long long)PP, (int)lines, piv, st);
  if (rc) return rc;
  li_any_kernel<<<cdiv_up((long long)lines, 256), 256, 0, s>>>(st, (long long)lines, bad);
  count_launch();
  RCWA_LAUNCH_CHECK();
  const long long warps = (long long)PP * (2 * Pb - 1);
  li_cross_kernel<<<dim3(cdiv_up(warps, 8), nl), 256, 0, s>>>(aug, nb, Pa, Pb, tw_b, Cg);
  count_launch();
  RCWA_LAUNCH_CHECK();
  const long long NN = (long long)d.N * d.N;
  li_gather_kernel<<<dim3(cdiv_up(NN, 256), nl), 256, 0, s>>>(Cg, d.P, d.Q, axis_y, out);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int wave_vectors(cudaStream_t s, const SourceDev* src_dev, int B, const ModeDims& d,
                 double2 er_ref, double2 ur_ref, double2 er_trn, double2 ur_trn,
                 const WaveVecs& w, uint32_t* status) {
  wavevec_kernel<<<B, 256, 0, s>>>(src_dev, d.nxh, d.nyh, d.Q, d.N, er_ref, ur_ref, er_trn,
                                   ur_trn, w, status);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int assemble_pq(cudaStream_t s, int B, const ModeDims& d, const double2* exx, const double2* eyy,
                const double2* mxx, const double2* myy, const double2* einv, const double2* uinv,
                long long s_item, const WaveVecs& w, double2* P, double2* Qm) {
  const long long nn = (long long)d.n * d.n;
  assemble_pq_kernel<<<dim3(cdiv_up(nn, 256), B), 256, 0, s>>>(d.N, exx, eyy, mxx, myy, einv, uinv,
                                                                s_item, w.Kx, w.Ky, P, Qm);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int layer_modes(cudaStream_t s, int B, int n, const double2* lam2, const double2* kinc, double t,
                const double* t_item, int t_stride, double2* lam, double2* ilam, double2* X) {
  layer_modes_kernel<<<dim3(cdiv_up(n, 256), B), 256, 0, s>>>(n, lam2, kinc, t, t_item, t_stride,
                                                               lam, ilam, X);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int assemble_ab(cudaStream_t s, int B, const ModeDims& d, const double2* Wi, long long sWi,
                const double2* Vi, long long sVi, const double2* V0, double2* A, double2* Bm) {
  const long long nn = (long long)d.n * d.n;
  assemble_ab_kernel<<<dim3(cdiv_up(nn, 256), B), 256, 0, s>>>(d.N, Wi, sWi, Vi, sVi, V0, A, Bm);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int uniform_layer(cudaStream_t s, int B, const ModeDims& d, double2 eps, double2 mu, double t,
                  const double2* eps_item, const double2* mu_item, const double* t_item,
                  int stride, const WaveVecs& w, double2* S11, double2* S12, long long sS, int bd) {
  uniform_layer_kernel<<<dim3(cdiv_up(d.N, 128), B), 128, 0, s>>>(d.N, eps, mu, t, eps_item, mu_item,
                                                                   t_item, stride, w, S11, S12, sS, bd);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int port_smatrix(cudaStream_t s, int B, const ModeDims& d, int side, double2 er, double2 ur,
                 const WaveVecs& w, double2* S11, double2* S12, double2* S21, double2* S22,
                 long long sS, int bd) {
  port_smatrix_kernel<<<dim3(cdiv_up(d.N, 128), B), 128, 0, s>>>(d.N, side, er, ur, w, S11, S12,
                                                                  S21, S22, sS, bd);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int efficiencies(cudaStream_t s, int B, const ModeDims& d, const SourceDev* src_dev,
                 double2 ur_ref, double2 ur_trn, const WaveVecs& w, const double2* S11,
                 const double2* S21, long long sS, int compact, double* R, double* T, double* tot,
                 uint32_t* status, const int* map, const int* oidx, const uint32_t* ustatus) {
  if (B <= 0) return RCWA_OK;
  efficiencies_kernel<<<B, 256, 0, s>>>(d.N, src_dev, ur_ref, ur_trn, w, S11, S21, sS, compact, map,
                                         oidx, ustatus, R, T, tot, status);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int bd_apply(cudaStream_t s, int side, int N, int rows, int cols, const double2* X, long long sX,
             const double2* M, int ldm, long long sM, double2* C, int ldc, long long sC,
             double2 alpha, double2 beta, int addI, int batch) {
  const long long ne = (long long)rows * cols;
  bd_apply_kernel<<<dim3(cdiv_up(ne, 256), batch), 256, 0, s>>>(side, N, rows, cols, X, sX, M, ldm, sM,
                                                                 C, ldc, sC, alpha, beta, addI);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int bd_cols(cudaStream_t s, int N, int a, const double2* X, long long sX, double2* C, int ldc,
            long long sC, double2 alpha, double2 beta, int batch) {
  bd_cols_kernel<<<dim3(cdiv_up(4 * N, 256), batch), 256, 0, s>>>(N, a, X, sX, C, ldc, sC, alpha, beta);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int bd_dense(cudaStream_t s, int N, const double2* X, long long sX, double2* C, long long sC,
             int accumulate, int batch) {
  const long long nn = 4LL * N * N;
  bd_dense_kernel<<<dim3(cdiv_up(nn, 256), batch), 256, 0, s>>>(N, X, sX, C, sC, accumulate);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int gap_v0(cudaStream_t s, int N, const double2* Kx, const double2* Ky, double2* V0) {
  gap_v0_kernel<<<cdiv_up(N, 128), 128, 0, s>>>(N, Kx, Ky, V0);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int set_identity(cudaStream_t s, double2* M, int n, int ld, long long stride, int /*ncols_total*/,
                 int col0, int batch, double2 diag) {
  const long long nn = (long long)n * n;
  set_identity_kernel<<<dim3(cdiv_up(nn, 256), batch), 256, 0, s>>>(M, n, ld, stride, col0, diag);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int fill_zero(cudaStream_t s, double2* M, size_t count) {
  RCWA_CUDA_TRY(cudaMemsetAsync(M, 0, count * sizeof(double2), s));
  return RCWA_OK;
}

int scale_rows(cudaStream_t s, double2* M, int n, int ncols, int ld, long long stride,
               const double2* d, long long sd, int batch) {
  const long long ne = (long long)n * ncols;
  scale_rows_kernel<<<dim3(cdiv_up(ne, 256), batch), 256, 0, s>>>(M, n, ncols, ld, stride, d, sd);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

int copy_blocks(cudaStream_t s, double2* dst, long long sdst, const double2* src, long long ssrc,
                size_t count, int batch) {
  RCWA_CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)sdst * sizeof(double2), src,
                                  (size_t)ssrc * sizeof(double2), count * sizeof(double2), batch,
                                  cudaMemcpyDeviceToDevice, s));
  return RCWA_OK;
}

int any_nonuniform(cudaStream_t s, const double2* grid, size_t count, int* flag) {
  nonuniform_kernel<<<256, 256, 0, s>>>(grid, count, flag);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

}  // namespace rcwa
