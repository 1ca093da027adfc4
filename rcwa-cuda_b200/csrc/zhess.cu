// Blocked Householder reduction to upper Hessenberg form, A = Q H Q^H, and the
// explicit Q, for a batch of packed n x n complex matrices (steps 1-2 of the
// eigensolver that replaces Eigen::ComplexEigenSolver, rcwa.cpp:298).
//
// Compact-WY formulation (Golub & Van Loan 5.1.7, 7.4.3): the reflectors
// G_c = I - tau_c v_c v_c^H of a panel of NB columns form
// Q_p = G_k ... G_{k+NB-1} = I - V T V^H, and with Y = A V T
//     A Q_p = A - Y V^H,        Q_p^H (A Q_p) = (A Q_p) - V T^H V^H (A Q_p).
// Per panel:
//   panel kernel (one CTA per matrix): column by column, applies the panel's
//     earlier reflectors to the next column (right: -Y V^H, left: -V T^H V^H),
//     forms the reflector, and extends Y (rows k+1..n-1) and T.  Its one pass
//     over the trailing matrix per column is the GEMV  A v_c;
//   batched GEMMs: the top rows of Y, the right update of the trailing
//     columns and of the rows above the panel, and the left update of the
//     trailing block -- the trailing matrix is read and written once per
//     panel instead of several times per column.
// Q is accumulated backwards over the panels, Z <- (I - V T V^H) Z, as GEMMs.
// V of every panel is kept densely (zeros above, unit at the subdiagonal) in
// an n x n side buffer; T of every panel in a small side buffer.
#include "common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {

constexpr int NB = 32;      // panel width
constexpr int PNT = 512;    // panel kernel threads

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// One panel: columns k .. k+jb-1.  A: packed matrices; V: n x n dense
// reflectors (column c holds v_c); Y: n x NB; T: NB x NB (of this panel).
__global__ void __launch_bounds__(PNT)
hess_panel_kernel(double2* __restrict__ Ag, int n, int k, int jb, double2* __restrict__ Vg,
                  double2* __restrict__ Yg, double2* __restrict__ Tg, long long sT) {
  extern __shared__ __align__(16) double2 sh[];
  double2* a = sh;          // [n] working column
  double2* v = sh + n;      // [n] current reflector
  __shared__ double2 vc[NB], w[NB], u[NB];
  __shared__ double red[PNT / 32];
  __shared__ double2 s_tau, s_scale;
  __shared__ double s_beta;
  const int b = blockIdx.x;
  const long long nn = (long long)n * n;
  double2* A = Ag + b * nn;
  double2* V = Vg + b * nn;
  double2* Y = Yg + (long long)b * n * NB;
  double2* T = Tg + (long long)b * sT;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int NW = PNT / 32;

  for (int j = 0; j < jb; ++j) {
    const int c = k + j;
    for (int r = k + 1 + tid; r < n; r += PNT) a[r] = A[(long long)c * n + r];
    if (tid < j) vc[tid] = V[(long long)(k + tid) * n + c];   // V[c, j'] (row c of the panel's V)
    __syncthreads();
    if (j > 0) {
      // right: a -= Y_{<j} conj(V[c, 0:j])
      for (int r = k + 1 + tid; r < n; r += PNT) {
        double2 acc = a[r];
        for (int q = 0; q < j; ++q) {
          const double2 y = Y[(long long)q * n + r], vq = cconj(vc[q]);
          acc.x -= y.x * vq.x - y.y * vq.y;
          acc.y -= y.x * vq.y + y.y * vq.x;
        }
        a[r] = acc;
      }
      __syncthreads();
      // left: w = V_{<j}^H a, w <- T^H w, a -= V_{<j} w
      for (int q = wid; q < j; q += NW) {
        const double2* vq = V + (long long)(k + q) * n;
        double sr = 0.0, si = 0.0;
        for (int r = k + 1 + q + lane; r < n; r += 32) {   // v_q is zero above row k+q+1
          const double2 x = vq[r], y = a[r];
          sr += x.x * y.x + x.y * y.y;
          si += x.x * y.y - x.y * y.x;
        }
        sr = wsum(sr);
        si = wsum(si);
        if (lane == 0) u[q] = cmk(sr, si);
      }
      __syncthreads();
      if (tid < j) {   // w[p] = sum_{q <= p} conj(T[q, p]) u[q]
        double2 acc = cmk(0.0, 0.0);
        for (int q = 0; q <= tid; ++q) cfma(acc, cconj(T[(long long)tid * NB + q]), u[q]);
        w[tid] = acc;
      }
      __syncthreads();
      for (int r = k + 1 + tid; r < n; r += PNT) {
        double2 acc = a[r];
        for (int q = 0; q < j; ++q) {
          const double2 x = V[(long long)(k + q) * n + r], y = w[q];
          acc.x -= x.x * y.x - x.y * y.y;
          acc.y -= x.x * y.y + x.y * y.x;
        }
        a[r] = acc;
      }
      __syncthreads();
    }
    // final H entries of column c (rows k+1..c) and the reflector from a[c+1:]
    for (int r = k + 1 + tid; r <= c; r += PNT) A[(long long)c * n + r] = a[r];
    double part = 0.0;
    for (int r = c + 2 + tid; r < n; r += PNT) part += cabs2(a[r]);
    part = wsum(part);
    if (lane == 0) red[wid] = part;
    __syncthreads();
    if (tid == 0) {
      double xn2 = 0.0;
      for (int q = 0; q < NW; ++q) xn2 += red[q];
      const double2 alpha = a[c + 1];
      double2 tau = cmk(0.0, 0.0), scale = cmk(0.0, 0.0);
      double beta = alpha.x;
      if (!(xn2 == 0.0 && alpha.y == 0.0)) {
        const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
        beta = -copysign(nrm, alpha.x);
        tau = cmk((beta - alpha.x) / beta, -alpha.y / beta);
        scale = crcp(cmk(alpha.x - beta, alpha.y));
      }
      s_tau = tau;
      s_scale = scale;
      s_beta = beta;
    }
    __syncthreads();
    const double2 tau = s_tau, scale = s_scale;
    for (int r = tid; r < n; r += PNT) {
      double2 x = cmk(0.0, 0.0);
      if (r == c + 1) x = cmk(1.0, 0.0);
      else if (r > c + 1) x = cmul(a[r], scale);
      v[r] = x;
      V[(long long)c * n + r] = x;
      if (r == c + 1) A[(long long)c * n + r] = cmk(s_beta, 0.0);
      else if (r > c + 1) A[(long long)c * n + r] = cmk(0.0, 0.0);
    }
    __syncthreads();
    // u = V_{<j}^H v  (v is zero above row c+1)
    for (int q = wid; q < j; q += NW) {
      const double2* vq = V + (long long)(k + q) * n;
      double sr = 0.0, si = 0.0;
      for (int r = c + 1 + lane; r < n; r += 32) {
        const double2 x = vq[r], y = v[r];
        sr += x.x * y.x + x.y * y.y;
        si += x.x * y.y - x.y * y.x;
      }
      sr = wsum(sr);
      si = wsum(si);
      if (lane == 0) u[q] = cmk(sr, si);
    }
    // Y[:, j] = tau (A v - Y_{<j} u), rows k+1..n-1; A v over the columns
    // c+1..n-1 of the panel-start matrix (not yet touched in this panel)
    __syncthreads();
    for (int r = k + 1 + tid; r < n; r += PNT) {
      double2 acc = cmk(0.0, 0.0);
      const double2* ar = A + r;
      for (int col = c + 1; col < n; ++col) cfma(acc, ar[(long long)col * n], v[col]);
      for (int q = 0; q < j; ++q) {
        const double2 y = Y[(long long)q * n + r], uq = u[q];
        acc.x -= y.x * uq.x - y.y * uq.y;
        acc.y -= y.x * uq.y + y.y * uq.x;
      }
      Y[(long long)j * n + r] = cmul(tau, acc);
    }
    // T[0:j, j] = -tau T_{<j} u, T[j, j] = tau
    if (tid < j) {
      double2 acc = cmk(0.0, 0.0);
      for (int q = tid; q < j; ++q) cfma(acc, T[(long long)q * NB + tid], u[q]);
      T[(long long)j * NB + tid] = cneg(cmul(tau, acc));
    }
    if (tid == 0) T[(long long)j * NB + j] = tau;
    for (int p = j + 1 + tid; p < NB; p += PNT) T[(long long)j * NB + p] = cmk(0.0, 0.0);
    __syncthreads();
  }
}

__global__ void identity_kernel(double2* Z, int n) {
  const int b = blockIdx.y;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nn = (long long)n * n;
  if (e >= nn) return;
  const int i = (int)(e % n), j = (int)(e / n);
  Z[b * nn + e] = cmk(i == j ? 1.0 : 0.0, 0.0);
}

}  // namespace

size_t hess_ws_bytes(int n, int batch) {
  const size_t npan = (size_t)(n + NB - 1) / NB + 1;
  // Y, Ytmp (n x NB), W, W2 (NB x n), T store (npan x NB x NB)
  return (size_t)batch * ((size_t)4 * n * NB + npan * NB * NB) * sizeof(double2);
}

// Reduces packed A (n x n, batch) to Hessenberg form in place (zero below the
// subdiagonal), writes Z = Q, uses V (n x n per matrix) and ws.
int hess_blocked(cudaStream_t s, int n, int batch, double2* A, double2* Z, double2* V, void* ws) {
  const long long nn = (long long)n * n;
  const size_t npan = (size_t)(n + NB - 1) / NB + 1;
  double2* Y = (double2*)ws;
  double2* Ytmp = Y + (size_t)batch * n * NB;
  double2* W = Ytmp + (size_t)batch * n * NB;
  double2* W2 = W + (size_t)batch * n * NB;
  double2* Tst = W2 + (size_t)batch * n * NB;
  const long long sY = (long long)n * NB, sW = (long long)NB * n, sT = (long long)npan * NB * NB;
  const double2 one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0), zero = cmk(0.0, 0.0);
  const size_t shm = (size_t)2 * n * sizeof(double2);
  if (shm > 48 * 1024) {
    if (shm > 200 * 1024) {
      set_last_error("hess: n=%d too large", n);
      return RCWA_ERR_INVALID;
    }
    // the attribute is per function and device, shared by every thread: set
    // the bound once instead of this call's size (concurrent callers with
    // different n would otherwise undercut each other's launches)
    static bool set[64] = {};
    int dev = 0;
    RCWA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !set[dev]) {
      RCWA_CUDA_TRY(cudaFuncSetAttribute(hess_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024));
      if (dev < 64) set[dev] = true;
    }
  }
  auto gemm = [&](int m, int ncol, int kd, double2 alpha, const double2* X, int ldx, long long sx,
                  int opx, const double2* Yb, int ldy, long long sy, int opy, double2 beta,
                  double2* C, int ldc, long long sc) {
    ZGemm g;
    g.m = m; g.n = ncol; g.k = kd; g.batch = batch;
    g.alpha = alpha; g.beta = beta;
    g.A = X; g.lda = ldx; g.sA = sx; g.opA = opx;
    g.B = Yb; g.ldb = ldy; g.sB = sy; g.opB = opy;
    g.C = C; g.ldc = ldc; g.sC = sc;
    return zgemm(s, g);
  };
  int rc;
  int p = 0;
  for (int k = 0; k < n - 2; k += NB, ++p) {
    const int jb = min(NB, n - 2 - k);
    double2* Tp = Tst + (size_t)p * NB * NB;
    void* tok = prof_begin(s);
    hess_panel_kernel<<<batch, PNT, shm, s>>>(A, n, k, jb, V, Y, Tp, sT);
    prof_end(s, tok, "hess_panel");
    count_launch();
    RCWA_LAUNCH_CHECK();
    const double2* Vp = V + (long long)k * n;   // columns k..k+jb-1 of V
    // Y[0:k+1, :] = A[0:k+1, k+1:n] V[k+1:n, :] T
    if ((rc = gemm(k + 1, jb, n - k - 1, one, A + (long long)(k + 1) * n, n, nn, 0, Vp + k + 1, n, nn, 0,
                   zero, Ytmp, n, sY)))
      return rc;
    if ((rc = gemm(k + 1, jb, jb, one, Ytmp, n, sY, 0, Tp, NB, sT, 0, zero, Y, n, sY))) return rc;
    // right: A[:, k+jb:n] -= Y V[k+jb:n, :]^H ; A[0:k+1, k+1:k+jb] -= Y[0:k+1, :] V[k+1:k+jb, :]^H
    if (k + jb < n) {
      if ((rc = gemm(n, n - k - jb, jb, mone, Y, n, sY, 0, Vp + k + jb, n, nn, 1, one,
                     A + (long long)(k + jb) * n, n, nn)))
        return rc;
    }
    if (jb > 1) {
      if ((rc = gemm(k + 1, jb - 1, jb, mone, Y, n, sY, 0, Vp + k + 1, n, nn, 1, one,
                     A + (long long)(k + 1) * n, n, nn)))
        return rc;
    }
    // left: A[k+1:n, k+jb:n] -= V T^H V^H A[k+1:n, k+jb:n]
    if (k + jb < n) {
      const int nc = n - k - jb;
      if ((rc = gemm(jb, nc, n - k - 1, one, Vp + k + 1, n, nn, 1, A + (long long)(k + jb) * n + k + 1, n,
                     nn, 0, zero, W, NB, sW)))
        return rc;
      if ((rc = gemm(jb, nc, jb, one, Tp, NB, sT, 1, W, NB, sW, 0, zero, W2, NB, sW))) return rc;
      if ((rc = gemm(n - k - 1, nc, jb, mone, Vp + k + 1, n, nn, 0, W2, NB, sW, 0, one,
                     A + (long long)(k + jb) * n + k + 1, n, nn)))
        return rc;
    }
  }
  // Z = Q = Q_0 Q_1 ... accumulated backwards: Z[k+1:, k+1:] <- (I - V T V^H) Z[k+1:, k+1:]
  identity_kernel<<<dim3(cdiv_up(nn, 256), batch), 256, 0, s>>>(Z, n);
  count_launch();
  RCWA_LAUNCH_CHECK();
  for (int q = p - 1; q >= 0; --q) {
    const int k = q * NB;
    const int jb = min(NB, n - 2 - k);
    const double2* Tp = Tst + (size_t)q * NB * NB;
    const double2* Vp = V + (long long)k * n + k + 1;
    double2* Zs = Z + (long long)(k + 1) * n + k + 1;
    const int m = n - k - 1;
    if ((rc = gemm(jb, m, m, one, Vp, n, nn, 1, Zs, n, nn, 0, zero, W, NB, sW))) return rc;
    if ((rc = gemm(jb, m, jb, one, Tp, NB, sT, 0, W, NB, sW, 0, zero, W2, NB, sW))) return rc;
    if ((rc = gemm(m, m, jb, mone, Vp, n, nn, 0, W2, NB, sW, 0, one, Zs, n, nn))) return rc;
  }
  return RCWA_OK;
}

}  // namespace rcwa
