// Device helpers shared by the eigensolver kernels (zeig.cu, zschur.cu).
#pragma once

#include <cfloat>

#include "common.cuh"

namespace rcwa {
namespace eig {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// 2x2 Householder reflector (zlarfg with n = 2): beta (real), tau, v2 with
// (I - tau [1 v2]^T [1 v2]^* )^H [alpha; x] = [beta; 0].
// It sits on the serial critical path of every QR chase step, so the common
// case uses one square root and two divisions: the norm is formed unscaled
// when all components lie in [1e-140, 1e140] (no over- or underflow of the
// squares), v2 = x conj(d) / |d|^2 with d = alpha - beta (|d| >= |beta|).
// Other magnitudes take the scaled path.
__device__ __forceinline__ void larfg2(double2 alpha, double2 x, double& beta, double2& tau,
                                       double2& v2) {
  if (x.x == 0.0 && x.y == 0.0 && alpha.y == 0.0) {
    tau = cmk(0.0, 0.0);
    v2 = cmk(0.0, 0.0);
    beta = alpha.x;
    return;
  }
  const double mx = fmax(fmax(fabs(alpha.x), fabs(alpha.y)), fmax(fabs(x.x), fabs(x.y)));
  double nrm;
  if (mx > 1e-140 && mx < 1e140) {
    nrm = sqrt(fma(alpha.x, alpha.x, fma(alpha.y, alpha.y, fma(x.x, x.x, x.y * x.y))));
  } else {
    const double a = alpha.x / mx, c = alpha.y / mx, e = x.x / mx, f = x.y / mx;
    nrm = mx * sqrt(a * a + c * c + e * e + f * f);
  }
  beta = -copysign(nrm, alpha.x);
  const double rb = 1.0 / beta;
  tau = cmk((beta - alpha.x) * rb, -alpha.y * rb);
  const double2 d = cmk(alpha.x - beta, alpha.y);
  if (mx > 1e-140 && mx < 1e140) {
    const double rd = 1.0 / fma(d.x, d.x, d.y * d.y);
    v2 = cmk((x.x * d.x + x.y * d.y) * rd, (x.y * d.x - x.x * d.y) * rd);
  } else {
    v2 = cmul(x, crcp(d));
  }
}

// Left application of G^H = I - conj(tau) v v^H, v = [1, v2], to (a; q).
__device__ __forceinline__ void refl_left(double2& a, double2& q, double2 tau, double2 v2) {
  const double2 sum = cmulc(tau, cadd(a, cmulc(v2, q)));
  a = csub(a, sum);
  q = csub(q, cmul(sum, v2));
}
// Right application of G = I - tau v v^H to the row pair (a, q).
__device__ __forceinline__ void refl_right(double2& a, double2& q, double2 tau, double2 v2) {
  const double2 sum = cmul(tau, cadd(a, cmul(q, v2)));
  a = csub(a, sum);
  q = csub(q, cmulc(v2, sum));
}

// Deflation test of zlahqr (Ahues & Tisseur) for the subdiagonal entry
// (k, k-1) of a column-major matrix H with leading dimension ld.
__device__ __forceinline__ bool negligible(const double2* H, int ld, int n, int k, double ulp,
                                           double smlnum) {
  const double2 h = H[(long long)(k - 1) * ld + k];
  const double ah = cabs1(h);
  if (ah <= smlnum) return true;
  const double2 hkk = H[(long long)k * ld + k];
  const double2 hk1 = H[(long long)(k - 1) * ld + k - 1];
  double tst = cabs1(hk1) + cabs1(hkk);
  if (tst == 0.0) {
    if (k - 2 >= 0) tst += cabs1(H[(long long)(k - 2) * ld + k - 1]);
    if (k + 1 <= n - 1) tst += cabs1(H[(long long)k * ld + k + 1]);
  }
  if (ah <= ulp * tst) {
    const double2 hup = H[(long long)k * ld + k - 1];
    const double ab = fmax(ah, cabs1(hup)), ba = fmin(ah, cabs1(hup));
    const double2 dd = csub(hk1, hkk);
    const double aa = fmax(cabs1(hkk), cabs1(dd)), bb = fmin(cabs1(hkk), cabs1(dd));
    const double s = aa + ab;
    if (ba * (ab / s) <= fmax(smlnum, ulp * (bb * (aa / s)))) return true;
  }
  return false;
}

// Wilkinson shift of zlahqr from the trailing 2x2 [[h11, h12], [h21, h22]]:
// the eigenvalue of the block closer to h22.
__device__ __forceinline__ double2 wilkinson_shift(double2 h11, double2 h12, double2 h21,
                                                   double2 h22) {
  double2 t = h22;
  const double2 u = cmul(csqrt_principal(h12), csqrt_principal(h21));
  double s = cabs1(u);
  if (s != 0.0) {
    const double2 x = cscale(csub(h11, t), 0.5);
    const double sx = cabs1(x);
    s = fmax(s, sx);
    const double2 xs = cscale(x, 1.0 / s), us = cscale(u, 1.0 / s);
    double2 y = cscale(csqrt_principal(cadd(cmul(xs, xs), cmul(us, us))), s);
    if (sx > 0.0) {
      const double2 xx = cscale(x, 1.0 / sx);
      if (xx.x * y.x + xx.y * y.y < 0.0) y = cneg(y);
    }
    t = csub(t, cmul(u, cdiv(u, cadd(x, y))));
  }
  return t;
}

}  // namespace eig
}  // namespace rcwa
