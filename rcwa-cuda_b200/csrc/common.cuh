// Shared device helpers for the RCWA kernels: complex128 arithmetic on
// double2, launch checks, status bits.  All matrices are column-major
// complex128 (double2), matching the reference's Eigen default layout
// (rcwa.hpp:13).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/rcwa_b200.h"

namespace rcwa {

// ----------------------------------------------------------------------------
// complex128 helpers
// ----------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return cmk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return cmk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cneg(double2 a) { return cmk(-a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return cmk(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return cmk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return cmk(a.x * s, a.y * s); }
// acc += a*b
__host__ __device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
__host__ __device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }
__device__ __forceinline__ double cabs(double2 a) { return hypot(a.x, a.y); }

// a / b with Smith's scaling (robust complex division).
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  if (fabs(b.y) <= fabs(b.x)) {
    double r = b.y / b.x;
    double d = b.x + b.y * r;
    return cmk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y;
    double d = b.y + b.x * r;
    return cmk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}
__host__ __device__ __forceinline__ double2 crcp(double2 b) { return cdiv(cmk(1.0, 0.0), b); }

// Principal complex square root (branch cut on the negative real axis,
// Im(result) carries the sign of Im(z)), written from the half-angle
// identities: for z = x + iy, t = sqrt((|x| + |z|)/2); if x >= 0 the root is
// t + i y/(2t), else |y|/(2t) + i sign(y) t.  |z| uses hypot to avoid
// overflow.  This matches std::sqrt(std::complex) including the sign of a
// zero imaginary part.
__device__ __forceinline__ double2 csqrt_principal(double2 z) {
  double x = z.x, y = z.y;
  if (x == 0.0 && y == 0.0) return cmk(0.0, y);
  double t = sqrt(0.5 * (fabs(x) + hypot(x, y)));
  if (x >= 0.0) return cmk(t, y / (2.0 * t));
  return cmk(fabs(y) / (2.0 * t), copysign(t, y));
}
// unsigned_sqrt (rcwa.hpp:24-28): an imaginary -0 is turned into +0 first.
__device__ __forceinline__ double2 usqrt(double2 z) {
  if (z.y == 0.0) z.y = 0.0;  // -0.0 == 0.0 -> store +0
  return csqrt_principal(z);
}
__device__ __forceinline__ double2 cexp(double2 z) {
  double e = exp(z.x);
  double s, c;
  sincos(z.y, &s, &c);
  return cmk(e * c, e * s);
}
__device__ __forceinline__ bool cfinite(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// complex64 (float2) counterparts used by the FP32 factorisation of the
// mixed-precision LU (zlu.cu)
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float cabs1(float2 a) { return fabsf(a.x) + fabsf(a.y); }
__host__ __device__ __forceinline__ float2 cdiv(float2 a, float2 b) {
  if (fabsf(b.y) <= fabsf(b.x)) {
    float r = b.y / b.x;
    float d = b.x + b.y * r;
    return make_float2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    float r = b.x / b.y;
    float d = b.y + b.x * r;
    return make_float2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}
__host__ __device__ __forceinline__ float2 crcp(float2 b) { return cdiv(make_float2(1.0f, 0.0f), b); }

// ----------------------------------------------------------------------------
// host-side checking
// ----------------------------------------------------------------------------
#define RCWA_CUDA_TRY(expr)                                                        \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      rcwa::set_last_error("%s:%d %s: %s", __FILE__, __LINE__, #expr,              \
                           cudaGetErrorString(_e));                                \
      return RCWA_ERR_CUDA;                                                        \
    }                                                                              \
  } while (0)

#define RCWA_LAUNCH_CHECK()                                                        \
  do {                                                                             \
    cudaError_t _e = cudaGetLastError();                                           \
    if (_e != cudaSuccess) {                                                       \
      rcwa::set_last_error("%s:%d launch: %s", __FILE__, __LINE__,                 \
                           cudaGetErrorString(_e));                                \
      return RCWA_ERR_CUDA;                                                        \
    }                                                                              \
  } while (0)

void set_last_error(const char* fmt, ...);

// Per-matrix status bits written by kernels (OR-ed into a uint32 per problem).
enum : uint32_t {
  ST_SINGULAR = RCWA_STATUS_SINGULAR,
  ST_EIG_NOCONV = RCWA_STATUS_EIG_NOCONV,
  ST_NONFINITE = RCWA_STATUS_NONFINITE,
  ST_WOOD = RCWA_STATUS_WOOD_ANOMALY,
};

inline unsigned cdiv_up(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace rcwa
