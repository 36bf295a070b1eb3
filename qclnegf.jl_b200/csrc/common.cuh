// Shared device/host helpers for the B200 SCBA library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/qclb200.h"

namespace qcl {

// ---------------------------------------------------------------------------
// Complex numbers: interleaved (re, im) pairs, identical in memory to Julia's
// ComplexF64 / ComplexF32 and numpy's complex128 / complex64.
// ---------------------------------------------------------------------------
template <typename R> struct Cx;
template <> struct __align__(16) Cx<double> { double x, y; };
template <> struct __align__(8) Cx<float> { float x, y; };

template <typename R> __host__ __device__ __forceinline__ Cx<R> cx(R re, R im) {
  Cx<R> z;
  z.x = re;
  z.y = im;
  return z;
}
template <typename R, typename S> __host__ __device__ __forceinline__ Cx<R> cvt(Cx<S> z) {
  return cx<R>((R)z.x, (R)z.y);
}
template <typename R> __host__ __device__ __forceinline__ Cx<R> operator+(Cx<R> a, Cx<R> b) {
  return cx<R>(a.x + b.x, a.y + b.y);
}
template <typename R> __host__ __device__ __forceinline__ Cx<R> operator-(Cx<R> a, Cx<R> b) {
  return cx<R>(a.x - b.x, a.y - b.y);
}
template <typename R> __host__ __device__ __forceinline__ Cx<R> operator*(Cx<R> a, Cx<R> b) {
  return cx<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename R> __host__ __device__ __forceinline__ Cx<R> operator*(R s, Cx<R> a) {
  return cx<R>(s * a.x, s * a.y);
}
template <typename R> __host__ __device__ __forceinline__ Cx<R> conj(Cx<R> a) { return cx<R>(a.x, -a.y); }
// acc += a * b
template <typename R> __device__ __forceinline__ void cfma(Cx<R>& acc, Cx<R> a, Cx<R> b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc -= a * b
template <typename R> __device__ __forceinline__ void cfms(Cx<R>& acc, Cx<R> a, Cx<R> b) {
  acc.x = fma(-a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(-a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
// acc += a * conj(b)
template <typename R> __device__ __forceinline__ void cfma_conj(Cx<R>& acc, Cx<R> a, Cx<R> b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(-a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// |re| + |im|: the pivot magnitude of LAPACK izamax (dcabs1).
template <typename R> __device__ __forceinline__ R cabs1(Cx<R> a) { return fabs(a.x) + fabs(a.y); }
// 1 / z by Smith's scaled division (robust against over/underflow of |z|^2).
template <typename R> __device__ __forceinline__ Cx<R> crecip(Cx<R> z) {
  if (fabs(z.x) >= fabs(z.y)) {
    R r = z.y / z.x;
    R d = z.x + z.y * r;
    return cx<R>(R(1) / d, -r / d);
  } else {
    R r = z.x / z.y;
    R d = z.x * r + z.y;
    return cx<R>(r / d, R(-1) / d);
  }
}

// 1 / z with one real division: both parts are scaled by a power of two
// (exact) so that |z|^2 can neither overflow nor underflow.
template <typename R> __device__ __forceinline__ Cx<R> crecip_scaled(Cx<R> z) {
  const R mx = fmax(fabs(z.x), fabs(z.y));
  int ex = 0;
  frexp(mx, &ex);
  const R xs = ldexp(z.x, -ex), ys = ldexp(z.y, -ex);
  const R r = R(1) / (xs * xs + ys * ys);
  return cx<R>(ldexp(xs * r, -ex), ldexp(-ys * r, -ex));
}

// 1 / z for the pivots of the elimination.  Both parts are multiplied by the
// power of two 2^(bias - e) built from the exponent field e of max(|re|, |im|)
// (exact), so that d = |z|^2 lies in [1, 8); 1 / d is refined by Newton-Raphson
// (r <- r + r (1 - d r)) from a single-precision seed, two steps for double
// (relative error ~2^-92 before the final rounding).  Valid for finite
// non-zero z; the caller flags zero pivots and never uses their reciprocal.
__device__ __forceinline__ Cx<double> crecip_pivot(Cx<double> z) {
  const double mx = fmax(fabs(z.x), fabs(z.y));
  const int e = min((__double2hiint(mx) >> 20) & 0x7ff, 2045);
  const double sc = __hiloint2double((2046 - e) << 20, 0);
  const double xs = z.x * sc, ys = z.y * sc;
  const double d = fma(xs, xs, ys * ys);
  double r = (double)__frcp_rn((float)d);
  r = fma(r, fma(-d, r, 1.0), r);
  r = fma(r, fma(-d, r, 1.0), r);
  return cx<double>((xs * r) * sc, (-ys * r) * sc);
}
__device__ __forceinline__ Cx<float> crecip_pivot(Cx<float> z) {
  const float mx = fmaxf(fabsf(z.x), fabsf(z.y));
  const int e = min((__float_as_int(mx) >> 23) & 0xff, 253);
  const float sc = __int_as_float((254 - e) << 23);
  const float xs = z.x * sc, ys = z.y * sc;
  const float d = fmaf(xs, xs, ys * ys);
  float r = __frcp_rn(d);
  return cx<float>((xs * r) * sc, (-ys * r) * sc);
}

template <typename R> struct Real;
template <> struct Real<double> { static constexpr int dtype = QCL_C128; };
template <> struct Real<float> { static constexpr int dtype = QCL_C64; };

// ---------------------------------------------------------------------------
// Device status word: [0] = first error code, [1] = linear block index of it.
// Kernels never trap; they record and carry on, the host maps the code to the
// reference's exception.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void record_status(int* status, int code, long long where) {
  if (status == nullptr) return;
  if (atomicCAS(status, 0, code) == 0) status[1] = (int)where;
}

// A QCL_SINGULAR status stores block * kSingularPivotSpan + k, k the index of
// SingularException(k) (0: zero scale; else the 1-based first zero pivot).
constexpr long long kSingularPivotSpan = 64;

// Host-side error plumbing --------------------------------------------------
void set_last_error(const char* fmt, ...);
// Records a QCL_SINGULAR device status word (block * 64 + k) for
// qcl_last_singular_pivot and formats the message; returns QCL_SINGULAR.
int singular_status(const char* what, int where);
int cuda_status(cudaError_t e, const char* where);

#define QCL_CUDA_CHECK(expr)                                   \
  do {                                                         \
    cudaError_t _e = (expr);                                   \
    if (_e != cudaSuccess) return ::qcl::cuda_status(_e, #expr); \
  } while (0)

#define QCL_LAUNCH_CHECK(where)                                  \
  do {                                                           \
    cudaError_t _e = cudaGetLastError();                         \
    if (_e != cudaSuccess) return ::qcl::cuda_status(_e, where); \
  } while (0)

inline size_t field_elems(int NE, int Nk, int Nb) { return (size_t)NE * Nk * Nb * Nb; }

}  // namespace qcl
