// Shared device/host helpers: complex arithmetic on double2/float2-like structs, error status.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace bwpm {

// Complex number of real type T (double or float); 16-/8-byte aligned for vector loads.
template <typename T>
struct alignas(2 * sizeof(T)) cx {
  T re, im;
};

using cd = cx<double>;
using cf = cx<float>;

template <typename T>
__host__ __device__ __forceinline__ cx<T> mk(T a, T b) {
  return cx<T>{a, b};
}
template <typename T>
__host__ __device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) {
  return {a.re + b.re, a.im + b.im};
}
template <typename T>
__host__ __device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) {
  return {a.re - b.re, a.im - b.im};
}
template <typename T>
__host__ __device__ __forceinline__ cx<T> operator-(cx<T> a) {
  return {-a.re, -a.im};
}
template <typename T>
__host__ __device__ __forceinline__ cx<T> operator*(cx<T> a, cx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
__host__ __device__ __forceinline__ cx<T> operator*(cx<T> a, T s) {
  return {a.re * s, a.im * s};
}
template <typename T>
__host__ __device__ __forceinline__ cx<T> operator*(T s, cx<T> a) {
  return {a.re * s, a.im * s};
}
template <typename T>
__host__ __device__ __forceinline__ cx<T> operator/(cx<T> a, T s) {
  return {a.re / s, a.im / s};
}
template <typename T>
__host__ __device__ __forceinline__ cx<T> conj(cx<T> a) {
  return {a.re, -a.im};
}
// multiply by +i (dir > 0) or -i (dir < 0)
template <int DIR, typename T>
__host__ __device__ __forceinline__ cx<T> mul_i(cx<T> a) {
  return DIR > 0 ? cx<T>{-a.im, a.re} : cx<T>{a.im, -a.re};
}
template <typename T>
__host__ __device__ __forceinline__ T norm2(cx<T> a) {
  return a.re * a.re + a.im * a.im;
}

// Complex quotient a/b by Smith's method (scaled, no premature overflow).
template <typename T>
__host__ __device__ __forceinline__ cx<T> cdiv(cx<T> a, cx<T> b) {
  if (fabs(b.re) >= fabs(b.im)) {
    const T r = b.im / b.re;
    const T d = b.re + b.im * r;
    return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  }
  const T r = b.re / b.im;
  const T d = b.im + b.re * r;
  return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}

template <typename T>
__host__ __device__ __forceinline__ T cabs(cx<T> a) {
  return hypot(a.re, a.im);
}

// Principal square root (Re ≥ 0), from sqrt(z) = t + i·b/(2t), t = sqrt((|a| + |z|)/2).
__host__ __device__ __forceinline__ cd csqrt(cd z) {
  const double a = z.re, b = z.im;
  if (a == 0.0 && b == 0.0) return {0.0, b};
  const double t = sqrt((fabs(a) + hypot(a, b)) * 0.5);
  if (a >= 0.0) return {t, b / (2.0 * t)};
  return {fabs(b) / (2.0 * t), copysign(t, b)};
}

// exp(z) = e^Re·(cos Im + i sin Im)
__host__ __device__ __forceinline__ cd cexp(cd z) {
  const double m = exp(z.re);
  double s, c;
  sincos(z.im, &s, &c);
  return {m * c, m * s};
}

template <typename To, typename From>
__host__ __device__ __forceinline__ cx<To> cast(cx<From> a) {
  return {static_cast<To>(a.re), static_cast<To>(a.im)};
}

// ---- host-side error status -------------------------------------------------------------------

// Thrown for invalid arguments; maps to status BWPM_EINVAL (ValueError in Python).
struct invalid_argument : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};

// Throws on a failed runtime call. The runtime also keeps a failed call's code as its "last
// error", which the next launch check (cudaGetLastError) would report against an unrelated
// kernel: it is read (and so cleared, unless the context itself is lost) before throwing.
inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
  }
}

inline unsigned ceil_div(std::size_t a, std::size_t b) { return static_cast<unsigned>((a + b - 1) / b); }

}  // namespace bwpm
