// dual.cuh -- forward-mode dual numbers for the pointwise Jacobians of the
// discrete adjoint.  Dual<N> carries a value and N tangents; instantiating the
// pointwise physics (inviscid flux, Rusanov / Roe / Lax-Friedrichs, boundary
// ghost states) with it gives every Jacobian column in one pass, and the
// adjoint contracts those columns with the incoming adjoint (J^T v).
//
// The type lives in its own namespace: the math overloads below are found by
// argument-dependent lookup for Dual arguments only, so unqualified sqrt/fabs
// on doubles inside namespace frg still resolve to CUDA's own functions.
#pragma once
#include <cuda_runtime.h>

namespace frg {
namespace ad {

template <int N>
struct Dual {
  double v;
  double d[N];
  __device__ __forceinline__ Dual() : v(0) {
#pragma unroll
    for (int i = 0; i < N; i++) d[i] = 0;
  }
  __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
    for (int i = 0; i < N; i++) d[i] = 0;
  }
  __device__ __forceinline__ Dual &operator+=(const Dual &b) { return *this = *this + b; }
  __device__ __forceinline__ Dual &operator-=(const Dual &b) { return *this = *this - b; }
  __device__ __forceinline__ Dual &operator*=(const Dual &b) { return *this = *this * b; }

  friend __device__ __forceinline__ Dual operator+(const Dual &a, const Dual &b) {
    Dual r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
  }
  friend __device__ __forceinline__ Dual operator-(const Dual &a, const Dual &b) {
    Dual r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
  }
  friend __device__ __forceinline__ Dual operator-(const Dual &a) {
    Dual r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
  }
  friend __device__ __forceinline__ Dual operator*(const Dual &a, const Dual &b) {
    Dual r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
  }
  friend __device__ __forceinline__ Dual operator/(const Dual &a, const Dual &b) {
    Dual r;
    const double ib = 1.0 / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
  }
  friend __device__ __forceinline__ bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
  friend __device__ __forceinline__ bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
  friend __device__ __forceinline__ bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
  friend __device__ __forceinline__ bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }
};

template <int N>
__device__ __forceinline__ Dual<N> sqrt(const Dual<N> &a) {
  Dual<N> r;
  r.v = ::sqrt(a.v);
  const double h = r.v > 0 ? 0.5 / r.v : 0.0;  // d sqrt(x) = dx / (2 sqrt x)
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = a.d[i] * h;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> fabs(const Dual<N> &a) {
  return a.v < 0 ? -a : a;
}
template <int N>
__device__ __forceinline__ Dual<N> fmax(const Dual<N> &a, const Dual<N> &b) {
  return a.v >= b.v ? a : b;
}
// x^e for a constant exponent: d(x^e) = e x^(e-1) dx
template <int N>
__device__ __forceinline__ Dual<N> pow(const Dual<N> &a, double e) {
  Dual<N> r;
  r.v = ::pow(a.v, e);
  const double g = e * ::pow(a.v, e - 1.0);
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = a.d[i] * g;
  return r;
}

// x^e with a constant exponent given as a dual (its tangents are ignored)
template <int N>
__device__ __forceinline__ Dual<N> pow(const Dual<N> &a, const Dual<N> &e) {
  return pow(a, e.v);
}

}  // namespace ad
}  // namespace frg
