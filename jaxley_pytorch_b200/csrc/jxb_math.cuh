// Scalar helpers shared by the step kernels: float/double overloads and a
// forward-mode dual number used by the adjoint to differentiate rate functions.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace jxb {

// float32 uses the hardware approximations (exp2-based exponential, approximate
// reciprocal and division: a few ulp, well inside the float32 tolerance of the
// simulator); float64 stays correctly rounded.
__device__ __forceinline__ float ex(float x) { return __expf(x); }
__device__ __forceinline__ double ex(double x) { return exp(x); }
// exp(x) - 1 in float32: the Taylor series to degree 7 (Horner form) for |x| < 1/4,
// where it is accurate to 2e-9 relative before rounding, else exp(x) - 1 from the
// hardware exponential (no cancellation for |x| >= 1/4).
__device__ __forceinline__ float exm1(float x) {
  if (fabsf(x) < 0.25f) {
    float p = 1.0f / 5040.0f;
    p = fmaf(p, x, 1.0f / 720.0f);
    p = fmaf(p, x, 1.0f / 120.0f);
    p = fmaf(p, x, 1.0f / 24.0f);
    p = fmaf(p, x, 1.0f / 6.0f);
    p = fmaf(p, x, 0.5f);
    p = fmaf(p, x, 1.0f);
    return p * x;
  }
  return __expf(x) - 1.0f;
}
__device__ __forceinline__ double exm1(double x) { return expm1(x); }
__device__ __forceinline__ float lg(float x) { return logf(x); }
__device__ __forceinline__ double lg(double x) { return log(x); }
__device__ __forceinline__ float pw(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double pw(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float fab(float x) { return fabsf(x); }
__device__ __forceinline__ double fab(double x) { return fabs(x); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float rcp(float b) { return __fdividef(1.0f, b); }
__device__ __forceinline__ double rcp(double b) { return 1.0 / b; }

// (rcp/fdiv for float/double are defined above.)
// Dual number a + b*eps (eps^2 = 0): `d` carries the derivative with respect to
// one seeded input.
template <typename T>
struct Dual {
  T v, d;
  __host__ __device__ __forceinline__ Dual() {}
  __host__ __device__ __forceinline__ Dual(T a) : v(a), d(T(0)) {}
  __host__ __device__ __forceinline__ Dual(T a, T b) : v(a), d(b) {}
  __device__ __forceinline__ Dual& operator+=(Dual b) { v += b.v; d += b.d; return *this; }
  __device__ __forceinline__ Dual& operator-=(Dual b) { v -= b.v; d -= b.d; return *this; }
  __device__ __forceinline__ Dual& operator*=(Dual b) { d = d * b.v + v * b.d; v *= b.v; return *this; }
};
// Comparisons look at the value (a branch of the function, not of its derivative).
template <typename T> __device__ __forceinline__ bool operator<(Dual<T> a, Dual<T> b) { return a.v < b.v; }
template <typename T> __device__ __forceinline__ bool operator>(Dual<T> a, Dual<T> b) { return a.v > b.v; }
template <typename T> __device__ __forceinline__ bool operator!=(Dual<T> a, Dual<T> b) { return a.v != b.v || a.d != b.d; }
__device__ __forceinline__ bool is_finite(float x) { return ::isfinite(x); }
__device__ __forceinline__ bool is_finite(double x) { return ::isfinite(x); }
template <typename T> __device__ __forceinline__ bool is_finite(Dual<T> a) { return is_finite(a.v) && is_finite(a.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator+(Dual<T> a, Dual<T> b) { return Dual<T>(a.v + b.v, a.d + b.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator-(Dual<T> a, Dual<T> b) { return Dual<T>(a.v - b.v, a.d - b.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator-(Dual<T> a) { return Dual<T>(-a.v, -a.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator*(Dual<T> a, Dual<T> b) { return Dual<T>(a.v * b.v, a.d * b.v + a.v * b.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator/(Dual<T> a, Dual<T> b) {
  T ib = rcp(b.v);
  T q = a.v * ib;
  return Dual<T>(q, (a.d - q * b.d) * ib);
}
template <typename T> __device__ __forceinline__ Dual<T> operator+(Dual<T> a, T b) { return Dual<T>(a.v + b, a.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator+(T a, Dual<T> b) { return Dual<T>(a + b.v, b.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator-(Dual<T> a, T b) { return Dual<T>(a.v - b, a.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator-(T a, Dual<T> b) { return Dual<T>(a - b.v, -b.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator*(Dual<T> a, T b) { return Dual<T>(a.v * b, a.d * b); }
template <typename T> __device__ __forceinline__ Dual<T> operator*(T a, Dual<T> b) { return Dual<T>(a * b.v, a * b.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator/(Dual<T> a, T b) { return Dual<T>(a.v / b, a.d / b); }
template <typename T> __device__ __forceinline__ Dual<T> operator/(T a, Dual<T> b) {
  T ib = rcp(b.v);
  T q = a * ib;
  return Dual<T>(q, -q * b.d * ib);
}
template <typename T> __device__ __forceinline__ Dual<T> ex(Dual<T> a) { T e = ex(a.v); return Dual<T>(e, e * a.d); }
template <typename T> __device__ __forceinline__ Dual<T> exm1(Dual<T> a) { return Dual<T>(exm1(a.v), ex(a.v) * a.d); }
template <typename T> __device__ __forceinline__ Dual<T> lg(Dual<T> a) { return Dual<T>(lg(a.v), a.d / a.v); }
template <typename T> __device__ __forceinline__ Dual<T> pw(Dual<T> a, T y) {
  T p = pw(a.v, y);
  return Dual<T>(p, y * pw(a.v, y - T(1)) * a.d);
}
template <typename T> __device__ __forceinline__ Dual<T> fab(Dual<T> a) { return a.v < T(0) ? -a : a; }
template <typename T> __device__ __forceinline__ Dual<T> fdiv(Dual<T> a, Dual<T> b) { return a / b; }
template <typename T> __device__ __forceinline__ Dual<T> rcp(Dual<T> b) { return T(1) / b; }

template <typename T> __device__ __forceinline__ T val(T a) { return a; }
template <typename T> __device__ __forceinline__ T val(Dual<T> a) { return a.v; }

template <typename S> struct Base { typedef S type; };
template <typename T> struct Base<Dual<T>> { typedef T type; };

// `min(x, 20)` keeping NaN (torch.clamp semantics); the derivative is zero on the
// clamped side.
template <typename T> __device__ __forceinline__ T clamp20(T x) { return x > T(20) ? T(20) : x; }
template <typename T> __device__ __forceinline__ Dual<T> clamp20(Dual<T> x) {
  return x.v > T(20) ? Dual<T>(T(20), T(0)) : x;
}

// solver_gate.py:8-11
template <typename S> __device__ __forceinline__ S save_exp(S x) { return ex(clamp20(x)); }

// solver_gate.py:14-30: x / (exp(x/y) - 1), series y*(1 - z/2 + z^2/12) for |z| < 1e-4.
template <typename S, typename T> __device__ __forceinline__ S x_over_expm1(S x, T y) {
  typedef typename Base<S>::type B;
  S z = clamp20(x * (B(1) / B(y)));
  bool small = fab(val(z)) < B(1e-4);
  if (small) return y * (B(1) - z * B(0.5) + z * z * B(1.0 / 12.0));
  return fdiv(x, exm1(z));
}

}  // namespace jxb
