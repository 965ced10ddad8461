// Reciprocal, quotient and square-root helpers for the fast kernel builds.
//
// FP64: start from the PTX approximations rcp.approx.ftz.f64 /
// rsqrt.approx.ftz.f64 and refine with Newton-Raphson iterations
//   reciprocal:   y <- y + y (1 - x y)
//   inverse root: y <- y + y (1 - x y^2) / 2
// followed, for quotients and roots, by one residual correction
//   q <- q + r (a - b q),   s <- s + (y/2) (x - s^2)
// (the classical Newton/Markstein refinements).  Results are within a couple
// of units in the last place of the correctly rounded value for the normal,
// positive operands the flux uses (densities, sound speeds, 1 + r); they are
// not IEEE-exact, which is why the exact build does not use them.
// Measured on B200 over [0.25, 16) against IEEE division and square root:
// the approximations alone 9.9e-7 (rcp) and 9.2e-7 (rsqrt) relative, after
// one Newton step (rcp1, rsqrt1) 9.8e-13 and 1.3e-12, after two (rcp, rsqrt)
// 0 and 2.7e-16.  One step is used only where the result scales a
// dissipation term or a limited slope; anything that reaches a central flux
// or the primitive recovery takes two.
// FP32 (mixed precision): the PTX single-precision approximations directly.
#pragma once

#include <cuda_runtime.h>

namespace ibgpu {

template <typename R>
struct FastMath;

template <>
struct FastMath<double> {
  static __device__ __forceinline__ double rcp(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    return y;
  }
  static __device__ __forceinline__ double rcp1(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return fma(y, fma(-x, y, 1.0), y);
  }
  static __device__ __forceinline__ double rsqrt1(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return fma(y, fma(-0.5 * x * y, y, 0.5), y);
  }
  static __device__ __forceinline__ double div(double a, double b) {
    double r = rcp(b);
    double q = a * r;
    return fma(fma(-b, q, a), r, q);
  }
  static __device__ __forceinline__ double rsqrt(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double h = 0.5 * x;
    y = fma(y, fma(-h * y, y, 0.5), y);
    y = fma(y, fma(-h * y, y, 0.5), y);
    return y;
  }
  static __device__ __forceinline__ double sqrt(double x) {
    double y = rsqrt(x);
    double s = x * y;
    return fma(0.5 * y, fma(-s, s, x), s);
  }
};

template <>
struct FastMath<float> {
  static __device__ __forceinline__ float rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
  }
  static __device__ __forceinline__ float rcp1(float x) { return rcp(x); }
  static __device__ __forceinline__ float div(float a, float b) { return a * rcp(b); }
  static __device__ __forceinline__ float rsqrt(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
  }
  static __device__ __forceinline__ float rsqrt1(float x) { return rsqrt(x); }
  static __device__ __forceinline__ float sqrt(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
  }
};

}  // namespace ibgpu
