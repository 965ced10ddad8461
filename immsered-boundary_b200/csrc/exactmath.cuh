// Powers the reference takes through libm pow(): x^3 (Sutherland viscosity,
// NS_Solver.cpp:564) and x^3.5 (pressure inlet, BCValues.H:199).  Both are
// evaluated with error-free transformations (Dekker/Knuth two-product via
// fma, a residual-corrected square root) and rounded once, which gives the
// correctly rounded value except for operands that fall within ~2^-100 of a
// rounding tie; a correctly rounded libm pow agrees with it.
#pragma once

#include <cuda_runtime.h>

namespace ibgpu {

// x^3 as hi + lo (|lo| <= ulp(hi)/2 of the exact value's remainder)
__device__ __forceinline__ void cube_dd(double x, double &hi, double &lo) {
  double a = x * x;
  double b = fma(x, x, -a);  // x^2 = a + b exactly
  double c = a * x;
  double d = fma(a, x, -c);  // a*x = c + d exactly
  double t = fma(b, x, d);   // d + b*x (b*x is far below ulp(c))
  hi = c + t;
  lo = t - (hi - c);
}

__device__ __forceinline__ double cube_rn(double x) {
  double hi, lo;
  cube_dd(x, hi, lo);
  return hi + lo;
}

__device__ __forceinline__ double pow3p5_rn(double x) {
  double ch, cl;
  cube_dd(x, ch, cl);
  double s = sqrt(x);
  double sl = fma(-s, s, x) / (2.0 * s);  // sqrt(x) = s + sl to ~2^-106
  double p = ch * s;
  double pl = fma(ch, s, -p);             // ch*s = p + pl exactly
  pl = pl + (ch * sl + cl * s);
  return p + pl;
}

}  // namespace ibgpu
