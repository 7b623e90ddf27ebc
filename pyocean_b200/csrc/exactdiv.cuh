// Correctly rounded division of binary64 values by the constants 3 and 6 in four FP64 operations.
//
// The reference divides by 6 three times per WENO face ((2v1 - 7v2 + 11v3)/6 ...) and by 3 in the RK3 flux
// combination.  An IEEE division is an iterative sequence of ~10 FP64 instructions; for these constant divisors
// the same correctly rounded result comes from one multiplication and two FMAs:
//
//   y  = RN(1/3)                      (a compile-time constant)
//   q  = RN(x * y)                    |q - x/3| <= ulp(x/3): x*y = (x/3)(1 + d), |d| = 2^-54, plus one rounding
//   r  = fma(-q, 3, x)                exact: x and 3q are multiples of ulp(x/3)/2 and |x - 3q| <= 3 ulp(x/3)
//   q' = RN(q + r * y) = RN(x/3)      the FMA's argument is x/3 + (x/3 - q) d, within 2^-54 ulp of x/3, while
//                                     x/3 is at least ulp/6 away from every rounding midpoint (x - 3m is an odd
//                                     multiple of ulp/2 for any midpoint m), so both round to the same double.
//
// This is Markstein's correction step for division with a correctly rounded reciprocal (P. Markstein, "IA-64 and
// Elementary Functions", 2000, ch. 8) specialised to the divisor 3.  x/6 is (x/2)/3 with x/2 exact.  Arguments
// outside [2^-899, 2^899] in magnitude (zero, subnormal range, near overflow, inf, NaN) take the IEEE division,
// so the result equals `x / 3.0` / `x / 6.0` for every input.  tests/hostcore checks the identity on the host.
#pragma once

#ifdef __CUDACC__
#define PO_XD __host__ __device__ __forceinline__
#else
#include <math.h>
#define PO_XD inline
#endif

namespace po {

PO_XD double div3_exact(double x)
{
    const double y = 1.0 / 3.0;
    const double ax = fabs(x);
    if (!(ax >= 0x1p-899 && ax <= 0x1p899)) return x / 3.0;
    const double q = x * y;
    const double r = fma(-q, 3.0, x);
    return fma(r, y, q);
}

PO_XD double div6_exact(double x)
{
    const double y = 1.0 / 3.0;
    const double ax = fabs(x);
    if (!(ax >= 0x1p-898 && ax <= 0x1p899)) return x / 6.0;
    const double h = x * 0.5;
    const double q = h * y;
    const double r = fma(-q, 3.0, h);
    return fma(r, y, q);
}

}  // namespace po
