// WENO5 face reconstruction in FP64 with the reference's arithmetic.
//
// The face value of an upwind-ordered 5-cell stencil v1..v5 (v3 = the upwind cell) follows
// core/dynamics/sigma_baroclinic.py:204-233 (`_wval`): WENO5-Z (Borges et al. 2008, tau5 = |b2 - b0|, eps 1e-40) or
// WENO5-JS (Jiang & Shu 1996, eps 1e-6) when all five cells are valid, WENO3 (eps 1e-6) when v2..v4 are, else the
// upwind value.  Every operation is written in the reference's evaluation order; the translation unit is compiled
// with -fmad=false so no multiply-add is contracted, which makes the result bit-identical to the reference's
// IEEE-754 FP64 evaluation (correctly rounded division included).
#pragma once

#include "common.cuh"

namespace po {

__device__ __forceinline__ double weno5_value(double v1, double v2, double v3, double v4, double v5,
                                              bool k1, bool k2, bool k3, bool k4, bool k5, bool z_variant)
{
    if (k1 && k2 && k3 && k4 && k5) {
        const double q0 = (2.0 * v1 - 7.0 * v2 + 11.0 * v3) / 6.0;
        const double q1 = (-v2 + 5.0 * v3 + 2.0 * v4) / 6.0;
        const double q2 = (2.0 * v3 + 5.0 * v4 - v5) / 6.0;
        const double c1312 = 13.0 / 12.0;
        double d = v1 - 2.0 * v2 + v3, e = v1 - 4.0 * v2 + 3.0 * v3;
        const double b0 = c1312 * (d * d) + 0.25 * (e * e);
        d = v2 - 2.0 * v3 + v4;
        e = v2 - v4;
        const double b1 = c1312 * (d * d) + 0.25 * (e * e);
        d = v3 - 2.0 * v4 + v5;
        e = 3.0 * v3 - 4.0 * v4 + v5;
        const double b2 = c1312 * (d * d) + 0.25 * (e * e);
        double a0, a1, a2;
        if (z_variant) {
            const double tau = fabs(b2 - b0);
            a0 = 0.1 * (1.0 + tau / (1e-40 + b0));
            a1 = 0.6 * (1.0 + tau / (1e-40 + b1));
            a2 = 0.3 * (1.0 + tau / (1e-40 + b2));
        } else {
            const double s0 = 1e-6 + b0, s1 = 1e-6 + b1, s2 = 1e-6 + b2;
            a0 = 0.1 / (s0 * s0);
            a1 = 0.6 / (s1 * s1);
            a2 = 0.3 / (s2 * s2);
        }
        return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
    }
    if (k2 && k3 && k4) {
        const double c0 = (-v2 + 3.0 * v3) / 2.0, c1 = (v3 + v4) / 2.0;
        const double s0 = 1e-6 + (v3 - v2) * (v3 - v2), s1 = 1e-6 + (v4 - v3) * (v4 - v3);
        const double e0 = (1.0 / 3.0) / (s0 * s0);
        const double e1 = (2.0 / 3.0) / (s1 * s1);
        return (e0 * c0 + e1 * c1) / (e0 + e1);
    }
    return v3;
}

}  // namespace po
