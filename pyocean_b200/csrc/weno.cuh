// WENO5 face reconstruction in FP64 with the reference's arithmetic.
//
// The face value of an upwind-ordered 5-cell stencil v1..v5 (v3 = the upwind cell) follows
// core/dynamics/sigma_baroclinic.py:204-233 (`_wval`): WENO5-Z (Borges et al. 2008, tau5 = |b2 - b0|, eps 1e-40) or
// WENO5-JS (Jiang & Shu 1996, eps 1e-6) when all five cells are valid, WENO3 (eps 1e-6) when v2..v4 are, else the
// upwind value.  Every operation is written in the reference's evaluation order; the translation unit is compiled
// with -fmad=false so no multiply-add is contracted, which makes the result bit-identical to the reference's
// IEEE-754 FP64 evaluation.  Divisions by the constants 6 and 2 give the same correctly rounded quotients as the
// reference's divisions, in fewer instructions (exactdiv.cuh; x * 0.5 is x / 2 exactly).
#pragma once

#include "common.cuh"
#include "exactdiv.cuh"

namespace po {

__device__ __forceinline__ double weno5_value(double v1, double v2, double v3, double v4, double v5,
                                              bool k1, bool k2, bool k3, bool k4, bool k5, bool z_variant)
{
    if (k1 && k2 && k3 && k4 && k5) {
        const double q0 = div6_exact(2.0 * v1 - 7.0 * v2 + 11.0 * v3);
        const double q1 = div6_exact(-v2 + 5.0 * v3 + 2.0 * v4);
        const double q2 = div6_exact(2.0 * v3 + 5.0 * v4 - v5);
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
        const double c0 = (-v2 + 3.0 * v3) * 0.5, c1 = (v3 + v4) * 0.5;
        const double s0 = 1e-6 + (v3 - v2) * (v3 - v2), s1 = 1e-6 + (v4 - v3) * (v4 - v3);
        const double e0 = (1.0 / 3.0) / (s0 * s0);
        const double e1 = (2.0 / 3.0) / (s1 * s1);
        return (e0 * c0 + e1 * c1) / (e0 + e1);
    }
    return v3;
}

// Upwind WENO5 value of the face between cells f-1 and f from the six cells f-3 .. f+2 (w[0..5] with stride
// `step`, validity v[..]).  The upwind ordering is selected per face without branching, so a warp whose faces
// have transports of both signs runs one reconstruction, not two.
__device__ __forceinline__ double upwind_face_value(const double* w, const uint8_t* v, int step, double q, bool z)
{
    const bool pos = q >= 0.0;
    const double w0 = w[0], w1 = w[step], w2 = w[2 * step], w3 = w[3 * step], w4 = w[4 * step], w5 = w[5 * step];
    const bool b0 = v[0], b1 = v[step], b2 = v[2 * step], b3 = v[3 * step], b4 = v[4 * step], b5 = v[5 * step];
    return weno5_value(pos ? w0 : w5, pos ? w1 : w4, pos ? w2 : w3, pos ? w3 : w2, pos ? w4 : w1,
                       pos ? b0 : b5, pos ? b1 : b4, pos ? b2 : b3, pos ? b3 : b2, pos ? b4 : b1, z);
}

}  // namespace po
