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

// ---------------------------------------------------------------------------------------------------------------
// Mixed-precision WENO5 face value: the smoothness indicators, the nonlinear weights and the weighted candidate
// run in FP32 on the differences of the stencil from the upwind cell (formed in FP64, then rounded), normalised by
// their largest magnitude s; the result is added back to the FP64 upwind value: face = v3 + s * w(d/s).  Every
// quantity of the scheme is a function of these differences (q_r - v3 and beta_r are linear / quadratic forms in
// them), so the FP32 rounding acts on the local variation only (relative face error ~1e-7 of s, not of v3).  The
// normalisation keeps beta_r in [0, 40] so FP32 cannot overflow; WENO5-Z's epsilon, 1e-40 in FP64, becomes 1e-30 on
// the normalised scale (both are negligible against any non-zero beta_r, and both give the same limit when a
// beta_r vanishes).  Stencils whose variation is outside what the FP32 forms represent safely (s below 1e-30 or,
// for the absolute-epsilon forms WENO5-JS and WENO3, above 1e8) keep the FP64 arithmetic of weno5_value.

__device__ __forceinline__ double weno5_value_mixed(double v1, double v2, double v3, double v4, double v5,
                                                    bool k1, bool k2, bool k3, bool k4, bool k5, bool z_variant)
{
    if (k1 && k2 && k3 && k4 && k5) {
        const float e1 = (float)(v1 - v3), e2 = (float)(v2 - v3), e4 = (float)(v4 - v3), e5 = (float)(v5 - v3);
        const float sc = fmaxf(fmaxf(fabsf(e1), fabsf(e2)), fmaxf(fabsf(e4), fabsf(e5)));
        if (sc == 0.f) {
            if (v1 == v3 && v2 == v3 && v4 == v3 && v5 == v3) return v3;      // flat: every candidate is v3
            return weno5_value(v1, v2, v3, v4, v5, k1, k2, k3, k4, k5, z_variant);
        }
        if (!(sc > 1e-30f) || (!z_variant && sc > 1e8f))
            return weno5_value(v1, v2, v3, v4, v5, k1, k2, k3, k4, k5, z_variant);
        const float inv = 1.f / sc;
        const float d1 = e1 * inv, d2 = e2 * inv, d4 = e4 * inv, d5 = e5 * inv;
        const float c1312 = 13.f / 12.f;
        float t = fmaf(-2.f, d2, d1), u = fmaf(-4.f, d2, d1);
        const float b0 = fmaf(c1312 * t, t, 0.25f * u * u);
        t = d2 + d4;
        u = d2 - d4;
        const float b1 = fmaf(c1312 * t, t, 0.25f * u * u);
        t = fmaf(-2.f, d4, d5);
        u = fmaf(-4.f, d4, d5);
        const float b2 = fmaf(c1312 * t, t, 0.25f * u * u);
        const float tau = fabsf(b2 - b0);
        float a0, a1, a2;
        if (z_variant) {
            a0 = 0.1f * (1.f + __fdividef(tau, 1e-30f + b0));
            a1 = 0.6f * (1.f + __fdividef(tau, 1e-30f + b1));
            a2 = 0.3f * (1.f + __fdividef(tau, 1e-30f + b2));
        } else {
            // JS weights use an absolute epsilon (1e-6): un-normalise beta (s <= 1e8 keeps the squares finite)
            const float s2 = sc * sc;
            const float g0 = fmaf(s2, b0, 1e-6f), g1 = fmaf(s2, b1, 1e-6f), g2 = fmaf(s2, b2, 1e-6f);
            a0 = __fdividef(0.1f, g0 * g0);
            a1 = __fdividef(0.6f, g1 * g1);
            a2 = __fdividef(0.3f, g2 * g2);
        }
        // 6 (q_r - v3) / s
        const float p0 = fmaf(2.f, d1, -7.f * d2), p1 = fmaf(2.f, d4, -d2), p2 = fmaf(5.f, d4, -d5);
        const float num = fmaf(a0, p0, fmaf(a1, p1, a2 * p2));
        const float den = 6.f * (a0 + a1 + a2);
        return v3 + (double)(sc * __fdividef(num, den));
    }
    if (k2 && k3 && k4) {
        // WENO3 (absolute eps 1e-6): candidates v3 - e2/2 and v3 + e4/2
        const float d2 = (float)(v2 - v3), d4 = (float)(v4 - v3);
        if (!(fmaxf(fabsf(d2), fabsf(d4)) <= 1e8f)) return weno5_value(v1, v2, v3, v4, v5, k1, k2, k3, k4, k5, z_variant);
        const float g0 = fmaf(d2, d2, 1e-6f), g1 = fmaf(d4, d4, 1e-6f);
        const float w0 = __fdividef(1.f / 3.f, g0 * g0), w1 = __fdividef(2.f / 3.f, g1 * g1);
        const float corr = __fdividef(fmaf(w1, 0.5f * d4, -w0 * 0.5f * d2), w0 + w1);
        return v3 + (double)corr;
    }
    return v3;
}

template <bool MIX>
__device__ __forceinline__ double weno5_face(double v1, double v2, double v3, double v4, double v5, bool k1, bool k2,
                                             bool k3, bool k4, bool k5, bool z)
{
    if (MIX) return weno5_value_mixed(v1, v2, v3, v4, v5, k1, k2, k3, k4, k5, z);
    return weno5_value(v1, v2, v3, v4, v5, k1, k2, k3, k4, k5, z);
}

}  // namespace po
