// Column remap arithmetic of core/vertical/remap.py, written once for the device kernels (and compiled for the
// host only by the CPU self-test of tests/hostcore/).
//
// Two column algorithms share the per-cell formulas:
//   remap_column_stream  one pass over the source cells with a 6-cell register window: the reconstruction of cell i
//                        (PLM slopes, PPM_H4 edge values, bounding, discontinuity check, CW84 limiter) is built
//                        from its neighbours as the window slides, then cell i is integrated over the targets it
//                        overlaps (two passes over those targets: the first finds the thickest piece, the second
//                        accumulates the others and gives the thickest the residual, remap.py:359-366).  No column
//                        array is stored; finished targets are written as the sweep passes them.
//   remap_column_general the reference's array formulation (column arrays in thread-local memory), used for the
//                        columns the sweep cannot take in one pass: a target thickness that is negative or NaN.
// Both evaluate every expression in the reference's order; compiled without FMA contraction they give the
// reference's numbers bit for bit.
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define PO_HD __host__ __device__ __forceinline__
#define PO_HDT __host__ __device__
#else
#define PO_HD inline
#define PO_HDT
#endif

namespace po {
namespace rc {

enum { PCM = 0, PLM = 1, PPM_H4 = 2 };
constexpr double H_NEGLECT = 1e-30;        // remap.py:42
constexpr double H_NEGLECT_EDGE = 1e-10;   // remap.py:43
constexpr double H_MIN_FRAC = 1e-5;        // remap.py:100
constexpr double EPS = 2.220446049250313e-16;

PO_HD double pmax(double a, double b) { return (b > a) ? b : a; }
PO_HD double pmin(double a, double b) { return (b < a) ? b : a; }

PO_HD int effective_scheme(int n_active, int scheme)          // remap.py:46-53
{
    if (n_active <= 1) return PCM;
    if (n_active <= 3 && scheme > PLM) return PLM;
    return scheme;
}

PO_HD double plm_slope(double h_l, double h_c, double h_r, double u_l, double u_c, double u_r)   // remap.py:59-80
{
    const double sigma_r = u_r - u_c;
    const double sigma_l = u_c - u_l;
    const double sigma_c = 2.0 * (u_r - u_l) * (h_c / (h_l + 2.0 * h_c + h_r + H_NEGLECT));
    const double u_min = pmin(pmin(u_l, u_c), u_r);
    const double u_max = pmax(pmax(u_l, u_c), u_r);
    double slope = 0.0;
    if (sigma_l * sigma_r > 0.0) {
        const double m = pmin(fabs(sigma_c), 2.0 * pmin(u_c - u_min, u_max - u_c));
        slope = sigma_c >= 0.0 ? m : -m;
    }
    if (u_c - 0.5 * fabs(slope) < u_min || u_c + 0.5 * fabs(slope) > u_max) slope = slope * (1.0 - EPS);
    if (fabs(slope) < 1e-140) slope = 0.0;
    return slope;
}

PO_HD double plm_monotonized(double u_l, double u_c, double u_r, double s_l, double s_c, double s_r)   // :83-97
{
    const double almost_two = 2.0 * (1.0 - EPS);
    const double e_r = u_l + 0.5 * s_l;
    const double e_l = u_r - 0.5 * s_r;
    double slp = fabs(s_c);
    double edge = u_c - 0.5 * s_c;
    if ((edge - e_r) * (u_c - edge) < 0.0) {
        edge = 0.5 * (edge + e_r);
        slp = pmin(slp, fabs(edge - u_c) * almost_two);
    }
    edge = u_c + 0.5 * s_c;
    if ((edge - u_c) * (e_l - edge) < 0.0) {
        edge = 0.5 * (edge + e_l);
        slp = pmin(slp, fabs(edge - u_c) * almost_two);
    }
    return s_c >= 0.0 ? slp : -slp;
}

// PLM coefficients of cell k from its slope data (remap.py:271-282): c0 = u_l, c1 = u_r - u_l (times 1 - eps when
// the right edge is not monotone with the next cell's left edge).
PO_HD void plm_coef(double u_c, double u_next, double mslp, double mslp_next, double slp_next, double& c0,
                    double& c1)
{
    const double u_l = u_c - 0.5 * mslp;
    const double u_r = u_c + 0.5 * mslp;
    c0 = u_l;
    c1 = u_r - u_l;
    const double edge = c1 + c0;
    const double am = fabs(mslp_next);
    const double e_r = u_next - 0.5 * (slp_next >= 0.0 ? am : -am);
    if ((edge - u_c) * (e_r - edge) < 0.0) c1 = c1 * (1.0 - EPS);
}

// (C(0), C(dz1)) of the cubic whose means over the 4 end cells are u1..u4, thicknesses h1..h4 from the end
// (remap.py:103-156; the caller applies max(h_neglect_edge, h)).
PO_HD void end_values(double h1, double h2, double h3, double h4, double u1, double u2, double u3, double u4,
                      double& e_end, double& e_in)
{
    const double min_frac = 1.0e-6;
    const double d0 = h1;
    if ((h2 + h3) < min_frac * h1) h3 = min_frac * h1 - h2;
    if ((h3 + h4) < min_frac * h1) h4 = min_frac * h1 - h3;
    const double h12 = h1 + h2, h23 = h2 + h3, h34 = h3 + h4;
    const double h123 = h12 + h3, h234 = h2 + h34, h1234 = h12 + h34;
    const double I_denB3 = 1.0 / (h123 * h12 * h23);
    const double I_h12 = (h123 * h23) * I_denB3;
    const double I_h23 = (h12 * h123) * I_denB3;
    const double I_h123 = (h12 * h23) * I_denB3;
    const double I_denom = 1.0 / (h1234 * (h234 * h34));
    const double I_h234 = (h1234 * h34) * I_denom;
    const double I_h1234 = (h234 * h34) * I_denom;
    const double w11 = -h1 * (I_h1234 + I_h123 + I_h12);
    const double w21 = h1 * h12 * (I_h234 * I_h1234 + I_h23 * (I_h234 + I_h123));
    const double w31 = -h1 * h12 * h123 * I_denom;
    const double w12 = 2.0 * (I_h12 * (1.0 + (h1 + h12) * (I_h1234 + I_h123)) + h1 * I_h1234 * I_h123);
    const double w22 = -2.0 * ((h1 * h12 * I_h1234) * (I_h23 * (I_h234 + I_h123)) +
                               (h1 + h12) * (I_h1234 * I_h234 + I_h23 * (I_h234 + I_h123)));
    const double w32 = 2.0 * ((h1 + h12) * h123 + h1 * h12) * I_denom;
    const double w13 = -3.0 * I_h12 * I_h123 * (1.0 + I_h1234 * ((h1 + h12) + h123));
    const double w23 = 3.0 * I_h23 * (I_h123 + I_h1234 * ((h1 + h12) + h123) * (I_h123 + I_h234));
    const double w33 = -3.0 * ((h1 + h12) + h123) * I_denom;
    const double w14 = 4.0 * I_h1234 * I_h123 * I_h12;
    const double w24 = -4.0 * I_h1234 * (I_h23 * (I_h123 + I_h234));
    const double w34 = 4.0 * I_denom;
    const double d1 = u2 - u1, d2 = u3 - u2, d3 = u4 - u3;
    const double c0 = ((u1 + (w11 * d1)) + (w21 * d2)) + (w31 * d3);
    const double c1 = ((w12 * d1) + (w22 * d2)) + (w32 * d3);
    const double c2 = ((w13 * d1) + (w23 * d2)) + (w33 * d3);
    const double c3 = ((w14 * d1) + (w24 * d2)) + (w34 * d3);
    e_end = c0;
    e_in = c0 + d0 * (c1 + d0 * (c2 + d0 * c3));
}

// Thickness factors of the explicit 4th-order edge value between cells i-1 and i (stencil h0..h3 = cells
// i-2..i+1), remap.py:167-181: the edge is (w1 u1 + w2 u2 + g2 (u1 - u0) + g3 (u2 - u3)) / den, split so that the
// thickness-only part is shared by every field of the column.
struct H4Weights {
    double w1, w2, g2, g3, den;
};

PO_HD H4Weights h4_weights(double h0, double h1, double h2, double h3)
{
    if (h0 + h1 == 0.0 || h1 + h2 == 0.0 || h2 + h3 == 0.0) {
        const double h_min = H_MIN_FRAC * pmax(H_NEGLECT_EDGE, (h0 + h1) + (h2 + h3));
        h0 = pmax(h_min, h0);
        h1 = pmax(h_min, h1);
        h2 = pmax(h_min, h2);
        h3 = pmax(h_min, h3);
    }
    const double I_h12 = 1.0 / (h1 + h2);
    const double I_den_et2 = 1.0 / (((h0 + h1) + h2) * (h0 + h1));
    const double I_h012 = (h0 + h1) * I_den_et2;
    const double I_den_et3 = 1.0 / ((h1 + (h2 + h3)) * (h2 + h3));
    const double I_h123 = (h2 + h3) * I_den_et3;
    H4Weights w;
    w.w1 = (1.0 + (h1 * I_h012 + (h0 + h1) * I_h123)) * I_h12 * (h2 * (h2 + h3));
    w.w2 = (1.0 + (h2 * I_h123 + (h2 + h3) * I_h012)) * I_h12 * (h1 * (h0 + h1));
    w.g2 = h1 * (h2 * (h2 + h3)) * I_den_et2;
    w.g3 = h2 * (h1 * (h0 + h1)) * I_den_et3;
    w.den = (h0 + h1) + (h2 + h3);
    return w;
}

PO_HD double h4_edge(const H4Weights& w, double u0, double u1, double u2, double u3)
{
    const double et1 = w.w1 * u1 + w.w2 * u2;
    const double et2 = w.g2 * (u1 - u0);
    const double et3 = w.g3 * (u2 - u3);
    return (et1 + (et2 + et3)) / w.den;
}

// Limited slope of bound_edges for cell k with neighbours km1 / kp1 (remap.py:203-213).
PO_HD double bound_slope(double h_m, double h_c, double h_p, double u_m, double u_c, double u_p)
{
    double slope_x_h = 0.0;
    if ((h_m + h_p) + 2.0 * h_c > 0.0) {
        const double sl = u_c - u_m;
        const double sc = (u_p - u_m) * (h_c / ((h_m + h_p) + 2.0 * h_c));
        const double sr = u_p - u_c;
        if (sl * sr > 0.0) {
            const double m = pmin(pmin(fabs(sl), fabs(sc)), fabs(sr));
            slope_x_h = sc >= 0.0 ? m : -m;
        }
    }
    return slope_x_h;
}

// The left (sign = -1) or right (+1) edge of a cell after bound_edges (remap.py:214-220): u_n is the neighbour on
// that side (u_km1 for the left edge, u_kp1 for the right one).
PO_HD double bound_edge(double e, double u_n, double u_c, double slope_x_h, double side)
{
    const double sgn = slope_x_h >= 0.0 ? 1.0 : -1.0;
    if ((u_n - e) * (e - u_c) < 0.0) e = u_c + side * sgn * pmin(fabs(slope_x_h), fabs(e - u_c));
    return pmax(pmin(e, pmax(u_n, u_c)), pmin(u_n, u_c));
}

// check_discontinuous at the interface between cells k and k+1 (remap.py:223-231): (right of k, left of k+1).
PO_HD void check_pair(double& er_k, double& el_k1, double u_k, double u_k1)
{
    if ((el_k1 - er_k) * (u_k1 - u_k) < 0.0) {
        double a = 0.5 * (er_k + el_k1);
        a = pmax(pmin(a, pmax(u_k, u_k1)), pmin(u_k, u_k1));
        er_k = a;
        el_k1 = a;
    }
}

// Colella & Woodward limiter and PPM coefficients of an interior cell (remap.py:265-294).
PO_HD void ppm_coef(double u_l, double u_c, double u_r, double el, double er, double& c0, double& c1, double& c2)
{
    if ((u_r - u_c) * (u_c - u_l) <= 0.0) {
        el = u_c;
        er = u_c;
    } else {
        const double expr1 = 3.0 * (er - el) * ((u_c - el) + (u_c - er));
        const double expr2 = (er - el) * (er - el);
        if (expr1 > expr2) {
            el = u_c + 2.0 * (u_c - er);
            el = pmax(pmin(el, pmax(u_l, u_c)), pmin(u_l, u_c));
        } else if (expr1 < -expr2) {
            er = u_c + 2.0 * (u_c - el);
            er = pmax(pmin(er, pmax(u_r, u_c)), pmin(u_r, u_c));
        }
    }
    if (fabs(er - el) < pmax(1e-60, EPS * fabs(u_c))) {
        el = u_c;
        er = u_c;
    }
    c0 = el;
    c1 = 4.0 * (u_c - el) + 2.0 * (u_c - er);
    c2 = 3.0 * ((er - u_c) + (el - u_c));
}

PO_HD double average(double c0, double c1, double c2, double xa, double xb)      // remap.py:297-303
{
    if (xb - xa <= 1e-14) {
        const double x = 0.5 * (xa + xb);
        return c0 + x * (c1 + x * c2);
    }
    return c0 + 0.5 * c1 * (xa + xb) + c2 * (xa * xa + xa * xb + xb * xb) / 3.0;
}

// ------------------------------------------------------------------------------------------------------------
// One-pass column remap.  IO: hs(k), ht(k), f(m, k) loads and put(m, k, v) stores; NF fields share the
// thickness work.  Preconditions: the column is wet, has at least one active source cell, and every target
// thickness is >= 0 (the caller routes other columns to remap_column_general).
template <int NF, class IO>
PO_HDT void remap_column_stream(IO& io, int n0, int n1, int scheme, int n_active, int last)
{
    const int sch = effective_scheme(n_active, scheme);
    const bool plm = sch == PLM && n0 >= 3;
    const bool ppm = sch == PPM_H4 && n0 >= 4;

    // window: slot s holds cell i - 2 + s (s = 0..5) of the current step i
    double wh[6];
    double wu[NF][6];
    for (int s = 0; s < 6; ++s) {
        const int k = s - 2;
        const bool in = k >= 0 && k < n0;
        wh[s] = in ? io.hs(k) : 0.0;
        for (int m = 0; m < NF; ++m) wu[m][s] = in ? io.f(m, k) : 0.0;
    }
    // PLM state: raw slope of cells i-1, i, i+1 and monotonized slope of cells i, i+1 (zeros at the ends)
    double slp_m1[NF], slp_0[NF], slp_p1[NF], mslp_0[NF], mslp_p1[NF];
    // PPM state: bounded/checked left edge of cell i, bound slopes of cells i and i+1, raw edge of interface i+1
    double el_i[NF], sl_i[NF], top_in[NF], top_out[NF];
    for (int m = 0; m < NF; ++m) {
        slp_m1[m] = slp_0[m] = slp_p1[m] = mslp_0[m] = mslp_p1[m] = 0.0;
        el_i[m] = sl_i[m] = top_in[m] = top_out[m] = 0.0;
    }
    if (plm) {
        // slopes of cells 0 (zero), 1; monotonized slope of cell 0 is zero
        for (int m = 0; m < NF; ++m) {
            slp_0[m] = 0.0;
            slp_p1[m] = n0 - 1 > 1 ? plm_slope(wh[2], wh[3], wh[4], wu[m][2], wu[m][3], wu[m][4]) : 0.0;
            mslp_0[m] = 0.0;
        }
    }
    if (ppm) {
        // end values: bottom from cells 0..3, top from cells n0-1..n0-4 (thicknesses floored at h_neglect_edge)
        double hb[4], ht4[4];
        for (int q = 0; q < 4; ++q) {
            hb[q] = pmax(H_NEGLECT_EDGE, io.hs(q));
            ht4[q] = pmax(H_NEGLECT_EDGE, io.hs(n0 - 1 - q));
        }
        for (int m = 0; m < NF; ++m) {
            double e00, e01;
            end_values(hb[0], hb[1], hb[2], hb[3], io.f(m, 0), io.f(m, 1), io.f(m, 2), io.f(m, 3), e00, e01);
            end_values(ht4[0], ht4[1], ht4[2], ht4[3], io.f(m, n0 - 1), io.f(m, n0 - 2), io.f(m, n0 - 3),
                       io.f(m, n0 - 4), top_out[m], top_in[m]);
            // cell 0: km1 = 0, kp1 = 1
            const double s0 = bound_slope(wh[2], wh[2], wh[3], wu[m][2], wu[m][2], wu[m][3]);
            sl_i[m] = s0;
            el_i[m] = bound_edge(e00, wu[m][2], wu[m][2], s0, -1.0);
            // raw edge of interface 1 kept in slp_p1 (reused as the PPM "next raw edge")
            slp_p1[m] = e01;
        }
    }

    // target sweep state
    int j = 0;
    double t_lo = 0.0, t_hi = io.ht(0);   // t_edge[j], t_edge[j+1]
    double acc[NF];
    for (int m = 0; m < NF; ++m) acc[m] = 0.0;
    bool last_target_reached = n1 == 1;   // target n1-1 reached (its vanished value then comes from that cell)
    double last_target_val[NF];
    bool last_val_set = false;
    double a = 0.0;

    for (int i = 0; i < n0; ++i) {
        // ---- coefficients of cell i (window slots: 1 = i-1, 2 = i, 3 = i+1, 4 = i+2, 5 = i+3)
        double c0[NF], c1[NF], c2[NF];
        for (int m = 0; m < NF; ++m) { c0[m] = wu[m][2]; c1[m] = 0.0; c2[m] = 0.0; }
        if (plm) {
            for (int m = 0; m < NF; ++m) {
                // slope of cell i+2 and monotonized slope of cell i+1
                const double slp_p2 = (i + 2 <= n0 - 2) ? plm_slope(wh[3], wh[4], wh[5], wu[m][3], wu[m][4], wu[m][5])
                                                         : 0.0;
                mslp_p1[m] = (i + 1 >= 1 && i + 1 <= n0 - 2)
                                 ? plm_monotonized(wu[m][2], wu[m][3], wu[m][4], slp_0[m], slp_p1[m], slp_p2)
                                 : 0.0;
                if (i >= 1 && i <= n0 - 2)
                    plm_coef(wu[m][2], wu[m][3], mslp_0[m], mslp_p1[m], slp_p1[m], c0[m], c1[m]);
                slp_m1[m] = slp_0[m];
                slp_0[m] = slp_p1[m];
                slp_p1[m] = slp_p2;
                mslp_0[m] = mslp_p1[m];
            }
        } else if (ppm) {
            // raw edge of interface i+2 (stencil cells i..i+3): interior H4, or the top end values
            H4Weights w{};
            const bool interior = i + 2 >= 2 && i + 2 <= n0 - 2;
            if (interior) w = h4_weights(wh[2], wh[3], wh[4], wh[5]);
            for (int m = 0; m < NF; ++m) {
                // raw edges: interface i (left of i) is already in el_i (bounded), interface i+1 raw in slp_p1
                const double e_ip1 = slp_p1[m];
                double e_ip2 = 0.0;
                if (i + 2 <= n0) {
                    if (interior) e_ip2 = h4_edge(w, wu[m][2], wu[m][3], wu[m][4], wu[m][5]);
                    else if (i + 2 == n0 - 1) e_ip2 = top_in[m];
                    else e_ip2 = top_out[m];
                }
                // bound slope of cell i+1 (km1 = i, kp1 = min(i+2, n0-1))
                double sl_ip1 = 0.0;
                if (i + 1 <= n0 - 1) {
                    const int sp = i + 2 <= n0 - 1 ? 4 : 3;
                    sl_ip1 = bound_slope(wh[2], wh[3], wh[sp], wu[m][2], wu[m][3], wu[m][sp]);
                }
                // right edge of cell i (kp1 = min(i+1, n0-1)) and left edge of cell i+1 (km1 = i), then the check
                const int rp = i + 1 <= n0 - 1 ? 3 : 2;
                double er = bound_edge(e_ip1, wu[m][rp], wu[m][2], sl_i[m], 1.0);
                double el_next = 0.0;
                if (i + 1 <= n0 - 1) {
                    el_next = bound_edge(e_ip1, wu[m][2], wu[m][3], sl_ip1, -1.0);
                    check_pair(er, el_next, wu[m][2], wu[m][3]);
                }
                if (i >= 1 && i <= n0 - 2) ppm_coef(wu[m][1], wu[m][2], wu[m][3], el_i[m], er, c0[m], c1[m], c2[m]);
                el_i[m] = el_next;
                sl_i[m] = sl_ip1;
                slp_p1[m] = e_ip2;
            }
        }

        // ---- integrate cell i over the targets it overlaps (remap.py:331-367)
        const double hi = wh[2];
        if (hi > 0.0) {
            const double b = a + hi;
            // pass 1: targets touched, thickest piece (first maximum)
            int jj = j;
            double tl = t_lo, th = t_hi, thick = -1.0;
            int jthick = -1;
            while (true) {
                const double lo = pmax(a, tl);
                const double hi_t = jj < n1 - 1 ? th : pmax(th, b);
                const double up = pmin(b, hi_t);
                const double L = up - lo;
                if (L > 0.0 && L > thick) { thick = L; jthick = jj; }
                if (hi_t <= b && jj < n1 - 1) {
                    ++jj;
                    tl = th;
                    th = th + io.ht(jj);
                } else {
                    break;
                }
            }
            const int j_end = jj;
            // pass 2: pieces, the residual of the thickest, finished targets written as they are passed
            double s[NF], base_thick[NF];
            for (int m = 0; m < NF; ++m) { s[m] = 0.0; base_thick[m] = 0.0; }
            jj = j;
            tl = t_lo;
            th = t_hi;
            double h_jj = th - tl;   // placeholder; the target thickness is reloaded below
            (void)h_jj;
            while (true) {
                const double lo = pmax(a, tl);
                const double hi_t = jj < n1 - 1 ? th : pmax(th, b);
                const double up = pmin(b, hi_t);
                const double L = up - lo;
                double content[NF];
                for (int m = 0; m < NF; ++m) content[m] = jj == j ? acc[m] : 0.0;
                if (L > 0.0) {
                    const double xa = (lo - a) / hi, xb = (up - a) / hi;
                    if (jj == jthick) {
                        for (int m = 0; m < NF; ++m) base_thick[m] = content[m];
                    } else {
                        for (int m = 0; m < NF; ++m) {
                            const double piece = L * average(c0[m], c1[m], c2[m], xa, xb);
                            s[m] += piece;
                            content[m] += piece;
                        }
                    }
                }
                if (jj < j_end) {
                    if (jj != jthick) {
                        const double hgt = io.ht(jj);
                        for (int m = 0; m < NF; ++m) {
                            double val;
                            if (hgt > 0.0) {
                                val = content[m] / hgt;
                            } else {           // vanished target: value of this cell's polynomial at its position
                                const double xi = (tl - a) / hi;
                                val = c0[m] + xi * (c1[m] + xi * c2[m]);
                            }
                            io.put(m, jj, val);
                        }
                    }
                    ++jj;
                    tl = th;
                    th = th + io.ht(jj);
                } else {
                    if (jj != jthick)
                        for (int m = 0; m < NF; ++m) acc[m] = content[m];
                    break;
                }
            }
            if (jthick >= 0) {
                for (int m = 0; m < NF; ++m) {
                    const double piece = wu[m][2] * hi - s[m];
                    const double cth = base_thick[m] + piece;
                    if (jthick < j_end) {
                        const double hgt = io.ht(jthick);
                        io.put(m, jthick, hgt > 0.0 ? cth / hgt : cth);   // hgt > 0: a piece needs a thickness
                    } else {
                        acc[m] = cth;
                    }
                }
            }
            // the last target, reached for the first time in this cell, takes this cell's polynomial if vanished
            if (!last_target_reached && j_end == n1 - 1) last_target_reached = true;
            if (last_target_reached && !last_val_set) {
                // x = t_edge[n1-1] = tl at the end of pass 2 when j_end == n1-1
                const double xi = (tl - a) / hi;
                for (int m = 0; m < NF; ++m) last_target_val[m] = c0[m] + xi * (c1[m] + xi * c2[m]);
                last_val_set = true;
            }
            j = j_end;
            t_lo = tl;
            t_hi = th;
            a = b;
        }
        // ---- slide the window by one cell
        for (int s = 0; s < 5; ++s) {
            wh[s] = wh[s + 1];
            for (int m = 0; m < NF; ++m) wu[m][s] = wu[m][s + 1];
        }
        const int knew = i + 4;
        const bool in = knew < n0;
        wh[5] = in ? io.hs(knew) : 0.0;
        for (int m = 0; m < NF; ++m) wu[m][5] = in ? io.f(m, knew) : 0.0;
    }

    // targets from the current one to the top: the current one holds its accumulated content; the ones above it
    // were never reached (content 0, or the last source value when vanished)
    for (int jj = j; jj < n1; ++jj) {
        const double hgt = io.ht(jj);
        for (int m = 0; m < NF; ++m) {
            double val;
            if (hgt > 0.0) {
                val = (jj == j ? acc[m] : 0.0) / hgt;
            } else if (jj == n1 - 1 && last_val_set) {
                val = last_target_val[m];
            } else {
                val = io.f(m, last);
            }
            io.put(m, jj, val);
        }
    }
}

}  // namespace rc
}  // namespace po
