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
// The sweep needs non-negative target thicknesses (a vanished target then sits in the cell that passes it); the
// kernel sends a column with a negative or NaN target thickness to the reference's array formulation instead.
// Every expression is evaluated in the reference's order; compiled without FMA contraction the results are the
// reference's numbers bit for bit.
#pragma once

#include <math.h>
#include <stdint.h>

#include "exactdiv.cuh"

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

// Thickness factor h_c / (h_l + 2 h_c + h_r + h_neglect) of the PLM slope, shared by every field of a column.
PO_HD double plm_ratio(double h_l, double h_c, double h_r) { return h_c / (h_l + 2.0 * h_c + h_r + H_NEGLECT); }

// The PLM steps are written with selects instead of branches, as the PPM_H4 limiter steps below are (same values).
PO_HD double plm_slope(double ratio, double u_l, double u_c, double u_r)   // remap.py:59-80
{
    const double sigma_r = u_r - u_c;
    const double sigma_l = u_c - u_l;
    const double sigma_c = 2.0 * (u_r - u_l) * ratio;
    const double u_min = pmin(pmin(u_l, u_c), u_r);
    const double u_max = pmax(pmax(u_l, u_c), u_r);
    const double m = pmin(fabs(sigma_c), 2.0 * pmin(u_c - u_min, u_max - u_c));
    double slope = sigma_l * sigma_r > 0.0 ? (sigma_c >= 0.0 ? m : -m) : 0.0;
    const bool shrink = (u_c - 0.5 * fabs(slope) < u_min) | (u_c + 0.5 * fabs(slope) > u_max);
    slope = shrink ? slope * (1.0 - EPS) : slope;
    return fabs(slope) < 1e-140 ? 0.0 : slope;
}

PO_HD double plm_monotonized(double u_l, double u_c, double u_r, double s_l, double s_c, double s_r)   // :83-97
{
    const double almost_two = 2.0 * (1.0 - EPS);
    const double e_r = u_l + 0.5 * s_l;
    const double e_l = u_r - 0.5 * s_r;
    double slp = fabs(s_c);
    const double edge_l = u_c - 0.5 * s_c;
    const double mid_l = 0.5 * (edge_l + e_r);
    const double slp_l = pmin(slp, fabs(mid_l - u_c) * almost_two);
    slp = (edge_l - e_r) * (u_c - edge_l) < 0.0 ? slp_l : slp;
    const double edge_r = u_c + 0.5 * s_c;
    const double mid_r = 0.5 * (edge_r + e_l);
    const double slp_r = pmin(slp, fabs(mid_r - u_c) * almost_two);
    slp = (edge_r - u_c) * (e_l - edge_r) < 0.0 ? slp_r : slp;
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
    c1 = (edge - u_c) * (e_r - edge) < 0.0 ? c1 * (1.0 - EPS) : c1;
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

// The limiter steps below (bound_slope, bound_edge, check_pair, ppm_coef) are written without branches: each
// candidate value is formed and the reference's condition selects it, so the columns of a warp, which take
// different limiter branches where the fields are rough, stay in step.  The selected values are the reference's
// bit for bit; at 512 x 512 x 50 the T/S remap of fields advected for 20 to 100 steps takes 4-5 % less time.
//
// Thickness part of bound_edges' slope for cell k with neighbours km1 / kp1 (remap.py:205-207): whether the slope
// is formed at all, and h_k / ((h_km1 + h_kp1) + 2 h_k); shared by every field of a column.
struct BoundRatio {
    bool active;
    double ratio;
};

PO_HD BoundRatio bound_ratio(double h_m, double h_c, double h_p)
{
    BoundRatio b;
    b.active = (h_m + h_p) + 2.0 * h_c > 0.0;
    b.ratio = b.active ? h_c / ((h_m + h_p) + 2.0 * h_c) : 0.0;
    return b;
}

// Limited slope of bound_edges for cell k (remap.py:203-213).
PO_HD double bound_slope(const BoundRatio& br, double u_m, double u_c, double u_p)
{
    const double sl = u_c - u_m;
    const double sc = (u_p - u_m) * br.ratio;
    const double sr = u_p - u_c;
    const double m = pmin(pmin(fabs(sl), fabs(sc)), fabs(sr));
    const double v = sc >= 0.0 ? m : -m;
    return (br.active && sl * sr > 0.0) ? v : 0.0;
}

// The left (sign = -1) or right (+1) edge of a cell after bound_edges (remap.py:214-220): u_n is the neighbour on
// that side (u_km1 for the left edge, u_kp1 for the right one).
PO_HD double bound_edge(double e, double u_n, double u_c, double slope_x_h, double side)
{
    const double sgn = slope_x_h >= 0.0 ? 1.0 : -1.0;
    const double e2 = u_c + side * sgn * pmin(fabs(slope_x_h), fabs(e - u_c));
    e = (u_n - e) * (e - u_c) < 0.0 ? e2 : e;
    return pmax(pmin(e, pmax(u_n, u_c)), pmin(u_n, u_c));
}

// check_discontinuous at the interface between cells k and k+1 (remap.py:223-231): (right of k, left of k+1).
PO_HD void check_pair(double& er_k, double& el_k1, double u_k, double u_k1)
{
    double a = 0.5 * (er_k + el_k1);
    a = pmax(pmin(a, pmax(u_k, u_k1)), pmin(u_k, u_k1));
    const bool jump = (el_k1 - er_k) * (u_k1 - u_k) < 0.0;
    er_k = jump ? a : er_k;
    el_k1 = jump ? a : el_k1;
}

// Colella & Woodward limiter and PPM coefficients of an interior cell (remap.py:265-294), without branches: both
// candidate edges are formed and selected by the reference's conditions.
PO_HD void ppm_coef(double u_l, double u_c, double u_r, double el, double er, double& c0, double& c1, double& c2)
{
    const bool flat = (u_r - u_c) * (u_c - u_l) <= 0.0;
    const double expr1 = 3.0 * (er - el) * ((u_c - el) + (u_c - er));
    const double expr2 = (er - el) * (er - el);
    double el2 = u_c + 2.0 * (u_c - er);
    el2 = pmax(pmin(el2, pmax(u_l, u_c)), pmin(u_l, u_c));
    double er2 = u_c + 2.0 * (u_c - el);
    er2 = pmax(pmin(er2, pmax(u_r, u_c)), pmin(u_r, u_c));
    const bool left = expr1 > expr2;
    const bool right = !left && expr1 < -expr2;
    el = flat ? u_c : (left ? el2 : el);
    er = flat ? u_c : (right ? er2 : er);
    const bool collapse = fabs(er - el) < pmax(1e-60, EPS * fabs(u_c));
    el = collapse ? u_c : el;
    er = collapse ? u_c : er;
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
    return c0 + 0.5 * c1 * (xa + xb) + div3_exact(c2 * (xa * xa + xa * xb + xb * xb));
}

// ------------------------------------------------------------------------------------------------------------
// One-pass column remap.  IO: hs(k), ht(k), f(m, k) loads and put(m, k, v) stores; NF fields share the
// thickness work.  Preconditions: the column is wet, has n_active >= 1 source cells with h > 0 (the last one is
// `last`), and every target thickness is >= 0 (the caller sends other columns to the general algorithm).
//
// Window: slot s holds source cell i - 2 + s (s = 0..5) while cell i is processed; out-of-range slots hold 0 and
// are never read by the formulas (each use is guarded by its cell range).
template <int NF, class IO>
PO_HDT void remap_column_stream(IO& io, int n0, int n1, int scheme, int n_active, int last)
{
    const int sch = effective_scheme(n_active, scheme);
    const bool plm = sch == PLM && n0 >= 3;
    const bool ppm = sch == PPM_H4 && n0 >= 4;

    double wh[6];
    double wu[NF][6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const int k = s - 2;
        const bool in = k >= 0 && k < n0;
        wh[s] = in ? io.hs(k) : 0.0;
#pragma unroll
        for (int m = 0; m < NF; ++m) wu[m][s] = in ? io.f(m, k) : 0.0;
    }
    // PLM: raw slopes of cells i, i+1 and the monotonized slope of cell i (remap.py:248-262; zero at both ends).
    // PPM: checked left edge of cell i, bound slope of cell i, raw edge of interface i+1, and the top end values.
    double st_a[NF], st_b[NF], st_c[NF], top_in[NF], top_out[NF];
#pragma unroll
    for (int m = 0; m < NF; ++m) st_a[m] = st_b[m] = st_c[m] = top_in[m] = top_out[m] = 0.0;
    BoundRatio br_i{false, 0.0};
    if (plm) {
        const double r1 = plm_ratio(wh[2], wh[3], wh[4]);          // slope of cell 1 (cells 0, 1, 2)
#pragma unroll
        for (int m = 0; m < NF; ++m) {
            st_a[m] = 0.0;                                           // slp[0]
            st_b[m] = plm_slope(r1, wu[m][2], wu[m][3], wu[m][4]);   // slp[1] (n0 >= 3)
            st_c[m] = 0.0;                                           // mslp[0]
        }
    }
    if (ppm) {
        double hb[4], ht4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            hb[q] = pmax(H_NEGLECT_EDGE, io.hs(q));
            ht4[q] = pmax(H_NEGLECT_EDGE, io.hs(n0 - 1 - q));
        }
        br_i = bound_ratio(wh[2], wh[2], wh[3]);                      // cell 0: km1 = 0, kp1 = 1
#pragma unroll
        for (int m = 0; m < NF; ++m) {
            double e00, e01;
            end_values(hb[0], hb[1], hb[2], hb[3], io.f(m, 0), io.f(m, 1), io.f(m, 2), io.f(m, 3), e00, e01);
            end_values(ht4[0], ht4[1], ht4[2], ht4[3], io.f(m, n0 - 1), io.f(m, n0 - 2), io.f(m, n0 - 3),
                       io.f(m, n0 - 4), top_out[m], top_in[m]);
            const double s0 = bound_slope(br_i, wu[m][2], wu[m][2], wu[m][3]);
            st_b[m] = s0;                                                     // bound slope of cell 0
            st_a[m] = bound_edge(e00, wu[m][2], wu[m][2], s0, -1.0);          // left edge of cell 0 (interface 0)
            st_c[m] = e01;                                                    // raw edge of interface 1
        }
    }

    // target sweep state: current target j with edges t_lo = t_edge[j], t_hi = t_edge[j+1]; acc = its content
    int j = 0;
    double t_lo = 0.0, t_hi = 0.0 + io.ht(0);
    double acc[NF], last_val[NF];
#pragma unroll
    for (int m = 0; m < NF; ++m) acc[m] = last_val[m] = 0.0;
    bool last_reached = n1 == 1;      // target n1-1 reached: a vanished last target takes that cell's polynomial
    bool last_set = false;
    double a = 0.0;

    for (int i = 0; i < n0; ++i) {
        // ---- polynomial of cell i (slots: 1 = i-1, 2 = i, 3 = i+1, 4 = i+2, 5 = i+3)
        double c0[NF], c1[NF], c2[NF];
#pragma unroll
        for (int m = 0; m < NF; ++m) { c0[m] = wu[m][2]; c1[m] = 0.0; c2[m] = 0.0; }
        if (plm) {
            const bool have_p2 = i + 2 <= n0 - 2;                        // slope of cell i+2 is formed
            const double r2 = have_p2 ? plm_ratio(wh[3], wh[4], wh[5]) : 0.0;
            const bool have_m1 = i + 1 >= 1 && i + 1 <= n0 - 2;          // monotonized slope of cell i+1
#pragma unroll
            for (int m = 0; m < NF; ++m) {
                const double slp_p2 = have_p2 ? plm_slope(r2, wu[m][3], wu[m][4], wu[m][5]) : 0.0;
                const double mslp_p1 = have_m1 ? plm_monotonized(wu[m][2], wu[m][3], wu[m][4], st_a[m], st_b[m],
                                                                 slp_p2)
                                               : 0.0;
                if (i >= 1 && i <= n0 - 2) plm_coef(wu[m][2], wu[m][3], st_c[m], mslp_p1, st_b[m], c0[m], c1[m]);
                st_a[m] = st_b[m];
                st_b[m] = slp_p2;
                st_c[m] = mslp_p1;
            }
        } else if (ppm) {
            const bool interior = i + 2 <= n0 - 2;                        // interface i+2 from cells i..i+3
            const H4Weights w = interior ? h4_weights(wh[2], wh[3], wh[4], wh[5]) : H4Weights{0, 0, 0, 0, 1};
            const bool has_next = i + 1 <= n0 - 1;                        // cell i+1 exists
            const bool next_has_p = i + 2 <= n0 - 1;                      // cell i+1 has a cell above it
            const BoundRatio br_n = has_next ? bound_ratio(wh[2], wh[3], next_has_p ? wh[4] : wh[3])
                                             : BoundRatio{false, 0.0};
#pragma unroll
            for (int m = 0; m < NF; ++m) {
                const double e_ip1 = st_c[m];
                double e_ip2 = 0.0;
                if (interior) e_ip2 = h4_edge(w, wu[m][2], wu[m][3], wu[m][4], wu[m][5]);
                else if (i + 2 == n0 - 1) e_ip2 = top_in[m];
                else if (i + 2 == n0) e_ip2 = top_out[m];
                const double u_n = next_has_p ? wu[m][4] : wu[m][3];
                const double sl_n = has_next ? bound_slope(br_n, wu[m][2], wu[m][3], u_n) : 0.0;
                const double u_r = has_next ? wu[m][3] : wu[m][2];        // kp1 of cell i
                double er = bound_edge(e_ip1, u_r, wu[m][2], st_b[m], 1.0);
                double el_next = 0.0;
                if (has_next) {
                    el_next = bound_edge(e_ip1, wu[m][2], wu[m][3], sl_n, -1.0);
                    check_pair(er, el_next, wu[m][2], wu[m][3]);
                }
                if (i >= 1 && i <= n0 - 2) ppm_coef(wu[m][1], wu[m][2], wu[m][3], st_a[m], er, c0[m], c1[m], c2[m]);
                st_a[m] = el_next;
                st_b[m] = sl_n;
                st_c[m] = e_ip2;
            }
        }

        // ---- integrate cell i over the targets it overlaps (remap.py:331-367)
        const double hi = wh[2];
        if (hi > 0.0) {
            const double b = a + hi;
            // pass 1: which targets the cell reaches, and the first thickest piece.  The edges here are sums of
            // non-negative thicknesses from +0 (never NaN: such columns go to the general algorithm, such source
            // cells are skipped; never -0), so the native fmax / fmin give pmax / pmin's values bit for bit.
            int jj = j, jthick = -1;
            double tl = t_lo, th = t_hi, thick = -1.0;
            while (true) {
                const double lo = fmax(a, tl);
                const double hi_t = jj < n1 - 1 ? th : fmax(th, b);
                const double L = fmin(b, hi_t) - lo;
                if (L > 0.0 && L > thick) {
                    thick = L;
                    jthick = jj;
                }
                if (hi_t <= b && jj < n1 - 1) {
                    ++jj;
                    tl = th;
                    th = th + io.ht(jj);
                } else {
                    break;
                }
            }
            const int j_end = jj;
            // pass 2: pieces in target order; every piece but the thickest is summed, the thickest gets the
            // residual u h - sum (Hallberg); targets the sweep leaves behind are final and written
            double s[NF], base_thick[NF];
#pragma unroll
            for (int m = 0; m < NF; ++m) s[m] = base_thick[m] = 0.0;
            jj = j;
            tl = t_lo;
            th = t_hi;
            while (true) {
                const double lo = fmax(a, tl);
                const double hi_t = jj < n1 - 1 ? th : fmax(th, b);
                const double up = fmin(b, hi_t);
                const double L = up - lo;
                double content[NF];
#pragma unroll
                for (int m = 0; m < NF; ++m) content[m] = jj == j ? acc[m] : 0.0;
                if (L > 0.0) {
                    if (jj == jthick) {
#pragma unroll
                        for (int m = 0; m < NF; ++m) base_thick[m] = content[m];
                    } else {
                        const double xa = (lo - a) / hi, xb = (up - a) / hi;
#pragma unroll
                        for (int m = 0; m < NF; ++m) {
                            const double piece = L * average(c0[m], c1[m], c2[m], xa, xb);
                            s[m] += piece;
                            content[m] += piece;
                        }
                    }
                }
                if (jj == j_end) {
                    if (jj != jthick) {
#pragma unroll
                        for (int m = 0; m < NF; ++m) acc[m] = content[m];
                    }
                    break;
                }
                if (jj != jthick) {
                    const double hgt = io.ht(jj);
                    if (hgt > 0.0) {
#pragma unroll
                        for (int m = 0; m < NF; ++m) io.put(m, jj, content[m] / hgt);
                    } else {                                   // vanished target: this cell's value at its position
                        const double xi = (tl - a) / hi;
#pragma unroll
                        for (int m = 0; m < NF; ++m) io.put(m, jj, c0[m] + xi * (c1[m] + xi * c2[m]));
                    }
                }
                ++jj;
                tl = th;
                th = th + io.ht(jj);
            }
            if (jthick >= 0) {
                const double hgt = jthick < j_end ? io.ht(jthick) : 0.0;
#pragma unroll
                for (int m = 0; m < NF; ++m) {
                    const double cth = base_thick[m] + (wu[m][2] * hi - s[m]);
                    if (jthick < j_end) io.put(m, jthick, cth / hgt);     // a piece implies a positive thickness
                    else acc[m] = cth;
                }
            }
            if (j_end == n1 - 1) last_reached = true;
            if (last_reached && !last_set) {                       // x = t_edge[n1-1] = tl when j_end = n1-1
                const double xi = (tl - a) / hi;
#pragma unroll
                for (int m = 0; m < NF; ++m) last_val[m] = c0[m] + xi * (c1[m] + xi * c2[m]);
                last_set = true;
            }
            j = j_end;
            t_lo = tl;
            t_hi = th;
            a = b;
        }
        // ---- slide the window
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            wh[s] = wh[s + 1];
#pragma unroll
            for (int m = 0; m < NF; ++m) wu[m][s] = wu[m][s + 1];
        }
        const bool in = i + 4 < n0;
        wh[5] = in ? io.hs(i + 4) : 0.0;
#pragma unroll
        for (int m = 0; m < NF; ++m) wu[m][5] = in ? io.f(m, i + 4) : 0.0;
    }

    // the current target keeps its content; targets above it were never reached: content 0, or (vanished) the
    // value of the last source cell, except a vanished last target reached by some cell (remap.py:382-397)
    for (int jj = j; jj < n1; ++jj) {
        const double hgt = io.ht(jj);
#pragma unroll
        for (int m = 0; m < NF; ++m) {
            double val;
            if (hgt > 0.0) val = (jj == j ? acc[m] : 0.0) / hgt;
            else if (jj == n1 - 1 && last_set) val = last_val[m];
            else val = io.f(m, last);
            io.put(m, jj, val);
        }
    }
}

// Column with no active source cell (remap.py:375-381): copied when n0 == n1, else every target takes the mean.
template <int NF, class IO>
PO_HDT void remap_column_dry(IO& io, int n0, int n1)
{
#pragma unroll
    for (int m = 0; m < NF; ++m) {
        if (n0 == n1) {
            for (int k = 0; k < n1; ++k) io.put(m, k, io.f(m, k));
        } else {
            double mean = 0.0;
            for (int k = 0; k < n0; ++k) mean += io.f(m, k) / n0;
            for (int k = 0; k < n1; ++k) io.put(m, k, mean);
        }
    }
}

// reconstruct (remap.py:234-294): the coefficients (c0, c1, c2) of p(xi) = c0 + c1 xi + c2 xi^2 in each of the n0
// cells (PCM; PLM from 3 cells on; PPM_H4 from 4: H4 edges, end values, edge bounding, discontinuity check, CW84
// limiter); e0, e1: scratch of n0 entries.
PO_HD void reconstruct_column(const double* h, const double* u, int n0, int sch, double* c0, double* c1, double* c2,
                               double* e0, double* e1)
{
    for (int k = 0; k < n0; ++k) { c0[k] = u[k]; c1[k] = 0.0; c2[k] = 0.0; }
    if (sch == PLM && n0 >= 3) {                           // remap.py:248-262 (e0 = slp, e1 = mslp)
        e0[0] = e0[n0 - 1] = e1[0] = e1[n0 - 1] = 0.0;
        for (int k = 1; k < n0 - 1; ++k) e0[k] = plm_slope(plm_ratio(h[k - 1], h[k], h[k + 1]), u[k - 1], u[k], u[k + 1]);
        for (int k = 1; k < n0 - 1; ++k) e1[k] = plm_monotonized(u[k - 1], u[k], u[k + 1], e0[k - 1], e0[k], e0[k + 1]);
        for (int k = 1; k < n0 - 1; ++k) plm_coef(u[k], u[k + 1], e1[k], e1[k + 1], e0[k + 1], c0[k], c1[k]);
    } else if (sch == PPM_H4 && n0 >= 4) {                 // remap.py:263-294 (e0 = left edges, e1 = right edges)
        for (int i = 2; i < n0 - 1; ++i) {
            e0[i] = h4_edge(h4_weights(h[i - 2], h[i - 1], h[i], h[i + 1]), u[i - 2], u[i - 1], u[i], u[i + 1]);
            e1[i - 1] = e0[i];
        }
        end_values(pmax(H_NEGLECT_EDGE, h[0]), pmax(H_NEGLECT_EDGE, h[1]), pmax(H_NEGLECT_EDGE, h[2]),
                   pmax(H_NEGLECT_EDGE, h[3]), u[0], u[1], u[2], u[3], e0[0], e1[0]);
        e0[1] = e1[0];
        end_values(pmax(H_NEGLECT_EDGE, h[n0 - 1]), pmax(H_NEGLECT_EDGE, h[n0 - 2]), pmax(H_NEGLECT_EDGE, h[n0 - 3]),
                   pmax(H_NEGLECT_EDGE, h[n0 - 4]), u[n0 - 1], u[n0 - 2], u[n0 - 3], u[n0 - 4], e1[n0 - 1],
                   e0[n0 - 1]);
        e1[n0 - 2] = e0[n0 - 1];
        for (int k = 0; k < n0; ++k) {
            const int km1 = k > 0 ? k - 1 : 0, kp1 = k < n0 - 1 ? k + 1 : n0 - 1;
            const double sl = bound_slope(bound_ratio(h[km1], h[k], h[kp1]), u[km1], u[k], u[kp1]);
            e0[k] = bound_edge(e0[k], u[km1], u[k], sl, -1.0);
            e1[k] = bound_edge(e1[k], u[kp1], u[k], sl, 1.0);
        }
        for (int k = 0; k < n0 - 1; ++k) check_pair(e1[k], e0[k + 1], u[k], u[k + 1]);
        for (int k = 1; k < n0 - 1; ++k) ppm_coef(u[k - 1], u[k], u[k + 1], e0[k], e1[k], c0[k], c1[k], c2[k]);
    }
}

// ------------------------------------------------------------------------------------------------------------
// The reference's array formulation of remap_column (remap.py:306-397) for one field, with the column held in
// thread-local arrays of NMAX entries (n0, n1 <= NMAX).  Used for the columns outside the one-pass sweep's domain
// (a negative or NaN target thickness); same arithmetic, same results.
template <int NMAX, class IO>
PO_HDT void remap_column_general(IO& io, int m, int n0, int n1, int scheme)
{
    double h[NMAX], u[NMAX], c0[NMAX], c1[NMAX], c2[NMAX], e0[NMAX], e1[NMAX];
    double t_edge[NMAX + 1], content[NMAX], piece[NMAX + 1];
    int piece_j[NMAX + 1];
    int n_active = 0;
    for (int k = 0; k < n0; ++k) {
        h[k] = io.hs(k);
        u[k] = io.f(m, k);
        if (h[k] > 0.0) ++n_active;
    }
    const int sch = effective_scheme(n_active, scheme);
    reconstruct_column(h, u, n0, sch, c0, c1, c2, e0, e1);
    t_edge[0] = 0.0;
    for (int j = 0; j < n1; ++j) {
        t_edge[j + 1] = t_edge[j] + io.ht(j);
        content[j] = 0.0;
    }
    double a = 0.0;
    int j = 0, last = -1;
    for (int i = 0; i < n0; ++i) {
        const double hi = h[i];
        if (hi <= 0.0) continue;
        last = i;
        const double b = a + hi;
        int npc = 0, ithick = 0;
        double thick = -1.0;
        while (j < n1) {
            const double lo = pmax(a, t_edge[j]);
            const double hi_t = j < n1 - 1 ? t_edge[j + 1] : pmax(t_edge[n1], b);
            const double up = pmin(b, hi_t);
            const double L = up - lo;
            if (L > 0.0) {
                piece[npc] = L * average(c0[i], c1[i], c2[i], (lo - a) / hi, (up - a) / hi);
                piece_j[npc] = j;
                if (L > thick) { thick = L; ithick = npc; }
                ++npc;
            }
            if (hi_t <= b && j < n1 - 1) ++j;
            else break;
        }
        if (npc > 0) {
            double s = 0.0;
            for (int q = 0; q < npc; ++q) if (q != ithick) s += piece[q];
            piece[ithick] = u[i] * hi - s;
            for (int q = 0; q < npc; ++q) content[piece_j[q]] += piece[q];
        }
        a = b;
    }
    if (last < 0) {
        double mean = 0.0;
        for (int i = 0; i < n0; ++i) mean += u[i] / n0;
        for (int jj = 0; jj < n1; ++jj) io.put(m, jj, n0 == n1 ? u[jj] : mean);
        return;
    }
    for (int jj = 0; jj < n1; ++jj) {
        const double ht = io.ht(jj);
        double val;
        if (ht > 0.0) {
            val = content[jj] / ht;
        } else {
            const double x = t_edge[jj];
            double aa = 0.0;
            val = u[last];
            for (int i = 0; i < n0; ++i) {
                if (h[i] <= 0.0) continue;
                if (x <= aa + h[i]) {
                    const double xi = (x - aa) / h[i];
                    val = c0[i] + xi * (c1[i] + xi * c2[i]);
                    break;
                }
                aa += h[i];
            }
        }
        io.put(m, jj, val);
    }
}

}  // namespace rc
}  // namespace po
