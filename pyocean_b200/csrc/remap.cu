// FP64 conservative vertical remap (PCM / PLM / PPM_H4) of water columns on B200.
//
// Reference: core/vertical/remap.py — remap_column :306-397, reconstruct :234-294 (PLM :59-97, PPM_H4 edges
// :100-231), _average :297-303, _remap_columns :400-415.
//
// One thread owns one (field, column).  Consecutive threads take consecutive i, so every per-layer load and store
// of a warp is one contiguous 256-byte segment of the (k, j, i) arrays.  The column's reconstruction and overlap
// sweep run in the reference's order with every expression evaluated as written (-fmad=false): results equal the
// reference bit for bit, including the Hallberg residual that keeps the column content exact.
#include <cmath>

#include "common.cuh"

namespace po {
namespace remap {

constexpr double H_NEGLECT = 1e-30;        // remap.py:42
constexpr double H_NEGLECT_EDGE = 1e-10;   // remap.py:43
constexpr double H_MIN_FRAC = 1e-5;        // remap.py:100
constexpr double EPS = 2.220446049250313e-16;

__device__ __forceinline__ int effective_scheme(int n_active, int scheme)
{
    if (n_active <= 1) return POCEAN_PCM;
    if (n_active <= 3 && scheme > POCEAN_PLM) return POCEAN_PLM;
    return scheme;
}

// Limited PLM slope (remap.py:59-80).
__device__ __forceinline__ double plm_slope(double h_l, double h_c, double h_r, double u_l, double u_c, double u_r)
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

// Edge-monotonic PLM slope (remap.py:83-97).
__device__ __forceinline__ double plm_monotonized(double u_l, double u_c, double u_r, double s_l, double s_c,
                                                  double s_r)
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

// Edge values (C(0), C(dz1)) of the cubic whose means over the 4 end cells are u1..u4 (remap.py:103-156).
__device__ __forceinline__ void end_values(double h1, double h2, double h3, double h4, double u1, double u2,
                                           double u3, double u4, double& e_end, double& e_in)
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

// Explicit 4th-order edge value at the interface between cells i-1 and i of the stencil h0..h3 / u0..u3
// (cells i-2 .. i+1), remap.py:159-183.
__device__ __forceinline__ double h4_edge(double h0, double h1, double h2, double h3, double u0, double u1,
                                          double u2, double u3)
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
    const double et1 = ((1.0 + (h1 * I_h012 + (h0 + h1) * I_h123)) * I_h12 * (h2 * (h2 + h3)) * u1 +
                        (1.0 + (h2 * I_h123 + (h2 + h3) * I_h012)) * I_h12 * (h1 * (h0 + h1)) * u2);
    const double et2 = (h1 * (h2 * (h2 + h3)) * I_den_et2) * (u1 - u0);
    const double et3 = (h2 * (h1 * (h0 + h1)) * I_den_et3) * (u2 - u3);
    return (et1 + (et2 + et3)) / ((h0 + h1) + (h2 + h3));
}

// Polynomial coefficients of every cell (remap.py:234-294); c0/c1/c2 and the scratch e[2*NMAX].
template <int NMAX>
__device__ void reconstruct(const double* h, const double* u, int n, int scheme, double* c0, double* c1,
                            double* c2, double* e)
{
    for (int k = 0; k < n; ++k) { c0[k] = u[k]; c1[k] = 0.0; c2[k] = 0.0; }
    if (scheme == POCEAN_PCM || n < 3) return;
    if (scheme == POCEAN_PLM) {
        double* slp = e;
        double* mslp = e + NMAX;
        slp[0] = 0.0; slp[n - 1] = 0.0; mslp[0] = 0.0; mslp[n - 1] = 0.0;
        for (int k = 1; k < n - 1; ++k) slp[k] = plm_slope(h[k - 1], h[k], h[k + 1], u[k - 1], u[k], u[k + 1]);
        for (int k = 1; k < n - 1; ++k)
            mslp[k] = plm_monotonized(u[k - 1], u[k], u[k + 1], slp[k - 1], slp[k], slp[k + 1]);
        const double almost_one = 1.0 - EPS;
        for (int k = 1; k < n - 1; ++k) {
            const double u_l = u[k] - 0.5 * mslp[k];
            const double u_r = u[k] + 0.5 * mslp[k];
            c0[k] = u_l;
            c1[k] = u_r - u_l;
            const double edge = c1[k] + c0[k];
            const double am = fabs(mslp[k + 1]);
            const double e_r = u[k + 1] - 0.5 * (slp[k + 1] >= 0.0 ? am : -am);
            if ((edge - u[k]) * (e_r - edge) < 0.0) c1[k] = c1[k] * almost_one;
        }
        return;
    }
    if (scheme != POCEAN_PPM_H4 || n < 4) return;
    double* eL = e;          // left (bottom) edge of each cell
    double* eR = e + NMAX;   // right (top) edge
    for (int i = 2; i < n - 1; ++i) {
        eL[i] = h4_edge(h[i - 2], h[i - 1], h[i], h[i + 1], u[i - 2], u[i - 1], u[i], u[i + 1]);
        eR[i - 1] = eL[i];
    }
    end_values(pmax(H_NEGLECT_EDGE, h[0]), pmax(H_NEGLECT_EDGE, h[1]), pmax(H_NEGLECT_EDGE, h[2]),
               pmax(H_NEGLECT_EDGE, h[3]), u[0], u[1], u[2], u[3], eL[0], eR[0]);
    eL[1] = eR[0];
    end_values(pmax(H_NEGLECT_EDGE, h[n - 1]), pmax(H_NEGLECT_EDGE, h[n - 2]), pmax(H_NEGLECT_EDGE, h[n - 3]),
               pmax(H_NEGLECT_EDGE, h[n - 4]), u[n - 1], u[n - 2], u[n - 3], u[n - 4], eR[n - 1], eL[n - 1]);
    eR[n - 2] = eL[n - 1];
    // bound_edges (remap.py:199-220)
    for (int k = 0; k < n; ++k) {
        const int km1 = k > 0 ? k - 1 : 0, kp1 = k < n - 1 ? k + 1 : n - 1;
        double slope_x_h = 0.0;
        if ((h[km1] + h[kp1]) + 2.0 * h[k] > 0.0) {
            const double sl = u[k] - u[km1];
            const double sc = (u[kp1] - u[km1]) * (h[k] / ((h[km1] + h[kp1]) + 2.0 * h[k]));
            const double sr = u[kp1] - u[k];
            if (sl * sr > 0.0) {
                const double m = pmin(pmin(fabs(sl), fabs(sc)), fabs(sr));
                slope_x_h = sc >= 0.0 ? m : -m;
            }
        }
        const double sgn = slope_x_h >= 0.0 ? 1.0 : -1.0;
        double l = eL[k], r = eR[k];
        if ((u[km1] - l) * (l - u[k]) < 0.0) l = u[k] - sgn * pmin(fabs(slope_x_h), fabs(l - u[k]));
        if ((u[kp1] - r) * (r - u[k]) < 0.0) r = u[k] + sgn * pmin(fabs(slope_x_h), fabs(r - u[k]));
        eL[k] = pmax(pmin(l, pmax(u[km1], u[k])), pmin(u[km1], u[k]));
        eR[k] = pmax(pmin(r, pmax(u[kp1], u[k])), pmin(u[kp1], u[k]));
    }
    // check_discontinuous (remap.py:223-231)
    for (int k = 0; k < n - 1; ++k) {
        if ((eL[k + 1] - eR[k]) * (u[k + 1] - u[k]) < 0.0) {
            double a = 0.5 * (eR[k] + eL[k + 1]);
            a = pmax(pmin(a, pmax(u[k], u[k + 1])), pmin(u[k], u[k + 1]));
            eR[k] = a;
            eL[k + 1] = a;
        }
    }
    // Colella & Woodward (1984) limiter (remap.py:265-294)
    for (int k = 1; k < n - 1; ++k) {
        const double u_l = u[k - 1], u_c = u[k], u_r = u[k + 1];
        double el = eL[k], er = eR[k];
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
        c0[k] = el;
        c1[k] = 4.0 * (u_c - el) + 2.0 * (u_c - er);
        c2[k] = 3.0 * ((er - u_c) + (el - u_c));
    }
}

// Mean of c0 + c1 x + c2 x^2 over [xa, xb] (remap.py:297-303).
__device__ __forceinline__ double average(double c0, double c1, double c2, double xa, double xb)
{
    if (xb - xa <= 1e-14) {
        const double x = 0.5 * (xa + xb);
        return c0 + x * (c1 + x * c2);
    }
    return c0 + 0.5 * c1 * (xa + xb) + c2 * (xa * xa + xa * xb + xb * xb) / 3.0;
}

template <int NMAX>
__global__ void __launch_bounds__(128) remap_columns_kernel(const double* __restrict__ h_src,
                                                            const double* __restrict__ f_src,
                                                            const double* __restrict__ h_tgt,
                                                            const uint8_t* __restrict__ wet, int n0, int n1,
                                                            int ny, int nx, int scheme, double* __restrict__ out)
{
    const i64 plane = (i64)ny * nx;
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    const double* fs = f_src + (i64)blockIdx.y * n0 * plane + c;
    double* o = out + (i64)blockIdx.y * n1 * plane + c;
    if (!wet[c]) {                                   // remap.py:405-408
        for (int k = 0; k < n1; ++k) o[k * plane] = n0 == n1 ? fs[k * plane] : nan("");
        return;
    }
    double h[NMAX], u[NMAX], c0[NMAX], c1[NMAX], c2[NMAX], e[2 * NMAX];
    double t_edge[NMAX + 1], content[NMAX], piece[NMAX + 1];
    int piece_j[NMAX + 1];
    int n_active = 0;
    for (int k = 0; k < n0; ++k) {
        h[k] = h_src[k * plane + c];
        u[k] = fs[k * plane];
        if (h[k] > 0.0) n_active++;
    }
    reconstruct<NMAX>(h, u, n0, effective_scheme(n_active, scheme), c0, c1, c2, e);

    t_edge[0] = 0.0;
    for (int j = 0; j < n1; ++j) {
        t_edge[j + 1] = t_edge[j] + h_tgt[j * plane + c];
        content[j] = 0.0;
    }
    double a = 0.0;
    int j = 0, last = -1;
    for (int i = 0; i < n0; ++i) {                   // remap.py:331-367
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
                npc++;
            }
            if (hi_t <= b && j < n1 - 1) j++;
            else break;
        }
        if (npc > 0) {
            double sacc = 0.0;
            for (int q = 0; q < npc; ++q) if (q != ithick) sacc += piece[q];
            piece[ithick] = u[i] * hi - sacc;        // Hallberg residual: exact cell content
            for (int q = 0; q < npc; ++q) content[piece_j[q]] += piece[q];
        }
        a = b;
    }
    if (last < 0) {                                  // no source thickness: keep the values (remap.py:375-381)
        double mean = 0.0;
        for (int i = 0; i < n0; ++i) mean += u[i] / n0;
        for (int jj = 0; jj < n1; ++jj) o[jj * plane] = n0 == n1 ? u[jj] : mean;
        return;
    }
    for (int jj = 0; jj < n1; ++jj) {                // remap.py:382-397
        const double ht = h_tgt[jj * plane + c];
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
        o[jj * plane] = val;
    }
}

}  // namespace remap
}  // namespace po

using namespace po;

extern "C" int pocean_remap_columns_f64(const double* h_src, const double* f_src, const double* h_tgt,
                                        const uint8_t* wet, int n0, int n1, int ny, int nx, int nfields, int scheme,
                                        double* out, void* stream)
{
    const char* fn = "pocean_remap_columns_f64";
    if (n0 < 1 || n1 < 1 || ny < 1 || nx < 1 || nfields < 1)
        return pocean_fail(POCEAN_EINVAL, "%s: sizes must be >= 1 (n0=%d n1=%d ny=%d nx=%d nfields=%d)", fn, n0, n1,
                           ny, nx, nfields);
    if (n0 > 256 || n1 > 256)
        return pocean_fail(POCEAN_EINVAL, "%s: at most 256 layers per column (n0=%d n1=%d)", fn, n0, n1);
    if (nfields > 65535) return pocean_fail(POCEAN_EINVAL, "%s: nfields=%d exceeds 65535", fn, nfields);
    if (scheme < POCEAN_PCM || scheme > POCEAN_PPM_H4)
        return pocean_fail(POCEAN_EINVAL, "%s: unknown scheme %d", fn, scheme);
    if (!h_src || !f_src || !h_tgt || !wet || !out) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const i64 plane = (i64)ny * nx;
    const dim3 grid((unsigned)((plane + 127) / 128), (unsigned)nfields);
    const int nm = n0 > n1 ? n0 : n1;
    if (nm <= 32)
        remap::remap_columns_kernel<32><<<grid, 128, 0, st>>>(h_src, f_src, h_tgt, wet, n0, n1, ny, nx, scheme, out);
    else if (nm <= 64)
        remap::remap_columns_kernel<64><<<grid, 128, 0, st>>>(h_src, f_src, h_tgt, wet, n0, n1, ny, nx, scheme, out);
    else if (nm <= 128)
        remap::remap_columns_kernel<128><<<grid, 128, 0, st>>>(h_src, f_src, h_tgt, wet, n0, n1, ny, nx, scheme,
                                                               out);
    else
        remap::remap_columns_kernel<256><<<grid, 128, 0, st>>>(h_src, f_src, h_tgt, wet, n0, n1, ny, nx, scheme,
                                                               out);
    return pocean_check_launch(fn);
}
