// The kernels either side of the tracer step: the z* / sigma / hybrid regrid that produces the remap target (with the
// remap in the same call); the velocity remap in fraction space with its face fractions; the ALE horizontal
// diffusion.
//
// Reference: core/vertical/regrid.py:44-98 (zstar_column, sigma_column, enforce_min_thickness), :100-289
// (the hybrid rule: _p1m_h2_positions, _keep_consistent, hycom1_column, transition_weight, window_shallow_sigma)
// and :309-395 (regrid_columns), core/vertical/remap.py:199-220 (_bound_edges), core/components/vertical_coordinate.py:69-111, 142-153 (ALECoordinate.regrid_remap / regrid /
// remap_faces), core/vertical/ale.py:883-902 (_fractions_kernel), core/dynamics/sigma_baroclinic.py:533-561
// (_diffuse_ale_kernel) with the periodic pad/crop of core/components/tracers.py:436-447.
//
// Every expression keeps the reference's order (compiled with -fmad=false), so results are bit-identical.
#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "remap_io.cuh"

namespace po {
namespace nb {

__device__ __forceinline__ double nan_to_num(double x)          // numpy.nan_to_num
{
    if (isnan(x)) return 0.0;
    if (isinf(x)) return x > 0.0 ? DBL_MAX : -DBL_MAX;
    return x;
}

// regrid.py:44-61 `zstar_column` into e (surface first, n+1 heights); the bed-first interfaces are e[n - j].
__device__ __forceinline__ void zstar_heights(double H, double eta, const double* __restrict__ dz_top, int n,
                                              double h_min, double* e)
{
    const double D = H + eta;
    const double hm = pmin(h_min, D / n);
    const double s = D / H;
    e[0] = eta;
    for (int k = 0; k < n; ++k) e[k + 1] = e[k] - s * __ldg(dz_top + k);
    e[n] = -H;
    for (int k = n - 1; k >= 0; --k)
        if (e[k] < e[k + 1] + hm) e[k] = e[k + 1] + hm;
}

// regrid.py:63-78 `sigma_column` with `enforce_min_thickness` (:87-98) into zw (bed first, n+1 heights).
__device__ __forceinline__ void sigma_heights(double H, double eta, const double* __restrict__ dsigma, int n,
                                              double h_min, double* zw)
{
    const double D = H + eta;
    zw[0] = -H;
    for (int j = 0; j < n; ++j) zw[j + 1] = zw[j] + D * __ldg(dsigma + j);
    zw[n] = eta;
    const double hm = pmin(h_min, (zw[n] - zw[0]) / n);
    for (int j = n - 1; j > 0; --j)
        if (zw[j] > zw[j + 1] - hm) zw[j] = zw[j + 1] - hm;
    for (int j = 1; j < n; ++j)
        if (zw[j] < zw[j - 1] + hm) zw[j] = zw[j - 1] + hm;
}

// One thread per column: wet = active & (H + eta > 0) & (sum_k h_src > 0) and h_new (the rule's thicknesses where
// wet, else h_src).  The remap that follows is the ordinary column remap with h_new as the target: a single kernel
// that remapped from the heights it had just built was measured 6-8 % slower at 512 x 512 x 50 (the remap is
// latency-bound and the regrid's registers and column array cost it occupancy), so the two stay separate launches.
template <int NMAX>
__global__ void __launch_bounds__(128) regrid_kernel(int rule, const double* __restrict__ Hin,
                                                     const double* __restrict__ eta, const double* __restrict__ h_src,
                                                     const uint8_t* __restrict__ active,
                                                     const double* __restrict__ coord, double h_min, int n, i64 plane,
                                                     double* __restrict__ h_new, uint8_t* __restrict__ wet_out,
                                                     int* __restrict__ bad)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    const double H = nan_to_num(__ldg(Hin + c));
    double tot = 0.0;                                          // h_src.sum(axis=0), k = 0 .. n-1
    for (int k = 0; k < n; ++k) tot += __ldg(h_src + k * plane + c);
    const double et = __ldg(eta + c);
    const bool wet = __ldg(active + c) != 0 && H + et > 0.0 && tot > 0.0;
    wet_out[c] = wet;
    if (!wet) {
        for (int k = 0; k < n; ++k) h_new[k * plane + c] = __ldg(h_src + k * plane + c);
        return;
    }
    double z[NMAX + 1];
    if (rule == 0) {
        if (!(H > 0.0) && bad) atomicAdd(bad, 1);
        zstar_heights(H, et, coord, n, h_min, z);
        for (int k = 0; k < n; ++k) h_new[k * plane + c] = z[n - k - 1] - z[n - k];   // zw[k] = e[n - k]
    } else {
        sigma_heights(H, et, coord, n, h_min, z);
        for (int k = 0; k < n; ++k) h_new[k * plane + c] = z[k + 1] - z[k];
    }
}

// ---------------------------------------------------------------------------------------------------------------
// The hybrid (HYCOM1) rule (regrid.py:100-289, 309-342), one thread per column.
//
// The reference builds 2n edge densities per column and, for each of the n-1 target densities, scans them in order
// for the first match (a point hit on an interface, else the layer whose edges bracket it).  Here the column keeps
// only the n+1 interface densities I: after the reference's running minimum the layer densities are nondecreasing
// downwards, each bounded edge lies between its layer's and its neighbour's density (the bound of `_bound_edges`),
// and the two edges meeting at an interface are equal after the averaging step (their mean, computed as
// 0.5 * (a + b), stays between the same two densities), so I is nondecreasing and the first match is found by a
// binary search, bit for bit the same position.  The per-thread state is four (n+1)-arrays (interface densities,
// positions, cumulative thickness, the modified densities, later reused for the windowed grids) plus a bitmask of
// the kept interfaces; the thicknesses and the columns' own densities are re-read from global memory (coalesced
// across the warp's columns).  Non-finite densities make I unordered: the search stays in bounds and the column is
// reported as bad, as the reference raises for it.

// regrid.py:87-98 `enforce_min_thickness` on bed-first interfaces.
__device__ __forceinline__ void enforce_min_thickness(double* zw, int n, double h_min)
{
    const double hm = pmin(h_min, (zw[n] - zw[0]) / n);
    for (int j = n - 1; j > 0; --j)
        if (zw[j] > zw[j + 1] - hm) zw[j] = zw[j + 1] - hm;
    for (int j = 1; j < n; ++j)
        if (zw[j] < zw[j - 1] + hm) zw[j] = zw[j - 1] + hm;
}

struct HybridParams {
    const double* rho_target;      // n+1, surface first
    const double* dz_top;          // n, surface first
    const double* max_h_top;       // n
    const double* dsigma;          // n, bed first
    double d_sigma, d_hybrid, h_min;
    int keep;
};

// One column's thickness and own density, surface first (k = 0 is the top layer).
struct HybridColumn {
    const double* h;               // h_src + c
    const double* r;               // rho + c
    i64 plane;
    int n;
    __device__ __forceinline__ double th(int k) const { return __ldg(h + (i64)(n - 1 - k) * plane); }
    __device__ __forceinline__ double rho(int k) const { return __ldg(r + (i64)(n - 1 - k) * plane); }
};

// The weighted edge density between top-first layers k-1 and k (regrid.py:112-117).
__device__ __forceinline__ double edge_weighted(double h0, double h1, double r0, double r1)
{
    if (h0 + h1 == 0.0) return 0.5 * (r0 + r1);
    return (r0 * h1 + r1 * h0) / (h0 + h1);
}

// regrid.py:100-154 `_p1m_h2_positions` for m target layers (m + 1 target densities).  u: the modified densities;
// I out: interface densities; G out: cumulative thickness from the surface; x out: the m + 1 interface depths.
__device__ __forceinline__ void p1m_h2_positions(const HybridColumn& col, const double* u,
                                                 const double* __restrict__ targets, int m, double* I, double* G,
                                                 double* x)
{
    const int n = col.n;
    double hm = col.th(0), hc = hm;                   // sliding h[k-1], h[k], h[k+1]
    double hp = n > 1 ? col.th(1) : hc;
    double wl = u[0];                                 // left edge of layer k before bounding
    double er_prev = 0.0;
    G[0] = 0.0;
    for (int k = 0; k < n; ++k) {
        const int km1 = k - 1 > 0 ? k - 1 : 0;
        const int kp1 = k + 1 < n - 1 ? k + 1 : n - 1;
        const double um = u[km1], uc = u[k], up = u[kp1];
        const double wr = k == n - 1 ? u[n - 1] : edge_weighted(hc, hp, uc, up);
        // remap.py:199-220 `_bound_edges` for layer k
        double slope_x_h = 0.0;
        if ((hm + hp) + 2.0 * hc > 0.0) {
            const double sl = uc - um;
            const double sc = (up - um) * (hc / ((hm + hp) + 2.0 * hc));
            const double sr = up - uc;
            if (sl * sr > 0.0) {
                const double m = pmin(pmin(fabs(sl), fabs(sc)), fabs(sr));
                slope_x_h = sc >= 0.0 ? m : -m;
            }
        }
        const double sg = slope_x_h >= 0.0 ? 1.0 : -1.0;
        double el = wl, er = wr;
        if ((um - el) * (el - uc) < 0.0) el = uc - sg * pmin(fabs(slope_x_h), fabs(el - uc));
        if ((up - er) * (er - uc) < 0.0) er = uc + sg * pmin(fabs(slope_x_h), fabs(er - uc));
        el = pmax(pmin(el, pmax(um, uc)), pmin(um, uc));
        er = pmax(pmin(er, pmax(up, uc)), pmin(up, uc));
        // regrid.py:120-124: the two edges meeting at interface k are replaced by their mean where they differ
        I[k] = k == 0 ? el : (er_prev != el ? 0.5 * (er_prev + el) : er_prev);
        er_prev = er;
        G[k + 1] = G[k] + hc;
        wl = wr;
        hm = hc;
        hc = hp;
        hp = k + 2 < n ? col.th(k + 2) : hc;
    }
    I[n] = er_prev;
    // the fallback where no cell matches (a non-finite density): the source grid, or uniform for another count
    for (int k = 0; k <= m; ++k) x[k] = m == n ? G[k] : G[n] * (double)k / (double)m;
    for (int kk = 1; kk < m; ++kk) {
        const double t = __ldg(targets + kk);
        int lo = 0, len = n + 1;                      // p = first index with I[p] >= t (n + 1 if none)
        while (len > 0) {
            const int half = len >> 1;
            if (!(I[lo + half] >= t)) {
                lo += half + 1;
                len -= half + 1;
            } else {
                len = half;
            }
        }
        const int p = lo;
        if (t <= I[0]) x[kk] = G[0];
        else if (p >= 1 && p <= n - 1 && I[p] == t) x[kk] = G[p];
        else if (t >= I[n]) x[kk] = G[n];
        else if (p >= 1 && p <= n && I[p - 1] < t && t < I[p]) {
            const double xi = (t - I[p - 1]) / (I[p] - I[p - 1]);
            x[kk] = G[p - 1] + pmin(pmax(xi, 0.0), 1.0) * col.th(p - 1);
        }
    }
}

// regrid.py:158-201 `_keep_consistent`: interfaces between layers already in their density class stay put.
template <int NMAX>
__device__ __forceinline__ void keep_consistent(const HybridColumn& col, const double* __restrict__ targets,
                                                double h_mass, const double* G, double* x)
{
    const int n = col.n;
    uint32_t kept[(NMAX + 32) / 32];
    for (int w = 0; w <= n / 32; ++w) kept[w] = 0u;
    double h0 = col.th(0), r0 = col.rho(0);
    bool ok0 = h0 < h_mass || (__ldg(targets) <= r0 && r0 <= __ldg(targets + 1));
    for (int j = 1; j < n; ++j) {
        const double h1 = col.th(j), r1 = col.rho(j);
        const double tj = __ldg(targets + j);
        const bool ok1 = h1 < h_mass || (tj <= r1 && r1 <= __ldg(targets + j + 1));
        const bool straddle = h0 >= h_mass && h1 >= h_mass && r0 <= tj && tj <= r1;
        if ((ok0 && ok1) || straddle) {
            x[j] = G[j];
            kept[j >> 5] |= 1u << (j & 31);
        }
        h0 = h1;
        r0 = r1;
        ok0 = ok1;
    }
    double lo = G[0];
    for (int j = 1; j < n; ++j) {
        if ((kept[j >> 5] >> (j & 31)) & 1u) lo = x[j];
        else if (x[j] < lo) x[j] = lo;
    }
    double hi = G[n];
    for (int j = n - 1; j > 0; --j) {
        if ((kept[j >> 5] >> (j & 31)) & 1u) hi = x[j];
        else if (x[j] > hi) x[j] = hi;
    }
}

// regrid.py:204-252 `hycom1_column` for m target layers into zw (bed first, m+1); A, B, G scratch of
// max(n, m) + 1 each.  The isopycnal test (`keep`) applies only when m == n, as in the reference.
template <int NMAX>
__device__ __forceinline__ void hycom1_column(double H, double eta, const HybridColumn& col, const HybridParams& P,
                                              int m, double* zw, double* A, double* B, double* G)
{
    const int n = col.n;
    const double D = H + eta;
    const double h_mass = 2.0 * P.h_min;
    double last = -1.0;                       // massless layers take the density of the massive layer above
    int k0 = -1;                              // the first massive layer
    for (int k = 0; k < n; ++k) {
        double r = col.rho(k);
        if (col.th(k) >= h_mass) {
            last = r;
            if (k0 < 0) k0 = k;
        } else if (last >= 0.0) {
            r = last;
        }
        A[k] = r;
    }
    if (k0 > 0)                               // massless top layers take the first massive layer's density
        for (int kk = 0; kk < k0; ++kk) A[kk] = A[k0];
    for (int k = n - 2; k >= 0; --k) A[k] = pmin(A[k], A[k + 1]);
    double* x = zw;                           // depths in zw's storage, reversed into A below
    p1m_h2_positions(col, A, P.rho_target, m, B, G, x);
    if (P.keep && m == n) keep_consistent<NMAX>(col, P.rho_target, 2.0 * P.h_min, G, x);
    const double s = D / H;
    double nominal = 0.0;
    for (int k = 1; k <= m; ++k) {
        nominal += __ldg(P.dz_top + k - 1) * s;
        x[k] = pmin(pmax(x[k], nominal), D);
    }
    for (int k = 1; k < m; ++k) x[k] = pmin(x[k], x[k - 1] + __ldg(P.max_h_top + k - 1));
    for (int k = 1; k <= m; ++k) x[k] = pmax(x[k], x[k - 1]);
    x[m] = D;
    for (int j = 0; j <= m; ++j) A[j] = eta - x[m - j];
    A[0] = -H;
    A[m] = eta;
    enforce_min_thickness(A, m, P.h_min);
    for (int j = 0; j <= m; ++j) zw[j] = A[j];
}

// regrid.py:255-260 `transition_weight`.
__device__ __forceinline__ double transition_weight(double D, double d_sigma, double d_hybrid)
{
    if (d_hybrid <= d_sigma) return D > d_sigma ? 1.0 : 0.0;
    return pmin(pmax((D - d_sigma) / (d_hybrid - d_sigma), 0.0), 1.0);
}

// The hybrid rule of `_regrid_columns` (regrid.py:322-340) for one wet column: sigma where the shallow-sigma weight
// is 0 (or H <= 0 with a sigma zone), else hycom1_column, windowed towards sigma where 0 < q < 1; zw bed first (m+1).
template <int NMAX>
__device__ __forceinline__ void hybrid_column(double H, double et, const HybridColumn& hc, const HybridParams& P,
                                              int m, double* col, double* A, double* B, double* G)
{
    const double q = P.d_hybrid > 0.0 ? transition_weight(H + et, P.d_sigma, P.d_hybrid) : 1.0;
    const double qq = (P.d_hybrid > 0.0 && H <= 0.0) ? 0.0 : q;     // flooded land: sigma at any depth
    if (qq <= 0.0) {
        sigma_heights(H, et, P.dsigma, m, P.h_min, col);
        return;
    }
    hycom1_column<NMAX>(H, et, hc, P, m, col, A, B, G);
    if (qq < 1.0) {                                   // regrid.py:263-289 `window_shallow_sigma`
        double* sig = A;
        double* zs = B;
        sigma_heights(H, et, P.dsigma, m, P.h_min, sig);
        zstar_heights(H, et, P.dz_top, m, P.h_min, zs);   // surface first: bed-first interface j is zs[m - j]
        for (int j = 0; j <= m; ++j) {
            const double lo = qq * (-H) + (1.0 - qq) * sig[j];
            const double hi = qq * zs[m - j] + (1.0 - qq) * sig[j];
            col[j] = pmin(pmax(col[j], lo), hi);
        }
        col[0] = -H;
        col[m] = sig[m];
        enforce_min_thickness(col, m, P.h_min);
    }
}

// One thread per column: the hybrid rule of `_regrid_columns` (code 2) with the wet mask and h_new of
// regrid_kernel.  bad counts wet columns with H <= 0 and no sigma zone, or a non-finite density.
template <int NMAX>
__global__ void __launch_bounds__(128) regrid_hybrid_kernel(const double* __restrict__ Hin,
                                                            const double* __restrict__ eta,
                                                            const double* __restrict__ h_src,
                                                            const uint8_t* __restrict__ active,
                                                            const double* __restrict__ rho, HybridParams P, int n,
                                                            i64 plane, double* __restrict__ h_new,
                                                            uint8_t* __restrict__ wet_out, int* __restrict__ bad)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    const double H = nan_to_num(__ldg(Hin + c));
    double tot = 0.0;
    for (int k = 0; k < n; ++k) tot += __ldg(h_src + k * plane + c);
    const double et = __ldg(eta + c);
    const bool wet = __ldg(active + c) != 0 && H + et > 0.0 && tot > 0.0;
    wet_out[c] = wet;
    if (!wet) {
        for (int k = 0; k < n; ++k) h_new[k * plane + c] = __ldg(h_src + k * plane + c);
        return;
    }
    bool finite = true;
    for (int k = 0; k < n; ++k) finite = finite && isfinite(__ldg(rho + k * plane + c));
    if ((!finite || (P.d_hybrid <= 0.0 && !(H > 0.0))) && bad) atomicAdd(bad, 1);
    double col[NMAX + 1], A[NMAX + 1], B[NMAX + 1], G[NMAX + 1];
    const HybridColumn hc{h_src + c, rho + c, plane, n};
    hybrid_column<NMAX>(H, et, hc, P, n, col, A, B, G);
    for (int k = 0; k < n; ++k) h_new[k * plane + c] = col[k + 1] - col[k];
}

// One thread per column: `_regrid_columns` (regrid.py:309-342) itself, target interface heights zw (m+1, bed first)
// of every column that `wet` marks (the others NaN, as the reference leaves them); code 0 z*, 1 sigma, 2 hybrid on
// the n source layers h, rho (m may differ from n only for the hybrid rule).
template <int NMAX>
__global__ void __launch_bounds__(128) regrid_columns_kernel(int code, const double* __restrict__ Hin,
                                                             const double* __restrict__ eta,
                                                             const double* __restrict__ h,
                                                             const double* __restrict__ rho,
                                                             const uint8_t* __restrict__ wet, HybridParams P, int n,
                                                             int m, i64 plane, double* __restrict__ zw)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    if (!__ldg(wet + c)) {
        for (int k = 0; k <= m; ++k) zw[k * plane + c] = nan("");
        return;
    }
    const double H = nan_to_num(__ldg(Hin + c)), et = __ldg(eta + c);
    double col[NMAX + 1], A[NMAX + 1], B[NMAX + 1], G[NMAX + 1];
    if (code == 0) {
        zstar_heights(H, et, P.dz_top, m, P.h_min, A);
        for (int j = 0; j <= m; ++j) col[j] = A[m - j];
    } else if (code == 1) {
        sigma_heights(H, et, P.dsigma, m, P.h_min, col);
    } else {
        const HybridColumn hc{h + c, rho + c, plane, n};
        hybrid_column<NMAX>(H, et, hc, P, m, col, A, B, G);
    }
    for (int k = 0; k <= m; ++k) zw[k * plane + c] = col[k];
}

// Column IO of the velocity remap in fraction space (vertical_coordinate.py:142-153): source thickness
// w_src,k S and target w_tgt,k S, with w = hf / sum(hf) (1/n where the sum is not positive, ale.py:883-892) and S the
// source column total (1 where it is not positive); the fractions are formed on the fly, never stored.
template <int NF>
struct FractionIO {
    const double* __restrict__ hfs;
    const double* __restrict__ hft;
    const double* __restrict__ wt;             // given target fractions, or null
    const double* __restrict__ u[NF];
    double* __restrict__ o[NF];
    i64 plane;
    int n;
    double tot_s, tot_t, S;
    __device__ __forceinline__ double hs(int k) const
    {
        const double w = tot_s > 0.0 ? __ldg(hfs + k * plane) / tot_s : 1.0 / n;
        return w * S;
    }
    __device__ __forceinline__ double ht(int k) const
    {
        const double w = wt ? __ldg(wt + k * plane) : (tot_t > 0.0 ? __ldg(hft + k * plane) / tot_t : 1.0 / n);
        return w * S;
    }
    __device__ __forceinline__ double f(int m, int k) const { return __ldg(u[m] + k * plane); }
    __device__ __forceinline__ void put(int m, int k, double v) { o[m][k * plane] = v; }
};

template <int NF>
__device__ __forceinline__ void fraction_io(FractionIO<NF>& io, const double* hf_src, const double* hf_tgt,
                                            const double* w_tgt, int n, i64 plane, i64 c)
{
    io.hfs = hf_src + c;
    io.hft = hf_tgt ? hf_tgt + c : nullptr;
    io.wt = w_tgt ? w_tgt + c : nullptr;
    io.plane = plane;
    io.n = n;
    double ts = 0.0, tt = 0.0;
    for (int k = 0; k < n; ++k) ts += __ldg(io.hfs + k * plane);
    if (!w_tgt)
        for (int k = 0; k < n; ++k) tt += __ldg(io.hft + k * plane);
    io.tot_s = ts;
    io.tot_t = tt;
    io.S = ts > 0.0 ? ts : 1.0;
}

// Register budgets of the velocity remap as resident 128-thread CTAs per SM, one field per thread (NF = 1) or two:
// fitted to 7 and 5 (u-faces of 512 x 512 x 50: 1.17 and 1.93 ms against 1.43 and 2.48 at ptxas's own choice of
// 108 / 152 registers; 5 / 6 and 3 / 4 in between).
#ifndef POCEAN_VREMAP1_CTAS
#define POCEAN_VREMAP1_CTAS 7
#endif
#ifndef POCEAN_VREMAP2_CTAS
#define POCEAN_VREMAP2_CTAS 5
#endif
// One thread per face column and field group (NF fields from NF * blockIdx.y).
template <int NF>
__global__ void __launch_bounds__(128, NF == 1 ? POCEAN_VREMAP1_CTAS : POCEAN_VREMAP2_CTAS)
remap_faces_kernel(const double* __restrict__ vel, const double* __restrict__ hf_src, const double* __restrict__ hf_tgt,
                   const double* __restrict__ w_tgt, int n, i64 plane, int field0, int scheme, double* __restrict__ out)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    FractionIO<NF> io;
    fraction_io(io, hf_src, hf_tgt, w_tgt, n, plane, c);
    const int m0 = field0 + NF * (int)blockIdx.y;
#pragma unroll
    for (int m = 0; m < NF; ++m) {
        io.u[m] = vel + (i64)(m0 + m) * n * plane + c;
        io.o[m] = out + (i64)(m0 + m) * n * plane + c;
    }
    remap::remap_column_io<NF>(io, io.tot_s > 0.0, n, n, scheme);
}

// The general algorithm for the sentinel columns of the velocity remap.
template <int NMAX>
__global__ void __launch_bounds__(128) remap_faces_general_kernel(const double* __restrict__ vel,
                                                                  const double* __restrict__ hf_src,
                                                                  const double* __restrict__ hf_tgt,
                                                                  const double* __restrict__ w_tgt, int n,
                                                                  i64 plane, int scheme, double* __restrict__ out)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    double* o = out + (i64)blockIdx.y * n * plane + c;
    if (__double_as_longlong(o[0]) != remap::kRedo) return;
    FractionIO<1> io;
    fraction_io(io, hf_src, hf_tgt, w_tgt, n, plane, c);
    io.u[0] = vel + (i64)blockIdx.y * n * plane + c;
    io.o[0] = o;
    rc::remap_column_general<NMAX>(io, 0, n, n, scheme);
}

// ale.py:883-892 `_fractions_kernel`.
__global__ void __launch_bounds__(128) face_fractions_kernel(const double* __restrict__ hf, int n, i64 plane,
                                                             double* __restrict__ w)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    double tot = 0.0;
    for (int k = 0; k < n; ++k) tot += __ldg(hf + k * plane + c);
    for (int k = 0; k < n; ++k) w[k * plane + c] = tot > 0.0 ? __ldg(hf + k * plane + c) / tot : 1.0 / n;
}

// sigma_baroclinic.py:533-561 `_diffuse_ale_kernel` for nt stacked fields sharing the geometry; periodic axes
// natively (the wrap face of cells 0 and n-1 is face 0, as the reference's halo-1 pad/crop reads it).  One thread
// per (j, i) column and DKL consecutive layers: the column's masks and metrics are read once for its layers;
// consecutive threads take consecutive i.  Every index is valid whether or not its face exists, so each layer's
// loads are issued together and the masks applied afterwards.
constexpr int DTI = 32, DTJ = 4, DKL = 4;

// Register budget of the diffusion as resident 128-thread CTAs per SM: fitted to 12 (T and S at 512 x 512 x 50:
// 0.236 ms against 0.334 at ptxas's choice of 80 registers, 0.273 at 8 and 0.246 at 10).
#ifndef POCEAN_DIFF_CTAS
#define POCEAN_DIFF_CTAS 12
#endif
#if POCEAN_DIFF_CTAS > 0
#define DIFF_BOUNDS __launch_bounds__(DTI * DTJ, POCEAN_DIFF_CTAS)
#else
#define DIFF_BOUNDS __launch_bounds__(DTI * DTJ)
#endif
__global__ void DIFF_BOUNDS diffuse_ale_kernel(const double* __restrict__ T,
                                                                const double* __restrict__ Tw,
                                                                const double* __restrict__ h,
                                                                const uint8_t* __restrict__ act,
                                                                const double* __restrict__ cx,
                                                                const double* __restrict__ cy,
                                                                const uint8_t* __restrict__ okx,
                                                                const uint8_t* __restrict__ oky,
                                                                const double* __restrict__ V, int nt, int n, int ny,
                                                                int nx, bool per_x, bool per_y, double kh, double dt,
                                                                double* __restrict__ out)
{
    const int i = blockIdx.x * DTI + threadIdx.x % DTI;
    const int j = blockIdx.y * DTJ + threadIdx.x / DTI;
    if (i >= nx || j >= ny) return;
    const int k0 = blockIdx.z * DKL, k1 = min(k0 + DKL, n);
    const i64 plane = (i64)ny * nx;
    const i64 a = (i64)j * nx + i;
    const bool has_w = (i > 0 || per_x), has_e = (i < nx - 1 || per_x);
    const bool has_s = (j > 0 || per_y), has_n = (j < ny - 1 || per_y);
    const int iw = i > 0 ? i - 1 : nx - 1, ie = i < nx - 1 ? i + 1 : 0;
    const int js = j > 0 ? j - 1 : ny - 1, jn = j < ny - 1 ? j + 1 : 0;
    const i64 fw_i = (i64)j * (nx + 1) + i, fe_i = (i64)j * (nx + 1) + ie;
    const i64 fs_i = (i64)j * nx + i, fn_i = (i64)jn * nx + i;
    const i64 aw = (i64)j * nx + iw, ae = (i64)j * nx + ie, as = (i64)js * nx + i, an = (i64)jn * nx + i;
    const bool ow = has_w && __ldg(okx + fw_i), oe = has_e && __ldg(okx + fe_i);
    const bool os = has_s && __ldg(oky + fs_i), on = has_n && __ldg(oky + fn_i);
    const bool ac = __ldg(act + a) != 0;
    const bool bw = __ldg(act + aw) && ac, be = ac && __ldg(act + ae);
    const bool bs = __ldg(act + as) && ac, bn = ac && __ldg(act + an);
    const double cxw = __ldg(cx + fw_i), cxe = __ldg(cx + fe_i), cys = __ldg(cy + fs_i), cyn = __ldg(cy + fn_i);
#pragma unroll 2
    for (int k = k0; k < k1; ++k) {
        const i64 hk = (i64)k * plane;
        const double hc = __ldg(h + hk + a), hw = __ldg(h + hk + aw), he = __ldg(h + hk + ae),
                     hs = __ldg(h + hk + as), hn = __ldg(h + hk + an);
        const double v = __ldg(V + hk + a);
        const double hu_w = bw ? pmin(hw, hc) : 0.0;
        const double hu_e = be ? pmin(hc, he) : 0.0;
        const double hv_s = bs ? pmin(hs, hc) : 0.0;
        const double hv_n = bn ? pmin(hc, hn) : 0.0;
        for (int t = 0; t < nt; ++t) {
            const i64 to = (i64)t * n * plane + hk;
            const double* tw = Tw + to;
            const double twc = __ldg(tw + a), tww = __ldg(tw + aw), twe = __ldg(tw + ae), tws = __ldg(tw + as),
                         twn = __ldg(tw + an);
            const double tc = __ldg(T + to + a);
            const double fw = ow ? -kh * cxw * hu_w * (twc - tww) : 0.0;
            const double fe = oe ? -kh * cxe * hu_e * (twe - twc) : 0.0;
            const double fs = os ? -kh * cys * hv_s * (twc - tws) : 0.0;
            const double fn = on ? -kh * cyn * hv_n * (twn - twc) : 0.0;
            const double div = fe - fw + fn - fs;
            out[to + a] = v > 0.0 ? tc - dt * div / v : tc;
        }
    }
}

}  // namespace nb
}  // namespace po

using namespace po;

extern "C" int pocean_regrid_remap_f64(int rule, const double* H, const double* eta, const double* h_src,
                                       const uint8_t* active, const double* coord, double h_min,
                                       const double* f_src, int nz, int ny, int nx, int nfields, int scheme,
                                       double* h_new, uint8_t* wet, double* out, int* bad_columns, void* stream)
{
    const char* fn = "pocean_regrid_remap_f64";
    if (rule != POCEAN_REGRID_ZSTAR && rule != POCEAN_REGRID_SIGMA)
        return pocean_fail(POCEAN_EINVAL, "%s: unknown rule %d (z* = 0, sigma = 1)", fn, rule);
    if (nz < 1 || ny < 1 || nx < 1 || nfields < 0)
        return pocean_fail(POCEAN_EINVAL, "%s: bad sizes nz=%d ny=%d nx=%d nfields=%d", fn, nz, ny, nx, nfields);
    if (nz > 256) return pocean_fail(POCEAN_EINVAL, "%s: at most 256 layers per column (nz=%d)", fn, nz);
    if (nfields > 65535) return pocean_fail(POCEAN_EINVAL, "%s: nfields=%d exceeds 65535", fn, nfields);
    if (nfields > 0 && (scheme < POCEAN_PCM || scheme > POCEAN_PPM_H4))
        return pocean_fail(POCEAN_EINVAL, "%s: unknown scheme %d", fn, scheme);
    if (!H || !eta || !h_src || !active || !coord || !h_new || !wet || (nfields > 0 && (!f_src || !out)))
        return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const i64 plane = (i64)ny * nx;
    const unsigned gx = (unsigned)((plane + 127) / 128);
    if (nz <= 64)
        nb::regrid_kernel<64><<<gx, 128, 0, st>>>(rule, H, eta, h_src, active, coord, h_min, nz, plane, h_new, wet,
                                                  bad_columns);
    else if (nz <= 128)
        nb::regrid_kernel<128><<<gx, 128, 0, st>>>(rule, H, eta, h_src, active, coord, h_min, nz, plane, h_new, wet,
                                                   bad_columns);
    else
        nb::regrid_kernel<256><<<gx, 128, 0, st>>>(rule, H, eta, h_src, active, coord, h_min, nz, plane, h_new, wet,
                                                   bad_columns);
    rc = pocean_check_launch(fn);
    if (rc || nfields == 0) return rc;
    return pocean_remap_columns_f64(h_src, f_src, h_new, wet, nz, nz, ny, nx, nfields, scheme, out, stream);
}

extern "C" int pocean_regrid_hybrid_remap_f64(const double* H, const double* eta, const double* h_src,
                                              const uint8_t* active, const double* rho, const double* rho_target,
                                              const double* dz_top, const double* max_h_top, const double* dsigma,
                                              double d_sigma, double d_hybrid, double h_min, int keep,
                                              const double* f_src, int nz, int ny, int nx, int nfields, int scheme,
                                              double* h_new, uint8_t* wet, double* out, int* bad_columns,
                                              void* stream)
{
    const char* fn = "pocean_regrid_hybrid_remap_f64";
    if (nz < 1 || ny < 1 || nx < 1 || nfields < 0)
        return pocean_fail(POCEAN_EINVAL, "%s: bad sizes nz=%d ny=%d nx=%d nfields=%d", fn, nz, ny, nx, nfields);
    if (nz > 256) return pocean_fail(POCEAN_EINVAL, "%s: at most 256 layers per column (nz=%d)", fn, nz);
    if (nfields > 65535) return pocean_fail(POCEAN_EINVAL, "%s: nfields=%d exceeds 65535", fn, nfields);
    if (nfields > 0 && (scheme < POCEAN_PCM || scheme > POCEAN_PPM_H4))
        return pocean_fail(POCEAN_EINVAL, "%s: unknown scheme %d", fn, scheme);
    if (!H || !eta || !h_src || !active || !rho || !rho_target || !dz_top || !max_h_top || !dsigma || !h_new ||
        !wet || (nfields > 0 && (!f_src || !out)))
        return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const i64 plane = (i64)ny * nx;
    const unsigned gx = (unsigned)((plane + 127) / 128);
    const nb::HybridParams P{rho_target, dz_top, max_h_top, dsigma, d_sigma, d_hybrid, h_min, keep};
    if (nz <= 64)
        nb::regrid_hybrid_kernel<64><<<gx, 128, 0, st>>>(H, eta, h_src, active, rho, P, nz, plane, h_new, wet,
                                                         bad_columns);
    else if (nz <= 128)
        nb::regrid_hybrid_kernel<128><<<gx, 128, 0, st>>>(H, eta, h_src, active, rho, P, nz, plane, h_new, wet,
                                                          bad_columns);
    else
        nb::regrid_hybrid_kernel<256><<<gx, 128, 0, st>>>(H, eta, h_src, active, rho, P, nz, plane, h_new, wet,
                                                          bad_columns);
    rc = pocean_check_launch(fn);
    if (rc || nfields == 0) return rc;
    return pocean_remap_columns_f64(h_src, f_src, h_new, wet, nz, nz, ny, nx, nfields, scheme, out, stream);
}

extern "C" int pocean_face_fractions_f64(const double* hf, int nz, int ny, int nx, double* w, void* stream)
{
    const char* fn = "pocean_face_fractions_f64";
    if (nz < 1 || ny < 1 || nx < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (!hf || !w) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    const i64 plane = (i64)ny * nx;
    nb::face_fractions_kernel<<<(unsigned)((plane + 127) / 128), 128, 0, (cudaStream_t)stream>>>(hf, nz, plane, w);
    return pocean_check_launch(fn);
}

extern "C" int pocean_remap_faces_f64(const double* vel, const double* hf_src, const double* hf_tgt,
                                      const double* w_tgt, int nz, int ny, int nx, int nfields, int scheme,
                                      double* out, void* stream)
{
    const char* fn = "pocean_remap_faces_f64";
    if (nz < 1 || ny < 1 || nx < 1 || nfields < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (nz > 256) return pocean_fail(POCEAN_EINVAL, "%s: at most 256 layers per column (nz=%d)", fn, nz);
    if (nfields > 65535) return pocean_fail(POCEAN_EINVAL, "%s: nfields=%d exceeds 65535", fn, nfields);
    if (scheme < POCEAN_PCM || scheme > POCEAN_PPM_H4) return pocean_fail(POCEAN_EINVAL, "%s: unknown scheme", fn);
    if (!vel || !hf_src || (!hf_tgt && !w_tgt) || !out) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const i64 plane = (i64)ny * nx;
    const unsigned gx = (unsigned)((plane + 127) / 128);
    if (nfields / 2 > 0)
        nb::remap_faces_kernel<2><<<dim3(gx, nfields / 2), 128, 0, st>>>(vel, hf_src, hf_tgt, w_tgt, nz, plane, 0,
                                                                          scheme, out);
    if (nfields & 1)
        nb::remap_faces_kernel<1><<<dim3(gx, 1), 128, 0, st>>>(vel, hf_src, hf_tgt, w_tgt, nz, plane, nfields - 1,
                                                                scheme, out);
    const dim3 g2(gx, (unsigned)nfields);
    if (nz <= 64)
        nb::remap_faces_general_kernel<64><<<g2, 128, 0, st>>>(vel, hf_src, hf_tgt, w_tgt, nz, plane, scheme, out);
    else if (nz <= 128)
        nb::remap_faces_general_kernel<128><<<g2, 128, 0, st>>>(vel, hf_src, hf_tgt, w_tgt, nz, plane, scheme, out);
    else
        nb::remap_faces_general_kernel<256><<<g2, 128, 0, st>>>(vel, hf_src, hf_tgt, w_tgt, nz, plane, scheme, out);
    return pocean_check_launch(fn);
}

extern "C" int pocean_diffuse_ale_f64(const double* T, const double* Tw, const double* h, const uint8_t* act,
                                      const double* cx, const double* cy, const uint8_t* okx, const uint8_t* oky,
                                      const double* V, int nt, int nz, int ny, int nx, unsigned flags, double kh,
                                      double dt, double* out, void* stream)
{
    const char* fn = "pocean_diffuse_ale_f64";
    if (nt < 1 || nz < 1 || ny < 1 || nx < 1 || nz > 65535)
        return pocean_fail(POCEAN_EINVAL, "%s: bad sizes nt=%d nz=%d ny=%d nx=%d", fn, nt, nz, ny, nx);
    if (flags & ~(unsigned)(POCEAN_PERIODIC_X | POCEAN_PERIODIC_Y))
        return pocean_fail(POCEAN_EINVAL, "%s: only the periodic flags apply (0x%x)", fn, flags);
    if (!T || !Tw || !h || !act || !cx || !cy || !okx || !oky || !V || !out)
        return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    const dim3 grid((unsigned)((nx + nb::DTI - 1) / nb::DTI), (unsigned)((ny + nb::DTJ - 1) / nb::DTJ),
                    (unsigned)((nz + nb::DKL - 1) / nb::DKL));
    nb::diffuse_ale_kernel<<<grid, nb::DTI * nb::DTJ, 0, (cudaStream_t)stream>>>(
        T, Tw, h, act, cx, cy, okx, oky, V, nt, nz, ny, nx, (flags & POCEAN_PERIODIC_X) != 0,
        (flags & POCEAN_PERIODIC_Y) != 0, kh, dt, out);
    return pocean_check_launch(fn);
}

extern "C" int pocean_regrid_columns_f64(int code, const double* H, const double* eta, const double* h,
                                         const double* rho, const uint8_t* wet, const double* dz_top,
                                         const double* dsigma, const double* rho_target, const double* max_h_top,
                                         double d_sigma, double d_hybrid, double h_min, int keep, int n, int m,
                                         int ny, int nx, double* zw, void* stream)
{
    const char* fn = "pocean_regrid_columns_f64";
    if (code < 0 || code > 2) return pocean_fail(POCEAN_EINVAL, "%s: unknown rule %d", fn, code);
    if (n < 1 || m < 1 || ny < 1 || nx < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (n > 256 || m > 256) return pocean_fail(POCEAN_EINVAL, "%s: at most 256 layers (n=%d m=%d)", fn, n, m);
    if (code != 2 && n != m)
        return pocean_fail(POCEAN_EINVAL, "%s: a target layer count other than the source's is only for the hybrid "
                           "rule", fn);
    if (!H || !eta || !wet || !zw || (code == 0 && !dz_top) || (code == 1 && !dsigma) ||
        (code == 2 && (!h || !rho || !dz_top || !rho_target || !max_h_top || (d_hybrid > 0.0 && !dsigma))))
        return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    nb::HybridParams P{rho_target, dz_top, max_h_top, dsigma, d_sigma, d_hybrid, h_min, keep};
    const i64 plane = (i64)ny * nx;
    const unsigned gx = (unsigned)((plane + 127) / 128);
    const int nm = n > m ? n : m;
    cudaStream_t st = (cudaStream_t)stream;
    if (nm <= 64) nb::regrid_columns_kernel<64><<<gx, 128, 0, st>>>(code, H, eta, h, rho, wet, P, n, m, plane, zw);
    else if (nm <= 128)
        nb::regrid_columns_kernel<128><<<gx, 128, 0, st>>>(code, H, eta, h, rho, wet, P, n, m, plane, zw);
    else nb::regrid_columns_kernel<256><<<gx, 128, 0, st>>>(code, H, eta, h, rho, wet, P, n, m, plane, zw);
    return pocean_check_launch(fn);
}
