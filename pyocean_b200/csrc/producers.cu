// The producers of the tracer step's inputs on B200: face transport thicknesses, the transport velocity, the PPM
// layer transport with its barotropic correction, the outflow limiter and the Lagrangian thickness, so that Qx, Qy,
// h-dagger (and from it V1) never leave HBM between the momentum step and the tracer step.
//
// Reference: core/vertical/ale.py — _ftt_kernel :177-210, _transport_velocity_kernel :789-808, _ppm_edges_kernel
// :582-626, _face_flux :629-647, _ppm_transport_kernel :650-740, _exceeds_kernel / limit_outflow / _give_back
// :300-441, lagrangian_thickness :278-294.  Every expression keeps the reference's order (-fmad=false); sums over
// layers run k = 0 .. n-1 as the reference's loops and numpy's first-axis reductions do, so results are bit-identical.
//
// Mapping: one thread per face column (j, f) or per cell column / cell-layer; consecutive threads take consecutive
// i (or f), so every per-layer access of a warp is one contiguous segment.  The Newton iteration of the PPM
// transport stops when every face has converged (the reference's global test): iteration i is one launch that
// first reads how many faces iteration i-1 left unconverged and returns at once when none, so max_iter launches are
// enqueued without a host round trip.  The outflow limiter's passes end on a global test too; it is rare (nothing
// to limit in the common case) and synchronises once per pass.
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace po {
namespace pr {

__device__ __forceinline__ double nan0(double x) { return x == x ? x : 0.0; }
__device__ __forceinline__ double nan_to_num(double x)
{
    if (isnan(x)) return 0.0;
    if (isinf(x)) return x > 0.0 ? DBL_MAX : -DBL_MAX;
    return x;
}
__device__ __forceinline__ double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : (x == 0.0 ? 0.0 : x)); }

// ale.py:177-210: one face column (j, f) of the u-faces.
__global__ void __launch_bounds__(128) ftt_kernel(const double* __restrict__ h, const double* __restrict__ H,
                                                  const uint8_t* __restrict__ active, int n, int ny, int nx, bool clip,
                                                  double* __restrict__ q_e, double* __restrict__ q_w)
{
    const int nf = nx + 1;
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (i64)ny * nf) return;
    const int j = (int)(t / nf), f = (int)(t - (i64)j * nf);
    const int iw = f > 0 ? f - 1 : 0, ie = f < nx ? f : nx - 1;
    const i64 pc = (i64)ny * nx, pf = (i64)ny * nf;
    const i64 cw = (i64)j * nx + iw, ce = (i64)j * nx + ie;
    if (!(__ldg(active + cw) && __ldg(active + ce))) {
        for (int k = 0; k < n; ++k) q_e[k * pf + t] = q_w[k * pf + t] = 0.0;
        return;
    }
    if (clip) {
        const double Hw = nan0(__ldg(H + cw)), He = nan0(__ldg(H + ce));
        const double z_bed = pmax(-Hw, -He);
        double sw = 0.0, se = 0.0;
        for (int k = 0; k < n; ++k) {
            const double hw = nan0(__ldg(h + k * pc + cw)), he = nan0(__ldg(h + k * pc + ce));
            sw += hw;
            se += he;
            q_e[k * pf + t] = pmin(hw, pmax(0.0, (-Hw + sw) - z_bed));
            q_w[k * pf + t] = pmin(he, pmax(0.0, (-He + se) - z_bed));
        }
    } else {
        for (int k = 0; k < n; ++k) {
            q_e[k * pf + t] = nan0(__ldg(h + k * pc + cw));
            q_w[k * pf + t] = nan0(__ldg(h + k * pc + ce));
        }
    }
}

// ale.py:789-808: one face column c of an (n, plane) face array.
__global__ void __launch_bounds__(128) transport_velocity_kernel(const double* __restrict__ u_new,
                                                                 const double* __restrict__ u_old,
                                                                 const uint8_t* __restrict__ last_wet,
                                                                 const double* __restrict__ w,
                                                                 const double* __restrict__ L,
                                                                 const double* __restrict__ D, int n, i64 plane,
                                                                 double theta, double theta_bc,
                                                                 double* __restrict__ ut, double* __restrict__ Qb)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    const bool lw = __ldg(last_wet + c) != 0;
    double m1 = 0.0, m0 = 0.0;
    for (int k = 0; k < n; ++k) {
        const double un = lw ? __ldg(u_old + k * plane + c) : 0.0;
        m1 += __ldg(w + k * plane + c) * __ldg(u_new + k * plane + c);
        m0 += __ldg(w + k * plane + c) * un;
    }
    const double d = (theta - theta_bc) * (m1 - m0);
    double s = 0.0;
    for (int k = 0; k < n; ++k) {
        const double un = lw ? __ldg(u_old + k * plane + c) : 0.0;
        const double x = theta_bc * __ldg(u_new + k * plane + c) + (1 - theta_bc) * un + d;
        ut[k * plane + c] = x;
        s += __ldg(w + k * plane + c) * x;
    }
    Qb[c] = __ldg(L + c) * __ldg(D + c) * s;
}

// The masked thickness the PPM kernels read: where(active, nan_to_num(h), 0) (ale.py:755).  Offsets are 32-bit:
// the PPM entry points bound every field by 2^31 entries.
struct Thick {
    const double* __restrict__ h;
    const uint8_t* __restrict__ act;
    int pc;
    int nx;
    __device__ __forceinline__ double at(int k, int j, int i) const
    {
        return __ldg(act + (j * nx + i)) ? nan_to_num(__ldg(h + (k * pc + j * nx + i))) : 0.0;
    }
    __device__ __forceinline__ double m(int j, int i) const { return __ldg(act + (j * nx + i)) ? 1.0 : 0.0; }
};

// The limited slope of cell i (first loop of _ppm_edges_kernel).
__device__ __forceinline__ double ppm_slope(const Thick& T, int k, int j, int i)
{
    const int nx = T.nx;
    const double m = T.m(j, i);
    const double mw = i > 0 ? T.m(j, i - 1) : 0.0;
    const double me = i < nx - 1 ? T.m(j, i + 1) : 0.0;
    const double hc = T.at(k, j, i);
    const double hm1 = i > 0 ? mw * T.at(k, j, i - 1) + (1.0 - mw) * hc : hc;
    const double hp1 = i < nx - 1 ? me * T.at(k, j, i + 1) + (1.0 - me) * hc : hc;
    double s = 0.5 * (hp1 - hm1);
    const double dmx = pmax(pmax(hp1, hm1), hc) - hc;
    const double dmn = hc - pmin(pmin(hp1, hm1), hc);
    const double a = pmin(fabs(s), 2.0 * pmin(dmx, dmn));
    s = s > 0.0 ? a : (s < 0.0 ? -a : 0.0);
    return mw * me * m > 0.0 ? s : 0.0;
}

// ale.py:582-626: edge values of cell (k, j, i); the neighbours' slopes are recomputed from h, not stored.
__global__ void __launch_bounds__(128) ppm_edges_kernel(Thick T, int n, int ny, double h_min, double* __restrict__ h_w,
                                                        double* __restrict__ h_e)
{
    const int nx = T.nx;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= nx) return;
    const double mw = i > 0 ? T.m(j, i - 1) : 0.0;
    const double me = i < nx - 1 ? T.m(j, i + 1) : 0.0;
    const double hc = T.at(k, j, i);
    const double hm1 = i > 0 ? mw * T.at(k, j, i - 1) + (1.0 - mw) * hc : hc;
    const double hp1 = i < nx - 1 ? me * T.at(k, j, i + 1) + (1.0 - me) * hc : hc;
    const double sc_ = ppm_slope(T, k, j, i);
    const double sw = i > 0 ? ppm_slope(T, k, j, i - 1) : 0.0;
    const double se = i < nx - 1 ? ppm_slope(T, k, j, i + 1) : 0.0;
    const double hw = 0.5 * (hm1 + hc) + (sw - sc_) / 6.0;
    const double he = 0.5 * (hp1 + hc) + (sc_ - se) / 6.0;
    const double curv = 3.0 * ((hw + he) - 2.0 * hc);
    const double dh = he - hw;
    const bool inside = curv > 0.0 && fabs(dh) < curv;
    const int o = k * T.pc + j * nx + i;
    if (inside && hc <= h_min) {
        h_w[o] = hc;
        h_e[o] = hc;
        return;
    }
    double sc = 1.0;
    if (inside) {
        const double num = 12.0 * curv * (hc - h_min);
        const double den = curv * curv + 3.0 * dh * dh;
        if (num < den) sc = num / den;
    }
    h_w[o] = hc + sc * (hw - hc);
    h_e[o] = hc + sc * (he - hc);
}

struct PPMArgs {
    Thick T;
    const double* __restrict__ h_w;
    const double* __restrict__ h_e;
    const double* __restrict__ ut;
    const double* __restrict__ L;
    const double* __restrict__ Q_bt;
    const double* __restrict__ q_e;
    const double* __restrict__ q_w;
    const double* __restrict__ dx;
    double dt;
    int n, ny, nx;
    double* du;
    double* lo;
    double* hi;
    double* err;
    double* dsum;
    int* unconverged;      // per iteration: faces left unconverged (max_iter + 1 counters, zeroed)
};

// ale.py:629-647 `_face_flux` for layer k of a face at velocity u, with the face's metrics and masks given once
// and both cells' values loaded before the upwind choice, so a layer's loads do not wait for its velocity (the
// per-layer chains of a Newton step are load-latency bound: 15 % faster than loading the upwind side after the
// test, at 512 x 512 x 50).
struct FaceCells {
    double dxw, dxe;
    bool aw, ae;
    int cw, ce;          // cell offsets (j, iw), (j, ie) in a plane
};

__device__ __forceinline__ FaceCells face_cells(const PPMArgs& a, int j, int f)
{
    const int nx = a.nx;
    const int iw = f > 0 ? f - 1 : 0, ie = f < nx ? f : nx - 1;
    FaceCells c;
    c.cw = j * nx + iw;
    c.ce = j * nx + ie;
    c.dxw = __ldg(a.dx + c.cw);
    c.dxe = __ldg(a.dx + c.ce);
    c.aw = __ldg(a.T.act + c.cw) != 0;
    c.ae = __ldg(a.T.act + c.ce) != 0;
    return c;
}

__device__ __forceinline__ void face_flux(const PPMArgs& a, const FaceCells& fc, int k, int of, double u, double L_f,
                                          double& F, double& dF)
{
    const int pf = a.ny * (a.nx + 1);
    const int ow = k * a.T.pc + fc.cw, oe = k * a.T.pc + fc.ce;
    const double hw_ = fc.aw ? nan_to_num(__ldg(a.T.h + ow)) : 0.0, he_ = fc.ae ? nan_to_num(__ldg(a.T.h + oe)) : 0.0;
    const double wwW = __ldg(a.h_w + ow), eeW = __ldg(a.h_e + ow), wwE = __ldg(a.h_w + oe), eeE = __ldg(a.h_e + oe);
    const double qE = __ldg(a.q_e + k * pf + of), qW = __ldg(a.q_w + k * pf + of);
    double c, hu, curv3, dh, edge, q;
    if (u >= 0.0) {
        c = pmin(fabs(u) * a.dt / fc.dxw, 1.0);
        hu = hw_; curv3 = (wwW + eeW) - 2.0 * hu; dh = wwW - eeW; edge = eeW; q = qE;
    } else {
        c = pmin(fabs(u) * a.dt / fc.dxe, 1.0);
        hu = he_; curv3 = (wwE + eeE) - 2.0 * hu; dh = eeE - wwE; edge = wwE; q = qW;
    }
    double mean = edge + c * (0.5 * dh + curv3 * (c - 1.5));
    double marg = edge + c * (dh + 3.0 * curv3 * (c - 1.0));
    if (q < hu) {
        mean = pmin(mean, q);
        marg = pmin(marg, q);
    }
    F = L_f * u * pmax(mean, 0.0);
    dF = L_f * pmax(marg, 0.0);
}

__device__ __forceinline__ bool face_open(const PPMArgs& a, int j, int f)
{
    const int iw = f > 0 ? f - 1 : 0, ie = f < a.nx ? f : a.nx - 1;
    return __ldg(a.T.act + (j * a.nx + iw)) && __ldg(a.T.act + (j * a.nx + ie));
}

// Sum over the layers of (F, dF) at velocities ut + du (shift) or ut itself (the first evaluation, as the reference
// passes ut unchanged there: ut + 0.0 would turn a -0.0 velocity into +0.0).
__device__ __forceinline__ void column_flux(const PPMArgs& a, int j, int f, double du, bool shift, double& s,
                                            double& sd)
{
    const int pf = a.ny * (a.nx + 1), o = j * (a.nx + 1) + f;
    const double L_f = __ldg(a.L + o);
    s = 0.0;
    sd = 0.0;
    if (!face_open(a, j, f)) return;
    const FaceCells fc = face_cells(a, j, f);
    for (int k = 0; k < a.n; ++k) {
        double F, dF;
        const double u = __ldg(a.ut + k * pf + o);
        face_flux(a, fc, k, o, shift ? u + du : u, L_f, F, dF);
        s += F;
        sd += dF;
    }
}

// Register budget of the PPM Newton passes as resident 128-thread CTAs per SM: fitted to 7 (the layer loops are
// load-latency bound; 512 x 512 x 50 u-faces, 20 iterations: 3.98 ms against 5.00 at ptxas's choice of 79-94
// registers, 4.29 at 8, 4.79 at 9, 5.26 at 12).
#ifndef POCEAN_PPM_CTAS
#define POCEAN_PPM_CTAS 7
#endif
#if POCEAN_PPM_CTAS > 0
#define PPM_BOUNDS __launch_bounds__(128, POCEAN_PPM_CTAS)
#else
#define PPM_BOUNDS __launch_bounds__(128)
#endif

// The first pass of _ppm_transport_kernel: bracket, fluxes at du = 0.
__global__ void PPM_BOUNDS ppm_init_kernel(PPMArgs a)
{
    const int nx = a.nx, nf = nx + 1;
    const i64 ot = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (ot >= (i64)a.ny * nf) return;
    const int o = (int)ot, j = o / nf, f = o - j * nf;
    const int iw = f > 0 ? f - 1 : 0, ie = f < nx ? f : nx - 1;
    const int pf = a.ny * nf;
    const double limw = 0.5 * __ldg(a.dx + (j * nx + iw)) / a.dt, lime = 0.5 * __ldg(a.dx + (j * nx + ie)) / a.dt;
    double mnw = INFINITY, mxe = -INFINITY;
    for (int k = 0; k < a.n; ++k) {
        const double u = __ldg(a.ut + k * pf + o);
        mnw = pmin(mnw, limw - u);
        mxe = pmax(mxe, -(lime + u));
    }
    a.hi[o] = pmax(pmin(limw, mnw), 0.0);
    a.lo[o] = pmin(pmax(-lime, mxe), 0.0);
    a.du[o] = 0.0;
    double s, sd;
    column_flux(a, j, f, 0.0, false, s, sd);
    a.err[o] = s - __ldg(a.Q_bt + o);
    a.dsum[o] = sd;
}

// Newton step `it` (0-based) with bracketing bisection; skipped when iteration it-1 left no face unconverged.
__global__ void PPM_BOUNDS ppm_iter_kernel(PPMArgs a, int it)
{
    if (it > 0 && *(volatile int*)(a.unconverged + it - 1) == 0) return;
    const int nf = a.nx + 1;
    const i64 ot = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (ot >= (i64)a.ny * nf) return;
    const int o = (int)ot, j = o / nf, f = o - j * nf;
    const double e = a.err[o], d = a.du[o];
    if (e > 0.0) a.hi[o] = d;
    if (e < 0.0) a.lo[o] = d;
    const double ds = a.dsum[o];
    const double step = ds > 0.0 ? -e / ds : 0.0;
    double nw = d + step;
    if (step > 0.0 && nw >= a.hi[o]) nw = 0.5 * (d + a.hi[o]);
    if (step < 0.0 && nw <= a.lo[o]) nw = 0.5 * (d + a.lo[o]);
    a.du[o] = nw;
    const double q = __ldg(a.Q_bt + o);
    double er = e;
    // a face whose correction did not change (bit for bit) since the iteration that computed its err and dsum at
    // that same correction keeps both: the column sum would give them again (iteration 0 always sums, since the
    // first pass evaluated the layers at ut itself, not at ut + du).  The ALE layer-transport step at 512 x 512 x
    // 50 with the PPM flux: 8.48 against 8.89 ms, the same results bit for bit.
    if (it == 0 || __double_as_longlong(nw) != __double_as_longlong(d)) {
        double s, sd;
        column_flux(a, j, f, nw, true, s, sd);
        er = s - q;
        a.err[o] = er;
        a.dsum[o] = sd;
    }
    if (fabs(er) > 1e-12 * pmax(fabs(q), 1.0)) atomicAdd(a.unconverged + it, 1);
}

// Final fluxes with the converged correction and the residual share (cnuity.F90 style, ale.py:718-740).
__global__ void PPM_BOUNDS ppm_final_kernel(PPMArgs a, double* __restrict__ out)
{
    const int nf = a.nx + 1;
    const i64 ot = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (ot >= (i64)a.ny * nf) return;
    const int o = (int)ot, j = o / nf, f = o - j * nf;
    const int pf = a.ny * nf;
    if (!face_open(a, j, f)) {
        for (int k = 0; k < a.n; ++k) out[k * pf + o] = 0.0;
        return;
    }
    const double du = a.du[o], L_f = __ldg(a.L + o);
    const FaceCells fc = face_cells(a, j, f);
    double s = 0.0;
    for (int k = 0; k < a.n; ++k) {
        double F, dF;
        face_flux(a, fc, k, o, __ldg(a.ut + k * pf + o) + du, L_f, F, dF);
        out[k * pf + o] = F;                   // Fk, completed below
        s += F;
    }
    const double R = __ldg(a.Q_bt + o) - s;
    double te = 0.0, tw = 0.0;
    for (int k = 0; k < a.n; ++k) {
        te += __ldg(a.q_e + k * pf + o);
        tw += __ldg(a.q_w + k * pf + o);
    }
    bool use_e = R >= 0.0;
    double tot = use_e ? te : tw;
    if (tot <= 0.0) {
        use_e = !use_e;
        tot = use_e ? te : tw;
    }
    const double den = tot > 0.0 ? tot : 1.0;
    const double* qs = use_e ? a.q_e : a.q_w;
    for (int k = 0; k < a.n; ++k) out[k * pf + o] = out[k * pf + o] + R * __ldg(qs + k * pf + o) / den;
}

// ---------------------------------------------------------------------------------------------------------------
// Outflow limiter (ale.py:300-441).

struct LimArgs {
    const double* __restrict__ h;
    double* Qx;
    double* Qy;
    const double* __restrict__ area;
    const uint8_t* __restrict__ act;
    double dt, h_floor;
    int n, ny, nx;
    bool per_x, per_y;
    double* room0;
    double* room;
    double* r;
    uint8_t* over;
    double* delta;
    int* flags;            // [0] any over / exceeds, [1] over count, [2] dry donor, [3] spare
};

__device__ __forceinline__ double outflow(const LimArgs& a, int k, int j, int i)
{
    const int nx = a.nx, ny = a.ny;
    const i64 ox = (i64)k * ny * (nx + 1) + (i64)j * (nx + 1) + i, oy = (i64)k * (ny + 1) * nx + (i64)j * nx + i;
    return pmax(a.Qx[ox + 1], 0.0) - pmin(a.Qx[ox], 0.0) + pmax(a.Qy[oy + nx], 0.0) - pmin(a.Qy[oy], 0.0);
}

__device__ __forceinline__ bool cell_of(i64 t, const LimArgs& a, int& k, int& j, int& i)
{
    const i64 pc = (i64)a.ny * a.nx;
    if (t >= (i64)a.n * pc) return false;
    k = (int)(t / pc);
    const i64 c = t - (i64)k * pc;
    j = (int)(c / a.nx);
    i = (int)(c - (i64)j * a.nx);
    return true;
}

// _exceeds_kernel: does any active cell-layer lose more than it holds?
__global__ void __launch_bounds__(256) exceeds_kernel(LimArgs a)
{
    int k, j, i;
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (!cell_of(t, a, k, j, i)) return;
    const i64 c = (i64)j * a.nx + i;
    if (!__ldg(a.act + c)) return;
    if (outflow(a, k, j, i) > pmax(__ldg(a.h + t) - a.h_floor, 0.0) * __ldg(a.area + c) / a.dt) a.flags[0] = 1;
}

// room0 and the first `over` (pass == 0), or the end-of-pass `over` with the 1e-12 tolerance.
__global__ void __launch_bounds__(256) over_kernel(LimArgs a, int first)
{
    int k, j, i;
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (!cell_of(t, a, k, j, i)) return;
    const i64 c = (i64)j * a.nx + i;
    const bool ac = __ldg(a.act + c) != 0;
    if (first) {
        const double A = ac ? __ldg(a.area + c) : 0.0;
        a.room0[t] = pmax(__ldg(a.h + t) - a.h_floor, 0.0) * A / a.dt;
    }
    const double O = outflow(a, k, j, i);
    const bool ov = ac && (first ? O > a.room0[t] : O > a.room0[t] * (1.0 + 1e-12));
    a.over[t] = ov;
    if (ov) a.flags[0] = 1;
}

// r = room0 / O on the cells over the limit (1 elsewhere), and their count.
__global__ void __launch_bounds__(256) ratio_kernel(LimArgs a)
{
    int k, j, i;
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (!cell_of(t, a, k, j, i)) return;
    const double O = outflow(a, k, j, i);
    const bool ov = a.over[t] != 0;
    a.r[t] = ov ? a.room0[t] / (O > 0 ? O : 1.0) : 1.0;
    if (ov) atomicAdd(a.flags + 1, 1);
}

__global__ void __launch_bounds__(256) room_kernel(LimArgs a)
{
    int k, j, i;
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (!cell_of(t, a, k, j, i)) return;
    a.room[t] = a.room0[t] - outflow(a, k, j, i);
}

// Face column geometry of axis ax (0: x faces (j, f), f = 0 .. nx; 1: y faces (f, i), f = 0 .. ny).
struct FaceCol {
    i64 q;          // offset of layer 0 of the face in Q
    i64 sq;         // layer stride of Q
    i64 clo, chi;   // donor cells (row-major (j, i)) on the low / high side
    bool lo_ok, hi_ok;
};

__device__ __forceinline__ bool face_col(const LimArgs& a, int ax, i64 t, FaceCol& fc)
{
    const int nx = a.nx, ny = a.ny;
    if (ax == 0) {
        const int nf = nx + 1;
        if (t >= (i64)ny * nf) return false;
        const int j = (int)(t / nf), f = (int)(t - (i64)j * nf);
        const int lo = f > 0 ? f - 1 : (a.per_x ? nx - 1 : -1), hi = f < nx ? f : (a.per_x ? 0 : -1);
        fc.q = t;
        fc.sq = (i64)ny * nf;
        fc.lo_ok = lo >= 0;
        fc.hi_ok = hi >= 0;
        fc.clo = (i64)j * nx + (lo >= 0 ? lo : 0);
        fc.chi = (i64)j * nx + (hi >= 0 ? hi : 0);
    } else {
        if (t >= (i64)(ny + 1) * nx) return false;
        const int f = (int)(t / nx), i = (int)(t - (i64)f * nx);
        const int lo = f > 0 ? f - 1 : (a.per_y ? ny - 1 : -1), hi = f < ny ? f : (a.per_y ? 0 : -1);
        fc.q = t;
        fc.sq = (i64)(ny + 1) * nx;
        fc.lo_ok = lo >= 0;
        fc.hi_ok = hi >= 0;
        fc.clo = (i64)(lo >= 0 ? lo : 0) * nx + i;
        fc.chi = (i64)(hi >= 0 ? hi : 0) * nx + i;
    }
    return true;
}

// Scale the outgoing flux of every face by the donor's ratio; delta = the net cut of the face column.
__global__ void __launch_bounds__(256) cut_kernel(LimArgs a, int ax)
{
    FaceCol fc;
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (!face_col(a, ax, t, fc)) return;
    double* Q = ax == 0 ? a.Qx : a.Qy;
    const i64 pc = (i64)a.ny * a.nx;
    double d = 0.0;
    for (int k = 0; k < a.n; ++k) {
        const double rlo = fc.lo_ok ? a.r[k * pc + fc.clo] : 1.0, rhi = fc.hi_ok ? a.r[k * pc + fc.chi] : 1.0;
        const double q = Q[fc.q + k * fc.sq];
        const double nw = q > 0 ? q * rlo : (q < 0 ? q * rhi : q);
        d += q - nw;
        Q[fc.q + k * fc.sq] = nw;
    }
    a.delta[t] = d;
}

// _give_back for one face column (ale.py:398-441).
__global__ void __launch_bounds__(256) give_back_kernel(LimArgs a, int ax)
{
    FaceCol fc;
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (!face_col(a, ax, t, fc)) return;
    double* Q = (ax == 0 ? a.Qx : a.Qy) + fc.q;
    const i64 sq = fc.sq, pc = (i64)a.ny * a.nx;
    const int n = a.n;
    const double delta = a.delta[t];
    const double s = sgn(delta);
    auto rooms = [&](int k, double& rl, double& rh) {
        rl = pmax(fc.lo_ok ? a.room[k * pc + fc.clo] : 0.0, 0.0);
        rh = pmax(fc.hi_ok ? a.room[k * pc + fc.chi] : 0.0, 0.0);
    };
    double tot = 0.0;
    for (int k = 0; k < n; ++k) {
        double rl, rh;
        rooms(k, rl, rh);
        const double q = Q[k * sq];
        const bool same = sgn(q) == s && q != 0.0 && s != 0.0;
        tot += same ? (s > 0 ? rl : rh) : 0.0;
    }
    const double need = fabs(delta);
    const double give = need < tot ? need : tot;
    const double X = tot > 0 ? give / (tot > 0 ? tot : 1.0) : 0.0;
    for (int k = 0; k < n; ++k) {
        double rl, rh;
        rooms(k, rl, rh);
        const double q = Q[k * sq];
        const bool same = sgn(q) == s && q != 0.0 && s != 0.0;
        const double rm = same ? (s > 0 ? rl : rh) : 0.0;
        Q[k * sq] = q + s * rm * X;
    }
    double rest = need - give;
    double cap = 0.0;
    for (int k = 0; k < n; ++k) {
        const double q = Q[k * sq];
        cap += (sgn(q) == -s && s != 0.0) ? fabs(q) : 0.0;
    }
    const double mrc = rest < cap ? rest : cap;
    const double frac = cap > 0 ? mrc / (cap > 0 ? cap : 1.0) : 0.0;
    for (int k = 0; k < n; ++k) {
        const double q = Q[k * sq];
        Q[k * sq] = q - ((sgn(q) == -s && s != 0.0) ? q * frac : 0.0);
    }
    rest = rest - mrc;
    const double rp = rest > 0 ? 1.0 : 0.0;
    double ftot = 0.0;
    for (int k = 0; k < n; ++k) {
        const double fl = fc.lo_ok ? a.room0[k * pc + fc.clo] : 0.0, fh = fc.hi_ok ? a.room0[k * pc + fc.chi] : 0.0;
        ftot += (s > 0 ? fl : fh) * rp;
    }
    if (rest > 0 && ftot <= 0) {
        a.flags[2] = 1;
        return;
    }
    const double Y = ftot > 0 ? rest / (ftot > 0 ? ftot : 1.0) : 0.0;
    for (int k = 0; k < n; ++k) {
        const double fl = fc.lo_ok ? a.room0[k * pc + fc.clo] : 0.0, fh = fc.hi_ok ? a.room0[k * pc + fc.chi] : 0.0;
        Q[k * sq] = Q[k * sq] + s * ((s > 0 ? fl : fh) * rp) * Y;
    }
}

// After max_pass passes: the smallest h-dagger (ale.py:385-387), as an ordered bit pattern for atomicMin.
__device__ __forceinline__ unsigned long long ordered(double x)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void __launch_bounds__(256) hdag_min_kernel(LimArgs a, unsigned long long* mn)
{
    int k, j, i;
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (!cell_of(t, a, k, j, i)) return;
    const int nx = a.nx, ny = a.ny;
    const i64 c = (i64)j * nx + i;
    const i64 ox = (i64)k * ny * (nx + 1) + (i64)j * (nx + 1) + i, oy = (i64)k * (ny + 1) * nx + (i64)j * nx + i;
    const double div = a.Qx[ox + 1] - a.Qx[ox] + a.Qy[oy + nx] - a.Qy[oy];
    const bool ac = __ldg(a.act + c) != 0;
    const double A = ac ? __ldg(a.area + c) : 0.0;
    const double hd = ac ? __ldg(a.h + t) - a.dt * div / (A > 0 ? A : 1.0) : 0.0;
    atomicMin(mn, ordered(hd));
}

// ale.py:278-294 `lagrangian_thickness`; the flat index of the first cell-layer below -tol goes to *bad.
__global__ void __launch_bounds__(256) lagrangian_kernel(const double* __restrict__ h, const double* __restrict__ divq,
                                                         const double* __restrict__ area, i64 pc, i64 total, double dt,
                                                         double tol, double* __restrict__ out,
                                                         unsigned long long* __restrict__ bad)
{
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const double A = __ldg(area + t % pc);
    const double v = __ldg(h + t) - dt * __ldg(divq + t) / (A > 0 ? A : 1.0);
    if (v < -tol) atomicMin(bad, (unsigned long long)t);
    out[t] = (v > 0.0 || isnan(v)) ? v : 0.0;                         // numpy.maximum(v, 0.0): +0.0 for v = -0.0
}

// ale.py:233-251 `upwind_transport_x`: one face column (numpy semantics: sums over k from 0.0 in layer order).
__global__ void __launch_bounds__(128) upwind_kernel(const double* __restrict__ q_e, const double* __restrict__ q_w,
                                                     const double* __restrict__ ut, const double* __restrict__ L,
                                                     const double* __restrict__ Q_bt, int n, i64 pf,
                                                     double* __restrict__ out)
{
    const i64 o = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= pf) return;
    const double Lo = __ldg(L + o);
    double S = 0.0;
    for (int k = 0; k < n; ++k) {
        const i64 x = k * pf + o;
        const double u = __ldg(ut + x);
        const double F = (Lo * u) * (u >= 0 ? __ldg(q_e + x) : __ldg(q_w + x));
        out[x] = F;
        S += F;
    }
    const double R = __ldg(Q_bt + o) - S;
    const bool pos = R >= 0;
    double sq = 0.0;
    for (int k = 0; k < n; ++k) sq += pos ? __ldg(q_e + k * pf + o) : __ldg(q_w + k * pf + o);
    const bool use_e = sq > 0 ? pos : !pos;                          // the other side if this column is empty
    const double* q = use_e ? q_e : q_w;
    double tot = 0.0;
    for (int k = 0; k < n; ++k) tot += __ldg(q + k * pf + o);
    const double den = tot > 0 ? tot : 1.0;
    for (int k = 0; k < n; ++k) {
        const i64 x = k * pf + o;
        out[x] = out[x] + R * __ldg(q + x) / den;
    }
}

__device__ __forceinline__ double np_min(double a, double b) { return (a < b || isnan(a)) ? a : b; }
__device__ __forceinline__ double np_max(double a, double b) { return (a > b || isnan(a)) ? a : b; }

// core/components/freshwater.py:31-58 `freshwater_volumes`: one column per thread.
__global__ void __launch_bounds__(128) freshwater_kernel(const double* __restrict__ V, const double* __restrict__ dV,
                                                         const double* __restrict__ floor_arr, double floor_value,
                                                         int n, i64 pc, double* __restrict__ out,
                                                         int* __restrict__ n_limited)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= pc) return;
    const double d = __ldg(dV + c);
    const double fl = floor_arr ? __ldg(floor_arr + c) : floor_value;
    const i64 top = (i64)(n - 1) * pc + c;
    const double vtop = __ldg(V + top);
    const double top_new = vtop + d;
    if (!(d < 0 && top_new < fl)) {
        for (int k = 0; k < n - 1; ++k) out[k * pc + c] = __ldg(V + k * pc + c);
        out[top] = top_new;
        return;
    }
    if (n_limited) atomicAdd(n_limited, 1);
    double deficit = -d;
    for (int k = n - 1; k >= 0; --k) {                               // first keep the floor
        const double col = __ldg(V + k * pc + c);
        const double take = np_min(deficit, np_max(col - fl, 0.0));
        out[k * pc + c] = col - take;
        deficit = deficit - take;
    }
    for (int k = n - 1; k >= 0; --k) {                               // then down to zero
        const double col = out[k * pc + c];
        const double take = np_min(deficit, np_max(col - 0.0, 0.0));
        out[k * pc + c] = col - take;
        deficit = deficit - take;
    }
}

// div Q of each cell-layer: Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:, :] - Qy[:, :-1, :] (layer_transport.py:146).
__global__ void __launch_bounds__(256) divergence_kernel(const double* __restrict__ Qx, const double* __restrict__ Qy,
                                                         int ny, int nx, i64 total, double* __restrict__ out)
{
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const i64 pc = (i64)ny * nx;
    const int k = (int)(t / pc);
    const i64 c = t - k * pc;
    const int j = (int)(c / nx), i = (int)(c - (i64)j * nx);
    const i64 ox = ((i64)k * ny + j) * (nx + 1) + i, oy = ((i64)k * (ny + 1) + j) * nx + i;
    out[t] = __ldg(Qx + ox + 1) - __ldg(Qx + ox) + __ldg(Qy + oy + nx) - __ldg(Qy + oy);
}

// Layer volumes h A of the ALE coordinate (sigma_baroclinic.py:1812-1815) and ok = active & V > 0.
__global__ void __launch_bounds__(256) volumes_kernel(const double* __restrict__ h, const double* __restrict__ area,
                                                      const uint8_t* __restrict__ active, i64 pc, i64 total,
                                                      double* __restrict__ V, uint8_t* __restrict__ ok)
{
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const i64 c = t % pc;
    const double v = __ldg(h + t) * __ldg(area + c);
    V[t] = v;
    if (ok) ok[t] = __ldg(active + c) != 0 && v > 0.0;
}

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace pr
}  // namespace po

using namespace po;

extern "C" int pocean_face_transport_thickness_f64(const double* h, const double* H, const uint8_t* active, int nz,
                                                   int ny, int nx, int clip, double* q_e, double* q_w, void* stream)
{
    const char* fn = "pocean_face_transport_thickness_f64";
    if (nz < 1 || ny < 1 || nx < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (!h || !H || !active || !q_e || !q_w) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    const i64 faces = (i64)ny * (nx + 1);
    pr::ftt_kernel<<<(unsigned)((faces + 127) / 128), 128, 0, (cudaStream_t)stream>>>(h, H, active, nz, ny, nx,
                                                                                      clip != 0, q_e, q_w);
    return pocean_check_launch(fn);
}

extern "C" int pocean_transport_velocity_f64(const double* u_new, const double* u_old, const uint8_t* last_wet,
                                             const double* w, const double* L, const double* D, int nz, int na,
                                             int nb, double theta, double theta_bc, double* ut, double* Qb,
                                             void* stream)
{
    const char* fn = "pocean_transport_velocity_f64";
    if (nz < 1 || na < 1 || nb < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (!u_new || !u_old || !last_wet || !w || !L || !D || !ut || !Qb)
        return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    const i64 plane = (i64)na * nb;
    pr::transport_velocity_kernel<<<(unsigned)((plane + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        u_new, u_old, last_wet, w, L, D, nz, plane, theta, theta_bc, ut, Qb);
    return pocean_check_launch(fn);
}

static int ppm_sizes(const char* fn, int nz, int ny, int nx)
{
    if (nz < 1 || ny < 1 || nx < 1 || ny > 65535 || nz > 65535)
        return pocean_fail(POCEAN_EINVAL, "%s: bad sizes nz=%d ny=%d nx=%d", fn, nz, ny, nx);
    if ((i64)nz * (ny + 1) * (nx + 1) >= (1ll << 31))
        return pocean_fail(POCEAN_EINVAL, "%s: nz=%d ny=%d nx=%d exceeds 2^31 entries per field", fn, nz, ny, nx);
    return POCEAN_OK;
}

extern "C" int pocean_ppm_edges_f64(const double* h, const uint8_t* active, int nz, int ny, int nx, double h_min,
                                    double* h_w, double* h_e, void* stream)
{
    const char* fn = "pocean_ppm_edges_f64";
    int rc = ppm_sizes(fn, nz, ny, nx);
    if (rc) return rc;
    if (!h || !active || !h_w || !h_e) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    rc = pocean_check_device();
    if (rc) return rc;
    const pr::Thick T{h, active, ny * nx, nx};
    pr::ppm_edges_kernel<<<dim3((unsigned)((nx + 127) / 128), ny, nz), 128, 0, (cudaStream_t)stream>>>(T, nz, ny, h_min,
                                                                                                      h_w, h_e);
    return pocean_check_launch(fn);
}

extern "C" size_t pocean_ppm_transport_workspace_bytes(int nz, int ny, int nx, int max_iter)
{
    if (nz < 1 || ny < 1 || nx < 1 || max_iter < 0) return 0;
    const size_t cells = (size_t)nz * ny * nx * sizeof(double), faces = (size_t)ny * (nx + 1) * sizeof(double);
    return 2 * pr::align256(cells) + 5 * pr::align256(faces) + pr::align256((size_t)(max_iter + 1) * sizeof(int));
}

extern "C" int pocean_ppm_transport_f64(const double* h, const double* ut, const double* L, const double* Q_bt,
                                        const double* q_e, const double* q_w, const uint8_t* active, const double* dx,
                                        int nz, int ny, int nx, double dt, int max_iter, double* Qx, void* workspace,
                                        size_t workspace_bytes, void* stream)
{
    const char* fn = "pocean_ppm_transport_f64";
    int rc = ppm_sizes(fn, nz, ny, nx);
    if (rc) return rc;
    if (max_iter < 0 || max_iter > 1000) return pocean_fail(POCEAN_EINVAL, "%s: max_iter=%d", fn, max_iter);
    if (!h || !ut || !L || !Q_bt || !q_e || !q_w || !active || !dx || !Qx)
        return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    const size_t need = pocean_ppm_transport_workspace_bytes(nz, ny, nx, max_iter);
    if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255))
        return pocean_fail(POCEAN_EWORKSPACE, "%s: workspace of %zu bytes (256-byte aligned) needed", fn, need);
    rc = pocean_check_device();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    char* w = (char*)workspace;
    const size_t cells = pr::align256((size_t)nz * ny * nx * sizeof(double));
    const size_t faces = pr::align256((size_t)ny * (nx + 1) * sizeof(double));
    pr::PPMArgs a;
    a.T = pr::Thick{h, active, ny * nx, nx};
    double* h_w = (double*)w; w += cells;
    double* h_e = (double*)w; w += cells;
    a.h_w = h_w; a.h_e = h_e;
    a.du = (double*)w; w += faces;
    a.lo = (double*)w; w += faces;
    a.hi = (double*)w; w += faces;
    a.err = (double*)w; w += faces;
    a.dsum = (double*)w; w += faces;
    a.unconverged = (int*)w;
    a.ut = ut; a.L = L; a.Q_bt = Q_bt; a.q_e = q_e; a.q_w = q_w; a.dx = dx;
    a.dt = dt; a.n = nz; a.ny = ny; a.nx = nx;
    cudaError_t e = cudaMemsetAsync(a.unconverged, 0, (size_t)(max_iter + 1) * sizeof(int), st);
    if (e != cudaSuccess) return pocean_fail(POCEAN_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
    pr::ppm_edges_kernel<<<dim3((unsigned)((nx + 127) / 128), ny, nz), 128, 0, st>>>(a.T, nz, ny, 2e-10, h_w, h_e);
    const i64 nfaces = (i64)ny * (nx + 1);
    const unsigned g = (unsigned)((nfaces + 127) / 128);
    pr::ppm_init_kernel<<<g, 128, 0, st>>>(a);
    for (int it = 0; it < max_iter; ++it) pr::ppm_iter_kernel<<<g, 128, 0, st>>>(a, it);
    pr::ppm_final_kernel<<<g, 128, 0, st>>>(a, Qx);
    return pocean_check_launch(fn);
}

extern "C" size_t pocean_limit_outflow_workspace_bytes(int nz, int ny, int nx)
{
    if (nz < 1 || ny < 1 || nx < 1) return 0;
    const size_t cells = (size_t)nz * ny * nx;
    const size_t fx = (size_t)ny * (nx + 1), fy = (size_t)(ny + 1) * nx;
    return 3 * pr::align256(cells * sizeof(double)) + pr::align256(cells) +
           pr::align256((fx > fy ? fx : fy) * sizeof(double)) + 256 + 256;
}

extern "C" int pocean_limit_outflow_f64(const double* h, double* Qx, double* Qy, const double* area,
                                        const uint8_t* active, int nz, int ny, int nx, double dt, double h_floor,
                                        int max_pass, unsigned flags, int* n_limited, int* warned, void* workspace,
                                        size_t workspace_bytes, void* stream)
{
    const char* fn = "pocean_limit_outflow_f64";
    if (nz < 1 || ny < 1 || nx < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (max_pass < 0) return pocean_fail(POCEAN_EINVAL, "%s: max_pass=%d", fn, max_pass);
    if (flags & ~(unsigned)(POCEAN_PERIODIC_X | POCEAN_PERIODIC_Y))
        return pocean_fail(POCEAN_EINVAL, "%s: only the periodic flags apply (0x%x)", fn, flags);
    if (!h || !Qx || !Qy || !area || !active) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    const size_t need = pocean_limit_outflow_workspace_bytes(nz, ny, nx);
    if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255))
        return pocean_fail(POCEAN_EWORKSPACE, "%s: workspace of %zu bytes (256-byte aligned) needed", fn, need);
    int rc = pocean_check_device();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t cells = (size_t)nz * ny * nx;
    const size_t fx = (size_t)ny * (nx + 1), fy = (size_t)(ny + 1) * nx;
    char* w = (char*)workspace;
    pr::LimArgs a;
    a.h = h; a.Qx = Qx; a.Qy = Qy; a.area = area; a.act = active; a.dt = dt; a.h_floor = h_floor;
    a.n = nz; a.ny = ny; a.nx = nx;
    a.per_x = (flags & POCEAN_PERIODIC_X) != 0;
    a.per_y = (flags & POCEAN_PERIODIC_Y) != 0;
    a.room0 = (double*)w; w += pr::align256(cells * sizeof(double));
    a.room = (double*)w; w += pr::align256(cells * sizeof(double));
    a.r = (double*)w; w += pr::align256(cells * sizeof(double));
    a.over = (uint8_t*)w; w += pr::align256(cells);
    a.delta = (double*)w; w += pr::align256((fx > fy ? fx : fy) * sizeof(double));
    a.flags = (int*)w; w += 256;
    unsigned long long* mn = (unsigned long long*)w;
    int hflags[4];
    auto fetch = [&]() -> int {
        cudaError_t e = cudaMemcpyAsync(hflags, a.flags, sizeof(hflags), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return pocean_fail(POCEAN_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
        return POCEAN_OK;
    };
    const unsigned gc = (unsigned)((cells + 255) / 256);
    const unsigned gx = (unsigned)((fx + 255) / 256), gy = (unsigned)((fy + 255) / 256);
    if (n_limited) *n_limited = 0;
    if (warned) *warned = 0;
    cudaError_t e = cudaMemsetAsync(a.flags, 0, 4 * sizeof(int), st);
    if (e != cudaSuccess) return pocean_fail(POCEAN_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
    pr::exceeds_kernel<<<gc, 256, 0, st>>>(a);
    if ((rc = pocean_check_launch(fn)) || (rc = fetch())) return rc;
    if (!hflags[0]) return POCEAN_OK;                                   // the common case: nothing to limit
    cudaMemsetAsync(a.flags, 0, 4 * sizeof(int), st);
    pr::over_kernel<<<gc, 256, 0, st>>>(a, 1);
    for (int pass = 0; pass < max_pass; ++pass) {
        cudaMemsetAsync(a.flags, 0, sizeof(int), st);                   // any-over of this pass (count accumulates)
        pr::ratio_kernel<<<gc, 256, 0, st>>>(a);
        for (int ax = 0; ax < 2; ++ax) {
            pr::cut_kernel<<<ax == 0 ? gx : gy, 256, 0, st>>>(a, ax);
            pr::room_kernel<<<gc, 256, 0, st>>>(a);
            pr::give_back_kernel<<<ax == 0 ? gx : gy, 256, 0, st>>>(a, ax);
        }
        pr::over_kernel<<<gc, 256, 0, st>>>(a, 0);
        if ((rc = pocean_check_launch(fn)) || (rc = fetch())) return rc;
        if (n_limited) *n_limited = hflags[1];
        if (hflags[2])
            return pocean_fail(POCEAN_ESTEP, "%s: a face must carry flow out of a donor column that holds no water "
                               "(barotropic CFL, or the flow has already blown up)", fn);
        if (!hflags[0]) return POCEAN_OK;
    }
    // still over after max_pass: accepted if h-dagger stays >= -h_floor (the reference warns), else it raises
    e = cudaMemsetAsync(mn, 0xFF, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return pocean_fail(POCEAN_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
    pr::hdag_min_kernel<<<gc, 256, 0, st>>>(a, mn);
    unsigned long long hm = 0;
    e = cudaMemcpyAsync(&hm, mn, sizeof(hm), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return pocean_fail(POCEAN_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
    const unsigned long long bits = (hm >> 63) ? (hm & 0x7FFFFFFFFFFFFFFFull) : ~hm;
    double hmin;
    memcpy(&hmin, &bits, sizeof(hmin));
    if (hmin >= -h_floor) {
        if (warned) *warned = 1;
        return POCEAN_OK;
    }
    return pocean_fail(POCEAN_ESTEP, "%s: a layer would reach h = %.3g m after %d passes: the column cannot supply "
                       "the free-surface flux (barotropic CFL)", fn, hmin, max_pass);
}

extern "C" int pocean_lagrangian_thickness_f64(const double* h, const double* divq, const double* area, int nz,
                                               int ny, int nx, double dt, double tol, double* h_dag,
                                               unsigned long long* first_bad, void* stream)
{
    const char* fn = "pocean_lagrangian_thickness_f64";
    if (nz < 1 || ny < 1 || nx < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (!h || !divq || !area || !h_dag || !first_bad) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(first_bad, 0xFF, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return pocean_fail(POCEAN_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
    const i64 pc = (i64)ny * nx, total = pc * nz;
    pr::lagrangian_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(h, divq, area, pc, total, dt, tol, h_dag,
                                                                            first_bad);
    return pocean_check_launch(fn);
}

extern "C" int pocean_upwind_transport_f64(const double* q_e, const double* q_w, const double* ut, const double* L,
                                           const double* Q_bt, int nz, int a, int b, double* Q, void* stream)
{
    const char* fn = "pocean_upwind_transport_f64";
    if (nz < 1 || a < 1 || b < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (!q_e || !q_w || !ut || !L || !Q_bt || !Q) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    const i64 pf = (i64)a * b;
    pr::upwind_kernel<<<(unsigned)((pf + 127) / 128), 128, 0, (cudaStream_t)stream>>>(q_e, q_w, ut, L, Q_bt, nz, pf,
                                                                                        Q);
    return pocean_check_launch(fn);
}

extern "C" int pocean_freshwater_volumes_f64(const double* V, const double* dV, const double* floor_,
                                             double floor_value, int nz, int ny, int nx, double* V_new,
                                             int* n_limited, void* stream)
{
    const char* fn = "pocean_freshwater_volumes_f64";
    if (nz < 1 || ny < 1 || nx < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (!V || !dV || !V_new) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    if (V_new == V) return pocean_fail(POCEAN_EINVAL, "%s: V_new must not alias V", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    const i64 pc = (i64)ny * nx;
    pr::freshwater_kernel<<<(unsigned)((pc + 127) / 128), 128, 0, (cudaStream_t)stream>>>(V, dV, floor_, floor_value,
                                                                                           nz, pc, V_new, n_limited);
    return pocean_check_launch(fn);
}

extern "C" int pocean_flux_divergence_f64(const double* Qx, const double* Qy, int nz, int ny, int nx, double* divq,
                                          void* stream)
{
    const char* fn = "pocean_flux_divergence_f64";
    if (nz < 1 || ny < 1 || nx < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (!Qx || !Qy || !divq) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    const i64 total = (i64)nz * ny * nx;
    pr::divergence_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(Qx, Qy, ny, nx, total,
                                                                                              divq);
    return pocean_check_launch(fn);
}

extern "C" int pocean_layer_volumes_f64(const double* h, const double* area, const uint8_t* active, int nz, int ny,
                                        int nx, double* V, uint8_t* ok, void* stream)
{
    const char* fn = "pocean_layer_volumes_f64";
    if (nz < 1 || ny < 1 || nx < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes", fn);
    if (!h || !area || !V || (ok && !active)) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    const i64 pc = (i64)ny * nx, total = (i64)nz * pc;
    pr::volumes_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(h, area, active, pc, total,
                                                                                           V, ok);
    return pocean_check_launch(fn);
}

// ---------------------------------------------------------------------------------------------------------------
// Periodic halo of a producer's inputs (core/model/periodic.py:72-94 `Periodic.pad` / `crop`).  The reference
// reaches the wrap of its PPM layer flux by running the kernel on inputs extended by `halo` wrapped positions on
// each periodic axis and cropping the result (core/components/layer_transport.py:121-128); these copies give the
// CUDA kernels the same extended inputs, so the fluxes (and the Newton iteration's global stop test, which sees the
// halo faces too) are the reference's bit for bit.
namespace po {
namespace pr {

// dst (nlead, Yd, Xd) from src (nlead, Ys, Xs): position y of dst reads row (y - oy) mod ny of src when `wy` (the
// wrapped axis of ny unique positions), else row y + oy; the same for x.
template <typename T>
__global__ void __launch_bounds__(256) window_kernel(const T* __restrict__ src, int Ys, int Xs, T* __restrict__ dst,
                                                     int Yd, int Xd, i64 total, int oy, int ox, int wy, int wx,
                                                     int ny, int nx)
{
    const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int x = (int)(e % Xd);
    const i64 r = e / Xd;
    const int y = (int)(r % Yd);
    const i64 l = r / Yd;
    const int sy = wy ? wrap(y - oy, ny) : y + oy;
    const int sx = wx ? wrap(x - ox, nx) : x + ox;
    dst[e] = src[(l * Ys + sy) * Xs + sx];
}

}  // namespace pr
}  // namespace po

template <typename T>
static int periodic_window(const char* fn, const T* src, int nlead, int ny, int nx, int face_y, int face_x, int py,
                           int px, int halo, T* dst, bool pad, void* stream)
{
    if (nlead < 1 || ny < 1 || nx < 1 || halo < 0 || (face_y & ~1) || (face_x & ~1))
        return pocean_fail(POCEAN_EINVAL, "%s: bad sizes (nlead=%d ny=%d nx=%d halo=%d)", fn, nlead, ny, nx, halo);
    if (!src || !dst) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    const int Yc = ny + face_y, Xc = nx + face_x;                               // the unpadded array
    const int Yp = py ? ny + 2 * halo + face_y : Yc, Xp = px ? nx + 2 * halo + face_x : Xc;
    const int Ys = pad ? Yc : Yp, Xs = pad ? Xc : Xp, Yd = pad ? Yp : Yc, Xd = pad ? Xp : Xc;
    const i64 total = (i64)nlead * Yd * Xd;
    pr::window_kernel<T><<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        src, Ys, Xs, dst, Yd, Xd, total, py ? halo : 0, px ? halo : 0, pad && py, pad && px, ny, nx);
    return pocean_check_launch(fn);
}

extern "C" int pocean_periodic_pad_f64(const double* src, int nlead, int ny, int nx, int face_y, int face_x, int py,
                                       int px, int halo, double* dst, void* stream)
{
    return periodic_window("pocean_periodic_pad_f64", src, nlead, ny, nx, face_y, face_x, py, px, halo, dst, true,
                           stream);
}

extern "C" int pocean_periodic_pad_u8(const uint8_t* src, int nlead, int ny, int nx, int face_y, int face_x, int py,
                                      int px, int halo, uint8_t* dst, void* stream)
{
    return periodic_window("pocean_periodic_pad_u8", src, nlead, ny, nx, face_y, face_x, py, px, halo, dst, true,
                           stream);
}

extern "C" int pocean_periodic_crop_f64(const double* src, int nlead, int ny, int nx, int face_y, int face_x, int py,
                                        int px, int halo, double* dst, void* stream)
{
    return periodic_window("pocean_periodic_crop_f64", src, nlead, ny, nx, face_y, face_x, py, px, halo, dst, false,
                           stream);
}

// ---------------------------------------------------------------------------------------------------------------
// Layer fluxes through the faces of one open edge (core/vertical/ale.py:841-861 `open_face_transport`, as
// core/components/open_boundary.py:334-352 `open_face_transports` applies it in place where the open face depth
// D > 0): Q_k = w_k Q_bt + L h_k (theta_bc u'_k^new + (1 - theta_bc) u'_k^old), w_k = h_k / sum h, u' = u - sum w u;
// 0 in a column without water.  One thread per face of the edge; the column sums run over k in order, as numpy's
// reduction over the leading axis does.
namespace po {
namespace pr {

__global__ void __launch_bounds__(128) open_face_kernel(const double* __restrict__ h, i64 hk, i64 hm,
                                                        const double* __restrict__ un, const double* __restrict__ uo,
                                                        i64 uk, i64 um, const double* __restrict__ Qbt,
                                                        const double* __restrict__ L, const double* __restrict__ D,
                                                        i64 qm, int n, int m, double tb, double* __restrict__ Q,
                                                        i64 Qk, i64 Qm)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    if (!(D[c * qm] > 0)) return;
    const double* hc = h + c * hm;
    double tot = 0.0;
    for (int k = 0; k < n; ++k) tot += hc[k * hk];
    const bool wet = tot > 0;
    const double dn = wet ? tot : 1.0;
    double sn = 0.0, so = 0.0;
    for (int k = 0; k < n; ++k) {
        const double w = wet ? hc[k * hk] / dn : 0.0;
        sn += w * un[c * um + k * uk];
    }
    for (int k = 0; k < n; ++k) {
        const double w = wet ? hc[k * hk] / dn : 0.0;
        so += w * uo[c * um + k * uk];
    }
    const double qb = Qbt[c * qm], Lc = L[c * qm];
    for (int k = 0; k < n; ++k) {
        const double hk_ = hc[k * hk];
        const double w = wet ? hk_ / dn : 0.0;
        const double pn = un[c * um + k * uk] - sn;
        const double po = uo[c * um + k * uk] - so;
        const double q = w * qb + Lc * hk_ * (tb * pn + (1.0 - tb) * po);
        Q[c * Qm + k * Qk] = wet ? q : 0.0;
    }
}

}  // namespace pr
}  // namespace po

extern "C" int pocean_open_face_transport_f64(const double* h_int, long long h_stride_k, long long h_stride_m,
                                              const double* u_new, const double* u_old, long long u_stride_k,
                                              long long u_stride_m, const double* Q_bt, const double* L,
                                              const double* D, long long col_stride, int n, int m, double theta_bc,
                                              double* Q, long long Q_stride_k, long long Q_stride_m, void* stream)
{
    const char* fn = "pocean_open_face_transport_f64";
    if (n < 1 || m < 1) return pocean_fail(POCEAN_EINVAL, "%s: bad sizes (n=%d m=%d)", fn, n, m);
    if (!h_int || !u_new || !u_old || !Q_bt || !L || !D || !Q) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    pr::open_face_kernel<<<(unsigned)((m + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        h_int, h_stride_k, h_stride_m, u_new, u_old, u_stride_k, u_stride_m, Q_bt, L, D, col_stride, n, m, theta_bc, Q,
        Q_stride_k, Q_stride_m);
    return pocean_check_launch(fn);
}
