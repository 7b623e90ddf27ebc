// FP64 tracer advection on B200: SSP-RK3 WENO5 with Zalesak FCT (TracerAdvection.advect_fct) and without limiter
// (TracerAdvection.advect).
//
// Reference: core/components/tracers.py:208-254, 342-375 and the Numba kernels of
// core/dynamics/sigma_baroclinic.py:265-364 (faces, RHS), 407-530 (FCT), 856-875 (RK stage).
//
// Design.  The reference runs 9 kernels over ~15 full-size temporaries per FCT step.  Here one step is 7 launches:
//   1-5. for RK stages 1 and 2 a face pass and a cell pass, for stage 3 a face pass (fct_split.cuh): one thread per
//        cell computes the west x-face and the south y-face of its cell from global memory (L1 serves the
//        overlapping stencils; no shared memory, no barrier, high occupancy, two independent WENO5 chains per
//        thread), then a streaming pass updates the cells from the stored faces.
//        1: S <- F0;  c1 = safe(q0 - dt div F0, Va).
//        2: T <- F1;  q1 recomputed from F0, c2 = safe(3/4 q0 + 1/4 (q1 - dt div F1), Vb).
//        3: S <- A = ((F0 + F1)/6 + 2 F2/3) - F_L, and c_L = safe(q0 - dt div F_L, V1) from the donor fluxes F_L
//           of the cell's four faces (recomputed, never stored).
//   6. coeff  Zalesak R+ / R- per cell from the 7-point (x, y, k +- 1) bounds of C and c_L (tracers looped per
//             thread: the stencil geometry is read once).
//   7. final  face coefficients from R of both neighbours; C_out = safe(q0 - dt div(F_L + C A), V1).
// The unlimited step (tracers.py:289-291) runs stages 1-2, then a face pass storing the RK3 flux
// F_H = (F0 + F1)/6 + 2 F2/3 and a cell pass C_out = safe(q0 - dt div F_H, V1).
// q0 = V0 C, Va, Vb and q1 are recomputed where needed instead of stored.  Planes run k-major (the tracers of one
// layer follow each other) so a layer's geometry is re-read from L2.  Periodic axes wrap natively in every stencil
// (the reference pads by TRACER_HALO = 13 cells and crops; with the dependency radius of the step, 10 cells, both
// give the same numbers).  Workspace: 3 cell stacks (c1 -> R+, c2 -> R-, c_L) and 4 face stacks (S, T).
// An earlier form marched warps along 31-cell strips with a shared-memory row ring and did each stage in one pass;
// the split form is 14 % faster at 512 x 512 x 50 (the passes are bound by instruction issue and latency, and the
// simple face threads run at twice the occupancy).
//
// Arithmetic: every expression in the reference's order, no FMA contraction (-fmad=false), IEEE division; the
// results equal the reference's FP64 Numba path bit for bit.
#include <cstdio>

#include "common.cuh"
#include "fct_args.cuh"
#include "weno.cuh"

namespace po {

constexpr int TI = 32;          // tile width (i, contiguous in memory)
constexpr int TJ = 8;           // tile height (j)
constexpr int NTHREADS = TI * TJ;

// Launch bounds of the coefficient and final passes; POCEAN_*_CTAS (resident CTAs per SM) sets their register
// budget when defined, else ptxas chooses.  The final pass is fitted to 4 CTAs (32 warps, 64 registers) per SM:
// 1.5 % faster for the step than 3 CTAs, measured at 512 x 512 x 50; the coefficient pass keeps ptxas's choice
// (5 CTAs, which spills, was slower).
#ifndef POCEAN_FINAL_CTAS
#define POCEAN_FINAL_CTAS 4
#endif
#ifdef POCEAN_COEFF_CTAS
#define COEFF_BOUNDS __launch_bounds__(NTHREADS, POCEAN_COEFF_CTAS)
#else
#define COEFF_BOUNDS __launch_bounds__(NTHREADS)
#endif
#ifdef POCEAN_FINAL_CTAS
#define FINAL_BOUNDS __launch_bounds__(NTHREADS, POCEAN_FINAL_CTAS)
#else
#define FINAL_BOUNDS __launch_bounds__(NTHREADS)
#endif
// The batched coefficient and final passes have budgets of their own (the domains of a batch usually carry one
// tracer, so a thread's loop over the tracers runs once).  The batched coefficient pass at 6 CTAs per SM (40
// registers, spilling to L1): the 64-domain batched step 40.92 ms against 42.99 ms at ptxas's choice (68 registers,
// 3 CTAs), 41.14 / 41.16 ms at 4 / 5 CTAs; the batched final pass keeps the single-domain budget (5 CTAs: slower).
#ifndef POCEAN_COEFF_BATCHED_CTAS
#define POCEAN_COEFF_BATCHED_CTAS 6
#endif
#ifdef POCEAN_COEFF_BATCHED_CTAS
#define COEFF_BATCHED_BOUNDS __launch_bounds__(NTHREADS, POCEAN_COEFF_BATCHED_CTAS)
#else
#define COEFF_BATCHED_BOUNDS COEFF_BOUNDS
#endif
#ifdef POCEAN_FINAL_BATCHED_CTAS
#define FINAL_BATCHED_BOUNDS __launch_bounds__(NTHREADS, POCEAN_FINAL_BATCHED_CTAS)
#else
#define FINAL_BATCHED_BOUNDS FINAL_BOUNDS
#endif

// ---------------------------------------------------------------------------------------------------------------
// Donor-cell flux F_L of x-face gf (sigma_baroclinic.py:486-494; periodic: every face interior, face nx = face 0).
__device__ __forceinline__ double donor_x(const double* __restrict__ cp, const double* __restrict__ ep,
                                          const double* __restrict__ Qx, const Shape& s, const Flags& fl, int k,
                                          int j, int f)
{
    const i64 row = (i64)j * s.nx;
    if (fl.per_x) {
        const int ff = f == s.nx ? 0 : f;
        const double q = Qx[s.qx(k, j, ff)];
        return q * (q >= 0 ? cp[row + wrap(ff - 1, s.nx)] : cp[row + ff]);
    }
    const double q = Qx[s.qx(k, j, f)];
    if (f >= 1 && f <= s.nx - 1) return q * (q >= 0 ? cp[row + f - 1] : cp[row + f]);
    if (f == 0) return fl.open_w ? q * (q > 0 ? ep[row] : cp[row]) : 0.0;
    return fl.open_e ? q * (q < 0 ? ep[row + s.nx - 1] : cp[row + s.nx - 1]) : 0.0;
}

__device__ __forceinline__ double donor_y(const double* __restrict__ cp, const double* __restrict__ ep,
                                          const double* __restrict__ Qy, const Shape& s, const Flags& fl, int k,
                                          int f, int i)
{
    if (fl.per_y) {
        const int ff = f == s.ny ? 0 : f;
        const double q = Qy[s.qy(k, ff, i)];
        return q * (q >= 0 ? cp[(i64)wrap(ff - 1, s.ny) * s.nx + i] : cp[(i64)ff * s.nx + i]);
    }
    const double q = Qy[s.qy(k, f, i)];
    if (f >= 1 && f <= s.ny - 1) return q * (q >= 0 ? cp[(i64)(f - 1) * s.nx + i] : cp[(i64)f * s.nx + i]);
    if (f == 0) return fl.open_s ? q * (q > 0 ? ep[i] : cp[i]) : 0.0;
    const i64 o = (i64)(s.ny - 1) * s.nx + i;
    return fl.open_n ? q * (q < 0 ? ep[o] : cp[o]) : 0.0;
}

}  // namespace po

#include "fct_split.cuh"

namespace po {


// Pass 4: Zalesak R+ / R- (sigma_baroclinic.py:407-432): bounds over the cell, its x / y neighbours and the layers
// k +- 1 (ok cells), P from the antidiffusive fluxes of the cell's faces, Q from V1 and c_L.
__device__ __forceinline__ void coeff_body(const StepArgs& a, int i, int j, int k)
{
    const Shape s = a.s;
    const Flags fl(a.flags);
    if (i >= s.nx || j >= s.ny) return;
    const double* cL = a.q1;
    // the 7-point stencil of the bounds: cell, x / y neighbours, layers k -+ 1 (ok cells only); its geometry is
    // the same for every tracer
    const int dk[7] = {0, 0, 0, 0, 0, -1, 1};
    const int dj[7] = {0, 0, 0, -1, 1, 0, 0};
    const int di[7] = {0, -1, 1, 0, 0, 0, 0};
    // 32-bit offsets within a field (every field holds fewer than 2^31 entries)
    const int pl = s.ny * s.nx, gc = k * pl + j * s.nx + i;
    const bool self_ok = a.ok[gc];
    int nb[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) {
        int kk = k + dk[m], jj = j + dj[m], ii = i + di[m];
        bool in = kk >= 0 && kk < s.n;
        if (fl.per_y) jj = wrap(jj, s.ny); else in = in && jj >= 0 && jj < s.ny;
        if (fl.per_x) ii = wrap(ii, s.nx); else in = in && ii >= 0 && ii < s.nx;
        const int o = in ? kk * pl + jj * s.nx + ii : 0;
        nb[m] = (in && a.ok[o]) ? o : -1;
    }
    const double v1 = a.V1[gc];
    const int tstride = s.n * pl;
    for (int t = 0; t < s.nt; ++t) {
        const i64 ci = plane_at(t, tstride) + gc;
        double rin = 0.0, rout = 0.0;
        if (self_ok) {
            // every load of the tracer first (independent, in flight together), then the bounds in stencil order
            double vc[7], vl[7];
#pragma unroll
            for (int m = 0; m < 7; ++m) {
                const i64 o = plane_at(t, tstride) + (nb[m] >= 0 ? nb[m] : nb[0]);
                vc[m] = __ldg(a.C + o);
                vl[m] = cL[o];
            }
            const int p = t * s.n + k;
            const i64 w = plane_at(p, s.ny * (s.nx + 1)) + (j * (s.nx + 1) + i), so = plane_at(p, (s.ny + 1) * s.nx) + (j * s.nx + i);
            const double axw = a.Sx[w], axe = a.Sx[w + 1], ays = a.Sy[so], ayn = a.Sy[so + s.nx];
            double cmax = -INFINITY, cmin = INFINITY;
#pragma unroll
            for (int m = 0; m < 7; ++m) {
                if (nb[m] < 0) continue;
                cmax = pmax(pmax(cmax, vc[m]), vl[m]);
                cmin = pmin(pmin(cmin, vc[m]), vl[m]);
            }
            const double p_in = a.dt * (pmax(axw, 0.0) - pmin(axe, 0.0) + pmax(ays, 0.0) - pmin(ayn, 0.0));
            const double p_out = a.dt * (pmax(axe, 0.0) - pmin(axw, 0.0) + pmax(ayn, 0.0) - pmin(ays, 0.0));
            const double q_in = pmax(v1 * (cmax - cL[ci]), 0.0);
            const double q_out = pmax(v1 * (cL[ci] - cmin), 0.0);
            rin = p_in > 0.0 ? pmin(1.0, q_in / p_in) : 0.0;
            rout = p_out > 0.0 ? pmin(1.0, q_out / p_out) : 0.0;
        }
        a.c1[ci] = rin;            // R+ over c1
        a.c2[ci] = rout;           // R- over c2
    }
}

// Face coefficient C of x-face f of row j (sigma_baroclinic.py:435-442): min(R+ downstream, R- upstream) by the
// sign of A; 0 on the domain edges unless periodic.
__device__ __forceinline__ double coef_x(const StepArgs& a, const Shape& s, const Flags& fl, int t, int k, int j,
                                         int f, double A)
{
    int l = f - 1, r = f;
    if (fl.per_x) { l = wrap(l, s.nx); r = wrap(r, s.nx); }
    else if (f < 1 || f > s.nx - 1) return 0.0;
    const i64 ol = s.cell(t, k, j, l), orr = s.cell(t, k, j, r);
    return A >= 0.0 ? pmin(a.c1[orr], a.c2[ol]) : pmin(a.c1[ol], a.c2[orr]);
}

__device__ __forceinline__ double coef_y(const StepArgs& a, const Shape& s, const Flags& fl, int t, int k, int f,
                                         int i, double A)
{
    int l = f - 1, r = f;
    if (fl.per_y) { l = wrap(l, s.ny); r = wrap(r, s.ny); }
    else if (f < 1 || f > s.ny - 1) return 0.0;
    const i64 ol = s.cell(t, k, l, i), orr = s.cell(t, k, r, i);
    return A >= 0.0 ? pmin(a.c1[orr], a.c2[ol]) : pmin(a.c1[ol], a.c2[orr]);
}

// Pass 5: C_out = safe(q0 - dt div(F_L + C A), V1) (sigma_baroclinic.py:514-530).  One thread per column cell
// (k, j, i) loops over the tracers, so the geometry is read once; every value a tracer needs (C, R+ and R- at the
// cell and its four neighbours, A on the four faces) is loaded before any is used, so the loads of a thread are
// independent and in flight together.

// Effective flux F_L + C A through one face from its preloaded neighbourhood: `interior` faces take the donor value
// and the limited antidiffusive flux; domain-edge faces (closed, or open with the upstream rule) carry no
// antidiffusive part (C = 0 there).
__device__ __forceinline__ double face_flux(bool interior, bool open, bool inflow_side_pos, double q, double A,
                                            double c_l, double c_r, double rin_l, double rin_r, double rout_l,
                                            double rout_r, double ext, double c_edge)
{
    if (interior) {
        const double fl = q * (q >= 0 ? c_l : c_r);
        const double cf = A >= 0.0 ? pmin(rin_r, rout_l) : pmin(rin_l, rout_r);
        return fl + cf * A;
    }
    // edge: inflow when q > 0 on the west/south edge (inflow_side_pos) or q < 0 on the east/north edge
    const double fl = open ? q * ((inflow_side_pos ? q > 0 : q < 0) ? ext : c_edge) : 0.0;
    return fl + 0.0 * A;
}

__device__ __forceinline__ void final_body(const StepArgs& a, int i, int j, int k)
{
    const Shape s = a.s;
    const Flags fl(a.flags);
    if (i >= s.nx || j >= s.ny) return;
    // neighbours (wrapped on periodic axes, -1 outside the domain) and which faces are interior
    const int iw = fl.per_x ? wrap(i - 1, s.nx) : i - 1, ie = fl.per_x ? wrap(i + 1, s.nx) : (i + 1 < s.nx ? i + 1 : -1);
    const int js = fl.per_y ? wrap(j - 1, s.ny) : j - 1, jn = fl.per_y ? wrap(j + 1, s.ny) : (j + 1 < s.ny ? j + 1 : -1);
    const bool in_w = fl.per_x || i >= 1, in_e = fl.per_x || i + 1 <= s.nx - 1;
    const bool in_s = fl.per_y || j >= 1, in_n = fl.per_y || j + 1 <= s.ny - 1;
    // 32-bit offsets within a field (every field holds fewer than 2^31 entries)
    const int pl = s.ny * s.nx, xpl = s.ny * (s.nx + 1), ypl = (s.ny + 1) * s.nx;
    const int g = k * pl + j * s.nx + i, gx = k * xpl + j * (s.nx + 1) + i, gy = k * ypl + j * s.nx + i;
    const double v0 = __ldg(a.V0 + g), v1 = __ldg(a.V1 + g);
    const double qw = __ldg(a.Qx + gx);
    const double qe = __ldg(a.Qx + ((fl.per_x && i + 1 == s.nx) ? gx + 1 - s.nx : gx + 1));
    const double qs = __ldg(a.Qy + gy);
    const double qn = __ldg(a.Qy + ((fl.per_y && j + 1 == s.ny) ? gy - j * s.nx : gy + s.nx));
    const i64 row = (i64)j * s.nx;
    const i64 o_c = row + i, o_w = row + (iw >= 0 ? iw : i), o_e = row + (ie >= 0 ? ie : i);
    const i64 o_s = (i64)(js >= 0 ? js : j) * s.nx + i, o_n = (i64)(jn >= 0 ? jn : j) * s.nx + i;
    for (int t = 0; t < s.nt; ++t) {
        const int p = t * s.n + k;
        const i64 pc = plane_at(p, pl);
        const double* C = a.C + pc;
        const double* Rp = a.c1 + pc;
        const double* Rm = a.c2 + pc;
        const double c0 = __ldg(C + o_c), cw = __ldg(C + o_w), ce = __ldg(C + o_e), cs = __ldg(C + o_s),
                     cn = __ldg(C + o_n);
        const double rp0 = Rp[o_c], rpw = Rp[o_w], rpe = Rp[o_e], rps = Rp[o_s], rpn = Rp[o_n];
        const double rm0 = Rm[o_c], rmw = Rm[o_w], rme = Rm[o_e], rms = Rm[o_s], rmn = Rm[o_n];
        const i64 w = plane_at(p, xpl) + (gx - k * xpl), so = plane_at(p, ypl) + (gy - k * ypl);
        const double aw = a.Sx[w], ae = a.Sx[w + 1], as = a.Sy[so], an = a.Sy[so + s.nx];
        double ext_c = c0;
        if (a.inflow && ((!in_w && fl.open_w) || (!in_e && fl.open_e) || (!in_s && fl.open_s) ||
                         (!in_n && fl.open_n)))
            ext_c = __ldg(a.inflow + pc + o_c);
        const double fw = face_flux(in_w, fl.open_w, true, qw, aw, cw, c0, rpw, rp0, rmw, rm0, ext_c, c0);
        const double fe = face_flux(in_e, fl.open_e, false, qe, ae, c0, ce, rp0, rpe, rm0, rme, ext_c, c0);
        const double fs = face_flux(in_s, fl.open_s, true, qs, as, cs, c0, rps, rp0, rms, rm0, ext_c, c0);
        const double fn = face_flux(in_n, fl.open_n, false, qn, an, c0, cn, rp0, rpn, rm0, rmn, ext_c, c0);
        const double d = fe - fw + fn - fs;
        const double q = v0 * c0 - a.dt * d;
        a.out[pc + o_c] = v1 > 0 ? q / v1 : c0;
    }
}

// Single-domain launches of passes 4 and 5: a 32 x 8 tile of one layer per CTA.
__global__ void COEFF_BOUNDS fct_coeff_kernel(StepArgs a)
{
    coeff_body(a, blockIdx.x * TI + threadIdx.x % TI, blockIdx.y * TJ + threadIdx.x / TI, a.k0 + blockIdx.z);
}

__global__ void FINAL_BOUNDS fct_final_kernel(StepArgs a)
{
    final_body(a, blockIdx.x * TI + threadIdx.x % TI, blockIdx.y * TJ + threadIdx.x / TI, a.k0 + blockIdx.z);
}

// Batched launches of passes 4 and 5: domain d owns CTAs off[d] .. off[d+1]-1, one 32 x 8 tile of one layer each.
__global__ void COEFF_BATCHED_BOUNDS fct_coeff_batched(const BatchDomain* __restrict__ doms,
                                                               const int* __restrict__ off, int ndom)
{
    __shared__ BlockTile bt;
    __shared__ StepArgs sh;
    const StepArgs& a = block_tile<false, TJ>(doms, off, ndom, bt, sh);
    coeff_body(a, bt.bx * TI + threadIdx.x % TI, bt.by * TJ + threadIdx.x / TI, bt.k);
}

__global__ void FINAL_BATCHED_BOUNDS fct_final_batched(const BatchDomain* __restrict__ doms,
                                                               const int* __restrict__ off, int ndom)
{
    __shared__ BlockTile bt;
    __shared__ StepArgs sh;
    const StepArgs& a = block_tile<false, TJ>(doms, off, ndom, bt, sh);
    final_body(a, bt.bx * TI + threadIdx.x % TI, bt.by * TJ + threadIdx.x / TI, bt.k);
}

// Effective flux F_L + C A of the step through u-face column face_i, (nt, n, ny) (tracers.py:251-254).
__global__ void fct_tef_kernel(StepArgs a)
{
    const Shape s = a.s;
    const Flags fl(a.flags);
    const i64 total = (i64)s.nt * s.n * s.ny;
    const i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= total) return;
    const int j = (int)(r % s.ny);
    const int k = (int)((r / s.ny) % s.n);
    const int t = (int)(r / ((i64)s.n * s.ny));
    const double* Cp = a.C + s.cell(t, k, 0, 0);
    const double* eL = a.inflow ? a.inflow + s.cell(t, k, 0, 0) : Cp;
    const double A = a.Sx[s.ux(t, k, j, a.face_i)];
    a.fx_face[r] = donor_x(Cp, eL, a.Qx, s, fl, k, j, a.face_i) + coef_x(a, s, fl, t, k, j, a.face_i, A) * A;
}

// Net inflow through the open edges per tracer (tracers.py:65-78): one block per tracer, a fixed-order reduction
// so that the result does not change from run to run.
__global__ void __launch_bounds__(256) fct_open_flux_kernel(StepArgs a, double* open_flux)
{
    __shared__ double red[256];
    const Shape s = a.s;
    const Flags fl(a.flags);
    const int t = blockIdx.x;
    double acc = 0.0;
    const i64 nxe = (i64)s.n * s.ny, nye = (i64)s.n * s.nx;
    for (i64 r = threadIdx.x; r < nxe; r += blockDim.x) {
        const int j = (int)(r % s.ny), k = (int)(r / s.ny);
        const double* Cp = a.C + s.cell(t, k, 0, 0);
        const double* eL = a.inflow ? a.inflow + s.cell(t, k, 0, 0) : Cp;
        if (fl.open_w) {
            const double A = a.Sx[s.ux(t, k, j, 0)];
            acc += donor_x(Cp, eL, a.Qx, s, fl, k, j, 0) + coef_x(a, s, fl, t, k, j, 0, A) * A;
        }
        if (fl.open_e) {
            const double A = a.Sx[s.ux(t, k, j, s.nx)];
            acc -= donor_x(Cp, eL, a.Qx, s, fl, k, j, s.nx) + coef_x(a, s, fl, t, k, j, s.nx, A) * A;
        }
    }
    for (i64 r = threadIdx.x; r < nye; r += blockDim.x) {
        const int i = (int)(r % s.nx), k = (int)(r / s.nx);
        const double* Cp = a.C + s.cell(t, k, 0, 0);
        const double* eL = a.inflow ? a.inflow + s.cell(t, k, 0, 0) : Cp;
        if (fl.open_s) {
            const double A = a.Sy[s.vy(t, k, 0, i)];
            acc += donor_y(Cp, eL, a.Qy, s, fl, k, 0, i) + coef_y(a, s, fl, t, k, 0, i, A) * A;
        }
        if (fl.open_n) {
            const double A = a.Sy[s.vy(t, k, s.ny, i)];
            acc -= donor_y(Cp, eL, a.Qy, s, fl, k, s.ny, i) + coef_y(a, s, fl, t, k, s.ny, i, A) * A;
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) open_flux[t] = red[0];
}

// ---------------------------------------------------------------------------------------------------------------
// SSP-RK3 without limiter (tracers.py:342-375): per stage a face pass (the x, y and z WENO5 faces of _advect_div)
// and a cell pass (the stage update of _rk_stage).

// z-face flux through interface kf (between layers kf-1 and kf) of column (j, i): WENO5 in k on the layers of the
// column, valid cells only, 0 on the bed and surface interfaces (sigma_baroclinic.py:335-353).
__device__ __forceinline__ double zface_flux(const StepArgs& a, const Shape& s, const Flags& fl, const double* cin,
                                             int t, int kf, int j, int i)
{
    if (a.Fz == nullptr || kf < 1 || kf > s.n - 1) return 0.0;
    const int pl = s.ny * s.nx, ij = j * s.nx + i;            // 32-bit offsets within a field
    const double q = a.Fz[kf * pl + ij];
    if (q == 0.0) return 0.0;
    const double* ct = cin + plane_at(t, s.n * pl);
    // the five upwind layers in upwind order, as the reference passes them to _wval: kf-3 .. kf+1 when q >= 0,
    // kf+2 .. kf-2 when q < 0 (no per-value selects)
    const bool pos = q >= 0.0;
    const int k0 = pos ? kf - 3 : kf + 2, dk = pos ? 1 : -1;
    double w[5];
    bool v[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const int kk = k0 + m * dk;
        const bool in = kk >= 0 && kk < s.n;
        w[m] = in ? ct[kk * pl + ij] : 0.0;
        v[m] = in && a.ok[(in ? kk : 0) * pl + ij] != 0;
    }
    return q * weno5_value(w[0], w[1], w[2], w[3], w[4], v[0], v[1], v[2], v[3], v[4], fl.z);
}

// Face values of the reference's NumPy RHS (tracers.py:110-151), used by `advect` for the upwind-3 / upwind-1
// schemes and by the centred predictor of the 'pc' time stepping: FS_UP3 and FS_UP1 (_up3_faces,
// sigma_baroclinic.py:164-188), FS_CEN (_centred_faces, :632-652); FS_WENO is the fused WENO5 path above.  The
// NumPy path multiplies every face value by its transport (no skip where Q = 0) and gives the closed boundary faces
// the value 0, so the fluxes here are Q * value there too.
enum FaceScheme { FS_WENO = 0, FS_UP3 = 1, FS_UP1 = 2, FS_CEN = 3 };

// Cells f-3 .. f+2 around face f of a line of n cells (stride `st`), with validity `in range and ok`; out of range
// 0 and invalid (the reference's _shift), periodic lines wrap.
__device__ __forceinline__ void line6(const double* __restrict__ c, const uint8_t* __restrict__ ok, int st, int n,
                                      bool per, int f, double* w, bool* v)
{
    if (f >= 3 && f + 2 < n) {
#pragma unroll
        for (int m = 0; m < 6; ++m) {
            w[m] = __ldg(c + (f - 3 + m) * st);
            v[m] = __ldg(ok + (f - 3 + m) * st) != 0;
        }
        return;
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        int g = f - 3 + m;
        bool in = true;
        if (per) g = wrap(g, n); else in = g >= 0 && g < n;
        w[m] = in ? __ldg(c + g * st) : 0.0;
        v[m] = in && __ldg(ok + (in ? g : 0) * st) != 0;
    }
}

// The value on face f from its six cells w[0..5] = c[f-3 .. f+2] (the same expressions, in the same order, as the
// NumPy functions named above; the divisions are IEEE divisions, as NumPy's).
template <int FS>
__device__ __forceinline__ double lin_face_value(const double* w, const bool* v, double q)
{
    const double lo = w[2], hi = w[3];
    if (FS == FS_UP1) return q >= 0.0 ? lo : hi;
    if (FS == FS_UP3) {
        if (q >= 0.0) return (v[1] && v[2] && v[3]) ? (-w[1] + 5.0 * lo + 2.0 * hi) / 6.0 : lo;
        return (v[2] && v[3] && v[4]) ? (2.0 * lo + 5.0 * hi - w[4]) / 6.0 : hi;
    }
    const double near = lo + hi, mid = w[1] + w[4];
    if (v[0] && v[1] && v[2] && v[3] && v[4] && v[5]) return (37.0 * near - 8.0 * mid + (w[0] + w[5])) / 60.0;
    if (v[1] && v[2] && v[3] && v[4]) return (7.0 * near - mid) / 12.0;
    return 0.5 * near;
}

// x-face flux of the NumPy path through face f of row j (open edges: upstream, the exterior on inflow).
template <int FS>
__device__ __forceinline__ double x_face_lin(const FacePlane& P, const Shape& s, const Flags& fl, int j, int f)
{
    const int row = j * s.nx;
    const double q = __ldg(P.qx + j * (s.nx + 1) + ((fl.per_x && f == s.nx) ? 0 : f));
    if (fl.per_x || (f >= 1 && f <= s.nx - 1)) {
        double w[6];
        bool v[6];
        line6(P.c + row, P.ok + row, 1, s.nx, fl.per_x, f, w, v);
        return q * lin_face_value<FS>(w, v, q);
    }
    if (f == 0) return q * (fl.open_w ? (q > 0.0 ? P.e[row] : P.c[row]) : 0.0);
    return q * (fl.open_e ? (q < 0.0 ? P.e[row + s.nx - 1] : P.c[row + s.nx - 1]) : 0.0);
}

template <int FS>
__device__ __forceinline__ double y_face_lin(const FacePlane& P, const Shape& s, const Flags& fl, int f, int i)
{
    const double q = __ldg(P.qy + ((fl.per_y && f == s.ny) ? 0 : f) * s.nx + i);
    if (fl.per_y || (f >= 1 && f <= s.ny - 1)) {
        double w[6];
        bool v[6];
        line6(P.c + i, P.ok + i, s.nx, s.ny, fl.per_y, f, w, v);
        return q * lin_face_value<FS>(w, v, q);
    }
    const int o = (s.ny - 1) * s.nx + i;
    if (f == 0) return q * (fl.open_s ? (q > 0.0 ? P.e[i] : P.c[i]) : 0.0);
    return q * (fl.open_n ? (q < 0.0 ? P.e[o] : P.c[o]) : 0.0);
}

// z-face flux of the NumPy path through interface kf of column (j, i): Fz[kf] * value on kf = 1 .. n-1, Fz[0] * 0
// on the bed, 0 on the surface (tracers.py:148-150).
template <int FS>
__device__ __forceinline__ double zface_lin(const StepArgs& a, const Shape& s, const double* cin, int t, int kf,
                                            int j, int i)
{
    if (a.Fz == nullptr || kf > s.n - 1) return 0.0;
    const int pl = s.ny * s.nx, ij = j * s.nx + i;
    const double q = a.Fz[kf * pl + ij];
    if (kf == 0) return q * 0.0;
    double w[6];
    bool v[6];
    line6(cin + plane_at(t, s.n * pl) + ij, a.ok + ij, pl, s.n, false, kf, w, v);
    return q * lin_face_value<FS>(w, v, q);
}

// The step as face and cell passes (the FCT stages' design): the face pass of stage s has one thread per cell
// compute the west x-face, the south y-face and the bottom z-face of its cell (the last column / row also the
// east / north domain face) into Sx, Sy and the z-face stack; the cell pass forms -div F from the stored faces
// (x, y, then z, the reference's order), updates the stage and keeps the TEF column.  Each face is computed once.
// A single kernel per stage on shared-memory tiles, which computed every z-face twice (once for each of its two
// cells), took 6.68 ms at 512 x 512 x 50 with a vertical transport; these passes take 3.86 ms, bit-identical.
// Stages 1-3: SSP-RK3 (input C, c1, c2); 4: the 'pc' predictor (input C, centred faces, half step to c1); 5: the
// 'pc' corrector (input c1, the scheme's faces, full step from C).
template <int STAGE>
__device__ __forceinline__ const double* rk3_stage_field(const StepArgs& a)
{
    return (STAGE == 1 || STAGE == 4) ? a.C : ((STAGE == 2 || STAGE == 5) ? a.c1 : a.c2);
}

template <int STAGE, bool ZV, int FS>
__device__ __forceinline__ void rk3_faces_body(const StepArgs& a, int t, int k, int i, int j)
{
    const Shape s = a.s;
    const Flags fl(a.flags);
    if (i >= s.nx || j >= s.ny) return;
    const int pl = s.ny * s.nx, xpl = s.ny * (s.nx + 1), ypl = (s.ny + 1) * s.nx, p = t * s.n + k;
    const i64 pc = plane_at(p, pl);
    const double* cin = rk3_stage_field<STAGE>(a);
    FacePlane P;
    P.c = cin + pc;
    P.e = a.inflow ? a.inflow + pc : P.c;
    P.c0 = P.c;
    P.e0 = P.e;
    P.ok = a.ok + plane_at(k, pl);
    P.qx = a.Qx + plane_at(k, xpl);
    P.qy = a.Qy + plane_at(k, ypl);
    double* sx = a.Sx + plane_at(p, xpl);
    double* sy = a.Sy + plane_at(p, ypl);
    const int fxo = j * (s.nx + 1) + i, fyo = j * s.nx + i;
    if (FS != FS_WENO) {
        sx[fxo] = x_face_lin<FS>(P, s, fl, j, i);
        sy[fyo] = y_face_lin<FS>(P, s, fl, j, i);
        a.Tx[pc + fyo] = zface_lin<FS>(a, s, cin, t, k, j, i);
        if (i == s.nx - 1) sx[fxo + 1] = x_face_lin<FS>(P, s, fl, j, s.nx);
        if (j == s.ny - 1) sy[fyo + s.nx] = y_face_lin<FS>(P, s, fl, s.ny, i);
        return;
    }
    double F, unused;
    x_face<ZV, false, false>(P, s, fl, j, i, F, unused);
    sx[fxo] = F;
    y_face<ZV, false, false>(P, s, fl, j, i, F, unused);
    sy[fyo] = F;
    a.Tx[pc + fyo] = zface_flux(a, s, fl, cin, t, k, j, i);          // bottom interface k (0 at the bed)
    if (i == s.nx - 1) {
        x_face<ZV, false, false>(P, s, fl, j, s.nx, F, unused);
        sx[fxo + 1] = F;
    }
    if (j == s.ny - 1) {
        y_face<ZV, false, false>(P, s, fl, s.ny, i, F, unused);
        sy[fyo + s.nx] = F;
    }
}

// Register budget of the RK3 face passes as resident 256-thread blocks per SM: 6 (40 registers); 8 (32 registers,
// which the FCT face passes prefer) is 1.4 % slower here.
#ifndef POCEAN_RK3_FACES_MINB
#define POCEAN_RK3_FACES_MINB 6
#endif
template <int STAGE, bool ZV, int FS, int TJR>
__global__ void __launch_bounds__(TI * TJR, POCEAN_RK3_FACES_MINB * 256 / (TI * TJR)) rk3_faces_kernel(StepArgs a)
{
    int k, t;
    split_plane(blockIdx.z, a.s.nt, a.tdiv, k, t);
    rk3_faces_body<STAGE, ZV, FS>(a, t, k, blockIdx.x * TI + threadIdx.x % TI,
                                  blockIdx.y * TJR + threadIdx.x / TI);
}

template <int STAGE, int TJR>
__global__ void __launch_bounds__(TI * TJR) rk3_update_kernel(StepArgs a)
{
    int k, t;
    split_plane(blockIdx.z, a.s.nt, a.tdiv, k, t);
    const int gi = blockIdx.x * TI + threadIdx.x % TI, gj = blockIdx.y * TJR + threadIdx.x / TI;
    const Shape s = a.s;
    if (gi >= s.nx || gj >= s.ny) return;
    const int pl = s.ny * s.nx, p = t * s.n + k, ij = gj * s.nx + gi;
    const i64 w = plane_at(p, s.ny * (s.nx + 1)) + (gj * (s.nx + 1) + gi), so = plane_at(p, (s.ny + 1) * s.nx) + ij;
    const i64 ci = plane_at(p, pl) + ij;
    if (a.fx_face != nullptr && gi == (a.face_i == s.nx ? s.nx - 1 : a.face_i)) {
        const double F = a.Sx[a.face_i == s.nx ? w + 1 : w];
        const i64 r = ((i64)t * s.n + k) * s.ny + gj;
        if (STAGE == 1) a.tef0[r] = F;
        else if (STAGE == 2) a.tef1[r] = F;
        else if (STAGE == 3) a.fx_face[r] = div6_exact(a.tef0[r] + a.tef1[r]) + div3_exact(2.0 * F);
        else if (STAGE == 5) a.fx_face[r] = F;                    // 'pc': the corrector's flux F(c^{n+1/2})
    }
    const double fzb = a.Tx[ci];
    const double fzt = k + 1 < s.n ? a.Tx[ci + pl] : 0.0;      // the surface interface carries no flux
    const double r = -(a.Sx[w + 1] - a.Sx[w] + a.Sy[so + s.nx] - a.Sy[so] + fzt - fzb);
    const int g = k * pl + ij;
    const double v0 = a.V0[g], v1 = a.V1[g], c0 = a.C[ci];
    const double q0 = v0 * c0, dv = v1 - v0;
    double q, v;
    if (STAGE == 1) {
        q = q0 + a.dt * r;
        v = v0 + dv;
        a.q1[ci] = q;
        a.c1[ci] = v > 0 ? q / v : c0;
    } else if (STAGE == 2) {
        q = 0.75 * q0 + 0.25 * (a.q1[ci] + a.dt * r);
        v = v0 + 0.5 * dv;
        a.q2[ci] = q;
        a.c2[ci] = v > 0 ? q / v : c0;
    } else if (STAGE == 3) {
        q = div3_exact(q0) + 2.0 / 3.0 * (a.q2[ci] + a.dt * r);
        a.out[ci] = v1 > 0 ? q / v1 : c0;
    } else if (STAGE == 4) {                                     // tracers.py:327-328
        q = q0 + 0.5 * a.dt * r;
        v = v0 + 0.5 * dv;
        a.c1[ci] = v > 0 ? q / v : c0;
    } else {                                                     // tracers.py:329
        q = q0 + a.dt * r;
        a.out[ci] = v1 > 0 ? q / v1 : c0;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// The single-stage helpers of TracerAdvection (tracers.py:139-206): the horizontal face fluxes of a field
// (`faces_h`: the WENO5 faces of _advect_faces_h; `flux_x`: the faces `rhs` differences, WENO5, the NumPy path's
// upwind-3 / upwind-1 or centred faces; `upwind_faces_h`: donor cell) and the RHS -div(Q c) itself (`rhs`,
// `rhs_numpy`).  The reference runs them on the arrays it is given (a periodic caller pads them first), so they
// take no periodic flag.

// x- and y-face fluxes of plane (t, k) for cell (j, i): its west and south faces, plus the east / north domain
// faces on the last column / row.  KIND: FS_WENO, FS_UP3, FS_UP1, FS_CEN, or FACES_DONOR.
constexpr int FACES_DONOR = 4;

template <int KIND, bool ZV>
__device__ __forceinline__ double any_x_face(const FacePlane& P, const StepArgs& a, const Shape& s, const Flags& fl,
                                             int k, int j, int f)
{
    if (KIND == FACES_DONOR) return donor_x(P.c, P.e, a.Qx, s, fl, k, j, f);
    if (KIND == FS_WENO) {
        double F, unused;
        x_face<ZV, false, false>(P, s, fl, j, f, F, unused);
        return F;
    }
    return x_face_lin<KIND>(P, s, fl, j, f);
}

template <int KIND, bool ZV>
__device__ __forceinline__ double any_y_face(const FacePlane& P, const StepArgs& a, const Shape& s, const Flags& fl,
                                             int k, int f, int i)
{
    if (KIND == FACES_DONOR) return donor_y(P.c, P.e, a.Qy, s, fl, k, f, i);
    if (KIND == FS_WENO) {
        double F, unused;
        y_face<ZV, false, false>(P, s, fl, f, i, F, unused);
        return F;
    }
    return y_face_lin<KIND>(P, s, fl, f, i);
}

template <int KIND, bool ZV>
__global__ void __launch_bounds__(TI * TJ) helper_faces_kernel(StepArgs a, double* __restrict__ fx,
                                                               double* __restrict__ fy)
{
    int k, t;
    split_plane(blockIdx.z, a.s.nt, a.tdiv, k, t);
    const Shape s = a.s;
    const Flags fl(a.flags);
    const int i = blockIdx.x * TI + threadIdx.x % TI, j = blockIdx.y * TJ + threadIdx.x / TI;
    if (i >= s.nx || j >= s.ny) return;
    const int pl = s.ny * s.nx, xpl = s.ny * (s.nx + 1), ypl = (s.ny + 1) * s.nx, p = t * s.n + k;
    const i64 pc = plane_at(p, pl);
    FacePlane P;
    P.c = a.C + pc;
    P.e = a.inflow ? a.inflow + pc : P.c;
    P.c0 = P.c;
    P.e0 = P.e;
    P.ok = a.ok + plane_at(k, pl);
    P.qx = a.Qx + plane_at(k, xpl);
    P.qy = a.Qy + plane_at(k, ypl);
    double* sx = fx + plane_at(p, xpl);
    double* sy = fy + plane_at(p, ypl);
    const int fxo = j * (s.nx + 1) + i, fyo = j * s.nx + i;
    sx[fxo] = any_x_face<KIND, ZV>(P, a, s, fl, k, j, i);
    sy[fyo] = any_y_face<KIND, ZV>(P, a, s, fl, k, j, i);
    if (i == s.nx - 1) sx[fxo + 1] = any_x_face<KIND, ZV>(P, a, s, fl, k, j, s.nx);
    if (j == s.ny - 1) sy[fyo + s.nx] = any_y_face<KIND, ZV>(P, a, s, fl, k, s.ny, i);
}

// -div(Q c) of cell (t, k, j, i) from the stored faces, x then y then z (the reference's order, tracers.py:151 and
// sigma_baroclinic.py:357-362).
__global__ void __launch_bounds__(TI * TJ) helper_rhs_kernel(StepArgs a, double* __restrict__ out)
{
    int k, t;
    split_plane(blockIdx.z, a.s.nt, a.tdiv, k, t);
    const Shape s = a.s;
    const int gi = blockIdx.x * TI + threadIdx.x % TI, gj = blockIdx.y * TJ + threadIdx.x / TI;
    if (gi >= s.nx || gj >= s.ny) return;
    const int pl = s.ny * s.nx, p = t * s.n + k, ij = gj * s.nx + gi;
    const i64 w = plane_at(p, s.ny * (s.nx + 1)) + (gj * (s.nx + 1) + gi), so = plane_at(p, (s.ny + 1) * s.nx) + ij;
    const i64 ci = plane_at(p, pl) + ij;
    const double fzb = a.Tx[ci];
    const double fzt = k + 1 < s.n ? a.Tx[ci + pl] : 0.0;
    out[ci] = -(a.Sx[w + 1] - a.Sx[w] + a.Sy[so + s.nx] - a.Sy[so] + fzt - fzb);
}

}  // namespace po

// =================================================================================================================
// C ABI
using namespace po;

static size_t align_up(size_t b) { return (b + 255) & ~(size_t)255; }

// The FCT workspace of shape a.s cut into its buffers (layout of pocean_advect_fct_workspace_bytes).
void po::carve_fct_workspace(StepArgs& a, void* workspace)
{
    const Shape& s = a.s;
    char* w = (char*)workspace;
    const size_t cells = align_up((size_t)s.nt * s.n * s.ny * s.nx * sizeof(double));
    a.q1 = (double*)w; w += cells;
    a.c1 = (double*)w; w += cells;
    a.c2 = (double*)w; w += cells;
    const size_t xf = align_up((size_t)s.nt * s.n * s.ny * (s.nx + 1) * sizeof(double));
    const size_t yf = align_up((size_t)s.nt * s.n * (s.ny + 1) * s.nx * sizeof(double));
    a.Sx = (double*)w; w += xf;
    a.Sy = (double*)w; w += yf;
    a.Tx = (double*)w; w += xf;
    a.Ty = (double*)w;
    a.q2 = nullptr; a.tef0 = a.tef1 = nullptr;
}

static int check_shape(const char* fn, int nt, int nz, int ny, int nx)
{
    if (nt < 1 || nz < 1 || ny < 1 || nx < 1)
        return pocean_fail(POCEAN_EINVAL, "%s: sizes must be >= 1 (nt=%d nz=%d ny=%d nx=%d)", fn, nt, nz, ny, nx);
    if ((i64)nt * nz > 65535)
        return pocean_fail(POCEAN_EINVAL, "%s: nt*nz = %lld exceeds 65535", fn, (long long)nt * nz);
    if ((i64)nz * (ny + 1) * (nx + 1) >= (1ll << 31))
        return pocean_fail(POCEAN_EINVAL, "%s: one field of %d x %d x %d cells exceeds 2^31 entries", fn, nz, ny, nx);
    return POCEAN_OK;
}

extern "C" size_t pocean_advect_fct_workspace_bytes(int nt, int nz, int ny, int nx)
{
    if (nt < 1 || nz < 1 || ny < 1 || nx < 1) return 0;
    const size_t cells = (size_t)nt * nz * ny * nx * sizeof(double);
    const size_t xf = (size_t)nt * nz * ny * (nx + 1) * sizeof(double);
    const size_t yf = (size_t)nt * nz * (ny + 1) * nx * sizeof(double);
    return 3 * align_up(cells) + 2 * (align_up(xf) + align_up(yf));
}

extern "C" size_t pocean_advect_rk3_workspace_bytes(int nt, int nz, int ny, int nx)
{
    if (nt < 1 || nz < 1 || ny < 1 || nx < 1) return 0;
    const size_t cells = (size_t)nt * nz * ny * nx * sizeof(double);
    const size_t col = (size_t)nt * nz * ny * sizeof(double);
    const size_t xf = (size_t)nt * nz * ny * (nx + 1) * sizeof(double);
    const size_t yf = (size_t)nt * nz * (ny + 1) * nx * sizeof(double);
    return 5 * align_up(cells) + 2 * align_up(col) + align_up(xf) + align_up(yf);      // stages, TEF, faces
}

static int common_checks(const char* fn, const void* C, const void* V0, const void* V1, const void* Qx,
                         const void* Qy, const void* ok, const void* out, int nt, int nz, int ny, int nx,
                         unsigned flags, int face_i, const void* fx_face, void* ws, size_t ws_bytes, size_t need,
                         unsigned allowed = 0xFFu)
{
    int rc = check_shape(fn, nt, nz, ny, nx);
    if (rc) return rc;
    if (!C || !V0 || !V1 || !Qx || !Qy || !ok || !out)
        return pocean_fail(POCEAN_EINVAL, "%s: null input or output pointer", fn);
    if (flags & ~allowed) return pocean_fail(POCEAN_EINVAL, "%s: unknown flag bits 0x%x", fn, flags & ~allowed);
    if (fx_face && (face_i < 0 || face_i > nx))
        return pocean_fail(POCEAN_EINVAL, "%s: face_i=%d outside 0..nx=%d", fn, face_i, nx);
    if (!ws || ws_bytes < need)
        return pocean_fail(POCEAN_EWORKSPACE, "%s: workspace of %zu bytes needed, %zu given", fn, need,
                           ws ? ws_bytes : (size_t)0);
    if (((uintptr_t)ws & 255) != 0) return pocean_fail(POCEAN_EWORKSPACE, "%s: workspace not 256-byte aligned", fn);
    return pocean_check_device();
}

// Rows of the 32-wide cell tiles of the single-domain stage passes.
#ifndef POCEAN_FACE_ROWS
#define POCEAN_FACE_ROWS 8
#endif

template <bool ZV, bool MIX>
static void launch_split(const StepArgs& a, int stage, cudaStream_t st, int nlayers = -1)
{
    constexpr int R = POCEAN_FACE_ROWS;
    const Shape& s = a.s;
    const dim3 grid(ceil_div(s.nx, TI), ceil_div(s.ny, R), s.nt * (nlayers < 0 ? s.n : nlayers));
    if (stage == 1) {
        fct_faces_kernel<1, ZV, MIX, R><<<grid, TI * R, 0, st>>>(a);
        fct_update_kernel<1, R><<<grid, TI * R, 0, st>>>(a);
    } else if (stage == 2) {
        fct_faces_kernel<2, ZV, MIX, R><<<grid, TI * R, 0, st>>>(a);
        fct_update_kernel<2, R><<<grid, TI * R, 0, st>>>(a);
    } else {
        fct_faces3_kernel<ZV, MIX, R><<<grid, TI * R, 0, st>>>(a);
    }
}

// The FCT step with FP64 (mixed = false) or FP32-weight (mixed = true) WENO faces; everything else FP64.
static int advect_fct_impl(const char* fn, bool mixed, const double* C, const double* V0, const double* V1,
                           const double* Qx, const double* Qy, const uint8_t* ok, const double* inflow, int nt,
                           int nz, int ny, int nx, unsigned flags, double dt, double* C_out, int face_i,
                           double* fx_face, double* open_flux, void* workspace, size_t workspace_bytes, void* stream)
{
    int rc = common_checks(fn, C, V0, V1, Qx, Qy, ok, C_out, nt, nz, ny, nx, flags, face_i, fx_face, workspace,
                           workspace_bytes, pocean_advect_fct_workspace_bytes(nt, nz, ny, nx));
    if (rc) return rc;
    if ((flags & POCEAN_FCT_UNLIMITED) && open_flux)
        return pocean_fail(POCEAN_EINVAL, "%s: open_flux is only defined for the limited step", fn);
    if (open_flux && (((flags & POCEAN_PERIODIC_X) && (flags & (POCEAN_OPEN_W | POCEAN_OPEN_E))) ||
                      ((flags & POCEAN_PERIODIC_Y) && (flags & (POCEAN_OPEN_S | POCEAN_OPEN_N)))))
        return pocean_fail(POCEAN_EINVAL, "%s: open_flux is not defined for an open edge on a periodic axis", fn);
    cudaStream_t st = (cudaStream_t)stream;
    StepArgs a{};
    a.s = Shape{nt, nz, ny, nx};
    a.tdiv = plane_magic(nt);
    a.flags = flags;
    a.dt = dt;
    a.C = C; a.V0 = V0; a.V1 = V1; a.Qx = Qx; a.Qy = Qy; a.Fz = nullptr; a.ok = ok; a.inflow = inflow;
    carve_fct_workspace(a, workspace);
    a.out = C_out; a.face_i = face_i; a.fx_face = fx_face;

    const dim3 grid(ceil_div(nx, TI), ceil_div(ny, TJ), nt * nz);
    const bool zv = !(flags & POCEAN_WENO_JS);
    auto stage_passes = [&](int stage) {
        if (zv && !mixed) launch_split<true, false>(a, stage, st);
        else if (!zv && !mixed) launch_split<false, false>(a, stage, st);
        else if (zv) launch_split<true, true>(a, stage, st);
        else launch_split<false, true>(a, stage, st);
    };
    stage_passes(1);
    stage_passes(2);
    if (flags & POCEAN_FCT_UNLIMITED) {
        constexpr int R = POCEAN_FACE_ROWS;
        const dim3 g2(ceil_div(nx, TI), ceil_div(ny, R), nt * nz);
        if (zv && !mixed) fct_faces_kernel<4, true, false, R><<<g2, TI * R, 0, st>>>(a);
        else if (!zv && !mixed) fct_faces_kernel<4, false, false, R><<<g2, TI * R, 0, st>>>(a);
        else if (zv) fct_faces_kernel<4, true, true, R><<<g2, TI * R, 0, st>>>(a);
        else fct_faces_kernel<4, false, true, R><<<g2, TI * R, 0, st>>>(a);
        fct_update_kernel<4, R><<<g2, TI * R, 0, st>>>(a);
        return pocean_check_launch(fn);
    }
    stage_passes(3);
    fct_coeff_kernel<<<dim3(ceil_div(nx, TI), ceil_div(ny, TJ), nz), NTHREADS, 0, st>>>(a);
    fct_final_kernel<<<dim3(ceil_div(nx, TI), ceil_div(ny, TJ), nz), NTHREADS, 0, st>>>(a);
    if (fx_face) {
        const i64 rows = (i64)nt * nz * ny;
        fct_tef_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(a);
    }
    if (open_flux) fct_open_flux_kernel<<<nt, 256, 0, st>>>(a, open_flux);
    return pocean_check_launch(fn);
}

namespace po {

// The FCT passes of every domain of a batch, one launch per pass (off_host: the CTA offsets also held on the device).
template <bool ZV, bool MIX, int TJR>
static void fct_batched_stages(const BatchDomain* doms, const int* po, unsigned np, int ndom, cudaStream_t st)
{
    fct_faces_batched<1, ZV, MIX, TJR><<<np, TI * TJR, 0, st>>>(doms, po, ndom);
    fct_update_batched<1, TJR><<<np, TI * TJR, 0, st>>>(doms, po, ndom);
    fct_faces_batched<2, ZV, MIX, TJR><<<np, TI * TJR, 0, st>>>(doms, po, ndom);
    fct_update_batched<2, TJR><<<np, TI * TJR, 0, st>>>(doms, po, ndom);
    fct_faces3_batched<ZV, MIX, TJR><<<np, TI * TJR, 0, st>>>(doms, po, ndom);
}

// The FCT passes of every domain of a batch, one launch per pass (off_host: the CTA offsets also held on the device).
template <bool ZV, bool MIX>
static void fct_batched_impl(const BatchDomain* doms, const int* off_dev, const int* off_host, int ndom, int tile_rows,
                             cudaStream_t st)
{
    const int* po = off_dev + BP_PTILE * (ndom + 1);
    const int* to = off_dev + BP_TILE * (ndom + 1);
    const unsigned np = (unsigned)off_host[BP_PTILE * (ndom + 1) + ndom];
    const unsigned nt = (unsigned)off_host[BP_TILE * (ndom + 1) + ndom];
    if (tile_rows == 4) fct_batched_stages<ZV, MIX, 4>(doms, po, np, ndom, st);
    else if (tile_rows == 16) fct_batched_stages<ZV, MIX, 16>(doms, po, np, ndom, st);
    else fct_batched_stages<ZV, MIX, 8>(doms, po, np, ndom, st);
    fct_coeff_batched<<<nt, NTHREADS, 0, st>>>(doms, to, ndom);
    fct_final_batched<<<nt, NTHREADS, 0, st>>>(doms, to, ndom);
}

void fct_batched_launch(const BatchDomain* doms, const int* off_dev, const int* off_host, int ndom, bool zv,
                        bool mixed, int tile_rows, cudaStream_t st)
{
    if (zv && !mixed) fct_batched_impl<true, false>(doms, off_dev, off_host, ndom, tile_rows, st);
    else if (!zv && !mixed) fct_batched_impl<false, false>(doms, off_dev, off_host, ndom, tile_rows, st);
    else if (zv) fct_batched_impl<true, true>(doms, off_dev, off_host, ndom, tile_rows, st);
    else fct_batched_impl<false, true>(doms, off_dev, off_host, ndom, tile_rows, st);
}

// CTAs of each batched FCT pass for one domain: 32 x tile_rows tiles x planes (stage passes); 32 x 8 tiles x
// layers (coefficient and final passes).
void fct_batched_ctas(const Shape& s, int tile_rows, int& plane_ctas, int& tile_ctas)
{
    plane_ctas = ceil_div(s.nx, TI) * ceil_div(s.ny, tile_rows) * s.nt * s.n;
    tile_ctas = ceil_div(s.nx, TI) * ceil_div(s.ny, TJ) * s.n;
}

}  // namespace po

using namespace po;

extern "C" int pocean_advect_fct_f64(const double* C, const double* V0, const double* V1, const double* Qx,
                                     const double* Qy, const uint8_t* ok, const double* inflow, int nt, int nz,
                                     int ny, int nx, unsigned flags, double dt, double* C_out, int face_i,
                                     double* fx_face, double* open_flux, void* workspace, size_t workspace_bytes,
                                     void* stream)
{
    return advect_fct_impl("pocean_advect_fct_f64", false, C, V0, V1, Qx, Qy, ok, inflow, nt, nz, ny, nx, flags, dt,
                           C_out, face_i, fx_face, open_flux, workspace, workspace_bytes, stream);
}

extern "C" int pocean_advect_fct_mixed(const double* C, const double* V0, const double* V1, const double* Qx,
                                       const double* Qy, const uint8_t* ok, const double* inflow, int nt, int nz,
                                       int ny, int nx, unsigned flags, double dt, double* C_out, int face_i,
                                       double* fx_face, double* open_flux, void* workspace, size_t workspace_bytes,
                                       void* stream)
{
    return advect_fct_impl("pocean_advect_fct_mixed", true, C, V0, V1, Qx, Qy, ok, inflow, nt, nz, ny, nx, flags,
                           dt, C_out, face_i, fx_face, open_flux, workspace, workspace_bytes, stream);
}

// The passes of `advect`: three SSP-RK3 stages, or the 'pc' predictor (centred faces) and corrector (the
// scheme's faces).
template <bool ZV, int FS>
static void launch_rk3(const StepArgs& a, bool pc, dim3 grid, cudaStream_t st)
{
    constexpr int R = POCEAN_FACE_ROWS;
    if (pc) {
        rk3_faces_kernel<4, false, FS_CEN, R><<<grid, TI * R, 0, st>>>(a);
        rk3_update_kernel<4, R><<<grid, TI * R, 0, st>>>(a);
        rk3_faces_kernel<5, ZV, FS, R><<<grid, TI * R, 0, st>>>(a);
        rk3_update_kernel<5, R><<<grid, TI * R, 0, st>>>(a);
        return;
    }
    rk3_faces_kernel<1, ZV, FS, R><<<grid, TI * R, 0, st>>>(a);
    rk3_update_kernel<1, R><<<grid, TI * R, 0, st>>>(a);
    rk3_faces_kernel<2, ZV, FS, R><<<grid, TI * R, 0, st>>>(a);
    rk3_update_kernel<2, R><<<grid, TI * R, 0, st>>>(a);
    rk3_faces_kernel<3, ZV, FS, R><<<grid, TI * R, 0, st>>>(a);
    rk3_update_kernel<3, R><<<grid, TI * R, 0, st>>>(a);
}

extern "C" int pocean_advect_rk3_f64(const double* C, const double* V0, const double* V1, const double* Qx,
                                     const double* Qy, const double* Fz, const uint8_t* ok, const double* inflow,
                                     int nt, int nz, int ny, int nx, unsigned flags, double dt, double* C_out,
                                     int face_i, double* fx_face, void* workspace, size_t workspace_bytes,
                                     void* stream)
{
    const char* fn = "pocean_advect_rk3_f64";
    if ((flags & POCEAN_FACES_UP3) && (flags & POCEAN_FACES_UP1))
        return pocean_fail(POCEAN_EINVAL, "%s: POCEAN_FACES_UP3 and POCEAN_FACES_UP1 are exclusive", fn);
    int rc = common_checks(fn, C, V0, V1, Qx, Qy, ok, C_out, nt, nz, ny, nx, flags, face_i, fx_face, workspace,
                           workspace_bytes, pocean_advect_rk3_workspace_bytes(nt, nz, ny, nx),
                           0xFFu | POCEAN_FACES_UP3 | POCEAN_FACES_UP1 | POCEAN_TIME_PC);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    StepArgs a{};
    a.s = Shape{nt, nz, ny, nx};
    a.tdiv = plane_magic(nt);
    a.flags = flags;
    a.dt = dt;
    a.C = C; a.V0 = V0; a.V1 = V1; a.Qx = Qx; a.Qy = Qy; a.Fz = Fz; a.ok = ok; a.inflow = inflow;
    char* w = (char*)workspace;
    const size_t cells = align_up((size_t)nt * nz * ny * nx * sizeof(double));
    a.q1 = (double*)w; w += cells;
    a.c1 = (double*)w; w += cells;
    a.q2 = (double*)w; w += cells;
    a.c2 = (double*)w; w += cells;
    a.tef0 = (double*)w; w += align_up((size_t)nt * nz * ny * sizeof(double));
    a.tef1 = (double*)w; w += align_up((size_t)nt * nz * ny * sizeof(double));
    a.Sx = a.Sy = a.Tx = a.Ty = nullptr;
    a.out = C_out; a.face_i = face_i; a.fx_face = fx_face;
    a.Tx = (double*)w; w += cells;                                       // z-faces (interface k of each cell)
    a.Sx = (double*)w; w += align_up((size_t)nt * nz * ny * (nx + 1) * sizeof(double));
    a.Sy = (double*)w;
    const dim3 grid(ceil_div(nx, TI), ceil_div(ny, POCEAN_FACE_ROWS), nt * nz);
    const bool pc = flags & POCEAN_TIME_PC;
    if (flags & POCEAN_FACES_UP3) launch_rk3<false, FS_UP3>(a, pc, grid, st);
    else if (flags & POCEAN_FACES_UP1) launch_rk3<false, FS_UP1>(a, pc, grid, st);
    else if (flags & POCEAN_WENO_JS) launch_rk3<false, FS_WENO>(a, pc, grid, st);
    else launch_rk3<true, FS_WENO>(a, pc, grid, st);
    return pocean_check_launch(fn);
}

// The single-stage helpers (tracers.py:139-206).  kind 0: the advect scheme's faces (WENO5-Z / -JS, or with
// POCEAN_FACES_UP3 / _UP1 the NumPy path's upwind faces); 1: centred faces; 2: donor cell (upwind_faces_h).
static int helper_checks(const char* fn, const void* c, const void* Qx, const void* Qy, const void* ok, int nt,
                         int nz, int ny, int nx, unsigned flags)
{
    int rc = check_shape(fn, nt, nz, ny, nx);
    if (rc) return rc;
    if (!c || !Qx || !Qy || !ok) return pocean_fail(POCEAN_EINVAL, "%s: null input pointer", fn);
    const unsigned allowed = POCEAN_OPEN_W | POCEAN_OPEN_E | POCEAN_OPEN_S | POCEAN_OPEN_N | POCEAN_WENO_JS |
                             POCEAN_FACES_UP3 | POCEAN_FACES_UP1;
    if (flags & ~allowed)
        return pocean_fail(POCEAN_EINVAL, "%s: flag bits 0x%x not taken (the helpers do not wrap periodic axes: "
                           "the caller pads)", fn, flags & ~allowed);
    if ((flags & POCEAN_FACES_UP3) && (flags & POCEAN_FACES_UP1))
        return pocean_fail(POCEAN_EINVAL, "%s: POCEAN_FACES_UP3 and POCEAN_FACES_UP1 are exclusive", fn);
    return POCEAN_OK;
}

extern "C" int pocean_advect_faces_f64(const double* c, const double* Qx, const double* Qy, const uint8_t* ok,
                                       const double* ext, int nt, int nz, int ny, int nx, unsigned flags, int kind,
                                       double* fx, double* fy, void* stream)
{
    const char* fn = "pocean_advect_faces_f64";
    int rc = helper_checks(fn, c, Qx, Qy, ok, nt, nz, ny, nx, flags);
    if (rc) return rc;
    if (kind < 0 || kind > 2) return pocean_fail(POCEAN_EINVAL, "%s: kind %d (0, 1 or 2)", fn, kind);
    if (!fx || !fy) return pocean_fail(POCEAN_EINVAL, "%s: null output pointer", fn);
    rc = pocean_check_device();
    if (rc) return rc;
    StepArgs a{};
    a.s = Shape{nt, nz, ny, nx};
    a.tdiv = plane_magic(nt);
    a.flags = flags;
    a.C = c; a.Qx = Qx; a.Qy = Qy; a.ok = ok; a.inflow = ext;
    const dim3 grid(ceil_div(nx, TI), ceil_div(ny, TJ), nt * nz);
    cudaStream_t st = (cudaStream_t)stream;
    if (kind == 2) helper_faces_kernel<FACES_DONOR, true><<<grid, NTHREADS, 0, st>>>(a, fx, fy);
    else if (kind == 1) helper_faces_kernel<FS_CEN, true><<<grid, NTHREADS, 0, st>>>(a, fx, fy);
    else if (flags & POCEAN_FACES_UP3) helper_faces_kernel<FS_UP3, true><<<grid, NTHREADS, 0, st>>>(a, fx, fy);
    else if (flags & POCEAN_FACES_UP1) helper_faces_kernel<FS_UP1, true><<<grid, NTHREADS, 0, st>>>(a, fx, fy);
    else if (flags & POCEAN_WENO_JS) helper_faces_kernel<FS_WENO, false><<<grid, NTHREADS, 0, st>>>(a, fx, fy);
    else helper_faces_kernel<FS_WENO, true><<<grid, NTHREADS, 0, st>>>(a, fx, fy);
    return pocean_check_launch(fn);
}

extern "C" size_t pocean_advect_rhs_workspace_bytes(int nt, int nz, int ny, int nx)
{
    if (nt < 1 || nz < 1 || ny < 1 || nx < 1) return 0;
    const size_t cells = (size_t)nt * nz * ny * nx * sizeof(double);
    const size_t xf = (size_t)nt * nz * ny * (nx + 1) * sizeof(double);
    const size_t yf = (size_t)nt * nz * (ny + 1) * nx * sizeof(double);
    return align_up(cells) + align_up(xf) + align_up(yf);
}

extern "C" int pocean_advect_rhs_f64(const double* c, const double* Qx, const double* Qy, const double* Fz,
                                     const uint8_t* ok, const double* ext, int nt, int nz, int ny, int nx,
                                     unsigned flags, int centred, double* rhs, void* workspace,
                                     size_t workspace_bytes, void* stream)
{
    const char* fn = "pocean_advect_rhs_f64";
    int rc = helper_checks(fn, c, Qx, Qy, ok, nt, nz, ny, nx, flags);
    if (rc) return rc;
    if (!rhs) return pocean_fail(POCEAN_EINVAL, "%s: null output pointer", fn);
    const size_t need = pocean_advect_rhs_workspace_bytes(nt, nz, ny, nx);
    if (!workspace || workspace_bytes < need)
        return pocean_fail(POCEAN_EWORKSPACE, "%s: workspace of %zu bytes needed, %zu given", fn, need,
                           workspace ? workspace_bytes : (size_t)0);
    if (((uintptr_t)workspace & 255) != 0)
        return pocean_fail(POCEAN_EWORKSPACE, "%s: workspace not 256-byte aligned", fn);
    rc = pocean_check_device();
    if (rc) return rc;
    StepArgs a{};
    a.s = Shape{nt, nz, ny, nx};
    a.tdiv = plane_magic(nt);
    a.flags = flags;
    a.C = c; a.Qx = Qx; a.Qy = Qy; a.Fz = Fz; a.ok = ok; a.inflow = ext;
    char* w = (char*)workspace;
    a.Tx = (double*)w; w += align_up((size_t)nt * nz * ny * nx * sizeof(double));
    a.Sx = (double*)w; w += align_up((size_t)nt * nz * ny * (nx + 1) * sizeof(double));
    a.Sy = (double*)w;
    constexpr int R = POCEAN_FACE_ROWS;
    const dim3 grid(ceil_div(nx, TI), ceil_div(ny, R), nt * nz);
    cudaStream_t st = (cudaStream_t)stream;
    if (centred) rk3_faces_kernel<4, false, FS_CEN, R><<<grid, TI * R, 0, st>>>(a);
    else if (flags & POCEAN_FACES_UP3) rk3_faces_kernel<1, false, FS_UP3, R><<<grid, TI * R, 0, st>>>(a);
    else if (flags & POCEAN_FACES_UP1) rk3_faces_kernel<1, false, FS_UP1, R><<<grid, TI * R, 0, st>>>(a);
    else if (flags & POCEAN_WENO_JS) rk3_faces_kernel<1, false, FS_WENO, R><<<grid, TI * R, 0, st>>>(a);
    else rk3_faces_kernel<1, true, FS_WENO, R><<<grid, TI * R, 0, st>>>(a);
    helper_rhs_kernel<<<dim3(ceil_div(nx, TI), ceil_div(ny, TJ), nt * nz), NTHREADS, 0, st>>>(a, rhs);
    return pocean_check_launch(fn);
}

// Layer-range FCT passes (no counterpart in the reference; the host-array path of the Python layer streams layer
// blocks through them).  part 0: the three stage passes of layers k0 .. k1-1 (they read only those layers);
// part 1: the coefficient and final passes of those layers, whose bounds read layers k0-1 and k1, so part 0 of
// the neighbouring layers must have run first on the same stream.  Parts 0 and 1 over blocks covering 0 .. nz-1
// give the result of pocean_advect_fct_f64 / _mixed bit for bit.  The workspace is the whole step's
// (pocean_advect_fct_workspace_bytes); the unlimited step and the side outputs are not offered here.
extern "C" int pocean_advect_fct_layers(int mixed, const double* C, const double* V0, const double* V1,
                                        const double* Qx, const double* Qy, const uint8_t* ok, const double* inflow,
                                        int nt, int nz, int ny, int nx, unsigned flags, double dt, double* C_out,
                                        void* workspace, size_t workspace_bytes, int k0, int k1, int part,
                                        void* stream)
{
    const char* fn = "pocean_advect_fct_layers";
    if (flags & POCEAN_FCT_UNLIMITED) return pocean_fail(POCEAN_EINVAL, "%s: the unlimited step is not offered", fn);
    if (k0 < 0 || k1 > nz || k0 >= k1) return pocean_fail(POCEAN_EINVAL, "%s: layers %d .. %d of %d", fn, k0, k1, nz);
    if (part != 0 && part != 1) return pocean_fail(POCEAN_EINVAL, "%s: part %d (0 or 1)", fn, part);
    int rc = common_checks(fn, C, V0, V1, Qx, Qy, ok, C_out, nt, nz, ny, nx, flags, 0, nullptr, workspace,
                           workspace_bytes, pocean_advect_fct_workspace_bytes(nt, nz, ny, nx));
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    StepArgs a{};
    a.s = Shape{nt, nz, ny, nx};
    a.tdiv = plane_magic(nt);
    a.flags = flags;
    a.dt = dt;
    a.C = C; a.V0 = V0; a.V1 = V1; a.Qx = Qx; a.Qy = Qy; a.Fz = nullptr; a.ok = ok; a.inflow = inflow;
    carve_fct_workspace(a, workspace);
    a.out = C_out;
    a.k0 = k0;
    const int nl = k1 - k0;
    if (part == 0) {
        const bool zv = !(flags & POCEAN_WENO_JS);
        for (int stage = 1; stage <= 3; ++stage) {
            if (zv && !mixed) launch_split<true, false>(a, stage, st, nl);
            else if (!zv && !mixed) launch_split<false, false>(a, stage, st, nl);
            else if (zv) launch_split<true, true>(a, stage, st, nl);
            else launch_split<false, true>(a, stage, st, nl);
        }
    } else {
        fct_coeff_kernel<<<dim3(ceil_div(nx, TI), ceil_div(ny, TJ), nl), NTHREADS, 0, st>>>(a);
        fct_final_kernel<<<dim3(ceil_div(nx, TI), ceil_div(ny, TJ), nl), NTHREADS, 0, st>>>(a);
    }
    return pocean_check_launch(fn);
}
