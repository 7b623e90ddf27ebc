// The three WENO passes of the FCT step split into a face pass and a cell pass each (included by advect.cu).
//
// Face pass of stage s: one thread per cell (t, k, j, i) computes the west x-face and the south y-face of its cell
// (the last column / row also the east / north domain face) straight from global memory (the five upwind cells of
// a face, loaded in upwind order, overlap between neighbouring threads and are served by L1), with no shared memory
// and no barrier, so the pass runs
// at high occupancy and the two independent WENO5 chains of a thread overlap.  Cell pass of stage s: the stage
// update from the stored faces.  Faces per stage are stored once:
//   stage 1: S <- F0;  stage 2: T <- F1;  stage 3: S <- A = ((F0 + F1)/6 + 2 F2/3) - F_L,
// with (F0 + F1)/6 and 2 F2/3 formed by the same exact divisions as the reference.  Stage 3 has no cell pass: its
// face pass also forms the donor-cell solution c_L of its cell, recomputing the cheap donor fluxes F_L of the
// cell's east and north faces, so F_L is never stored.  The arithmetic of every face and
// update is the reference's (weno.cuh; sigma_baroclinic.py:265-321, 452-511), so results equal the reference's bit
// for bit.  Addresses are formed once per thread as plane pointers with 32-bit offsets; interior stencils (all six
// candidate cells inside the domain, the common case) load without checks, edge and periodic stencils take a guarded
// path.
#pragma once

namespace po {

// The stage's input field (stages 1: C; 2: c1; 3: c2).
template <int STAGE>
__device__ __forceinline__ const double* stage_field(const StepArgs& a)
{
    return STAGE == 1 ? a.C : (STAGE == 2 ? a.c1 : a.c2);
}

// The five cells of the stencil of face f (between cells f-1 and f) in upwind order, as the reference passes them
// to _wval (sigma_baroclinic.py:277-297): v1..v5 = cells f-3 .. f+1 when the transport is >= 0, f+2 .. f-2 when it
// is negative, with their validity `0 <= g < n and ok[g]` (periodic lines wrap).  Loading in upwind order after the
// transport's sign is known replaces the per-value selects of a six-cell stencil (the loads wait for the transport
// anyway: faces with Q = 0 load nothing): 1.1 % of advect_fct at 512 x 512 x 50, and fewer live registers.
template <int ST>
__device__ __forceinline__ void upwind5(const double* __restrict__ c, const uint8_t* __restrict__ ok, int st, int n,
                                        bool per, int f, bool pos, double* w, bool* v)
{
    const int stride = ST > 0 ? ST : st;
    const int g0 = pos ? f - 3 : f + 2, dg = pos ? 1 : -1;
    if (f >= 3 && f + 2 < n) {
        const int o0 = g0 * stride, d = dg * stride;
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            w[m] = __ldg(c + (o0 + m * d));
            v[m] = __ldg(ok + (o0 + m * d)) != 0;
        }
        return;
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        int g = g0 + m * dg;
        bool in = true;
        if (per) g = wrap(g, n); else in = g >= 0 && g < n;
        w[m] = in ? __ldg(c + g * stride) : 0.0;
        v[m] = in && __ldg(ok + (in ? g : 0) * stride) != 0;
    }
}

// One plane (t, k) of the step as pointers; element offsets below are 32-bit.
struct FacePlane {
    const double* __restrict__ c;     // stage field
    const double* __restrict__ e;     // exterior on open edges (inflow, else the stage field)
    const double* __restrict__ c0;    // C (donor flux of stage 3)
    const double* __restrict__ e0;    // exterior of C
    const uint8_t* __restrict__ ok;
    const double* __restrict__ qx;
    const double* __restrict__ qy;
    double* sx;
    double* sy;
    double* tx;
    double* ty;
};

// Flux F through x-face f of row j (WENO5 on interior faces, 0 where Q = 0; open edges upstream with the exterior
// on inflow; closed edges 0) and, for stage 3, the donor flux FL of C through the same face
// (sigma_baroclinic.py:277-297, 486-494).
template <bool ZV, bool MIX, bool DONOR>
__device__ __forceinline__ void x_face(const FacePlane& P, const Shape& s, const Flags& fl, int j, int f, double& F,
                                       double& FL)
{
    const int row = j * s.nx;
    const bool interior = fl.per_x || (f >= 1 && f <= s.nx - 1);
    const double q = __ldg(P.qx + j * (s.nx + 1) + ((fl.per_x && f == s.nx) ? 0 : f));
    F = 0.0;
    FL = 0.0;
    if (interior) {
        if (q != 0.0) {
            double w[5];
            bool v[5];
            upwind5<1>(P.c + row, P.ok + row, 1, s.nx, fl.per_x, f, q >= 0.0, w, v);
            F = q * weno5_face<MIX>(w[0], w[1], w[2], w[3], w[4], v[0], v[1], v[2], v[3], v[4], ZV);
        }
        if (DONOR) {
            const int ff = f == s.nx ? 0 : f;
            const int fm = ff >= 1 ? ff - 1 : s.nx - 1;          // f >= 1 unless periodic
            FL = q * (q >= 0 ? __ldg(P.c0 + row + fm) : __ldg(P.c0 + row + ff));
        }
        return;
    }
    if (f == 0) {
        if (fl.open_w) {
            F = q * (q > 0.0 ? P.e[row] : P.c[row]);
            if (DONOR) FL = q * (q > 0 ? __ldg(P.e0 + row) : __ldg(P.c0 + row));
        }
    } else if (fl.open_e) {
        F = q * (q < 0.0 ? P.e[row + s.nx - 1] : P.c[row + s.nx - 1]);
        if (DONOR) FL = q * (q < 0 ? __ldg(P.e0 + row + s.nx - 1) : __ldg(P.c0 + row + s.nx - 1));
    }
}

template <bool ZV, bool MIX, bool DONOR>
__device__ __forceinline__ void y_face(const FacePlane& P, const Shape& s, const Flags& fl, int f, int i, double& F,
                                       double& FL)
{
    const bool interior = fl.per_y || (f >= 1 && f <= s.ny - 1);
    const double q = __ldg(P.qy + ((fl.per_y && f == s.ny) ? 0 : f) * s.nx + i);
    F = 0.0;
    FL = 0.0;
    if (interior) {
        if (q != 0.0) {
            double w[5];
            bool v[5];
            upwind5<0>(P.c + i, P.ok + i, s.nx, s.ny, fl.per_y, f, q >= 0.0, w, v);
            F = q * weno5_face<MIX>(w[0], w[1], w[2], w[3], w[4], v[0], v[1], v[2], v[3], v[4], ZV);
        }
        if (DONOR) {
            const int ff = f == s.ny ? 0 : f;
            const int fm = ff >= 1 ? ff - 1 : s.ny - 1;
            FL = q * (q >= 0 ? __ldg(P.c0 + fm * s.nx + i) : __ldg(P.c0 + ff * s.nx + i));
        }
        return;
    }
    if (f == 0) {
        if (fl.open_s) {
            F = q * (q > 0.0 ? P.e[i] : P.c[i]);
            if (DONOR) FL = q * (q > 0 ? __ldg(P.e0 + i) : __ldg(P.c0 + i));
        }
    } else if (fl.open_n) {
        const int o = (s.ny - 1) * s.nx + i;
        F = q * (q < 0.0 ? P.e[o] : P.c[o]);
        if (DONOR) FL = q * (q < 0 ? __ldg(P.e0 + o) : __ldg(P.c0 + o));
    }
}

// Store the stage's quantity of one face (S, T: the face arrays of this plane).  Stages 3 and 4 read the face's F0
// and F1 here, after the face computation: holding them across the WENO chains cost registers, and at the face
// passes' 32-register budget the spills outweighed the overlap (2.2 % of advect_fct at 512 x 512 x 50).
template <int STAGE>
__device__ __forceinline__ void put_face(double* S, double* T, int fo, double F, double FL)
{
    if (STAGE == 1) {
        S[fo] = F;
    } else if (STAGE == 2) {
        T[fo] = F;
    } else if (STAGE == 3) {
        S[fo] = (div6_exact(S[fo] + T[fo]) + div3_exact(2.0 * F)) - FL;
    } else {                     // the unlimited step: S <- the RK3 flux F_H = (F0 + F1)/6 + 2 F2/3
        S[fo] = div6_exact(S[fo] + T[fo]) + div3_exact(2.0 * F);
    }
}

// Face pass of stage STAGE for cell (t, k, j, i); blocks are 32 x TJR cells of one (t, k) plane, planes k-major (the
// tracers of a layer in a row share the layer's transports in L2).
template <int STAGE, bool ZV, bool MIX>
__device__ __forceinline__ void faces_body(const StepArgs& a, int t, int k, int i, int j)
{
    const Shape s = a.s;
    const Flags fl(a.flags);
    if (i >= s.nx || j >= s.ny) return;
    const int pl = s.ny * s.nx, xpl = s.ny * (s.nx + 1), ypl = (s.ny + 1) * s.nx, p = t * s.n + k;
    const i64 pc = plane_at(p, pl), pu = plane_at(p, xpl), pv = plane_at(p, ypl);
    FacePlane P;
    P.c = stage_field<STAGE>(a) + pc;
    P.e = a.inflow ? a.inflow + pc : P.c;
    P.c0 = a.C + pc;
    P.e0 = a.inflow ? a.inflow + pc : P.c0;
    P.ok = a.ok + plane_at(k, pl);
    P.qx = a.Qx + plane_at(k, xpl);
    P.qy = a.Qy + plane_at(k, ypl);
    P.sx = a.Sx + pu;
    P.sy = a.Sy + pv;
    P.tx = a.Tx + pu;
    P.ty = a.Ty + pv;
    const int fxo = j * (s.nx + 1) + i, fyo = j * s.nx + i;
    const bool last_x = i == s.nx - 1, last_y = j == s.ny - 1;
    double fw, lw, fs, ls, le = 0.0, ln = 0.0;
    x_face<ZV, MIX, STAGE == 3>(P, s, fl, j, i, fw, lw);
    y_face<ZV, MIX, STAGE == 3>(P, s, fl, j, i, fs, ls);
    put_face<STAGE>(P.sx, P.tx, fxo, fw, lw);
    put_face<STAGE>(P.sy, P.ty, fyo, fs, ls);
    if (last_x) {
        double fe;
        x_face<ZV, MIX, STAGE == 3>(P, s, fl, j, s.nx, fe, le);
        put_face<STAGE>(P.sx, P.tx, fxo + 1, fe, le);
    }
    if (last_y) {
        double fn;
        y_face<ZV, MIX, STAGE == 3>(P, s, fl, s.ny, i, fn, ln);
        put_face<STAGE>(P.sy, P.ty, fyo + s.nx, fn, ln);
    }
    if (STAGE == 3) {
        // c_L = safe(q0 - dt div F_L, V1) of this cell (sigma_baroclinic.py:509-511): the donor fluxes of its east
        // and north faces are recomputed here (they are its neighbours' west and south faces), so F_L is never
        // stored and no separate cell pass runs
        // faces i + 1 <= nx - 1 and j + 1 <= ny - 1 are interior on any axis (periodic or not)
        const double c0 = __ldg(P.c0 + fyo);
        if (!last_x) {
            const double q = __ldg(P.qx + fxo + 1);
            le = q * (q >= 0 ? c0 : __ldg(P.c0 + fyo + 1));
        }
        if (!last_y) {
            const double q = __ldg(P.qy + fyo + s.nx);
            ln = q * (q >= 0 ? c0 : __ldg(P.c0 + fyo + s.nx));
        }
        const double dl = le - lw + ln - ls;
        const i64 g = plane_at(k, pl) + fyo;
        const double v0 = __ldg(a.V0 + g), v1 = __ldg(a.V1 + g);
        const double q0 = v0 * c0;
        const double q = 0.0 * q0 + 1.0 * (q0 - a.dt * dl);
        a.q1[pc + fyo] = v1 > 0 ? q / v1 : c0;
    }
}

// Register budget of the face passes, as resident 256-thread blocks per SM (scaled for other block sizes): 7 for
// all three stages, which ptxas rounds to 32 registers and full occupancy (64 warps per SM; stages 1-2 and 3 spill
// a few values to L1).  Measured at 512 x 512 x 50: 2.0 % faster for advect_fct than 6 (40 registers), and 1.0 %
// faster than 32 registers for stages 1-2 with 40 for stage 3 or the reverse; 40 registers had been 8.5 % faster
// than ptxas's own choice (58 / 80 registers), whose lower occupancy left the FP64 chains and the loads exposed.
#ifndef POCEAN_FACES12_MINB
#define POCEAN_FACES12_MINB 7
#endif
#ifndef POCEAN_FACES3_MINB
#define POCEAN_FACES3_MINB 7
#endif
// The mixed-precision face passes (FP32 weights) hold fewer FP64 values: 7 blocks of 256 (1 % faster than 6; 5 and
// 8 slower).
#ifndef POCEAN_FACES12_MINB_MIX
#define POCEAN_FACES12_MINB_MIX 7
#endif
#ifndef POCEAN_FACES3_MINB_MIX
#define POCEAN_FACES3_MINB_MIX 7
#endif
#define FACES12_BOUNDS(n) __launch_bounds__(n, (MIX ? POCEAN_FACES12_MINB_MIX : POCEAN_FACES12_MINB) * 256 / (n))
#define FACES3_BOUNDS(n) __launch_bounds__(n, (MIX ? POCEAN_FACES3_MINB_MIX : POCEAN_FACES3_MINB) * 256 / (n))
template <int STAGE, bool ZV, bool MIX, int TJR>
__device__ __forceinline__ void faces_plane(const StepArgs& a)
{
    int k, t;
    split_plane(a.k0 * a.s.nt + blockIdx.z, a.s.nt, a.tdiv, k, t);
    faces_body<STAGE, ZV, MIX>(a, t, k, blockIdx.x * TI + threadIdx.x % TI, blockIdx.y * TJR + threadIdx.x / TI);
}

template <int STAGE, bool ZV, bool MIX, int TJR>
__global__ void FACES12_BOUNDS(TI * TJR) fct_faces_kernel(StepArgs a)
{
    faces_plane<STAGE, ZV, MIX, TJR>(a);
}

template <bool ZV, bool MIX, int TJR>
__global__ void FACES3_BOUNDS(TI * TJR) fct_faces3_kernel(StepArgs a)
{
    faces_plane<3, ZV, MIX, TJR>(a);
}

// Where a batched CTA works (domain d owns CTAs off[d] .. off[d+1]-1): its domain d, tracer t and layer k, and its
// 32 x TJR tile (bx, by).  The first thread of
// the CTA works it out (a binary search over the domains' CTA offsets and two integer divisions, the same for every
// thread of the CTA) and shares it, with the domain's argument block, through shared memory: done by every thread,
// that set-up cost the batched cell passes as many instructions again as their own work.
struct BlockTile {
    int d, t, k, bx, by;
};

// The CTA's tile (bt) and its domain's argument block (sh), both in shared memory.  PLANES: the CTA's index counts
// 32 x TJR tiles of the (t, k) planes (k-major: the stage passes); else tiles of the layers (t = 0: the coefficient
// and final passes).  Call before any thread returns: it contains block barriers.
template <bool PLANES, int TJR>
__device__ __forceinline__ const StepArgs& block_tile(const BatchDomain* __restrict__ doms, const int* __restrict__ off,
                                                      int ndom, BlockTile& bt, StepArgs& sh)
{
    if (threadIdx.x == 0) {
        const int d = find_domain(off, ndom, blockIdx.x);
        const Shape s = doms[d].a.s;
        const int tx = ceil_div(s.nx, TI), ty = ceil_div(s.ny, TJR);
        int local = blockIdx.x - __ldg(off + d);
        const int p = local / (tx * ty);
        local -= p * tx * ty;
        int t = 0, k = p;
        if (PLANES) split_plane(p, s.nt, doms[d].a.tdiv, k, t);
        const int by = local / tx;
        bt.d = d;
        bt.t = t;
        bt.k = k;
        bt.by = by;
        bt.bx = local - by * tx;
    }
    __syncthreads();
    return block_args(doms, bt.d, sh);
}

template <int STAGE, bool ZV, bool MIX, int TJR>
__device__ __forceinline__ void faces_batched_body(const BatchDomain* __restrict__ doms, const int* __restrict__ off,
                                                   int ndom)
{
    __shared__ BlockTile bt;
    __shared__ StepArgs sh;
    const StepArgs& a = block_tile<true, TJR>(doms, off, ndom, bt, sh);
    faces_body<STAGE, ZV, MIX>(a, bt.t, bt.k, bt.bx * TI + threadIdx.x % TI, bt.by * TJR + threadIdx.x / TI);
}

template <int STAGE, bool ZV, bool MIX, int TJR>
__global__ void FACES12_BOUNDS(TI * TJR) fct_faces_batched(const BatchDomain* __restrict__ doms,
                                                           const int* __restrict__ off, int ndom)
{
    faces_batched_body<STAGE, ZV, MIX, TJR>(doms, off, ndom);
}

template <bool ZV, bool MIX, int TJR>
__global__ void FACES3_BOUNDS(TI * TJR) fct_faces3_batched(const BatchDomain* __restrict__ doms,
                                                           const int* __restrict__ off, int ndom)
{
    faces_batched_body<3, ZV, MIX, TJR>(doms, off, ndom);
}

// Cell pass of stage STAGE = 1, 2 (sigma_baroclinic.py:452-468 `_fct_stage`); stage 3 has none (its face pass
// writes c_L); STAGE = 4 is the unlimited step's final update from the RK3 flux.
template <int STAGE>
__device__ __forceinline__ void update_body(const StepArgs& a, int t, int k, int i, int j)
{
    const Shape s = a.s;
    if (i >= s.nx || j >= s.ny) return;
    const int pl = s.ny * s.nx, p = t * s.n + k, ij = j * s.nx + i;
    const i64 w = plane_at(p, s.ny * (s.nx + 1)) + (j * (s.nx + 1) + i), so = plane_at(p, (s.ny + 1) * s.nx) + ij;
    const i64 g = plane_at(k, pl) + ij, cc = plane_at(p, pl) + ij;
    const double v0 = __ldg(a.V0 + g), v1 = __ldg(a.V1 + g), c0 = __ldg(a.C + cc);
    const double q0 = v0 * c0;
    if (STAGE == 1) {
        const double d = a.Sx[w + 1] - a.Sx[w] + a.Sy[so + s.nx] - a.Sy[so];
        const double q = 0.0 * q0 + 1.0 * (q0 - a.dt * d);
        const double v = v0 + (v1 - v0);
        a.c1[cc] = v > 0.0 ? q / v : c0;
    } else if (STAGE == 2) {
        const double d0 = a.Sx[w + 1] - a.Sx[w] + a.Sy[so + s.nx] - a.Sy[so];
        const double d = a.Tx[w + 1] - a.Tx[w] + a.Ty[so + s.nx] - a.Ty[so];
        const double q1 = 0.0 * q0 + 1.0 * (q0 - a.dt * d0);
        const double q = 0.75 * q0 + 0.25 * (q1 - a.dt * d);
        const double v = v0 + 0.5 * (v1 - v0);
        a.c2[cc] = v > 0.0 ? q / v : c0;
    } else if (STAGE == 4) {     // the unlimited step (tracers.py:289-291): C_out = safe(q0 - dt div F_H, V1)
        const double d = a.Sx[w + 1] - a.Sx[w] + a.Sy[so + s.nx] - a.Sy[so];
        if (a.fx_face != nullptr && i == (a.face_i == s.nx ? s.nx - 1 : a.face_i))
            a.fx_face[((i64)t * s.n + k) * s.ny + j] = a.face_i == s.nx ? a.Sx[w + 1] : a.Sx[w];
        const double q = q0 - a.dt * d;
        a.out[cc] = v1 > 0 ? q / v1 : c0;
    }
}

template <int STAGE, int TJR>
__global__ void __launch_bounds__(TI * TJR) fct_update_kernel(StepArgs a)
{
    int k, t;
    split_plane(a.k0 * a.s.nt + blockIdx.z, a.s.nt, a.tdiv, k, t);
    update_body<STAGE>(a, t, k, blockIdx.x * TI + threadIdx.x % TI, blockIdx.y * TJR + threadIdx.x / TI);
}

template <int STAGE, int TJR>
__global__ void __launch_bounds__(TI * TJR) fct_update_batched(const BatchDomain* __restrict__ doms,
                                                               const int* __restrict__ off, int ndom)
{
    __shared__ BlockTile bt;
    __shared__ StepArgs sh;
    const StepArgs& a = block_tile<true, TJR>(doms, off, ndom, bt, sh);
    update_body<STAGE>(a, bt.t, bt.k, bt.bx * TI + threadIdx.x % TI, bt.by * TJR + threadIdx.x / TI);
}

}  // namespace po
