// Warp-strip marching for the three WENO5 passes of the FCT step (included by advect.cu).
//
// Each warp owns one strip of 31 cells along i (lanes 0..30; lane 31 computes the strip's 32nd x-face, which is
// the east face of lane 30's cell) and a segment of SEG rows of one (t, k) plane, and marches in j.  Rows of the
// input field (columns i0-3 .. i0+33 with their validity bytes) pass through a per-warp ring of RING rows in
// shared memory: the row j+4 is loaded (coalesced) into registers while row j is computed and written to the ring
// one step later, so the ring holds rows j-3 .. j+3.  A lane's y-stencil is its ring column, its x-stencil six
// neighbouring ring entries of row j; both need only __syncwarp, never a block barrier, and the warp keeps just
// the in-flight row and the faces of the previous step in registers (a register budget that lets 32 warps share
// an SM, which the FP64 dependency chains of WENO5 need).  The cell update of row j-1 uses the x-faces of the
// previous step (the east one from lane+1 by shuffle) and the y-faces of the previous and current steps.
// Faces per cell: 32/31 in x and 32/31 (1 + 1/SEG) in y.  The arithmetic is the reference's (weno.cuh).
#pragma once

namespace po {

constexpr int STRIP = 31;            // cells per warp along i
constexpr int SEG = 64;              // default rows per warp segment (a launch parameter)
constexpr int SWARPS = 4;            // warps per CTA (independent)
constexpr int RXW = 40;              // ring row pitch (37 used: columns i0-3 .. i0+33)
constexpr int RING = 8;              // ring rows (rows j-3 .. j+3 plus the one being refilled)

// Resident CTAs per SM the register allocation is fitted to, per pass (stages 1 and 2 / stage 3).
#ifndef POCEAN_STRIP_CTAS_12
#define POCEAN_STRIP_CTAS_12 5
#endif
#ifndef POCEAN_STRIP_CTAS_3
#define POCEAN_STRIP_CTAS_3 8
#endif

struct StripSmem {
    double row[SWARPS][RING][RXW];
    uint8_t val[SWARPS][RING][RXW];
};

// Global row index of row r (periodic wrap, or -1 outside a closed/open domain).
__device__ __forceinline__ int row_of(int r, const Shape& s, const Flags& fl)
{
    if (fl.per_y) return wrap(r, s.ny);
    return (r >= 0 && r < s.ny) ? r : -1;
}

// One warp's work: (segment, strip) pair `pair` of plane p (k-major) of the domain described by `a`.
template <int STAGE, bool ZV, bool MIX>
__device__ __forceinline__ void strip_body(const StepArgs& a, StripSmem& SM, int seglen, int nstrips, int pair, int p)
{
    const Shape s = a.s;
    const Flags fl(a.flags);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int seg = pair / nstrips, strip = pair - seg * nstrips;
    const int i0 = strip * STRIP;
    const int jA = seg * seglen;
    const int jB = min(jA + seglen, s.ny);                     // cells jA..jB-1; y-faces jA..jB
    const int k = p / s.nt, t = p - k * s.nt;                  // k-major: the tracers of a layer in a row

    const i64 pc = s.cell(t, k, 0, 0);
    const i64 pg = s.geo(k, 0, 0);
    // plane base pointers: every per-step address below is a 32-bit offset from one of them
    const double* __restrict__ cin = (STAGE == 1 ? a.C : (STAGE == 2 ? a.c1 : a.c2)) + pc;
    const uint8_t* __restrict__ okk = a.ok + pg;
    const double* __restrict__ qxk = a.Qx + s.qx(k, 0, 0);
    const double* __restrict__ qyk = a.Qy + s.qy(k, 0, 0);
    const double* __restrict__ v0k = a.V0 + pg;
    const double* __restrict__ v1k = a.V1 + pg;
    const double* __restrict__ ck = a.C + pc;
    const double* __restrict__ ek = a.inflow ? a.inflow + pc : cin;
    double* __restrict__ sxk = a.Sx + s.ux(t, k, 0, 0);
    double* __restrict__ syk = a.Sy + s.vy(t, k, 0, 0);
    double* __restrict__ txk = a.Tx + s.ux(t, k, 0, 0);
    double* __restrict__ tyk = a.Ty + s.vy(t, k, 0, 0);
    const int nx1 = s.nx + 1;
    double* ring = &SM.row[warp][0][0];
    uint8_t* ringv = &SM.val[warp][0][0];

    // this lane's column (main) and, for lanes 0..4, its halo column of the ring row
    const int ci = i0 + lane;
    const int mcol = fl.per_x ? wrap(ci, s.nx) : (ci < s.nx ? ci : -1);
    int hslot = -1, hcol = -1;
    if (lane < 5) {
        hslot = lane < 3 ? lane : 32 + lane;                   // slots 0,1,2 (i0-3..i0-1) and 35,36 (i0+32, i0+33)
        const int hc = i0 - 3 + hslot;
        hcol = fl.per_x ? wrap(hc, s.nx) : ((hc >= 0 && hc < s.nx) ? hc : -1);
    }
    const bool has_x = ci <= s.nx;                              // x-face ci exists
    const bool x_interior = fl.per_x || (ci >= 1 && ci <= s.nx - 1);
    const int qx_col = (fl.per_x && ci == s.nx) ? 0 : ci;
    const bool has_col = ci < s.nx;                             // column ci exists (its y-faces, its cells)
    const bool cell_lane = lane < STRIP && has_col;

    auto load_row = [&](int r, double& mv, uint8_t& mo, double& hv, uint8_t& ho) {
        const int g = row_of(r, s, fl);
        mv = 0.0; mo = 0; hv = 0.0; ho = 0;
        if (g >= 0) {
            const int base = g * s.nx;
            if (mcol >= 0) { mv = __ldg(cin + base + mcol); mo = __ldg(okk + base + mcol); }
            if (hcol >= 0) { hv = __ldg(cin + base + hcol); ho = __ldg(okk + base + hcol); }
        }
    };
    auto slot_of = [&](int r) { return (r - jA + 8 * RING) % RING; };
    auto put_ring = [&](int r, double mv, uint8_t mo, double hv, uint8_t ho) {
        const int sl = slot_of(r);
        ring[sl * RXW + lane + 3] = mv;
        ringv[sl * RXW + lane + 3] = mo;
        if (hslot >= 0) {
            ring[sl * RXW + hslot] = hv;
            ringv[sl * RXW + hslot] = ho;
        }
    };

    // prologue: rows jA-3 .. jA+2 into the ring, row jA+3 in flight
    double in_mv, in_hv;
    uint8_t in_mo, in_ho;
#pragma unroll 1
    for (int r = jA - 3; r <= jA + 2; ++r) {
        load_row(r, in_mv, in_mo, in_hv, in_ho);
        put_ring(r, in_mv, in_mo, in_hv, in_ho);
    }
    load_row(jA + 3, in_mv, in_mo, in_hv, in_ho);

    // C, V0, V1 of this lane's cell are loaded one row ahead of the cell update; pass 3 also forms the donor fluxes
    // F_L of its faces from these values (left neighbour by shuffle, the row below from the previous step)
    const int lcol = fl.per_x ? wrap(i0 - 1, s.nx) : i0 - 1;  // lane 0's left neighbour column
    auto crow_at = [&](int r) -> double {
        const int g = row_of(r, s, fl);
        return (g >= 0 && mcol >= 0) ? __ldg(ck + g * s.nx + mcol) : 0.0;   // periodic: column nx is column 0
    };
    double c_prev = STAGE == 3 ? crow_at(jA - 1) : 0.0;     // C of row j-1 (pass 3: the cell below face j)
    double v0_prev = 0.0, v1_prev = 0.0;
    double flx_prev = 0.0, fly_prev = 0.0;

    // stage 2 recomputes q1 = q0 - dt div F0 from the F0 faces kept by stage 1 (the same arithmetic as the value
    // stage 1 formed), so q1 is never stored
    double fx_prev = 0.0, fy_prev = 0.0, f0x_prev = 0.0, f0y_prev = 0.0;
#pragma unroll 1
    for (int j = jA; j <= jB; ++j) {
        __syncwarp();
        // face transports of this step (and F0 in stage 2)
        const double qx = (j < jB && has_x) ? __ldg(qxk + j * nx1 + qx_col) : 0.0;
        const double qy = has_col ? __ldg(qyk + ((fl.per_y && j == s.ny) ? 0 : j) * s.nx + ci) : 0.0;
        double f0x = 0.0, f0y = 0.0;
        if (STAGE == 2) {
            f0x = (j < jB && has_x) ? sxk[j * nx1 + ci] : 0.0;
            f0y = has_col ? syk[j * s.nx + ci] : 0.0;
        }
        // C, V0, V1 of row j (used by the update of row j at the next step, and by pass 3's donor fluxes now)
        const double crow = (STAGE == 3 || j < jB) ? crow_at(j) : 0.0;
        const bool row_in = j < jB && has_col;
        const double v0row = row_in ? __ldg(v0k + j * s.nx + ci) : 0.0;
        const double v1row = row_in ? __ldg(v1k + j * s.nx + ci) : 0.0;
        double flx = 0.0, fly = 0.0;
        if (STAGE == 3) {
            // donor flux of x-face (j, ci) (sigma_baroclinic.py:486-494): left cell by shuffle (lane 0 loads it)
            double cleft = __shfl_up_sync(0xffffffffu, crow, 1);
            if (lane == 0) cleft = (lcol >= 0 && j < jB) ? __ldg(ck + j * s.nx + lcol) : 0.0;
            if (j < jB && has_x) {
                if (x_interior) {
                    flx = qx * (qx >= 0 ? cleft : crow);
                } else if (ci == 0) {
                    flx = fl.open_w ? qx * (qx > 0 ? __ldg(a.inflow ? a.inflow + pc + j * s.nx : ck + j * s.nx) : crow)
                                    : 0.0;
                } else {
                    flx = fl.open_e ? qx * (qx < 0 ? __ldg((a.inflow ? a.inflow + pc : ck) + j * s.nx + s.nx - 1)
                                                   : cleft)
                                    : 0.0;
                }
            }
            // donor flux of y-face (j, ci) (:498-507): the cell below from the previous step
            if (has_col) {
                if (fl.per_y || (j >= 1 && j <= s.ny - 1)) {
                    fly = qy * (qy >= 0 ? c_prev : crow);
                } else if (j == 0) {
                    fly = fl.open_s ? qy * (qy > 0 ? __ldg((a.inflow ? a.inflow + pc : ck) + ci) : crow) : 0.0;
                } else {
                    fly = fl.open_n ? qy * (qy < 0 ? __ldg((a.inflow ? a.inflow + pc : ck) + (s.ny - 1) * s.nx + ci)
                                                   : c_prev)
                                    : 0.0;
                }
            }
        }
        // x-face of row j (west face of column ci)
        double fx = 0.0;
        if (j < jB && has_x) {
            if (x_interior) {
                if (qx != 0.0) {
                    const int sl = slot_of(j);
                    fx = qx * upwind_face<MIX>(ring + sl * RXW + lane, ringv + sl * RXW + lane, 1, qx, ZV);
                }
            } else {
                const int row = j * s.nx;
                if (ci == 0) fx = fl.open_w ? qx * (qx > 0.0 ? ek[row] : cin[row]) : 0.0;
                else fx = fl.open_e ? qx * (qx < 0.0 ? ek[row + s.nx - 1] : cin[row + s.nx - 1]) : 0.0;
            }
        }
        // y-face j of this column: cells j-3 .. j+2 are ring rows
        double fy = 0.0;
        if (has_col) {
            if (fl.per_y || (j >= 1 && j <= s.ny - 1)) {
                if (qy != 0.0) {
                    const int s0 = slot_of(j - 3);
                    double w[6];
                    uint8_t v[6];
#pragma unroll
                    for (int m = 0; m < 6; ++m) {
                        const int sl = (s0 + m) & (RING - 1);
                        w[m] = ring[sl * RXW + lane + 3];
                        v[m] = ringv[sl * RXW + lane + 3];
                    }
                    fy = qy * upwind_face<MIX>(w, v, 1, qy, ZV);
                }
            } else {
                if (j == 0) {
                    fy = fl.open_s ? qy * (qy > 0.0 ? ek[ci] : cin[ci]) : 0.0;
                } else {
                    const int o = (s.ny - 1) * s.nx + ci;
                    fy = fl.open_n ? qy * (qy < 0.0 ? ek[o] : cin[o]) : 0.0;
                }
            }
        }
        // row j+3 enters the ring (its slot held row j-5, read for the last time two steps ago), row j+4 in flight
        put_ring(j + 3, in_mv, in_mo, in_hv, in_ho);
        if (j + 1 <= jB) load_row(j + 4, in_mv, in_mo, in_hv, in_ho);

        // cell update of row j-1: west fx_prev, east = lane+1's fx_prev, south fy_prev, north fy
        const double fx_east = __shfl_down_sync(0xffffffffu, fx_prev, 1);
        const double f0_east = STAGE == 2 ? __shfl_down_sync(0xffffffffu, f0x_prev, 1) : 0.0;
        const double fl_east = STAGE == 3 ? __shfl_down_sync(0xffffffffu, flx_prev, 1) : 0.0;
        if (j > jA && cell_lane) {
            const int jc = j - 1;
            const int w = jc * nx1 + ci, so = jc * s.nx + ci, cc = jc * s.nx + ci;
            const double v0 = v0_prev, v1 = v1_prev, c0 = c_prev;
            const double d = fx_east - fx_prev + fy - fy_prev;
            const double q0 = v0 * c0;
            if (STAGE == 1) {
                sxk[w] = fx_prev;
                syk[so] = fy_prev;
                if (ci == s.nx - 1) sxk[w + 1] = fx_east;
                if (jc == s.ny - 1) syk[so + s.nx] = fy;
                const double q = 0.0 * q0 + 1.0 * (q0 - a.dt * d);
                const double v = v0 + (v1 - v0);
                a.c1[pc + cc] = v > 0.0 ? q / v : c0;
            } else if (STAGE == 2) {
                txk[w] = div6_exact(f0x_prev + fx_prev);
                tyk[so] = div6_exact(f0y_prev + fy_prev);
                if (ci == s.nx - 1) txk[w + 1] = div6_exact(f0_east + fx_east);
                if (jc == s.ny - 1) tyk[so + s.nx] = div6_exact(f0y + fy);
                const double d0 = f0_east - f0x_prev + f0y - f0y_prev;
                const double q1 = 0.0 * q0 + 1.0 * (q0 - a.dt * d0);
                const double q = 0.75 * q0 + 0.25 * (q1 - a.dt * d);
                const double v = v0 + 0.5 * (v1 - v0);
                a.c2[pc + cc] = v > 0.0 ? q / v : c0;
            } else {
                const double flw = flx_prev, fle = fl_east, fls = fly_prev, fln = fly;
                sxk[w] = (txk[w] + div3_exact(2.0 * fx_prev)) - flw;
                syk[so] = (tyk[so] + div3_exact(2.0 * fy_prev)) - fls;
                if (ci == s.nx - 1) sxk[w + 1] = (txk[w + 1] + div3_exact(2.0 * fx_east)) - fle;
                if (jc == s.ny - 1) syk[so + s.nx] = (tyk[so + s.nx] + div3_exact(2.0 * fy)) - fln;
                const double dl = fle - flw + fln - fls;
                const double q = 0.0 * q0 + 1.0 * (q0 - a.dt * dl);
                a.q1[pc + cc] = v1 > 0 ? q / v1 : c0;          // c_L
            }
        }
        c_prev = crow;
        v0_prev = v0row;
        v1_prev = v1row;
        flx_prev = flx;
        fly_prev = fly;
        fx_prev = fx;
        fy_prev = fy;
        f0x_prev = f0x;
        f0y_prev = f0y;
    }
}

// Single-domain launch: blockIdx.x covers the (segment, strip) pairs SWARPS at a time, blockIdx.y the planes.
template <int STAGE, bool ZV, bool MIX>
__global__ void __launch_bounds__(SWARPS * 32, STAGE == 3 ? POCEAN_STRIP_CTAS_3 : POCEAN_STRIP_CTAS_12)
    fct_strip_kernel(StepArgs a, int seglen, int nstrips, int nsegs)
{
    __shared__ StripSmem SM;
    const int pair = blockIdx.x * SWARPS + (threadIdx.x >> 5);
    if (pair >= nstrips * nsegs) return;                       // whole warp leaves together
    strip_body<STAGE, ZV, MIX>(a, SM, seglen, nstrips, pair, blockIdx.y);
}

// Batched launch over many domains: domain d owns CTAs off[d] .. off[d+1]-1, each a block of SWARPS pairs of one
// of its planes.
template <int STAGE, bool ZV, bool MIX>
__global__ void __launch_bounds__(SWARPS * 32, STAGE == 3 ? POCEAN_STRIP_CTAS_3 : POCEAN_STRIP_CTAS_12)
    fct_strip_batched(const BatchDomain* __restrict__ doms, const int* __restrict__ off, int ndom)
{
    __shared__ StripSmem SM;
    const int d = find_domain(off, ndom, blockIdx.x);
    const BatchDomain& D = doms[d];
    const int local = blockIdx.x - __ldg(off + d);
    const int npairs = D.nstrips * D.nsegs;
    const int per_plane = (npairs + SWARPS - 1) / SWARPS;
    const int p = local / per_plane;
    const int pair = (local - p * per_plane) * SWARPS + (threadIdx.x >> 5);
    if (pair >= npairs) return;
    const StepArgs a = D.a;
    strip_body<STAGE, ZV, MIX>(a, SM, D.seglen, D.nstrips, pair, p);
}

}  // namespace po
