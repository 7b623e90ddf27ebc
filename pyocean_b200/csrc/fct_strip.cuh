// Warp-strip marching for the three WENO5 passes of the FCT step (included by advect.cu).
//
// Each warp owns one strip of 31 cells along i (lanes 0..30; lane 31 computes the strip's 32nd x-face, which is
// the east face of lane 30's cell) and a segment of SEG rows of one (t, k) plane, and marches in j:
//   * y-faces: every lane keeps the 6-cell y-stencil of its column in registers and slides it by one row a step,
//     so a y-face costs one new load;
//   * x-faces: the row being finished is staged in a small per-warp ring in shared memory (columns i0-3 .. i0+33,
//     read by the warp's own lanes after __syncwarp), one x-face per lane;
//   * row j+3 is loaded (coalesced) while row j is computed, and the cell update of row j-1 uses the x-faces of the
//     previous step (the east face from lane+1 by shuffle) and the y-faces of the previous and current steps.
// There is no block-level barrier: warps march independently.  Faces per cell: 32/31 x-faces and 32/31 +
// 1/SEG y-faces, against 2 + 1/32 + 1/8 for 32 x 8 tiles.  The arithmetic is the reference's (weno.cuh).
#pragma once

namespace po {

constexpr int STRIP = 31;            // cells per warp along i
constexpr int SEG = 32;              // rows per warp segment
constexpr int SWARPS = 4;            // warps per CTA (independent)
constexpr int RXW = 37;              // ring row: columns i0-3 .. i0+33
constexpr int RING = 4;              // ring rows

struct StripSmem {
    double row[SWARPS][RING][RXW + 3];
    uint8_t val[SWARPS][RING][RXW + 3];
};

// Upwind WENO5 face value from register stencils (cells f-3 .. f+2 in w0..w5, validity bits in vb bits 0..5).
__device__ __forceinline__ double upwind_face_reg(double w0, double w1, double w2, double w3, double w4, double w5,
                                                  unsigned vb, double q, bool z)
{
    const bool pos = q >= 0.0;
    const bool b0 = vb & 1u, b1 = vb & 2u, b2 = vb & 4u, b3 = vb & 8u, b4 = vb & 16u, b5 = vb & 32u;
    return weno5_value(pos ? w0 : w5, pos ? w1 : w4, pos ? w2 : w3, pos ? w3 : w2, pos ? w4 : w1,
                       pos ? b0 : b5, pos ? b1 : b4, pos ? b2 : b3, pos ? b3 : b2, pos ? b4 : b1, z);
}

// Global row index of row r (periodic wrap, or -1 outside a closed/open domain).
__device__ __forceinline__ int row_of(int r, const Shape& s, const Flags& fl)
{
    if (fl.per_y) return wrap(r, s.ny);
    return (r >= 0 && r < s.ny) ? r : -1;
}

template <int STAGE>
__global__ void __launch_bounds__(SWARPS * 32) fct_strip_kernel(StepArgs a)
{
    __shared__ StripSmem SM;
    const Shape s = a.s;
    const Flags fl(a.flags);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int strip = blockIdx.x * SWARPS + warp;
    const int i0 = strip * STRIP;
    if (i0 >= s.nx) return;                                   // whole warp leaves together
    const int jA = blockIdx.y * SEG;
    const int jB = min(jA + SEG, s.ny);                        // cells jA..jB-1; y-faces jA..jB
    const int p = blockIdx.z, k = p / s.nt, t = p - k * s.nt;   // k-major: the tracers of a layer in a row

    const double* cin = STAGE == 1 ? a.C : (STAGE == 2 ? a.c1 : a.c2);
    const double* cp = cin + s.cell(t, k, 0, 0);
    const double* ep = (a.inflow ? a.inflow : cin) + s.cell(t, k, 0, 0);
    const uint8_t* okp = a.ok + s.geo(k, 0, 0);
    const double* qxp = a.Qx + s.qx(k, 0, 0);
    const double* qyp = a.Qy + s.qy(k, 0, 0);
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
    // x-face of this lane: face f = ci (between cells ci-1 and ci)
    const bool has_x = ci <= s.nx;
    const bool x_interior = fl.per_x || (ci >= 1 && ci <= s.nx - 1);
    const int qx_col = (fl.per_x && ci == s.nx) ? 0 : ci;
    // y-faces of this lane's column exist for ci < nx
    const bool has_col = ci < s.nx;
    const bool cell_lane = lane < STRIP && has_col;

    auto load_row = [&](int r, double& mv, uint8_t& mo, double& hv, uint8_t& ho) {
        const int g = row_of(r, s, fl);
        mv = 0.0; mo = 0; hv = 0.0; ho = 0;
        if (g >= 0) {
            const i64 base = (i64)g * s.nx;
            if (mcol >= 0) { mv = __ldg(cp + base + mcol); mo = __ldg(okp + base + mcol); }
            if (hcol >= 0) { hv = __ldg(cp + base + hcol); ho = __ldg(okp + base + hcol); }
        }
    };
    auto put_ring = [&](int r, double mv, uint8_t mo, double hv, uint8_t ho) {
        const int slot = ((r % RING) + RING) % RING;
        ring[slot * (RXW + 3) + lane + 3] = mv;
        ringv[slot * (RXW + 3) + lane + 3] = mo;
        if (hslot >= 0) {
            ring[slot * (RXW + 3) + hslot] = hv;
            ringv[slot * (RXW + 3) + hslot] = ho;
        }
    };

    // prologue: y-window rows jA-3 .. jA+1 (slots 1..5 before the first shift), ring rows jA, jA+1, incoming jA+2
    double w0 = 0.0, w1, w2, w3, w4, w5;
    unsigned vb = 0;
    {
        double mv[5], hv[5];
        uint8_t mo[5], ho[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) load_row(jA - 3 + r, mv[r], mo[r], hv[r], ho[r]);
        w1 = mv[0]; w2 = mv[1]; w3 = mv[2]; w4 = mv[3]; w5 = mv[4];
        vb = ((unsigned)mo[0] << 1) | ((unsigned)mo[1] << 2) | ((unsigned)mo[2] << 3) | ((unsigned)mo[3] << 4) |
             ((unsigned)mo[4] << 5);
        put_ring(jA, mv[3], mo[3], hv[3], ho[3]);
        put_ring(jA + 1, mv[4], mo[4], hv[4], ho[4]);
    }
    double in_mv, in_hv;
    uint8_t in_mo, in_ho;
    load_row(jA + 2, in_mv, in_mo, in_hv, in_ho);
    // x- and y-face transports of the first step
    double qx_next = (has_x && jA < s.ny) ? __ldg(qxp + (i64)jA * (s.nx + 1) + qx_col) : 0.0;
    const int qy_row0 = (fl.per_y && jA == s.ny) ? 0 : jA;
    double qy_next = has_col ? __ldg(qyp + (i64)qy_row0 * s.nx + ci) : 0.0;

    // stage 2 recomputes q1 = q0 - dt div F0 from the F0 faces kept by stage 1 (the same arithmetic as the stored
    // value), so q1 is never stored; F0 of this lane's x-face of row j and y-face j are loaded one step ahead
    const double* f0x = a.Sx + s.ux(t, k, 0, 0);
    const double* f0y = a.Sy + s.vy(t, k, 0, 0);
    auto load_f0 = [&](int j, double& x, double& y) {
        x = (STAGE == 2 && has_x && j < s.ny) ? f0x[(i64)j * (s.nx + 1) + ci] : 0.0;
        y = (STAGE == 2 && has_col && j <= s.ny) ? f0y[(i64)j * s.nx + ci] : 0.0;
    };
    double f0x_next, f0y_next;
    load_f0(jA, f0x_next, f0y_next);

    double fx_prev = 0.0, fy_prev = 0.0, f0x_prev = 0.0, f0y_prev = 0.0;
    for (int j = jA; j <= jB; ++j) {
        // 1. slide the y-window: rows j-3 .. j+2
        w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = in_mv;
        vb = (vb >> 1) | ((unsigned)in_mo << 5);
        // 2. stage row j+2 in the ring
        put_ring(j + 2, in_mv, in_mo, in_hv, in_ho);
        // 3. loads for the next step
        const double qx_cur = qx_next, qy_cur = qy_next;
        const double f0x_cur = f0x_next, f0y_cur = f0y_next;
        if (j + 1 <= jB) {
            load_f0(j + 1, f0x_next, f0y_next);
            load_row(j + 3, in_mv, in_mo, in_hv, in_ho);
            const int jn = j + 1;
            qx_next = (has_x && jn < s.ny) ? __ldg(qxp + (i64)jn * (s.nx + 1) + qx_col) : 0.0;
            const int qyr = (fl.per_y && jn == s.ny) ? 0 : jn;
            qy_next = (has_col && jn <= s.ny) ? __ldg(qyp + (i64)qyr * s.nx + ci) : 0.0;
        }
        __syncwarp();
        // 4. x-face of row j (west face of column ci)
        double fx = 0.0;
        if (j < jB && has_x) {
            if (x_interior) {
                if (qx_cur != 0.0) {
                    const int slot = j % RING;
                    fx = qx_cur * upwind_face_value(ring + slot * (RXW + 3) + lane, ringv + slot * (RXW + 3) + lane,
                                                    1, qx_cur, fl.z);
                }
            } else {
                const i64 row = (i64)j * s.nx;
                if (ci == 0) fx = fl.open_w ? qx_cur * (qx_cur > 0.0 ? ep[row] : cp[row]) : 0.0;
                else fx = fl.open_e ? qx_cur * (qx_cur < 0.0 ? ep[row + s.nx - 1] : cp[row + s.nx - 1]) : 0.0;
            }
        }
        // 5. y-face j of this column
        double fy = 0.0;
        if (has_col) {
            if (fl.per_y || (j >= 1 && j <= s.ny - 1)) {
                if (qy_cur != 0.0) fy = qy_cur * upwind_face_reg(w0, w1, w2, w3, w4, w5, vb, qy_cur, fl.z);
            } else if (j == 0) {
                fy = fl.open_s ? qy_cur * (qy_cur > 0.0 ? ep[ci] : cp[ci]) : 0.0;
            } else {
                const i64 o = (i64)(s.ny - 1) * s.nx + ci;
                fy = fl.open_n ? qy_cur * (qy_cur < 0.0 ? ep[o] : cp[o]) : 0.0;
            }
        }
        // 6. cell update of row j-1 with faces: west fx_prev, east = lane+1's fx_prev, south fy_prev, north fy
        const double fx_east = __shfl_down_sync(0xffffffffu, fx_prev, 1);
        const double f0_east = __shfl_down_sync(0xffffffffu, f0x_prev, 1);
        if (j > jA && cell_lane) {
            const int jc = j - 1;
            const i64 w = s.ux(t, k, jc, ci), so = s.vy(t, k, jc, ci);
            const i64 g = s.geo(k, jc, ci), cc = s.cell(t, k, jc, ci);
            const double v0 = __ldg(a.V0 + g), v1 = __ldg(a.V1 + g), c0 = __ldg(a.C + cc);
            const double d = fx_east - fx_prev + fy - fy_prev;
            const double q0 = v0 * c0;
            if (STAGE == 1) {
                a.Sx[w] = fx_prev;
                a.Sy[so] = fy_prev;
                if (ci == s.nx - 1) a.Sx[w + 1] = fx_east;
                if (jc == s.ny - 1) a.Sy[so + s.nx] = fy;
                const double q = 0.0 * q0 + 1.0 * (q0 - a.dt * d);
                const double v = v0 + (v1 - v0);
                a.c1[cc] = v > 0.0 ? q / v : c0;
            } else if (STAGE == 2) {
                a.Tx[w] = div6_exact(f0x_prev + fx_prev);
                a.Ty[so] = div6_exact(f0y_prev + fy_prev);
                if (ci == s.nx - 1) a.Tx[w + 1] = div6_exact(f0_east + fx_east);
                if (jc == s.ny - 1) a.Ty[so + s.nx] = div6_exact(f0y_cur + fy);
                const double d0 = f0_east - f0x_prev + f0y_cur - f0y_prev;
                const double q1 = 0.0 * q0 + 1.0 * (q0 - a.dt * d0);
                const double q = 0.75 * q0 + 0.25 * (q1 - a.dt * d);
                const double v = v0 + 0.5 * (v1 - v0);
                a.c2[cc] = v > 0.0 ? q / v : c0;
            } else {
                const double* Cp = a.C + s.cell(t, k, 0, 0);
                const double* eL = a.inflow ? a.inflow + s.cell(t, k, 0, 0) : Cp;
                const double flw = donor_x(Cp, eL, a.Qx, s, fl, k, jc, ci);
                const double fle = donor_x(Cp, eL, a.Qx, s, fl, k, jc, ci + 1);
                const double fls = donor_y(Cp, eL, a.Qy, s, fl, k, jc, ci);
                const double fln = donor_y(Cp, eL, a.Qy, s, fl, k, jc + 1, ci);
                a.Sx[w] = (a.Tx[w] + div3_exact(2.0 * fx_prev)) - flw;
                a.Sy[so] = (a.Ty[so] + div3_exact(2.0 * fy_prev)) - fls;
                if (ci == s.nx - 1) a.Sx[w + 1] = (a.Tx[w + 1] + div3_exact(2.0 * fx_east)) - fle;
                if (jc == s.ny - 1) a.Sy[so + s.nx] = (a.Ty[so + s.nx] + div3_exact(2.0 * fy)) - fln;
                const double dl = fle - flw + fln - fls;
                const double q = 0.0 * q0 + 1.0 * (q0 - a.dt * dl);
                a.q1[cc] = v1 > 0 ? q / v1 : c0;               // c_L
            }
        }
        f0x_prev = f0x_cur;
        f0y_prev = f0y_cur;
        fx_prev = fx;
        fy_prev = fy;
    }
}

}  // namespace po
