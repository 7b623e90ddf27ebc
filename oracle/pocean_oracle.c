/*
 * CPU restatement of pyOCEAN's tracer hot path, written as the parity oracle of this repository.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (pyocean_b200/, libpocean_b200.so) links, loads or calls
 * this file; it is used by tests/, by __graft_entry__.smoke() as the checker, and by bench.py's CPU-baseline
 * leg ("port" of the reference's Numba kernels timed on the host cores).
 *
 * Every function restates one Numba kernel of the reference in plain C with the same expression order, so that,
 * compiled without FMA contraction (-ffp-contract=off) and without fast-math, it reproduces the reference's FP64
 * results bit for bit (pinned against golden vectors generated from the reference, tests/golden/).
 * Parallelism mirrors the reference's `prange` loops with OpenMP (results do not depend on the thread count).
 *
 * Layouts (C order, k = 0 at the bed): stacks (nt, n, ny, nx); geometry (n, ny, nx); u-faces (.., ny, nx+1);
 * v-faces (.., ny+1, nx); `ok` is one byte per cell (0/1).
 *
 * Reference files (paths inside the pyOCEAN project):
 *   core/dynamics/sigma_baroclinic.py  _wval :204-233, _advect_faces_h :265-321, _advect_div :324-364,
 *                                      _fct_coeff_kernel :407-449, _fct_stage :452-468, _fct_fluxes :471-511,
 *                                      _fct_final :514-530, _rk_stage :856-875
 *   core/components/tracers.py         TracerAdvection.advect_fct :208-254 (orchestration in oracle.py)
 *   core/vertical/remap.py             remap_column :306-397 and its helpers :46-303, _remap_columns :400-415
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t i64;

/* Python's builtin max/min on two floats: the first argument unless the second is strictly larger/smaller. */
static inline double pmax(double a, double b) { return (b > a) ? b : a; }
static inline double pmin(double a, double b) { return (b < a) ? b : a; }

/* ------------------------------------------------------------------------------------------------------------
 * WENO5 face value (sigma_baroclinic.py:204-233, `_wval`).  v3 is the upwind cell; k1..k5 validity flags.
 * ---------------------------------------------------------------------------------------------------------- */
static inline double wval(double v1, double v2, double v3, double v4, double v5,
                          int k1, int k2, int k3, int k4, int k5, int z_variant)
{
    if (k1 && k2 && k3 && k4 && k5) {
        double q0 = (2 * v1 - 7 * v2 + 11 * v3) / 6;
        double q1 = (-v2 + 5 * v3 + 2 * v4) / 6;
        double q2 = (2 * v3 + 5 * v4 - v5) / 6;
        double d;
        d = v1 - 2 * v2 + v3;  double e = v1 - 4 * v2 + 3 * v3;
        double b0 = (13.0 / 12.0) * (d * d) + 0.25 * (e * e);
        d = v2 - 2 * v3 + v4;  e = v2 - v4;
        double b1 = (13.0 / 12.0) * (d * d) + 0.25 * (e * e);
        d = v3 - 2 * v4 + v5;  e = 3 * v3 - 4 * v4 + v5;
        double b2 = (13.0 / 12.0) * (d * d) + 0.25 * (e * e);
        double a0, a1, a2;
        if (z_variant) {
            double tau = fabs(b2 - b0), ez = 1e-40;
            a0 = 0.1 * (1 + tau / (ez + b0));
            a1 = 0.6 * (1 + tau / (ez + b1));
            a2 = 0.3 * (1 + tau / (ez + b2));
        } else {
            double s0 = 1e-6 + b0, s1 = 1e-6 + b1, s2 = 1e-6 + b2;
            a0 = 0.1 / (s0 * s0);
            a1 = 0.6 / (s1 * s1);
            a2 = 0.3 / (s2 * s2);
        }
        return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
    }
    if (k2 && k3 && k4) {
        double c0 = (-v2 + 3 * v3) / 2, c1 = (v3 + v4) / 2;
        double s0 = 1e-6 + (v3 - v2) * (v3 - v2), s1 = 1e-6 + (v4 - v3) * (v4 - v3);
        double e0 = (1.0 / 3.0) / (s0 * s0);
        double e1 = (2.0 / 3.0) / (s1 * s1);
        return (e0 * c0 + e1 * c1) / (e0 + e1);
    }
    return v3;
}

/* Upwind-ordered 5-cell stencil of face f (between cells f-1 and f) of a line of n cells with stride `st`. */
static inline double face_line(const double* c, const uint8_t* ok, i64 st, int n, int f, double q, int z)
{
    int i1, i2, i3, i4, i5;
    if (q >= 0.0) { i1 = f - 3; i2 = f - 2; i3 = f - 1; i4 = f; i5 = f + 1; }
    else          { i1 = f + 2; i2 = f + 1; i3 = f;     i4 = f - 1; i5 = f - 2; }
    int b1 = 0 <= i1 && i1 < n, b2 = 0 <= i2 && i2 < n, b3 = 0 <= i3 && i3 < n, b4 = 0 <= i4 && i4 < n,
        b5 = 0 <= i5 && i5 < n;
    return wval(b1 ? c[i1 * st] : 0.0, b2 ? c[i2 * st] : 0.0, b3 ? c[i3 * st] : 0.0, b4 ? c[i4 * st] : 0.0,
                b5 ? c[i5 * st] : 0.0, b1 && ok[i1 * st], b2 && ok[i2 * st], b3 && ok[i3 * st],
                b4 && ok[i4 * st], b5 && ok[i5 * st], z);
}

/* sigma_baroclinic.py:265-321 `_advect_faces_h`.  fx (nt,n,ny,nx+1), fy (nt,n,ny+1,nx) are fully written. */
void oracle_advect_faces_h(const double* c, const double* Qx, const double* Qy, const uint8_t* ok,
                           const double* ext, int nt, int n, int ny, int nx, int open_w, int open_e, int open_s,
                           int open_n, int z_variant, double* fx, double* fy)
{
    const i64 cs = (i64)ny * nx, xs = (i64)ny * (nx + 1), ys = (i64)(ny + 1) * nx;
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < (i64)nt * n; ++p) {
        int t = (int)(p / n), k = (int)(p % n);
        const double* cp = c + p * cs;
        const double* ep = ext + p * cs;
        const uint8_t* op = ok + (i64)k * cs;
        double* fxp = fx + p * xs;
        double* fyp = fy + p * ys;
        const double* qx = Qx + (i64)k * xs;
        const double* qy = Qy + (i64)k * ys;
        (void)t;
        memset(fxp, 0, sizeof(double) * xs);
        memset(fyp, 0, sizeof(double) * ys);
        for (int j = 0; j < ny; ++j) {
            const double* row = cp + (i64)j * nx;
            const uint8_t* orow = op + (i64)j * nx;
            for (int i = 1; i < nx; ++i) {
                double q = qx[(i64)j * (nx + 1) + i];
                if (q == 0.0) continue;
                double v = face_line(row, orow, 1, nx, i, q, z_variant);
                fxp[(i64)j * (nx + 1) + i] = q * v;
            }
            double q = qx[(i64)j * (nx + 1)];
            if (open_w) fxp[(i64)j * (nx + 1)] = q * (q > 0.0 ? ep[(i64)j * nx] : row[0]);
            q = qx[(i64)j * (nx + 1) + nx];
            if (open_e) fxp[(i64)j * (nx + 1) + nx] = q * (q < 0.0 ? ep[(i64)j * nx + nx - 1] : row[nx - 1]);
        }
        for (int j = 1; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) {
                double q = qy[(i64)j * nx + i];
                if (q == 0.0) continue;
                double v = face_line(cp + i, op + i, nx, ny, j, q, z_variant);
                fyp[(i64)j * nx + i] = q * v;
            }
        }
        for (int i = 0; i < nx; ++i) {
            double q = qy[i];
            if (open_s) fyp[i] = q * (q > 0.0 ? ep[i] : cp[i]);
            q = qy[(i64)ny * nx + i];
            if (open_n) fyp[(i64)ny * nx + i] = q * (q < 0.0 ? ep[(i64)(ny - 1) * nx + i] : cp[(i64)(ny - 1) * nx + i]);
        }
    }
}

/* sigma_baroclinic.py:324-364 `_advect_div`: out = -div(F) with WENO5 faces in x, y and (if vert) z. */
void oracle_advect_div(const double* c, const double* Qx, const double* Qy, const double* Fz, const uint8_t* ok,
                       const double* ext, int nt, int n, int ny, int nx, int open_w, int open_e, int open_s,
                       int open_n, int z_variant, int vert, double* out)
{
    const i64 cs = (i64)ny * nx, xs = (i64)ny * (nx + 1), ys = (i64)(ny + 1) * nx;
    double* fx = (double*)malloc(sizeof(double) * (size_t)(nt * (i64)n * xs));
    double* fy = (double*)malloc(sizeof(double) * (size_t)(nt * (i64)n * ys));
    double* fz = vert ? (double*)calloc((size_t)(nt * (i64)(n + 1) * cs), sizeof(double)) : NULL;
    oracle_advect_faces_h(c, Qx, Qy, ok, ext, nt, n, ny, nx, open_w, open_e, open_s, open_n, z_variant, fx, fy);
    if (vert) {
#pragma omp parallel for schedule(static)
        for (i64 p = 0; p < (i64)nt * ny; ++p) {
            int t = (int)(p / ny), j = (int)(p % ny);
            for (int k = 1; k < n; ++k) {
                for (int i = 0; i < nx; ++i) {
                    double q = Fz[(i64)k * cs + (i64)j * nx + i];
                    if (q == 0.0) continue;
                    const double* col = c + (i64)t * n * cs + (i64)j * nx + i;
                    const uint8_t* ocol = ok + (i64)j * nx + i;
                    double v = face_line(col, ocol, cs, n, k, q, z_variant);
                    fz[((i64)t * (n + 1) + k) * cs + (i64)j * nx + i] = q * v;
                }
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < (i64)nt * n; ++p) {
        int t = (int)(p / n), k = (int)(p % n);
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) {
                const double* fxr = fx + p * xs + (i64)j * (nx + 1);
                const double* fyr = fy + p * ys;
                double d = fxr[i + 1] - fxr[i] + fyr[(i64)(j + 1) * nx + i] - fyr[(i64)j * nx + i];
                if (vert) {
                    const double* fzt = fz + (i64)t * (n + 1) * cs;
                    d = d + fzt[(i64)(k + 1) * cs + (i64)j * nx + i] - fzt[(i64)k * cs + (i64)j * nx + i];
                }
                out[p * cs + (i64)j * nx + i] = -d;
            }
        }
    }
    free(fx); free(fy); free(fz);
}

/* sigma_baroclinic.py:856-875 `_rk_stage` (flattened arrays; V broadcast over tracers). */
void oracle_rk_stage(const double* qa, const double* qb, const double* r, double dt, const double* V,
                     const double* C, int stage, i64 size, i64 nv, double* q_out, double* c_out)
{
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < size; ++p) {
        double q;
        if (stage == 1)      q = qa[p] + dt * r[p];
        else if (stage == 2) q = 0.75 * qa[p] + 0.25 * (qb[p] + dt * r[p]);
        else                 q = qa[p] / 3.0 + 2.0 / 3.0 * (qb[p] + dt * r[p]);
        q_out[p] = q;
        double v = V[p % nv];
        c_out[p] = v > 0 ? q / v : C[p];
    }
}

/* sigma_baroclinic.py:452-468 `_fct_stage`. */
void oracle_fct_stage(const double* q0, const double* qp, const double* fx, const double* fy, double a, double b,
                      double dt, const double* V, const double* C, int nt, int n, int ny, int nx,
                      double* q_out, double* c_out)
{
    const i64 cs = (i64)ny * nx, xs = (i64)ny * (nx + 1), ys = (i64)(ny + 1) * nx;
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < (i64)nt * n; ++p) {
        int k = (int)(p % n);
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) {
                i64 ci = p * cs + (i64)j * nx + i;
                const double* fxr = fx + p * xs + (i64)j * (nx + 1);
                const double* fyr = fy + p * ys;
                double d = fxr[i + 1] - fxr[i] + fyr[(i64)(j + 1) * nx + i] - fyr[(i64)j * nx + i];
                double q = a * q0[ci] + b * (qp[ci] - dt * d);
                q_out[ci] = q;
                double v = V[(i64)k * cs + (i64)j * nx + i];
                c_out[ci] = v > 0 ? q / v : C[ci];
            }
        }
    }
}

/* sigma_baroclinic.py:471-511 `_fct_fluxes`: donor flux F_L and antidiffusive flux A = F_H - F_L. */
void oracle_fct_fluxes(const double* c, const double* Qx, const double* Qy, const double* ext, int nt, int n,
                       int ny, int nx, int open_w, int open_e, int open_s, int open_n,
                       const double* fx0, const double* fy0, const double* fx1, const double* fy1,
                       const double* fx2, const double* fy2, double* FLx, double* FLy, double* Ax, double* Ay)
{
    const i64 cs = (i64)ny * nx, xs = (i64)ny * (nx + 1), ys = (i64)(ny + 1) * nx;
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < (i64)nt * n; ++p) {
        int k = (int)(p % n);
        const double* cp = c + p * cs;
        const double* ep = ext + p * cs;
        const double* qx = Qx + (i64)k * xs;
        const double* qy = Qy + (i64)k * ys;
        double* flx = FLx + p * xs; double* fly = FLy + p * ys;
        double* ax = Ax + p * xs;   double* ay = Ay + p * ys;
        memset(flx, 0, sizeof(double) * xs);
        memset(fly, 0, sizeof(double) * ys);
        for (int j = 0; j < ny; ++j) {
            i64 r = (i64)j * (nx + 1);
            for (int f = 1; f < nx; ++f) {
                double q = qx[r + f];
                flx[r + f] = q * (q >= 0 ? cp[(i64)j * nx + f - 1] : cp[(i64)j * nx + f]);
            }
            double q = qx[r];
            if (open_w) flx[r] = q * (q > 0 ? ep[(i64)j * nx] : cp[(i64)j * nx]);
            q = qx[r + nx];
            if (open_e) flx[r + nx] = q * (q < 0 ? ep[(i64)j * nx + nx - 1] : cp[(i64)j * nx + nx - 1]);
            for (int f = 0; f <= nx; ++f) {
                double fh = (fx0[p * xs + r + f] + fx1[p * xs + r + f]) / 6.0 + 2.0 * fx2[p * xs + r + f] / 3.0;
                ax[r + f] = fh - flx[r + f];
            }
        }
        for (int i = 0; i < nx; ++i) {
            for (int f = 1; f < ny; ++f) {
                double q = qy[(i64)f * nx + i];
                fly[(i64)f * nx + i] = q * (q >= 0 ? cp[(i64)(f - 1) * nx + i] : cp[(i64)f * nx + i]);
            }
            double q = qy[i];
            if (open_s) fly[i] = q * (q > 0 ? ep[i] : cp[i]);
            q = qy[(i64)ny * nx + i];
            if (open_n) fly[(i64)ny * nx + i] = q * (q < 0 ? ep[(i64)(ny - 1) * nx + i] : cp[(i64)(ny - 1) * nx + i]);
            for (int f = 0; f <= ny; ++f) {
                i64 o = (i64)f * nx + i;
                double fh = (fy0[p * ys + o] + fy1[p * ys + o]) / 6.0 + 2.0 * fy2[p * ys + o] / 3.0;
                ay[o] = fh - fly[o];
            }
        }
    }
}

/* sigma_baroclinic.py:407-449 `_fct_coeff_kernel`: Zalesak coefficients Cx, Cy (fully written). */
void oracle_fct_coeff(const double* c0, const double* cL, const double* V1, const double* Ax, const double* Ay,
                      const uint8_t* ok, double dt, int nt, int n, int ny, int nx, double* Cx, double* Cy)
{
    const i64 cs = (i64)ny * nx, xs = (i64)ny * (nx + 1), ys = (i64)(ny + 1) * nx;
    double* r_in = (double*)calloc((size_t)(nt * (i64)n * cs), sizeof(double));
    double* r_out = (double*)calloc((size_t)(nt * (i64)n * cs), sizeof(double));
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < (i64)nt * n; ++p) {
        int t = (int)(p / n), k = (int)(p % n);
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) {
                if (!ok[(i64)k * cs + (i64)j * nx + i]) continue;
                double cmax = -INFINITY, cmin = INFINITY;
                const int kk[7] = {k, k, k, k, k, k - 1, k + 1};
                const int jj[7] = {j, j, j, j - 1, j + 1, j, j};
                const int ii[7] = {i, i - 1, i + 1, i, i, i, i};
                for (int s = 0; s < 7; ++s) {
                    if (0 <= kk[s] && kk[s] < n && 0 <= jj[s] && jj[s] < ny && 0 <= ii[s] && ii[s] < nx &&
                        ok[(i64)kk[s] * cs + (i64)jj[s] * nx + ii[s]]) {
                        i64 o = ((i64)t * n + kk[s]) * cs + (i64)jj[s] * nx + ii[s];
                        /* max(cmax, c0, cL) / min(cmin, c0, cL) as Python's 3-argument max/min */
                        cmax = pmax(pmax(cmax, c0[o]), cL[o]);
                        cmin = pmin(pmin(cmin, c0[o]), cL[o]);
                    }
                }
                const double* ax = Ax + p * xs + (i64)j * (nx + 1);
                const double* ay = Ay + p * ys;
                double axw = ax[i], axe = ax[i + 1], ays = ay[(i64)j * nx + i], ayn = ay[(i64)(j + 1) * nx + i];
                double p_in = dt * (pmax(axw, 0.0) - pmin(axe, 0.0) + pmax(ays, 0.0) - pmin(ayn, 0.0));
                double p_out = dt * (pmax(axe, 0.0) - pmin(axw, 0.0) + pmax(ayn, 0.0) - pmin(ays, 0.0));
                i64 ci = p * cs + (i64)j * nx + i;
                double v1 = V1[(i64)k * cs + (i64)j * nx + i];
                double q_in = pmax(v1 * (cmax - cL[ci]), 0.0);
                double q_out = pmax(v1 * (cL[ci] - cmin), 0.0);
                r_in[ci] = p_in > 0.0 ? pmin(1.0, q_in / p_in) : 0.0;
                r_out[ci] = p_out > 0.0 ? pmin(1.0, q_out / p_out) : 0.0;
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < (i64)nt * n; ++p) {
        const double* ri = r_in + p * cs; const double* ro = r_out + p * cs;
        double* cx = Cx + p * xs; double* cy = Cy + p * ys;
        const double* ax = Ax + p * xs; const double* ay = Ay + p * ys;
        memset(cx, 0, sizeof(double) * xs);
        memset(cy, 0, sizeof(double) * ys);
        for (int j = 0; j < ny; ++j) {
            for (int f = 1; f < nx; ++f) {
                i64 o = (i64)j * (nx + 1) + f, c = (i64)j * nx + f;
                cx[o] = ax[o] >= 0.0 ? pmin(ri[c], ro[c - 1]) : pmin(ri[c - 1], ro[c]);
            }
        }
        for (int f = 1; f < ny; ++f) {
            for (int i = 0; i < nx; ++i) {
                i64 o = (i64)f * nx + i;
                cy[o] = ay[o] >= 0.0 ? pmin(ri[o], ro[o - nx]) : pmin(ri[o - nx], ro[o]);
            }
        }
    }
    free(r_in); free(r_out);
}

/* sigma_baroclinic.py:514-530 `_fct_final`. */
void oracle_fct_final(const double* q0, const double* FLx, const double* FLy, const double* Ax, const double* Ay,
                      const double* Cx, const double* Cy, double dt, const double* V1, const double* C, int nt,
                      int n, int ny, int nx, double* out)
{
    const i64 cs = (i64)ny * nx, xs = (i64)ny * (nx + 1), ys = (i64)(ny + 1) * nx;
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < (i64)nt * n; ++p) {
        int k = (int)(p % n);
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) {
                i64 e = p * xs + (i64)j * (nx + 1) + i + 1, w = e - 1;
                i64 nn = p * ys + (i64)(j + 1) * nx + i, s = p * ys + (i64)j * nx + i;
                double d = (FLx[e] + Cx[e] * Ax[e]
                            - (FLx[w] + Cx[w] * Ax[w])
                            + (FLy[nn] + Cy[nn] * Ay[nn])
                            - (FLy[s] + Cy[s] * Ay[s]));
                i64 ci = p * cs + (i64)j * nx + i;
                double q = q0[ci] - dt * d;
                double v = V1[(i64)k * cs + (i64)j * nx + i];
                out[ci] = v > 0 ? q / v : C[ci];
            }
        }
    }
}

/* ============================================================================================================
 * Vertical remap (core/vertical/remap.py)
 * ========================================================================================================== */
enum { PCM = 0, PLM = 1, PPM_H4 = 2 };
#define H_NEGLECT 1e-30
#define H_NEGLECT_EDGE 1e-10
#define H_MIN_FRAC 1e-5
static const double EPS = 2.220446049250313e-16;   /* np.finfo(np.float64).eps */

/* remap.py:46-53 */
static int effective_scheme(int n_active, int scheme)
{
    if (n_active <= 1) return PCM;
    if (n_active <= 3 && scheme > PLM) return PLM;
    return scheme;
}

/* remap.py:59-80 */
static double plm_slope_wa(double h_l, double h_c, double h_r, double h_neglect, double u_l, double u_c, double u_r)
{
    double sigma_r = u_r - u_c;
    double sigma_l = u_c - u_l;
    double sigma_c = 2.0 * (u_r - u_l) * (h_c / (h_l + 2.0 * h_c + h_r + h_neglect));
    double u_min = pmin(pmin(u_l, u_c), u_r);
    double u_max = pmax(pmax(u_l, u_c), u_r);
    double slope;
    if (sigma_l * sigma_r > 0.0) {
        double s = pmin(fabs(sigma_c), 2.0 * pmin(u_c - u_min, u_max - u_c));
        slope = sigma_c >= 0.0 ? s : -s;
    } else {
        slope = 0.0;
    }
    if (u_c - 0.5 * fabs(slope) < u_min || u_c + 0.5 * fabs(slope) > u_max) slope = slope * (1.0 - EPS);
    if (fabs(slope) < 1e-140) slope = 0.0;
    return slope;
}

/* remap.py:83-97 */
static double plm_monotonized_slope(double u_l, double u_c, double u_r, double s_l, double s_c, double s_r)
{
    double almost_two = 2.0 * (1.0 - EPS);
    double e_r = u_l + 0.5 * s_l;
    double e_l = u_r - 0.5 * s_r;
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

/* remap.py:103-156 `_end_values_h4`: (C(0), C(dz[0])). */
static void end_values_h4(const double* dz, const double* u, double* e0, double* e1)
{
    double min_frac = 1.0e-6;
    double h1 = dz[0], h2 = dz[1], h3 = dz[2], h4 = dz[3];
    if ((h2 + h3) < min_frac * h1) h3 = min_frac * h1 - h2;
    if ((h3 + h4) < min_frac * h1) h4 = min_frac * h1 - h3;
    double h12 = h1 + h2, h23 = h2 + h3, h34 = h3 + h4;
    double h123 = h12 + h3, h234 = h2 + h34, h1234 = h12 + h34;
    double I_denB3 = 1.0 / (h123 * h12 * h23);
    double I_h12 = (h123 * h23) * I_denB3;
    double I_h23 = (h12 * h123) * I_denB3;
    double I_h123 = (h12 * h23) * I_denB3;
    double I_denom = 1.0 / (h1234 * (h234 * h34));
    double I_h234 = (h1234 * h34) * I_denom;
    double I_h1234 = (h234 * h34) * I_denom;

    double w11 = -h1 * (I_h1234 + I_h123 + I_h12);
    double w21 = h1 * h12 * (I_h234 * I_h1234 + I_h23 * (I_h234 + I_h123));
    double w31 = -h1 * h12 * h123 * I_denom;
    double w12 = 2.0 * (I_h12 * (1.0 + (h1 + h12) * (I_h1234 + I_h123)) + h1 * I_h1234 * I_h123);
    double w22 = -2.0 * ((h1 * h12 * I_h1234) * (I_h23 * (I_h234 + I_h123))
                         + (h1 + h12) * (I_h1234 * I_h234 + I_h23 * (I_h234 + I_h123)));
    double w32 = 2.0 * ((h1 + h12) * h123 + h1 * h12) * I_denom;
    double w13 = -3.0 * I_h12 * I_h123 * (1.0 + I_h1234 * ((h1 + h12) + h123));
    double w23 = 3.0 * I_h23 * (I_h123 + I_h1234 * ((h1 + h12) + h123) * (I_h123 + I_h234));
    double w33 = -3.0 * ((h1 + h12) + h123) * I_denom;
    double w14 = 4.0 * I_h1234 * I_h123 * I_h12;
    double w24 = -4.0 * I_h1234 * (I_h23 * (I_h123 + I_h234));
    double w34 = 4.0 * I_denom;

    double d1 = u[1] - u[0], d2 = u[2] - u[1], d3 = u[3] - u[2];
    double c0 = ((u[0] + (w11 * d1)) + (w21 * d2)) + (w31 * d3);
    double c1 = ((w12 * d1) + (w22 * d2)) + (w32 * d3);
    double c2 = ((w13 * d1) + (w23 * d2)) + (w33 * d3);
    double c3 = ((w14 * d1) + (w24 * d2)) + (w34 * d3);
    double d = dz[0];
    *e0 = c0;
    *e1 = c0 + d * (c1 + d * (c2 + d * c3));
}

/* remap.py:159-196 `_edges_h4`; e is (n, 2). */
static void edges_h4(const double* h, const double* u, int n, double h_neglect, double* e)
{
    for (int i = 2; i < n - 1; ++i) {
        double h0 = h[i - 2], h1 = h[i - 1], h2 = h[i], h3 = h[i + 1];
        if (h0 + h1 == 0.0 || h1 + h2 == 0.0 || h2 + h3 == 0.0) {
            double h_min = H_MIN_FRAC * pmax(h_neglect, (h0 + h1) + (h2 + h3));
            h0 = pmax(h_min, h0); h1 = pmax(h_min, h1); h2 = pmax(h_min, h2); h3 = pmax(h_min, h3);
        }
        double I_h12 = 1.0 / (h1 + h2);
        double I_den_et2 = 1.0 / (((h0 + h1) + h2) * (h0 + h1));
        double I_h012 = (h0 + h1) * I_den_et2;
        double I_den_et3 = 1.0 / ((h1 + (h2 + h3)) * (h2 + h3));
        double I_h123 = (h2 + h3) * I_den_et3;
        double et1 = ((1.0 + (h1 * I_h012 + (h0 + h1) * I_h123)) * I_h12 * (h2 * (h2 + h3)) * u[i - 1]
                      + (1.0 + (h2 * I_h123 + (h2 + h3) * I_h012)) * I_h12 * (h1 * (h0 + h1)) * u[i]);
        double et2 = (h1 * (h2 * (h2 + h3)) * I_den_et2) * (u[i - 1] - u[i - 2]);
        double et3 = (h2 * (h1 * (h0 + h1)) * I_den_et3) * (u[i] - u[i + 1]);
        e[2 * i + 0] = (et1 + (et2 + et3)) / ((h0 + h1) + (h2 + h3));
        e[2 * (i - 1) + 1] = e[2 * i + 0];
    }
    double dz[4], ut[4];
    for (int i = 0; i < 4; ++i) { dz[i] = pmax(h_neglect, h[i]); ut[i] = u[i]; }
    end_values_h4(dz, ut, &e[0], &e[1]);
    e[2 * 1 + 0] = e[1];
    for (int i = 0; i < 4; ++i) { dz[i] = pmax(h_neglect, h[n - 1 - i]); ut[i] = u[n - 1 - i]; }
    end_values_h4(dz, ut, &e[2 * (n - 1) + 1], &e[2 * (n - 1) + 0]);
    e[2 * (n - 2) + 1] = e[2 * (n - 1) + 0];
}

/* remap.py:199-220 `_bound_edges`. */
static void bound_edges(const double* h, const double* u, int n, double* e)
{
    for (int k = 0; k < n; ++k) {
        int km1 = k - 1 > 0 ? k - 1 : 0;
        int kp1 = k + 1 < n - 1 ? k + 1 : n - 1;
        double slope_x_h = 0.0;
        if ((h[km1] + h[kp1]) + 2.0 * h[k] > 0.0) {
            double sl = u[k] - u[km1];
            double sc = (u[kp1] - u[km1]) * (h[k] / ((h[km1] + h[kp1]) + 2.0 * h[k]));
            double sr = u[kp1] - u[k];
            if (sl * sr > 0.0) {
                double m = pmin(pmin(fabs(sl), fabs(sc)), fabs(sr));
                slope_x_h = sc >= 0.0 ? m : -m;
            }
        }
        double sgn = slope_x_h >= 0.0 ? 1.0 : -1.0;
        double* el = &e[2 * k + 0];
        double* er = &e[2 * k + 1];
        if ((u[km1] - *el) * (*el - u[k]) < 0.0) *el = u[k] - sgn * pmin(fabs(slope_x_h), fabs(*el - u[k]));
        if ((u[kp1] - *er) * (*er - u[k]) < 0.0) *er = u[k] + sgn * pmin(fabs(slope_x_h), fabs(*er - u[k]));
        *el = pmax(pmin(*el, pmax(u[km1], u[k])), pmin(u[km1], u[k]));
        *er = pmax(pmin(*er, pmax(u[kp1], u[k])), pmin(u[kp1], u[k]));
    }
}

/* remap.py:223-231 `_check_discontinuous`. */
static void check_discontinuous(const double* u, int n, double* e)
{
    for (int k = 0; k < n - 1; ++k) {
        if ((e[2 * (k + 1) + 0] - e[2 * k + 1]) * (u[k + 1] - u[k]) < 0.0) {
            double a = 0.5 * (e[2 * k + 1] + e[2 * (k + 1) + 0]);
            a = pmax(pmin(a, pmax(u[k], u[k + 1])), pmin(u[k], u[k + 1]));
            e[2 * k + 1] = a;
            e[2 * (k + 1) + 0] = a;
        }
    }
}

/* remap.py:234-294 `reconstruct`; coef is (n, 3); work holds >= 4n doubles. */
static void reconstruct(const double* h, const double* u, int n, int scheme, double h_neglect,
                        double h_neglect_edge, double* coef, double* work)
{
    for (int k = 0; k < n; ++k) { coef[3 * k] = u[k]; coef[3 * k + 1] = 0.0; coef[3 * k + 2] = 0.0; }
    if (scheme == PCM || n < 3) return;
    if (scheme == PLM) {
        double* slp = work;
        double* mslp = work + n;
        for (int k = 0; k < n; ++k) { slp[k] = 0.0; mslp[k] = 0.0; }
        for (int k = 1; k < n - 1; ++k)
            slp[k] = plm_slope_wa(h[k - 1], h[k], h[k + 1], h_neglect, u[k - 1], u[k], u[k + 1]);
        for (int k = 1; k < n - 1; ++k)
            mslp[k] = plm_monotonized_slope(u[k - 1], u[k], u[k + 1], slp[k - 1], slp[k], slp[k + 1]);
        double almost_one = 1.0 - EPS;
        for (int k = 1; k < n - 1; ++k) {
            double u_l = u[k] - 0.5 * mslp[k];
            double u_r = u[k] + 0.5 * mslp[k];
            coef[3 * k] = u_l;
            coef[3 * k + 1] = u_r - u_l;
            double edge = coef[3 * k + 1] + coef[3 * k];
            double am = fabs(mslp[k + 1]);
            double e_r = u[k + 1] - 0.5 * (slp[k + 1] >= 0.0 ? am : -am);
            if ((edge - u[k]) * (e_r - edge) < 0.0) coef[3 * k + 1] = coef[3 * k + 1] * almost_one;
        }
        return;
    }
    if (scheme == PPM_H4 && n >= 4) {
        double* e = work;    /* (n, 2) */
        edges_h4(h, u, n, h_neglect_edge, e);
        bound_edges(h, u, n, e);
        check_discontinuous(u, n, e);
        for (int k = 1; k < n - 1; ++k) {
            double u_l = u[k - 1], u_c = u[k], u_r = u[k + 1];
            double el = e[2 * k], er = e[2 * k + 1];
            if ((u_r - u_c) * (u_c - u_l) <= 0.0) {
                el = u_c; er = u_c;
            } else {
                double expr1 = 3.0 * (er - el) * ((u_c - el) + (u_c - er));
                double expr2 = (er - el) * (er - el);
                if (expr1 > expr2) {
                    el = u_c + 2.0 * (u_c - er);
                    el = pmax(pmin(el, pmax(u_l, u_c)), pmin(u_l, u_c));
                } else if (expr1 < -expr2) {
                    er = u_c + 2.0 * (u_c - el);
                    er = pmax(pmin(er, pmax(u_r, u_c)), pmin(u_r, u_c));
                }
            }
            if (fabs(er - el) < pmax(1e-60, EPS * fabs(u_c))) { el = u_c; er = u_c; }
            coef[3 * k] = el;
            coef[3 * k + 1] = 4.0 * (u_c - el) + 2.0 * (u_c - er);
            coef[3 * k + 2] = 3.0 * ((er - u_c) + (el - u_c));
        }
    }
}

/* remap.py:297-303 `_average`. */
static inline double average(double c0, double c1, double c2, double xa, double xb)
{
    if (xb - xa <= 1e-14) {
        double x = 0.5 * (xa + xb);
        return c0 + x * (c1 + x * c2);
    }
    return c0 + 0.5 * c1 * (xa + xb) + c2 * (xa * xa + xa * xb + xb * xb) / 3.0;
}

/* remap.py:306-397 `remap_column`.  work must hold 10*max(n0,n1)+16 doubles. */
void oracle_remap_column(const double* h_src, const double* u_src, int n0, const double* h_tgt, int n1,
                         int scheme, double* u_tgt, double* work)
{
    int n_active = 0;
    for (int k = 0; k < n0; ++k) if (h_src[k] > 0.0) n_active++;
    double* coef = work;                       /* 3*n0 */
    double* rwork = coef + 3 * n0;             /* 4*n0 */
    double* t_edge = rwork + 4 * n0 + 4;       /* n1+1 */
    double* content = t_edge + n1 + 1;         /* n1 */
    double* piece = content + n1;              /* n1+1 */
    int* piece_j = (int*)malloc(sizeof(int) * (size_t)(n1 + 1));
    reconstruct(h_src, u_src, n0, effective_scheme(n_active, scheme), H_NEGLECT, H_NEGLECT_EDGE, coef, rwork);

    t_edge[0] = 0.0;
    for (int j = 0; j < n1; ++j) t_edge[j + 1] = t_edge[j] + h_tgt[j];
    for (int j = 0; j < n1; ++j) content[j] = 0.0;

    double a = 0.0;
    int j = 0, last = -1;
    for (int i = 0; i < n0; ++i) {
        double hi = h_src[i];
        if (hi <= 0.0) continue;
        last = i;
        double b = a + hi;
        int npc = 0, ithick = 0;
        double thick = -1.0;
        while (j < n1) {
            double lo = pmax(a, t_edge[j]);
            double hi_t = j < n1 - 1 ? t_edge[j + 1] : pmax(t_edge[n1], b);
            double up = pmin(b, hi_t);
            double L = up - lo;
            if (L > 0.0) {
                piece[npc] = L * average(coef[3 * i], coef[3 * i + 1], coef[3 * i + 2], (lo - a) / hi, (up - a) / hi);
                piece_j[npc] = j;
                if (L > thick) { thick = L; ithick = npc; }
                npc++;
            }
            if (hi_t <= b && j < n1 - 1) j++;
            else break;
        }
        if (npc > 0) {
            double s = 0.0;
            for (int p = 0; p < npc; ++p) if (p != ithick) s += piece[p];
            piece[ithick] = u_src[i] * hi - s;
            for (int p = 0; p < npc; ++p) content[piece_j[p]] += piece[p];
        }
        a = b;
    }
    if (last < 0) {
        double mean = 0.0;
        for (int i = 0; i < n0; ++i) mean += u_src[i] / n0;
        for (int jj = 0; jj < n1; ++jj) u_tgt[jj] = n0 == n1 ? u_src[jj] : mean;
        free(piece_j);
        return;
    }
    for (int jj = 0; jj < n1; ++jj) {
        if (h_tgt[jj] > 0.0) {
            u_tgt[jj] = content[jj] / h_tgt[jj];
        } else {
            double x = t_edge[jj], aa = 0.0, val = u_src[last];
            for (int i = 0; i < n0; ++i) {
                if (h_src[i] <= 0.0) continue;
                if (x <= aa + h_src[i]) {
                    double xi = (x - aa) / h_src[i];
                    val = coef[3 * i] + xi * (coef[3 * i + 1] + xi * coef[3 * i + 2]);
                    break;
                }
                aa += h_src[i];
            }
            u_tgt[jj] = val;
        }
    }
    free(piece_j);
}

/* Polynomial coefficients of one column (remap.py:234-294), for the reconstruction known-answer tests. */
void oracle_reconstruct(const double* h, const double* u, int n, int scheme, double* coef)
{
    double* work = (double*)malloc(sizeof(double) * (size_t)(4 * n + 8));
    reconstruct(h, u, n, scheme, H_NEGLECT, H_NEGLECT_EDGE, coef, work);
    free(work);
}

/* remap.py:400-415 `_remap_columns`: f_src (n0,ny,nx) -> out (n1,ny,nx); wet one byte per column. */
void oracle_remap_columns(const double* h_src, const double* f_src, const double* h_tgt, int n0, int n1, int ny,
                          int nx, int scheme, const uint8_t* wet, double* out)
{
    const i64 cs = (i64)ny * nx;
    const int nm = n0 > n1 ? n0 : n1;
#pragma omp parallel
    {
        double* col = (double*)malloc(sizeof(double) * (size_t)(4 * nm + 10 * nm + 16));
        double* hs = col + n1;
        double* us = hs + n0;
        double* ht = us + n0;
        double* work = ht + n1;
#pragma omp for schedule(static)
        for (i64 c = 0; c < cs; ++c) {
            if (!wet[c]) {
                for (int k = 0; k < n1; ++k) out[(i64)k * cs + c] = n0 == n1 ? f_src[(i64)k * cs + c] : NAN;
                continue;
            }
            for (int k = 0; k < n0; ++k) { hs[k] = h_src[(i64)k * cs + c]; us[k] = f_src[(i64)k * cs + c]; }
            for (int k = 0; k < n1; ++k) ht[k] = h_tgt[(i64)k * cs + c];
            oracle_remap_column(hs, us, n0, ht, n1, scheme, col, work);
            for (int k = 0; k < n1; ++k) out[(i64)k * cs + c] = col[k];
        }
        free(col);
    }
}

/* ============================================================================================================
 * Whole FCT step (tracers.py:208-254 `advect_fct`, non-periodic arrays; the periodic pad/crop is in oracle.py).
 * inflow: the inflow stack, or NULL (then stages 2 and 3 use their own values at open edges).
 * Fx_eff, Fy_eff (optional, full face arrays): the step's effective flux F_L + C A (tracers.py:249-254).
 * ========================================================================================================== */
int oracle_advect_fct(const double* C, const double* V0, const double* V1, const double* Qx, const double* Qy,
                      const uint8_t* okc, const double* inflow, int nt, int n, int ny, int nx, int open_w,
                      int open_e, int open_s, int open_n, int z_variant, double dt, double* out,
                      double* Fx_eff, double* Fy_eff)
{
    const i64 cs = (i64)ny * nx, xs = (i64)ny * (nx + 1), ys = (i64)(ny + 1) * nx;
    const i64 N3 = (i64)n * cs, NC = (i64)nt * N3, NX = (i64)nt * n * xs, NY = (i64)nt * n * ys;
    double* mem = (double*)malloc(sizeof(double) * (size_t)(3 * N3 + 5 * NC + 6 * (NX + NY)));
    if (!mem) return 1;
    double* dV = mem; double* Va = dV + N3; double* Vb = Va + N3;
    double* q0 = Vb + N3; double* q1 = q0 + NC; double* c1 = q1 + NC; double* q2 = c1 + NC; double* c2 = q2 + NC;
    double* fx0 = c2 + NC; double* fy0 = fx0 + NX; double* fx1 = fy0 + NY; double* fy1 = fx1 + NX;
    double* fx2 = fy1 + NY; double* fy2 = fx2 + NX; double* FLx = fy2 + NY; double* FLy = FLx + NX;
    double* Ax = FLy + NY; double* Ay = Ax + NX; double* Cx = Ay + NY; double* Cy = Cx + NX;
    for (i64 p = 0; p < N3; ++p) dV[p] = V1[p] - V0[p];
    for (i64 p = 0; p < N3; ++p) { Va[p] = V0[p] + dV[p]; Vb[p] = V0[p] + 0.5 * dV[p]; }
    for (i64 p = 0; p < NC; ++p) q0[p] = V0[p % N3] * C[p];
    const double* ext = inflow ? inflow : C;
    oracle_advect_faces_h(C, Qx, Qy, okc, ext, nt, n, ny, nx, open_w, open_e, open_s, open_n, z_variant, fx0, fy0);
    oracle_fct_stage(q0, q0, fx0, fy0, 0.0, 1.0, dt, Va, C, nt, n, ny, nx, q1, c1);
    oracle_advect_faces_h(c1, Qx, Qy, okc, inflow ? inflow : c1, nt, n, ny, nx, open_w, open_e, open_s, open_n,
                          z_variant, fx1, fy1);
    oracle_fct_stage(q0, q1, fx1, fy1, 0.75, 0.25, dt, Vb, C, nt, n, ny, nx, q2, c2);
    oracle_advect_faces_h(c2, Qx, Qy, okc, inflow ? inflow : c2, nt, n, ny, nx, open_w, open_e, open_s, open_n,
                          z_variant, fx2, fy2);
    oracle_fct_fluxes(C, Qx, Qy, ext, nt, n, ny, nx, open_w, open_e, open_s, open_n, fx0, fy0, fx1, fy1, fx2, fy2,
                      FLx, FLy, Ax, Ay);
    /* stage buffers reused: qL, cL = q1, c1 */
    oracle_fct_stage(q0, q0, FLx, FLy, 0.0, 1.0, dt, V1, C, nt, n, ny, nx, q1, c1);
    oracle_fct_coeff(C, c1, V1, Ax, Ay, okc, dt, nt, n, ny, nx, Cx, Cy);
    oracle_fct_final(q0, FLx, FLy, Ax, Ay, Cx, Cy, dt, V1, C, nt, n, ny, nx, out);
    if (Fx_eff) for (i64 p = 0; p < NX; ++p) Fx_eff[p] = FLx[p] + Cx[p] * Ax[p];
    if (Fy_eff) for (i64 p = 0; p < NY; ++p) Fy_eff[p] = FLy[p] + Cy[p] * Ay[p];
    free(mem);
    return 0;
}

/* ============================================================================================================
 * Neighbours of the path: the z* / sigma regrid that produces the remap target, the ALE horizontal diffusion and the
 * face fractions of the velocity remap.
 * ========================================================================================================== */

/* core/vertical/regrid.py:87-98 `enforce_min_thickness` (zw bed first, n+1 interfaces). */
static void enforce_min_thickness(double* zw, int n, double h_min)
{
    const double hm = pmin(h_min, (zw[n] - zw[0]) / n);
    for (int j = n - 1; j > 0; --j)
        if (zw[j] > zw[j + 1] - hm) zw[j] = zw[j + 1] - hm;
    for (int j = 1; j < n; ++j)
        if (zw[j] < zw[j - 1] + hm) zw[j] = zw[j - 1] + hm;
}

/* regrid.py:44-61 `zstar_column`: interfaces bed first; dz_top surface first; e holds n+1 doubles. */
static void zstar_column(double H, double eta, const double* dz_top, int n, double h_min, double* e, double* zw)
{
    const double D = H + eta;
    const double hm = pmin(h_min, D / n);
    const double s = D / H;
    e[0] = eta;
    for (int k = 0; k < n; ++k) e[k + 1] = e[k] - s * dz_top[k];
    e[n] = -H;
    for (int k = n - 1; k >= 0; --k)
        if (e[k] < e[k + 1] + hm) e[k] = e[k + 1] + hm;
    for (int j = 0; j <= n; ++j) zw[j] = e[n - j];
}

/* regrid.py:63-78 `sigma_column`: fractions dsigma bed first. */
static void sigma_column(double H, double eta, const double* dsigma, int n, double h_min, double* zw)
{
    const double D = H + eta;
    zw[0] = -H;
    for (int j = 0; j < n; ++j) zw[j + 1] = zw[j] + D * dsigma[j];
    zw[n] = eta;
    enforce_min_thickness(zw, n, h_min);
}

static double nan_to_num(double x)
{
    if (isnan(x)) return 0.0;
    if (isinf(x)) return x > 0 ? DBL_MAX : -DBL_MAX;
    return x;
}

/*
 * ALECoordinate.regrid_remap's regrid half for the z* (rule 0) and sigma (rule 1) rules
 * (core/components/vertical_coordinate.py:69-78, 96-111; regrid.py:309-395): per column
 * wet = active & (H + eta > 0) & (sum_k h_src > 0) with H = nan_to_num(H) and the sum taken k = 0 .. n-1;
 * h_new = diff(zw) where wet, else h_src.  coord: dz_top (surface first, z*) or dsigma (bed first, sigma).
 * Returns the number of wet columns that break the rule's precondition (z*: H > 0), which the reference
 * raises for.
 */
int oracle_regrid(int rule, const double* Hin, const double* eta, const double* h_src, const uint8_t* active,
                  const double* coord, double h_min, int n, int ny, int nx, double* h_new, uint8_t* wet)
{
    const i64 plane = (i64)ny * nx;
    int bad = 0;
#pragma omp parallel for reduction(+ : bad)
    for (i64 c = 0; c < plane; ++c) {
        const double H = nan_to_num(Hin[c]);
        double tot = 0.0;
        for (int k = 0; k < n; ++k) tot += h_src[k * plane + c];
        const int w = active[c] && (H + eta[c] > 0) && (tot > 0);
        wet[c] = (uint8_t)w;
        if (!w) {
            for (int k = 0; k < n; ++k) h_new[k * plane + c] = h_src[k * plane + c];
            continue;
        }
        double* zw = (double*)malloc(2 * (size_t)(n + 1) * sizeof(double));
        if (rule == 0) {
            if (!(H > 0)) ++bad;
            zstar_column(H, eta[c], coord, n, h_min, zw + n + 1, zw);
        } else {
            sigma_column(H, eta[c], coord, n, h_min, zw);
        }
        for (int k = 0; k < n; ++k) h_new[k * plane + c] = zw[k + 1] - zw[k];
        free(zw);
    }
    return bad;
}

/* regrid.py:100-154 `_p1m_h2_positions`: depths (0 at the surface) of the m+1 target interface densities in a
 * column of n layers (h, rho surface first); e holds 2n doubles, xg n+1. */
static void p1m_h2_positions(const double* h, const double* rho, int n, const double* targets, int m, double* x,
                             double* e, double* xg)
{
    e[0] = rho[0];
    e[2 * (n - 1) + 1] = rho[n - 1];
    for (int k = 1; k < n; ++k) {
        if (h[k - 1] + h[k] == 0.0) e[2 * k] = 0.5 * (rho[k - 1] + rho[k]);
        else e[2 * k] = (rho[k - 1] * h[k] + rho[k] * h[k - 1]) / (h[k - 1] + h[k]);
        e[2 * (k - 1) + 1] = e[2 * k];
    }
    bound_edges(h, rho, n, e);
    for (int k = 0; k < n - 1; ++k)
        if (e[2 * k + 1] != e[2 * (k + 1)]) {
            const double a = 0.5 * (e[2 * k + 1] + e[2 * (k + 1)]);
            e[2 * k + 1] = a;
            e[2 * (k + 1)] = a;
        }
    xg[0] = 0.0;
    for (int k = 0; k < n; ++k) xg[k + 1] = xg[k] + h[k];
    for (int k = 0; k <= m; ++k) x[k] = m == n ? xg[k] : xg[n] * k / m;
    for (int kk = 1; kk < m; ++kk) {
        const double t = targets[kk];
        if (t <= e[0]) {
            x[kk] = xg[0];
            continue;
        }
        int found = 0;
        for (int k = 1; k < n; ++k)
            if (t >= e[2 * (k - 1) + 1] && t <= e[2 * k]) {
                x[kk] = xg[k];
                found = 1;
                break;
            }
        if (found) continue;
        if (t >= e[2 * (n - 1) + 1]) {
            x[kk] = xg[n];
            continue;
        }
        for (int k = 0; k < n; ++k)
            if (e[2 * k] < t && t < e[2 * k + 1]) {
                const double xi = (t - e[2 * k]) / (e[2 * k + 1] - e[2 * k]);
                x[kk] = xg[k] + pmin(pmax(xi, 0.0), 1.0) * h[k];
                break;
            }
    }
}

/* regrid.py:158-201 `_keep_consistent` (x: n+1 depths, overwritten); xg n+1, ok / kept scratch. */
static void keep_consistent(const double* h, const double* rho, int n, const double* targets, double h_mass, double* x,
                            double* xg, uint8_t* ok, uint8_t* kept)
{
    for (int j = 0; j < n; ++j) ok[j] = h[j] < h_mass || (targets[j] <= rho[j] && rho[j] <= targets[j + 1]);
    xg[0] = 0.0;
    for (int j = 0; j < n; ++j) xg[j + 1] = xg[j] + h[j];
    for (int j = 0; j <= n; ++j) kept[j] = 0;
    kept[0] = kept[n] = 1;
    for (int j = 1; j < n; ++j) {
        const int straddle = h[j - 1] >= h_mass && h[j] >= h_mass && rho[j - 1] <= targets[j] && targets[j] <= rho[j];
        if ((ok[j - 1] && ok[j]) || straddle) {
            x[j] = xg[j];
            kept[j] = 1;
        }
    }
    double lo = xg[0];
    for (int j = 1; j < n; ++j) {
        if (kept[j]) lo = x[j];
        else if (x[j] < lo) x[j] = lo;
    }
    double hi = xg[n];
    for (int j = n - 1; j > 0; --j) {
        if (kept[j]) hi = x[j];
        else if (x[j] > hi) x[j] = hi;
    }
}

/* regrid.py:204-252 `hycom1_column`: n source layers (h_bed, rho_bed), m target layers (rho_target m+1, dz_top and
 * max_h_top m, zw bed first m+1); the isopycnal test (keep) only when n == m.  work: >= 6n + m + 8 doubles, bwork
 * >= 2n+2 bytes. */
static void hycom1_column(double H, double eta, const double* h_bed, const double* rho_bed, const double* rho_target,
                          const double* dz_top, const double* max_h_top, double h_min, int keep, int n, int m,
                          double* zw, double* work, uint8_t* bwork)
{
    const double D = H + eta;
    double* h_top = work;
    double* rho_own = h_top + n;
    double* rho = rho_own + n;
    double* x = rho + n;                 /* m+1 */
    double* e = x + m + 1;               /* 2n */
    double* xg = e + 2 * n;              /* n+1 */
    for (int k = 0; k < n; ++k) {
        h_top[k] = h_bed[n - 1 - k];
        rho_own[k] = rho_bed[n - 1 - k];
        rho[k] = rho_own[k];
    }
    const double h_mass = 2.0 * h_min;
    double last = -1.0;
    for (int k = 0; k < n; ++k) {
        if (h_top[k] >= h_mass) last = rho[k];
        else if (last >= 0.0) rho[k] = last;
    }
    int k0 = 0;
    for (k0 = 0; k0 < n; ++k0)
        if (h_top[k0] >= h_mass) break;
    if (k0 == n) k0 = n - 1;             /* the loop variable's last value when nothing breaks */
    if (k0 > 0 && h_top[k0] >= h_mass)
        for (int kk = 0; kk < k0; ++kk) rho[kk] = rho[k0];
    for (int k = n - 2; k >= 0; --k) rho[k] = pmin(rho[k], rho[k + 1]);
    p1m_h2_positions(h_top, rho, n, rho_target, m, x, e, xg);
    if (keep && n == m) keep_consistent(h_top, rho_own, n, rho_target, 2.0 * h_min, x, xg, bwork, bwork + n + 1);
    const double s = D / H;
    double nominal = 0.0;
    for (int k = 1; k <= m; ++k) {
        nominal += dz_top[k - 1] * s;
        x[k] = pmin(pmax(x[k], nominal), D);
    }
    for (int k = 1; k < m; ++k) x[k] = pmin(x[k], x[k - 1] + max_h_top[k - 1]);
    for (int k = 1; k <= m; ++k) x[k] = pmax(x[k], x[k - 1]);
    x[m] = D;
    for (int j = 0; j <= m; ++j) zw[j] = eta - x[m - j];
    zw[0] = -H;
    zw[m] = eta;
    enforce_min_thickness(zw, m, h_min);
}

/* regrid.py:255-260 `transition_weight`. */
static double transition_weight(double D, double d_sigma, double d_hybrid)
{
    if (d_hybrid <= d_sigma) return D > d_sigma ? 1.0 : 0.0;
    return pmin(pmax((D - d_sigma) / (d_hybrid - d_sigma), 0.0), 1.0);
}

/* regrid.py:263-289 `window_shallow_sigma` into zw (zw_hyb may alias nothing). */
static void window_shallow_sigma(const double* zw_hyb, const double* zw_sig, const double* zw_zs, double H, double D,
                                 double d_sigma, double d_hybrid, double h_min, int n, double* zw)
{
    const double q = transition_weight(D, d_sigma, d_hybrid);
    if (q >= 1.0) {
        for (int j = 0; j <= n; ++j) zw[j] = zw_hyb[j];
        return;
    }
    for (int j = 0; j <= n; ++j) {
        const double lo = q * (-H) + (1.0 - q) * zw_sig[j];
        const double hi = q * zw_zs[j] + (1.0 - q) * zw_sig[j];
        zw[j] = pmin(pmax(zw_hyb[j], lo), hi);
    }
    zw[0] = -H;
    zw[n] = zw_sig[n];
    enforce_min_thickness(zw, n, h_min);
}

/*
 * The hybrid rule of `_regrid_columns` (regrid.py:309-342, code 2) as ALECoordinate.regrid uses it: per column the
 * wet mask as oracle_regrid, then sigma where the shallow-sigma weight is 0 (or H <= 0 with a sigma zone),
 * else hycom1_column, windowed towards sigma where 0 < q < 1.  rho (n, ny, nx) bed first; rho_target (n+1) surface
 * first; dz_top, max_h_top (n) surface first; dsigma (n) bed first.  Returns the number of wet columns that break
 * the rule's preconditions (H <= 0 without a sigma zone, or a non-finite density), for which the reference raises.
 */
int oracle_regrid_hybrid(const double* Hin, const double* eta, const double* h_src, const uint8_t* active,
                         const double* rho, const double* rho_target, const double* dz_top, const double* max_h_top,
                         const double* dsigma, double d_sigma, double d_hybrid, double h_min, int keep, int n, int ny,
                         int nx, double* h_new, uint8_t* wet)
{
    const i64 plane = (i64)ny * nx;
    int bad = 0;
#pragma omp parallel for reduction(+ : bad)
    for (i64 c = 0; c < plane; ++c) {
        const double H = nan_to_num(Hin[c]);
        double tot = 0.0;
        for (int k = 0; k < n; ++k) tot += h_src[k * plane + c];
        const int w = active[c] && (H + eta[c] > 0) && (tot > 0);
        wet[c] = (uint8_t)w;
        if (!w) {
            for (int k = 0; k < n; ++k) h_new[k * plane + c] = h_src[k * plane + c];
            continue;
        }
        double* buf = (double*)malloc((size_t)(16 * n + 32) * sizeof(double));
        uint8_t* bwork = (uint8_t*)malloc((size_t)(2 * n + 4));
        double* hb = buf;                      /* n */
        double* rb = hb + n;                   /* n */
        double* col = rb + n;                  /* n+1 */
        double* sig = col + n + 1;             /* n+1 */
        double* zs = sig + n + 1;              /* n+1 */
        double* hyb = zs + n + 1;              /* n+1 */
        double* work = hyb + n + 1;            /* 8n+8 */
        int finite = 1;
        for (int k = 0; k < n; ++k) {
            hb[k] = h_src[k * plane + c];
            rb[k] = rho[k * plane + c];
            finite = finite && isfinite(rb[k]);
        }
        if (!finite || (d_hybrid <= 0.0 && !(H > 0))) ++bad;
        const double q = d_hybrid > 0.0 ? transition_weight(H + eta[c], d_sigma, d_hybrid) : 1.0;
        const double qq = (d_hybrid > 0.0 && H <= 0.0) ? 0.0 : q;
        if (qq <= 0.0) {
            sigma_column(H, eta[c], dsigma, n, h_min, col);
        } else {
            hycom1_column(H, eta[c], hb, rb, rho_target, dz_top, max_h_top, h_min, keep, n, n, col, work, bwork);
            if (qq < 1.0) {
                sigma_column(H, eta[c], dsigma, n, h_min, sig);
                zstar_column(H, eta[c], dz_top, n, h_min, work, zs);
                for (int j = 0; j <= n; ++j) hyb[j] = col[j];
                window_shallow_sigma(hyb, sig, zs, H, H + eta[c], d_sigma, d_hybrid, h_min, n, col);
            }
        }
        for (int k = 0; k < n; ++k) h_new[k * plane + c] = col[k + 1] - col[k];
        free(buf);
        free(bwork);
    }
    return bad;
}

/*
 * regrid.py:309-342 `_regrid_columns`: target interface heights zw (m+1, ny, nx), bed first, of every column wet[c]
 * (the others are left as they are; the caller fills NaN).  code 0 z*, 1 sigma, 2 hybrid; h, rho (n, ny, nx) bed
 * first (n = m unless hybrid); dz_top, max_h_top (m) surface first; dsigma (m) bed first; rho_target (m+1) surface
 * first; H already numpy.nan_to_num'ed by the caller, as the reference passes it.
 */
void oracle_regrid_columns(int code, const double* H, const double* eta, const double* h, const double* rho,
                           const double* dz_top, const double* dsigma, const double* rho_target,
                           const double* max_h_top, double d_sigma, double d_hybrid, double h_min, int keep,
                           const uint8_t* wet, int n, int m, int ny, int nx, double* zw)
{
    const i64 plane = (i64)ny * nx;
    const int nn = n > m ? n : m;
#pragma omp parallel for
    for (i64 c = 0; c < plane; ++c) {
        if (!wet[c]) continue;
        double* buf = (double*)malloc((size_t)(14 * nn + 32) * sizeof(double));
        uint8_t* bwork = (uint8_t*)malloc((size_t)(2 * n + 4));
        double* hb = buf;                      /* n */
        double* rb = hb + nn;                  /* n */
        double* col = rb + nn;                 /* m+1 */
        double* sig = col + nn + 1;            /* m+1 */
        double* zs = sig + nn + 1;             /* m+1 */
        double* hyb = zs + nn + 1;             /* m+1 */
        double* work = hyb + nn + 1;           /* 6n + m + 8 */
        const double Hc = H[c], ec = eta[c];
        if (code == 0) {
            zstar_column(Hc, ec, dz_top, m, h_min, work, col);
        } else if (code == 1) {
            sigma_column(Hc, ec, dsigma, m, h_min, col);
        } else {
            for (int k = 0; k < n; ++k) {
                hb[k] = h[k * plane + c];
                rb[k] = rho[k * plane + c];
            }
            double q = d_hybrid > 0.0 ? transition_weight(Hc + ec, d_sigma, d_hybrid) : 1.0;
            if (d_hybrid > 0.0 && Hc <= 0.0) q = 0.0;
            if (q <= 0.0) {
                sigma_column(Hc, ec, dsigma, m, h_min, col);
            } else {
                hycom1_column(Hc, ec, hb, rb, rho_target, dz_top, max_h_top, h_min, keep, n, m, col, work, bwork);
                if (q < 1.0) {
                    sigma_column(Hc, ec, dsigma, m, h_min, sig);
                    zstar_column(Hc, ec, dz_top, m, h_min, work, zs);
                    for (int j = 0; j <= m; ++j) hyb[j] = col[j];
                    window_shallow_sigma(hyb, sig, zs, Hc, Hc + ec, d_sigma, d_hybrid, h_min, m, col);
                }
            }
        }
        for (int k = 0; k <= m; ++k) zw[k * plane + c] = col[k];
        free(buf);
        free(bwork);
    }
}

/* sigma_baroclinic.py:533-561 `_diffuse_ale_kernel` on one field (n, ny, nx); faces (ny, nx+1) / (ny+1, nx). */
void oracle_diffuse_ale(const double* T, const double* Tw, const double* h, const uint8_t* act, const double* cx,
                        const double* cy, const uint8_t* okx, const uint8_t* oky, const double* V, double kh,
                        double dt, int n, int ny, int nx, double* out)
{
#pragma omp parallel for
    for (int p = 0; p < n * ny; ++p) {
        const int k = p / ny, j = p % ny;
        const i64 r = ((i64)k * ny + j) * nx;
        for (int i = 0; i < nx; ++i) {
            double fw = 0.0, fe = 0.0, fs = 0.0, fn = 0.0;
            const i64 ux = (i64)j * (nx + 1) + i, vy = (i64)j * nx + i, a = (i64)j * nx + i;
            if (0 < i && okx[ux]) {
                const double hu = (act[a - 1] && act[a]) ? pmin(h[r + i - 1], h[r + i]) : 0.0;
                fw = -kh * cx[ux] * hu * (Tw[r + i] - Tw[r + i - 1]);
            }
            if (i < nx - 1 && okx[ux + 1]) {
                const double hu = (act[a] && act[a + 1]) ? pmin(h[r + i], h[r + i + 1]) : 0.0;
                fe = -kh * cx[ux + 1] * hu * (Tw[r + i + 1] - Tw[r + i]);
            }
            if (0 < j && oky[vy]) {
                const double hv = (act[a - nx] && act[a]) ? pmin(h[r + i - nx], h[r + i]) : 0.0;
                fs = -kh * cy[vy] * hv * (Tw[r + i] - Tw[r + i - nx]);
            }
            if (j < ny - 1 && oky[vy + nx]) {
                const double hv = (act[a] && act[a + nx]) ? pmin(h[r + i], h[r + i + nx]) : 0.0;
                fn = -kh * cy[vy + nx] * hv * (Tw[r + i + nx] - Tw[r + i]);
            }
            const double div = fe - fw + fn - fs;
            out[r + i] = V[r + i] > 0.0 ? T[r + i] - dt * div / V[r + i] : T[r + i];
        }
    }
}

/* core/vertical/ale.py:883-892 `_fractions_kernel`: w_k = hf_k / sum_k hf_k (sequential sum), 1/n where the sum
 * is not positive; hf (n, a, b). */
void oracle_face_fractions(const double* hf, int n, int a, int b, double* w)
{
    const i64 plane = (i64)a * b;
#pragma omp parallel for
    for (i64 c = 0; c < plane; ++c) {
        double tot = 0.0;
        for (int k = 0; k < n; ++k) tot += hf[k * plane + c];
        for (int k = 0; k < n; ++k) w[k * plane + c] = tot > 0.0 ? hf[k * plane + c] / tot : 1.0 / n;
    }
}

/* ============================================================================================================
 * Producers of the step's inputs (core/vertical/ale.py): face transport thicknesses, transport velocity, PPM layer
 * transport with the barotropic correction, the outflow limiter and the Lagrangian thickness.
 * ========================================================================================================== */

/* ale.py:177-210 `_ftt_kernel`: q_e, q_w (n, ny, nx+1) from h (n, ny, nx), H (ny, nx). */
void oracle_ftt(const double* h, const double* H, const uint8_t* active, int clip, int n, int ny, int nx,
                double* q_e, double* q_w)
{
    const int nf = nx + 1;
    const i64 pc = (i64)ny * nx, pf = (i64)ny * nf;
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int f = 0; f < nf; ++f) {
            const int iw = f > 0 ? f - 1 : 0, ie = f < nx ? f : nx - 1;
            const i64 o = (i64)j * nf + f;
            if (!(active[j * nx + iw] && active[j * nx + ie])) {
                for (int k = 0; k < n; ++k) q_e[k * pf + o] = q_w[k * pf + o] = 0.0;
                continue;
            }
            if (clip) {
                const double Hw0 = H[j * nx + iw], He0 = H[j * nx + ie];
                const double Hw = Hw0 == Hw0 ? Hw0 : 0.0, He = He0 == He0 ? He0 : 0.0;
                const double z_bed = pmax(-Hw, -He);
                double cw = 0.0, ce = 0.0;
                for (int k = 0; k < n; ++k) {
                    const double a = h[k * pc + j * nx + iw], b = h[k * pc + j * nx + ie];
                    const double hw = a == a ? a : 0.0, he = b == b ? b : 0.0;
                    cw += hw;
                    ce += he;
                    q_e[k * pf + o] = pmin(hw, pmax(0.0, (-Hw + cw) - z_bed));
                    q_w[k * pf + o] = pmin(he, pmax(0.0, (-He + ce) - z_bed));
                }
            } else {
                for (int k = 0; k < n; ++k) {
                    const double a = h[k * pc + j * nx + iw], b = h[k * pc + j * nx + ie];
                    q_e[k * pf + o] = a == a ? a : 0.0;
                    q_w[k * pf + o] = b == b ? b : 0.0;
                }
            }
        }
}

/* ale.py:789-808 `_transport_velocity_kernel` on (n, a, b) face arrays. */
void oracle_transport_velocity(const double* u_new, const double* u_old, const uint8_t* last_wet, const double* w,
                               const double* L, const double* D, double theta, double theta_bc, int n, int a, int b,
                               double* ut, double* Qb)
{
    const i64 plane = (i64)a * b;
#pragma omp parallel for
    for (i64 c = 0; c < plane; ++c) {
        double m1 = 0.0, m0 = 0.0;
        for (int k = 0; k < n; ++k) {
            const double un = last_wet[c] ? u_old[k * plane + c] : 0.0;
            m1 += w[k * plane + c] * u_new[k * plane + c];
            m0 += w[k * plane + c] * un;
        }
        const double d = (theta - theta_bc) * (m1 - m0);
        double s = 0.0;
        for (int k = 0; k < n; ++k) {
            const double un = last_wet[c] ? u_old[k * plane + c] : 0.0;
            const double x = theta_bc * u_new[k * plane + c] + (1 - theta_bc) * un + d;
            ut[k * plane + c] = x;
            s += w[k * plane + c] * x;
        }
        Qb[c] = L[c] * D[c] * s;
    }
}

/* ale.py:582-626 `_ppm_edges_kernel` (h already masked: where(active, nan_to_num(h), 0)). */
void oracle_ppm_edges(const double* h, const uint8_t* active, double h_min, int n, int ny, int nx, double* h_w,
                      double* h_e)
{
    const i64 pc = (i64)ny * nx;
#pragma omp parallel for
    for (int j = 0; j < ny; ++j) {
        double* slp = (double*)malloc((size_t)nx * sizeof(double));
        for (int k = 0; k < n; ++k) {
            const double* hr = h + k * pc + (i64)j * nx;
            const uint8_t* ar = active + (i64)j * nx;
            for (int i = 0; i < nx; ++i) {
                const double m = ar[i] ? 1.0 : 0.0;
                const double mw = i > 0 ? (ar[i - 1] ? 1.0 : 0.0) : 0.0;
                const double me = i < nx - 1 ? (ar[i + 1] ? 1.0 : 0.0) : 0.0;
                const double hc = hr[i];
                const double hm1 = i > 0 ? mw * hr[i - 1] + (1.0 - mw) * hc : hc;
                const double hp1 = i < nx - 1 ? me * hr[i + 1] + (1.0 - me) * hc : hc;
                double sl = 0.5 * (hp1 - hm1);
                const double dmx = pmax(pmax(hp1, hm1), hc) - hc;
                const double dmn = hc - pmin(pmin(hp1, hm1), hc);
                const double a = pmin(fabs(sl), 2.0 * pmin(dmx, dmn));
                sl = sl > 0.0 ? a : (sl < 0.0 ? -a : 0.0);
                slp[i] = mw * me * m > 0.0 ? sl : 0.0;
            }
            for (int i = 0; i < nx; ++i) {
                const double mw = i > 0 ? (ar[i - 1] ? 1.0 : 0.0) : 0.0;
                const double me = i < nx - 1 ? (ar[i + 1] ? 1.0 : 0.0) : 0.0;
                const double hc = hr[i];
                const double hm1 = i > 0 ? mw * hr[i - 1] + (1.0 - mw) * hc : hc;
                const double hp1 = i < nx - 1 ? me * hr[i + 1] + (1.0 - me) * hc : hc;
                const double sw = i > 0 ? slp[i - 1] : 0.0, se = i < nx - 1 ? slp[i + 1] : 0.0;
                const double hw = 0.5 * (hm1 + hc) + (sw - slp[i]) / 6.0;
                const double he = 0.5 * (hp1 + hc) + (slp[i] - se) / 6.0;
                const double curv = 3.0 * ((hw + he) - 2.0 * hc);
                const double dh = he - hw;
                const int inside = curv > 0.0 && fabs(dh) < curv;
                const i64 o = k * pc + (i64)j * nx + i;
                if (inside && hc <= h_min) {
                    h_w[o] = hc;
                    h_e[o] = hc;
                    continue;
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
        }
        free(slp);
    }
}

/* ale.py:629-647 `_face_flux`: (F, dF/du) of layer k at u-face (j, f). */
static void face_flux(int k, int j, int f, double u, const double* h, const double* h_w, const double* h_e,
                      const double* dx, const double* q_e, const double* q_w, double L_f, double dt, int ny, int nx,
                      double* F, double* dF)
{
    const int iw = f > 0 ? f - 1 : 0, ie = f < nx ? f : nx - 1;
    const i64 pc = (i64)ny * nx, pf = (i64)ny * (nx + 1);
    double c, hu, ww, ee, curv3, dh, edge, q;
    if (u >= 0.0) {
        c = pmin(fabs(u) * dt / dx[j * nx + iw], 1.0);
        const i64 o = k * pc + (i64)j * nx + iw;
        hu = h[o]; ww = h_w[o]; ee = h_e[o];
        curv3 = (ww + ee) - 2.0 * hu; dh = ww - ee; edge = ee; q = q_e[k * pf + (i64)j * (nx + 1) + f];
    } else {
        c = pmin(fabs(u) * dt / dx[j * nx + ie], 1.0);
        const i64 o = k * pc + (i64)j * nx + ie;
        hu = h[o]; ww = h_w[o]; ee = h_e[o];
        curv3 = (ww + ee) - 2.0 * hu; dh = ee - ww; edge = ww; q = q_w[k * pf + (i64)j * (nx + 1) + f];
    }
    double mean = edge + c * (0.5 * dh + curv3 * (c - 1.5));
    double marg = edge + c * (dh + 3.0 * curv3 * (c - 1.0));
    if (q < hu) {
        mean = pmin(mean, q);
        marg = pmin(marg, q);
    }
    *F = L_f * u * pmax(mean, 0.0);
    *dF = L_f * pmax(marg, 0.0);
}

/* ale.py:650-740 `_ppm_transport_kernel`; h masked, h_w / h_e its edges; out (n, ny, nx+1).  Returns the number of
 * Newton iterations taken. */
int oracle_ppm_transport(const double* h, const double* h_w, const double* h_e, const double* ut, const double* L,
                         const double* Q_bt, const double* q_e, const double* q_w, const uint8_t* active, double dt,
                         const double* dx, int max_iter, int n, int ny, int nx, double* out)
{
    const int nf = nx + 1;
    const i64 pf = (i64)ny * nf;
    double* du = (double*)calloc((size_t)pf, sizeof(double));
    double* lo = (double*)malloc((size_t)pf * sizeof(double));
    double* hi = (double*)malloc((size_t)pf * sizeof(double));
    double* err = (double*)malloc((size_t)pf * sizeof(double));
    double* dsum = (double*)malloc((size_t)pf * sizeof(double));
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int f = 0; f < nf; ++f) {
            const i64 o = (i64)j * nf + f;
            const int iw = f > 0 ? f - 1 : 0, ie = f < nx ? f : nx - 1;
            const double limw = 0.5 * dx[j * nx + iw] / dt, lime = 0.5 * dx[j * nx + ie] / dt;
            double mnw = INFINITY, mxe = -INFINITY;
            for (int k = 0; k < n; ++k) {
                mnw = pmin(mnw, limw - ut[k * pf + o]);
                mxe = pmax(mxe, -(lime + ut[k * pf + o]));
            }
            hi[o] = pmax(pmin(limw, mnw), 0.0);
            lo[o] = pmin(pmax(-lime, mxe), 0.0);
            double s = 0.0, sd = 0.0;
            if (active[j * nx + iw] && active[j * nx + ie])
                for (int k = 0; k < n; ++k) {
                    double F, dF;
                    face_flux(k, j, f, ut[k * pf + o], h, h_w, h_e, dx, q_e, q_w, L[o], dt, ny, nx, &F, &dF);
                    s += F;
                    sd += dF;
                }
            err[o] = s - Q_bt[o];
            dsum[o] = sd;
        }
    int it = 0;
    for (; it < max_iter;) {
#pragma omp parallel for
        for (int j = 0; j < ny; ++j)
            for (int f = 0; f < nf; ++f) {
                const i64 o = (i64)j * nf + f;
                const double e = err[o], d = du[o];
                if (e > 0.0) hi[o] = d;
                if (e < 0.0) lo[o] = d;
                const double step = dsum[o] > 0.0 ? -e / dsum[o] : 0.0;
                double nw = d + step;
                if (step > 0.0 && nw >= hi[o]) nw = 0.5 * (d + hi[o]);
                if (step < 0.0 && nw <= lo[o]) nw = 0.5 * (d + lo[o]);
                du[o] = nw;
                const int iw = f > 0 ? f - 1 : 0, ie = f < nx ? f : nx - 1;
                double s = 0.0, sd = 0.0;
                if (active[j * nx + iw] && active[j * nx + ie])
                    for (int k = 0; k < n; ++k) {
                        double F, dF;
                        face_flux(k, j, f, ut[k * pf + o] + nw, h, h_w, h_e, dx, q_e, q_w, L[o], dt, ny, nx, &F, &dF);
                        s += F;
                        sd += dF;
                    }
                err[o] = s - Q_bt[o];
                dsum[o] = sd;
            }
        ++it;
        int done = 1;
        for (i64 o = 0; o < pf; ++o)
            if (fabs(err[o]) > 1e-12 * pmax(fabs(Q_bt[o]), 1.0)) done = 0;
        if (done) break;
    }
#pragma omp parallel for
    for (int j = 0; j < ny; ++j) {
        double* Fk = (double*)malloc((size_t)n * sizeof(double));
        for (int f = 0; f < nf; ++f) {
            const i64 o = (i64)j * nf + f;
            const int iw = f > 0 ? f - 1 : 0, ie = f < nx ? f : nx - 1;
            if (!(active[j * nx + iw] && active[j * nx + ie])) {
                for (int k = 0; k < n; ++k) out[k * pf + o] = 0.0;
                continue;
            }
            double s = 0.0;
            for (int k = 0; k < n; ++k) {
                double F, dF;
                face_flux(k, j, f, ut[k * pf + o] + du[o], h, h_w, h_e, dx, q_e, q_w, L[o], dt, ny, nx, &F, &dF);
                Fk[k] = F;
                s += Fk[k];
            }
            const double R = Q_bt[o] - s;
            double te = 0.0, tw = 0.0;
            for (int k = 0; k < n; ++k) {
                te += q_e[k * pf + o];
                tw += q_w[k * pf + o];
            }
            int use_e = R >= 0.0;
            double tot = use_e ? te : tw;
            if (tot <= 0.0) {
                use_e = !use_e;
                tot = use_e ? te : tw;
            }
            const double den = tot > 0.0 ? tot : 1.0;
            for (int k = 0; k < n; ++k)
                out[k * pf + o] = Fk[k] + R * (use_e ? q_e[k * pf + o] : q_w[k * pf + o]) / den;
        }
        free(Fk);
    }
    free(du); free(lo); free(hi); free(err); free(dsum);
    return it;
}

/* Outflow of a cell-layer through its four faces, ale.py:300-303. */
static inline double outflow_at(const double* Qx, const double* Qy, int k, int j, int i, int ny, int nx)
{
    const i64 ox = (i64)k * ny * (nx + 1) + (i64)j * (nx + 1) + i, oy = (i64)k * (ny + 1) * nx + (i64)j * nx + i;
    return pmax(Qx[ox + 1], 0.0) - pmin(Qx[ox], 0.0) + pmax(Qy[oy + nx], 0.0) - pmin(Qy[oy], 0.0);
}

/* ale.py:306-321 `_exceeds_kernel`. */
int oracle_outflow_exceeds(const double* h, const double* Qx, const double* Qy, const double* area, double dt,
                           const uint8_t* active, double h_floor, int n, int ny, int nx)
{
    int hit = 0;
    for (int k = 0; k < n && !hit; ++k)
        for (int j = 0; j < ny && !hit; ++j)
            for (int i = 0; i < nx; ++i) {
                if (!active[j * nx + i]) continue;
                const double o = outflow_at(Qx, Qy, k, j, i, ny, nx);
                if (o > pmax(h[(i64)k * ny * nx + (i64)j * nx + i] - h_floor, 0.0) * area[j * nx + i] / dt) {
                    hit = 1;
                    break;
                }
            }
    return hit;
}

static inline double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : (x == 0.0 ? 0.0 : x)); }

/*
 * One face column of the give-back (ale.py:398-441 `_give_back`) for face (j, f) of one axis: nq layers of Q with
 * stride sq, the donor cells' room (lo / hi side) and whole content (full) with stride sc.  lo_ok / hi_ok: the
 * donor exists (otherwise the edge value, 0).  Returns 1 if the face must carry flow out of a dry donor column.
 */
static int give_back_face(double* Q, i64 sq, int nq, double delta, const double* room_lo, const double* room_hi,
                          const double* full_lo, const double* full_hi, i64 sc, int lo_ok, int hi_ok)
{
    const double s = sgn(delta);
    double tot = 0.0;
    for (int k = 0; k < nq; ++k) {
        const double rl = pmax(lo_ok ? room_lo[k * sc] : 0.0, 0.0), rh = pmax(hi_ok ? room_hi[k * sc] : 0.0, 0.0);
        const double q = Q[k * sq];
        const int same = sgn(q) == s && q != 0.0 && s != 0.0;
        tot += same ? (s > 0 ? rl : rh) : 0.0;
    }
    const double need = fabs(delta);
    const double give = need < tot ? need : tot;                    /* np.minimum */
    const double X = tot > 0 ? give / (tot > 0 ? tot : 1.0) : 0.0;
    for (int k = 0; k < nq; ++k) {
        const double rl = pmax(lo_ok ? room_lo[k * sc] : 0.0, 0.0), rh = pmax(hi_ok ? room_hi[k * sc] : 0.0, 0.0);
        const double q = Q[k * sq];
        const int same = sgn(q) == s && q != 0.0 && s != 0.0;
        const double rm = same ? (s > 0 ? rl : rh) : 0.0;
        Q[k * sq] = q + s * rm * X;
    }
    double rest = need - give;
    double cap = 0.0;
    for (int k = 0; k < nq; ++k) {
        const double q = Q[k * sq];
        const int opp = sgn(q) == -s && s != 0.0;
        cap += opp ? fabs(q) : 0.0;
    }
    const double mrc = rest < cap ? rest : cap;
    const double frac = cap > 0 ? mrc / (cap > 0 ? cap : 1.0) : 0.0;
    for (int k = 0; k < nq; ++k) {
        const double q = Q[k * sq];
        const int opp = sgn(q) == -s && s != 0.0;
        Q[k * sq] = q - (opp ? q * frac : 0.0);
    }
    rest = rest - mrc;
    const double rp = rest > 0 ? 1.0 : 0.0;
    double ftot = 0.0;
    for (int k = 0; k < nq; ++k) {
        const double fl = lo_ok ? full_lo[k * sc] : 0.0, fh = hi_ok ? full_hi[k * sc] : 0.0;
        ftot += (s > 0 ? fl : fh) * rp;
    }
    if (rest > 0 && ftot <= 0) return 1;
    const double Y = ftot > 0 ? rest / (ftot > 0 ? ftot : 1.0) : 0.0;
    for (int k = 0; k < nq; ++k) {
        const double fl = lo_ok ? full_lo[k * sc] : 0.0, fh = hi_ok ? full_hi[k * sc] : 0.0;
        const double fm = (s > 0 ? fl : fh) * rp;
        Q[k * sq] = Q[k * sq] + s * fm * Y;
    }
    return 0;
}

/*
 * ale.py:331-395 `limit_outflow` after its fast check found a cell to limit; Qx, Qy are limited in place.
 * Returns 0 (limited), 1 (accepted with the reference's warning), 2 (raises: barotropic CFL), 3 (raises: a face must
 * carry flow out of a dry donor column); *n_lim the count of limited cell-layers over the passes.
 */
int oracle_limit_outflow(const double* h, double* Qx, double* Qy, const double* area, double dt,
                         const uint8_t* active, double h_floor, int max_pass, int per_x, int per_y, int n, int ny,
                         int nx, int* n_lim)
{
    const i64 pc = (i64)ny * nx, px = (i64)ny * (nx + 1), py = (i64)(ny + 1) * nx;
    double* room0 = (double*)malloc((size_t)(n * pc) * sizeof(double));
    double* room = (double*)malloc((size_t)(n * pc) * sizeof(double));
    double* r = (double*)malloc((size_t)(n * pc) * sizeof(double));
    uint8_t* over = (uint8_t*)malloc((size_t)(n * pc));
    double* Qn = (double*)malloc((size_t)(n * (px > py ? px : py)) * sizeof(double));
    for (int k = 0; k < n; ++k)
        for (i64 c = 0; c < pc; ++c) {
            const double A = active[c] ? area[c] : 0.0;
            room0[k * pc + c] = pmax(h[k * pc + c] - h_floor, 0.0) * A / dt;
        }
    int status = -1, cnt = 0, any = 0;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const i64 o = k * pc + (i64)j * nx + i;
                over[o] = active[j * nx + i] && outflow_at(Qx, Qy, k, j, i, ny, nx) > room0[o];
            }
    for (int pass = 0; pass < max_pass && status < 0; ++pass) {
        for (i64 o = 0; o < n * pc; ++o) cnt += over[o];
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const i64 o = k * pc + (i64)j * nx + i;
                    const double O = outflow_at(Qx, Qy, k, j, i, ny, nx);
                    r[o] = over[o] ? room0[o] / (O > 0 ? O : 1.0) : 1.0;
                }
        for (int ax = 0; ax < 2 && status < 0; ++ax) {
            /* ax 0: x faces (j, f), f = 0 .. nx; ax 1: y faces (f, i), f = 0 .. ny */
            const int wrap = ax == 0 ? per_x : per_y;
            double* Q = ax == 0 ? Qx : Qy;
            const int na = ax == 0 ? ny : nx, nc = ax == 0 ? nx : ny;  /* columns across, cells along the axis */
            const i64 pq = ax == 0 ? px : py;
            double* delta = (double*)malloc((size_t)(na * (nc + 1)) * sizeof(double));
            for (int a = 0; a < na; ++a)
                for (int f = 0; f <= nc; ++f) {
                    double d = 0.0;
                    for (int k = 0; k < n; ++k) {
                        const i64 oq = ax == 0 ? k * pq + (i64)a * (nx + 1) + f : k * pq + (i64)f * nx + a;
                        const int lo_c = f > 0 ? f - 1 : (wrap ? nc - 1 : -1), hi_c = f < nc ? f : (wrap ? 0 : -1);
                        const double rlo = lo_c < 0 ? 1.0 : r[k * pc + (ax == 0 ? (i64)a * nx + lo_c : (i64)lo_c * nx + a)];
                        const double rhi = hi_c < 0 ? 1.0 : r[k * pc + (ax == 0 ? (i64)a * nx + hi_c : (i64)hi_c * nx + a)];
                        const double q = Q[oq];
                        const double nw = q > 0 ? q * rlo : (q < 0 ? q * rhi : q);
                        d += q - nw;
                        Qn[oq] = nw;
                    }
                    delta[a * (nc + 1) + f] = d;
                }
            for (i64 o = 0; o < n * pq; ++o) Q[o] = Qn[o];
            for (int k = 0; k < n; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        const i64 o = k * pc + (i64)j * nx + i;
                        room[o] = room0[o] - outflow_at(Qx, Qy, k, j, i, ny, nx);
                    }
            for (int a = 0; a < na && status < 0; ++a)
                for (int f = 0; f <= nc; ++f) {
                    const int lo_c = f > 0 ? f - 1 : (wrap ? nc - 1 : -1), hi_c = f < nc ? f : (wrap ? 0 : -1);
                    const i64 clo = lo_c < 0 ? 0 : (ax == 0 ? (i64)a * nx + lo_c : (i64)lo_c * nx + a);
                    const i64 chi = hi_c < 0 ? 0 : (ax == 0 ? (i64)a * nx + hi_c : (i64)hi_c * nx + a);
                    const i64 oq = ax == 0 ? (i64)a * (nx + 1) + f : (i64)f * nx + a;
                    if (give_back_face(Q + oq, pq, n, delta[a * (nc + 1) + f], room + clo, room + chi, room0 + clo,
                                       room0 + chi, pc, lo_c >= 0, hi_c >= 0)) {
                        status = 3;
                        break;
                    }
                }
            free(delta);
        }
        if (status >= 0) break;
        any = 0;
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const i64 o = k * pc + (i64)j * nx + i;
                    over[o] = active[j * nx + i] && outflow_at(Qx, Qy, k, j, i, ny, nx) > room0[o] * (1.0 + 1e-12);
                    any |= over[o];
                }
        if (!any) status = 0;
    }
    if (status < 0) {
        double mn = INFINITY;
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const i64 c = (i64)j * nx + i;
                    const i64 ox = (i64)k * px + (i64)j * (nx + 1) + i, oy = (i64)k * py + (i64)j * nx + i;
                    const double div = Qx[ox + 1] - Qx[ox] + Qy[oy + nx] - Qy[oy];
                    const double A = active[c] ? area[c] : 0.0;
                    const double hd = active[c] ? h[k * pc + c] - dt * div / (A > 0 ? A : 1.0) : 0.0;
                    mn = hd < mn ? hd : mn;
                }
        status = mn >= -h_floor ? 1 : 2;
    }
    *n_lim = cnt;
    free(room0); free(room); free(r); free(over); free(Qn);
    return status;
}

/* ale.py:278-294 `lagrangian_thickness`: out = max(h - dt divq / A, 0); returns the flat index of the first
 * cell-layer below -tol (the reference raises there), or -1. */
long long oracle_lagrangian_thickness(const double* h, const double* divq, double dt, const double* area, double tol,
                                      int n, int ny, int nx, double* out)
{
    const i64 pc = (i64)ny * nx;
    long long bad = -1;
    for (int k = 0; k < n; ++k)
        for (i64 c = 0; c < pc; ++c) {
            const i64 o = k * pc + c;
            const double v = h[o] - dt * divq[o] / (area[c] > 0 ? area[c] : 1.0);
            if (v < -tol && bad < 0) bad = o;
            out[o] = (v > 0.0 || isnan(v)) ? v : 0.0;                 /* np.maximum(v, 0.0): +0.0 for v = -0.0 */
        }
    return bad;
}

/*
 * ale.py:233-251 `upwind_transport_x` on one face column (a, b) of nq layers: F_k = (L u_k) q_k(u_k) with q_e for
 * u >= 0, q_w otherwise; R = Q_bt - sum_k F_k; the column's thicknesses on R's upwind side (the other side if that
 * column is empty) share R in proportion.  Sums run k = 0 .. n-1 from 0.0, as numpy's first-axis reductions do.
 */
void oracle_upwind_transport(const double* q_e, const double* q_w, const double* ut, const double* L,
                             const double* Q_bt, int n, int a, int b, double* out)
{
    const i64 pf = (i64)a * b;
#pragma omp parallel for
    for (i64 o = 0; o < pf; ++o) {
        double S = 0.0;
        for (int k = 0; k < n; ++k) {
            const i64 x = k * pf + o;
            const double F = (L[o] * ut[x]) * (ut[x] >= 0 ? q_e[x] : q_w[x]);
            out[x] = F;
            S += F;
        }
        const double R = Q_bt[o] - S;
        const int pos = R >= 0;
        double sq = 0.0;
        for (int k = 0; k < n; ++k) sq += pos ? q_e[k * pf + o] : q_w[k * pf + o];
        const int use_e = sq > 0 ? pos : !pos;
        double tot = 0.0;
        for (int k = 0; k < n; ++k) tot += use_e ? q_e[k * pf + o] : q_w[k * pf + o];
        const double den = tot > 0 ? tot : 1.0;
        for (int k = 0; k < n; ++k) {
            const i64 x = k * pf + o;
            out[x] = out[x] + R * (use_e ? q_e[x] : q_w[x]) / den;
        }
    }
}

static inline double np_min(double a, double b) { return (a < b || isnan(a)) ? a : b; }   /* numpy.minimum */
static inline double np_max(double a, double b) { return (a > b || isnan(a)) ? a : b; }   /* numpy.maximum */

/*
 * core/components/freshwater.py:31-58 `freshwater_volumes`: dV (ny, nx) added to the top layer (k = n-1) of V
 * (n, ny, nx); a removal that would take the top layer below floor (ny, nx) is taken from the layers below, top
 * down, each kept at the floor, then down to zero.  Returns the number of such columns.
 */
int oracle_freshwater_volumes(const double* V, const double* dV, const double* floor_, int n, int ny, int nx,
                              double* out)
{
    const i64 pc = (i64)ny * nx;
    int spilled = 0;
    for (i64 c = 0; c < pc; ++c) {
        for (int k = 0; k < n; ++k) out[k * pc + c] = V[k * pc + c];
        out[(n - 1) * pc + c] += dV[c];
        if (!(dV[c] < 0 && out[(n - 1) * pc + c] < floor_[c])) continue;
        ++spilled;
        double deficit = -dV[c];
        for (int pass = 0; pass < 2; ++pass) {
            const double keep = pass == 0 ? floor_[c] : 0.0;
            for (int k = n - 1; k >= 0; --k) {
                const double col = pass == 0 && k == n - 1 ? V[k * pc + c] : out[k * pc + c];
                const double take = np_min(deficit, np_max(col - keep, 0.0));
                out[k * pc + c] = col - take;
                deficit = deficit - take;
            }
        }
    }
    return spilled;
}

/* Threads available to the OpenMP loops (for reporting the CPU baseline's core count). */
#ifdef _OPENMP
#include <omp.h>
int oracle_num_threads(void) { return omp_get_max_threads(); }
void oracle_set_threads(int n) { omp_set_num_threads(n); }
#else
int oracle_num_threads(void) { return 1; }
void oracle_set_threads(int n) { (void)n; }
#endif
