/*
 * pocean_b200.h — C ABI of libpocean_b200.so, the B200 (sm_100a) implementation of pyOCEAN's baroclinic tracer
 * hot path: SSP-RK3 WENO5-Z advection with Zalesak FCT, and the conservative ALE vertical remap.
 *
 * Conventions shared by every entry point:
 *   - All array arguments are DEVICE pointers (cudaMalloc / torch CUDA tensors), C-contiguous, k = 0 at the bed:
 *       tracer stacks (nt, nz, ny, nx) float64; layer geometry (nz, ny, nx) float64;
 *       u-face arrays (nz, ny, nx+1); v-face arrays (nz, ny+1, nx); `ok` / `wet` one byte per cell (0 or 1).
 *   - `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream).  Calls are stream-ordered:
 *     they enqueue kernels and return without synchronising; status codes report argument errors and launch
 *     failures known at return time.
 *   - Inputs are never written.  Outputs are fully written.
 *   - The library allocates no device memory: scratch comes from the caller's `workspace`, sized by the matching
 *     *_workspace_bytes() query.  A workspace may be reused by consecutive calls on the same stream; calls that
 *     run concurrently need distinct workspaces.
 *   - Return value: 0 on success, a POCEAN_E* code otherwise; pocean_last_error() gives the message (per thread).
 */
#ifndef POCEAN_B200_H
#define POCEAN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define POCEAN_OK 0
#define POCEAN_EINVAL 1       /* bad sizes, null pointers, unknown flags or scheme */
#define POCEAN_EWORKSPACE 2   /* workspace missing, misaligned or too small */
#define POCEAN_ECUDA 3        /* a CUDA launch or API call failed */
#define POCEAN_EDEVICE 4      /* the current device is not an sm_100 part */
#define POCEAN_ESTEP 5        /* the step cannot proceed where the reference raises RuntimeError (CFL, dry donor) */

/* Flags of the advection entry points (bitwise OR). */
#define POCEAN_OPEN_W 0x1u    /* open western edge (ob.open contains "west"), tracers.py:163 */
#define POCEAN_OPEN_E 0x2u
#define POCEAN_OPEN_S 0x4u
#define POCEAN_OPEN_N 0x8u
#define POCEAN_PERIODIC_X 0x10u /* periodic in x (core/model/periodic.py); u-face nx is u-face 0 */
#define POCEAN_PERIODIC_Y 0x20u
#define POCEAN_WENO_JS 0x40u  /* WENO5-JS weights (tracer_scheme != "weno5"); default WENO5-Z */
#define POCEAN_FCT_UNLIMITED 0x80u /* advect_fct only: no limiter, C_out = the SSP-RK3 result (tracers.py:289-291) */
/* advect (pocean_advect_rk3_f64) only: the face schemes and the time stepping of the reference's NumPy RHS path
 * (tracers.py:110-151, 303-330).  POCEAN_FACES_UP3: tracer_scheme "upwind3" (and any other non-WENO5 name),
 * POCEAN_FACES_UP1: "upwind1" (_up3_faces, sigma_baroclinic.py:164-188); neither: the WENO5 faces.
 * POCEAN_TIME_PC: tracer_time "pc", a centred half step (_centred_faces, sigma_baroclinic.py:632-652) and a full step
 * from the start with the scheme's faces of the half-step tracer; fx_face is then the corrector's flux. */
#define POCEAN_FACES_UP3 0x100u
#define POCEAN_FACES_UP1 0x200u
#define POCEAN_TIME_PC 0x400u

/* Remap schemes (core/vertical/remap.py:40). */
#define POCEAN_PCM 0
#define POCEAN_PLM 1
#define POCEAN_PPM_H4 2

/* Message of the last failed call on this host thread ("" when none). */
const char* pocean_last_error(void);

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int pocean_version(void);

/* Utility (no counterpart in the reference): a stream-ordered strided 2-D copy, height rows of width bytes from
 * src (row pitch spitch) to dst (row pitch dpitch), in any direction the pointers allow (host pinned <-> device,
 * device <-> device).  The host-array paths of the Python layer use it to stream row blocks so that copies overlap
 * the kernels of other blocks. */
int pocean_memcpy2d_async(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                          void* stream);

/*
 * Workspace (bytes) that pocean_advect_fct_f64 needs for this shape.
 */
size_t pocean_advect_fct_workspace_bytes(int nt, int nz, int ny, int nx);

/*
 * One SSP-RK3 WENO5 advection step of the tracer stack C with Zalesak FCT, layer volumes linear from V0 to V1.
 * Replaces TracerAdvection.advect_fct (core/components/tracers.py:208-254) and the Numba kernels it calls
 * (_advect_faces_h, _fct_stage, _fct_fluxes, _fct_coeff_kernel, _fct_final in
 * core/dynamics/sigma_baroclinic.py:265-321, 407-530).
 *   inflow     (nt, nz, ny, nx) upstream values on open edges during inflow, or NULL: then stage 1 and the donor
 *              flux use C, and stages 2 and 3 their own values (tracers.py:230-241).
 *   C_out      (nt, nz, ny, nx) result.
 *   face_i, fx_face  if fx_face != NULL: the step's effective flux F_L + C·A through u-face column face_i
 *              (0 <= face_i <= nx), written as (nt, nz, ny) (tracers.py:251-254).
 *   open_flux  if != NULL: (nt,) net inflow rate through the open edges, Σ_W F − Σ_E F + Σ_S F − Σ_N F of the
 *              effective flux (tracers.py:65-78, 249-250).  Not defined for an open edge on a periodic axis.
 */
int pocean_advect_fct_f64(const double* C, const double* V0, const double* V1, const double* Qx,
                          const double* Qy, const uint8_t* ok, const double* inflow, int nt, int nz, int ny,
                          int nx, unsigned flags, double dt, double* C_out, int face_i, double* fx_face,
                          double* open_flux, void* workspace, size_t workspace_bytes, void* stream);

/*
 * The FCT step of pocean_advect_fct_f64 with mixed precision: the WENO5 smoothness indicators, nonlinear weights
 * and face values are computed in FP32 (on the stencil's differences from the upwind cell, normalised), while the
 * fluxes, the Zalesak limiter, the donor-cell bookkeeping and every stage update stay in FP64, so tracer content is
 * conserved to FP64 round-off.  Same arguments and workspace as pocean_advect_fct_f64.  Replaces the same
 * reference function (core/components/tracers.py:208-254) at reduced precision of the high-order face values;
 * its error against the FP64 path is measured, not bit-exact.
 */
int pocean_advect_fct_mixed(const double* C, const double* V0, const double* V1, const double* Qx,
                            const double* Qy, const uint8_t* ok, const double* inflow, int nt, int nz, int ny,
                            int nx, unsigned flags, double dt, double* C_out, int face_i, double* fx_face,
                            double* open_flux, void* workspace, size_t workspace_bytes, void* stream);

/* Layer-range FCT passes (no counterpart in the reference): part 0 runs the three RK stage passes of layers
 * k0 .. k1-1, part 1 the Zalesak coefficient and final passes of those layers (their bounds read layers k0-1 and
 * k1, so part 0 of those layers must have run before, in stream order).  Blocks of layers covering 0 .. nz-1, each
 * part 1 after part 0 of the next block, give pocean_advect_fct_f64 (mixed = 0) or _mixed (mixed = 1) bit for bit.
 * The host-array path of the Python layer uses it to overlap the upload of later layers with the passes of earlier
 * ones.  Same arguments as pocean_advect_fct_f64 without the side outputs; the unlimited flag is refused. */
int pocean_advect_fct_layers(int mixed, const double* C, const double* V0, const double* V1, const double* Qx,
                             const double* Qy, const uint8_t* ok, const double* inflow, int nt, int nz, int ny,
                             int nx, unsigned flags, double dt, double* C_out, void* workspace,
                             size_t workspace_bytes, int k0, int k1, int part, void* stream);

/*
 * The same FCT step as pocean_advect_fct_f64 for callers that cannot allocate device memory (a host model that
 * reaches the GPU only through this ABI with no device allocator of its own, or one whose device memory belongs
 * to a pool that forbids side allocations).  No counterpart in the reference: it is an addition of this library.
 * It allocates nothing; its scratch is a fixed array of POCEAN_NOALLOC_SCRATCH_BYTES inside the library, held by
 * every GPU that loads it until the process exits.  Shapes whose pocean_advect_fct_workspace_bytes() exceeds that
 * size are rejected with POCEAN_EINVAL.  Every call looks up the array's address in the current context (so a
 * device reset between calls is safe); the first call on a device loads the library's module there, so make it
 * before any stream capture.  All calls on a device share the array: calls that overlap on the GPU race, so order
 * them on one stream.
 */
#define POCEAN_NOALLOC_SCRATCH_BYTES (64u << 20)
int pocean_advect_fct_f64_noalloc(const double* C, const double* V0, const double* V1, const double* Qx,
                                  const double* Qy, const uint8_t* ok, const double* inflow, int nt, int nz, int ny,
                                  int nx, unsigned flags, double dt, double* C_out, int face_i, double* fx_face,
                                  double* open_flux, void* stream);

/*
 * Workspace (bytes) that pocean_advect_rk3_f64 needs for this shape.
 */
size_t pocean_advect_rk3_workspace_bytes(int nt, int nz, int ny, int nx);

/*
 * One SSP-RK3 step without limiter, WENO5 faces in x, y and z (interface transports Fz (nz+1, ny, nx), or NULL
 * for none).  Replaces TracerAdvection.advect (core/components/tracers.py:342-375) with _advect_div and _rk_stage
 * (core/dynamics/sigma_baroclinic.py:324-364, 856-875).  fx_face: (nt, nz, ny) SSP-RK3 combination
 * (F(c0) + F(c1))/6 + 2F(c2)/3 of the x-face fluxes through column face_i, or NULL.  With POCEAN_FACES_UP3 /
 * POCEAN_FACES_UP1 the faces of the reference's NumPy RHS (tracers.py:139-151), with POCEAN_TIME_PC the 'pc'
 * predictor-corrector step (tracers.py:324-330).
 */
int pocean_advect_rk3_f64(const double* C, const double* V0, const double* V1, const double* Qx,
                          const double* Qy, const double* Fz, const uint8_t* ok, const double* inflow, int nt,
                          int nz, int ny, int nx, unsigned flags, double dt, double* C_out, int face_i,
                          double* fx_face, void* workspace, size_t workspace_bytes, void* stream);

/*
 * The single-stage helpers of TracerAdvection (core/components/tracers.py:139-206), which the reference runs on the
 * arrays it is given (a periodic caller pads them first, so the periodic flags are refused here); ext: the
 * exterior values on open edges (the reference's `ext` / `inflow`), or NULL for the field's own.
 * pocean_advect_faces_f64: the horizontal face fluxes fx (nt, nz, ny, nx+1), fy (nt, nz, ny+1, nx) of the stack c:
 *   kind POCEAN_HELPER_SCHEME   the advect scheme's faces — WENO5-Z, or WENO5-JS with POCEAN_WENO_JS, as
 *                               `faces_h` (_advect_faces_h, sigma_baroclinic.py:265-321); with POCEAN_FACES_UP3 /
 *                               _UP1 the NumPy path's upwind faces times Q (`flux_x`, tracers.py:195-206);
 *   kind POCEAN_HELPER_CENTRED  the centred faces times Q (`flux_x(centred=True)`, _centred_faces);
 *   kind POCEAN_HELPER_DONOR    the donor-cell fluxes of `upwind_faces_h` (tracers.py:178-193).
 * pocean_advect_rhs_f64: -div(Q c) (nt, nz, ny, nx) with the scheme's faces (`rhs`: _advect_div for WENO5,
 *   sigma_baroclinic.py:324-364; the NumPy RHS for the upwind schemes) or centred faces (centred != 0,
 *   `rhs(centred=True)`), Fz (nz+1, ny, nx) or NULL; workspace pocean_advect_rhs_workspace_bytes.
 */
#define POCEAN_HELPER_SCHEME 0
#define POCEAN_HELPER_CENTRED 1
#define POCEAN_HELPER_DONOR 2
int pocean_advect_faces_f64(const double* c, const double* Qx, const double* Qy, const uint8_t* ok,
                            const double* ext, int nt, int nz, int ny, int nx, unsigned flags, int kind, double* fx,
                            double* fy, void* stream);
size_t pocean_advect_rhs_workspace_bytes(int nt, int nz, int ny, int nx);
int pocean_advect_rhs_f64(const double* c, const double* Qx, const double* Qy, const double* Fz, const uint8_t* ok,
                          const double* ext, int nt, int nz, int ny, int nx, unsigned flags, int centred,
                          double* rhs, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Conservative remap of nfields stacked fields f_src (nfields, n0, ny, nx) from thicknesses h_src (n0, ny, nx)
 * onto h_tgt (n1, ny, nx); out (nfields, n1, ny, nx).  wet (ny, nx): dry columns are copied when n0 == n1, else
 * NaN.  scheme: POCEAN_PCM / POCEAN_PLM / POCEAN_PPM_H4.  Replaces core.vertical.remap.remap_columns
 * (core/vertical/remap.py:400-427; one call per field there) and remap_column (:306-397).  Needs no workspace.
 */
int pocean_remap_columns_f64(const double* h_src, const double* f_src, const double* h_tgt, const uint8_t* wet,
                             int n0, int n1, int ny, int nx, int nfields, int scheme, double* out, void* stream);

/*
 * reconstruct (core/vertical/remap.py:234-294) of ncols columns of n cells: h and u (n, ncols), coef (n, ncols, 3),
 * the coefficients (c0, c1, c2) of p(xi) = c0 + c1 xi + c2 xi^2 in each cell with the reference's default
 * negligible thicknesses (H_NEGLECT, H_NEGLECT_EDGE); the scheme as given (no reduction by active cells).
 */
int pocean_reconstruct_f64(const double* h, const double* u, int n, long long ncols, int scheme, double* coef,
                           void* stream);

/*
 * The neighbours of the tracer step.
 *
 * Regrid + remap (ALECoordinate.regrid_remap, core/components/vertical_coordinate.py:69-78, with the z* and sigma
 * rules of core/vertical/regrid.py:44-98, 309-395): per column wet = active & (H + eta > 0) & (sum_k h_src > 0)
 * (H with NaN read as 0, numpy.nan_to_num), h_new = the rule's layer thicknesses where wet, else h_src; then the
 * nfields stacked fields f_src (nfields, nz, ny, nx) are remapped from h_src onto h_new into out, as
 * remap_columns(h_src, f, h_new, scheme, wet) does for each field (a regrid launch, then the remap launches of
 * pocean_remap_columns_f64).  rule POCEAN_REGRID_ZSTAR: coord = dz_top (nz, surface first);
 * POCEAN_REGRID_SIGMA: coord = dsigma (nz, bed first).  h_min: the rules' minimum thickness (the reference's
 * default is 1e-3 m).  wet (ny, nx) bytes out.  nfields = 0: the regrid alone.  bad_columns (device int, may be
 * NULL): incremented for every wet column that breaks the rule's precondition (z*: H > 0), for which the reference
 * raises ValueError; those columns' outputs are undefined.
 */
#define POCEAN_REGRID_ZSTAR 0
#define POCEAN_REGRID_SIGMA 1
int pocean_regrid_remap_f64(int rule, const double* H, const double* eta, const double* h_src, const uint8_t* active,
                            const double* coord, double h_min, const double* f_src, int nz, int ny, int nx,
                            int nfields, int scheme, double* h_new, uint8_t* wet, double* out, int* bad_columns,
                            void* stream);

/*
 * Regrid with the hybrid (HYCOM1) rule + remap (ALECoordinate.regrid_remap with rule 'hybrid',
 * core/vertical/regrid.py:100-289 and the code-2 branch of :309-342): per wet column (the mask of
 * pocean_regrid_remap_f64) the interfaces follow the target densities rho_target (nz+1, surface first) through the
 * P1M/H2 positions of the layer densities rho (nz, ny, nx, bed first), kept where layers already sit in their
 * density class (keep != 0, the default `keep_isopycnal`), floored at the z* grid dz_top (nz, surface first) and
 * capped at max_h_top (nz; +inf = no cap); with d_hybrid > 0 the columns shallower than d_hybrid are windowed
 * towards sigma (dsigma, nz, bed first) and fully sigma below d_sigma or where H <= 0.  Then the nfields stacked
 * fields are remapped onto h_new as pocean_regrid_remap_f64 does.  bad_columns (device int, may be NULL) counts the
 * wet columns with a non-finite density, or with H <= 0 when d_hybrid <= 0, for which the reference raises
 * ValueError.  nz <= 256.  (A target layer count other than the source's: pocean_regrid_columns_f64.)
 */
int pocean_regrid_hybrid_remap_f64(const double* H, const double* eta, const double* h_src, const uint8_t* active,
                                   const double* rho, const double* rho_target, const double* dz_top,
                                   const double* max_h_top, const double* dsigma, double d_sigma, double d_hybrid,
                                   double h_min, int keep, const double* f_src, int nz, int ny, int nx, int nfields,
                                   int scheme, double* h_new, uint8_t* wet, double* out, int* bad_columns,
                                   void* stream);

/* Face fractions w_k = hf_k / sum_k hf_k (1/nz where the sum is not positive) of hf (nz, ny, nx); replaces
 * core/vertical/ale.py:883-902 (face_fractions / _fractions_kernel). */
int pocean_face_fractions_f64(const double* hf, int nz, int ny, int nx, double* w, void* stream);

/* Velocity remap in fraction space (ALECoordinate.remap_faces, vertical_coordinate.py:142-153): each face column of
 * the nfields stacked fields vel (nfields, nz, ny, nx) goes from thicknesses w_src S to w_tgt S, S = sum_k hf_src
 * (1 where not positive, those columns copied), w_src = face_fractions(hf_src), w_tgt = the given fractions or
 * face_fractions(hf_tgt) when w_tgt is NULL.  The fractions are formed in the kernel. */
int pocean_remap_faces_f64(const double* vel, const double* hf_src, const double* hf_tgt, const double* w_tgt,
                           int nz, int ny, int nx, int nfields, int scheme, double* out, void* stream);

/* ALE horizontal diffusion (sigma_baroclinic.py:533-561 `_diffuse_ale_kernel`, as TracerAdvection.diffuse_h calls
 * it, core/components/tracers.py:421-447) of nt stacked fields T / Tw (nt, nz, ny, nx) sharing h, V (nz, ny, nx),
 * act (ny, nx), cx = L_u / dx_u and okx (ny, nx+1), cy and oky (ny+1, nx).  flags: POCEAN_PERIODIC_X / _Y (the wrap
 * faces read as the reference's halo-1 pad/crop reads them: face 0).  h is used as given (the reference passes
 * where(act, nan_to_num(h), 0)). */
int pocean_diffuse_ale_f64(const double* T, const double* Tw, const double* h, const uint8_t* act, const double* cx,
                           const double* cy, const uint8_t* okx, const uint8_t* oky, const double* V, int nt, int nz,
                           int ny, int nx, unsigned flags, double kh, double dt, double* out, void* stream);

/*
 * The producers of the step's inputs (core/vertical/ale.py), for u-faces (nz, ny, nx+1) of cells (nz, ny, nx); the
 * v-faces are the same calls on arrays with the horizontal axes swapped, as the reference makes them.
 */

/* ale.py:177-231 face_transport_thickness / _ftt_kernel: q_e (from the west cell), q_w (from the east cell);
 * clip != 0: only the part above the shallower bed (z*, hybrid).  NaN thickness or depth reads as 0. */
int pocean_face_transport_thickness_f64(const double* h, const double* H, const uint8_t* active, int nz, int ny,
                                        int nx, int clip, double* q_e, double* q_w, void* stream);

/* ale.py:767-825 transport_velocity / _transport_velocity_kernel on face arrays (nz, na, nb): ut (nz, na, nb) and
 * Qb (na, nb).  last_wet one byte per face column; w the layer fractions. */
int pocean_transport_velocity_f64(const double* u_new, const double* u_old, const uint8_t* last_wet, const double* w,
                                  const double* L, const double* D, int nz, int na, int nb, double theta,
                                  double theta_bc, double* ut, double* Qb, void* stream);

/* ale.py:445-480, 582-626 ppm_edges_x / _ppm_edges_kernel of where(active, nan_to_num(h), 0): h_w, h_e. */
int pocean_ppm_edges_f64(const double* h, const uint8_t* active, int nz, int ny, int nx, double h_min, double* h_w,
                         double* h_e, void* stream);

/* ale.py:743-764 ppm_transport_x: PPM layer fluxes Qx (nz, ny, nx+1) with the uniform per-face correction du that
 * makes sum_k Qx = Q_bt (Newton with bracketing bisection, max_iter iterations stopped when every face has
 * converged, then the residual share).  ut, q_e, q_w (nz, ny, nx+1); L, Q_bt (ny, nx+1); dx (ny, nx). */
size_t pocean_ppm_transport_workspace_bytes(int nz, int ny, int nx, int max_iter);
int pocean_ppm_transport_f64(const double* h, const double* ut, const double* L, const double* Q_bt,
                             const double* q_e, const double* q_w, const uint8_t* active, const double* dx, int nz,
                             int ny, int nx, double dt, int max_iter, double* Qx, void* workspace,
                             size_t workspace_bytes, void* stream);

/* ale.py:300-441 limit_outflow: Qx (nz, ny, nx+1) and Qy (nz, ny+1, nx) limited IN PLACE so that no active
 * cell-layer sends out more than (h - h_floor)+ area / dt, the cut flux given back to the other layers of each
 * face.  flags: POCEAN_PERIODIC_X / _Y.  Synchronises the stream (once when nothing exceeds, once per pass
 * otherwise).  *n_limited: limited cell-layers summed over the passes; *warned: still over after max_pass but
 * h-dagger >= -h_floor (the reference warns).  POCEAN_ESTEP where the reference raises (Qx, Qy then undefined). */
size_t pocean_limit_outflow_workspace_bytes(int nz, int ny, int nx);
int pocean_limit_outflow_f64(const double* h, double* Qx, double* Qy, const double* area, const uint8_t* active,
                             int nz, int ny, int nx, double dt, double h_floor, int max_pass, unsigned flags,
                             int* n_limited, int* warned, void* workspace, size_t workspace_bytes, void* stream);

/* ale.py:278-294 lagrangian_thickness: h_dag = max(h - dt divq / A, 0) with A = area where > 0, else 1;
 * *first_bad (DEVICE pointer) receives the flat (k, j, i) index of the first cell-layer below -tol, where the
 * reference raises, or ~0 when there is none. */
int pocean_lagrangian_thickness_f64(const double* h, const double* divq, const double* area, int nz, int ny, int nx,
                                    double dt, double tol, double* h_dag, unsigned long long* first_bad,
                                    void* stream);

/* ale.py:233-251 upwind_transport_x, the donor-cell layer flux of ALELayerTransport (thickness_flux != "ppm"):
 * Q_k = L u_k q_k(u_k) + R q_k(R) / sum_j q_j(R) with R = Q_bt - sum_k L u_k q_k(u_k), q = q_e for a non-negative
 * argument, q_w otherwise (the other side where that column is empty).  q_e, q_w, ut, Q (nz, a, b); L, Q_bt (a, b).
 * v-faces: the same call on swapped horizontal axes, as the reference makes it. */
int pocean_upwind_transport_f64(const double* q_e, const double* q_w, const double* ut, const double* L,
                                const double* Q_bt, int nz, int a, int b, double* Q, void* stream);

/* core/components/freshwater.py:31-58 freshwater_volumes: dV (ny, nx) added to the top layer (k = nz-1) of V
 * (nz, ny, nx); a removal that would take the top layer below the floor is taken from the layers below, top down,
 * first keeping each at the floor, then down to zero.  floor: (ny, nx) or NULL for floor_value everywhere.
 * *n_limited (DEVICE int, may be NULL; the caller zeroes it) is incremented for every such column.  V_new must not
 * alias V. */
int pocean_freshwater_volumes_f64(const double* V, const double* dV, const double* floor_, double floor_value,
                                  int nz, int ny, int nx, double* V_new, int* n_limited, void* stream);

/* Divergence of the layer fluxes, Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:, :] - Qy[:, :-1, :]
 * (core/components/layer_transport.py:146): Qx (nz, ny, nx+1), Qy (nz, ny+1, nx) -> divq (nz, ny, nx). */
int pocean_flux_divergence_f64(const double* Qx, const double* Qy, int nz, int ny, int nx, double* divq,
                               void* stream);

/* ALE layer volumes V = h A (core/dynamics/sigma_baroclinic.py:1812-1815) and, when ok is not NULL,
 * ok = active & (V > 0) (layer_transport.py:149). */
int pocean_layer_volumes_f64(const double* h, const double* area, const uint8_t* active, int nz, int ny, int nx,
                             double* V, uint8_t* ok, void* stream);

/* core/vertical/regrid.py:309-395 regrid_columns itself: target interface heights zw (m+1, ny, nx), bed first, of
 * every column that wet marks (NaN elsewhere) for rule code 0 (z*, dz_top m surface first), 1 (sigma, dsigma m bed
 * first) or 2 (hybrid: the n source layers h and densities rho (n, ny, nx) bed first, rho_target m+1 surface
 * first, dz_top and max_h_top m, with d_hybrid > 0 the shallow sigma window on dsigma; keep the isopycnal test,
 * applied only when m == n).  m != n only for the hybrid rule (regrid_columns' n_out: a finer or coarser source,
 * such as the data levels of an initial state).  H is read as numpy.nan_to_num(H).  n, m <= 256.  The reference's
 * argument checks (finite H and D > 0 in wet columns, ...) are the caller's. */
int pocean_regrid_columns_f64(int code, const double* H, const double* eta, const double* h, const double* rho,
                              const uint8_t* wet, const double* dz_top, const double* dsigma, const double* rho_target,
                              const double* max_h_top, double d_sigma, double d_hybrid, double h_min, int keep, int n,
                              int m, int ny, int nx, double* zw, void* stream);

/* Periodic halo of a producer's inputs (core/model/periodic.py:72-94 Periodic.pad / crop; used for the PPM layer
 * flux on periodic axes, core/components/layer_transport.py:121-128).  src (nlead, ny + face_y, nx + face_x) of ny x nx
 * cells (face_y / face_x = 1 for v- / u-faces); pad: dst with `halo` wrapped positions on each side of every periodic
 * axis (py, px), faces wrapping on the unique faces 0 .. n-1; crop: the inverse, from a padded src to the unpadded
 * dst. */
int pocean_periodic_pad_f64(const double* src, int nlead, int ny, int nx, int face_y, int face_x, int py, int px,
                            int halo, double* dst, void* stream);
int pocean_periodic_pad_u8(const uint8_t* src, int nlead, int ny, int nx, int face_y, int face_x, int py, int px,
                           int halo, uint8_t* dst, void* stream);
int pocean_periodic_crop_f64(const double* src, int nlead, int ny, int nx, int face_y, int face_x, int py, int px,
                             int halo, double* dst, void* stream);

/* core/vertical/ale.py:841-861 open_face_transport as core/components/open_boundary.py:334-352
 * open_face_transports applies it: the layer fluxes Q (n layers x m faces of one open edge) are replaced where the
 * open face depth D > 0 by the Flather flux Q_bt split with the interior cells' thickness fractions,
 * Q_k = w_k Q_bt + L h_k (theta_bc u'_k(new) + (1 - theta_bc) u'_k(old)).  Every array is addressed with its own
 * (layer, face) element strides; Q_bt, L and D share col_stride. */
int pocean_open_face_transport_f64(const double* h_int, long long h_stride_k, long long h_stride_m,
                                   const double* u_new, const double* u_old, long long u_stride_k,
                                   long long u_stride_m, const double* Q_bt, const double* L, const double* D,
                                   long long col_stride, int n, int m, double theta_bc, double* Q,
                                   long long Q_stride_k, long long Q_stride_m, void* stream);

/*
 * Batched steps of many independent domains (no counterpart in the reference, which advances one model at a time):
 * one ALE tracer step = advect_fct of the stack C then the remap of the advected stack C_adv onto the target grid,
 * into C_next.  Every pass is one launch over all domains; pocean_batch_step only enqueues kernels, so a sequence
 * of steps can be captured in a CUDA graph.  Parity 0 reads C and writes C_next, parity 1 reads C_next and writes C
 * (C is written: it is the ping-pong partner).  Results of each domain equal pocean_advect_fct_f64 (or _mixed)
 * followed by pocean_remap_columns_f64 on that domain alone.
 */
typedef struct pocean_domain {
    const double* C;          /* (nt, nz, ny, nx) stack at parity 0 */
    const double* V0;         /* (nz, ny, nx) */
    const double* V1;
    const double* Qx;         /* (nz, ny, nx+1) */
    const double* Qy;         /* (nz, ny+1, nx) */
    const uint8_t* ok;        /* (nz, ny, nx) */
    const double* inflow;     /* (nt, nz, ny, nx) or NULL */
    int nt, nz, ny, nx;
    unsigned flags;           /* POCEAN_OPEN_*, POCEAN_PERIODIC_*, POCEAN_WENO_JS (the same variant for all) */
    double dt;
    double* C_adv;            /* (nt, nz, ny, nx) advected stack */
    void* workspace;          /* pocean_advect_fct_workspace_bytes(nt, nz, ny, nx) bytes, 256-byte aligned */
    size_t workspace_bytes;
    const double* h_src;      /* (nz, ny, nx) source thicknesses of the remap */
    const double* h_tgt;      /* (nz, ny, nx) target thicknesses */
    const uint8_t* wet;       /* (ny, nx) */
    int remap_scheme;         /* POCEAN_PCM / POCEAN_PLM / POCEAN_PPM_H4 */
    double* C_next;           /* (nt, nz, ny, nx) remapped stack */
} pocean_domain;

typedef struct pocean_batch pocean_batch;   /* host-side plan of a batch */

/* Device bytes of the batch plan for ndom domains (descriptors of both parities and the CTA-offset tables). */
size_t pocean_batch_device_bytes(int ndom);

/* Validates the domains and writes the plan into device_buf with copies ordered on `stream` (after the steps
 * already enqueued there, which may still be reading an earlier plan in the same buffer); `domains` may be released
 * on return.  Not capturable: call outside stream capture.  tile_rows: 4, 8 or 16, the height of the 32-wide cell
 * tiles of the WENO face and stage passes (a tuning parameter; results do not depend on it).  A plan only refers to
 * the domains' buffers; steps enqueued with it must be ordered after the plan's copies (same stream, or an event). */
int pocean_batch_create(const pocean_domain* domains, int ndom, int tile_rows, void* device_buf, size_t device_bytes,
                        pocean_batch** out, void* stream);

/* Enqueues one step of every domain.  remap_nf: fields per remap thread (1 or 2, a tuning parameter); mixed: FP32
 * WENO weights (pocean_advect_fct_mixed) instead of FP64. */
int pocean_batch_step(const pocean_batch* b, int parity, int remap_nf, int mixed, void* stream);

void pocean_batch_destroy(pocean_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* POCEAN_B200_H */
