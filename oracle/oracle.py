"""
CPU oracle of pyOCEAN's tracer hot path (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` (as the checker) and ``bench.py``'s CPU-baseline leg import this
module.  The product package ``pyocean_b200`` never does: its path is the CUDA library, which fails loudly when it
is missing.

The arithmetic lives in ``pocean_oracle.c`` (one C function per Numba kernel of the reference, same expression
order, no FMA contraction), loaded through ctypes.  This module restates the Python orchestration around those
kernels with the reference's call signatures:

* ``TracerAdvection`` — ``core/components/tracers.py:50-375`` (``advect_fct`` :208-254, the unlimited NumPy path
  :256-301, ``advect`` :342-375 with the ``'pc'`` branch of ``advect_numpy`` :324-330, ``faces_h`` :166-176,
  ``upwind_faces_h`` :178-193, the NumPy RHS with its face rules :110-151, ``flux_x`` :195-206, periodic pad/crop
  :80-102, ``_open_inflow`` :65-78); the upwind-3/1 and centred face values of the NumPy path
  (``sigma_baroclinic.py:164-199, 632-652``) are restated here in NumPy.
* ``Periodic`` — ``core/model/periodic.py:31, 47-94`` (pad/crop with ``TRACER_HALO`` wrapped cells).
* ``remap_column`` / ``remap_columns`` / ``reconstruct`` — ``core/vertical/remap.py:234-427``.
* ``regrid`` / ``regrid_remap`` — the z* and sigma rules of ``core/vertical/regrid.py:44-98, 309-395`` as
  ``ALECoordinate.regrid_remap`` uses them (``core/components/vertical_coordinate.py:69-111``); ``regrid_hybrid``
  the hybrid (HYCOM1) rule of ``core/vertical/regrid.py:100-289, 309-342``.
* ``diffuse_ale`` — ``_diffuse_ale_kernel`` (``core/dynamics/sigma_baroclinic.py:533-561``) with the pad/crop of
  ``TracerAdvection.diffuse_h`` (``core/components/tracers.py:421-447``).
* ``face_fractions`` / ``remap_faces`` — ``core/vertical/ale.py:883-902`` and
  ``ALECoordinate.remap_faces`` (``vertical_coordinate.py:142-153``).
* The producers of the step's inputs (``core/vertical/ale.py``): ``face_transport_thickness`` (:177-231),
  ``transport_velocity`` (:789-825), ``ppm_edges_x`` / ``ppm_transport_x`` (:582-764), ``limit_outflow`` with
  ``_give_back`` (:300-441) and ``lagrangian_thickness`` (:278-294).

Parity of this restatement with the reference is pinned by ``tests/test_oracle_golden.py`` against the vectors in
``tests/golden/`` that ``tests/golden/make_golden.py`` generated by running the reference itself.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

TRACER_HALO = 13                       # core/model/periodic.py:31
PCM, PLM, PPM_H4 = 0, 1, 2             # core/vertical/remap.py:40
SCHEMES = {"pcm": PCM, "plm": PLM, "ppm_h4": PPM_H4}

_D = ctypes.POINTER(ctypes.c_double)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_LIB = None


def lib() -> ctypes.CDLL:
    """The compiled oracle (built on first use if the shared object is missing)."""
    global _LIB
    if _LIB is None:
        path = _build.LIB if os.path.exists(_build.LIB) else _build.build()
        L = ctypes.CDLL(path)
        i, d, v = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
        L.oracle_advect_faces_h.argtypes = [_D, _D, _D, _U8, _D, i, i, i, i, i, i, i, i, i, _D, _D]
        L.oracle_advect_div.argtypes = [_D, _D, _D, _D, _U8, _D, i, i, i, i, i, i, i, i, i, i, _D]
        L.oracle_rk_stage.argtypes = [_D, _D, _D, d, _D, _D, i, ctypes.c_int64, ctypes.c_int64, _D, _D]
        L.oracle_fct_stage.argtypes = [_D, _D, _D, _D, d, d, d, _D, _D, i, i, i, i, _D, _D]
        L.oracle_fct_fluxes.argtypes = [_D, _D, _D, _D, i, i, i, i, i, i, i, i, _D, _D, _D, _D, _D, _D, _D, _D,
                                        _D, _D]
        L.oracle_fct_coeff.argtypes = [_D, _D, _D, _D, _D, _U8, d, i, i, i, i, _D, _D]
        L.oracle_fct_final.argtypes = [_D, _D, _D, _D, _D, _D, _D, d, _D, _D, i, i, i, i, _D]
        L.oracle_advect_fct.argtypes = [_D, _D, _D, _D, _D, _U8, v, i, i, i, i, i, i, i, i, i, d, _D, v, v]
        L.oracle_advect_fct.restype = i
        L.oracle_remap_column.argtypes = [_D, _D, i, _D, i, i, _D, _D]
        L.oracle_reconstruct.argtypes = [_D, _D, i, i, _D]
        L.oracle_remap_columns.argtypes = [_D, _D, _D, i, i, i, i, i, _U8, _D]
        L.oracle_regrid.argtypes = [i, _D, _D, _D, _U8, _D, d, i, i, i, _D, _U8]
        L.oracle_regrid.restype = i
        L.oracle_regrid_hybrid.argtypes = [_D, _D, _D, _U8, _D, _D, _D, _D, _D, d, d, d, i, i, i, i, _D, _U8]
        L.oracle_regrid_hybrid.restype = i
        L.oracle_regrid_columns.argtypes = [i, _D, _D, _D, _D, _D, _D, _D, _D, d, d, d, i, _U8, i, i, i, i, _D]
        L.oracle_regrid_columns.restype = None
        L.oracle_diffuse_ale.argtypes = [_D, _D, _D, _U8, _D, _D, _U8, _U8, _D, d, d, i, i, i, _D]
        L.oracle_face_fractions.argtypes = [_D, i, i, i, _D]
        L.oracle_ftt.argtypes = [_D, _D, _U8, i, i, i, i, _D, _D]
        L.oracle_transport_velocity.argtypes = [_D, _D, _U8, _D, _D, _D, d, d, i, i, i, _D, _D]
        L.oracle_ppm_edges.argtypes = [_D, _U8, d, i, i, i, _D, _D]
        L.oracle_ppm_transport.argtypes = [_D, _D, _D, _D, _D, _D, _D, _D, _U8, d, _D, i, i, i, i, _D]
        L.oracle_ppm_transport.restype = i
        L.oracle_outflow_exceeds.argtypes = [_D, _D, _D, _D, d, _U8, d, i, i, i]
        L.oracle_outflow_exceeds.restype = i
        L.oracle_limit_outflow.argtypes = [_D, _D, _D, _D, d, _U8, d, i, i, i, i, i, i, ctypes.POINTER(i)]
        L.oracle_limit_outflow.restype = i
        L.oracle_lagrangian_thickness.argtypes = [_D, _D, d, _D, d, i, i, i, _D]
        L.oracle_lagrangian_thickness.restype = ctypes.c_longlong
        L.oracle_upwind_transport.argtypes = [_D, _D, _D, _D, _D, i, i, i, _D]
        L.oracle_freshwater_volumes.argtypes = [_D, _D, _D, i, i, i, _D]
        L.oracle_freshwater_volumes.restype = i
        L.oracle_num_threads.restype = i
        L.oracle_set_threads.argtypes = [i]
        _LIB = L
    return _LIB


def set_threads(n: int) -> None:
    """OpenMP threads of the oracle's loops (results are identical for any count, as in the reference)."""
    lib().oracle_set_threads(int(n))


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _u8(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=bool).view(np.uint8)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _pu8(a: np.ndarray):
    return a.ctypes.data_as(_U8)


# ------------------------------------------------------------------------------------------------ periodic
class Periodic:
    """Restatement of ``core/model/periodic.py:47-94``: which horizontal axes wrap, and the pad/crop halo."""

    def __init__(self, axes=()) -> None:
        if isinstance(axes, str):
            axes = (axes,)
        axes = tuple(axes or ())
        bad = [a for a in axes if a not in ("x", "y")]
        if bad:
            raise ValueError(f"unknown periodic axes {bad}; use 'x', 'y' or both")
        self.x, self.y = "x" in axes, "y" in axes
        self.axes = tuple(a for a in ("x", "y") if a in axes)

    def __bool__(self) -> bool:
        return self.x or self.y

    @staticmethod
    def _index(n_cells: int, face: bool, halo: int) -> np.ndarray:
        return np.arange(-halo, n_cells + halo + (1 if face else 0)) % n_cells

    def pad(self, a, kind: str, halo: int) -> np.ndarray:
        a = np.asarray(a)
        if self.x:
            face = kind in ("u", "q")
            a = np.take(a, self._index(a.shape[-1] - face, face, halo), axis=-1)
        if self.y:
            face = kind in ("v", "q")
            a = np.take(a, self._index(a.shape[-2] - face, face, halo), axis=-2)
        return a

    def crop(self, a: np.ndarray, kind: str, halo: int) -> np.ndarray:
        if self.x:
            a = a[..., halo:a.shape[-1] - halo]
        if self.y:
            a = a[..., halo:a.shape[-2] - halo, :]
        return np.ascontiguousarray(a)


NONE = Periodic()


class OpenEdges:
    """The part of the reference's open-boundary object that the tracer path reads: ``open`` (edge names)."""

    def __init__(self, open_=()) -> None:
        self.open = tuple(open_)


# ------------------------------------------------------------------------------------------------ kernels
def advect_faces_h(c, Qx, Qy, ok, ext, open_w, open_e, open_s, open_n, z_variant):
    """``sigma_baroclinic.py:265-321``: WENO5 horizontal face fluxes (fx, fy) of the stack c."""
    c = _f64(c)
    nt, n, ny, nx = c.shape
    Qx, Qy, ext = _f64(Qx), _f64(Qy), _f64(ext)
    okc = _u8(np.broadcast_to(ok, c.shape[1:]))
    fx = np.empty((nt, n, ny, nx + 1))
    fy = np.empty((nt, n, ny + 1, nx))
    lib().oracle_advect_faces_h(_p(c), _p(Qx), _p(Qy), _pu8(okc), _p(ext), nt, n, ny, nx, int(open_w), int(open_e),
                                int(open_s), int(open_n), int(z_variant), _p(fx), _p(fy))
    return fx, fy


def advect_div(c, Qx, Qy, Fz, ok, ext, open_w, open_e, open_s, open_n, z_variant, vert):
    """``sigma_baroclinic.py:324-364``: −∇·(Q c) with WENO5 faces in x, y and (``vert``) z."""
    c = _f64(c)
    nt, n, ny, nx = c.shape
    out = np.empty_like(c)
    okc = _u8(np.broadcast_to(ok, c.shape[1:]))
    Qx, Qy, Fz, ext = _f64(Qx), _f64(Qy), _f64(Fz), _f64(ext)
    lib().oracle_advect_div(_p(c), _p(Qx), _p(Qy), _p(Fz), _pu8(okc), _p(ext), nt, n, ny, nx, int(open_w),
                            int(open_e), int(open_s), int(open_n), int(z_variant), int(vert), _p(out))
    return out


def _cell_at(c, ok, s):
    """Values and validity of cells m + s along the last axis, m = 0 .. n-1 (0 and invalid out of range), as the
    reference's ``_shift`` (``sigma_baroclinic.py:191-199``)."""
    n = c.shape[-1]
    val = np.zeros_like(c)
    valid = np.zeros(ok.shape, bool)
    a, b = max(0, -s), min(n, n - s)
    if a < b:
        val[..., a:b] = c[..., a + s:b + s]
        valid[..., a:b] = ok[..., a + s:b + s]
    return val, valid


def up3_faces(c, flux, ok, axis, order=3):
    """``sigma_baroclinic.py:164-188``: face values on the interior faces f = 1 .. n-1 along ``axis`` (between cells
    f-1 and f), upwind with respect to ``flux``: third order (-c[f-2] + 5 c[f-1] + 2 c[f]) / 6 for flux >= 0 and
    (2 c[f-1] + 5 c[f] - c[f+1]) / 6 otherwise where the three stencil cells are ok, the upwind cell elsewhere
    (everywhere for ``order`` 1); the two boundary faces 0."""
    c = np.moveaxis(c, axis, -1)
    ok = np.moveaxis(ok, axis, -1)
    f = np.moveaxis(flux, axis, -1)
    n = c.shape[-1]
    cm2, km2 = _cell_at(c, ok, -2)
    cm1, km1 = _cell_at(c, ok, -1)
    k0 = ok
    cp1, kp1 = _cell_at(c, ok, 1)
    # indexed at cell m = f: lo = cell f-1, hi = cell f
    lo, hi = cm1, c
    if order == 1:
        pos, neg = lo, hi
    else:
        pos = np.where(km2 & km1 & k0, (-cm2 + 5.0 * lo + 2.0 * hi) / 6.0, lo)
        neg = np.where(km1 & k0 & kp1, (2.0 * lo + 5.0 * hi - cp1) / 6.0, hi)
    face = np.zeros(f.shape)
    face[..., 1:n] = np.where(f[..., 1:n] >= 0, pos[..., 1:n], neg[..., 1:n])
    return np.moveaxis(face, -1, axis)


def centred_faces(c, ok, axis, n_out=None):
    """``sigma_baroclinic.py:632-652``: centred face values on the interior faces along ``axis``, sixth order
    (37 (c[f-1] + c[f]) - 8 (c[f-2] + c[f+1]) + (c[f-3] + c[f+2])) / 60 where all six cells are ok, fourth order
    (7 (c[f-1] + c[f]) - (c[f-2] + c[f+1])) / 12 where the inner four are, the mean of the two neighbours
    elsewhere; ``n_out`` faces (default n + 1), 0 outside 1 .. n-1."""
    c = np.moveaxis(c, axis, -1)
    ok = np.moveaxis(ok, axis, -1)
    n = c.shape[-1]
    cell = {s: _cell_at(c, ok, s) for s in range(-3, 3)}
    near = cell[-1][0] + cell[0][0]
    mid = cell[-2][0] + cell[1][0]
    far = cell[-3][0] + cell[2][0]
    f6 = (37 * near - 8 * mid + far) / 60
    f4 = (7 * near - mid) / 12
    f2 = 0.5 * near
    m6 = cell[-3][1] & cell[-2][1] & cell[-1][1] & cell[0][1] & cell[1][1] & cell[2][1]
    m4 = cell[-2][1] & cell[-1][1] & cell[0][1] & cell[1][1]
    face = np.zeros(c.shape[:-1] + (n + 1 if n_out is None else n_out,))
    face[..., 1:n] = np.where(m6, f6, np.where(m4, f4, f2))[..., 1:n]
    return np.moveaxis(face, -1, axis)


def fct_coefficients(c0, cL, V1, Ax, Ay, ok, dt):
    """``sigma_baroclinic.py:407-449`` (``_fct_coeff_kernel``): Zalesak coefficients (Cx, Cy)."""
    c0, cL, V1, Ax, Ay = _f64(c0), _f64(cL), _f64(V1), _f64(Ax), _f64(Ay)
    nt, n, ny, nx = c0.shape
    okc = _u8(np.broadcast_to(ok, c0.shape[1:]))
    Cx, Cy = np.empty_like(Ax), np.empty_like(Ay)
    lib().oracle_fct_coeff(_p(c0), _p(cL), _p(V1), _p(Ax), _p(Ay), _pu8(okc), float(dt), nt, n, ny, nx, _p(Cx),
                           _p(Cy))
    return Cx, Cy


def _rk_stage(qa, qb, r, dt, V, C, stage):
    """``sigma_baroclinic.py:856-875``: one SSP-RK3 stage with the ``safe`` rule."""
    qa, qb, r, V, C = _f64(qa), _f64(qb), _f64(r), _f64(V), _f64(C)
    q, c = np.empty_like(C), np.empty_like(C)
    lib().oracle_rk_stage(_p(qa), _p(qb), _p(r), float(dt), _p(V), _p(C), int(stage), C.size, V.size, _p(q), _p(c))
    return q, c


# ------------------------------------------------------------------------------------------------ component
class TracerAdvection:
    """Restatement of ``core/components/tracers.py:50-375`` (WENO5 SSP-RK3 paths, FCT and unlimited)."""

    def __init__(self, *, scheme: str = "weno5", time: str = "ssprk3", dt: float, ob=None) -> None:
        self.tracer_scheme, self.tracer_time, self.dt = scheme, time, dt
        self.ob = ob if ob is not None else OpenEdges()
        self.per = NONE
        self.record_open_flux = False
        self.last_open_flux = None

    # tracers.py:65-78
    def _open_inflow(self, Fx, Fy):
        opn = self.ob.open
        out = np.zeros(Fx.shape[0])
        for edge, F, sl, sgn in (("west", Fx, np.s_[..., 0], 1.0), ("east", Fx, np.s_[..., -1], -1.0),
                                 ("south", Fy, np.s_[..., 0, :], 1.0), ("north", Fy, np.s_[..., -1, :], -1.0)):
            if edge in opn:
                out += sgn * F[sl].reshape(F.shape[0], -1).sum(axis=1)
        return out

    # tracers.py:80-102
    def _periodic(self, method, C, V0, V1, Qx, Qy, Fz, ok, inflow, flux_face_i, **kw):
        per, H = self.per, TRACER_HALO
        pad = lambda a, kind: None if a is None else per.pad(a, kind, H)          # noqa: E731
        fi = None if flux_face_i is None else flux_face_i + (H if per.x else 0)
        args = [pad(C, "c"), pad(V0, "c"), pad(V1, "c"), pad(Qx, "u"), pad(Qy, "v")]
        if Fz is not None:
            args.append(pad(Fz, "c"))
        args.append(pad(np.broadcast_to(ok, np.shape(C)[1:]), "c"))
        self.per = NONE
        try:
            res = method(*args, inflow=pad(inflow, "c"), flux_face_i=fi, **kw)
        finally:
            self.per = per
        if fi is None:
            return per.crop(res, "c", H)
        out, fx = res
        if per.y:
            fx = np.ascontiguousarray(fx[..., H:fx.shape[-1] - H])
        return per.crop(out, "c", H), fx

    def _open_flags(self):
        o = self.ob.open
        return "west" in o, "east" in o, "south" in o, "north" in o

    # tracers.py:166-176
    def faces_h(self, c, Qx, Qy, ok, ext=None, inflow=None):
        c = _f64(c)
        e = (c if inflow is None else inflow) if ext is None else ext
        return advect_faces_h(c, Qx, Qy, ok, e, *self._open_flags(), self.tracer_scheme == "weno5")

    # tracers.py:178-193
    def upwind_faces_h(self, c, Qx, Qy, inflow=None):
        ext = c if inflow is None else inflow
        fx = np.zeros(c.shape[:3] + (c.shape[3] + 1,))
        fy = np.zeros(c.shape[:2] + (c.shape[2] + 1, c.shape[3]))
        fx[..., 1:-1] = Qx[None, ..., 1:-1] * np.where(Qx[None, ..., 1:-1] >= 0, c[..., :-1], c[..., 1:])
        fy[..., 1:-1, :] = Qy[None, :, 1:-1, :] * np.where(Qy[None, :, 1:-1, :] >= 0, c[..., :-1, :], c[..., 1:, :])
        opn = self.ob.open
        if "west" in opn:
            fx[..., 0] = Qx[None, ..., 0] * np.where(Qx[None, ..., 0] > 0, ext[..., 0], c[..., 0])
        if "east" in opn:
            fx[..., -1] = Qx[None, ..., -1] * np.where(Qx[None, ..., -1] < 0, ext[..., -1], c[..., -1])
        if "south" in opn:
            fy[..., 0, :] = Qy[None, :, 0, :] * np.where(Qy[None, :, 0, :] > 0, ext[..., 0, :], c[..., 0, :])
        if "north" in opn:
            fy[..., -1, :] = Qy[None, :, -1, :] * np.where(Qy[None, :, -1, :] < 0, ext[..., -1, :], c[..., -1, :])
        return fx, fy

    # tracers.py:110-115: the face values of the NumPy path (centred, or the upwind-3/1 schemes)
    def faces(self, c, flux, ok, axis, centred=False):
        if centred:
            return centred_faces(c, ok, axis, n_out=flux.shape[axis])
        if self.tracer_scheme.startswith("weno5"):
            raise NotImplementedError("oracle: WENO5 faces are restated through the fused kernels only")
        return up3_faces(c, flux, ok, axis, order=1 if self.tracer_scheme == "upwind1" else 3)

    # tracers.py:117-137: upstream values on the open-edge faces (the exterior on inflow)
    def open_faces(self, face, c, Q, axis, inflow=None):
        if not self.ob.open:
            return face
        ext = c if inflow is None else inflow
        face = np.array(face, copy=True)
        lo, hi = ("west", "east") if axis == 3 else ("south", "north")
        for edge, f_i, sgn in ((lo, 0, 1.0), (hi, -1, -1.0)):
            if edge not in self.ob.open:
                continue
            q = np.take(Q, f_i, axis=axis - 1)
            cf = np.take(c, f_i, axis=axis)
            ef = np.take(ext, f_i, axis=axis)
            idx = [slice(None)] * face.ndim
            idx[axis] = f_i
            face[tuple(idx)] = np.where(sgn * q > 0, ef, cf)
        return face

    # tracers.py:139-151: -div(Q c) with the NumPy faces (x, y, then z differences, the reference's order)
    def rhs_numpy(self, c, Qx, Qy, Fz, ok, centred=False, inflow=None):
        c = _f64(c)
        Qx, Qy, Fz = _f64(Qx), _f64(Qy), _f64(Fz)
        okb = np.broadcast_to(np.asarray(ok, bool), c.shape)
        fx = Qx * self.open_faces(self.faces(c, np.broadcast_to(Qx, c.shape[:1] + Qx.shape), okb, 3, centred),
                                  c, Qx, 3, inflow)
        fy = Qy * self.open_faces(self.faces(c, np.broadcast_to(Qy, c.shape[:1] + Qy.shape), okb, 2, centred),
                                  c, Qy, 2, inflow)
        fz = np.zeros(c.shape[:1] + Fz.shape)
        fz[:, :-1] = Fz[:-1] * self.faces(c, np.broadcast_to(Fz[:-1], c.shape), okb, 1, centred)
        return -(fx[..., 1:] - fx[..., :-1] + fy[:, :, 1:, :] - fy[:, :, :-1, :] + fz[:, 1:] - fz[:, :-1])

    # tracers.py:195-206: the x-face fluxes that ``rhs`` differences
    def flux_x(self, c, Qx, Qy, ok, centred=False, inflow=None):
        if not centred and self.tracer_scheme.startswith("weno5"):
            return self.faces_h(c, Qx, Qy, np.broadcast_to(ok, np.shape(c)[1:]), inflow=inflow)[0]
        c = _f64(c)
        Qx = _f64(Qx)
        okb = np.broadcast_to(np.asarray(ok, bool), c.shape)
        return Qx * self.open_faces(self.faces(c, np.broadcast_to(Qx, c.shape[:1] + Qx.shape), okb, 3, centred),
                                    c, Qx, 3, inflow)

    # tracers.py:153-164: the fused compiled kernel for WENO5 upwind faces, else the NumPy path
    def rhs(self, c, Qx, Qy, Fz, ok, centred=False, inflow=None):
        if centred or not self.tracer_scheme.startswith("weno5"):
            return self.rhs_numpy(c, Qx, Qy, Fz, ok, centred, inflow)
        c = _f64(c)
        ext = c if inflow is None else inflow
        return advect_div(c, Qx, Qy, Fz, ok, ext, *self._open_flags(), self.tracer_scheme == "weno5",
                          bool(np.any(np.asarray(Fz) != 0.0)))

    # tracers.py:208-254
    def advect_fct(self, C, V0, V1, Qx, Qy, ok, unlimited=False, inflow=None, flux_face_i=None):
        if self.per:
            return self._periodic(self.advect_fct, C, V0, V1, Qx, Qy, None, ok, inflow, flux_face_i,
                                  unlimited=unlimited)
        if unlimited:
            return self.advect_fct_numpy(C, V0, V1, Qx, Qy, ok, unlimited=True, inflow=inflow,
                                         flux_face_i=flux_face_i)
        dt = float(self.dt)
        C_in = C
        C = _f64(C)
        own = inflow is None or (inflow is C_in and C is C_in)     # ``ext is C`` of the reference (identity)
        Qx, Qy, V0, V1 = _f64(Qx), _f64(Qy), _f64(V0), _f64(V1)
        nt, n, ny, nx = C.shape
        okc = _u8(np.broadcast_to(ok, C.shape[1:]))
        infl = None if own else _f64(inflow)
        out = np.empty_like(C)
        want = self.record_open_flux or flux_face_i is not None
        Fx = np.empty((nt, n, ny, nx + 1)) if want else None
        Fy = np.empty((nt, n, ny + 1, nx)) if want else None
        w, e, s, nn = self._open_flags()
        rc = lib().oracle_advect_fct(_p(C), _p(V0), _p(V1), _p(Qx), _p(Qy), _pu8(okc),
                                     None if infl is None else infl.ctypes.data, nt, n, ny, nx, int(w), int(e),
                                     int(s), int(nn), int(self.tracer_scheme == "weno5"), dt, _p(out),
                                     None if Fx is None else Fx.ctypes.data, None if Fy is None else Fy.ctypes.data)
        if rc != 0:
            raise MemoryError("oracle_advect_fct: out of host memory")
        if self.record_open_flux:
            self.last_open_flux = self._open_inflow(Fx, Fy)
        if flux_face_i is None:
            return out
        return out, np.ascontiguousarray(Fx[..., flux_face_i])

    # tracers.py:256-301 (the unlimited branch; the limited branch is ``advect_fct``)
    def advect_fct_numpy(self, C, V0, V1, Qx, Qy, ok, unlimited=False, inflow=None, flux_face_i=None):
        if self.per:
            return self._periodic(self.advect_fct_numpy, C, V0, V1, Qx, Qy, None, ok, inflow, flux_face_i,
                                  unlimited=unlimited)
        if not unlimited:
            return self.advect_fct(C, V0, V1, Qx, Qy, ok, inflow=inflow, flux_face_i=flux_face_i)
        dt = self.dt
        C = np.asarray(C, float)
        V0, V1, Qx, Qy = (np.asarray(a, float) for a in (V0, V1, Qx, Qy))
        dV = V1 - V0
        div = lambda fx, fy: fx[..., 1:] - fx[..., :-1] + fy[..., 1:, :] - fy[..., :-1, :]   # noqa: E731
        safe = lambda q, v: np.where(v > 0, q / np.where(v > 0, v, 1.0), C)                  # noqa: E731
        q0 = V0 * C
        fx0, fy0 = self.faces_h(C, Qx, Qy, ok, inflow=inflow)
        q1 = q0 - dt * div(fx0, fy0)
        c1 = safe(q1, V0 + dV)
        fx1, fy1 = self.faces_h(c1, Qx, Qy, ok, inflow=inflow)
        q2 = 0.75 * q0 + 0.25 * (q1 - dt * div(fx1, fy1))
        c2 = safe(q2, V0 + 0.5 * dV)
        fx2, fy2 = self.faces_h(c2, Qx, Qy, ok, inflow=inflow)
        FHx = (fx0 + fx1) / 6.0 + 2.0 * fx2 / 3.0
        FHy = (fy0 + fy1) / 6.0 + 2.0 * fy2 / 3.0
        out = safe(q0 - dt * div(FHx, FHy), V1)
        i = flux_face_i
        return out if i is None else (out, FHx[..., i])

    # tracers.py:324-330: the 'pc' branch of advect_numpy (centred predictor to the half step, corrector from the
    # step's start with the upwind faces of the half-step tracer)
    def _advect_pc(self, C, V0, V1, Qx, Qy, Fz, ok, inflow, flux_face_i):
        dt = self.dt
        C = _f64(C)
        V0, V1 = np.asarray(V0, float), np.asarray(V1, float)
        dV = V1 - V0
        safe = lambda q, v: np.where(v > 0, q / np.where(v > 0, v, 1.0), C)     # noqa: E731
        q0 = V0 * C
        Vh = V0 + 0.5 * dV
        ch = safe(q0 + 0.5 * dt * self.rhs(C, Qx, Qy, Fz, ok, centred=True, inflow=inflow), Vh)
        out = safe(q0 + dt * self.rhs(ch, Qx, Qy, Fz, ok, inflow=inflow), V1)
        if flux_face_i is None:
            return out
        return out, self.flux_x(ch, Qx, Qy, ok, inflow=inflow)[..., flux_face_i]

    # tracers.py:342-375 (SSP-RK3; the fused WENO5 RHS or the NumPy one), 'pc' as advect_numpy
    def advect(self, C, V0, V1, Qx, Qy, Fz, ok, inflow=None, flux_face_i=None):
        if self.per:
            return self._periodic(self.advect, C, V0, V1, Qx, Qy, Fz, ok, inflow, flux_face_i)
        if self.tracer_time == "pc":
            return self._advect_pc(C, V0, V1, Qx, Qy, Fz, ok, inflow, flux_face_i)
        dt = self.dt
        C = _f64(C)
        if np.shape(V0) != C.shape[1:] or np.shape(V1) != C.shape[1:]:
            raise ValueError(f"_advect: volume shape {np.shape(V0)}/{np.shape(V1)} vs tracer layers {C.shape[1:]}")
        V0, V1 = np.asarray(V0, float), np.asarray(V1, float)
        dV = V1 - V0
        Va, Vb = V0 + dV, V0 + 0.5 * dV
        q0 = V0 * C
        q1, c1 = _rk_stage(q0, q0, self.rhs(C, Qx, Qy, Fz, ok, inflow=inflow), dt, Va, C, 1)
        q2, c2 = _rk_stage(q0, q1, self.rhs(c1, Qx, Qy, Fz, ok, inflow=inflow), dt, Vb, C, 2)
        _, c3 = _rk_stage(q0, q2, self.rhs(c2, Qx, Qy, Fz, ok, inflow=inflow), dt, V1, C, 3)
        if flux_face_i is None:
            return c3
        fx = lambda c: self.flux_x(c, Qx, Qy, ok, inflow=inflow)[..., flux_face_i]            # noqa: E731
        return c3, (fx(C) + fx(c1)) / 6.0 + 2.0 * fx(c2) / 3.0


# ------------------------------------------------------------------------------------------------ remap
def reconstruct(h, u, scheme):
    """``remap.py:234-294``: polynomial coefficients (n, 3) of one column."""
    h, u = _f64(h), _f64(u)
    coef = np.empty((h.size, 3))
    lib().oracle_reconstruct(_p(h), _p(u), h.size, int(scheme), _p(coef))
    return coef


def remap_column(h_src, u_src, h_tgt, scheme, u_tgt=None):
    """``remap.py:306-397``: conservative remap of one column; returns (and fills) u_tgt."""
    h_src, u_src, h_tgt = _f64(h_src), _f64(u_src), _f64(h_tgt)
    n0, n1 = h_src.size, h_tgt.size
    out = np.empty(n1)
    work = np.empty(10 * max(n0, n1) + 16)
    lib().oracle_remap_column(_p(h_src), _p(u_src), n0, _p(h_tgt), n1, int(scheme), _p(out), _p(work))
    if u_tgt is not None:
        u_tgt[...] = out
    return out


def remap_columns(h_src, f_src, h_tgt, scheme, wet):
    """``remap.py:418-427``: remap every wet column of f_src (N0, ny, nx) onto h_tgt (N1, ny, nx)."""
    h_src, f_src, h_tgt = _f64(h_src), _f64(f_src), _f64(h_tgt)
    n0, ny, nx = h_src.shape
    n1 = h_tgt.shape[0]
    out = np.empty(h_tgt.shape)
    w = _u8(np.broadcast_to(wet, (ny, nx)))
    lib().oracle_remap_columns(_p(h_src), _p(f_src), _p(h_tgt), n0, n1, ny, nx, int(scheme), _pu8(w), _p(out))
    return out


# ---------------------------------------------------------------------------------------------------- neighbours
H_MIN = 1e-3                           # core/vertical/regrid.py:41
RULES = {"zstar": 0, "sigma": 1}


def regrid(rule: str, H, eta, h_src, active, coord, h_min: float = H_MIN):
    """z* / sigma target thicknesses of ``ALECoordinate.regrid_remap`` (vertical_coordinate.py:69-78, 96-111):
    returns (h_new, wet, bad) with bad = wet columns that break the rule's precondition."""
    h_src = _f64(h_src)
    n, ny, nx = h_src.shape
    h_new = np.empty_like(h_src)
    wet = np.empty((ny, nx), np.uint8)
    bad = lib().oracle_regrid(RULES[rule], _p(_f64(H)), _p(_f64(eta)), _p(h_src),
                              _pu8(_u8(np.broadcast_to(active, (ny, nx)))), _p(_f64(coord)), float(h_min), n, ny,
                              nx, _p(h_new), _pu8(wet))
    return h_new, wet.view(bool), int(bad)


def regrid_hybrid(H, eta, h_src, active, rho, params: dict):
    """The hybrid rule of ``_regrid_columns`` (regrid.py:309-342) as ``ALECoordinate.regrid`` uses it (n_out = the
    source layer count): (h_new, wet, bad)."""
    h_src = _f64(h_src)
    n, ny, nx = h_src.shape
    f = lambda key, default: _f64(params.get(key, default))                        # noqa: E731
    h_new = np.empty_like(h_src)
    wet = np.empty((ny, nx), np.uint8)
    bad = lib().oracle_regrid_hybrid(_p(_f64(H)), _p(_f64(eta)), _p(h_src),
                                     _pu8(_u8(np.broadcast_to(active, (ny, nx)))), _p(_f64(rho)),
                                     _p(f("rho_target", np.zeros(n + 1))), _p(f("dz_top", np.ones(n))),
                                     _p(f("max_h_top", np.full(n, np.inf))), _p(f("dsigma", np.full(n, 1.0 / n))),
                                     float(params.get("d_sigma", 0.0)), float(params.get("d_hybrid", 0.0)),
                                     float(params.get("h_min", H_MIN)), int(bool(params.get("keep_isopycnal", True))),
                                     n, ny, nx, _p(h_new), _pu8(wet))
    return h_new, wet.view(bool), int(bad)


def regrid_columns(rule: str, H, eta, h, rho, params: dict, wet, n_out=None):
    """``regrid_columns`` (core/vertical/regrid.py:345-395): target interface heights zw (N+1, ny, nx), bed first,
    N = n_out (default the source layer count; only the hybrid rule regrids a source of another count), NaN in the
    columns that are not wet; ValueError where the reference raises."""
    if rule not in ("zstar", "sigma", "hybrid"):
        raise ValueError(f"unknown rule {rule!r}; use 'zstar', 'sigma' or 'hybrid'")
    required = {"zstar": ("dz_top",), "sigma": ("dsigma",), "hybrid": ("dz_top", "rho_target")}[rule]
    if rule == "hybrid" and float(params.get("d_hybrid", 0.0)) > 0.0:
        required += ("dsigma",)
    for key in required:
        if key not in params:
            raise ValueError(f"regrid_columns({rule!r}) needs params[{key!r}]")
    if rule == "hybrid" and rho is None:
        raise ValueError("regrid_columns('hybrid') needs the layer densities rho")
    wet = np.asarray(wet, np.bool_)
    H = np.asarray(H, float)
    eta = np.asarray(eta, float)
    Hw, Dw = H[wet], (H + eta)[wet]
    if not (np.isfinite(Hw).all() and np.isfinite(Dw).all() and (Dw > 0).all()):
        raise ValueError("wet columns need finite H and D = H + eta > 0")
    if rule == "zstar" and not (Hw > 0).all():
        raise ValueError("z* needs H > 0 in every wet column")
    if rule == "hybrid" and float(params.get("d_hybrid", 0.0)) <= 0 and (Hw <= 0).any():
        raise ValueError("hybrid needs H > 0 unless it has a shallow sigma zone (d_hybrid > 0)")
    if rule == "hybrid" and not np.isfinite(np.asarray(rho, float)[:, wet]).all():
        raise ValueError("non-finite density in a wet column")
    h = _f64(h)
    n_src, ny, nx = h.shape
    m = n_src if n_out is None else int(n_out)
    if m != n_src and rule != "hybrid":
        raise ValueError("n_out != the source layer count is only for rule 'hybrid'")
    f = lambda key, default: _f64(params.get(key, default))                        # noqa: E731
    zw = np.full((m + 1, ny, nx), np.nan)
    lib().oracle_regrid_columns({"zstar": 0, "sigma": 1, "hybrid": 2}[rule], _p(_f64(np.nan_to_num(H))),
                                _p(_f64(eta)), _p(h), _p(h if rho is None else _f64(rho)),
                                _p(f("dz_top", np.ones(m))), _p(f("dsigma", np.full(m, 1.0 / m))),
                                _p(f("rho_target", np.zeros(m + 1))), _p(f("max_h_top", np.full(m, np.inf))),
                                float(params.get("d_sigma", 0.0)), float(params.get("d_hybrid", 0.0)),
                                float(params.get("h_min", H_MIN)), int(bool(params.get("keep_isopycnal", True))),
                                _pu8(_u8(wet)), n_src, m, ny, nx, _p(zw))
    return zw


def regrid_remap(rule: str, H, eta, h_src, active, fields, coord, scheme: int, h_min: float = H_MIN):
    """(h_new, [remap_columns(h_src, f, h_new, scheme, wet) for f in fields]) as ``ALECoordinate.regrid_remap``
    with the z* or sigma rule; ValueError where the reference's ``regrid_columns`` raises (z* and H <= 0)."""
    h_new, wet, bad = regrid(rule, H, eta, h_src, active, coord, h_min)
    if bad:
        raise ValueError("z* needs H > 0 in every wet column (cells that can dry: sigma, or hybrid with d_hybrid > 0)")
    return h_new, [remap_columns(h_src, f, h_new, scheme, wet) for f in fields]


def diffuse_ale(T, Tw, h, act, cx, cy, okx, oky, V, kh: float, dt: float, per=None):
    """``_diffuse_ale_kernel`` on one field (N, ny, nx); periodic axes by pad/crop with halo 1 as
    ``TracerAdvection.diffuse_h`` (tracers.py:436-447).  ``h`` is passed as the kernel receives it."""
    per = per or NONE

    def run(T, Tw, h, act, cx, cy, okx, oky, V):
        T, Tw, h, V = _f64(T), _f64(Tw), _f64(h), _f64(V)
        n, ny, nx = T.shape
        out = np.empty_like(T)
        lib().oracle_diffuse_ale(_p(T), _p(Tw), _p(h), _pu8(_u8(act)), _p(_f64(cx)), _p(_f64(cy)),
                                 _pu8(_u8(okx)), _pu8(_u8(oky)), _p(V), float(kh), float(dt), n, ny, nx, _p(out))
        return out

    args = (T, Tw, h, act, cx, cy, okx, oky, V)
    if per:
        kinds = ("c", "c", "c", "c", "u", "v", "u", "v", "c")
        return per.crop(run(*(per.pad(a, k, 1) for a, k in zip(args, kinds))), "c", 1)
    return run(*args)


def face_fractions(hf) -> np.ndarray:
    """``_fractions_kernel`` (ale.py:883-892) on (N, a, b)."""
    hf = _f64(hf)
    n, a, b = hf.shape
    w = np.empty_like(hf)
    lib().oracle_face_fractions(_p(hf), n, a, b, _p(w))
    return w


def remap_faces(vel, hf_src, hf_tgt, scheme: int, w_tgt=None):
    """``ALECoordinate.remap_faces`` (vertical_coordinate.py:142-153): the velocity remap in fraction space,
    thicknesses w_src S -> w_tgt S with the column total S of hf_src (summed k = 0 .. N-1)."""
    hf_src = _f64(hf_src)
    tot = np.zeros(hf_src.shape[1:])
    for k in range(hf_src.shape[0]):
        tot = tot + hf_src[k]
    wet = tot > 0
    S = np.where(wet, tot, 1.0)[None]
    w_tgt = face_fractions(hf_tgt) if w_tgt is None else _f64(w_tgt)
    return remap_columns(face_fractions(hf_src) * S, vel, w_tgt * S, scheme, wet)


# ---------------------------------------------------------------------------------------------------- producers
H_PPM_MIN = 2e-10                      # core/vertical/ale.py:297


def face_transport_thickness(h, H, active, clip: bool):
    """``_ftt_kernel`` (ale.py:177-210): (q_e, q_w) on the u-faces."""
    h = _f64(h)
    n, ny, nx = h.shape
    q_e, q_w = np.empty((n, ny, nx + 1)), np.empty((n, ny, nx + 1))
    lib().oracle_ftt(_p(h), _p(_f64(H)), _pu8(_u8(active)), int(bool(clip)), n, ny, nx, _p(q_e), _p(q_w))
    return q_e, q_w


def transport_velocity(u_new, u_old, last_wet, w, L, D, theta: float, theta_bc: float | None = None):
    """``_transport_velocity_kernel`` (ale.py:789-808): (u^theta, Q_bt)."""
    u_new = _f64(u_new)
    n, a, b = u_new.shape
    ut, Qb = np.empty((n, a, b)), np.empty((a, b))
    tb = theta if theta_bc is None else theta_bc
    lib().oracle_transport_velocity(_p(u_new), _p(_f64(u_old)), _pu8(_u8(last_wet)), _p(_f64(w)), _p(_f64(L)),
                                    _p(_f64(D)), float(theta), float(tb), n, a, b, _p(ut), _p(Qb))
    return ut, Qb


def _masked(h, active):
    return np.ascontiguousarray(np.where(np.asarray(active, bool)[None], np.nan_to_num(np.asarray(h, float)), 0.0))


def ppm_edges_x(h, active, h_min: float = H_PPM_MIN):
    """``_ppm_edges_kernel`` (ale.py:582-626) on where(active, nan_to_num(h), 0)."""
    hc = _masked(h, active)
    n, ny, nx = hc.shape
    h_w, h_e = np.empty_like(hc), np.empty_like(hc)
    lib().oracle_ppm_edges(_p(hc), _pu8(_u8(active)), float(h_min), n, ny, nx, _p(h_w), _p(h_e))
    return h_w, h_e


def ppm_transport_x(h, ut, L, Q_bt, q_e, q_w, active, dt: float, dx_t, max_iter: int = 20):
    """``ppm_transport_x`` (ale.py:743-764): PPM layer fluxes with the barotropic correction (u-faces)."""
    hc = _masked(h, active)
    n, ny, nx = hc.shape
    h_w, h_e = ppm_edges_x(hc, active)
    out = np.empty((n, ny, nx + 1))
    lib().oracle_ppm_transport(_p(hc), _p(h_w), _p(h_e), _p(_f64(ut)), _p(_f64(L)), _p(_f64(Q_bt)), _p(_f64(q_e)),
                               _p(_f64(q_w)), _pu8(_u8(active)), float(dt), _p(_f64(dx_t)), int(max_iter), n, ny, nx,
                               _p(out))
    return out


def limit_outflow(h, Qx, Qy, area, dt: float, active, h_floor: float = H_PPM_MIN, max_pass: int = 50,
                  periodic=(False, False)):
    """``limit_outflow`` (ale.py:331-395): (Qx, Qy, n_limited); the inputs themselves when nothing exceeds;
    RuntimeError where the reference raises."""
    h, Qx, Qy, area = _f64(h), _f64(Qx), _f64(Qy), _f64(area)
    n, ny, nx = h.shape
    act = _u8(active)
    if not lib().oracle_outflow_exceeds(_p(h), _p(Qx), _p(Qy), _p(area), float(dt), _pu8(act), float(h_floor), n,
                                        ny, nx):
        return Qx, Qy, 0
    Qx, Qy = Qx.copy(), Qy.copy()
    nl = ctypes.c_int(0)
    st = lib().oracle_limit_outflow(_p(h), _p(Qx), _p(Qy), _p(area), float(dt), _pu8(act), float(h_floor),
                                    int(max_pass), int(bool(periodic[0])), int(bool(periodic[1])), n, ny, nx,
                                    ctypes.byref(nl))
    if st >= 2:
        raise RuntimeError("limit_outflow: " + ("barotropic CFL" if st == 2 else "flow out of a dry donor column"))
    return Qx, Qy, int(nl.value)


def lagrangian_thickness(h, divq, dt: float, area, tol: float = 1e-9):
    """``lagrangian_thickness`` (ale.py:278-294)."""
    h = _f64(h)
    n, ny, nx = h.shape
    out = np.empty_like(h)
    bad = lib().oracle_lagrangian_thickness(_p(h), _p(_f64(divq)), float(dt), _p(_f64(area)), float(tol), n, ny, nx,
                                            _p(out))
    if bad >= 0:
        k, j, i = np.unravel_index(int(bad), h.shape)
        v = h[k, j, i] - dt * _f64(divq)[k, j, i] / (area[j, i] if area[j, i] > 0 else 1.0)
        raise RuntimeError(f"layer {k} of cell (j={j}, i={i}) emptied in the Lagrangian step: h† = {v:.3e} m "
                           f"(reduce dt)")
    return out


def upwind_transport_x(q_e, q_w, ut, L, Q_bt) -> np.ndarray:
    """``upwind_transport_x`` (ale.py:233-251): donor-cell layer fluxes consistent with the free-surface flux."""
    ut = _f64(ut)
    n, a, b = ut.shape
    out = np.empty_like(ut)
    lib().oracle_upwind_transport(_p(_f64(q_e)), _p(_f64(q_w)), _p(ut), _p(_f64(np.broadcast_to(L, (a, b)))),
                                  _p(_f64(np.broadcast_to(Q_bt, (a, b)))), n, a, b, _p(out))
    return out


DZ_FLOOR = 1e-6                        # core/vertical/ale.py:63


def open_face_transport(h_int, u_new, u_old, Q_bt, L, theta: float, theta_bc=None):
    """``open_face_transport`` (core/vertical/ale.py:841-861): the layer fluxes through the faces of one open edge,
    the Flather flux Q_bt split with the interior thickness fractions; h_int, u_new, u_old (N, m), Q_bt, L (m,)."""
    tot = h_int.sum(axis=0)
    wet = tot > 0
    w = np.where(wet[None], h_int / np.where(wet, tot, 1.0)[None], 0.0)
    pn = u_new - (w * u_new).sum(axis=0)[None]
    po = u_old - (w * u_old).sum(axis=0)[None]
    tb = theta if theta_bc is None else theta_bc
    Q = w * Q_bt[None] + L[None] * h_int * (tb * pn + (1.0 - tb) * po)
    return np.where(wet[None], Q, 0.0)


def open_face_transports(Qx, Qy, h, un, vn, u_new, v_new, open_, open_Du, open_Dv, open_Qu, open_Qv, Lu, Lv,
                         theta: float, theta_bc: float) -> None:
    """In place, the open faces of Qx / Qy where the open face depth is positive
    (core/components/open_boundary.py:334-352)."""
    for edge, Q, D, Qo, L, hc, vo, vn1 in (
            ("west", Qx[..., 0], open_Du[:, 0], open_Qu[:, 0], Lu[:, 0], h[..., 0], un[..., 0], u_new[..., 0]),
            ("east", Qx[..., -1], open_Du[:, -1], open_Qu[:, -1], Lu[:, -1], h[..., -1], un[..., -1],
             u_new[..., -1]),
            ("south", Qy[:, 0, :], open_Dv[0, :], open_Qv[0, :], Lv[0, :], h[:, 0, :], vn[:, 0, :], v_new[:, 0, :]),
            ("north", Qy[:, -1, :], open_Dv[-1, :], open_Qv[-1, :], Lv[-1, :], h[:, -1, :], vn[:, -1, :],
             v_new[:, -1, :])):
        if edge in open_:
            Q[...] = np.where((D > 0)[None], open_face_transport(hc, vn1, vo, Qo, L, theta, theta_bc), Q)


def ale_layer_transport(h, u_old, v_old, u_new, v_new, wet_u, wet_v, wu, wv, Lu, Lv, Du, Dv, qe, qw, qn, qs, active,
                        area, dx_t, dy_t, dt: float, theta: float, theta_bc: float, thickness_flux: str = "ppm",
                        periodic=(False, False), fw=None, open_=(), open_Du=None, open_Dv=None, open_Qu=None,
                        open_Qv=None) -> dict:
    """``ALELayerTransport.__call__`` (core/components/layer_transport.py:111-156) from the restatements above:
    transport velocities, the PPM or donor-cell layer fluxes (v-faces on swapped axes; the periodic PPM flux on
    inputs padded by four wrapped positions and cropped, as the reference does), the open faces, the outflow
    limiter, h-dagger, the layer volumes h A, ok = active & V1 > 0 and, with freshwater, h_fw and V_fw.  ``qn``,
    ``qs`` are the v-face thicknesses in the swapped (N, nx, ny+1) layout the reference passes."""
    sw = lambda a: np.ascontiguousarray(np.swapaxes(a, 1, 2))                       # noqa: E731
    utx, Qbx = transport_velocity(u_new, u_old, wet_u, wu, Lu, Du, theta, theta_bc)
    uty, Qby = transport_velocity(v_new, v_old, wet_v, wv, Lv, Dv, theta, theta_bc)
    if thickness_flux == "ppm":
        def both(h_, ux, uy, Lu_, Lv_, bx, by, e, w, n_, s_, a, dx, dy):
            return (ppm_transport_x(h_, ux, Lu_, bx, e, w, a, dt, dx),
                    sw(ppm_transport_x(sw(h_), sw(uy), np.ascontiguousarray(Lv_.T), np.ascontiguousarray(by.T),
                                       sw(n_), sw(s_), np.ascontiguousarray(a.T), dt, np.ascontiguousarray(dy.T))))
        if any(periodic):
            per = Periodic(tuple(ax for ax, f in zip(("x", "y"), periodic) if f))
            args = (h, utx, uty, Lu, Lv, Qbx, Qby, qe, qw, sw(qn), sw(qs), active, dx_t, dy_t)
            kinds = ("c", "u", "v", "u", "v", "u", "v", "u", "u", "v", "v", "c", "c", "c")
            Qx, Qy = both(*(np.ascontiguousarray(per.pad(a, k, 4)) for a, k in zip(args, kinds)))
            Qx, Qy = per.crop(Qx, "u", 4), per.crop(Qy, "v", 4)
        else:
            Qx, Qy = both(h, utx, uty, Lu, Lv, Qbx, Qby, qe, qw, sw(qn), sw(qs), active, dx_t, dy_t)
    else:
        Qx = upwind_transport_x(qe, qw, utx, Lu, Qbx)
        Qy = sw(upwind_transport_x(qn, qs, sw(uty), Lv.T, Qby.T))
    if open_:
        Qx, Qy = np.array(Qx), np.array(Qy)
        open_face_transports(Qx, Qy, h, u_old, v_old, u_new, v_new, tuple(open_), open_Du, open_Dv, open_Qu,
                             open_Qv, Lu, Lv, theta, theta_bc)
    Qx, Qy, n_lim = limit_outflow(h, Qx, Qy, area, dt, active, periodic=tuple(periodic))
    divh = Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:, :] - Qy[:, :-1, :]
    h_lag = lagrangian_thickness(h, divh, dt, area)
    V0, V1 = h * area[None], h_lag * area[None]
    ok = np.broadcast_to(active[None], V1.shape) & (V1 > 0)
    out = dict(Qx=Qx, Qy=Qy, V0=V0, V1=V1, ok=ok, h_dagger=h_lag, n_limited=n_lim)
    if fw is not None:
        h_fw, _ = freshwater_volumes(h_lag, dt * fw, DZ_FLOOR)
        out.update(h_fw=h_fw, V_fw=h_fw * area[None])
    return out


def freshwater_volumes(V, dV, floor):
    """``freshwater_volumes`` (core/components/freshwater.py:31-58): (V_new, n_limited)."""
    V = _f64(V)
    n, ny, nx = V.shape
    out = np.empty_like(V)
    nl = lib().oracle_freshwater_volumes(_p(V), _p(_f64(dV)), _p(_f64(np.broadcast_to(floor, (ny, nx)))), n, ny, nx,
                                         _p(out))
    return out, int(nl)
