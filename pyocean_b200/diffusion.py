"""
ALE horizontal diffusion of tracers along the layers, on B200: ``_diffuse_ale_kernel``
(core/dynamics/sigma_baroclinic.py:533-561) as ``TracerAdvection.diffuse_h`` calls it
(core/components/tracers.py:421-447), with periodic axes handled natively instead of by a halo-1 pad/crop.

    F_x = ((-K_h L_u / dx_u) min(h_L, h_R)) (Tw_i - Tw_{i-1})  on faces between active cells with okx,
    T_new = T - dt div F / V  where V > 0.

``diffuse_ale`` takes the kernel's arguments (the caller forms Tw and masks h, as ``diffuse_h`` does); ``T`` and
``Tw`` may be one field (N, ny, nx) or a stack (nt, N, ny, nx) sharing the geometry.
"""
from __future__ import annotations

from . import _lib
from ._device import Converter, shape_of
from .periodic import NONE


def diffuse_ale(T, Tw, h, act, cx, cy, okx, oky, V, kh: float, dt: float, per=None):
    per = per or NONE
    shp = shape_of(T)
    if len(shp) not in (3, 4) or shape_of(Tw) != shp:
        raise ValueError(f"T and Tw must be (N, ny, nx) or (nt, N, ny, nx) and alike, got {shp} and {shape_of(Tw)}")
    n, ny, nx = shp[-3:]
    nt = shp[0] if len(shp) == 4 else 1
    if shape_of(h) != (n, ny, nx) or shape_of(V) != (n, ny, nx):
        raise ValueError(f"h {shape_of(h)} and V {shape_of(V)} must be {(n, ny, nx)}")
    cv = Converter(T, Tw, h, V, cx, cy)
    Td, Twd, hd, Vd = cv.f64(T), cv.f64(Tw), cv.f64(h), cv.f64(V)
    cxd, cyd = cv.f64(cx, (ny, nx + 1)), cv.f64(cy, (ny + 1, nx))
    ad, oxd, oyd = cv.u8(act, (ny, nx)), cv.u8(okx, (ny, nx + 1)), cv.u8(oky, (ny + 1, nx))
    out = cv.empty(shp)
    flags = (_lib.PERIODIC_X if getattr(per, "x", False) else 0) | (_lib.PERIODIC_Y if getattr(per, "y", False) else 0)
    rc = _lib.lib().pocean_diffuse_ale_f64(Td.data_ptr(), Twd.data_ptr(), hd.data_ptr(), ad.data_ptr(),
                                           cxd.data_ptr(), cyd.data_ptr(), oxd.data_ptr(), oyd.data_ptr(),
                                           Vd.data_ptr(), nt, n, ny, nx, flags, float(kh), float(dt), out.data_ptr(),
                                           cv.stream())
    _lib.check(rc, "diffuse_ale")
    return cv.out(out)
