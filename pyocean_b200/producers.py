"""
The producers of the tracer step's inputs, with the reference's interface (core/vertical/ale.py), on B200:
``face_transport_thickness``, ``transport_velocity``, ``ppm_edges_x``, ``ppm_transport_x``, ``limit_outflow`` and
``lagrangian_thickness``.  With CUDA tensors the fluxes, h-dagger and everything in between stay in HBM, so a model
that keeps its state on the device runs the whole ALE tracer step (these, then ``TracerAdvection.advect_fct`` and
the remap) without a host round trip.  For v-faces call them on swapped horizontal axes, as the reference does
(non-contiguous arrays are made contiguous).  Results are the reference's, bit for bit.
"""
from __future__ import annotations

import ctypes
import warnings

import numpy as np
import torch

from . import _lib
from ._device import Converter, shape_of

H_PPM_MIN = 2e-10                      # core/vertical/ale.py:297


def face_transport_thickness(h, H, active, clip: bool):
    """(q_E, q_W) (N, ny, nx+1): the layer thickness available for transport from the west / east cell
    (ale.py:212-231)."""
    n, ny, nx = shape_of(h)
    cv = Converter(h, H)
    hd, Hd, ad = cv.f64(h), cv.f64(H, (ny, nx)), cv.u8(active, (ny, nx))
    q_e, q_w = cv.empty((n, ny, nx + 1)), cv.empty((n, ny, nx + 1))
    _lib.check(_lib.lib().pocean_face_transport_thickness_f64(hd.data_ptr(), Hd.data_ptr(), ad.data_ptr(), n, ny, nx,
                                                              int(bool(clip)), q_e.data_ptr(), q_w.data_ptr(),
                                                              cv.stream()), "face_transport_thickness")
    return cv.out(q_e), cv.out(q_w)


def transport_velocity(u_new, u_old, last_wet, w, L, D, theta: float, theta_bc: float | None = None):
    """(u^theta, Q_bt) of the ALE step (ale.py:811-825)."""
    n, a, b = shape_of(u_new)
    if shape_of(u_old) != (n, a, b) or shape_of(w) != (n, a, b) or any(
            shape_of(x) != (a, b) for x in (last_wet, L, D)):
        raise ValueError(f"transport_velocity: shapes u_new {shape_of(u_new)}, u_old {shape_of(u_old)}, "
                         f"w {shape_of(w)}, last_wet/L/D {shape_of(last_wet)}/{shape_of(L)}/{shape_of(D)}")
    cv = Converter(u_new, u_old, w, L, D)
    un, uo, wd, Ld, Dd = cv.f64(u_new), cv.f64(u_old), cv.f64(w), cv.f64(L), cv.f64(D)
    lw = cv.u8(last_wet, (a, b))
    ut, Qb = cv.empty((n, a, b)), cv.empty((a, b))
    tb = theta if theta_bc is None else theta_bc
    _lib.check(_lib.lib().pocean_transport_velocity_f64(un.data_ptr(), uo.data_ptr(), lw.data_ptr(), wd.data_ptr(),
                                                        Ld.data_ptr(), Dd.data_ptr(), n, a, b, float(theta), float(tb),
                                                        ut.data_ptr(), Qb.data_ptr(), cv.stream()),
               "transport_velocity")
    return cv.out(ut), cv.out(Qb)


def ppm_edges_x(h, active, h_min: float = H_PPM_MIN):
    """West and east PPM edge values of the layer thickness (ale.py:445-480)."""
    n, ny, nx = shape_of(h)
    cv = Converter(h)
    hd, ad = cv.f64(h), cv.u8(active, (ny, nx))
    h_w, h_e = cv.empty((n, ny, nx)), cv.empty((n, ny, nx))
    _lib.check(_lib.lib().pocean_ppm_edges_f64(hd.data_ptr(), ad.data_ptr(), n, ny, nx, float(h_min), h_w.data_ptr(),
                                               h_e.data_ptr(), cv.stream()), "ppm_edges_x")
    return cv.out(h_w), cv.out(h_e)


def ppm_transport_x(h, ut, L, Q_bt, q_e, q_w, active, dt: float, dx_t, max_iter: int = 20):
    """Layer volume fluxes through the u-faces with PPM thickness and the barotropic correction
    (ale.py:743-764)."""
    n, ny, nx = shape_of(h)
    cv = Converter(h, ut, L, Q_bt, q_e, q_w, dx_t)
    hd, utd, Ld, Qd = cv.f64(h), cv.f64(ut), cv.f64(L), cv.f64(Q_bt)
    qed, qwd, dxd, ad = cv.f64(q_e), cv.f64(q_w), cv.f64(dx_t, (ny, nx)), cv.u8(active, (ny, nx))
    out = cv.empty((n, ny, nx + 1))
    L_ = _lib.lib()
    nbytes = L_.pocean_ppm_transport_workspace_bytes(n, ny, nx, int(max_iter))
    ws = cv.workspace(nbytes)
    _lib.check(L_.pocean_ppm_transport_f64(hd.data_ptr(), utd.data_ptr(), Ld.data_ptr(), Qd.data_ptr(),
                                           qed.data_ptr(), qwd.data_ptr(), ad.data_ptr(), dxd.data_ptr(), n, ny, nx,
                                           float(dt), int(max_iter), out.data_ptr(), ws.data_ptr(), nbytes,
                                           cv.stream()), "ppm_transport_x")
    return cv.out(out)


def limit_outflow(h, Qx, Qy, area, dt: float, active, h_floor: float = H_PPM_MIN, max_pass: int = 50,
                  periodic=(False, False)):
    """(Qx, Qy, n_limited): no active layer sends out more than it holds in dt, the cut flux given back to the other
    layers of each face (ale.py:331-395).  The inputs themselves when nothing exceeds; RuntimeError where the
    reference raises; RuntimeWarning where it warns."""
    n, ny, nx = shape_of(h)
    cv = Converter(h, Qx, Qy, area)
    hd, ar, ad = cv.f64(h), cv.f64(area, (ny, nx)), cv.u8(active, (ny, nx))
    Qxd = cv.f64(Qx).clone() if isinstance(Qx, torch.Tensor) else cv.f64(Qx)
    Qyd = cv.f64(Qy).clone() if isinstance(Qy, torch.Tensor) else cv.f64(Qy)
    L_ = _lib.lib()
    nbytes = L_.pocean_limit_outflow_workspace_bytes(n, ny, nx)
    ws = cv.workspace(nbytes)
    nl, warned = ctypes.c_int(0), ctypes.c_int(0)
    flags = (_lib.PERIODIC_X if periodic[0] else 0) | (_lib.PERIODIC_Y if periodic[1] else 0)
    rc = L_.pocean_limit_outflow_f64(hd.data_ptr(), Qxd.data_ptr(), Qyd.data_ptr(), ar.data_ptr(), ad.data_ptr(), n,
                                     ny, nx, float(dt), float(h_floor), int(max_pass), flags, ctypes.byref(nl),
                                     ctypes.byref(warned), ws.data_ptr(), nbytes, cv.stream())
    _lib.check(rc, "limit_outflow")
    if nl.value == 0 and not warned.value:
        return Qx, Qy, 0
    if warned.value:
        warnings.warn(f"limit_outflow: a layer still sends out more than it holds after {max_pass} passes, but its "
                      f"inflow keeps h >= 0; the FCT bound is weaker there", RuntimeWarning, stacklevel=2)
    return cv.out(Qxd), cv.out(Qyd), int(nl.value)


def lagrangian_thickness(h, divq, dt: float, area, tol: float = 1e-9):
    """h-dagger = h - dt div(Q) / A, clamped at 0; RuntimeError for a layer emptied beyond tol (ale.py:278-294)."""
    n, ny, nx = shape_of(h)
    cv = Converter(h, divq, area)
    hd, dd, ar = cv.f64(h), cv.f64(divq), cv.f64(area, (ny, nx))
    out = cv.empty((n, ny, nx))
    bad = torch.empty(1, dtype=torch.int64, device=cv.device)
    _lib.check(_lib.lib().pocean_lagrangian_thickness_f64(hd.data_ptr(), dd.data_ptr(), ar.data_ptr(), n, ny, nx,
                                                          float(dt), float(tol), out.data_ptr(), bad.data_ptr(),
                                                          cv.stream()), "lagrangian_thickness")
    b = int(bad.item())
    if b != -1:                                           # ~0 read as a signed 64-bit integer
        k, j, i = np.unravel_index(b, (n, ny, nx))
        a = float(ar[j, i])
        v = float(hd[k, j, i]) - dt * float(dd[k, j, i]) / (a if a > 0 else 1.0)
        raise RuntimeError(f"layer {k} of cell (j={j}, i={i}) emptied in the Lagrangian step: h† = {v:.3e} m "
                           f"(reduce dt)")
    return cv.out(out)
