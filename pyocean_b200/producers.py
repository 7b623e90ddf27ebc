"""
The producers of the tracer step's inputs, with the reference's interface (core/vertical/ale.py), on B200:
``face_transport_thickness``, ``transport_velocity``, ``ppm_edges_x``, ``ppm_transport_x``, ``upwind_transport_x``,
``limit_outflow`` and ``lagrangian_thickness``; ``freshwater_volumes`` (core/components/freshwater.py); and the whole
Lagrangian step of ``ALELayerTransport`` (core/components/layer_transport.py:98-160) built from them.  With CUDA
tensors the fluxes, h-dagger and everything in between stay in HBM, so a model that keeps its state on the device
runs the whole ALE tracer step (these, then ``TracerAdvection.advect_fct`` and the remap) without a host round
trip.  For v-faces call them on swapped horizontal axes, as the reference does
(non-contiguous arrays are made contiguous).  Results are the reference's, bit for bit.
"""
from __future__ import annotations

import ctypes
import warnings
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._device import Converter, shape_of

H_PPM_MIN = 2e-10                      # core/vertical/ale.py:297
DZ_FLOOR = 1e-6                        # core/vertical/ale.py:63


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


def upwind_transport_x(q_e, q_w, ut, L, Q_bt):
    """Donor-cell layer fluxes through the u-faces consistent with the free-surface flux (ale.py:233-251)."""
    n, a, b = shape_of(ut)
    cv = Converter(q_e, q_w, ut, L, Q_bt)
    qe, qw, u = cv.f64(q_e), cv.f64(q_w), cv.f64(ut)
    Ld, Qd = cv.f64(L, (a, b)), cv.f64(Q_bt, (a, b))
    out = cv.empty((n, a, b))
    _lib.check(_lib.lib().pocean_upwind_transport_f64(qe.data_ptr(), qw.data_ptr(), u.data_ptr(), Ld.data_ptr(),
                                                      Qd.data_ptr(), n, a, b, out.data_ptr(), cv.stream()),
               "upwind_transport_x")
    return cv.out(out)


def freshwater_volumes(V, dV, floor):
    """(V_new, n_limited): dV added to the top layer, a removal beyond the floor taken from the layers below
    (core/components/freshwater.py:31-58).  ``floor`` a scalar or (ny, nx)."""
    n, ny, nx = shape_of(V)
    scalar = np.ndim(floor) == 0 and not isinstance(floor, torch.Tensor)
    cv = Converter(V, dV, *(() if scalar else (floor,)))
    Vd, dd = cv.f64(V), cv.f64(dV, (ny, nx))
    fd = None if scalar else cv.f64(floor, (ny, nx))
    out = cv.empty((n, ny, nx))
    nl = torch.zeros(1, dtype=torch.int32, device=cv.device)
    _lib.check(_lib.lib().pocean_freshwater_volumes_f64(Vd.data_ptr(), dd.data_ptr(),
                                                        None if fd is None else fd.data_ptr(),
                                                        float(floor) if scalar else 0.0, n, ny, nx, out.data_ptr(),
                                                        nl.data_ptr(), cv.stream()), "freshwater_volumes")
    return cv.out(out), int(nl.item())


@dataclass
class LayerFluxes:
    """The record ``ALELayerTransport`` returns (layer_transport.py:30-41)."""
    Qx: object
    Qy: object
    Fz: object
    V0: object
    V1: object
    ok: object
    h_dagger: object = None
    n_limited: int = 0
    V_fw: object = None
    h_fw: object = None


def _swap(t: torch.Tensor) -> torch.Tensor:
    return t.transpose(-1, -2).contiguous()


PPM_HALO = 4                           # core/components/layer_transport.py:122 (the PPM edges' stencil)


def _face_kind(kind: str) -> tuple[int, int]:
    """(face_y, face_x) of a staggering: 'c' cells, 'u' u-faces, 'v' v-faces."""
    return (1 if kind == "v" else 0), (1 if kind == "u" else 0)


def periodic_pad(t: torch.Tensor, kind: str, px: bool, py: bool, halo: int) -> torch.Tensor:
    """``t`` (leading axes, then y, x) with ``halo`` wrapped positions on each side of the periodic axes, as
    ``Periodic.pad`` (core/model/periodic.py:72-85): faces wrap on the unique faces 0 .. n-1."""
    fy, fx = _face_kind(kind)
    ny, nx = t.shape[-2] - fy, t.shape[-1] - fx
    lead = int(np.prod(t.shape[:-2])) if t.dim() > 2 else 1
    shape = tuple(t.shape[:-2]) + (ny + fy + (2 * halo if py else 0), nx + fx + (2 * halo if px else 0))
    out = torch.empty(shape, dtype=t.dtype, device=t.device)
    fn = _lib.lib().pocean_periodic_pad_u8 if t.dtype == torch.uint8 else _lib.lib().pocean_periodic_pad_f64
    src = t.contiguous()                      # held until the launch is enqueued
    _lib.check(fn(src.data_ptr(), lead, ny, nx, fy, fx, int(py), int(px), halo, out.data_ptr(),
                  torch.cuda.current_stream(t.device).cuda_stream), "periodic_pad")
    return out


def periodic_crop(t: torch.Tensor, kind: str, px: bool, py: bool, halo: int) -> torch.Tensor:
    """The interior positions of a padded ``t`` (``Periodic.crop``, core/model/periodic.py:87-93)."""
    fy, fx = _face_kind(kind)
    ny = t.shape[-2] - fy - (2 * halo if py else 0)
    nx = t.shape[-1] - fx - (2 * halo if px else 0)
    lead = int(np.prod(t.shape[:-2])) if t.dim() > 2 else 1
    out = torch.empty(tuple(t.shape[:-2]) + (ny + fy, nx + fx), dtype=t.dtype, device=t.device)
    src = t.contiguous()                      # held until the launch is enqueued
    _lib.check(_lib.lib().pocean_periodic_crop_f64(src.data_ptr(), lead, ny, nx, fy, fx, int(py), int(px), halo,
                                                   out.data_ptr(), torch.cuda.current_stream(t.device).cuda_stream),
               "periodic_crop")
    return out


def open_face_transports(Qx: torch.Tensor, Qy: torch.Tensor, h, un, vn, u_new, v_new, open_, open_Du, open_Dv,
                         open_Qu, open_Qv, Lu, Lv, theta_bc: float) -> None:
    """In place on device tensors: the layer fluxes through the open faces where the open face depth is positive,
    the Flather flux split with the interior cells' thickness fractions (core/components/open_boundary.py:334-352,
    core/vertical/ale.py:841-861).  h (N, ny, nx); un, u_new, Qx (N, ny, nx+1); vn, v_new, Qy (N, ny+1, nx);
    open_D*, open_Q*, L* face arrays of one layer."""
    n, ny, nx = h.shape
    L_ = _lib.lib()
    st = torch.cuda.current_stream(h.device).cuda_stream
    hs, us_x, us_y = (ny * nx, nx), (ny * (nx + 1), nx + 1), ((ny + 1) * nx, nx)
    for edge in open_:
        if edge == "west" or edge == "east":
            c = 0 if edge == "west" else -1
            ch, cu = (0 if c == 0 else nx - 1), (0 if c == 0 else nx)
            rc = L_.pocean_open_face_transport_f64(
                h.data_ptr() + 8 * ch, hs[0], hs[1], u_new.data_ptr() + 8 * cu, un.data_ptr() + 8 * cu, us_x[0],
                us_x[1], open_Qu.data_ptr() + 8 * cu, Lu.data_ptr() + 8 * cu, open_Du.data_ptr() + 8 * cu, nx + 1, n,
                ny, float(theta_bc), Qx.data_ptr() + 8 * cu, us_x[0], us_x[1], st)
        elif edge == "south" or edge == "north":
            r = 0 if edge == "south" else 1
            rh, rv = (0 if r == 0 else (ny - 1) * nx), (0 if r == 0 else ny * nx)
            rc = L_.pocean_open_face_transport_f64(
                h.data_ptr() + 8 * rh, hs[0], 1, v_new.data_ptr() + 8 * rv, vn.data_ptr() + 8 * rv, us_y[0], 1,
                open_Qv.data_ptr() + 8 * rv, Lv.data_ptr() + 8 * rv, open_Dv.data_ptr() + 8 * rv, 1, n, nx,
                float(theta_bc), Qy.data_ptr() + 8 * rv, us_y[0], 1, st)
        else:
            raise ValueError(f"unknown open edge {edge!r}")
        _lib.check(rc, "open_face_transport")


class ALELayerTransport:
    """The Lagrangian layer-transport step of the ALE core on B200, with the reference component's constructor and
    call (layer_transport.py:98-160): transport velocities, the PPM or donor-cell layer fluxes (v-faces on swapped
    axes; on periodic axes the PPM flux runs on inputs padded by four wrapped positions and is cropped, as the
    reference does), the open faces, the outflow limiter, h-dagger, the layer volumes h A, ``ok`` and, with
    ``fluxes.fw``, the freshwater thickness and volumes.  Open faces (``open_`` not empty)     are written in place on the device from ``fluxes.open_Du`` / ``open_Dv`` / ``open_Qu`` / ``open_Qv`` (the open
    boundary component's Flather split, core/components/open_boundary.py:334-352; ``theta_bc`` from ``ob`` when it
    has one, else the call's).  The ALE layer volumes are h A (sigma_baroclinic.py:1812-1815): the
    ``layer_volumes`` callable is kept for the interface and not called.  Arrays are NumPy (results come back as
    NumPy) or CUDA tensors (everything stays in HBM)."""

    def __init__(self, *, fs, H, area, dt: float, thickness_flux: str, vi_geom: dict, layer_volumes=None,
                 ob=None) -> None:
        if thickness_flux not in ("ppm", "upwind"):
            raise ValueError(f"thickness_flux {thickness_flux!r}: use 'ppm' or 'upwind'")
        self.fs, self.H, self.area, self.dt, self.thickness_flux = fs, H, area, float(dt), thickness_flux
        self.vi_geom, self.layer_volumes, self.ob = vi_geom, layer_volumes, ob
        self.per = None

    def __call__(self, st, eta_new, u_new, v_new, fluxes, theta_bc: float, open_, wu, wv, qe, qw, qn,
                 qs) -> LayerFluxes:
        px, py = bool(getattr(self.per, "x", False)), bool(getattr(self.per, "y", False))
        fw = getattr(fluxes, "fw", None)
        n, ny, nx = shape_of(st.h)
        fs, dt, L = self.fs, self.dt, _lib.lib()
        cv = Converter(st.h, st.u, st.v, u_new, v_new, wu, wv, qe, qw, qn, qs, self.area, *(() if fw is None else (fw,)))
        h = cv.f64(st.h)
        act = cv.u8(fs.active, (ny, nx))
        area = cv.f64(self.area, (ny, nx))
        tb = theta_bc
        utx, Qbx = transport_velocity(cv.f64(u_new), cv.f64(st.u), cv.u8(fluxes.wet_u, (ny, nx + 1)), cv.f64(wu),
                                      cv.f64(fs.Lu, (ny, nx + 1)), cv.f64(fluxes.Du, (ny, nx + 1)), fs.theta, tb)
        uty, Qby = transport_velocity(cv.f64(v_new), cv.f64(st.v), cv.u8(fluxes.wet_v, (ny + 1, nx)), cv.f64(wv),
                                      cv.f64(fs.Lv, (ny + 1, nx)), cv.f64(fluxes.Dv, (ny + 1, nx)), fs.theta, tb)
        Lv_t, Qby_t, uty_t = _swap(cv.f64(fs.Lv, (ny + 1, nx))), _swap(Qby), _swap(uty)
        qn_d, qs_d = cv.f64(qn), cv.f64(qs)
        if self.thickness_flux == "ppm":
            Lu_d, dx_d, dy_d = cv.f64(fs.Lu, (ny, nx + 1)), cv.f64(self.vi_geom["dx_t"], (ny, nx)), cv.f64(
                self.vi_geom["dy_t"], (ny, nx))
            Lv_d, qe_d, qw_d = cv.f64(fs.Lv, (ny + 1, nx)), cv.f64(qe), cv.f64(qw)
            if px or py:                               # pad-crop with the PPM halo (layer_transport.py:121-128)
                pad = lambda t, k: periodic_pad(t, k, px, py, PPM_HALO)                   # noqa: E731
                hp, uxp, uyp, Lup, Lvp = pad(h, "c"), pad(utx, "u"), pad(uty, "v"), pad(Lu_d, "u"), pad(Lv_d, "v")
                bxp, byp, ep, wp = pad(Qbx, "u"), pad(Qby, "v"), pad(qe_d, "u"), pad(qw_d, "u")
                np_, sp = pad(_swap(qn_d), "v"), pad(_swap(qs_d), "v")
                ap, dxp, dyp = pad(act, "c"), pad(dx_d, "c"), pad(dy_d, "c")
                Qx = periodic_crop(ppm_transport_x(hp, uxp, Lup, bxp, ep, wp, ap, dt, dxp), "u", px, py, PPM_HALO)
                Qy = periodic_crop(_swap(ppm_transport_x(_swap(hp), _swap(uyp), _swap(Lvp), _swap(byp), _swap(np_),
                                                         _swap(sp), _swap(ap), dt, _swap(dyp))), "v", px, py,
                                   PPM_HALO)
            else:
                Qx = ppm_transport_x(h, utx, Lu_d, Qbx, qe_d, qw_d, act, dt, dx_d)
                Qy = _swap(ppm_transport_x(_swap(h), uty_t, Lv_t, Qby_t, qn_d, qs_d, _swap(act), dt, _swap(dy_d)))
        else:
            Qx = upwind_transport_x(cv.f64(qe), cv.f64(qw), utx, cv.f64(fs.Lu, (ny, nx + 1)), Qbx)
            Qy = _swap(upwind_transport_x(qn_d, qs_d, uty_t, Lv_t, Qby_t))
        if open_:                                      # old velocity unmasked: the wet flag is False at edges
            if self.ob is None:
                raise ValueError("open edges need the open-boundary component (ob) of the reference's interface")
            tbc = getattr(self.ob, "theta_bc", None)
            tb = fs.theta if tbc is None else tbc          # ale.py:859
            Qx, Qy = Qx.clone(), Qy.clone()
            open_face_transports(Qx, Qy, h, cv.f64(st.u), cv.f64(st.v), cv.f64(u_new), cv.f64(v_new), tuple(open_),
                                 cv.f64(fluxes.open_Du, (ny, nx + 1)), cv.f64(fluxes.open_Dv, (ny + 1, nx)),
                                 cv.f64(fluxes.open_Qu, (ny, nx + 1)), cv.f64(fluxes.open_Qv, (ny + 1, nx)),
                                 cv.f64(fs.Lu, (ny, nx + 1)), cv.f64(fs.Lv, (ny + 1, nx)), tb)
        Qx, Qy, n_lim = limit_outflow(h, Qx, Qy, area, dt, act, periodic=(px, py))
        divh = cv.empty((n, ny, nx))
        _lib.check(L.pocean_flux_divergence_f64(Qx.data_ptr(), Qy.data_ptr(), n, ny, nx, divh.data_ptr(),
                                                cv.stream()), "flux_divergence")
        h_lag = lagrangian_thickness(h, divh, dt, area)
        V0, V1 = cv.empty((n, ny, nx)), cv.empty((n, ny, nx))
        ok = torch.empty((n, ny, nx), dtype=torch.uint8, device=cv.device)
        for hh, V, o in ((h, V0, None), (h_lag, V1, ok)):
            _lib.check(L.pocean_layer_volumes_f64(hh.data_ptr(), area.data_ptr(), act.data_ptr(), n, ny, nx,
                                                  V.data_ptr(), None if o is None else o.data_ptr(), cv.stream()),
                       "layer_volumes")
        Fz = torch.zeros((n + 1, ny, nx), dtype=torch.float64, device=cv.device)
        h_fw = V_fw = None
        if fw is not None:
            h_fw, _ = freshwater_volumes(h_lag, cv.f64(fw, (ny, nx)) * dt, DZ_FLOOR)
            V_fw = cv.empty((n, ny, nx))
            _lib.check(L.pocean_layer_volumes_f64(h_fw.data_ptr(), area.data_ptr(), act.data_ptr(), n, ny, nx,
                                                  V_fw.data_ptr(), None, cv.stream()), "layer_volumes")
        okb = ok.bool()
        return LayerFluxes(cv.out(Qx), cv.out(Qy), cv.out(Fz), cv.out(V0), cv.out(V1),
                           okb.cpu().numpy() if cv.numpy_out else okb, cv.out(h_lag), int(n_lim),
                           None if V_fw is None else cv.out(V_fw), None if h_fw is None else cv.out(h_fw))
