"""
``TracerAdvection`` with the reference's interface (core/components/tracers.py:50-375), computed on the GPU.

Drop-in use: construct it like the reference's component (``scheme``, ``time``, ``dt``, ``ob``), set ``per`` to the
model's periodic axes, and call ``advect_fct`` (ALE step with Zalesak FCT) or ``advect`` (SSP-RK3 without limiter).
Arrays are NumPy (copied to the GPU and back) or CUDA torch tensors (used in place, results stay on the device).
Inputs are never modified; results are new arrays, as in the reference.

``advect`` also covers what the reference runs through its NumPy RHS path (tracers.py:110-151, 303-330): the
``upwind3`` / ``upwind1`` face schemes (any other non-WENO5 name is upwind-3, as there) and the ``'pc'``
predictor-corrector time stepping (a centred half step, then a full step with the scheme's faces), in FP64 and
bit for bit.  ``advect_fct`` uses WENO5-Z for ``scheme='weno5'`` and WENO5-JS otherwise, exactly as the reference's
fused path does (tracers.py:176).  The single-stage helpers ``faces_h``, ``upwind_faces_h``, ``flux_x``, ``rhs``,
``rhs_numpy`` and the NumPy-named step methods, which ``SigmaBaroclinic`` delegates to, are here too.

Not provided: the per-axis face-value functions ``faces`` and ``open_faces`` (tracers.py:110-137), which the
reference calls only from inside ``rhs_numpy`` and ``flux_x`` (and from two ``SigmaBaroclinic`` delegators that
nothing calls); their results reach the caller through ``rhs``, ``rhs_numpy`` and ``flux_x``.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import _pipeline as _pl
from ._device import Converter, shape_of
from .periodic import NONE


class OpenEdges:
    """Minimal open-boundary descriptor: ``open`` is a tuple of edge names ('west', 'east', 'south', 'north')."""

    def __init__(self, open_=()) -> None:
        self.open = tuple(open_)


class TracerAdvection:
    """SSP-RK3 WENO5 tracer advection (with Zalesak FCT in ``advect_fct``) on frozen transports, on B200."""

    name = "tracer_advection"
    role = None                     # the model's Role enum; a drop-in copies the replaced component's
    reads = ("T", "tr", "Qx", "Qy", "Fz")
    writes = ("T", "tr")
    per = NONE

    def __init__(self, *, scheme: str, time: str, dt: float, ob=None, precision: str = "f64") -> None:
        """``precision``: "f64" (the reference's arithmetic, bit for bit) or "mixed" (WENO5 weights and face values
        in FP32, everything else in FP64; ``advect_fct`` only)."""
        if precision not in ("f64", "mixed"):
            raise ValueError(f"precision must be 'f64' or 'mixed', got {precision!r}")
        self.tracer_scheme, self.tracer_time, self.dt = scheme, time, dt
        self.precision = precision
        self.ob = ob if ob is not None else OpenEdges()
        self.record_open_flux = False
        self.last_open_flux: np.ndarray | None = None

    # ------------------------------------------------------------------------------------------------ component
    def check(self, ctx) -> list:
        """The model builder's consistency check (tracers.py:104-105): nothing to report."""
        return []

    def state_fields(self) -> dict:
        """Restart state (tracers.py:107-108): none — the component keeps nothing from step to step."""
        return {}

    def _flags(self) -> int:
        opn = tuple(getattr(self.ob, "open", ()) or ())
        f = 0
        f |= _lib.OPEN_W if "west" in opn else 0
        f |= _lib.OPEN_E if "east" in opn else 0
        f |= _lib.OPEN_S if "south" in opn else 0
        f |= _lib.OPEN_N if "north" in opn else 0
        per = self.per
        f |= _lib.PERIODIC_X if getattr(per, "x", False) else 0
        f |= _lib.PERIODIC_Y if getattr(per, "y", False) else 0
        f |= 0 if self.tracer_scheme == "weno5" else _lib.WENO_JS
        return f

    @staticmethod
    def _shapes(C, Qx, Qy):
        shp = shape_of(C)
        if len(shp) != 4:
            raise ValueError(f"tracer stack must be (ntr, N, ny, nx), got {shp}")
        nt, n, ny, nx = shp
        if shape_of(Qx) != (n, ny, nx + 1) or shape_of(Qy) != (n, ny + 1, nx):
            raise ValueError(f"transports {shape_of(Qx)}/{shape_of(Qy)} do not match the stack {shp}")
        return nt, n, ny, nx

    # ------------------------------------------------------------------------------------------------ FCT
    def advect_fct(self, C, V0, V1, Qx, Qy, ok, unlimited: bool = False, inflow=None, flux_face_i: int | None = None):
        """
        SSP-RK3 WENO5 step of the stack C (ntr, N, ny, nx) with Zalesak FCT (tracers.py:208-254).
        ``unlimited``: the plain RK3 result (C = 1).  ``inflow``: exterior values used on open edges during
        inflow (None: the stages' own values).  ``flux_face_i``: also return the step's effective flux through
        u-face column i, (ntr, N, ny).  With ``record_open_flux`` the net inflow rate per stack member through the
        open edges is left in ``last_open_flux`` (limited step only).
        """
        nt, n, ny, nx = self._shapes(C, Qx, Qy)
        if shape_of(V0) != (n, ny, nx) or shape_of(V1) != (n, ny, nx):
            raise ValueError(f"volume shape {shape_of(V0)}/{shape_of(V1)} vs tracer layers {(n, ny, nx)}")
        if (nt >= 2 and (inflow is None or inflow is C) and _pl.pinned(C, V0, V1, Qx, Qy, ok)
                and all(a.dtype == torch.float64 for a in (C, V0, V1, Qx, Qy))
                and ok.dtype in (torch.bool, torch.uint8) and tuple(ok.shape) in ((n, ny, nx), (ny, nx))
                and 8 * nt * n * ny * nx >= _pl.MIN_BYTES):
            if not unlimited and flux_face_i is None and not self.record_open_flux:
                return self._advect_fct_layered(C, V0, V1, Qx, Qy, ok)
            return self._advect_fct_pipelined(C, V0, V1, Qx, Qy, ok, unlimited, flux_face_i)
        cv = Converter(C, V0, V1, Qx, Qy, ok, inflow)
        # tracers.py:230-231: an inflow stack that *is* C means "no exterior values" (each stage its own)
        own = inflow is None or (inflow is C and (isinstance(C, torch.Tensor) or
                                                  (isinstance(C, np.ndarray) and C.dtype == np.float64 and
                                                   C.flags.c_contiguous)))
        Cd = cv.f64(C)
        V0d, V1d, Qxd, Qyd = cv.f64(V0), cv.f64(V1), cv.f64(Qx), cv.f64(Qy)
        okd = cv.u8(ok, (n, ny, nx))
        infl = None if own else cv.f64(inflow, (nt, n, ny, nx))
        out = cv.empty((nt, n, ny, nx))
        flags = self._flags() | (_lib.FCT_UNLIMITED if unlimited else 0)
        fx = None
        if flux_face_i is not None:
            fi = int(flux_face_i)
            if fi < 0:
                fi += nx + 1
            fx = cv.empty((nt, n, ny))
        else:
            fi = 0
        record = self.record_open_flux and not unlimited
        of = cv.empty((nt,)) if record else None
        L = _lib.lib()
        nbytes = L.pocean_advect_fct_workspace_bytes(nt, n, ny, nx)
        ws = cv.workspace(nbytes)
        fn = L.pocean_advect_fct_mixed if self.precision == "mixed" else L.pocean_advect_fct_f64
        rc = fn(Cd.data_ptr(), V0d.data_ptr(), V1d.data_ptr(), Qxd.data_ptr(), Qyd.data_ptr(),
                                     okd.data_ptr(), None if infl is None else infl.data_ptr(), nt, n, ny, nx, flags,
                                     float(self.dt), out.data_ptr(), fi, None if fx is None else fx.data_ptr(),
                                     None if of is None else of.data_ptr(), ws.data_ptr(), nbytes, cv.stream())
        _lib.check(rc, "advect_fct")
        if record:
            self.last_open_flux = of.cpu().numpy()
        if flux_face_i is None:
            return cv.out(out)
        return cv.out(out), cv.out(fx)

    def _advect_fct_layered(self, C, V0, V1, Qx, Qy, ok, download: bool = True, blocks=None):
        """advect_fct of pinned host tensors in blocks of layers: block b's tracers and geometry go to the device on
        the copy-in stream while the stage passes of block b-1 and the limiter passes of block b-2 run on the
        compute stream (``pocean_advect_fct_layers``: a block's limiter reads the layers either side of it) and
        finished blocks come back on the copy-out stream.  ``download=False``: the advected stack stays on the
        device and is returned as a tensor whose producing kernels are ordered on the compute stream
        (``_pipeline.streams``), for a caller that goes on with it there.  ``blocks``: (full blocks, tail), default
        ``_pipeline.FCT_BLOCKS``."""
        nt, n, ny, nx = C.shape
        dev = _pl.device_now()
        s_in, s_cmp, s_out = _pl.streams(dev)
        s_in.wait_stream(torch.cuda.current_stream(dev))
        L = _lib.lib()
        mixed = int(self.precision == "mixed")
        flags = self._flags()
        f64 = dict(dtype=torch.float64, device=dev)
        with torch.cuda.stream(s_in):
            Cd = torch.empty((nt, n, ny, nx), **f64)
            V0d, V1d = torch.empty((n, ny, nx), **f64), torch.empty((n, ny, nx), **f64)
            Qxd, Qyd = torch.empty((n, ny, nx + 1), **f64), torch.empty((n, ny + 1, nx), **f64)
            if ok.dim() == 2:                       # per column: uploaded once, broadcast over the layers
                okd = ok.to(dev, non_blocking=True)
                okd = (okd if okd.dtype == torch.uint8 else (okd != 0).to(torch.uint8)).expand((n, ny, nx)).contiguous()
            else:
                okd = torch.empty((n, ny, nx), dtype=torch.uint8, device=dev)
        nbytes = L.pocean_advect_fct_workspace_bytes(nt, n, ny, nx)
        with torch.cuda.stream(s_cmp):
            outd = torch.empty((nt, n, ny, nx), **f64)
            ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
        out = torch.empty((nt, n, ny, nx), dtype=torch.float64, pin_memory=True) if download else None
        for t in (Cd, V0d, V1d, Qxd, Qyd, okd):     # made on the copy-in stream, read on the compute stream
            t.record_stream(s_cmp)
        pl, px, py = ny * nx, ny * (nx + 1), (ny + 1) * nx

        def layers(k0, k1, part):
            _lib.check(L.pocean_advect_fct_layers(mixed, Cd.data_ptr(), V0d.data_ptr(), V1d.data_ptr(),
                                                  Qxd.data_ptr(), Qyd.data_ptr(), okd.data_ptr(), None, nt, n, ny,
                                                  nx, flags, float(self.dt), outd.data_ptr(), ws.data_ptr(), nbytes,
                                                  k0, k1, part, s_cmp.cuda_stream), "advect_fct")

        def fetch(k0, k1):
            if not download:
                return
            ev = torch.cuda.Event()
            ev.record(s_cmp)
            s_out.wait_event(ev)
            _pl.copy2d(out.data_ptr() + 8 * k0 * pl, 8 * n * pl, outd.data_ptr() + 8 * k0 * pl, 8 * n * pl,
                       8 * (k1 - k0) * pl, nt, s_out)

        blocks = _pl.row_blocks(n, *(blocks or _pl.FCT_BLOCKS))
        for b, (k0, k1) in enumerate(blocks):
            nl = k1 - k0
            _pl.copy2d(Cd.data_ptr() + 8 * k0 * pl, 8 * n * pl, C.data_ptr() + 8 * k0 * pl, 8 * n * pl, 8 * nl * pl,
                       nt, s_in)
            for dst, src, per in ((V0d, V0, pl), (V1d, V1, pl), (Qxd, Qx, px), (Qyd, Qy, py)):
                _pl.copy2d(dst.data_ptr() + 8 * k0 * per, 8 * nl * per, src.data_ptr() + 8 * k0 * per, 8 * nl * per,
                           8 * nl * per, 1, s_in)
            if ok.dim() == 3:                       # bool or uint8 bytes, one per cell
                _pl.copy2d(okd.data_ptr() + k0 * pl, nl * pl, ok.data_ptr() + k0 * pl, nl * pl, nl * pl, 1, s_in)
            ev = torch.cuda.Event()
            ev.record(s_in)
            s_cmp.wait_event(ev)
            layers(k0, k1, 0)
            if b > 0:
                layers(*blocks[b - 1], 1)
                fetch(*blocks[b - 1])
        layers(*blocks[-1], 1)
        fetch(*blocks[-1])
        if not download:
            return outd
        s_out.synchronize()
        return out

    def _advect_fct_pipelined(self, C, V0, V1, Qx, Qy, ok, unlimited: bool, flux_face_i):
        """advect_fct of pinned host tensors, one tracer of the stack at a time: the geometry goes to the device
        first, then tracer t's field on the copy-in stream while tracer t-1 steps on the compute stream and tracer
        t-2's result comes back on the copy-out stream (each tracer's step is independent of the others')."""
        nt, n, ny, nx = C.shape
        dev = _pl.device_now()
        s_in, s_cmp, s_out = _pl.streams(dev)
        s_in.wait_stream(torch.cuda.current_stream(dev))
        L = _lib.lib()
        fn = L.pocean_advect_fct_mixed if self.precision == "mixed" else L.pocean_advect_fct_f64
        flags = self._flags() | (_lib.FCT_UNLIMITED if unlimited else 0)
        fi = 0
        if flux_face_i is not None:
            fi = int(flux_face_i)
            if fi < 0:
                fi += nx + 1
        record = self.record_open_flux and not unlimited
        with torch.cuda.stream(s_in):
            V0d, V1d, Qxd, Qyd = (a.to(dev, non_blocking=True) for a in (V0, V1, Qx, Qy))
            okd = ok.to(dev, non_blocking=True)
            okd = (okd if okd.dtype == torch.uint8 else (okd != 0).to(torch.uint8)).expand((n, ny, nx)).contiguous()
        out = torch.empty((nt, n, ny, nx), dtype=torch.float64, pin_memory=True)
        fx = torch.empty((nt, n, ny), dtype=torch.float64, pin_memory=True) if flux_face_i is not None else None
        nbytes = L.pocean_advect_fct_workspace_bytes(1, n, ny, nx)
        with torch.cuda.stream(s_cmp):
            ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
            of = torch.empty((nt,), dtype=torch.float64, device=dev) if record else None
        keep = [V0d, V1d, Qxd, Qyd, okd]
        for t in range(nt):
            with torch.cuda.stream(s_in):
                ct = C[t].to(dev, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s_in)
            s_cmp.wait_event(ev)
            with torch.cuda.stream(s_cmp):
                ot = torch.empty((1, n, ny, nx), dtype=torch.float64, device=dev)
                ft = torch.empty((1, n, ny), dtype=torch.float64, device=dev) if fx is not None else None
            rc = fn(ct.data_ptr(), V0d.data_ptr(), V1d.data_ptr(), Qxd.data_ptr(), Qyd.data_ptr(), okd.data_ptr(),
                    None, 1, n, ny, nx, flags, float(self.dt), ot.data_ptr(), fi,
                    None if ft is None else ft.data_ptr(), None if of is None else of.data_ptr() + 8 * t,
                    ws.data_ptr(), nbytes, s_cmp.cuda_stream)
            _lib.check(rc, "advect_fct")
            ev = torch.cuda.Event()
            ev.record(s_cmp)
            s_out.wait_event(ev)
            with torch.cuda.stream(s_out):
                out[t].copy_(ot[0], non_blocking=True)
                if ft is not None:
                    fx[t].copy_(ft[0], non_blocking=True)
            keep += [ct, ot, ft]
        s_out.synchronize()
        if record:
            self.last_open_flux = of.cpu().numpy()
        if flux_face_i is None:
            return out
        return out, fx

    # ------------------------------------------------------------------------------------------------ helpers
    # The single-stage helpers (tracers.py:139-206), as the reference runs them: on the arrays given, with no
    # periodic wrap (a periodic caller pads first), the open edges of ``ob`` and their exterior values.
    def _helper_flags(self, scheme_faces: bool) -> int:
        f = self._flags() & ~(_lib.PERIODIC_X | _lib.PERIODIC_Y)
        if scheme_faces and not self.tracer_scheme.startswith("weno5"):
            f |= _lib.FACES_UP1 if self.tracer_scheme == "upwind1" else _lib.FACES_UP3
        return f

    def _faces(self, c, Qx, Qy, ok, ext, kind: int, scheme_faces: bool):
        nt, n, ny, nx = self._shapes(c, Qx, Qy)
        cv = Converter(c, Qx, Qy, ok, ext)
        # every device buffer is held by a name until the launch is enqueued (a temporary's memory could be handed
        # to the next upload before the kernel reads it)
        cd, Qxd, Qyd = cv.f64(c), cv.f64(Qx), cv.f64(Qy)
        ed = None if ext is None else cv.f64(ext, (nt, n, ny, nx))
        fx, fy = cv.empty((nt, n, ny, nx + 1)), cv.empty((nt, n, ny + 1, nx))
        okd = cv.u8(ok, (n, ny, nx)) if ok is not None else torch.ones((n, ny, nx), dtype=torch.uint8,
                                                                        device=cv.device)
        rc = _lib.lib().pocean_advect_faces_f64(cd.data_ptr(), Qxd.data_ptr(), Qyd.data_ptr(), okd.data_ptr(),
                                                None if ed is None else ed.data_ptr(), nt, n, ny, nx,
                                                self._helper_flags(scheme_faces), kind, fx.data_ptr(), fy.data_ptr(),
                                                cv.stream())
        _lib.check(rc, "faces")
        return cv.out(fx), cv.out(fy)

    def faces_h(self, c, Qx, Qy, ok, ext=None, inflow=None):
        """WENO5 horizontal face fluxes (fx, fy) of the stack, the terms _advect_div differences
        (tracers.py:166-176): WENO5-Z for scheme 'weno5', WENO5-JS otherwise; ``ext``: the exterior values on
        inflow, else ``inflow``, else the stack's own."""
        return self._faces(c, Qx, Qy, ok, inflow if ext is None else ext, _lib.HELPER_SCHEME, False)

    def upwind_faces_h(self, c, Qx, Qy, inflow=None):
        """Donor-cell face fluxes Q c_up (the FCT low-order flux; tracers.py:178-193)."""
        return self._faces(c, Qx, Qy, None, inflow, _lib.HELPER_DONOR, False)

    def flux_x(self, c, Qx, Qy, ok, centred: bool = False, inflow=None):
        """x-face fluxes (ntr, N, ny, nx+1) of the faces ``rhs`` differences (tracers.py:195-206)."""
        if not centred and self.tracer_scheme.startswith("weno5"):
            return self.faces_h(c, Qx, Qy, ok, inflow=inflow)[0]
        return self._faces(c, Qx, Qy, ok, inflow, _lib.HELPER_CENTRED if centred else _lib.HELPER_SCHEME, True)[0]

    def rhs(self, c, Qx, Qy, Fz, ok, centred: bool = False, inflow=None):
        """Advection RHS -div(Q c) of the stack (tracers.py:153-164): the fused WENO5 RHS, or the NumPy path's
        faces for the upwind schemes and for ``centred``."""
        nt, n, ny, nx = self._shapes(c, Qx, Qy)
        if Fz is not None and shape_of(Fz) != (n + 1, ny, nx):
            raise ValueError(f"Fz shape {shape_of(Fz)} vs {(n + 1, ny, nx)}")
        cv = Converter(c, Qx, Qy, Fz, ok, inflow)
        ed = None if inflow is None else cv.f64(inflow, (nt, n, ny, nx))
        out = cv.empty((nt, n, ny, nx))
        L = _lib.lib()
        nbytes = L.pocean_advect_rhs_workspace_bytes(nt, n, ny, nx)
        ws = cv.workspace(nbytes)
        cd, Qxd, Qyd, okd = cv.f64(c), cv.f64(Qx), cv.f64(Qy), cv.u8(ok, (n, ny, nx))
        Fzd = None if Fz is None else cv.f64(Fz)
        rc = L.pocean_advect_rhs_f64(cd.data_ptr(), Qxd.data_ptr(), Qyd.data_ptr(),
                                     None if Fzd is None else Fzd.data_ptr(), okd.data_ptr(),
                                     None if ed is None else ed.data_ptr(), nt, n, ny, nx, self._helper_flags(True),
                                     int(bool(centred)), out.data_ptr(), ws.data_ptr(), nbytes, cv.stream())
        _lib.check(rc, "rhs")
        return cv.out(out)

    def rhs_numpy(self, c, Qx, Qy, Fz, ok, centred: bool = False, inflow=None):
        """The reference's NumPy RHS (tracers.py:139-151); its values are those of ``rhs`` (the reference's fused
        and NumPy RHS agree), so this is ``rhs``."""
        return self.rhs(c, Qx, Qy, Fz, ok, centred, inflow)

    def advect_numpy(self, C, V0, V1, Qx, Qy, Fz, ok, inflow=None, flux_face_i: int | None = None):
        """The reference's NumPy form of ``advect`` (tracers.py:303-340), the same arithmetic as ``advect``."""
        return self.advect(C, V0, V1, Qx, Qy, Fz, ok, inflow=inflow, flux_face_i=flux_face_i)

    def advect_fct_numpy(self, C, V0, V1, Qx, Qy, ok, unlimited: bool = False, inflow=None,
                         flux_face_i: int | None = None):
        """The reference's NumPy form of ``advect_fct`` (tracers.py:256-301), which its fused path equals bit for
        bit: ``advect_fct``."""
        return self.advect_fct(C, V0, V1, Qx, Qy, ok, unlimited=unlimited, inflow=inflow, flux_face_i=flux_face_i)

    # ------------------------------------------------------------------------------------------------ RK3
    def advect(self, C, V0, V1, Qx, Qy, Fz, ok, inflow=None, flux_face_i: int | None = None):
        """
        SSP-RK3 flux-form advection of the stack C with frozen Qx, Qy, Fz (N+1, ny, nx); layer volumes linear from
        V0 to V1 (tracers.py:342-375); with ``time='pc'`` the predictor-corrector step (tracers.py:324-330).
        ``flux_face_i``: also return (F(c0) + F(c1))/6 + 2F(c2)/3 through u-face column i ('pc': the corrector's
        flux F(c^{n+1/2})).
        """
        if self.precision != "f64":
            raise NotImplementedError("advect (no limiter) is available in FP64 only")
        nt, n, ny, nx = self._shapes(C, Qx, Qy)
        if shape_of(V0) != (n, ny, nx) or shape_of(V1) != (n, ny, nx):
            raise ValueError(f"_advect: volume shape {shape_of(V0)}/{shape_of(V1)} vs tracer layers {(n, ny, nx)}")
        if Fz is not None and shape_of(Fz) != (n + 1, ny, nx):
            raise ValueError(f"Fz shape {shape_of(Fz)} vs {(n + 1, ny, nx)}")
        cv = Converter(C, V0, V1, Qx, Qy, Fz, ok, inflow)
        Cd = cv.f64(C)
        V0d, V1d, Qxd, Qyd = cv.f64(V0), cv.f64(V1), cv.f64(Qx), cv.f64(Qy)
        Fzd = None if Fz is None else cv.f64(Fz)
        okd = cv.u8(ok, (n, ny, nx))
        infl = None if inflow is None else cv.f64(inflow, (nt, n, ny, nx))
        out = cv.empty((nt, n, ny, nx))
        fx = None
        fi = 0
        if flux_face_i is not None:
            fi = int(flux_face_i)
            if fi < 0:
                fi += nx + 1
            fx = cv.empty((nt, n, ny))
        L = _lib.lib()
        nbytes = L.pocean_advect_rk3_workspace_bytes(nt, n, ny, nx)
        ws = cv.workspace(nbytes)
        # tracers.py:110-115, 153-156: non-WENO5 schemes take the NumPy path's upwind faces (order 1 for
        # "upwind1", else 3); 'pc' (tracers.py:355-356) the predictor-corrector step
        flags = self._flags()
        if not self.tracer_scheme.startswith("weno5"):
            flags |= _lib.FACES_UP1 if self.tracer_scheme == "upwind1" else _lib.FACES_UP3
        if self.tracer_time == "pc":
            flags |= _lib.TIME_PC
        rc = L.pocean_advect_rk3_f64(Cd.data_ptr(), V0d.data_ptr(), V1d.data_ptr(), Qxd.data_ptr(), Qyd.data_ptr(),
                                     None if Fzd is None else Fzd.data_ptr(), okd.data_ptr(),
                                     None if infl is None else infl.data_ptr(), nt, n, ny, nx, flags,
                                     float(self.dt), out.data_ptr(), fi, None if fx is None else fx.data_ptr(),
                                     ws.data_ptr(), nbytes, cv.stream())
        _lib.check(rc, "advect")
        if flux_face_i is None:
            return cv.out(out)
        return cv.out(out), cv.out(fx)
